// Counting kernels; see count.cuh.
//
// A piece is (row u, neighbours [s, min(s + 64, d+(u)))). A warp that takes a
// piece of u loads u's row into a per-warp shared-memory structure -- a
// bucketed hash of u's 32-column bit blocks (bitmap variant) or u's sorted
// neighbour list (merge variant) -- reusing it when its next piece is of the
// same row, then visits every item of every neighbour v of the piece: v's bit
// blocks (bitmap) or v's neighbours (merge), each looked up in u's structure.
// Neighbours with long lists are swept by all 32 lanes; short lists are
// flattened across lanes. Rows whose structure does not fit a warp's slice go
// whole to a CTA-wide pass, and rows too large for that to a global-memory
// pass, so every piece of every list is counted exactly once.
#include <cstddef>

#include "count.cuh"
#include "scan.cuh"

namespace tb {
namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kWarpsPerCta = 8;
constexpr int kWarpSlots = 512;                      // 8-byte words of shared memory per warp
constexpr uint32_t kWarpMaxBlocks = kWarpSlots / 2;  // bitmap rows up to this many bit blocks
constexpr int kCtaThreads = 512;
constexpr int kCtaLogSlots = 14;                     // 16384 slots = 128 KiB
constexpr uint32_t kCtaMaxBlocks = (1u << kCtaLogSlots) / 2;
constexpr uint32_t kLong = 24;                       // lists at least this long are swept by the whole warp
constexpr uint32_t kGrab = 4;                        // pieces taken per cursor update
constexpr uint64_t kEmptySlot = 0xFFFFFFFF00000000ull;

enum { kCurVariant0 = 0, kCurHubWarp = 3, kCurCta = 4, kCurGlobal = 5, kCurHeavy = 6, kCurHub = 7 };
// Heavy phase: CTA-shared table in the first 16 KiB of the kernel's shared
// memory, the row's per-neighbour item prefix in the second 16 KiB.
constexpr uint32_t kHeavyMaxBlocks = kWarpsPerCta * kWarpSlots / 4;
constexpr uint32_t kHeavyMaxDeg = kWarpsPerCta * kWarpSlots - 1;
constexpr uint32_t kHeavyMaxSpan = kWarpsPerCta * kWarpSlots;  // direct-mapped row: 16 KiB of masks
constexpr uint32_t kNoRow = 0xFFFFFFFFu;
enum { kOvfCta = 0, kOvfGlobal = 1 };

__device__ __forceinline__ int log2_ceil(uint32_t x) { return x <= 1 ? 0 : 32 - __clz(x - 1); }

__device__ __forceinline__ uint32_t hash_bucket(uint32_t blk, int logb) {
  return (blk * 0x9E3779B1u) >> (32 - logb);
}

// ---- bucketed hash of a row's bit blocks -----------------------------------
// 2^logb buckets of two 8-byte slots, (block << 32) | mask; a bucket's second
// slot fills only after its first, buckets probe linearly, and the table is at
// most half full, so every lookup ends at a bucket with an empty second slot.

__device__ __forceinline__ void table_clear(uint64_t* t, int logb, int tid, int nth) {
  for (int s = tid; s < (2 << logb); s += nth) t[s] = kEmptySlot;
}

__device__ __forceinline__ void table_insert(uint64_t* t, int logb, const uint64_t* __restrict__ bent, uint32_t bs,
                                             uint32_t be, int tid, int nth) {
  const uint32_t m = (1u << logb) - 1u;
  for (uint32_t k = bs + tid; k < be; k += nth) {
    const uint64_t e = bent[k];
    uint32_t b = hash_bucket((uint32_t)(e >> 32), logb);
    for (;;) {
      unsigned long long* slot = reinterpret_cast<unsigned long long*>(t + 2 * b);
      if (atomicCAS(slot, kEmptySlot, e) == kEmptySlot) break;
      if (atomicCAS(slot + 1, kEmptySlot, e) == kEmptySlot) break;
      b = (b + 1) & m;
    }
  }
}

__device__ __forceinline__ uint32_t table_find(const uint64_t* t, int logb, uint32_t blk) {
  const uint32_t m = (1u << logb) - 1u;
  uint32_t b = hash_bucket(blk, logb);
  for (;;) {
    const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(t + 2 * b);
    if ((uint32_t)(x.x >> 32) == blk) return (uint32_t)x.x;
    if ((uint32_t)(x.y >> 32) == blk) return (uint32_t)x.y;
    if ((uint32_t)(x.y >> 32) == 0xFFFFFFFFu) return 0u;
    b = (b + 1) & m;
  }
}

// Buckets for a row of nb bit blocks: at least nb (load <= 1/2), at least 16.
__device__ __forceinline__ int table_logb(uint32_t nb) { return max(4, log2_ceil(nb)); }

struct BitmapProbe {
  const uint64_t* t;
  int logb;
  uint32_t bmin, bmax;
  __device__ __forceinline__ uint32_t operator()(uint64_t e) const {
    const uint32_t blk = (uint32_t)(e >> 32);
    if (blk < bmin || blk > bmax) return 0u;
    return (uint32_t)__popc((uint32_t)e & table_find(t, logb, blk));
  }
  // Column id w (kept or not): 1 if w is in the staged row.
  __device__ __forceinline__ uint32_t col(uint32_t w, bool keep) const {
    const uint32_t blk = w >> 5;
    if (!keep || blk < bmin || blk > bmax) return 0u;
    return (table_find(t, logb, blk) >> (w & 31)) & 1u;
  }
  // e, or an entry that matches nothing.
  static __device__ __forceinline__ uint64_t drop(uint64_t e, bool keep) { return keep ? e : 0ull; }
};

// ---- the neighbour sweep ---------------------------------------------------
// Visits every item of the lists of slots [cs, ce), in chunks of 32 slots
// (chunk0, chunk0 + step, ...). desc(j, ib, il) gives slot j's first item and
// item count (il = 0 skips it); item(k, j) returns the matches of item k of
// slot j. Long lists are swept by all 32 lanes, two items per lane in flight;
// short lists are flattened across lanes. Must be called by all 32 lanes.

template <class Desc, class Item>
__device__ __forceinline__ uint64_t sweep_lists(uint32_t cs, uint32_t ce, uint32_t chunk0, uint32_t step,
                                                const Desc& desc, const Item& item) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t acc = 0;
  for (uint32_t c = cs + chunk0 * 32; c < ce; c += step * 32) {
    const uint32_t j = c + lane;
    uint32_t ib = 0, il = 0;
    if (j < ce) desc(j, ib, il);
    uint32_t longm = __ballot_sync(kFull, il >= kLong);
    while (longm) {
      const int s = __ffs(longm) - 1;
      longm &= longm - 1;
      const uint32_t sb = __shfl_sync(kFull, ib, s), sl = __shfl_sync(kFull, il, s);
      const uint32_t cj = c + s;
      uint32_t racc = 0;
      for (uint32_t k = lane; k < sl; k += 64) {
        const uint32_t k2 = k + 32;
        const uint32_t r0 = item(sb + k, cj);
        const uint32_t r1 = k2 < sl ? item(sb + k2, cj) : 0u;
        racc += r0 + r1;
      }
      acc += racc;
    }
    // Short lists: the owner of flattened item t is the lane whose inclusive
    // prefix first exceeds t.
    const uint32_t sl = il >= kLong ? 0u : il;
    const uint32_t incl = warp_inclusive_sum(sl);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - sl;
    uint32_t racc = 0;
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t t = base + lane;
      uint32_t s = 0;
#pragma unroll
      for (uint32_t st = 16; st >= 1; st >>= 1) {
        const uint32_t x = __shfl_sync(kFull, incl, s + st - 1);
        if (x <= t) s += st;
      }
      const uint32_t sb = __shfl_sync(kFull, ib, s);
      const uint32_t se = __shfl_sync(kFull, excl, s);
      if (t < total) racc += item(sb + (t - se), c + s);
    }
    acc += racc;
  }
  return acc;
}

// Flattened sweep for latency-bound lists: the lists of each chunk of 32
// slots are concatenated and lane l takes items t = base + l + 32 r, r <
// Depth, of the concatenation, issuing all Depth loads before it uses any, so
// a warp keeps 32 * Depth loads in flight however long or short the lists
// are. load(k) reads item k (index into the item array), probe(x) scores it;
// a loaded 0 must score 0. The owner slot of an item: the chunk's inclusive
// prefix and item offsets go to the warp's 64 words of shared memory (wsm);
// each lane finds the owner of its first item once by binary search and then
// only advances it (items of a lane only grow), so a long list costs one
// shared-memory compare per item. Chunks whose lists average under MinAvg
// items (measured: 8 for hub tails, 32 for bit rows) find each item's owner by
// a 5-step shuffle search over the prefix instead.
template <int Depth, uint32_t MinAvg, class Desc, class Load, class Probe>
__device__ __forceinline__ uint64_t sweep_runs(uint32_t cs, uint32_t ce, uint32_t chunk0, uint32_t step,
                                               const Desc& desc, const Load& load, const Probe& probe,
                                               uint32_t* wsm) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t acc = 0;
  for (uint32_t c = cs + chunk0 * 32; c < ce; c += step * 32) {
    const uint32_t j = c + lane;
    uint32_t ib = 0, il = 0;
    if (j < ce) desc(j, ib, il);
    const uint32_t incl = warp_inclusive_sum(il);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    if (total < 32 * MinAvg) {
      // Short lists: a lane would cross several lists per step; a shuffle
      // search per item is cheaper here.
      const uint32_t offs = ib - (incl - il);
      uint32_t racc = 0;
      for (uint32_t base = 0; base < total; base += 32 * Depth) {
        uint64_t x[Depth];
#pragma unroll
        for (int r = 0; r < Depth; ++r) {
          const uint32_t t = base + 32 * r + lane;
          uint32_t so = 0;
#pragma unroll
          for (uint32_t st = 16; st >= 1; st >>= 1) {
            const uint32_t y = __shfl_sync(kFull, incl, so + st - 1);
            if (y <= t) so += st;
          }
          const uint32_t o = __shfl_sync(kFull, offs, so);
          x[r] = t < total ? load(o + t) : 0ull;
        }
#pragma unroll
        for (int r = 0; r < Depth; ++r) racc += probe(x[r]);
      }
      acc += racc;
      continue;
    }
    __syncwarp();
    wsm[lane] = incl;
    wsm[32 + lane] = ib - (incl - il);  // item t of the chunk, owned by slot s, is item off_s + t
    __syncwarp();
    uint32_t s = 0;
#pragma unroll
    for (uint32_t st = 16; st >= 1; st >>= 1)
      if (wsm[s + st - 1] <= lane) s += st;
    uint32_t lim = wsm[s], off = wsm[32 + s];
    uint32_t racc = 0;
    for (uint32_t base = 0; base < total; base += 32 * Depth) {
      uint64_t x[Depth];
#pragma unroll
      for (int r = 0; r < Depth; ++r) {
        const uint32_t t = base + 32 * r + lane;
        while (t >= lim && s < 31) {
          ++s;
          lim = wsm[s];
          off = wsm[32 + s];
        }
        x[r] = t < total ? load(off + t) : 0ull;
      }
#pragma unroll
      for (int r = 0; r < Depth; ++r) racc += probe(x[r]);
    }
    acc += racc;
  }
  __syncwarp();
  return acc;
}

// Edge j of the CSR is counted by the hub pass (see k_hub) instead of by its
// row's sweep.
__device__ __forceinline__ bool edge_to_hub(const GraphView& g, uint32_t j) {
  return g.eflag && ((g.eflag[j >> 5] >> (j & 31)) & 1u);
}

// The neighbour sweep: slots are CSR positions j, each the list of v = col[j]:
// its bit blocks (Blocks) or its neighbour ids.
template <bool Blocks, class Item>
__device__ __forceinline__ uint64_t sweep(const GraphView& g, uint32_t cs, uint32_t ce, uint32_t chunk0,
                                          uint32_t step, const Item& item) {
  return sweep_lists(
      cs, ce, chunk0, step,
      [&](uint32_t j, uint32_t& ib, uint32_t& il) {
        if (edge_to_hub(g, j)) return;
        const uint32_t v = g.col[j];
        const uint64_t a = g.rp[v], b = g.rp[v + 1];
        ib = Blocks ? rp_blk(a) : rp_row(a);
        il = (Blocks ? rp_blk(b) : rp_row(b)) - ib;
      },
      item);
}

// Bit-row sweep: every bit block of v = col[j], j in the slots, scored by
// probe (a hash or direct-map lookup in u's staged row), flattened with
// kBitsDepth blocks in flight per lane (sweep_runs; wsm: the warp's 64 words).
#ifndef TB_BITS_DEPTH
#define TB_BITS_DEPTH 4
#endif
constexpr int kBitsDepth = TB_BITS_DEPTH;
// Column id w as a one-bit entry of its block; `keep` false: the block alone
// (matches nothing).
__device__ __forceinline__ uint64_t col_entry(uint32_t w, bool keep) {
  return ((uint64_t)(w >> 5) << 32) | (keep ? 1u << (w & 31) : 0u);
}

template <class Probe>
__device__ __forceinline__ uint64_t sweep_bits(const GraphView& g, uint32_t cs, uint32_t ce, uint32_t chunk0,
                                               uint32_t step, const Probe& probe, uint32_t* wsm) {
  return sweep_runs<kBitsDepth, 32>(
      cs, ce, chunk0, step,
      [&](uint32_t j, uint32_t& ib, uint32_t& il) {
        if (edge_to_hub(g, j)) return;
        const uint32_t v = g.col[j];
        const uint64_t a = g.rp[v], b = g.rp[v + 1];
        ib = rp_blk(a);
        il = rp_blk(b) - ib;
      },
      [&](uint32_t k) -> uint64_t { return g.bent[k]; }, probe, wsm);
}

// Mask of block x in the sorted bit row r[lo, end), or 0.
__device__ __forceinline__ uint32_t search_mask(const uint64_t* r, uint32_t lo, uint32_t end, uint32_t x) {
  uint32_t hi = end;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((uint32_t)(r[mid] >> 32) < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < end) {
    const uint64_t e = r[lo];
    if ((uint32_t)(e >> 32) == x) return (uint32_t)e;
  }
  return 0u;
}

// Sorted-list intersection of bit rows (the merge variant). u's bit row is in
// shared memory (urow, nbu entries, ascending block). For each neighbour v of
// the chunk, the shorter of u's tail -- u's entries from v's block on, the
// only ones that can meet N+(v) -- and v's bit row is walked, and every block
// of it is binary-searched in the other list. Edges given to the hub pass,
// where u's tail was the shorter list, are skipped. Must be called by all 32
// lanes.
__device__ __forceinline__ uint64_t sweep_merge(const GraphView& g, const uint64_t* urow, uint32_t nbu, uint32_t cs,
                                                uint32_t ce) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t acc = 0;
  auto item = [&](uint32_t k, bool walk_u, uint32_t ob, uint32_t oe) -> uint32_t {
    const uint64_t e = walk_u ? urow[k] : g.bent[k];
    const uint32_t m = walk_u ? search_mask(g.bent, ob, oe, (uint32_t)(e >> 32))
                              : search_mask(urow, ob, oe, (uint32_t)(e >> 32));
    return (uint32_t)__popc((uint32_t)e & m);
  };
  for (uint32_t c = cs; c < ce; c += 32) {
    const uint32_t j = c + lane;
    uint32_t ab = 0, len = 0, ob = 0, oe = 0, walk_u = 0;
    if (j < ce && !edge_to_hub(g, j)) {
      const uint32_t v = g.col[j];
      const uint64_t va = g.rp[v], vb = g.rp[v + 1];
      const uint32_t vbs = rp_blk(va), vbe = rp_blk(vb);
      uint32_t lo = 0, hi = nbu;  // position of v's block in u's row
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((uint32_t)(urow[mid] >> 32) < (v >> 5))
          lo = mid + 1;
        else
          hi = mid;
      }
      const uint32_t ta = nbu - lo, tb = vbe - vbs;
      walk_u = ta <= tb ? 1u : 0u;
      if (walk_u) {
        ab = lo, len = ta, ob = vbs, oe = vbe;
      } else {
        ab = vbs, len = tb, ob = lo, oe = nbu;
      }
    }
    uint32_t longm = __ballot_sync(kFull, len >= kLong);
    while (longm) {
      const int s = __ffs(longm) - 1;
      longm &= longm - 1;
      const uint32_t sab = __shfl_sync(kFull, ab, s), slen = __shfl_sync(kFull, len, s);
      const uint32_t sob = __shfl_sync(kFull, ob, s), soe = __shfl_sync(kFull, oe, s);
      const bool sw = __shfl_sync(kFull, walk_u, s) != 0;
      for (uint32_t k = lane; k < slen; k += 32) acc += item(sab + k, sw, sob, soe);
    }
    const uint32_t sl = len >= kLong ? 0u : len;
    const uint32_t incl = warp_inclusive_sum(sl);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - sl;
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t t = base + lane;
      uint32_t s = 0;
#pragma unroll
      for (uint32_t st = 16; st >= 1; st >>= 1) {
        const uint32_t x = __shfl_sync(kFull, incl, s + st - 1);
        if (x <= t) s += st;
      }
      const uint32_t sab = __shfl_sync(kFull, ab, s), sex = __shfl_sync(kFull, excl, s);
      const uint32_t sob = __shfl_sync(kFull, ob, s), soe = __shfl_sync(kFull, oe, s);
      const bool sw = __shfl_sync(kFull, walk_u, s) != 0;
      if (t < total) acc += item(sab + (t - sex), sw, sob, soe);
    }
  }
  return acc;
}

__device__ __forceinline__ void push_row(DeviceStats* stats, int which, uint32_t* list, uint32_t u) {
  const uint32_t i = atomicAdd(&stats->overflow[which], 1u);
  list[i] = u;
}

// SM cycle counter; a piece runs on one SM, so differences are meaningful.
__device__ __forceinline__ unsigned long long cycles() { return (unsigned long long)clock64(); }

// ---- warp-per-piece kernels (bitmap and merge variants) --------------------

// Merge row blocks' edges left to the row sweep (not taken by the hub pass)
// are walked by sorted-list merge with binary searches (0), or, like the
// bitmap variant's, as v's bit blocks probed in u's direct-mapped or hashed
// row (1). Build-time switch for measurement.
#ifndef TB_MERGE_BITS
#define TB_MERGE_BITS 0
#endif

// Shared memory of the row-piece bodies: the CTA's flat table (at least
// kWarpsPerCta * kWarpSlots words of 8 bytes, the warps' slices at `stride`
// words apart), the warps' run buffers (`run_stride` words apart, >= 64) and
// a CTA word.
struct PiecesShared {
  uint64_t* smem;
  uint32_t stride;
  uint32_t* runs;
  uint32_t run_stride;
  uint32_t* s_row;
};

// The row-piece variant V over its pieces (and, with `heavy`, first the heavy
// rows, one CTA per row); returns this thread's partial count.
template <int V>
__device__ __forceinline__ uint64_t pieces_body(const GraphView& g, const uint64_t* __restrict__ pieces,
                                                const uint32_t* __restrict__ piece_off, DeviceStats* stats,
                                                uint32_t* __restrict__ ovf_cta, unsigned long long* per_graph,
                                                unsigned long long* block_ns, const uint32_t* __restrict__ heavy,
                                                uint32_t width, const PiecesShared& sh) {
  constexpr bool kSorted = V == TRIBIT_VARIANT_MERGE && !TB_MERGE_BITS;  // u staged as a sorted row
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t* tbl = sh.smem + w * sh.stride;
  uint32_t* wruns = sh.runs + w * sh.run_stride;
  uint32_t& s_row = *sh.s_row;

  const uint32_t p0 = piece_off[V], len = piece_off[V + 1] - p0;
  uint64_t acc = 0;
  // Phase 1 (first kernel only): rows too wide for a warp's slice, one at a
  // time per CTA, with a CTA-shared table in the same shared memory and all
  // warps sweeping the row's neighbour chunks.
  if (heavy) {
    uint64_t* ctbl = sh.smem;
    uint32_t* pre = reinterpret_cast<uint32_t*>(sh.smem + (kWarpsPerCta / 2) * kWarpSlots);
    const uint32_t hlen = piece_off[TRIBIT_NUM_VARIANTS + 1];
    for (;;) {
      if (threadIdx.x == 0) {
        const uint32_t t = atomicAdd(&stats->cursor[kCurHeavy], 1u);
        s_row = t < hlen ? heavy[hlen - 1 - t] : kNoRow;
      }
      __syncthreads();
      const uint32_t u = s_row;
      if (u == kNoRow) break;
      const unsigned long long h_start = (block_ns && threadIdx.x == 0) ? cycles() : 0ull;
      const uint64_t a = g.rp[u], b = g.rp[u + 1];
      const uint32_t rs = rp_row(a), re = rp_row(b), bs = rp_blk(a), be = rp_blk(b), nb = be - bs;
      const uint32_t d = re - rs;
      if (nb > kHeavyMaxBlocks || d > kHeavyMaxDeg) {
        if (threadIdx.x == 0) push_row(stats, kOvfCta, ovf_cta, u);
        __syncthreads();
        continue;
      }
      // u's row: a direct-mapped mask array over its block span when that
      // fits the table's 16 KiB (the top-ranked rows), else the bucketed hash.
      const uint32_t bmin = (uint32_t)(g.bent[bs] >> 32), bmax = (uint32_t)(g.bent[be - 1] >> 32);
      const uint32_t span = bmax - bmin + 1;
      const bool direct = span <= kHeavyMaxSpan;
      uint32_t* cmap = reinterpret_cast<uint32_t*>(ctbl);
      const int logb = table_logb(nb);
      if (direct) {
        for (uint32_t i = threadIdx.x; i < span; i += blockDim.x) cmap[i] = 0u;
      } else {
        table_clear(ctbl, logb, threadIdx.x, blockDim.x);
      }
      // Item prefix: pre[j] = bit blocks of the neighbours before j, pre[d] = all.
      for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
        const uint32_t v = g.col[rs + j];
        pre[j] = edge_to_hub(g, rs + j) ? 0u : rp_blk(g.rp[v + 1]) - rp_blk(g.rp[v]);
      }
      __syncthreads();
      if (direct) {
        for (uint32_t k = bs + threadIdx.x; k < be; k += blockDim.x) {
          const uint64_t e = g.bent[k];
          cmap[(uint32_t)(e >> 32) - bmin] = (uint32_t)e;
        }
      } else {
        table_insert(ctbl, logb, g.bent, bs, be, threadIdx.x, blockDim.x);
      }
      {
        const uint32_t per = (d + blockDim.x - 1) / blockDim.x, j0 = threadIdx.x * per;
        uint32_t lsum = 0;
        for (uint32_t k = 0; k < per && j0 + k < d; ++k) lsum += pre[j0 + k];
        uint32_t tot;
        uint32_t ex = block_exclusive_scan<uint32_t>(lsum, OpSum{}, 0u, &tot);
        for (uint32_t k = 0; k < per && j0 + k < d; ++k) {
          const uint32_t x = pre[j0 + k];
          pre[j0 + k] = ex;
          ex += x;
        }
        if (threadIdx.x == 0) pre[d] = tot;
      }
      __syncthreads();
      // Warp w takes the neighbours whose first item falls in the w-th equal
      // share of the row's items, so the warps finish together.
      const uint32_t tot = pre[d];
      auto first_at = [&](uint32_t x) -> uint32_t {  // first j with pre[j] >= x
        uint32_t lo = 0, hi = d;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (pre[mid] < x)
            lo = mid + 1;
          else
            hi = mid;
        }
        return lo;
      };
      const uint32_t cs = first_at((uint32_t)((uint64_t)tot * w / kWarpsPerCta));
      const uint32_t ce = w + 1 == kWarpsPerCta ? d : first_at((uint32_t)((uint64_t)tot * (w + 1) / kWarpsPerCta));
      uint64_t racc;
      if (direct) {
        racc = sweep_bits(g, rs + cs, rs + ce, 0, 1, [&](uint64_t e) -> uint32_t {
          const uint32_t o = (uint32_t)(e >> 32) - bmin;
          return o < span ? (uint32_t)__popc((uint32_t)e & cmap[o]) : 0u;
        }, wruns);
      } else {
        const BitmapProbe probe{ctbl, logb, bmin, bmax};
        racc = sweep_bits(g, rs + cs, rs + ce, 0, 1, probe, wruns);
      }
      if (per_graph) {
        const uint64_t s = warp_sum(racc);
        if (lane == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
      }
      acc += racc;
      __syncthreads();  // the table and s_row are rewritten for the next row
      // Timing: the row's CTA cycles in warp-cycles, like the warp pieces'.
      if (block_ns && threadIdx.x == 0) atomicAdd(&block_ns[u >> 5], (cycles() - h_start) * kWarpsPerCta);
    }
    __syncthreads();
  }
  uint32_t cur = 0xFFFFFFFFu;  // row whose structure is loaded
  bool cur_ok = false, cur_direct = false;
  int logb = 0;
  uint32_t bmin = 0, bmax = 0, d = 0;
  uint32_t* wmap = reinterpret_cast<uint32_t*>(tbl);  // the slice as a direct-mapped row
  for (;;) {
    uint32_t t0 = 0;
    if (lane == 0) t0 = atomicAdd(&stats->cursor[kCurVariant0 + V], kGrab);
    t0 = __shfl_sync(kFull, t0, 0);
    if (t0 >= len) break;
    const uint32_t t1 = min(t0 + kGrab, len);
    for (uint32_t t = t0; t < t1; ++t) {
      const uint64_t pc = pieces[p0 + (len - 1 - t)];
      const uint32_t u = (uint32_t)(pc >> 32), first = (uint32_t)pc;
      const uint64_t a = g.rp[u], b = g.rp[u + 1];
      const uint32_t rs = rp_row(a), re = rp_row(b);
      unsigned long long t_start = 0;
      if (block_ns && lane == 0) t_start = cycles();
      if (u != cur) {
        __syncwarp();
        cur = u;
        if (kSorted) {
          const uint32_t bs = rp_blk(a), be = rp_blk(b);
          d = be - bs;  // u's bit-row length
          cur_ok = d <= kWarpMaxBlocks;
          if (cur_ok)
            for (uint32_t k = lane; k < d; k += 32) tbl[k] = g.bent[bs + k];
        } else {
          const uint32_t bs = rp_blk(a), be = rp_blk(b), nb = be - bs;
          cur_ok = nb <= kWarpMaxBlocks;
          if (cur_ok) {
            bmin = (uint32_t)(g.bent[bs] >> 32);
            bmax = (uint32_t)(g.bent[be - 1] >> 32);
            // A row whose blocks span at most the slice's 1,024 words is
            // direct-mapped (one load per probe); others are hashed.
            cur_direct = bmax - bmin < kWarpSlots * 2;
            if (cur_direct) {
              for (uint32_t i = lane; i <= bmax - bmin; i += 32) wmap[i] = 0u;
              __syncwarp();
              for (uint32_t k = bs + lane; k < be; k += 32) {
                const uint64_t e = g.bent[k];
                wmap[(uint32_t)(e >> 32) - bmin] = (uint32_t)e;
              }
            } else {
              logb = table_logb(nb);
              table_clear(tbl, logb, lane, 32);
              __syncwarp();
              table_insert(tbl, logb, g.bent, bs, be, lane, 32);
            }
          }
        }
        __syncwarp();
      }
      if (!cur_ok) {
        // The whole row goes to the CTA pass once, from its first piece.
        if (first == 0 && lane == 0) push_row(stats, kOvfCta, ovf_cta, u);
        continue;
      }
      const uint32_t cs = rs + first, ce = min(cs + width, re);
      uint64_t racc;
      if (kSorted) {
        racc = sweep_merge(g, tbl, d, cs, ce);
      } else if (cur_direct) {
        const uint32_t span = bmax - bmin + 1;
        racc = sweep_bits(g, cs, ce, 0, 1, [&](uint64_t e) -> uint32_t {
          const uint32_t o = (uint32_t)(e >> 32) - bmin;
          return o < span ? (uint32_t)__popc((uint32_t)e & wmap[o]) : 0u;
        }, wruns);
      } else {
        const BitmapProbe probe{tbl, logb, bmin, bmax};
        racc = sweep_bits(g, cs, ce, 0, 1, probe, wruns);
      }
      if (per_graph) {
        const uint64_t s = warp_sum(racc);
        if (lane == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
      }
      if (block_ns) {
        __syncwarp();
        if (lane == 0) atomicAdd(&block_ns[u >> 5], cycles() - t_start);
      }
      acc += racc;
    }
  }
  return acc;
}

template <int V>
__global__ void __launch_bounds__(kWarpsPerCta * 32) k_pieces_warp(GraphView g, const uint64_t* __restrict__ pieces,
                                                                    const uint32_t* __restrict__ piece_off,
                                                                    DeviceStats* stats, uint32_t* __restrict__ ovf_cta,
                                                                    unsigned long long* per_graph,
                                                                    unsigned long long* block_ns,
                                                                    const uint32_t* __restrict__ heavy,
                                                                    uint32_t width) {
  __shared__ __align__(16) uint64_t smem[kWarpsPerCta][kWarpSlots];
  __shared__ uint32_t runs[kWarpsPerCta][64];
  __shared__ uint32_t s_row;
  const PiecesShared sh{&smem[0][0], kWarpSlots, &runs[0][0], 64, &s_row};
  uint64_t acc = pieces_body<V>(g, pieces, piece_off, stats, ovf_cta, per_graph, block_ns, heavy, width, sh);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- bit-tile MMA variant -----------------------------------------------------
// One warp per 32-row block R. When every active row's bit blocks fall in one
// range [c0, c0 + K) of at most kTileMaxK blocks, the rows form the A tile
// (32 rows x K words, each word one 32-column mask); A is also the adjacency
// of R, so the neighbours V of R are the set bits of the OR of A's rows. For
// each group of 8 neighbours the warp gathers their masks on the same range
// (the B tile) and one m16n8k256 b1 AND+POPC MMA per 16 rows per 8 words
// gives D[r][j] = |N+(u_r) & N+(v_j)|; the count adds D[r][j] where A[r] has
// v_j. Each neighbour's row is read once per row block instead of once per
// edge. Row blocks that do not fit fall back to the bitmap sweep in place.

constexpr float kTileMinDensityInv = 8.f;      // plain rule: tiles need 1/8 of their cells set
constexpr int kTileStride = kTileMaxK + 4;      // padded: fragment loads hit 32 distinct banks
constexpr int kTileWarps = 4;
constexpr uint32_t kTileNbrPiece = 128;         // neighbours of V per tile piece (16 groups of 8)
struct TileSmem {
  uint32_t a[32 * kTileStride];                 // also the fallback hash table (4 KiB used)
  uint32_t b[8 * kTileStride];
  uint32_t vmask[kTileMaxK];                    // OR of the A rows: the neighbour set of R
};

__device__ __forceinline__ void mma_b1(int (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                       uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Per-row bitmap sweep of the active rows of a row block (the fallback).
__device__ uint64_t tile_fallback(const GraphView& g, uint32_t rb, uint64_t* tbl, uint32_t* wsm,
                                  unsigned long long* per_graph) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t acc = 0;
  for (uint32_t r = 0; r < 32; ++r) {
    const uint32_t u = rb * 32 + r;
    if (u >= g.n) break;
    const uint64_t a = g.rp[u], b = g.rp[u + 1];
    const uint32_t rs = rp_row(a), re = rp_row(b), bs = rp_blk(a), be = rp_blk(b), nb = be - bs;
    if (re - rs < 2 || nb > kWarpMaxBlocks) continue;
    const int logb = table_logb(nb);
    __syncwarp();
    table_clear(tbl, logb, lane, 32);
    __syncwarp();
    table_insert(tbl, logb, g.bent, bs, be, lane, 32);
    __syncwarp();
    const BitmapProbe probe{tbl, logb, (uint32_t)(g.bent[bs] >> 32), (uint32_t)(g.bent[be - 1] >> 32)};
    const uint64_t racc =
        sweep_bits(g, rs, re, 0, 1, probe, wsm);
    if (per_graph) {
      const uint64_t s = warp_sum(racc);
      if (lane == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
    }
    acc += racc;
  }
  return acc;
}

__global__ void __launch_bounds__(kTileWarps * 32) k_tiles_mma(GraphView g, const uint64_t* __restrict__ pieces,
                                                               const uint32_t* __restrict__ piece_off,
                                                               DeviceStats* stats, unsigned long long* per_graph,
                                                               unsigned long long* block_ns) {
  extern __shared__ __align__(16) unsigned char tile_raw[];
  TileSmem& sm = reinterpret_cast<TileSmem*>(tile_raw)[threadIdx.x >> 5];
  const uint32_t lane = threadIdx.x & 31, grp = lane >> 2, tig = lane & 3;
  const uint32_t p0 = piece_off[TRIBIT_VARIANT_MMA], len = piece_off[TRIBIT_VARIANT_MMA + 1] - p0;
  uint64_t acc = 0;
  for (;;) {
    uint32_t t0 = 0;
    if (lane == 0) t0 = atomicAdd(&stats->cursor[kCurVariant0 + TRIBIT_VARIANT_MMA], kGrab);
    t0 = __shfl_sync(kFull, t0, 0);
    if (t0 >= len) break;
    const uint32_t t1 = min(t0 + kGrab, len);
    for (uint32_t t = t0; t < t1; ++t) {
      // A piece is (first row of the block << 32) | index of its first neighbour in V.
      const uint64_t pc = pieces[p0 + (len - 1 - t)];
      const uint32_t rb = (uint32_t)(pc >> 32) >> 5, first = (uint32_t)pc;
      const unsigned long long t_start = (block_ns && lane == 0) ? cycles() : 0ull;
      // Row of this lane: activity and block range.
      const uint32_t u = rb * 32 + lane;
      uint32_t bs = 0, be = 0, lo = 0xFFFFFFFFu, hi = 0;
      bool active = false;
      if (u < g.n) {
        const uint64_t a = g.rp[u], b = g.rp[u + 1];
        bs = rp_blk(a);
        be = rp_blk(b);
        active = rp_row(b) - rp_row(a) >= 2 && be - bs <= kWarpMaxBlocks;
        if (active) {
          lo = (uint32_t)(g.bent[bs] >> 32);
          hi = (uint32_t)(g.bent[be - 1] >> 32);
        }
      }
      const uint32_t amask = __ballot_sync(kFull, active);
      if (!amask) continue;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
      }
      const uint32_t K = hi - lo + 1;
      uint64_t racc = 0;
      if (K > (uint32_t)kTileMaxK) {
        // Forced onto a block that fits no tile: its one piece sweeps the rows.
        if (first == 0) racc = tile_fallback(g, rb, reinterpret_cast<uint64_t*>(sm.a), sm.b, per_graph);
      } else {
        const uint32_t KP = (K + 7) & ~7u;  // words, whole 256-bit k-steps
        for (uint32_t i = lane; i < 32 * kTileStride; i += 32) sm.a[i] = 0u;
        __syncwarp();
        // A rows: each active row writes its own masks (distinct words).
        for (uint32_t r = 0; r < 32; ++r) {
          if (!((amask >> r) & 1u)) continue;
          const uint32_t rbs = __shfl_sync(kFull, bs, r), rbe = __shfl_sync(kFull, be, r);
          for (uint32_t k = rbs + lane; k < rbe; k += 32) {
            const uint64_t e = g.bent[k];
            sm.a[r * kTileStride + ((uint32_t)(e >> 32) - lo)] = (uint32_t)e;
          }
        }
        __syncwarp();
        // Neighbour set V: OR of the A rows.
        for (uint32_t w = lane; w < KP; w += 32) {
          uint32_t m = 0;
          if (w < K)
            for (uint32_t r = 0; r < 32; ++r) m |= sm.a[r * kTileStride + w];
          sm.vmask[w] = m;
        }
        __syncwarp();
        int rowsum[4] = {0, 0, 0, 0};  // rows grp, grp + 8, 16 + grp, 24 + grp
        uint32_t cw = 0, cbits = sm.vmask[0];  // warp-uniform cursor over V's set bits
        // This piece's neighbours: V[first, first + kTileNbrPiece).
        for (uint32_t skip = first; skip > 0;) {
          const uint32_t c = __popc(cbits);
          if (c > skip) {
            for (uint32_t q = 0; q < skip; ++q) cbits &= cbits - 1;
            break;
          }
          skip -= c;
          cbits = cw + 1 < K ? sm.vmask[++cw] : 0u;
          if (cbits == 0 && cw + 1 >= K) break;
        }
        for (uint32_t done = 0; done < kTileNbrPiece; done += 8) {
          // Next 8 neighbours, as column offsets from lo * 32 (0xFFFF = none).
          uint32_t vc[8];
          uint32_t nv = 0;
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            while (cbits == 0 && cw + 1 < K) cbits = sm.vmask[++cw];
            vc[jj] = 0xFFFFu;
            if (cbits) {
              vc[jj] = cw * 32 + __ffs(cbits) - 1;
              cbits &= cbits - 1;
              ++nv;
            }
          }
          if (nv == 0) break;
          for (uint32_t i = lane; i < 8 * kTileStride; i += 32) sm.b[i] = 0u;
          __syncwarp();
          // B tile: the neighbours' masks on [lo, lo + K).
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            if (vc[jj] == 0xFFFFu) continue;
            const uint32_t v = lo * 32 + vc[jj];
            const uint64_t va = g.rp[v], vb = g.rp[v + 1];
            const uint32_t vbs = rp_blk(va), vn = min(rp_blk(vb) - vbs, K);
            for (uint32_t k = lane; k < vn; k += 32) {
              const uint64_t e = g.bent[vbs + k];
              const uint32_t blk = (uint32_t)(e >> 32);
              if (blk <= hi) sm.b[jj * kTileStride + (blk - lo)] = (uint32_t)e;
            }
          }
          __syncwarp();
          int c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
          for (uint32_t ks = 0; ks < KP; ks += 8) {
            const uint32_t* a0p = sm.a + grp * kTileStride + ks + tig;
            const uint32_t* bp = sm.b + grp * kTileStride + ks + tig;
            const uint32_t b0 = bp[0], b1 = bp[4];
            mma_b1(c0, a0p[0], a0p[8 * kTileStride], a0p[4], a0p[8 * kTileStride + 4], b0, b1);
            mma_b1(c1, a0p[16 * kTileStride], a0p[24 * kTileStride], a0p[16 * kTileStride + 4],
                   a0p[24 * kTileStride + 4], b0, b1);
          }
          // D[row][col]: c[0] (grp, 2t), c[1] (grp, 2t+1), c[2] (grp+8, 2t), c[3] (grp+8, 2t+1).
          uint32_t vcol[2] = {vc[0], vc[1]};
#pragma unroll
          for (int q = 1; q < 4; ++q)
            if (tig == (uint32_t)q) vcol[0] = vc[2 * q], vcol[1] = vc[2 * q + 1];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t vo = vcol[q & 1];
            if (vo == 0xFFFFu) continue;
            const uint32_t ra = grp + ((q >> 1) ? 8 : 0), rbb = ra + 16;
            if ((sm.a[ra * kTileStride + (vo >> 5)] >> (vo & 31)) & 1u) rowsum[q >> 1] += c0[q];
            if ((sm.a[rbb * kTileStride + (vo >> 5)] >> (vo & 31)) & 1u) rowsum[2 + (q >> 1)] += c1[q];
          }
          __syncwarp();
        }
        // Reduce the four lanes of each row group; lane tig == 0 owns the rows.
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          rowsum[q] += __shfl_xor_sync(kFull, rowsum[q], 1);
          rowsum[q] += __shfl_xor_sync(kFull, rowsum[q], 2);
        }
        if (tig == 0) {
          const uint32_t rows[4] = {grp, grp + 8, 16 + grp, 24 + grp};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            racc += (uint64_t)rowsum[q];
            if (per_graph && rowsum[q]) atomicAdd(&per_graph[g.graph_of_rank[rb * 32 + rows[q]]],
                                                  (unsigned long long)rowsum[q]);
          }
        }
        __syncwarp();
      }
      if (block_ns) {
        __syncwarp();
        if (lane == 0) atomicAdd(&block_ns[rb], cycles() - t_start);
      }
      acc += racc;
    }
  }
  acc = warp_sum(acc);
  if (lane == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- bit-tile variant on the 5th-generation tensor cores (tcgen05) ----------
// Same pieces as k_tiles_mma (a row block R whose rows fit one column range of
// K <= kTileMaxK blocks, and 128 neighbours V[first, first + 128) of it), but
// the product runs as one tcgen05.mma kind::i8 per 32 columns: the 128
// neighbours' bits over the range, unpacked to 0/1 bytes, are the A operand
// (M = 128), the block's 32 rows the B operand (N = 32), both K-major in
// shared memory without swizzle; D[v][u] = |N+(v) & N+(u)| accumulates in
// TMEM as s32 (exact: at most K * 32 = 2048 per element). One elected thread
// issues the MMAs and commits them to an mbarrier that every thread waits on
// with a bounded wait; each warp then reads its 32 TMEM lanes (rows v) and
// adds D[v][u] where u has v. The CTA allocates its 32 TMEM columns once and
// frees them before it exits, also after a failed wait.

constexpr int kTcThreads = 128;
// 128-column rounds (7 CTAs an SM) measured faster than 256 (4 CTAs): dense
// cliques 0.276 vs 0.364 ms.
#ifndef TB_TC_CHUNK
#define TB_TC_CHUNK 128
#endif
constexpr uint32_t kTcChunk = TB_TC_CHUNK;         // K bytes (columns) unpacked per round
constexpr uint32_t kTcWords = kTcChunk / 32;       // bit words of a row per round
static_assert(kTcChunk == 128 || kTcChunk == 256, "a round is 4 or 8 MMAs of K = 32");
constexpr uint32_t kTcDrainPolls = 1u << 22;       // bounded wait for committed MMAs after a failed wait


// 29 KiB with 128-column rounds (49 KiB with 256): seven CTAs an SM (four),
// so one CTA's operand gathering runs while another's MMAs do.
struct TcSmem {
  uint8_t a[kTileNbrPiece * kTcChunk];             // A: 128 rows x kTcChunk K-bytes, core-matrix layout
  uint8_t b[32 * kTcChunk];                        // B: 32 rows x kTcChunk K-bytes
  uint32_t ubits[32][kTileMaxK];                   // the block's rows
  uint32_t vmask[kTileMaxK];                       // OR of the rows: V
  uint32_t vpre[kTileMaxK + 1];                    // popcount prefix of vmask
  uint32_t row_bs[32], row_be[32];
  unsigned long long mbar;
  uint32_t tmem;
  uint32_t lo, K, amask, cnt_v, fail;
};
constexpr int kTcCtasPerSm = kTcChunk == 256 ? 4 : 7;
static_assert(kTileMaxK == 64, "the vmask prefix is one warp scan of two words a lane");

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices, lbo bytes between core matrices along K, sbo along M/N.
__device__ __forceinline__ uint64_t umma_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((smem_addr(p) >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::i8: D s32, A and B unsigned 8-bit, both
// K-major, N = 32, M = 128.
constexpr uint32_t kTcIdesc = (2u << 4) | (0u << 7) | (0u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

// Unpacks 32 bits (LSB = first column) to 32 bytes of 0/1 as two uint4.
__device__ __forceinline__ void unpack32(uint32_t x, uint4& lo16, uint4& hi16) {
  auto nib = [](uint32_t v) -> uint32_t { return (v & 0xFu) * 0x00204081u & 0x01010101u; };
  lo16 = make_uint4(nib(x), nib(x >> 4), nib(x >> 8), nib(x >> 12));
  hi16 = make_uint4(nib(x >> 16), nib(x >> 20), nib(x >> 24), nib(x >> 28));
}

// Byte offset of (row, 16-byte K group) in a K-major no-swizzle operand of
// kTcChunk K-bytes: core matrices of 8 rows x 16 bytes, 128 bytes apart along
// K (LBO) and 16 * 128 bytes apart along the rows (SBO).
__device__ __forceinline__ uint32_t tc_off(uint32_t row, uint32_t kgroup) {
  return (row >> 3) * (kTcChunk / 16) * 128 + kgroup * 128 + (row & 7) * 16;
}

__device__ __forceinline__ bool tc_wait(unsigned long long* mbar, uint32_t parity, uint32_t max_polls) {
  uint32_t done = 0;
  for (uint32_t i = 0; i < max_polls && !done; ++i)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(mbar)), "r"(parity)
        : "memory");
  return done != 0;
}

// test_no_commit (failure-detection test only): the MMAs are neither issued
// nor committed, so the first wait runs out after max_polls and the kernel
// takes its error path.
__global__ void __launch_bounds__(kTcThreads) k_tiles_tc(GraphView g, const uint64_t* __restrict__ pieces,
                                                         const uint32_t* __restrict__ piece_off, DeviceStats* stats,
                                                         unsigned long long* per_graph,
                                                         unsigned long long* block_ns, uint32_t max_polls,
                                                         int test_no_commit) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t p0 = piece_off[TRIBIT_VARIANT_MMA], len = piece_off[TRIBIT_VARIANT_MMA + 1] - p0;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&sm.mbar)), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    sm.fail = 0;
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_addr(&sm.tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sm.tmem;
  uint32_t phase = 0;
  uint64_t acc = 0;
  __shared__ uint32_t s_t;
  for (;;) {
    if (tid == 0) s_t = atomicAdd(&stats->cursor[kCurVariant0 + TRIBIT_VARIANT_MMA], 1u);
    __syncthreads();
    const uint32_t t = s_t;
    if (t >= len || sm.fail) break;
    const unsigned long long t_start = (block_ns && tid == 0) ? cycles() : 0ull;
    const uint64_t pc = pieces[p0 + (len - 1 - t)];
    const uint32_t rb = (uint32_t)(pc >> 32) >> 5, first = (uint32_t)pc;
    // The block's rows: activity and the column range (warp 0).
    if (w == 0) {
      const uint32_t u = rb * 32 + lane;
      uint32_t bs = 0, be = 0, lo = 0xFFFFFFFFu, hi = 0;
      bool active = false;
      if (u < g.n) {
        const uint64_t a = g.rp[u], b = g.rp[u + 1];
        bs = rp_blk(a);
        be = rp_blk(b);
        active = rp_row(b) - rp_row(a) >= 2 && be - bs <= kWarpMaxBlocks;
        if (active) {
          lo = (uint32_t)(g.bent[bs] >> 32);
          hi = (uint32_t)(g.bent[be - 1] >> 32);
        }
      }
      const uint32_t amask = __ballot_sync(kFull, active);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
      }
      sm.row_bs[lane] = active ? bs : 0u;
      sm.row_be[lane] = active ? be : 0u;
      if (lane == 0) {
        sm.amask = amask;
        sm.lo = lo;
        sm.K = amask ? hi - lo + 1 : 0u;
      }
    }
    __syncthreads();
    const uint32_t K = sm.K, lo = sm.lo, amask = sm.amask;
    uint64_t racc = 0;
    if (K > (uint32_t)kTileMaxK) {
      // Forced onto a block that fits no tile: its one piece sweeps the rows
      // (warp 0; the operand buffers are its table and run buffer).
      if (first == 0 && w == 0)
        racc = tile_fallback(g, rb, reinterpret_cast<uint64_t*>(sm.a), reinterpret_cast<uint32_t*>(sm.b), per_graph);
    } else if (K > 0) {
      const uint32_t KW = (K + kTcWords - 1) & ~(kTcWords - 1);  // words, whole rounds
      for (uint32_t r = w; r < 32; r += kTcThreads / 32)
        for (uint32_t q = lane; q < KW; q += 32) sm.ubits[r][q] = 0u;
      __syncthreads();
      // The rows' bits: warp w takes rows w, w + 4, ...
      for (uint32_t r = w; r < 32; r += 4) {
        if (!((amask >> r) & 1u)) continue;
        for (uint32_t k = sm.row_bs[r] + lane; k < sm.row_be[r]; k += 32) {
          const uint64_t e = g.bent[k];
          sm.ubits[r][(uint32_t)(e >> 32) - lo] = (uint32_t)e;
        }
      }
      __syncthreads();
      if (tid < (uint32_t)kTileMaxK) {
        uint32_t m = 0;
        if (tid < K)
          for (uint32_t r = 0; r < 32; ++r) m |= sm.ubits[r][tid];
        sm.vmask[tid] = m;
      }
      __syncthreads();
      if (w == 0) {
        const uint32_t c0 = __popc(sm.vmask[2 * lane]), c1 = __popc(sm.vmask[2 * lane + 1]);
        const uint32_t incl = warp_inclusive_sum(c0 + c1);
        sm.vpre[2 * lane] = incl - c0 - c1;
        sm.vpre[2 * lane + 1] = incl - c1;
        if (lane == 31) {
          sm.vpre[kTileMaxK] = incl;
          sm.cnt_v = min(kTileNbrPiece, incl > first ? incl - first : 0u);
        }
      }
      __syncthreads();
      // Neighbour tid of the piece: the (first + tid)-th set bit of V. Its
      // bit row starts at or after block lo (v >= 32 lo) and ascends, so a
      // cursor walks it chunk by chunk: a chunk's kTcWords words hold at most
      // kTcWords of its entries, the next kTcWords from the cursor.
      const uint32_t nv = sm.cnt_v;
      uint32_t vcol = 0xFFFFFFFFu, vk = 0, vend = 0;
      if (tid < nv) {
        const uint32_t idx = first + tid;
        uint32_t wd = 0;
#pragma unroll
        for (uint32_t st = 32; st >= 1; st >>= 1)
          if (wd + st < (uint32_t)kTileMaxK && sm.vpre[wd + st] <= idx) wd += st;
        uint32_t m = sm.vmask[wd];
        for (uint32_t q = idx - sm.vpre[wd]; q > 0; --q) m &= m - 1;
        vcol = wd * 32 + __ffs(m) - 1;
        const uint32_t v = lo * 32 + vcol;
        const uint64_t va = g.rp[v], vb = g.rp[v + 1];
        vk = rp_blk(va);
        vend = vk + min(rp_blk(vb) - vk, K);
      }
      for (uint32_t c = 0; c < KW; c += kTcWords) {
        // This chunk of row tid of A: the neighbour's entries in blocks
        // [lo + c, lo + c + kTcWords) (kTcWords loads issued before any is
        // used), unpacked to kTcWords words = 2 kTcWords groups of 16 bytes.
        // B rows by all threads, a quarter row each.
        {
          constexpr uint32_t kW = kTcWords;
          uint64_t e[kW];
#pragma unroll
          for (uint32_t j = 0; j < kW; ++j) e[j] = vk + j < vend ? g.bent[vk + j] : ~0ull;
          uint32_t wv[kW], used = 0;
#pragma unroll
          for (uint32_t q = 0; q < kW; ++q) wv[q] = 0u;
#pragma unroll
          for (uint32_t j = 0; j < kW; ++j) {
            const uint32_t d = (uint32_t)(e[j] >> 32) - lo - c;  // a missing entry: ~0 - lo - c >= kW
            used += d < kW ? 1u : 0u;
#pragma unroll
            for (uint32_t q = 0; q < kW; ++q) wv[q] |= d == q ? (uint32_t)e[j] : 0u;
          }
          vk += used;
#pragma unroll
          for (uint32_t q = 0; q < kW; ++q) {
            uint4 x0, x1;
            unpack32(wv[q], x0, x1);
            *reinterpret_cast<uint4*>(sm.a + tc_off(tid, 2 * q)) = x0;
            *reinterpret_cast<uint4*>(sm.a + tc_off(tid, 2 * q + 1)) = x1;
          }
        }
        {
          const uint32_t r = tid & 31, q0 = (tid >> 5) * (kTcWords / 4);
          for (uint32_t q = q0; q < q0 + kTcWords / 4; ++q) {
            uint4 x0, x1;
            unpack32(sm.ubits[r][c + q], x0, x1);
            *reinterpret_cast<uint4*>(sm.b + tc_off(r, 2 * q)) = x0;
            *reinterpret_cast<uint4*>(sm.b + tc_off(r, 2 * q + 1)) = x1;
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !test_no_commit) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sbo = (kTcChunk / 16) * 128;
          for (uint32_t ks = 0; ks < kTcChunk / 32; ++ks) {
            const uint64_t ad = umma_desc(sm.a + ks * 256, 128, sbo);
            const uint64_t bd = umma_desc(sm.b + ks * 256, 128, sbo);
            const uint32_t accum = (c > 0 || ks > 0) ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(accum), "r"(0u)
                : "memory");
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&sm.mbar))
                       : "memory");
        }
        // One decision for the whole CTA: a thread whose own polls ran out
        // fails the chunk for every thread, so all threads leave the loop
        // together and no TMEM load follows a failed wait.
        const bool ok = __syncthreads_and(tc_wait(&sm.mbar, phase, max_polls) ? 1 : 0) != 0;
        phase ^= 1u;
        if (!ok) {
          if (tid == 0) {
            atomicOr(&stats->count_err, kErrTimeout);
            sm.fail = 1;
          }
          break;
        }
      }
      __syncthreads();
      if (!sm.fail) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]),
              "=r"(d[15]), "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]),
              "=r"(d[22]), "=r"(d[23]), "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]),
              "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
            : "r"(tmem + ((w * 32u) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // Lane = neighbour v = row 32w + lane of D; column r = row r of the block.
        if (tid < nv) {
          uint64_t sum = 0;
#pragma unroll
          for (int r = 0; r < 32; ++r)
            if ((sm.ubits[r][vcol >> 5] >> (vcol & 31)) & 1u) sum += d[r];
          racc += sum;
          if (per_graph && sum) atomicAdd(&per_graph[g.graph_of_rank[lo * 32 + vcol]], (unsigned long long)sum);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
    }
    acc += racc;
    __syncthreads();
    if (block_ns && tid == 0) atomicAdd(&block_ns[rb], (cycles() - t_start) * (kTcThreads / 32));
  }
  __syncthreads();
  // After a failed wait, the MMAs of the failed chunk may still be running
  // (they were committed; only the wait gave up): give them one more bounded
  // wait of their own budget before their accumulator columns are freed. With
  // nothing committed (the failure-detection test) there is nothing to drain.
  if (sm.fail && !test_no_commit) tc_wait(&sm.mbar, phase ^ 1u, kTcDrainPolls);
  __syncthreads();
  if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
  acc = warp_sum(acc);
  if (lane == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- CTA-per-row pass for rows deferred by the warp kernels ---------------

__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v) {
  __shared__ unsigned long long part[kCtaThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  uint64_t s = 0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0ull;
    s = warp_sum(s);
  }
  __syncthreads();
  return s;  // valid in thread 0
}

__global__ void __launch_bounds__(kCtaThreads) k_rows_cta(GraphView g, const uint32_t* __restrict__ rows,
                                                           DeviceStats* stats, uint32_t* __restrict__ ovf_global,
                                                           unsigned long long* per_graph,
                                                           unsigned long long* block_ns) {
  extern __shared__ __align__(16) uint64_t tbl[];
  __shared__ uint32_t runs[kCtaThreads / 32][64];
  __shared__ uint32_t s_t;
  const uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t len = stats->overflow[kOvfCta];
  uint64_t acc = 0;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(&stats->cursor[kCurCta], 1u);
    __syncthreads();
    const uint32_t t = s_t;
    __syncthreads();
    if (t >= len) break;
    const uint32_t u = rows[t];
    const uint64_t a = g.rp[u], b = g.rp[u + 1];
    const uint32_t rs = rp_row(a), re = rp_row(b), bs = rp_blk(a), be = rp_blk(b), nb = be - bs;
    if (nb > kCtaMaxBlocks) {
      if (threadIdx.x == 0) push_row(stats, kOvfGlobal, ovf_global, u);
      continue;
    }
    const unsigned long long t_start = block_ns ? cycles() : 0ull;
    const int logb = table_logb(nb);
    table_clear(tbl, logb, threadIdx.x, blockDim.x);
    __syncthreads();
    table_insert(tbl, logb, g.bent, bs, be, threadIdx.x, blockDim.x);
    __syncthreads();
    const BitmapProbe probe{tbl, logb, (uint32_t)(g.bent[bs] >> 32), (uint32_t)(g.bent[be - 1] >> 32)};
    const uint64_t racc =
        sweep_bits(g, rs, re, w, nw, probe, runs[w]);
    const uint64_t s = block_sum_u64(racc);  // also the barrier before the table is rebuilt
    if (threadIdx.x == 0) {
      if (per_graph && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
      if (block_ns) atomicAdd(&block_ns[u >> 5], (cycles() - t_start) * (blockDim.x >> 5));
    }
    acc += racc;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- global-memory pass: any row size, binary search in global memory -----

__global__ void __launch_bounds__(kCtaThreads) k_rows_global(GraphView g, const uint32_t* __restrict__ rows,
                                                              DeviceStats* stats, unsigned long long* per_graph) {
  __shared__ uint32_t s_t;
  const uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t len = stats->overflow[kOvfGlobal];
  uint64_t acc = 0;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(&stats->cursor[kCurGlobal], 1u);
    __syncthreads();
    const uint32_t t = s_t;
    __syncthreads();
    if (t >= len) break;
    const uint32_t u = rows[t];
    const uint32_t rs = rp_row(g.rp[u]), re = rp_row(g.rp[u + 1]);
    const uint32_t last = g.col[re - 1];
    const uint64_t racc = sweep<false>(g, rs, re, w, nw, [&](uint32_t k, uint32_t c) -> uint32_t {
      const uint32_t x = g.col[k];
      if (x > last) return 0u;
      uint32_t lo = c + 1, hi = re;
      while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (g.col[mid] < x)
          lo = mid + 1;
        else
          hi = mid;
      }
      return (lo < re && g.col[lo] == x) ? 1u : 0u;
    });
    const uint64_t s = block_sum_u64(racc);
    if (threadIdx.x == 0 && per_graph && s) atomicAdd(&per_graph[g.graph_of_rank[u]], (unsigned long long)s);
    acc += racc;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- hub pass: the merge variant's walks of u's tail ------------------------
// For an edge (u, v) of a merge row block, the sorted-list intersection walks
// the shorter of u's tail (u's bit blocks from v's block on: the only ones
// that can meet N+(v)) and v's bit row. Where the tail is shorter and v's row
// spans at most kHubMaxSpan blocks, the schedule groups the edge under v (the
// hub) and flags it so the row sweeps skip it. A CTA then stages v's bit row
// once as a direct-mapped array of masks over its block span, and its warps
// walk the tails of a piece of v's in-edges against it: per tail block one
// shared-memory load, AND and popc, and no search. A hub row spanning more
// than kHubMaxSpan blocks but holding at most kHubMaxHash blocks is staged as
// a bucketed hash instead (one bucket load per tail block). Hubs whose row fits a
// warp's slice of the map (kHubWarpSpan blocks) are staged and walked by one
// warp alone, with no CTA barrier per piece. Every edge is counted exactly
// once, here or by its row.

// Build-time tunables (-D...): measured defaults.
#ifndef TB_HUB_PIECE
#define TB_HUB_PIECE 512
#endif
#ifndef TB_HUB_DEPTH
#define TB_HUB_DEPTH 4
#endif
constexpr int kHubWarps = 8;
#ifndef TB_HUB_MAX_SPAN
#define TB_HUB_MAX_SPAN 8192
#endif
constexpr uint32_t kHubMaxSpan = TB_HUB_MAX_SPAN;  // blocks of v's row span staged direct-mapped by a CTA (4 bytes each)
constexpr uint32_t kHubWarpSpan = kHubMaxSpan / kHubWarps;  // spans up to this: one warp per piece
// A warp's slice of the map: its span plus a zero word past the staged masks,
// rounded to 16 bytes for the hash buckets (16-byte loads).
constexpr uint32_t kHubWarpStride = kHubWarpSpan + 4;
constexpr uint32_t kHubMapWords = kHubWarps * kHubWarpStride;  // >= kHubMaxSpan + 1
static_assert(kHubWarpStride % 4 == 0, "warp slices hold 16-byte hash buckets");
static_assert(kHubMapWords >= kHubMaxSpan + 1, "the CTA map needs its zero word");
// Rows spanning more than that are staged as a bucketed hash instead (the same
// 32 KiB, or a warp's 4 KiB slice, as 8-byte slots at most half full).
constexpr uint32_t kHubMaxHash = kHubMaxSpan / 4;          // bit blocks: CTA hash
#ifndef TB_HUB_HASH_MUL
#define TB_HUB_HASH_MUL 4
#endif
#ifndef TB_HUB_HASH_MIN
#define TB_HUB_HASH_MIN 1024
#endif
constexpr uint32_t kHubHashMul = TB_HUB_HASH_MUL;  // hashed hubs must save this many times their staging
constexpr uint32_t kHubHashMin = TB_HUB_HASH_MIN;  // ... plus this many blocks (0 / 0: no hashed hubs)
constexpr uint32_t kHubWarpHash = kHubWarpSpan / 4;        // bit blocks: warp hash
constexpr uint32_t kHubPiece = TB_HUB_PIECE;    // in-edges per CTA piece
#ifndef TB_HUB_WARP_PIECE
#define TB_HUB_WARP_PIECE 128
#endif
constexpr uint32_t kHubWarpPiece = TB_HUB_WARP_PIECE;  // in-edges per warp piece
#ifndef TB_HUB_WAVES
#define TB_HUB_WAVES 32
#endif
constexpr uint32_t kHubWaves = TB_HUB_WAVES;    // row ranges the hub pieces are ordered by (power of 2)
// Up to this many entries (bit rows of at most 64 MiB) the in-lists are filled
// in one launch instead of one per wave.
constexpr uint64_t kHubOneWaveEntries = 1ull << 23;
// Five CTAs per SM (48 registers), the occupancy the 41 KiB of shared memory
// allows; with four the pair loads' extra registers cost more than they save.
#ifndef TB_HUB_MIN_CTAS
#define TB_HUB_MIN_CTAS 5
#endif
constexpr int kHubCtasPerSm = TB_HUB_MIN_CTAS;
constexpr int kHubDepth = TB_HUB_DEPTH;         // tail blocks in flight per lane
#ifndef TB_HUB_PAIRS
#define TB_HUB_PAIRS 1
#endif
constexpr bool kHubPairs = TB_HUB_PAIRS != 0;   // tails read as 16-byte pairs of entries
// A hub tail holding at most TB_HUB_COL_RATIO / 100 neighbours a bit block is
// walked as u's column ids after v (4 bytes a neighbour) instead of its bit-row
// entries (8 bytes a block); 0 walks every tail as bit rows. Each hub's
// in-list holds its bit-row tails first (in_cnt[v] of them), then its column
// tails. 1.75 measured best on RMAT-24 and RMAT-22 (1.0 to 3.0 swept).
#ifndef TB_HUB_COL_RATIO
#define TB_HUB_COL_RATIO 175
#endif
constexpr uint32_t kHubColRatio = TB_HUB_COL_RATIO;
#ifndef TB_HUB_COL_DEPTH
#define TB_HUB_COL_DEPTH 2
#endif
constexpr int kHubColDepth = TB_HUB_COL_DEPTH;  // 16-byte quads of column ids in flight per lane

// Walks the tails of in-list entries [cs, ce) (at list) against v's staged row:
// direct-mapped masks over blocks [bmin, bmin + span) in map, or a bucketed
// hash (map as 8-byte slots, 2^logb buckets).
// The hub tails' walk (see sweep_runs) with 16-byte loads: a tail's blocks are
// read as aligned pairs of bit-row entries, so each load, address and owner
// check serves two blocks; the pair's entries outside the tail are masked.
// Chunks of short tails keep the per-item sweep. wsm: 128 words of the warp.
template <int DepthPairs, class Probe>
__device__ __forceinline__ uint64_t sweep_tail_pairs(const GraphView& g, const uint64_t* __restrict__ list,
                                                     uint32_t cs, uint32_t ce, const Probe& probe, uint32_t* wsm) {
  const uint32_t lane = threadIdx.x & 31;
  const ulonglong2* __restrict__ pairs = reinterpret_cast<const ulonglong2*>(g.bent);
  uint64_t acc = 0;
  for (uint32_t c = cs; c < ce; c += 32) {
    const uint32_t j = c + lane;
    uint32_t ib = 0, il = 0;
    if (j < ce) {
      const uint64_t x = list[j];
      ib = (uint32_t)(x >> 32);
      il = (uint32_t)x;
    }
    const uint32_t items = warp_sum(il);
    if (items < 32 * 8) {
      acc += sweep_runs<2 * DepthPairs, 8>(
          c, min(c + 32, ce), 0, 1,
          [&](uint32_t i, uint32_t& b, uint32_t& l) {
            const uint64_t x = list[i];
            b = (uint32_t)(x >> 32);
            l = (uint32_t)x;
          },
          [&](uint32_t k) -> uint64_t { return g.bent[k]; }, probe, wsm);
      continue;
    }
    const uint32_t ie = ib + il;
    const uint32_t p0 = ib >> 1, pn = il ? ((ie + 1) >> 1) - p0 : 0u;  // pairs covering [ib, ie)
    const uint32_t incl = warp_inclusive_sum(pn);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    __syncwarp();
    wsm[lane] = incl;
    wsm[32 + lane] = p0 - (incl - pn);  // pair t of the chunk, owned by slot s, is pair off_s + t
    wsm[64 + lane] = ib;
    wsm[96 + lane] = ie;
    __syncwarp();
    uint32_t s = 0;
#pragma unroll
    for (uint32_t st = 16; st >= 1; st >>= 1)
      if (wsm[s + st - 1] <= lane) s += st;
    uint32_t lim = wsm[s], off = wsm[32 + s], lo = wsm[64 + s], hi = wsm[96 + s];
    uint32_t racc = 0;
    for (uint32_t base = 0; base < total; base += 32 * DepthPairs) {
      ulonglong2 x[DepthPairs];
      uint32_t keep[DepthPairs];
#pragma unroll
      for (int r = 0; r < DepthPairs; ++r) {
        const uint32_t t = base + 32 * r + lane;
        while (t >= lim && s < 31) {
          ++s;
          lim = wsm[s];
          off = wsm[32 + s];
          lo = wsm[64 + s];
          hi = wsm[96 + s];
        }
        keep[r] = 0;
        x[r] = make_ulonglong2(0ull, 0ull);
        if (t < total) {
          const uint32_t p = off + t, k0 = 2 * p;
          x[r] = pairs[p];
          keep[r] = (k0 >= lo ? 1u : 0u) | (k0 + 1 < hi ? 2u : 0u);
        }
      }
#pragma unroll
      for (int r = 0; r < DepthPairs; ++r)
        racc += probe(Probe::drop(x[r].x, keep[r] & 1u)) + probe(Probe::drop(x[r].y, keep[r] & 2u));
    }
    acc += racc;
  }
  __syncwarp();
  return acc;
}

// Column tails (in-list entries (first CSR position << 32) | neighbours): u's
// neighbours after v, read as aligned 16-byte quads of column ids (the col
// array has three ids of padding past its end), each id probing v's staged
// row as a one-bit entry. Chunks of short tails keep the per-item sweep.
template <int DepthQuads, class Probe>
__device__ __forceinline__ uint64_t sweep_col_quads(const GraphView& g, const uint64_t* __restrict__ list,
                                                    uint32_t cs, uint32_t ce, const Probe& probe, uint32_t* wsm) {
  const uint32_t lane = threadIdx.x & 31;
  const uint4* __restrict__ quads = reinterpret_cast<const uint4*>(g.col);
  uint64_t acc = 0;
  for (uint32_t c = cs; c < ce; c += 32) {
    const uint32_t j = c + lane;
    uint32_t ib = 0, il = 0;
    if (j < ce) {
      const uint64_t x = list[j];
      ib = (uint32_t)(x >> 32);
      il = (uint32_t)x;
    }
    const uint32_t items = warp_sum(il);
    if (items < 32 * 8) {
      acc += sweep_runs<2 * DepthQuads, 8>(
          c, min(c + 32, ce), 0, 1,
          [&](uint32_t i, uint32_t& b, uint32_t& l) {
            const uint64_t x = list[i];
            b = (uint32_t)(x >> 32);
            l = (uint32_t)x;
          },
          [&](uint32_t k) -> uint64_t { return col_entry(g.col[k], true); }, probe, wsm);
      continue;
    }
    const uint32_t ie = ib + il;
    const uint32_t q0 = ib >> 2, qn = il ? ((ie + 3) >> 2) - q0 : 0u;  // quads covering [ib, ie)
    const uint32_t incl = warp_inclusive_sum(qn);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    __syncwarp();
    wsm[lane] = incl;
    wsm[32 + lane] = q0 - (incl - qn);  // quad t of the chunk, owned by slot s, is quad off_s + t
    wsm[64 + lane] = ib;
    wsm[96 + lane] = ie;
    __syncwarp();
    uint32_t s = 0;
#pragma unroll
    for (uint32_t st = 16; st >= 1; st >>= 1)
      if (wsm[s + st - 1] <= lane) s += st;
    uint32_t lim = wsm[s], off = wsm[32 + s], lo = wsm[64 + s], hi = wsm[96 + s];
    uint32_t racc = 0;
    for (uint32_t base = 0; base < total; base += 32 * DepthQuads) {
      uint4 x[DepthQuads];
      uint32_t keep[DepthQuads];  // bit i: id i of the quad lies in the tail
#pragma unroll
      for (int r = 0; r < DepthQuads; ++r) {
        const uint32_t t = base + 32 * r + lane;
        while (t >= lim && s < 31) {
          ++s;
          lim = wsm[s];
          off = wsm[32 + s];
          lo = wsm[64 + s];
          hi = wsm[96 + s];
        }
        x[r] = make_uint4(0u, 0u, 0u, 0u);
        keep[r] = 0u;
        if (t < total) {
          const uint32_t q = off + t, k = 4 * q;
          x[r] = quads[q];
          // ids [k, k + 4) within [lo, hi): 15 << 0..3 trimmed at both ends
          const uint32_t first = lo > k ? lo - k : 0u, last = hi - k < 4u ? hi - k : 4u;
          keep[r] = (0xFu >> (4u - last)) & (0xFu << first);
        }
      }
#pragma unroll
      for (int r = 0; r < DepthQuads; ++r)
        racc += probe.col(x[r].x, keep[r] & 1u) + probe.col(x[r].y, keep[r] & 2u) + probe.col(x[r].z, keep[r] & 4u) +
                probe.col(x[r].w, keep[r] & 8u);
    }
    acc += racc;
  }
  __syncwarp();
  return acc;
}

// v's row staged as direct-mapped masks over blocks [bmin, bmin + span), with
// map[span] = 0: a block outside the span reads that zero word instead of
// taking a branch.
struct DirectProbe {
  const uint32_t* map;
  uint32_t bmin, span;
  __device__ __forceinline__ uint32_t operator()(uint64_t e) const {
    return (uint32_t)__popc((uint32_t)e & map[min((uint32_t)(e >> 32) - bmin, span)]);
  }
  // Column id w: its bit of the staged mask word (a dropped id reads the zero word).
  __device__ __forceinline__ uint32_t col(uint32_t w, bool keep) const {
    return (map[keep ? min((w >> 5) - bmin, span) : span] >> (w & 31)) & 1u;
  }
  // e, or e with an empty mask: a dropped entry still probes, and matches nothing.
  static __device__ __forceinline__ uint64_t drop(uint64_t e, bool keep) {
    return keep ? e : e & 0xFFFFFFFF00000000ull;
  }
};

__device__ __forceinline__ uint64_t hub_sweep(const GraphView& g, const uint64_t* __restrict__ list, uint32_t cs,
                                              uint32_t ce, bool direct, const uint32_t* map, uint32_t bmin,
                                              uint32_t bmax, int logb, uint32_t* wsm) {
  auto desc = [&](uint32_t i, uint32_t& ib, uint32_t& il) {
    const uint64_t x = list[i];
    ib = (uint32_t)(x >> 32);
    il = (uint32_t)x;
  };
  auto load = [&](uint32_t k) -> uint64_t { return g.bent[k]; };
  if (direct) {
    const DirectProbe probe{map, bmin, bmax - bmin + 1};
    if (kHubPairs) return sweep_tail_pairs<kHubDepth / 2>(g, list, cs, ce, probe, wsm);
    return sweep_runs<kHubDepth, 8>(cs, ce, 0, 1, desc, load, probe, wsm);
  }
  const BitmapProbe probe{reinterpret_cast<const uint64_t*>(map), logb, bmin, bmax};
  if (kHubPairs) return sweep_tail_pairs<kHubDepth / 2>(g, list, cs, ce, probe, wsm);
  return sweep_runs<kHubDepth, 8>(cs, ce, 0, 1, desc, load, probe, wsm);
}

// Column tails [cs, ce) of the list against v's staged row (see sweep_col_quads).
__device__ __forceinline__ uint64_t hub_sweep_col(const GraphView& g, const uint64_t* __restrict__ list, uint32_t cs,
                                                  uint32_t ce, bool direct, const uint32_t* map, uint32_t bmin,
                                                  uint32_t bmax, int logb, uint32_t* wsm) {
  if (cs >= ce) return 0;  // uniform across the warp
  if (direct) return sweep_col_quads<kHubColDepth>(g, list, cs, ce, DirectProbe{map, bmin, bmax - bmin + 1}, wsm);
  const BitmapProbe probe{reinterpret_cast<const uint64_t*>(map), logb, bmin, bmax};
  return sweep_col_quads<kHubColDepth>(g, list, cs, ce, probe, wsm);
}

// Shared memory of the hub body: the map (kHubMapWords words; warp w's slice
// at w * kHubWarpStride), the tail-length prefix (kHubPiece + 1), the warps'
// run buffers (run_stride words apart, >= 128) and two CTA words.
struct HubShared {
  uint32_t* map;
  uint32_t* pre;
  uint32_t* runs;
  uint32_t run_stride;
  uint32_t* s_t;
  unsigned long long* s_dt;
};

// The hub pass: CTA pieces, then warp pieces; returns this thread's partial count.
__device__ __forceinline__ uint64_t hub_body(const GraphView& g, const uint64_t* __restrict__ hub_pieces,
                                             const uint32_t* __restrict__ piece_off,
                                             const uint32_t* __restrict__ in_off,
                                             const uint32_t* __restrict__ in_bits, const uint64_t* __restrict__ inl,
                                             const uint32_t* __restrict__ inrow, DeviceStats* stats,
                                             unsigned long long* per_graph, unsigned long long* block_ns,
                                             const HubShared& sh) {
  uint32_t* map = sh.map;
  uint32_t* pre = sh.pre;
  uint32_t& s_t = *sh.s_t;
  unsigned long long& s_dt = *sh.s_dt;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* wruns = sh.runs + w * sh.run_stride;
  const uint32_t len = piece_off[TRIBIT_NUM_VARIANTS + 2];  // CTA pieces; warp pieces follow them
  const uint32_t wlen = piece_off[TRIBIT_NUM_VARIANTS + 3] - len;
  uint64_t acc = 0;
  // Phase 1: hubs with wide rows, one CTA per piece.
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(&stats->cursor[kCurHub], 1u);
    __syncthreads();
    const uint32_t t = s_t;
    if (t >= len) break;
    const unsigned long long t_start = block_ns ? cycles() : 0ull;
    // Pieces are in wave order (see k_wave_bounds).
    const uint64_t pc = hub_pieces[t];
    const uint32_t v = (uint32_t)(pc >> 32);
    const uint32_t e0 = in_off[v] + (uint32_t)pc;
    const uint32_t cnt = min(kHubPiece, in_off[v + 1] - e0);
    const uint64_t a = g.rp[v], b = g.rp[v + 1];
    const uint32_t bs = rp_blk(a), be = rp_blk(b);
    const uint32_t bmin = (uint32_t)(g.bent[bs] >> 32), bmax = (uint32_t)(g.bent[be - 1] >> 32);
    const uint32_t span = bmax - bmin + 1;
    const bool direct = span <= kHubMaxSpan;  // else be - bs <= kHubMaxHash (schedule)
    uint64_t* htbl = reinterpret_cast<uint64_t*>(map);
    const int logb = table_logb(be - bs);
    if (direct) {
      for (uint32_t i = threadIdx.x; i <= span; i += blockDim.x) map[i] = 0u;  // and the zero word
    } else {
      table_clear(htbl, logb, threadIdx.x, blockDim.x);
    }
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) pre[i] = (uint32_t)inl[e0 + i];
    __syncthreads();
    if (direct) {
      for (uint32_t k = bs + threadIdx.x; k < be; k += blockDim.x) {
        const uint64_t e = g.bent[k];
        map[(uint32_t)(e >> 32) - bmin] = (uint32_t)e;
      }
    } else {
      table_insert(htbl, logb, g.bent, bs, be, threadIdx.x, blockDim.x);
    }
    // Tail-length prefix: pre[i] = blocks of the tails before i, pre[cnt] = all.
    {
      const uint32_t per = (cnt + blockDim.x - 1) / blockDim.x, j0 = threadIdx.x * per;
      uint32_t lsum = 0;
      for (uint32_t k = 0; k < per && j0 + k < cnt; ++k) lsum += pre[j0 + k];
      uint32_t tot;
      uint32_t ex = block_exclusive_scan<uint32_t>(lsum, OpSum{}, 0u, &tot);
      for (uint32_t k = 0; k < per && j0 + k < cnt; ++k) {
        const uint32_t x = pre[j0 + k];
        pre[j0 + k] = ex;
        ex += x;
      }
      if (threadIdx.x == 0) pre[cnt] = tot;
    }
    __syncthreads();
    // Warp w walks the tails whose first block falls in the w-th equal share.
    const uint32_t tot = pre[cnt];
    auto first_at = [&](uint32_t x) -> uint32_t {  // first i with pre[i] >= x
      uint32_t lo = 0, hi = cnt;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pre[mid] < x)
          lo = mid + 1;
        else
          hi = mid;
      }
      return lo;
    };
    const uint32_t cs = first_at((uint32_t)((uint64_t)tot * w / kHubWarps));
    const uint32_t ce = w + 1 == kHubWarps ? cnt : first_at((uint32_t)((uint64_t)tot * (w + 1) / kHubWarps));
    // Entries before nbits are bit-row tails, the rest column tails.
    const uint32_t nbits = kHubColRatio ? min(cnt, in_off[v] + in_bits[v] - min(e0, in_off[v] + in_bits[v]))
                                        : cnt;
    uint64_t racc = hub_sweep(g, inl + e0, cs, min(ce, nbits), direct, map, bmin, bmax, logb, wruns);
    if (kHubColRatio) racc += hub_sweep_col(g, inl + e0, max(cs, nbits), ce, direct, map, bmin, bmax, logb, wruns);
    if (per_graph) {
      const uint64_t s = warp_sum(racc);
      if (lane == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[v]], (unsigned long long)s);
    }
    acc += racc;
    __syncthreads();
    if (block_ns) {
      // The piece's warp-cycles, shared among its in-edges' row blocks by tail length.
      if (threadIdx.x == 0) s_dt = cycles() - t_start;
      __syncthreads();
      const double per_block = (double)s_dt * kHubWarps / (double)max(tot, 1u);  // warp-cycles per tail block
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
        atomicAdd(&block_ns[inrow[e0 + i] >> 5], (unsigned long long)(per_block * (pre[i + 1] - pre[i]) + 0.5));
      __syncthreads();
    }
  }
  // Phase 2: hubs whose row fits a warp's slice of the map, one warp per
  // piece, in wave order.
  uint32_t* wmap = map + w * kHubWarpStride;
  for (;;) {
    uint32_t t0 = 0;
    if (lane == 0) t0 = atomicAdd(&stats->cursor[kCurHubWarp], 1u);
    const uint32_t t = __shfl_sync(kFull, t0, 0);
    if (t >= wlen) break;
    const unsigned long long t_start = block_ns ? cycles() : 0ull;
    const uint64_t pc = hub_pieces[len + t];
    const uint32_t v = (uint32_t)(pc >> 32);
    const uint32_t e0 = in_off[v] + (uint32_t)pc;
    const uint32_t cnt = min(kHubWarpPiece, in_off[v + 1] - e0);
    const uint64_t a = g.rp[v], b = g.rp[v + 1];
    const uint32_t bs = rp_blk(a), be = rp_blk(b);
    const uint32_t bmin = (uint32_t)(g.bent[bs] >> 32), bmax = (uint32_t)(g.bent[be - 1] >> 32);
    const uint32_t span = bmax - bmin + 1;
    const bool direct = span <= kHubWarpSpan;  // else be - bs <= kHubWarpHash (schedule)
    const int logb = table_logb(be - bs);
    if (direct) {
      for (uint32_t i = lane; i <= span; i += 32) wmap[i] = 0u;  // and the zero word
      __syncwarp();
      for (uint32_t k = bs + lane; k < be; k += 32) {
        const uint64_t e = g.bent[k];
        wmap[(uint32_t)(e >> 32) - bmin] = (uint32_t)e;
      }
    } else {
      uint64_t* wtbl = reinterpret_cast<uint64_t*>(wmap);
      table_clear(wtbl, logb, lane, 32);
      __syncwarp();
      table_insert(wtbl, logb, g.bent, bs, be, lane, 32);
    }
    __syncwarp();
    const uint32_t nbits = kHubColRatio ? min(cnt, in_off[v] + in_bits[v] - min(e0, in_off[v] + in_bits[v]))
                                        : cnt;
    uint64_t racc = hub_sweep(g, inl + e0, 0, nbits, direct, wmap, bmin, bmax, logb, wruns);
    if (kHubColRatio) racc += hub_sweep_col(g, inl + e0, nbits, cnt, direct, wmap, bmin, bmax, logb, wruns);
    if (per_graph) {
      const uint64_t s = warp_sum(racc);
      if (lane == 0 && s) atomicAdd(&per_graph[g.graph_of_rank[v]], (unsigned long long)s);
    }
    acc += racc;
    if (block_ns) {
      // The piece's cycles, shared among its in-edges' row blocks by tail length.
      uint32_t tot = 0;
      for (uint32_t i = lane; i < cnt; i += 32) tot += (uint32_t)inl[e0 + i];
      tot = warp_sum(tot);
      const double per_block = (double)(cycles() - t_start) / (double)max(tot, 1u);
      for (uint32_t i = lane; i < cnt; i += 32)
        atomicAdd(&block_ns[inrow[e0 + i] >> 5], (unsigned long long)(per_block * (uint32_t)inl[e0 + i] + 0.5));
    }
    __syncwarp();  // the slice is rewritten for the next piece
  }
  return acc;
}

__global__ void __launch_bounds__(kHubWarps * 32, TB_HUB_MIN_CTAS) k_hub(GraphView g, const uint64_t* __restrict__ hub_pieces,
                                                        const uint32_t* __restrict__ piece_off,
                                                        const uint32_t* __restrict__ in_off,
                                                        const uint32_t* __restrict__ in_bits,
                                                        const uint64_t* __restrict__ inl,
                                                        const uint32_t* __restrict__ inrow, DeviceStats* stats,
                                                        unsigned long long* per_graph,
                                                        unsigned long long* block_ns) {
  __shared__ __align__(16) uint32_t map[kHubMapWords];
  __shared__ uint32_t pre[kHubPiece + 1];
  __shared__ uint32_t runs[kHubWarps][128];
  __shared__ uint32_t s_t;
  __shared__ unsigned long long s_dt;
  const HubShared sh{map, pre, &runs[0][0], 128, &s_t, &s_dt};
  uint64_t acc = hub_body(g, hub_pieces, piece_off, in_off, in_bits, inl, inrow, stats, per_graph, block_ns, sh);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}


// ---- one persistent kernel over the work queue ------------------------------
// The row-piece and hub work of one counting launch in one persistent kernel:
// each CTA takes, from the device cursors in turn, heavy rows (one CTA each),
// then each warp bitmap and merge pieces, then the CTA hub CTA pieces and each
// warp hub warp pieces, so no CTA waits at a kernel boundary for another
// kernel's tail. The
// bit tiles (128-thread CTAs with tensor memory) and the fallback rows (128
// KiB tables), which need other CTA shapes, keep their own kernels. Shared
// memory: warp w's slice at w * kHubWarpStride words serves both bodies (a
// row-piece table needs kWarpSlots 8-byte words), and the CTA phases use the
// whole map.
static_assert(kWarpsPerCta == kHubWarps, "the two bodies share the CTA shape");
static_assert(kHubWarpStride % 4 == 0 && kHubWarpStride * 4 >= kWarpSlots * 8, "a warp slice holds a row table");
static_assert(kHubMapWords * 4 >= kWarpsPerCta * kWarpSlots * 8, "the map holds the CTA row table and prefix");
__global__ void __launch_bounds__(kHubWarps * 32, TB_HUB_MIN_CTAS) k_queue(
    GraphView g, const uint64_t* __restrict__ pieces, const uint32_t* __restrict__ piece_off, DeviceStats* stats,
    uint32_t* __restrict__ ovf_cta, unsigned long long* per_graph, const uint32_t* __restrict__ heavy, uint32_t width,
    const uint64_t* __restrict__ hub_pieces, const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_bits,
    const uint64_t* __restrict__ inl) {
  __shared__ __align__(16) uint32_t map[kHubMapWords];
  __shared__ uint32_t pre[kHubPiece + 1];
  __shared__ uint32_t runs[kHubWarps][128];
  __shared__ uint32_t s_t;
  __shared__ unsigned long long s_dt;
  const PiecesShared ps{reinterpret_cast<uint64_t*>(map), kHubWarpStride / 2, &runs[0][0], 128, &s_t};
  const HubShared hs{map, pre, &runs[0][0], 128, &s_t, &s_dt};
  uint64_t acc = 0;
  // The separate kernels' order: heavy rows (CTA), bitmap and merge pieces
  // (warps), then, once the CTA's warps meet, the hub's CTA pieces and its
  // warp pieces. (Hub CTA pieces right after the heavy rows, before the warp
  // pieces, measured 0.5-3% slower on RMAT-18 to 24.)
  acc += pieces_body<TRIBIT_VARIANT_BITMAP>(g, pieces, piece_off, stats, ovf_cta, per_graph, nullptr, heavy, width, ps);
  acc += pieces_body<TRIBIT_VARIANT_MERGE>(g, pieces, piece_off, stats, ovf_cta, per_graph, nullptr, nullptr, width,
                                           ps);
  __syncthreads();  // the hub's CTA pieces take the whole map
  acc += hub_body(g, hub_pieces, piece_off, in_off, in_bits, inl, nullptr, stats, per_graph, nullptr, hs);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&stats->triangles, (unsigned long long)acc);
}

// ---- schedule ----------------------------------------------------------------

// Row-block features (one warp per row block) and the plain dispatcher's
// choice. Features are log-scaled so the learned dispatcher sees O(1) inputs.
__global__ void k_features(GraphView g, uint32_t nrb, int mode, float* __restrict__ feat,
                           uint8_t* __restrict__ variant_of, int full, float tile_min_nnz, float merge_ratio) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t rb = warp; rb < nrb; rb += nwarps) {
    const uint32_t u = rb * 32 + lane;
    uint32_t d = 0, nbu = 0, lo = 0xFFFFFFFFu, hi = 0;
    if (u < g.n) {
      const uint64_t a = g.rp[u], b = g.rp[u + 1];
      d = rp_row(b) - rp_row(a);
      nbu = rp_blk(b) - rp_blk(a);
      if (d >= 2 && nbu <= kWarpMaxBlocks) {
        lo = (uint32_t)(g.bent[rp_blk(a)] >> 32);
        hi = (uint32_t)(g.bent[rp_blk(b) - 1] >> 32);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(kFull, lo, o));
      hi = max(hi, __shfl_xor_sync(kFull, hi, o));
    }
    const float span = hi >= lo ? (float)(hi - lo + 1) : 0.f;  // column blocks the tile would cover
    const float fd = (float)d;
    const float rows = (float)warp_sum(d >= 2 ? 1u : 0u);
    const float nnz = (float)warp_sum(d);
    const float nb = (float)warp_sum(nbu);
    const float sq = warp_sum(fd * fd);
    uint32_t dmax = d;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(kFull, dmax, o));
    // Neighbour-side work: the bit blocks and ids the sweeps will read.
    float wb = 0.f, wm = 0.f, vmax = 0.f, top = 0.f;
    if (full) {
      for (uint32_t r = 0; r < 32; ++r) {
        const uint32_t ur = rb * 32 + r;
        if (ur >= g.n) break;
        const uint64_t a = g.rp[ur], b = g.rp[ur + 1];
        const uint32_t rs = rp_row(a), re = rp_row(b);
        if (re - rs < 2) continue;
        for (uint32_t k = rs + lane; k < re; k += 32) {
          const uint32_t v = g.col[k];
          const uint64_t va = g.rp[v], vb = g.rp[v + 1];
          const float dv = (float)(rp_row(vb) - rp_row(va));
          wb += (float)(rp_blk(vb) - rp_blk(va));
          wm += dv;
          vmax = fmaxf(vmax, dv);
          top += v + 4096u >= g.n ? 1.f : 0.f;
        }
      }
      wb = warp_sum(wb);
      wm = warp_sum(wm);
      top = warp_sum(top);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(kFull, vmax, o));
    }
    if (lane == 0) {
      float* f = feat + (size_t)rb * kNumFeatures;
      const float mean = rows > 0 ? nnz / fmaxf(rows, 1.f) : 0.f;
      f[0] = rows / 32.f;
      f[1] = log2f(1.f + nnz);
      f[2] = log2f(1.f + nb);
      f[3] = nb > 0 ? nnz / (32.f * nb) : 0.f;
      f[4] = log2f(1.f + mean);
      f[5] = log2f(1.f + (float)dmax);
      f[6] = log2f(1.f + sqrtf(fmaxf(sq / 32.f - (nnz / 32.f) * (nnz / 32.f), 0.f)));
      f[7] = log2f(1.f + wb);
      f[8] = log2f(1.f + wm);
      f[9] = wb > 0 ? log2f(wm / wb) : 0.f;
      f[10] = log2f(1.f + vmax);
      f[11] = nnz > 0 ? top / nnz : 0.f;
      f[12] = (float)rb * 32.f / fmaxf((float)g.n, 1.f);
      f[13] = log2f(1.f + span);
      f[14] = nnz > 0 ? log2f(1.f + wb / nnz) : 0.f;
      f[15] = log2f(1.f + sq);
      // Plain dispatcher: fixed thresholds. Bit tiles where the block's rows
      // share one narrow column range and are dense in it (at least 1/8 of
      // the 32 x 32 * span cells set, and tile_min_nnz edges): on disjoint
      // cliques tiles beat the sweeps, on sparse small graphs (1-2 % dense)
      // they lose. Otherwise the sorted-list merge where the neighbours' bit
      // rows average at least merge_ratio times the block's own (wb / nnz
      // against nb / rows; needs the neighbour-side pass): the power-law
      // case, where the merge's hub pass walks u's short tail against a long,
      // staged row of v instead of probing every block of v. The bitmap sweep
      // everywhere else (rows and neighbours of similar length).
      uint8_t var = TRIBIT_VARIANT_BITMAP;
      if (span > 0.f && span <= (float)kTileMaxK && nnz >= tile_min_nnz && nnz >= span * (1024.f / kTileMinDensityInv))
        var = TRIBIT_VARIANT_MMA;
      else if (full && rows > 0.f && nnz > 0.f && wb >= merge_ratio * nnz * (nb / rows))
        var = TRIBIT_VARIANT_MERGE;
      if (mode == TRIBIT_DISPATCH_BITMAP) var = TRIBIT_VARIANT_BITMAP;
      if (mode == TRIBIT_DISPATCH_MERGE) var = TRIBIT_VARIANT_MERGE;
      if (mode == TRIBIT_DISPATCH_MMA) var = TRIBIT_VARIANT_MMA;
      variant_of[rb] = var;
    }
  }
}

// Pieces of row u; rows wider than a warp's table are counted whole in the
// heavy phase instead and get none.
__device__ __forceinline__ uint32_t row_pieces(const GraphView& g, uint32_t u, uint32_t width) {
  if (u >= g.n) return 0u;
  const uint64_t a = g.rp[u], b = g.rp[u + 1];
  const uint32_t d = rp_row(b) - rp_row(a);
  if (d < 2 || rp_blk(b) - rp_blk(a) > kWarpMaxBlocks) return 0u;
  return (d + width - 1) / width;
}

__global__ void k_heavy_flags(GraphView g, uint32_t* __restrict__ flags) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u > g.n) return;
  uint32_t f = 0;
  if (u < g.n) {
    const uint64_t a = g.rp[u], b = g.rp[u + 1];
    f = (rp_row(b) - rp_row(a) >= 2 && rp_blk(b) - rp_blk(a) > kWarpMaxBlocks) ? 1u : 0u;
  }
  flags[u] = f;
}

__global__ void k_heavy_scatter(GraphView g, const uint32_t* __restrict__ pos, uint32_t* __restrict__ heavy,
                                uint32_t* __restrict__ piece_off) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < g.n && pos[u + 1] != pos[u]) heavy[pos[u]] = u;
  if (u == g.n) piece_off[TRIBIT_NUM_VARIANTS + 1] = pos[g.n];
}

// Pieces of a bit-tile row block: its neighbour set V (the OR of the active
// rows' bit rows over the block's column range) in chunks of kTileNbrPiece;
// one piece when the rows span more than kTileMaxK blocks (swept row by
// row). vm: kTileMaxK words of this warp's shared memory.
__device__ uint32_t tile_pieces(const GraphView& g, uint32_t rb, uint32_t* vm) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t u = rb * 32 + lane;
  uint32_t bs = 0, be = 0, lo = 0xFFFFFFFFu, hi = 0;
  bool active = false;
  if (u < g.n) {
    const uint64_t a = g.rp[u], b = g.rp[u + 1];
    bs = rp_blk(a);
    be = rp_blk(b);
    active = rp_row(b) - rp_row(a) >= 2 && be - bs <= kWarpMaxBlocks;
    if (active) {
      lo = (uint32_t)(g.bent[bs] >> 32);
      hi = (uint32_t)(g.bent[be - 1] >> 32);
    }
  }
  const uint32_t amask = __ballot_sync(kFull, active);
  if (!amask) return 0u;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(kFull, lo, o));
    hi = max(hi, __shfl_xor_sync(kFull, hi, o));
  }
  if (hi - lo + 1 > (uint32_t)kTileMaxK) return 1u;
  for (uint32_t i = lane; i < (uint32_t)kTileMaxK; i += 32) vm[i] = 0u;
  __syncwarp();
  for (uint32_t r = 0; r < 32; ++r) {
    if (!((amask >> r) & 1u)) continue;
    const uint32_t rbs = __shfl_sync(kFull, bs, r), rbe = __shfl_sync(kFull, be, r);
    for (uint32_t k = rbs + lane; k < rbe; k += 32) {
      const uint64_t e = g.bent[k];
      atomicOr(&vm[(uint32_t)(e >> 32) - lo], (uint32_t)e);
    }
  }
  __syncwarp();
  uint32_t c = 0;
  for (uint32_t i = lane; i < (uint32_t)kTileMaxK; i += 32) c += __popc(vm[i]);
  c = warp_sum(c);
  __syncwarp();
  return (c + kTileNbrPiece - 1) / kTileNbrPiece;
}

// Pieces of each row block (one warp per row block): bit-tile blocks by
// tile_pieces, the others one per piece_width neighbours of each row.
__global__ void __launch_bounds__(256) k_block_pieces(GraphView g, uint32_t nrb, const uint8_t* __restrict__ variant_of,
                                                      uint32_t* __restrict__ cnt, uint32_t width) {
  __shared__ uint32_t vm[8][kTileMaxK];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t rb = warp; rb < nrb; rb += nwarps) {
    const uint32_t s = variant_of[rb] == TRIBIT_VARIANT_MMA ? tile_pieces(g, rb, vm[threadIdx.x >> 5])
                                                            : warp_sum(row_pieces(g, rb * 32 + lane, width));
    if (lane == 0) cnt[rb] = s;
  }
}

__global__ void k_piece_flags(const uint8_t* __restrict__ variant_of, const uint32_t* __restrict__ cnt, uint32_t nrb,
                              int v, uint32_t* __restrict__ flags, uint32_t* __restrict__ list_len) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nrb) flags[i] = variant_of[i] == v ? cnt[i] : 0u;
  if (i == nrb) flags[i] = 0u;
  // row blocks per variant, for reporting
  if (i < nrb && variant_of[i] == v && cnt[i]) atomicAdd(&list_len[v], 1u);
}

__global__ void k_piece_segment(const uint32_t* __restrict__ off, uint32_t nrb, int v, uint32_t* piece_off) {
  if (v == 0) piece_off[0] = 0u;
  piece_off[v + 1] = piece_off[v] + off[nrb];
}

__global__ void k_piece_scatter(GraphView g, uint32_t nrb, const uint8_t* __restrict__ variant_of, int v,
                                const uint32_t* __restrict__ off, const uint32_t* __restrict__ piece_off,
                                uint64_t* __restrict__ pieces, uint32_t width) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t seg = piece_off[v];
  for (uint32_t rb = warp; rb < nrb; rb += nwarps) {
    if (variant_of[rb] != v) continue;
    if (v == TRIBIT_VARIANT_MMA) {
      const uint32_t base = seg + off[rb], np = off[rb + 1] - off[rb];
      for (uint32_t k = lane; k < np; k += 32) pieces[base + k] = ((uint64_t)(rb * 32) << 32) | (k * kTileNbrPiece);
      continue;
    }
    const uint32_t u = rb * 32 + lane;
    const uint32_t np = row_pieces(g, u, width);
    const uint32_t incl = warp_inclusive_sum(np);
    const uint32_t base = seg + off[rb] + incl - np;
    for (uint32_t k = 0; k < np; ++k) pieces[base + k] = ((uint64_t)u << 32) | (k * width);
  }
}

// ---- hub schedule -----------------------------------------------------------

// vinfo[v] = (span << 32) | nb: v's bit-row length and the blocks it spans.
__global__ void k_hub_vinfo(GraphView g, uint64_t* __restrict__ vinfo) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= g.n) return;
  const uint64_t a = g.rp[v], b = g.rp[v + 1];
  const uint32_t bs = rp_blk(a), be = rp_blk(b);
  uint64_t x = 0;
  if (be > bs) {
    const uint32_t span = (uint32_t)(g.bent[be - 1] >> 32) - (uint32_t)(g.bent[bs] >> 32) + 1;
    x = ((uint64_t)span << 32) | (be - bs);
  }
  vinfo[v] = x;
}

// Hub candidate: the edge at CSR position j (u -> v; v's block at index pos of
// u's bit row, u's tail `tail` blocks from it) whose tail is shorter than v's
// row, with v stageable. cost: what staging v's row costs (the direct map's
// span / 4 vector stores, or a hash's 2 nb slots cleared, plus nb inserts).
__device__ __forceinline__ unsigned long long hub_cost(uint32_t span, uint32_t nbv) {
  return span <= kHubMaxSpan ? (unsigned long long)(span / 4 + nbv)
                             : (unsigned long long)kHubHashMul * 3ull * nbv + kHubHashMin;
}

__device__ __forceinline__ bool hub_candidate(const uint64_t* __restrict__ vinfo, uint32_t v, uint32_t tail,
                                              uint32_t& nbv, unsigned long long& cost) {
  const uint64_t vi = vinfo[v];
  nbv = (uint32_t)vi;
  const uint32_t span = (uint32_t)(vi >> 32);
  cost = hub_cost(span, nbv);
  return nbv > 0 && tail < nbv && (span <= kHubMaxSpan || (kHubHashMul > 0 && nbv <= kHubMaxHash));
}

// One pass over the edges of the merge row blocks; rows of at most
// kHubLaneRow neighbours are walked by their own lane, longer rows by the
// whole warp (mode 1 on a small wave: one warp per row). For the edge at CSR
// position j, u's tail is u's bit blocks from v's block on.
// Mode 0: counts each hub's candidate in-edges (in_cnt) and adds to save[v]
// the blocks a hub walk saves (v's row length - tail), but only while save[v]
// is below the staging cost: the decision save[v] >= cost (k_hub_accept) is
// then the one the full sum gives, without one atomic per in-edge on the
// most popular hubs.
// Mode 1: every candidate edge of an accepted hub (a vertex whose vinfo
// k_hub_accept kept) is flagged and appended to the hub's in-list: a bit-row
// tail (first block, blocks) at the front (in_cnt[v] counts them), a column
// tail (first CSR position after v, neighbours) at the back (the low word of
// save[v] counts them). rows (may be null): the pass covers rows
// [rows[0], rows[1]).
constexpr uint32_t kHubLaneRow = 64;
#ifndef TB_HUB_TOP
#define TB_HUB_TOP 1024
#endif
// Mode 0 counts the in-edges of the kHubTop highest-ranked vertices in shared
// memory (under degree order they take a fifth to a third of all in-edges, so
// their global counters would see the most contended atomics), one flush per
// CTA.
constexpr uint32_t kHubTop = TB_HUB_TOP;

template <int Mode>
__global__ void k_hub_edges(GraphView g, const uint8_t* __restrict__ variant_of, const uint64_t* __restrict__ vinfo,
                            unsigned long long* __restrict__ save, uint32_t* __restrict__ eflag,
                            uint32_t* __restrict__ in_cnt, const uint32_t* __restrict__ in_off,
                            uint64_t* __restrict__ inl, uint32_t* __restrict__ inrow,
                            const uint32_t* __restrict__ rows) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t u0 = rows ? rows[0] : 0u, u1 = rows ? rows[1] : g.n;  // rows [u0, u1)
  // Mode 0: candidate counts and savings of the vertices ranked top_lo and
  // above, per CTA. A CTA adds to a saving only while it is below the cost,
  // as the global sums do, so a CTA's partial sum either is exact or already
  // reaches the cost by itself: the decision save[v] >= cost is unchanged.
  // Bounded: at most blockDim.x adds of at most nbv each past the cost.
  constexpr uint32_t kTop = Mode == 0 ? kHubTop : 0u;
  __shared__ uint32_t s_top[kTop ? 2 * kTop : 1];
  const uint32_t top_lo = g.n > kTop ? g.n - kTop : 0u;
  if constexpr (kTop != 0) {
    for (uint32_t t = threadIdx.x; t < 2 * kTop; t += blockDim.x) s_top[t] = 0;
    __syncthreads();
  }
  // Whether the edge to v (tail blocks) takes part: mode 0, a candidate;
  // mode 1, a candidate of an accepted hub (k_hub_accept clears the vinfo of
  // every other vertex, so one read decides).
  auto decide = [&](uint32_t v, uint32_t tail, uint32_t& nbv, unsigned long long& cost) -> bool {
    return hub_candidate(vinfo, v, tail, nbv, cost);
  };
  // Applies mode Mode to the taking-part edge at j (v = col[j]; u's row ends
  // at CSR position re) of row u.
  auto edge = [&](uint32_t u, uint32_t bs, uint32_t j, uint32_t re, uint32_t v, uint32_t pos, uint32_t tail,
                  uint32_t nbv, unsigned long long cost) {
    if (Mode == 0) {
      if (kTop && v >= top_lo) {
        uint32_t* c = s_top + 2 * (v - top_lo);
        atomicAdd(c, 1u);
        if (*(volatile uint32_t*)(c + 1) < cost) atomicAdd(c + 1, nbv - tail);
        return;
      }
      atomicAdd(&in_cnt[v], 1u);
      if (*(volatile const unsigned long long*)&save[v] < cost) atomicAdd(&save[v], (unsigned long long)(nbv - tail));
    } else {
      const uint32_t after = re - j - 1;  // u's neighbours after v
      uint32_t at;
      if (kHubColRatio && (uint64_t)after * 100u <= (uint64_t)tail * kHubColRatio) {
        at = in_off[v + 1] - 1u - atomicAdd(reinterpret_cast<uint32_t*>(&save[v]), 1u);
        inl[at] = ((uint64_t)(j + 1) << 32) | after;
      } else {
        at = in_off[v] + atomicAdd(&in_cnt[v], 1u);
        inl[at] = ((uint64_t)(bs + pos) << 32) | tail;
      }
      if (inrow) inrow[at] = u;  // timing mode only
    }
  };
  // Walks row u (CSR [rs, re), nb bit blocks from bs) with the whole warp.
  auto warp_row = [&](uint32_t u, uint32_t rs, uint32_t re, uint32_t bs, uint32_t nb) {
    uint32_t carry = 0, prev_last = 0xFFFFFFFFu;
    for (uint32_t c = rs; c < re; c += 32) {
      const uint32_t j = c + lane;
      const bool in = j < re;
      const uint32_t v = in ? g.col[j] : 0u;
      const uint32_t blk = in ? v >> 5 : 0xFFFFFFFFu;
      uint32_t prev = __shfl_up_sync(kFull, blk, 1);
      if (lane == 0) prev = prev_last;
      const uint32_t incl = warp_inclusive_sum((in && blk != prev) ? 1u : 0u);
      const uint32_t pos = carry + incl - 1;  // index of v's block in u's bit row
      carry += __shfl_sync(kFull, incl, 31);
      prev_last = __shfl_sync(kFull, blk, 31);
      const uint32_t tail = nb - pos;
      uint32_t nbv = 0;
      unsigned long long cost = 0;
      const bool hub = in && decide(v, tail, nbv, cost);
      if (Mode == 1) {
        const uint32_t bits = __ballot_sync(kFull, hub);
        if (lane == 0 && bits) {
          const uint32_t sh = c & 31;
          atomicOr(&eflag[c >> 5], bits << sh);
          if (sh && (bits >> (32 - sh))) atomicOr(&eflag[(c >> 5) + 1], bits >> (32 - sh));
        }
      }
      if (hub) edge(u, bs, j, re, v, pos, tail, nbv, cost);
    }
  };
  if (Mode == 1 && u1 - u0 < 32u * nwarps) {
    // The in-list fill runs once per row wave; a wave of fewer rows than the
    // grid has lanes keeps every warp busy with one warp per row. Larger waves
    // (the first ones: millions of short rows) take the row-block loop below.
    for (uint32_t u = u0 + warp; u < u1; u += nwarps) {
      if (variant_of[u >> 5] != TRIBIT_VARIANT_MERGE) continue;
      const uint64_t a = g.rp[u], b = g.rp[u + 1];
      const uint32_t rs = rp_row(a), re = rp_row(b), bs = rp_blk(a);
      if (re - rs >= 2) warp_row(u, rs, re, bs, rp_blk(b) - bs);
    }
  } else {
    for (uint32_t rb = (u0 >> 5) + warp; rb < ((u1 + 31) >> 5); rb += nwarps) {
      if (variant_of[rb] != TRIBIT_VARIANT_MERGE) continue;
      const uint32_t u = rb * 32 + lane;
      uint32_t rs = 0, re = 0, bs = 0, nbu = 0;
      bool mine = u >= u0 && u < u1;
      if (mine) {
        const uint64_t a = g.rp[u], b = g.rp[u + 1];
        rs = rp_row(a);
        re = rp_row(b);
        bs = rp_blk(a);
        nbu = rp_blk(b) - bs;
        mine = re - rs >= 2;
      }
      const bool own = mine && re - rs <= kHubLaneRow;
      if (own) {
        // Mode 1 gathers the row's flag bits word by word: one atomicOr per
        // 32 CSR positions (a word may hold the ends of other lanes' rows).
        uint32_t pos = 0xFFFFFFFFu, prev = 0xFFFFFFFFu, fw = 0xFFFFFFFFu, fb = 0;
        for (uint32_t j = rs; j < re; ++j) {
          const uint32_t v = g.col[j];
          if ((v >> 5) != prev) {
            ++pos;
            prev = v >> 5;
          }
          const uint32_t tail = nbu - pos;
          uint32_t nbv = 0;
          unsigned long long cost = 0;
          if (!decide(v, tail, nbv, cost)) continue;
          if (Mode == 1) {
            if ((j >> 5) != fw) {
              if (fb) atomicOr(&eflag[fw], fb);
              fw = j >> 5;
              fb = 0;
            }
            fb |= 1u << (j & 31);
          }
          edge(u, bs, j, re, v, pos, tail, nbv, cost);
        }
        if (Mode == 1 && fb) atomicOr(&eflag[fw], fb);
      }
      // Longer rows: the warp, one row at a time.
      uint32_t longm = __ballot_sync(kFull, mine && !own);
      while (longm) {
        const int r = __ffs(longm) - 1;
        longm &= longm - 1;
        warp_row(rb * 32 + r, __shfl_sync(kFull, rs, r), __shfl_sync(kFull, re, r), __shfl_sync(kFull, bs, r),
                 __shfl_sync(kFull, nbu, r));
      }
    }
  }
  if constexpr (kTop != 0) {
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < kTop && top_lo + t < g.n; t += blockDim.x) {
      const uint32_t c = s_top[2 * t], sv = s_top[2 * t + 1];
      if (c) atomicAdd(&in_cnt[top_lo + t], c);
      if (sv) atomicAdd(&save[top_lo + t], (unsigned long long)sv);
    }
  }
}

// After mode 0: a hub whose candidates save at least its staging cost keeps
// its candidate count (the length of its in-list) and is marked in save[v]
// (1 << 32: the low word then counts its column tails in mode 1); any other
// vertex gets no in-list, and its vinfo is cleared so that mode 1 takes none
// of its edges.
__global__ void k_hub_accept(uint64_t* __restrict__ vinfo, uint32_t n, unsigned long long* __restrict__ save,
                             uint32_t* __restrict__ in_cnt) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint64_t vi = vinfo[v];
  const bool acc = in_cnt[v] > 0 && save[v] >= hub_cost((uint32_t)(vi >> 32), (uint32_t)vi);
  if (!acc) {
    in_cnt[v] = 0;
    vinfo[v] = 0;  // no candidate in mode 1, no pieces
  }
  save[v] = acc ? (1ull << 32) : 0ull;
}

__global__ void k_hub_piece_count(const uint32_t* __restrict__ in_off, const uint64_t* __restrict__ vinfo,
                                  uint32_t n, uint32_t* __restrict__ cnt) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v > n) return;
  uint32_t c = 0, wc = 0;
  if (v < n) {
    const uint32_t k = in_off[v + 1] - in_off[v];
    const uint32_t span = (uint32_t)(vinfo[v] >> 32), nb = (uint32_t)vinfo[v];
    // The warp stages the row when its direct map fits the warp's slice, or,
    // for a row too wide for the CTA's direct map, when its hash does.
    const bool warp = span <= kHubWarpSpan || (span > kHubMaxSpan && nb <= kHubWarpHash);
    if (warp)
      wc = (k + kHubWarpPiece - 1) / kHubWarpPiece;
    else
      c = (k + kHubPiece - 1) / kHubPiece;
  }
  cnt[v] = c;
  cnt[n + 1 + v] = wc;
}

__global__ void k_hub_piece_scatter(const uint32_t* __restrict__ pos, uint32_t n, uint64_t* __restrict__ pieces,
                                    uint32_t* __restrict__ piece_off) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    for (uint32_t k = 0, np = pos[v + 1] - pos[v]; k < np; ++k)
      pieces[pos[v] + k] = ((uint64_t)v << 32) | (k * kHubPiece);
    const uint32_t* wpos = pos + n + 1;
    for (uint32_t k = 0, np = wpos[v + 1] - wpos[v]; k < np; ++k)
      pieces[wpos[v] + k] = ((uint64_t)v << 32) | (k * kHubWarpPiece);
  }
  if (v == n) {
    piece_off[TRIBIT_NUM_VARIANTS + 2] = pos[n];          // CTA pieces
    piece_off[TRIBIT_NUM_VARIANTS + 3] = pos[2 * n + 1];  // all pieces
  }
}

__global__ void k_hub_total(const uint32_t* __restrict__ in_off, uint32_t n, uint32_t* __restrict__ piece_off) {
  piece_off[TRIBIT_NUM_VARIANTS + 4] = in_off[n];
}

// Waves: kHubWaves ranges of rows with equal shares of the bit-row array.
// wave_lo[w] = first row whose bit row starts at or after w / kHubWaves of
// it (wave_lo[kHubWaves] = n). The in-lists are filled one wave of rows at a
// time, so each hub's in-list is ordered by wave, and the hub pieces are then
// ordered by the wave of their first tail: the CTAs working at one time walk
// the tails of rows of one wave, whose bit rows fit the L2.
// wave_bk[w] = the bit-row start of wave w's first row: the wave of row u is
// the last w with wave_bk[w] <= k for any bit-row index k of u's row (a tail
// start), so a piece's wave follows from its first tail without its row.
// wave_cp[w]: the same in CSR positions, for column tails.
__global__ void k_wave_bounds(GraphView g, uint32_t* __restrict__ wave_lo, uint32_t* __restrict__ wave_bk,
                              uint32_t* __restrict__ wave_cp) {
  const uint32_t w = threadIdx.x;
  if (w > kHubWaves) return;
  const uint64_t nb = rp_blk(g.rp[g.n]);
  const uint64_t target = nb * w / kHubWaves;
  uint32_t lo = 0, hi = g.n;  // first u with brow_ptr[u] >= target
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (rp_blk(g.rp[mid]) < target)
      lo = mid + 1;
    else
      hi = mid;
  }
  wave_lo[w] = w == kHubWaves ? g.n : lo;
  wave_bk[w] = w == kHubWaves ? 0xFFFFFFFFu : rp_blk(g.rp[lo]);
  wave_cp[w] = w == kHubWaves ? 0xFFFFFFFFu : rp_row(g.rp[lo]);
}

__device__ __forceinline__ uint32_t wave_of_block(const uint32_t* __restrict__ wave_bk, uint32_t k) {
  uint32_t w = 0;
#pragma unroll
  for (uint32_t st = kHubWaves / 2; st >= 1; st >>= 1)
    if (w + st < kHubWaves && wave_bk[w + st] <= k) w += st;
  return w;
}

// Counting sort of the hub pieces by the wave of their first tail, within
// each list (CTA pieces [0, Pc), warp pieces [Pc, P)). cnt: 2 kHubWaves.
__global__ void k_piece_waves(const uint64_t* __restrict__ pieces, const uint32_t* __restrict__ piece_off,
                              const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_bits,
                              const uint64_t* __restrict__ inl, const uint32_t* __restrict__ wave_bk,
                              const uint32_t* __restrict__ wave_cp, uint32_t* __restrict__ cnt,
                              uint8_t* __restrict__ wave) {
  const uint32_t pc_n = piece_off[TRIBIT_NUM_VARIANTS + 2], all = piece_off[TRIBIT_NUM_VARIANTS + 3];
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < all; p += gridDim.x * blockDim.x) {
    const uint64_t pc = pieces[p];
    const uint32_t v = (uint32_t)(pc >> 32), k = (uint32_t)pc;  // the piece's first entry: k of v's list
    const bool bits = !kHubColRatio || k < in_bits[v];
    const uint32_t w = wave_of_block(bits ? wave_bk : wave_cp, (uint32_t)(inl[in_off[v] + k] >> 32));
    wave[p] = (uint8_t)w;
    atomicAdd(&cnt[(p < pc_n ? 0 : kHubWaves) + w], 1u);
  }
}

__global__ void k_wave_scan(uint32_t* __restrict__ cnt, const uint32_t* __restrict__ piece_off) {
  uint32_t run = 0;
  for (uint32_t i = 0; i < 2 * kHubWaves; ++i) {
    if (i == kHubWaves) run = piece_off[TRIBIT_NUM_VARIANTS + 2];  // warp pieces follow the CTA pieces
    const uint32_t c = cnt[i];
    cnt[i] = run;
    run += c;
  }
}

__global__ void k_piece_wave_scatter(const uint64_t* __restrict__ pieces, const uint32_t* __restrict__ piece_off,
                                     const uint8_t* __restrict__ wave, uint32_t* __restrict__ pos,
                                     uint64_t* __restrict__ out) {
  const uint32_t pc_n = piece_off[TRIBIT_NUM_VARIANTS + 2], all = piece_off[TRIBIT_NUM_VARIANTS + 3];
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < all; p += gridDim.x * blockDim.x)
    out[atomicAdd(&pos[(p < pc_n ? 0 : kHubWaves) + wave[p]], 1u)] = pieces[p];
}

}  // namespace

Schedule take_schedule(Arena& ar, uint64_t n, uint64_t E, bool hubs) {
  Schedule s;
  const uint32_t nrb = (uint32_t)ceil_div<uint64_t>(n, 32);
  s.num_row_blocks = nrb;
  s.variant_of = ar.take<uint8_t>(nrb + 1);
  s.piece_cap = 2 * n + E / kMinPieceWidth + 64;  // row pieces, plus up to 16 per bit-tile block
  s.pieces = ar.take<uint64_t>(s.piece_cap);
  s.piece_off = ar.take<uint32_t>(TRIBIT_NUM_VARIANTS + 5);
  s.heavy = ar.take<uint32_t>(n + 1);
  s.row_flags = ar.take<uint32_t>(n + 1);
  s.row_scan_tmp = take_scan_temp<uint32_t>(ar, n + 1);
  s.list_len = ar.take<uint32_t>(TRIBIT_NUM_VARIANTS);
  s.block_pieces = ar.take<uint32_t>(nrb + 1);
  s.flags = ar.take<uint32_t>(nrb + 1);
  s.scan_tmp = take_scan_temp<uint32_t>(ar, nrb + 1);
  s.overflow_cap = (uint32_t)(n + 1);
  s.overflow = ar.take<uint32_t>(2 * (n + 1));
  s.features = ar.take<float>((uint64_t)nrb * kNumFeatures + 1);
  if (hubs) {
    s.eflag_words = E / 32 + 2;
    s.eflag = ar.take<uint32_t>(s.eflag_words);
    s.vinfo = ar.take<uint64_t>(n + 1);
    s.save = ar.take<unsigned long long>(n + 1);
    s.in_cnt = ar.take<uint32_t>(n + 1);
    s.in_off = ar.take<uint32_t>(n + 1);
    s.inl_cap = E + 1;
    s.inl = ar.take<uint64_t>(s.inl_cap);
    s.hub_pieces = ar.take<uint64_t>(2 * n + E / kHubWarpPiece + 64);
    s.hub_pieces2 = ar.take<uint64_t>(2 * n + E / kHubWarpPiece + 64);
    s.piece_wave = ar.take<uint8_t>(2 * n + E / kHubWarpPiece + 64);
    s.wave_lo = ar.take<uint32_t>(kHubWaves + 1);
    s.wave_bk = ar.take<uint32_t>(kHubWaves + 1);
    s.wave_cp = ar.take<uint32_t>(kHubWaves + 1);
    s.wave_cnt = ar.take<uint32_t>(2 * kHubWaves);
    s.hub_pos = ar.take<uint32_t>(2 * (n + 1));
    s.hub_scan_tmp = take_scan_temp<uint32_t>(ar, 2 * (n + 1));
  }
  return s;
}

// Hub in-lists and pieces of the merge row blocks (after the heavy-row list:
// its scan space is reused for the in-list offsets). Without hub arrays, or
// with hubs off, the hub pass gets no pieces and no edge is flagged.
static void build_hubs(const GraphView& g, Schedule& s, cudaStream_t st) {
  s.hubs_active = false;
  TB_CUDA(cudaMemsetAsync(s.piece_off + TRIBIT_NUM_VARIANTS + 2, 0, 3 * sizeof(uint32_t), st));
  if (!s.eflag || !s.hubs || g.n == 0) return;
  const uint64_t n = g.n;
  const unsigned vblocks = (unsigned)ceil_div<uint64_t>(n + 1, 256);
  const unsigned eblocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div<uint64_t>(n, 8), 148ull * 16));
  k_hub_vinfo<<<vblocks, 256, 0, st>>>(g, s.vinfo);
  TB_LAUNCH_CHECK();
  TB_CUDA(cudaMemsetAsync(s.save, 0, n * sizeof(unsigned long long), st));
  TB_CUDA(cudaMemsetAsync(s.eflag, 0, (s.eflag_words) * sizeof(uint32_t), st));
  TB_CUDA(cudaMemsetAsync(s.in_cnt, 0, (n + 1) * sizeof(uint32_t), st));
  // Candidates counted and savings summed in one pass; each hub accepted or
  // not as a whole; its in-list sized by its candidates, then filled.
  k_hub_edges<0><<<eblocks, 256, 0, st>>>(g, s.variant_of, s.vinfo, s.save, s.eflag, s.in_cnt, s.in_off, s.inl,
                                           nullptr, nullptr);
  TB_LAUNCH_CHECK();
  k_hub_accept<<<vblocks, 256, 0, st>>>(s.vinfo, (uint32_t)n, s.save, s.in_cnt);
  TB_LAUNCH_CHECK();
  device_scan<uint32_t, OpSum>(s.in_cnt, s.in_off, n + 1, true, OpSum{}, 0u, s.row_scan_tmp, st);
  TB_CUDA(cudaMemsetAsync(s.in_cnt, 0, (n + 1) * sizeof(uint32_t), st));
  k_wave_bounds<<<1, kHubWaves + 1, 0, st>>>(g, s.wave_lo, s.wave_bk, s.wave_cp);
  TB_LAUNCH_CHECK();
  if (s.inl_cap <= kHubOneWaveEntries) {
    // A graph whose bit rows fit the L2 many times over gains nothing from
    // the wave order: one launch fills every in-list.
    k_hub_edges<1><<<eblocks, 256, 0, st>>>(g, s.variant_of, s.vinfo, s.save, s.eflag, s.in_cnt, s.in_off, s.inl,
                                             s.hub_rows ? s.inrow : nullptr, nullptr);
    TB_LAUNCH_CHECK();
  } else {
    for (uint32_t w = 0; w < kHubWaves; ++w) {  // in-lists filled wave by wave: ordered by wave
      k_hub_edges<1><<<eblocks, 256, 0, st>>>(g, s.variant_of, s.vinfo, s.save, s.eflag, s.in_cnt, s.in_off, s.inl,
                                               s.hub_rows ? s.inrow : nullptr, s.wave_lo + w);
      TB_LAUNCH_CHECK();
    }
  }
  k_hub_piece_count<<<vblocks, 256, 0, st>>>(s.in_off, s.vinfo, (uint32_t)n, s.hub_pos);
  TB_LAUNCH_CHECK();
  device_scan<uint32_t, OpSum>(s.hub_pos, s.hub_pos, 2 * (n + 1), true, OpSum{}, 0u, s.hub_scan_tmp, st);
  k_hub_piece_scatter<<<vblocks, 256, 0, st>>>(s.hub_pos, (uint32_t)n, s.hub_pieces2, s.piece_off);
  TB_LAUNCH_CHECK();
  k_hub_total<<<1, 1, 0, st>>>(s.in_off, (uint32_t)n, s.piece_off);
  TB_LAUNCH_CHECK();
  TB_CUDA(cudaMemsetAsync(s.wave_cnt, 0, 2 * kHubWaves * sizeof(uint32_t), st));
  k_piece_waves<<<148 * 8, 256, 0, st>>>(s.hub_pieces2, s.piece_off, s.in_off, s.in_cnt, s.inl, s.wave_bk,
                                          s.wave_cp, s.wave_cnt, s.piece_wave);
  TB_LAUNCH_CHECK();
  k_wave_scan<<<1, 1, 0, st>>>(s.wave_cnt, s.piece_off);
  TB_LAUNCH_CHECK();
  k_piece_wave_scatter<<<148 * 8, 256, 0, st>>>(s.hub_pieces2, s.piece_off, s.piece_wave, s.wave_cnt, s.hub_pieces);
  TB_LAUNCH_CHECK();
  s.hubs_active = true;
}

void build_pieces(const GraphView& g, Schedule& s, cudaStream_t st) {
  const uint32_t nrb = s.num_row_blocks;
  const unsigned wblocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div<uint64_t>(nrb, 8), 148ull * 16));
  const unsigned fblocks = (unsigned)ceil_div<uint64_t>(nrb + 1, 256);
  TB_CUDA(cudaMemsetAsync(s.list_len, 0, TRIBIT_NUM_VARIANTS * sizeof(uint32_t), st));
  if (nrb) {
    k_block_pieces<<<wblocks, 256, 0, st>>>(g, nrb, s.variant_of, s.block_pieces, s.piece_width);
    TB_LAUNCH_CHECK();
  }
  for (int v = 0; v < TRIBIT_NUM_VARIANTS; ++v) {
    k_piece_flags<<<fblocks, 256, 0, st>>>(s.variant_of, s.block_pieces, nrb, v, s.flags, s.list_len);
    TB_LAUNCH_CHECK();
    device_scan<uint32_t, OpSum>(s.flags, s.flags, nrb + 1, true, OpSum{}, 0u, s.scan_tmp, st);
    k_piece_segment<<<1, 1, 0, st>>>(s.flags, nrb, v, s.piece_off);
    TB_LAUNCH_CHECK();
    if (nrb) {
      k_piece_scatter<<<wblocks, 256, 0, st>>>(g, nrb, s.variant_of, v, s.flags, s.piece_off, s.pieces,
                                               s.piece_width);
      TB_LAUNCH_CHECK();
    }
  }
  const unsigned rblocks = (unsigned)ceil_div<uint64_t>((uint64_t)g.n + 1, 256);
  k_heavy_flags<<<rblocks, 256, 0, st>>>(g, s.row_flags);
  TB_LAUNCH_CHECK();
  device_scan<uint32_t, OpSum>(s.row_flags, s.row_flags, (uint64_t)g.n + 1, true, OpSum{}, 0u, s.row_scan_tmp, st);
  k_heavy_scatter<<<rblocks, 256, 0, st>>>(g, s.row_flags, s.heavy, s.piece_off);
  TB_LAUNCH_CHECK();
  build_hubs(g, s, st);
}

void compute_features(const GraphView& g, Schedule& s, int mode, bool full_features, cudaStream_t st) {
  const uint32_t nrb = s.num_row_blocks;
  if (nrb == 0) return;
  const unsigned blocks = (unsigned)std::min<uint64_t>(ceil_div<uint64_t>(nrb, 8), 148ull * 16);
  k_features<<<blocks, 256, 0, st>>>(g, nrb, mode, s.features, s.variant_of, full_features ? 1 : 0,
                                     s.tile_min_nnz, s.merge_ratio);
  TB_LAUNCH_CHECK();
}

namespace {
__global__ void k_merge_to_bitmap(uint8_t* __restrict__ variant_of, uint32_t nrb) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nrb; i += gridDim.x * blockDim.x)
    if (variant_of[i] == TRIBIT_VARIANT_MERGE) variant_of[i] = TRIBIT_VARIANT_BITMAP;
}
}  // namespace

void merge_blocks_to_bitmap(Schedule& s, cudaStream_t st) {
  if (s.num_row_blocks == 0) return;
  k_merge_to_bitmap<<<(unsigned)ceil_div<uint64_t>(s.num_row_blocks, 256), 256, 0, st>>>(s.variant_of,
                                                                                         s.num_row_blocks);
  TB_LAUNCH_CHECK();
}

void build_schedule(const GraphView& g, Schedule& s, int mode, bool full_features, cudaStream_t st) {
  compute_features(g, s, mode, full_features, st);
  build_pieces(g, s, st);
}

LaunchInfo launch_count(const GraphView& graph, const Schedule& s, DeviceStats* stats, unsigned long long* per_graph,
                        const CountConfig& cfg, cudaStream_t st) {
  GraphView g = graph;
  g.eflag = s.hubs_active ? s.eflag : nullptr;
  once_per_device<0>([] {
    TB_CUDA(cudaFuncSetAttribute(k_rows_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(uint64_t) << kCtaLogSlots)));
    TB_CUDA(cudaFuncSetAttribute(k_tiles_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kTileWarps * sizeof(TileSmem))));
    TB_CUDA(cudaFuncSetAttribute(k_tiles_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
  });
  const int sms = cfg.num_sms > 0 ? cfg.num_sms : 148;
  const int per_sm = cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm : 6;
  const unsigned warp_grid = (unsigned)(sms * per_sm);
  LaunchInfo info;
  static_assert(offsetof(DeviceStats, cursor) == offsetof(DeviceStats, count_err) + sizeof(unsigned int) &&
                    offsetof(DeviceStats, overflow) == offsetof(DeviceStats, cursor) + sizeof(DeviceStats::cursor),
                "count_err, cursor and overflow are cleared by one memset");
  TB_CUDA(cudaMemsetAsync(&stats->count_err, 0,
                          sizeof(stats->count_err) + sizeof(stats->cursor) + sizeof(stats->overflow), st));
  TB_CUDA(cudaMemsetAsync(&stats->triangles, 0, sizeof(stats->triangles), st));
  uint32_t* ovf_cta = s.overflow;
  uint32_t* ovf_global = s.overflow + s.overflow_cap;
  if (cfg.queue && !cfg.block_ns && !cfg.variant_start) {
    // One persistent kernel for the row pieces and the hub pass; the tiles and
    // the fallback rows (whose list k_queue fills) after it.
    k_queue<<<(unsigned)(sms * kHubCtasPerSm), kHubWarps * 32, 0, st>>>(
        g, s.pieces, s.piece_off, stats, ovf_cta, per_graph, s.heavy, s.piece_width, s.hub_pieces, s.in_off,
        s.in_cnt, s.inl);
    TB_LAUNCH_CHECK();
    if (s.tile_engine == TRIBIT_TILES_TCGEN05)
      k_tiles_tc<<<(unsigned)(sms * kTcCtasPerSm), kTcThreads, sizeof(TcSmem), st>>>(
          g, s.pieces, s.piece_off, stats, per_graph, nullptr, cfg.tile_wait_polls, cfg.tile_test_no_commit);
    else
      k_tiles_mma<<<(unsigned)(sms * 5), kTileWarps * 32, kTileWarps * sizeof(TileSmem), st>>>(
          g, s.pieces, s.piece_off, stats, per_graph, nullptr);
    TB_LAUNCH_CHECK();
    k_rows_cta<<<(unsigned)sms, kCtaThreads, sizeof(uint64_t) << kCtaLogSlots, st>>>(g, ovf_cta, stats, ovf_global,
                                                                                     per_graph, nullptr);
    TB_LAUNCH_CHECK();
    k_rows_global<<<(unsigned)sms, kCtaThreads, 0, st>>>(g, ovf_global, stats, per_graph);
    TB_LAUNCH_CHECK();
    info.ctas = (uint64_t)(kHubCtasPerSm + (s.tile_engine == TRIBIT_TILES_TCGEN05 ? kTcCtasPerSm : 5) + 2) * sms;
    info.kernels = 4;
    return info;
  }
  // Timing mode: the events bracket every counting kernel, and every piece,
  // heavy row, tile block and hub piece adds its warp-cycles to its row block.
  if (cfg.variant_start) TB_CUDA(cudaEventRecord(cfg.variant_start, st));
  k_pieces_warp<TRIBIT_VARIANT_BITMAP><<<warp_grid, kWarpsPerCta * 32, 0, st>>>(
      g, s.pieces, s.piece_off, stats, ovf_cta, per_graph, cfg.block_ns, s.heavy, s.piece_width);
  TB_LAUNCH_CHECK();
  if (s.tile_engine == TRIBIT_TILES_TCGEN05)
    k_tiles_tc<<<(unsigned)(sms * kTcCtasPerSm), kTcThreads, sizeof(TcSmem), st>>>(
        g, s.pieces, s.piece_off, stats, per_graph, cfg.block_ns, cfg.tile_wait_polls, cfg.tile_test_no_commit);
  else
    k_tiles_mma<<<(unsigned)(sms * 5), kTileWarps * 32, kTileWarps * sizeof(TileSmem), st>>>(
        g, s.pieces, s.piece_off, stats, per_graph, cfg.block_ns);
  TB_LAUNCH_CHECK();
  k_pieces_warp<TRIBIT_VARIANT_MERGE><<<warp_grid, kWarpsPerCta * 32, 0, st>>>(g, s.pieces, s.piece_off, stats, ovf_cta,
                                                                               per_graph, cfg.block_ns, nullptr,
                                                                               s.piece_width);
  TB_LAUNCH_CHECK();
  k_rows_cta<<<(unsigned)sms, kCtaThreads, sizeof(uint64_t) << kCtaLogSlots, st>>>(g, ovf_cta, stats, ovf_global,
                                                                                   per_graph, cfg.block_ns);
  TB_LAUNCH_CHECK();
  k_rows_global<<<(unsigned)sms, kCtaThreads, 0, st>>>(g, ovf_global, stats, per_graph);
  TB_LAUNCH_CHECK();
  k_hub<<<(unsigned)(sms * kHubCtasPerSm), kHubWarps * 32, 0, st>>>(g, s.hub_pieces, s.piece_off, s.in_off, s.in_cnt,
                                                                     s.inl, s.inrow, stats, per_graph, cfg.block_ns);
  TB_LAUNCH_CHECK();
  if (cfg.variant_stop) TB_CUDA(cudaEventRecord(cfg.variant_stop, st));
  info.ctas = 2ull * warp_grid +
              (2ull + (s.tile_engine == TRIBIT_TILES_TCGEN05 ? (uint64_t)kTcCtasPerSm : 5ull) + kHubCtasPerSm) * sms;
  info.kernels = 6;
  return info;
}

}  // namespace tb
