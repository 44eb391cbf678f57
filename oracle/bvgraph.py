"""WebGraph BVGraph format -- TEST INFRASTRUCTURE ONLY.

The reference's multi-GPU loader reads LAW web graphs through the Rust
`webgraph` crate (0.6.1 in src/multi_gpu/Cargo.lock, with `dsi-bitstream`
0.7.0), `BvGraphSeq::with_basename(..).load()` (src/multi_gpu/src/main.rs:88),
and folds every arc (src, dst), src != dst, to the word (min << 32) | max
(main.rs:142-161). Neither the crate nor any BVGraph file is in this image, so
this module restates the published format (P. Boldi and S. Vigna, "The
WebGraph Framework I: Compression Techniques", WWW 2004, as implemented by
WebGraph's BVGraph) in plain Python: an encoder that writes
basename.graph / .offsets / .properties, and a decoder. The tests use them to
make BVGraph files and to check the product's C++ reader
(tribit_read_bvgraph) against them; parity with files written by WebGraph
itself is not pinned.

Format (big-endian bit streams, most significant bit of each byte first):
  unary(x)  x zeros, then a one
  gamma(x)  n = x + 1: unary(floor(log2 n)), then the low floor(log2 n) bits of n
  delta(x)  n = x + 1: gamma(floor(log2 n)), then the low floor(log2 n) bits of n
  zeta_k(x) n = x + 1, h = floor(log2(n) / k): unary(h), then n - 2^(hk) in the
            minimal binary code of [0, 2^((h+1)k) - 2^(hk))
Per node x, in order: outdegree d; if d > 0 and the window is not empty,
reference r (0 = none, else the list of node x - r); if r > 0, the copy
blocks of that list (block count, first block length, then lengths - 1;
blocks alternate copy / skip starting with copy; the rest of the list is
copied when the count is even); then, over the d - copied extra successors,
intervals (if minintervallength > 0: count, then the first left end as
nat(left - x) and length - minintervallength, then gaps left - prev - 1 and
length - minintervallength, prev = end of the previous interval) and
residuals (the first as nat(y - x), then gaps y - prev - 1), nat(v) = 2v for
v >= 0 and -2v - 1 for v < 0. .offsets: gamma of the first node's bit offset
and of every next offset difference.
"""
from __future__ import annotations

import os

DEFAULTS = {"windowsize": 7, "maxrefcount": 3, "minintervallength": 4, "zetak": 3}
CODES = {"OUTDEGREES": "GAMMA", "REFERENCES": "UNARY", "BLOCKS": "GAMMA", "INTERVALS": "GAMMA",
         "RESIDUALS": "ZETA", "OFFSETS": "GAMMA"}


def nat(v: int) -> int:
    return 2 * v if v >= 0 else -2 * v - 1


def unnat(x: int) -> int:
    return x >> 1 if x % 2 == 0 else -((x + 1) >> 1)


class BitWriter:
    def __init__(self):
        self.bits = []

    def __len__(self):
        return len(self.bits)

    def int(self, v: int, width: int):
        for b in range(width - 1, -1, -1):
            self.bits.append((v >> b) & 1)

    def unary(self, x: int):
        self.bits.extend([0] * x)
        self.bits.append(1)

    def gamma(self, x: int):
        n = x + 1
        m = n.bit_length() - 1
        self.unary(m)
        self.int(n, m)

    def delta(self, x: int):
        n = x + 1
        m = n.bit_length() - 1
        self.gamma(m)
        self.int(n, m)

    def zeta(self, x: int, k: int):
        n = x + 1
        h = (n.bit_length() - 1) // k
        self.unary(h)
        left, right = 1 << (h * k), 1 << ((h + 1) * k)
        # minimal binary code of n - left in [0, right - left)
        v, s = n - left, right - left
        w = (s - 1).bit_length()  # bits of the long codes
        short = (1 << w) - s      # values coded on w - 1 bits
        if v < short:
            self.int(v, w - 1)
        else:
            self.int(v + short, w)

    def code(self, kind: str, x: int, k: int):
        if kind == "GAMMA":
            self.gamma(x)
        elif kind == "DELTA":
            self.delta(x)
        elif kind == "UNARY":
            self.unary(x)
        elif kind == "ZETA":
            self.zeta(x, k)
        else:
            raise ValueError(kind)

    def tobytes(self) -> bytes:
        bits = self.bits + [0] * (-len(self.bits) % 8)
        out = bytearray(len(bits) // 8)
        for i in range(0, len(bits), 8):
            v = 0
            for b in bits[i:i + 8]:
                v = (v << 1) | b
            out[i // 8] = v
        return bytes(out)


class BitReader:
    def __init__(self, data: bytes, pos: int = 0):
        self.data = data
        self.pos = pos

    def bit(self) -> int:
        b = (self.data[self.pos >> 3] >> (7 - (self.pos & 7))) & 1
        self.pos += 1
        return b

    def int(self, width: int) -> int:
        v = 0
        for _ in range(width):
            v = (v << 1) | self.bit()
        return v

    def unary(self) -> int:
        x = 0
        while self.bit() == 0:
            x += 1
        return x

    def gamma(self) -> int:
        m = self.unary()
        return ((1 << m) | self.int(m)) - 1

    def delta(self) -> int:
        m = self.gamma()
        return ((1 << m) | self.int(m)) - 1

    def zeta(self, k: int) -> int:
        h = self.unary()
        left = 1 << (h * k)
        m = self.int(h * k + k - 1)
        if m < left:
            return m + left - 1
        return (m << 1) + self.bit() - 1

    def code(self, kind: str, k: int) -> int:
        return {"GAMMA": self.gamma, "DELTA": self.delta, "UNARY": self.unary}[kind]() if kind != "ZETA" \
            else self.zeta(k)


def _blocks(ref: list[int], mine: set[int]) -> tuple[list[int], list[int]]:
    """Copy blocks of `ref` against the successor set: (block lengths, copied)."""
    blocks, copied = [], []
    copying, run = True, 0
    for y in ref:
        if (y in mine) == copying:
            run += 1
        else:
            blocks.append(run)
            copying, run = not copying, 1
        if y in mine:
            copied.append(y)
    # the run in progress is the implicit last block: kept implicit only when
    # it is a copy run (even count); a trailing skip run is written out
    if not copying:
        blocks.append(run)
    return blocks, copied


def _intervals(extra: list[int], minlen: int):
    """Maximal runs of consecutive ids of length >= minlen, and the rest."""
    ivs, rest = [], []
    i = 0
    while i < len(extra):
        j = i
        while j + 1 < len(extra) and extra[j + 1] == extra[j] + 1:
            j += 1
        if minlen > 0 and j - i + 1 >= minlen:
            ivs.append((extra[i], j - i + 1))
        else:
            rest.extend(extra[i:j + 1])
        i = j + 1
    return ivs, rest


def encode(succ: list[list[int]], window: int = 7, maxref: int = 3, minint: int = 4, zetak: int = 3,
           codes: dict | None = None):
    """Compresses sorted successor lists -> (graph bytes, offsets bytes, properties dict)."""
    cd = dict(CODES, **(codes or {}))
    w = BitWriter()
    offsets = []
    chain = [0] * len(succ)
    for x, lst in enumerate(succ):
        offsets.append(len(w))
        d = len(lst)
        w.code(cd["OUTDEGREES"], d, zetak)
        if d == 0:
            continue
        mine = set(lst)
        best = (None, 0, [], [])  # (bits, r, blocks, copied)
        if window > 0:
            for r in range(0, min(window, x) + 1):
                if r and chain[x - r] >= maxref:
                    continue
                t = BitWriter()
                blocks, copied = ([], []) if r == 0 else _blocks(succ[x - r], mine)
                _write_body(t, x, lst, r, blocks, copied, minint, zetak, cd, window)
                if best[0] is None or len(t) < best[0]:
                    best = (len(t), r, blocks, copied)
        r, blocks, copied = best[1], best[2], best[3]
        chain[x] = chain[x - r] + 1 if r else 0
        _write_body(w, x, lst, r, blocks, copied, minint, zetak, cd, window)
    offsets.append(len(w))
    ow = BitWriter()
    prev = 0
    for o in offsets:
        ow.code(cd["OFFSETS"], o - prev, zetak)
        prev = o
    flags = "|".join(f"{k}_{v}" for k, v in cd.items() if CODES[k] != v)
    props = {"nodes": len(succ), "arcs": sum(map(len, succ)), "windowsize": window, "maxrefcount": maxref,
             "minintervallength": minint, "zetak": zetak, "compressionflags": flags, "version": 0,
             "graphclass": "it.unimi.dsi.webgraph.BVGraph"}
    return w.tobytes(), ow.tobytes(), props


def _write_body(w, x, lst, r, blocks, copied, minint, zetak, cd, window):
    if window > 0:
        w.code(cd["REFERENCES"], r, zetak)
    if r > 0:
        w.code(cd["BLOCKS"], len(blocks), zetak)
        for i, b in enumerate(blocks):
            w.code(cd["BLOCKS"], b if i == 0 else b - 1, zetak)
    cs = set(copied)
    extra = [y for y in lst if y not in cs]
    if not extra:
        return
    if minint > 0:
        ivs, rest = _intervals(extra, minint)
        w.code(cd["INTERVALS"], len(ivs), zetak)
        prev = None
        for left, ln in ivs:
            if prev is None:
                w.code(cd["INTERVALS"], nat(left - x), zetak)
            else:
                w.code(cd["INTERVALS"], left - prev - 1, zetak)
            w.code(cd["INTERVALS"], ln - minint, zetak)
            prev = left + ln
    else:
        rest = extra
    prev = None
    for y in rest:
        w.code(cd["RESIDUALS"], nat(y - x) if prev is None else y - prev - 1, zetak)
        prev = y


def decode(graph: bytes, props: dict) -> list[list[int]]:
    """Sequential decoder of the whole graph -> successor lists."""
    n = int(props["nodes"])
    window = int(props.get("windowsize", DEFAULTS["windowsize"]))
    minint = int(props.get("minintervallength", DEFAULTS["minintervallength"]))
    k = int(props.get("zetak", DEFAULTS["zetak"]))
    cd = dict(CODES)
    for f in filter(None, str(props.get("compressionflags", "")).split("|")):
        key, val = f.strip().split("_")
        cd[key] = val
    rd = BitReader(graph)
    out: list[list[int]] = []
    for x in range(n):
        d = rd.code(cd["OUTDEGREES"], k)
        if d == 0:
            out.append([])
            continue
        r = rd.code(cd["REFERENCES"], k) if window > 0 else 0
        copied = []
        if r > 0:
            ref = out[x - r]
            nb = rd.code(cd["BLOCKS"], k)
            blocks = [rd.code(cd["BLOCKS"], k) + (0 if i == 0 else 1) for i in range(nb)]
            i, copying = 0, True
            for b in blocks:
                if copying:
                    copied.extend(ref[i:i + b])
                i += b
                copying = not copying
            if copying:
                copied.extend(ref[i:])
        extra = d - len(copied)
        got = []
        if extra > 0 and minint > 0:
            ic = rd.code(cd["INTERVALS"], k)
            prev = None
            for _ in range(ic):
                left = x + unnat(rd.code(cd["INTERVALS"], k)) if prev is None else prev + rd.code(cd["INTERVALS"], k) + 1
                ln = rd.code(cd["INTERVALS"], k) + minint
                got.extend(range(left, left + ln))
                prev = left + ln
                extra -= ln
        prev = None
        for _ in range(extra):
            y = x + unnat(rd.code(cd["RESIDUALS"], k)) if prev is None else prev + rd.code(cd["RESIDUALS"], k) + 1
            got.append(y)
            prev = y
        out.append(sorted(copied + got))
    return out


def write(basename: str, succ: list[list[int]], offsets: bool = True, **kw):
    """Writes basename.graph, basename.properties (and basename.offsets)."""
    g, o, props = encode(succ, **kw)
    with open(basename + ".graph", "wb") as f:
        f.write(g)
    if offsets:
        with open(basename + ".offsets", "wb") as f:
            f.write(o)
    with open(basename + ".properties", "w") as f:
        f.write("#BVGraph properties\n")
        for key, v in props.items():
            f.write(f"{key}={v}\n")
    return props


def read_properties(basename: str) -> dict:
    out = {}
    with open(basename + ".properties") as f:
        for line in f:
            if "=" in line and not line.lstrip().startswith("#"):
                key, v = line.split("=", 1)
                out[key.strip()] = v.strip()
    return out


def entries(succ: list[list[int]]):
    """The reference loader's words (main.rs:142-161): every arc x -> y, x != y,
    as (min << 32) | max, in node order."""
    import numpy as np
    out = [(min(x, y) << 32) | max(x, y) for x, lst in enumerate(succ) for y in lst if y != x]
    return np.array(out, dtype=np.uint64)


def _check_tables():
    """Known code words from the format's definition (used by the tests)."""
    return {
        "gamma": {0: "1", 1: "010", 2: "011", 3: "00100", 6: "00111", 7: "0001000"},
        "delta": {0: "1", 1: "0100", 2: "0101", 3: "01100", 7: "00100000"},
        "zeta3": {0: "100", 1: "1010", 2: "1011", 3: "1100", 6: "1111", 7: "0100000", 63: "00100000000"},
        "unary": {0: "1", 3: "0001"},
    }


if __name__ == "__main__":  # pragma: no cover - quick self-check
    import random
    rnd = random.Random(1)
    g = [sorted(rnd.sample(range(200), rnd.randint(0, 20))) for _ in range(200)]
    b, o, p = encode(g)
    assert decode(b, p) == g
    print("ok", len(b), os.path.basename(__file__))
