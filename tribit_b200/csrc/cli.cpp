// `tribit` command line: a drop-in for the reference's single-GPU binary
// (src/single_gpu/tribit.cu:271-315 options, :840-866 main, :807-819 summary).
//
// Same invocation (`tribit -i <graph.mtx>`), same stdout lines in the same
// order, so the reference's benchmark harness regexes
// (artifact/sc26/run_benchmarks/run_single_gpu.py:78-83) parse it unchanged.
// Like the reference, a warm-up count precedes the reported one.
// Extensions (all optional): -d <auto|plain|learned|merge|bitmap|mma>
// dispatcher (auto, the default: learned with the weights shipped beside the
// binary, ../models/dispatch_mlp.bin, else plain), -o <degree|id>
// orientation, -m <model file> learned-dispatch weights, -v extra lines after
// the summary block.
#include <cuda_runtime.h>
#include <getopt.h>
#include <thrust/version.h>
#include <cub/version.cuh>

#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "tribit.h"

extern "C" tribit_status tribit_model_load(tribit_context* ctx, const char* path);

namespace {

struct Config {
  std::string input_file;
  std::string model;
  int dispatch = -1;  // auto
  int order = TRIBIT_ORDER_DEGREE;
  bool verbose = false;
  bool webgraph = false;  // -g: input_file is a WebGraph BVGraph basename
};

std::string usage(const char* prog) {
  return std::string("Usage: ") + prog +
         " -i <input_file>\n"
         "Options:\n"
         "  -i <input_file>    Path to the input file (required)\n"
         "  -d <dispatch>      auto (default: learned with the bundled model, else plain),\n"
         "                     plain, learned, merge, bitmap or mma\n"
         "  -o <order>         degree (default) or id\n"
         "  -m <model_file>    dispatcher weights for -d learned\n"
         "  -g <basename>      read a WebGraph BVGraph (basename.properties/.graph/.offsets)\n"
         "                     instead of a Matrix Market file\n"
         "  -v                 print extra statistics after the summary\n";
}

Config options(int argc, char* argv[]) {
  Config cfg;
  if (argc == 1) {
    std::fprintf(stderr, "%s", usage(argv[0]).c_str());
    std::exit(EXIT_FAILURE);
  }
  int opt;
  while ((opt = getopt(argc, argv, "i:d:o:m:vg:")) != -1) {
    switch (opt) {
      case 'i':
        cfg.input_file = optarg;
        break;
      case 'g':
        cfg.input_file = optarg;
        cfg.webgraph = true;
        break;
      case 'd':
        if (!std::strcmp(optarg, "auto")) cfg.dispatch = -1;
        else if (!std::strcmp(optarg, "plain")) cfg.dispatch = TRIBIT_DISPATCH_PLAIN;
        else if (!std::strcmp(optarg, "learned")) cfg.dispatch = TRIBIT_DISPATCH_LEARNED;
        else if (!std::strcmp(optarg, "merge")) cfg.dispatch = TRIBIT_DISPATCH_MERGE;
        else if (!std::strcmp(optarg, "bitmap")) cfg.dispatch = TRIBIT_DISPATCH_BITMAP;
        else if (!std::strcmp(optarg, "mma")) cfg.dispatch = TRIBIT_DISPATCH_MMA;
        else {
          std::fprintf(stderr, "Error: unknown dispatcher '%s'\n", optarg);
          std::fprintf(stderr, "%s", usage(argv[0]).c_str());
          std::exit(EXIT_FAILURE);
        }
        break;
      case 'o':
        if (!std::strcmp(optarg, "degree")) cfg.order = TRIBIT_ORDER_DEGREE;
        else if (!std::strcmp(optarg, "id")) cfg.order = TRIBIT_ORDER_ID;
        else {
          std::fprintf(stderr, "Error: unknown order '%s'\n", optarg);
          std::fprintf(stderr, "%s", usage(argv[0]).c_str());
          std::exit(EXIT_FAILURE);
        }
        break;
      case 'm':
        cfg.model = optarg;
        break;
      case 'v':
        cfg.verbose = true;
        break;
      case '?':
      default:
        std::fprintf(stderr, "Error: unknown option or missing argument\n");
        std::fprintf(stderr, "%s", usage(argv[0]).c_str());
        std::exit(EXIT_FAILURE);
    }
  }
  if (cfg.input_file.empty()) {
    std::fprintf(stderr, "Error: input file is required (-i option)\n");
    std::fprintf(stderr, "%s", usage(argv[0]).c_str());
    std::exit(EXIT_FAILURE);
  }
  if (optind < argc) std::fprintf(stderr, "Warning: extra arguments ignored\n");
  return cfg;
}

[[noreturn]] void fail(const char* what, tribit_status st, tribit_context* ctx) {
  std::fprintf(stderr, "Error: %s: %s", what, tribit_status_string(st));
  if (ctx && *tribit_last_error(ctx)) std::fprintf(stderr, " (%s)", tribit_last_error(ctx));
  std::fprintf(stderr, "\n");
  std::fflush(stdout);
  std::exit(EXIT_FAILURE);
}

// The dispatcher weights shipped with the binary: <dir of the executable>/../models/dispatch_mlp.bin.
std::string bundled_model() {
  char buf[4096];
  const ssize_t k = readlink("/proc/self/exe", buf, sizeof buf - 1);
  if (k <= 0) return {};
  buf[k] = 0;
  std::string dir(buf);
  dir = dir.substr(0, dir.find_last_of('/'));
  const std::string path = dir + "/../models/dispatch_mlp.bin";
  return access(path.c_str(), R_OK) == 0 ? path : std::string();
}

}  // namespace

int main(int argc, char* argv[]) {
  std::printf("Thrust version: %d.%d.%d\n", THRUST_MAJOR_VERSION, THRUST_MINOR_VERSION, THRUST_SUBMINOR_VERSION);
  std::printf("CUB version: %d\n", CUB_VERSION);
  Config cfg = options(argc, argv);

  std::printf("Reading data from %s...\n", cfg.input_file.c_str());
  std::fflush(stdout);
  const std::string probe = cfg.webgraph ? cfg.input_file + ".properties" : cfg.input_file;
  if (FILE* f = std::fopen(probe.c_str(), "rb")) {
    std::fclose(f);
  } else {
    fail(cfg.input_file.c_str(), TRIBIT_ERR_IO, nullptr);  // the reference throws here (tribit.cu:230)
  }
  tribit_status st = TRIBIT_OK;

  if (cfg.dispatch < 0) {
    if (cfg.model.empty()) cfg.model = bundled_model();
    cfg.dispatch = cfg.model.empty() ? TRIBIT_DISPATCH_PLAIN : TRIBIT_DISPATCH_LEARNED;
  }
  tribit_options o;
  tribit_default_options(&o);
  o.dispatch = cfg.dispatch;
  o.order = cfg.order;
  tribit_context* ctx = nullptr;
  st = tribit_create(&o, &ctx);
  if (st != TRIBIT_OK) fail("device setup", st, nullptr);
  if (!cfg.model.empty()) {
    st = tribit_model_load(ctx, cfg.model.c_str());
    if (st != TRIBIT_OK) fail(cfg.model.c_str(), st, ctx);
  }

  // The file goes to device memory and is parsed there (tribit_load_mtx);
  // then a warm-up count and the reported one (tribit.cu:858).
  // A BVGraph is decoded on the host threads and counted from host memory.
  uint64_t n = 0, ne = 0;
  uint64_t* web = nullptr;
  tribit_result res;
  if (cfg.webgraph) {
    st = tribit_read_bvgraph(cfg.input_file.c_str(), &n, &web, &ne);
    if (st != TRIBIT_OK) fail(cfg.input_file.c_str(), st, ctx);
    for (int k = 0; k < 2 && st == TRIBIT_OK; ++k) st = tribit_count_edges(ctx, web, ne, n, &res);
    tribit_free_host(web);
  } else {
    st = tribit_load_mtx(ctx, cfg.input_file.c_str(), &n, &ne);
    if (st != TRIBIT_OK) fail(cfg.input_file.c_str(), st, ctx);
    for (int k = 0; k < 2 && st == TRIBIT_OK; ++k) st = tribit_count_loaded(ctx, &res);
  }
  if (st != TRIBIT_OK) fail("count", st, ctx);

  std::printf(
      "============================================================\n"
      "                 Triangle Counting Summary\n"
      "============================================================\n"
      "Graph              : %s\n"
      "Blocks of threads  : %zu\n"
      "Preprocessing (ms) : %.3f\n"
      "Kernel (ms)        : %.3f\n"
      "Triangles          : %llu\n"
      "============================================================\n",
      cfg.input_file.c_str(), (size_t)res.blocks_of_threads, res.preprocess_ms, res.kernel_ms,
      (unsigned long long)res.triangles);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess)
    std::printf("Cuda error at %s:%d (%s): %s (code %d)\n", __FILE__, __LINE__, __func__, cudaGetErrorString(err),
                (int)err);
  else
    std::printf("No cuda error detected at %s:%d (%s)\n", __FILE__, __LINE__, __func__);
  if (cfg.verbose) {
    std::printf("Vertices           : %llu\n", (unsigned long long)res.num_nodes);
    std::printf("Entries            : %llu\n", (unsigned long long)res.entries);
    std::printf("Edges              : %llu\n", (unsigned long long)res.edges);
    std::printf("Read + parse (ms)  : %.3f (%s)\n", res.load_ms, res.load_gpu_parse ? "GPU parse" : "host parse");
    std::printf("Row blocks         : %llu (mma %llu, bitmap %llu, merge %llu)\n",
                (unsigned long long)res.row_blocks, (unsigned long long)res.row_blocks_by_variant[0],
                (unsigned long long)res.row_blocks_by_variant[1], (unsigned long long)res.row_blocks_by_variant[2]);
    std::printf("Edges/s (kernel)   : %.4g\n", res.kernel_ms > 0 ? res.edges / (res.kernel_ms * 1e-3) : 0.0);
  }
  tribit_destroy(ctx);
  return 0;
}
