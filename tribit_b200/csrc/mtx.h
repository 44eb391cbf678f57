// Matrix Market header parse shared by the host reader (mtx.cpp) and the GPU
// ingest (mtx_gpu.cu).
#pragma once
#include <stdint.h>

#include "tribit.h"

namespace tb {

// The banner line, then lines starting with '%', then "rows cols nnz" of the
// file mapped at [p, end), with the reference's semantics (read_mtx,
// tribit.cu:230-245): rows must equal cols. On success *body is the first byte
// after the size line, *num_nodes = rows and *nnz the declared entry count
// (the entry grammar does not depend on it).
tribit_status mtx_header(const char* p, const char* end, const char** body, uint64_t* num_nodes, uint64_t* nnz);

}  // namespace tb
