// Learned dispatcher (MLP over row-block features).
#include "tribit.h"

extern "C" tribit_status tribit_model_load(tribit_context* ctx, const char* path) {
  if (!ctx || !path) return TRIBIT_ERR_INVALID_ARGUMENT;
  return TRIBIT_ERR_NO_MODEL;
}
