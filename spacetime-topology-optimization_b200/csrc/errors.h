// Error bookkeeping shared by the entry points: a thread-local message and helpers
// that turn CUDA failures into STT_ERR_CUDA.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/sttb200.h"

namespace stt {

char* error_buffer();

inline int set_error(int code, const char* msg) {
  std::snprintf(error_buffer(), 512, "%s", msg);
  return code;
}

inline int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return STT_OK;
  std::snprintf(error_buffer(), 512, "%s: %s", what, cudaGetErrorString(e));
  return STT_ERR_CUDA;
}

inline int check_launch(const char* what) { return check_cuda(cudaGetLastError(), what); }

}  // namespace stt

#define STT_TRY(...)               \
  do {                             \
    int _stt_rc = (__VA_ARGS__);   \
    if (_stt_rc != STT_OK) return _stt_rc; \
  } while (0)
