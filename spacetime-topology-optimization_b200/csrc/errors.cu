// Thread-local last-error message behind stt_last_error().
#include "errors.h"

namespace stt {

char* error_buffer() {
  static thread_local char buf[512] = "";
  return buf;
}

}  // namespace stt

extern "C" const char* stt_last_error(void) { return stt::error_buffer(); }
