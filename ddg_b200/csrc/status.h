// Thread-local last-error message shared by every C-ABI entry point.
#pragma once
#include <string>

namespace ddg {
void set_error(const std::string& msg);
inline int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}
}  // namespace ddg
