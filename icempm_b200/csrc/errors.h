// errors.h -- status codes and the per-thread last-error message of the C ABI.
#pragma once
#include <string>

namespace icm {

// Records msg as the calling thread's last error and returns code.
int fail(int code, const std::string &msg);
const char *last_error();

}  // namespace icm
