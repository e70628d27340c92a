// errors.cpp -- per-thread last-error message of the C ABI.
#include "errors.h"
#include "../../include/icempm.h"

namespace icm {

static thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

const char *last_error() { return g_last_error.c_str(); }

}  // namespace icm

extern "C" const char *icm_last_error(void) { return icm::last_error(); }
extern "C" const char *icm_version(void) { return "icempm-b200 0.1 (sm_100a)"; }
