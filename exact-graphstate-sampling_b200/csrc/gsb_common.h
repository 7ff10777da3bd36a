// Error reporting shared by the translation units of libgsb: every ABI entry point returns a status and leaves a
// message for gsb_last_error() (thread-local).
#pragma once
#include <string>

namespace gsb {
int fail(int code, const std::string &msg);
}
