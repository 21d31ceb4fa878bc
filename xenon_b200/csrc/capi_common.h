// capi_common.h — status plumbing shared by the C ABI translation units.
#pragma once

#include <string>

namespace xb {
// Message of the last failure on this thread (returned by xb_last_error(NULL, ...)).
extern thread_local std::string g_last_error;
// Records a printf-style message as the last error and returns `code`.
int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
}  // namespace xb
