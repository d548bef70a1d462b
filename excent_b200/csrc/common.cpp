// common.cpp -- thread-local last-error string shared by every C entry point.
#include "common.h"

#include <cstring>

namespace excent {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

const char* get_error() { return g_err; }

}  // namespace excent

extern "C" const char* excent_last_error(void) { return excent::get_error(); }
extern "C" int excent_version(void) { return 100; }
