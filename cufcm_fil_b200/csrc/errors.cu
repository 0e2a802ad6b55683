// errors.cu -- thread-local error text behind cf_last_error().
#include "common.cuh"

namespace cufil {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

}  // namespace cufil

extern "C" const char *cf_last_error(void) { return cufil::g_last_error.c_str(); }

extern "C" int cf_version(void) { return 1 * 10000 + 0 * 100 + 0; }
