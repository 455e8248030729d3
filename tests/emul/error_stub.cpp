// mel_set_error for host sources of the library compiled alone into a test library (test
// infrastructure): the message is kept for emul_error().
#include <cstdarg>
#include <cstdio>

static char g_err[512];
void mel_set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

extern "C" const char* emul_error() { return g_err; }
