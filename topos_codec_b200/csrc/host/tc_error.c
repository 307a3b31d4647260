/* tc_error.c - thread-local error detail and status strings.
 * reference: native/src/common/error.c:9-31 (detail format "[status] text"),
 * native/src/version.c:148-171 (status strings). */
#include <stdarg.h>
#include <stdio.h>

#include "tc_internal.h"

static _Thread_local char g_detail[256];

int32_t tc_fail(int32_t status, const char* fmt, ...)
{
    int n = snprintf(g_detail, sizeof(g_detail), "[%d] ", (int)status);
    if (n < 0) {
        g_detail[0] = '\0';
        return status;
    }
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_detail + n, sizeof(g_detail) - (size_t)n, fmt, ap);
    va_end(ap);
    return status;
}

/* Exposed to the CUDA layer through tcg_device.h so device-side failures
 * report through the same thread-local detail. */
void tcg_host_set_error(int32_t status, const char* text)
{
    (void)tc_fail(status, "%s", text);
}

TC_EXPORT const char* tc_last_error(void) { return g_detail; }

TC_EXPORT const char* tc_status_message(int32_t status)
{
    switch (status) {
    case TC_OK: return "OK";
    case TC_WARN_CONCEALED: return "concealment applied to one or more slices";
    case TC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TC_ERR_OUT_OF_MEMORY: return "out of memory";
    case TC_ERR_UNSUPPORTED_VERSION: return "unsupported bitstream/ABI version";
    case TC_ERR_UNSUPPORTED_PROFILE: return "unsupported profile";
    case TC_ERR_UNSUPPORTED_PIXEL_FORMAT: return "unsupported pixel format or bit depth";
    case TC_ERR_UNSUPPORTED_MATRIX: return "unsupported quantization matrix id";
    case TC_ERR_UNSUPPORTED_ALPHA_MODE: return "unsupported alpha mode";
    case TC_ERR_LIMIT_EXCEEDED: return "decoder hard limit exceeded";
    case TC_ERR_MALFORMED: return "malformed bitstream";
    case TC_ERR_TRUNCATED: return "truncated bitstream";
    case TC_ERR_CHECKSUM_MISMATCH: return "checksum mismatch";
    case TC_ERR_STATE: return "invalid call order or context state";
    case TC_ERR_CANCELLED: return "operation cancelled";
    case TC_ERR_IO: return "I/O callback failure";
    case TC_ERR_BUFFER_TOO_SMALL: return "caller buffer too small";
    case TC_ERR_NOT_IMPLEMENTED: return "capability reserved but not implemented";
    default: return "unknown status";
    }
}
