// stubs.cpp — the few library functions the host parse layer calls outside
// itself, for the sanitizer build of tests/test_sanitizers.py (which builds
// framing.cpp, frameheader.cpp, symbol.cpp, walker*.cpp and decoder.cpp
// without CUDA).  The engine entry points are never reached: the decoder is
// created without an engine (parse only).
#include <string>

#include "av1g.h"

namespace av1g {
thread_local std::string t_err;
void set_last_error_text(const std::string& s) { t_err = s; }
}  // namespace av1g

extern "C" {
const char* av1g_last_error(void) { return av1g::t_err.c_str(); }

// count_units_in_frame (src/loop_restoration.rs:888)
int32_t av1g_lr_units_in_frame(int32_t unit_size, int32_t plane_size) {
    if (unit_size <= 0) return 1;
    int32_t n = (plane_size + (unit_size >> 1)) / unit_size;
    return n > 1 ? n : 1;
}

av1g_status av1g_stream_open(av1g_engine*, const av1g_seq_info*, av1g_stream**) { return AV1G_ENOTSUP; }
av1g_status av1g_stream_close(av1g_stream*) { return AV1G_ENOTSUP; }
av1g_status av1g_stream_reset_refs(av1g_stream*) { return AV1G_ENOTSUP; }
av1g_status av1g_submit_frame(av1g_stream*, const av1g_frame_desc*, uint64_t*) { return AV1G_ENOTSUP; }
av1g_status av1g_poll(av1g_engine*, uint64_t, int64_t, av1g_status*) { return AV1G_ENOTSUP; }
av1g_status av1g_fetch_output(av1g_stream*, uint64_t, av1g_frame_out*) { return AV1G_ENOTSUP; }
av1g_status av1g_release_output(av1g_stream*, uint64_t) { return AV1G_ENOTSUP; }
}
