// stubs.cu -- entry points whose kernels are not built yet report
// FG_ERR_UNSUPPORTED (never a CPU fallback).
#include "runtime.h"

using namespace fgrt;
extern "C" {
fg_status fg_server_start(fg_ctx*, size_t, int, int, fg_server**) {
    return set_error(FG_ERR_UNSUPPORTED, "server not built yet");
}
fg_status fg_server_submit(fg_server*, const fg_request*, uint64_t*) {
    return set_error(FG_ERR_UNSUPPORTED, "server not built yet");
}
fg_status fg_server_wait(fg_server*, uint64_t, int64_t) {
    return set_error(FG_ERR_UNSUPPORTED, "server not built yet");
}
fg_status fg_server_stats_get(fg_server*, fg_server_stats*) {
    return set_error(FG_ERR_UNSUPPORTED, "server not built yet");
}
fg_status fg_server_stop(fg_server*) { return FG_OK; }
}
