// Status, error-message and device-error-word plumbing of the C ABI.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "common.cuh"

namespace qsdvr {

static thread_local std::string t_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

int check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return QSDVR_OK;
    return set_error(QSDVR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_launch(const char *what) { return check_cuda(cudaGetLastError(), what); }

#define QSDVR_UNIT(name)                                         \
    cudaError_t error_word_##name(unsigned *, int, cudaStream_t); \
    cudaError_t bounds_record_##name(uint64_t *, int, cudaStream_t);
QSDVR_UNIT(camera)
QSDVR_UNIT(surface)
QSDVR_UNIT(render)
QSDVR_UNIT(fused)
QSDVR_UNIT(optim)
QSDVR_UNIT(gradcheck)
QSDVR_UNIT(proposal)
#undef QSDVR_UNIT

}  // namespace qsdvr

extern "C" const char *qsdvr_last_error(void) { return qsdvr::t_last_error.c_str(); }

extern "C" int qsdvr_version(void) { return 100; }

extern "C" int qsdvr_device_error(uint32_t *word, int clear, cudaStream_t stream) {
    using namespace qsdvr;
    if (!word) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_device_error: null output");
    unsigned w = 0;
    cudaError_t e = error_word_camera(&w, clear, stream);
    if (e == cudaSuccess) e = error_word_surface(&w, clear, stream);
    if (e == cudaSuccess) e = error_word_render(&w, clear, stream);
    if (e == cudaSuccess) e = error_word_fused(&w, clear, stream);
    if (e == cudaSuccess) e = error_word_optim(&w, clear, stream);
    if (e == cudaSuccess) e = error_word_gradcheck(&w, clear, stream);
    if (e == cudaSuccess) e = error_word_proposal(&w, clear, stream);
    *word = w;
    return check_cuda(e, "qsdvr_device_error");
}

extern "C" int qsdvr_bounds_checked(void) { return QSDVR_BOUNDS_CHECKED; }

extern "C" int qsdvr_bounds_record(uint64_t *record, int clear, cudaStream_t stream) {
    using namespace qsdvr;
    if (!record) return set_error(QSDVR_ERR_INVALID_ARGUMENT, "qsdvr_bounds_record: null output");
    // in the order of the source-file numbers the header lists
    cudaError_t (*const units[])(uint64_t *, int, cudaStream_t) = {
        bounds_record_camera, bounds_record_surface, bounds_record_render, bounds_record_fused,
        bounds_record_optim,  bounds_record_gradcheck, bounds_record_proposal};
    record[0] = record[1] = record[2] = record[3] = 0;
    cudaError_t e = cudaSuccess;
    for (int u = 0; u < 7 && e == cudaSuccess; ++u) {
        uint64_t rec[3] = {0, 0, 0};
        e = units[u](rec, clear, stream);
        if (e == cudaSuccess && rec[0] && !record[0]) {
            record[0] = (uint64_t)(u + 1);
            record[1] = rec[0];
            record[2] = rec[1];
            record[3] = rec[2];
        }
    }
    return check_cuda(e, "qsdvr_bounds_record");
}
