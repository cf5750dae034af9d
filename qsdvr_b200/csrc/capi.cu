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

cudaError_t error_word_camera(unsigned *, int, cudaStream_t);
cudaError_t error_word_surface(unsigned *, int, cudaStream_t);
cudaError_t error_word_render(unsigned *, int, cudaStream_t);
cudaError_t error_word_fused(unsigned *, int, cudaStream_t);
cudaError_t error_word_optim(unsigned *, int, cudaStream_t);
cudaError_t error_word_gradcheck(unsigned *, int, cudaStream_t);
cudaError_t error_word_proposal(unsigned *, int, cudaStream_t);

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
