// lucid_guide_capi.cpp — extern "C" access to the path-guiding network on
// its own (forward, encoding, loss gradient, Adam step), for checking it
// against a CPU restatement and for callers that train it themselves.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>

#include "../../include/lucid_cuda.h"
#include "lucid_guide_host.h"

struct LucidGuide {
    int device = 0;
    cudaStream_t stream = nullptr;
    lucid::GuideNet net;
    std::string err;
};

namespace {
int cuda_fail(LucidGuide* g, cudaError_t e, const char* what) {
    g->err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? LUCID_ERR_OOM : LUCID_ERR_CUDA;
}
// Device scratch for one call, freed on scope exit.
struct Dev {
    void* p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
};
}  // namespace

extern "C" {

int lucid_guide_create(int device, int seed, LucidGuide** out) {
    if (!out) return LUCID_ERR_INVALID;
    *out = nullptr;
    LucidGuide* g = new (std::nothrow) LucidGuide;
    if (!g) return LUCID_ERR_OOM;
    g->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete g; return LUCID_ERR_CUDA; }
    if (g->net.init(seed, g->stream) != 0 || cudaStreamSynchronize(g->stream) != cudaSuccess) {
        cudaStreamDestroy(g->stream);
        delete g;
        return LUCID_ERR_CUDA;
    }
    *out = g;
    return LUCID_OK;
}

void lucid_guide_destroy(LucidGuide* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

const char* lucid_guide_last_error(LucidGuide* g) { return g ? g->err.c_str() : "invalid guide"; }

int lucid_guide_num_params(void) { return lucid::kGuideParams; }

int lucid_guide_get_params(LucidGuide* g, float* out, size_t cap) {
    if (!g || !out || cap < (size_t)lucid::kGuideParams) return LUCID_ERR_INVALID;
    cudaSetDevice(g->device);
    if (g->net.get_params(out, g->stream) != 0) { g->err = g->net.error(); return LUCID_ERR_CUDA; }
    return lucid::kGuideParams;
}

int lucid_guide_set_params(LucidGuide* g, const float* in, size_t n) {
    if (!g || !in || n != (size_t)lucid::kGuideParams) return LUCID_ERR_INVALID;
    cudaSetDevice(g->device);
    if (g->net.set_params(in, g->stream) != 0) { g->err = g->net.error(); return LUCID_ERR_CUDA; }
    cudaError_t e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? LUCID_OK : cuda_fail(g, e, "set_params");
}

int lucid_guide_forward(LucidGuide* g, const float* inputs, int n, float* outputs) {
    if (!g || !inputs || !outputs || n <= 0) return LUCID_ERR_INVALID;
    cudaSetDevice(g->device);
    Dev din, dout;
    cudaError_t e = cudaMalloc(&din.p, (size_t)n * lucid::kGuideInputs * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&dout.p, (size_t)n * lucid::kGuideOutputs * sizeof(float));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(din.p, inputs, (size_t)n * lucid::kGuideInputs * sizeof(float), cudaMemcpyHostToDevice,
                            g->stream);
    if (e != cudaSuccess) return cuda_fail(g, e, "forward buffers");
    if (g->net.forward_rows((const float*)din.p, n, (float*)dout.p, g->stream) != 0) {
        g->err = g->net.error();
        return LUCID_ERR_CUDA;
    }
    e = cudaMemcpyAsync(outputs, dout.p, (size_t)n * lucid::kGuideOutputs * sizeof(float), cudaMemcpyDeviceToHost,
                        g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? LUCID_OK : cuda_fail(g, e, "forward");
}

int lucid_guide_encode(LucidGuide* g, const float* p01, const float* nrm, const float* wo, int n, float* out) {
    if (!g || !p01 || !nrm || !wo || !out || n <= 0) return LUCID_ERR_INVALID;
    cudaSetDevice(g->device);
    Dev d;
    const size_t in3 = (size_t)n * 3 * sizeof(float), outb = (size_t)n * lucid::kGuideInputs * sizeof(float);
    cudaError_t e = cudaMalloc(&d.p, 3 * in3 + outb);
    char* b = (char*)d.p;
    if (e == cudaSuccess) e = cudaMemcpyAsync(b, p01, in3, cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + in3, nrm, in3, cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + 2 * in3, wo, in3, cudaMemcpyHostToDevice, g->stream);
    if (e != cudaSuccess) return cuda_fail(g, e, "encode buffers");
    if (g->net.encode_rows((const float*)b, (const float*)(b + in3), (const float*)(b + 2 * in3), n,
                           (float*)(b + 3 * in3), g->stream) != 0) {
        g->err = g->net.error();
        return LUCID_ERR_CUDA;
    }
    e = cudaMemcpyAsync(out, b + 3 * in3, outb, cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    return e == cudaSuccess ? LUCID_OK : cuda_fail(g, e, "encode");
}

static int upload_records(LucidGuide* g, const float* records, int n, Dev& d) {
    cudaError_t e = cudaMalloc(&d.p, (size_t)n * sizeof(lucid::GuideRec));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d.p, records, (size_t)n * sizeof(lucid::GuideRec), cudaMemcpyHostToDevice, g->stream);
    return e == cudaSuccess ? LUCID_OK : cuda_fail(g, e, "records");
}

int lucid_guide_gradient(LucidGuide* g, const float* records, int n, float* grad_out) {
    if (!g || !records || !grad_out || n <= 0) return LUCID_ERR_INVALID;
    cudaSetDevice(g->device);
    Dev d;
    int rc = upload_records(g, records, n, d);
    if (rc != LUCID_OK) return rc;
    cudaError_t e = cudaMemsetAsync((void*)g->net.grad(), 0, lucid::kGuideParams * sizeof(float), g->stream);
    if (e != cudaSuccess) return cuda_fail(g, e, "gradient");
    if (g->net.gradient((const lucid::GuideRec*)d.p, n, g->stream) != 0) { g->err = g->net.error(); return LUCID_ERR_CUDA; }
    e = cudaMemcpyAsync(grad_out, g->net.grad(), lucid::kGuideParams * sizeof(float), cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync((void*)g->net.grad(), 0, lucid::kGuideParams * sizeof(float), g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return cuda_fail(g, e, "gradient");
    if (g->net.failed(g->stream) != 0) { g->err = g->net.error(); return LUCID_ERR_TIMEOUT; }
    return LUCID_OK;
}

int lucid_guide_train(LucidGuide* g, const float* records, int n, float lr) {
    if (!g || !records || n <= 0 || !(lr > 0.0f)) return LUCID_ERR_INVALID;
    cudaSetDevice(g->device);
    Dev d;
    int rc = upload_records(g, records, n, d);
    if (rc != LUCID_OK) return rc;
    if (g->net.train_step((const lucid::GuideRec*)d.p, n, g->stream, lr) != 0) { g->err = g->net.error(); return LUCID_ERR_CUDA; }
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return cuda_fail(g, e, "train");
    if (g->net.failed(g->stream) != 0) { g->err = g->net.error(); return LUCID_ERR_TIMEOUT; }
    return LUCID_OK;
}

}  // extern "C"
