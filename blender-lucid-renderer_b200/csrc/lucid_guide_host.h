// lucid_guide_host.h — host interface of the path-guiding network.
#pragma once

#include <cuda_runtime_api.h>

#include <string>

namespace lucid {

// One training sample: the guided vertex (position in [0,1]^3 of the scene
// box, normal, outgoing direction), the sampled direction, the pdf it was
// sampled with and the radiance estimate that arrived along it.
struct GuideRec {
    float p[3], n[3], wo[3], wi[3];
    float pdf;
    float L[3];
};
static_assert(sizeof(GuideRec) == 64, "GuideRec layout");

constexpr int kGuideParams = 22768;   // kGParams in lucid_guide.cuh
constexpr int kGuideInputs = 176;
constexpr int kGuideOutputs = 48;

// FP32 master weights, Adam moments and the BF16 copy the kernels read.
class GuideNet {
public:
    GuideNet() = default;
    ~GuideNet();
    GuideNet(const GuideNet&) = delete;
    GuideNet& operator=(const GuideNet&) = delete;
    int init(int seed, cudaStream_t st);                 // Xavier-uniform, seeded
    int set_params(const float* host_params, cudaStream_t st);
    int get_params(float* host_params, cudaStream_t st);
    // Loss gradient of n device records, added to the gradient buffer.
    int gradient(const GuideRec* d_recs, int n, cudaStream_t st);
    int adam(cudaStream_t st, float lr);                 // one step; clears the gradient
    int train_step(const GuideRec* d_recs, int n, cudaStream_t st, float lr);
    // Synchronises `st`; -3 (with error()) if a training kernel gave up a
    // bounded wait since init.
    int failed(cudaStream_t st);
    int forward_rows(const float* d_in, int n, float* d_out, cudaStream_t st);
    int encode_rows(const float* p01, const float* nrm, const float* wo, int n, float* out, cudaStream_t st);
    const void* weights_bf16() const { return wq_; }
    const float* master() const { return master_; }
    const float* grad() const { return grad_; }
    int steps() const { return step_; }
    const std::string& error() const { return err_; }

private:
    void release();
    float* master_ = nullptr;
    float* m_ = nullptr;
    float* v_ = nullptr;
    float* grad_ = nullptr;
    float* csum_ = nullptr;
    void* wq_ = nullptr;
    void* ws_ = nullptr;       // per-record layer inputs and gradients of the last batch (BF16)
    float* part_ = nullptr;    // per-block partial gradients
    int* flag_ = nullptr;      // set when a bounded device wait gave up
    int ws_rows_ = 0, part_blocks_ = 0;
    int step_ = 0;
    std::string err_;
};

}  // namespace lucid
