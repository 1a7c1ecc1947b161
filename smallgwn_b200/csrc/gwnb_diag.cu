// Machine-peak probe behind the traversal's compute roofline.
//
// The Taylor traversal is bound by instruction issue on the CUDA cores, not by HBM: its roofline
// denominator is the FP32 fused-multiply-add throughput of the GPU it runs on, measured here rather
// than taken from a datasheet (clocks under load, power capping and the part's SM count all enter).
// Each thread runs independent FMA chains, enough per warp and enough warps per SM that the FMA
// pipes never wait on a dependency; the device time of one launch, taken with CUDA events on the
// given stream, gives FLOP/s at 2 FLOP per FMA. No smallgwn counterpart.
#include "gwnb_internal.cuh"

namespace gwnb {
namespace {

constexpr int k_chains = 8;
constexpr int k_unroll = 16;

__global__ void __launch_bounds__(256) k_fma_peak(float *__restrict__ sink, int iters, float a, float b) {
    float x[k_chains];
#pragma unroll
    for (int c = 0; c < k_chains; ++c)
        x[c] = static_cast<float>(threadIdx.x + c) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < k_unroll; ++u) {
#pragma unroll
            for (int c = 0; c < k_chains; ++c)
                x[c] = __fmaf_rn(x[c], a, b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < k_chains; ++c)
        s += x[c];
    // a value the chains never reach (they converge to b / (1 - a)); keeps the work observable
    if (s == -1.0f)
        sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

int gwnb_fp32_fma_peak(int iters, double *tflops, double *ms, gwnb_stream_t stream) try {
    if (iters <= 0 || tflops == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "FP32 peak probe: iters must be positive and tflops non-null.");
    cudaStream_t const s = reinterpret_cast<cudaStream_t>(stream);
    int const sms = device_sm_count();
    unsigned const blocks = static_cast<unsigned>(sms) * 8u; // 2,048 threads per SM
    constexpr int threads = 256;
    float *sink = nullptr;
    GWNB_TRY(alloc(&sink, static_cast<std::uint64_t>(blocks) * threads, s));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GWNB_CUDA_TRY(cudaEventCreate(&e0));
    GWNB_CUDA_TRY(cudaEventCreate(&e1));
    // one untimed launch (module load, clocks up), then the timed one
    note_launch(), k_fma_peak<<<blocks, threads, 0, s>>>(sink, iters, 0.9999f, 1e-4f);
    GWNB_CUDA_TRY(cudaEventRecord(e0, s));
    note_launch(), k_fma_peak<<<blocks, threads, 0, s>>>(sink, iters, 0.9999f, 1e-4f);
    GWNB_CUDA_TRY(cudaEventRecord(e1, s));
    GWNB_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.0f;
    GWNB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release(sink, s);
    double const flop = 2.0 * k_chains * k_unroll * static_cast<double>(iters) * blocks * threads;
    *tflops = flop / (static_cast<double>(t) * 1e-3) / 1e12;
    if (ms != nullptr)
        *ms = t;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

} // extern "C"
