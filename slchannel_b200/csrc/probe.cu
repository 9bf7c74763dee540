// probe.cu -- FMA-pipe throughput of this GPU, measured with a
// register-resident FMA-chain kernel.  It is the denominator against which
// the trace+gather kernels' arithmetic rate is reported (their DRAM traffic
// is far below the HBM roofline, so HBM alone does not bound them).  Not on
// the step path.
#include <string>

#include "../../include/slc_b200.h"
#include "slc_internal.h"

namespace {

constexpr int kChains = 8;   // independent FMA chains per thread
constexpr int kUnroll = 16;  // chain steps per loop trip
constexpr int kThreadsP = 256;

// x <- x * a + b on kChains chains; a < 1 so every chain settles near
// b / (1 - a) (no overflow, no subnormals).  The sums are stored so that
// nothing is dead code.
template <typename T>
__global__ void __launch_bounds__(kThreadsP) k_fma_chain(T a, T b, int trips, T *out)
{
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int t = 0; t < trips; ++t) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
        }
    }
    T s = (T)0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[(size_t)blockIdx.x * kThreadsP + threadIdx.x] = s;
}

template <typename T>
int run(int sms, int trips, cudaStream_t s, double *gflops)
{
    const int blocks = sms * (2048 / kThreadsP);
    T *out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * (size_t)blocks * kThreadsP) != cudaSuccess) {
        cudaGetLastError();
        return slc_report_error(SLC_E_NOMEM, "slc_fma_peak: device allocation failed");
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = SLC_OK;
    float best = 0.f;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = SLC_E_CUDA;
    } else {
        const T a = (T)0.999999, b = (T)1e-6;
        k_fma_chain<T><<<blocks, kThreadsP, 0, s>>>(a, b, trips, out);  // warm-up
        count_launches(1);
        for (int r = 0; r < 3 && rc == SLC_OK; ++r) {
            cudaEventRecord(e0, s);
            k_fma_chain<T><<<blocks, kThreadsP, 0, s>>>(a, b, trips, out);
            count_launches(1);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = SLC_E_CUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r == 0 || ms < best) best = ms;
        }
        if (cudaGetLastError() != cudaSuccess) rc = SLC_E_CUDA;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    if (rc != SLC_OK) return slc_report_error(rc, "slc_fma_peak: a CUDA call failed");
    const double fmas = (double)blocks * kThreadsP * trips * kUnroll * kChains;
    *gflops = 2.0 * fmas / (best * 1e-3) / 1e9;
    return SLC_OK;
}

}  // namespace

extern "C" int slc_fma_peak(int fp64, double *gflops, void *stream)
{
    if (!gflops) return slc_report_error(SLC_E_INVALID, "slc_fma_peak: null output");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return slc_report_error(SLC_E_CUDA, "slc_fma_peak: no CUDA device");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    return fp64 ? run<double>(sms, 1024, s, gflops) : run<float>(sms, 2048, s, gflops);
}
