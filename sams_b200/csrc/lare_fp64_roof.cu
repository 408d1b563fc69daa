// lare_fp64_roof.cu -- measured FP64 instruction throughput of this GPU.
//
// The LARE3D step is FP64 arithmetic with many IEEE divisions and square
// roots by data, so next to the HBM roofline it has a compute roof: the
// number of FP64 operations a step needs divided by the rate the GPU
// sustains for each kind.  This file measures those rates with CUDA events:
// every thread runs eight independent dependency chains of one operation
// (enough independent work per warp to hide its latency), on a grid of
// eight 256-thread blocks per SM.  Rates are thread-level operations per
// second (one division = one operation, whatever it compiles to).
//
// Measured kinds (the rates[] order):
//   0 add   x = x + c
//   1 mul   x = x * c
//   2 fma   x = fma(x, c, d)                  (explicit fused multiply-add)
//   3 div   x = c / x                         (IEEE round-to-nearest division)
//   4 sqrt  x = sqrt(x * c)                   (one multiply + one IEEE sqrt)
//   5 rcp   x = __drcp_rn(x) * c              (one correctly rounded reciprocal + one multiply)
#include "sams_lare.h"

#include <cuda_runtime.h>
#include <string>

void sams_capi_set_last_error(const std::string &msg);

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

template <int OP>
__global__ void __launch_bounds__(kThreads) k_fp64_chain(double *out, double c, double d, int iters)
{
    double x[kChains];
#pragma unroll
    for (int q = 0; q < kChains; ++q) x[q] = 1.0 + 1e-3 * (double)(q + (threadIdx.x & 7));
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < kChains; ++q) {
            if (OP == 0) x[q] = x[q] + c;
            if (OP == 1) x[q] = x[q] * c;
            if (OP == 2) x[q] = fma(x[q], c, d);
            if (OP == 3) x[q] = c / x[q];
            if (OP == 4) x[q] = sqrt(x[q] * c);
            if (OP == 5) x[q] = __drcp_rn(x[q]) * c;
        }
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kChains; ++q) s += x[q];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live; one slot per thread
}

template <int OP>
int time_op(double *out, int blocks, int iters, cudaEvent_t e0, cudaEvent_t e1, double c, double d, double *rate)
{
    k_fp64_chain<OP><<<blocks, kThreads>>>(out, c, d, iters / 8);  // warm-up
    cudaEventRecord(e0);
    k_fp64_chain<OP><<<blocks, kThreads>>>(out, c, d, iters);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) return (int)e;
    float ms = 0.f;
    if ((e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) return (int)e;
    *rate = (double)blocks * kThreads * kChains * (double)iters / (ms * 1e-3);
    return 0;
}

}  // namespace

extern "C" int sams_lare_fp64_rates(int device, double rates[6])
{
    if (!rates) {
        sams_capi_set_last_error("sams_lare_fp64_rates: null output");
        return SAMS_ERR_INVALID;
    }
    int sms = 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        sams_capi_set_last_error(std::string("sams_lare_fp64_rates: ") + cudaGetErrorString(e));
        return SAMS_ERR_CUDA;
    }
    const int blocks = 8 * sms;
    double *out = nullptr;
    if ((e = cudaMalloc(&out, (size_t)blocks * kThreads * sizeof(double))) != cudaSuccess) {
        sams_capi_set_last_error(std::string("sams_lare_fp64_rates: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? SAMS_ERR_NOMEM : SAMS_ERR_CUDA;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = 0;
    // constants keep every chain finite and normal: x + 1e-9, x * (1 + 1e-12),
    // fma towards a fixed point near 1, c / x and c * rcp(x) alternate around
    // sqrt(c), sqrt(2.25 x) converges to 2.25
    if (!rc) rc = time_op<0>(out, blocks, 1 << 16, e0, e1, 1e-9, 0.0, &rates[0]);
    if (!rc) rc = time_op<1>(out, blocks, 1 << 16, e0, e1, 1.0 + 1e-12, 0.0, &rates[1]);
    if (!rc) rc = time_op<2>(out, blocks, 1 << 16, e0, e1, 0.5, 0.5, &rates[2]);
    if (!rc) rc = time_op<3>(out, blocks, 1 << 13, e0, e1, 1.5, 0.0, &rates[3]);
    if (!rc) rc = time_op<4>(out, blocks, 1 << 13, e0, e1, 2.25, 0.0, &rates[4]);
    if (!rc) rc = time_op<5>(out, blocks, 1 << 13, e0, e1, 1.5, 0.0, &rates[5]);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (rc) {
        sams_capi_set_last_error(std::string("sams_lare_fp64_rates: ") + cudaGetErrorString((cudaError_t)rc));
        return SAMS_ERR_CUDA;
    }
    return SAMS_OK;
}
