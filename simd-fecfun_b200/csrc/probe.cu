// Integer issue-rate microbenchmark: the denominator of the decoder's ALU
// roofline.  Each thread runs eight interleaved chains of one 32-bit logic op
// (lop3) or add (iadd3); inline PTX keeps the compiler from folding them.
#include <algorithm>

#include "internal.h"

namespace ldpc {
namespace {

template <int OP>
__global__ void int_peak_kernel(uint32_t* out, int iters, uint32_t seed) {
    uint32_t x[8];
    const uint32_t y = seed ^ (threadIdx.x * 0x9E3779B9u);
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = seed + c * 0x01010101u + blockIdx.x;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (OP == 0)
                asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[c]) : "r"(y), "r"(x[(c + 1) & 7]));
            else
                asm volatile("add.u32 %0, %0, %1;" : "+r"(x[c]) : "r"(x[(c + 3) & 7]));
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) r ^= x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// FP32 fused multiply-add (OP 0) or MUFU base-2 exponential (OP 1) chains,
// eight per thread: the denominators of the float decoders' roofline.
template <int OP>
__global__ void fp_peak_kernel(float* out, int iters, float seed) {
    float x[8];
    const float y = 0.999999f, z = 1e-7f * (float)(threadIdx.x & 7);
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = seed + 0.01f * (float)c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (OP == 0)
                asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(x[c]) : "f"(y), "f"(z));
            else
                asm volatile("ex2.approx.ftz.f32 %0, %0;" : "+f"(x[c]));
        }
    }
    float r = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) r += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

// Best rate over repetitions of a probe kernel (ops/s), or -1 on a CUDA error.
template <class Launch>
double time_ops(Launch launch, double ops) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        launch(rep);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms > 0) best = std::max(best, ops / (ms * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? best : -1.0;
}

}  // namespace
}  // namespace ldpc

using ldpc::fail;

extern "C" int ldpc_probe_fp32_peak(int device, double* fma_per_s, double* mufu_per_s) {
    if (!fma_per_s || !mufu_per_s) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int threads = 256, blocks = sms * 8, iters = 8192;
    float* out = nullptr;
    CUDA_TRY(cudaMalloc(&out, sizeof(float) * threads * blocks));
    const double ops = (double)threads * blocks * iters * 8;
    const double f = ldpc::time_ops([&](int rep) { ldpc::fp_peak_kernel<0><<<blocks, threads>>>(out, iters, 1.0f + rep); }, ops);
    const double m = ldpc::time_ops([&](int rep) { ldpc::fp_peak_kernel<1><<<blocks, threads>>>(out, iters / 8, 0.5f + rep); },
                                    ops / 8);
    cudaFree(out);
    if (f < 0 || m < 0) return fail(LDPC_ERR_CUDA, "fp32 probe kernel failed");
    *fma_per_s = f;
    *mufu_per_s = m;
    return LDPC_OK;
}

extern "C" int ldpc_probe_int32_peak(int device, double* ops_per_s) {
    if (!ops_per_s) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int threads = 256, blocks = sms * 8, iters = 8192;
    uint32_t* out = nullptr;
    CUDA_TRY(cudaMalloc(&out, sizeof(uint32_t) * threads * blocks));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int op = 0; op < 2; ++op) {
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0);
            if (op == 0)
                ldpc::int_peak_kernel<0><<<blocks, threads>>>(out, iters, 0x12345678u + rep);
            else
                ldpc::int_peak_kernel<1><<<blocks, threads>>>(out, iters, 0x12345678u + rep);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && ms > 0) best = std::max(best, (double)threads * blocks * iters * 8 / (ms * 1e-3));
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    CUDA_TRY(cudaGetLastError());
    *ops_per_s = best;
    return LDPC_OK;
}
