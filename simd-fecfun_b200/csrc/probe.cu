// Integer issue-rate microbenchmark: the denominator of the decoder's ALU
// roofline.  Each thread runs eight interleaved chains of one 32-bit logic op
// (lop3) or add (iadd3); inline PTX keeps the compiler from folding them.
#include <algorithm>
#include <utility>

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

// Throughput of single operations on packed lanes, the measurements behind
// the int8 decoder's choice of f16x2 arithmetic: each thread runs eight
// independent chains of one operation.  OP indexes kOpNames.
__device__ __forceinline__ uint32_t op_apply(int op, uint32_t a, uint32_t b) {
    uint32_t d = a;
    switch (op) {
        case 0: d = __vsubss4(a, b); break;
        case 1: d = __vaddss4(a, b); break;
        case 2: d = __vabsss4(a) ^ b; break;
        case 3: d = __vmins4(a, b); break;
        case 4: d = __vsub4(a, b); break;
        case 5: d = __vsubss2(a, b); break;
        case 6: asm("min.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); break;
        case 7: asm("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); break;
        case 8: asm("min.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); break;
        case 9: asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); break;
        case 10: asm("fma.rn.f16x2 %0, %1, %2, %1;" : "=r"(d) : "r"(a), "r"(b)); break;
        case 11: asm("min.xorsign.abs.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); break;
        case 12: asm("set.eq.u32.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b)); d ^= a; break;
        case 13: {
            float f;
            asm volatile("min.f32 %0, %1, %2;" : "=f"(f) : "f"(__uint_as_float(a)), "f"(__uint_as_float(b)));
            d = __float_as_uint(f);
            break;
        }
        case 14: d = __float_as_uint(__fadd_rn(__uint_as_float(a), __uint_as_float(b))); break;
        case 15: d = __byte_perm(a, b, 0x5410); break;
        default: asm("lop3.b32 %0, %1, %2, %1, 0x96;" : "=r"(d) : "r"(a), "r"(b)); break;
    }
    return d;
}

template <int OP>
__global__ void op_rate_kernel(uint32_t* out, int iters, uint32_t seed) {
    uint32_t x[8];
    const uint32_t y = 0x3c003c00u ^ (threadIdx.x & 7);   // 1.0 in both f16 lanes, perturbed
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = 0x40004000u + seed + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = op_apply(OP, x[c], y);
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) r ^= x[c];
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

namespace {
const char* const kOpNames[] = {"vsubss4 (int8x4 saturating sub)", "vaddss4", "vabsss4", "vmins4", "vsub4 (wrapping)",
                                "vsubss2 (int16x2 saturating sub)", "min.s16x2", "add.s16x2", "min.f16x2",
                                "add.rn.f16x2", "fma.rn.f16x2", "min.xorsign.abs.f16x2", "set.eq.u32.f16x2",
                                "fmin (f32)", "add.rn.f32", "prmt", "lop3"};
constexpr int kNumOps = 17;

template <int... Ops>
void launch_op(int op, int blocks, int threads, uint32_t* out, int iters, uint32_t seed, std::integer_sequence<int, Ops...>) {
    ((op == Ops ? (ldpc::op_rate_kernel<Ops><<<blocks, threads>>>(out, iters, seed), 0) : 0), ...);
}
}  // namespace

extern "C" int ldpc_probe_op_rates(int device, double* ops_per_clk_sm, int n_ops, const char** names) {
    if (!ops_per_clk_sm || n_ops < 0) return fail(LDPC_ERR_INVALID_ARG, "NULL argument");
    if (n_ops > kNumOps) n_ops = kNumOps;
    CUDA_TRY(cudaSetDevice(device));
    int sms = 0, clk_khz = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CUDA_TRY(cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device));
    const int threads = 256, blocks = sms * 8, iters = 4096;
    uint32_t* out = nullptr;
    CUDA_TRY(cudaMalloc(&out, sizeof(uint32_t) * threads * blocks));
    for (int op = 0; op < n_ops; ++op) {
        const double ops = (double)threads * blocks * iters * 8;
        const double r = ldpc::time_ops(
            [&](int rep) { launch_op(op, blocks, threads, out, iters, 17u + rep, std::make_integer_sequence<int, kNumOps>()); },
            ops);
        if (r < 0) {
            cudaFree(out);
            return fail(LDPC_ERR_CUDA, "op-rate probe kernel %d failed", op);
        }
        ops_per_clk_sm[op] = r / ((double)sms * clk_khz * 1e3);
        if (names) names[op] = kOpNames[op];
    }
    cudaFree(out);
    return LDPC_OK;
}
