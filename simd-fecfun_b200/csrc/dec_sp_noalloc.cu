// ldpc_decode_f32_noalloc: the float decoders (sum-product, offset min-sum)
// without a context and without allocating device memory.
//
// Who needs it.  ldpc_ctx_create allocates device memory: work counters,
// encoder tables and, for codes whose check messages do not fit in shared
// memory (802.3ca, large 5G lifts), a message scratch area of several tens of
// MB.  Some callers cannot allocate.  For example:
//   - their device memory is reserved at start-up by another allocator (a
//     framework's caching pool, a fixed per-process budget);
//   - they share the GPU with latency-sensitive streams, since cudaFree, and
//     at times cudaMalloc, synchronise the whole device;
//   - they have no way to recover from an out-of-memory error in the middle
//     of a run.
// This entry point takes the code and the configuration directly, and keeps
// the check messages in the fixed array below, reserved once when the
// library's module loads on a device.
//
// Limits.
//   - The array holds kScratchBytes.  Each CTA needs E * threads * 4 bytes
//     (E = edges per lifted row block, threads = the CTA size).  The grid is
//     capped at the number of CTAs the array holds.  A code whose single CTA
//     needs more than the whole array is rejected with LDPC_ERR_UNSUPPORTED.
//   - Nothing in the array needs to start at zero: the kernel clears the
//     messages of every codeword it starts.
//   - There is one array per device.  Calls whose kernels can overlap on one
//     device (different streams, or host threads without ordering) share it
//     and corrupt each other's messages.  Order them on one stream, or with
//     events.
//   - The first call on each device looks up the array's address and sets the
//     kernels' shared-memory limit.  Make it before any stream capture.  Later
//     calls take no lock: they read a per-device ready flag.
//   - The cached address belongs to the device's current context: after
//     cudaDeviceReset on a device that has used this entry point, the entry
//     point must not be called again in that process.
//   - Shared memory: posteriors and LLR staging of G codewords per CTA, G as
//     the context path picks it, within the same 220 KB limit; a code whose
//     single codeword does not fit with its staging buffer runs without it
//     (5G NR base graph 1 at Z=384, 802.3ca), as the context path does.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

#include "internal.h"
#include "sp_f32.cuh"

namespace {

constexpr size_t kScratchBytes = 32u << 20;     // 32 MiB per device
constexpr int kMaxDevices = 64;
constexpr int kThreads = 512;                   // __launch_bounds__ of the kernels below
// The kernels are the context path's instances (sp_f32_kernel<D, P, false, 512>),
// and a kernel's shared-memory limit is a property of the function: both
// paths set it to the same maximum, so neither lowers it under the other.
constexpr int kMaxSmem = ldpc::kSpMaxSmem;

__device__ __align__(256) float g_sp_scratch[kScratchBytes / sizeof(float)];

struct NoallocKernel {
    int dmax;
    bool prod;
    ldpc::sp_fn k;
};
#define SPN(D_, P_) {D_, P_, ldpc::sp_f32_kernel<D_, P_, false, kThreads>}
const NoallocKernel kKernels[] = {SPN(8, true), SPN(8, false), SPN(16, true), SPN(16, false), SPN(32, true), SPN(32, false)};
#undef SPN

struct DeviceState {
    std::atomic<bool> ready{false};
    float* scratch = nullptr;
    int sms = 0;
};
DeviceState g_dev[kMaxDevices];
std::mutex g_setup_mu;

// Once per device, with that device current: the scratch address, the SM
// count, and the dynamic shared-memory limit of every kernel variant.  After
// that a call reads the ready flag (acquire) and takes no lock.
int device_setup(int dev, DeviceState** out) {
    DeviceState& d = g_dev[dev];
    if (d.ready.load(std::memory_order_acquire)) {
        *out = &d;
        return LDPC_OK;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!d.ready.load(std::memory_order_relaxed)) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_sp_scratch);
        if (e != cudaSuccess)
            return ldpc::fail(LDPC_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", dev,
                              cudaGetErrorString(e));
        if (((uintptr_t)p & 255) != 0) return ldpc::fail(LDPC_ERR_CUDA, "scratch of device %d is not 256-byte aligned", dev);
        CUDA_TRY(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
        for (const NoallocKernel& k : kKernels)
            CUDA_TRY(cudaFuncSetAttribute((const void*)k.k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem));
        d.scratch = (float*)p;
        d.ready.store(true, std::memory_order_release);
    }
    *out = &d;
    return LDPC_OK;
}

}  // namespace

extern "C" int ldpc_decode_f32_noalloc(const ldpc_code* code, const ldpc_cfg* cfg, const float* llr, size_t n,
                                       float* post_out, uint32_t* hard_out, uint8_t* iters_out, void* stream) {
    using ldpc::fail;
    if (!code || !cfg) return fail(LDPC_ERR_INVALID_ARG, "code or cfg is NULL");
    if (cfg->variant != LDPC_F32_SP && cfg->variant != LDPC_F32_OMS)
        return fail(LDPC_ERR_INVALID_ARG, "ldpc_decode_f32_noalloc takes the float variants only (got %d)", cfg->variant);
    if (cfg->max_iter < 1 || cfg->max_iter > 255)
        return fail(LDPC_ERR_UNSUPPORTED, "max_iter=%u outside 1..255", cfg->max_iter);
    if (n && !llr) return fail(LDPC_ERR_INVALID_ARG, "llr is NULL");
    if (n > (size_t)1 << 40) return fail(LDPC_ERR_INVALID_ARG, "n=%zu too large", n);
    const ldpc_code& c = *code;
    if (c.mrow > ldpc::SP_MAX_L || (int)c.row_cols.size() > ldpc::SP_MAX_E)
        return fail(LDPC_ERR_UNSUPPORTED, "float decoder: %d layers / %zu edges exceed the tables", c.mrow,
                    c.row_cols.size());
    const int dmax = c.max_row_weight <= 8 ? 8 : c.max_row_weight <= 16 ? 16 : c.max_row_weight <= 32 ? 32 : 0;
    if (!dmax) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: row weight %d > 32", c.max_row_weight);
    if (c.z > kThreads) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: Z=%d > %d", c.z, kThreads);

    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(LDPC_ERR_UNSUPPORTED, "device %d beyond %d", dev, kMaxDevices);
    DeviceState* ds = nullptr;
    if (int rc = device_setup(dev, &ds)) return rc;
    if (n == 0) return LDPC_OK;

    // tables by value in the kernel parameters, codewords per CTA and the
    // staging rule of the context path (setup_sp); the messages always live
    // in the scratch array
    ldpc::SpTables t;
    int G = std::max(1, std::min(32, 128 / c.z));
    while (G > 1 && ((G * c.z + 31) / 32) * 32 > kThreads) --G;
    const int nstage = (c.z * c.mcol + 3) & ~3;
    auto base_bytes = [&](int g, bool stage) {
        ldpc::fill_sp_tables(c, g, &t);
        return ((((size_t)g * t.stride + 3) & ~(size_t)3) + (stage ? (size_t)g * nstage : 0)) * sizeof(float);
    };
    while (G > 1 && base_bytes(G, true) > (size_t)kMaxSmem) --G;
    const bool nostage = base_bytes(G, true) > (size_t)kMaxSmem;
    const size_t smem = base_bytes(G, !nostage);   // leaves t filled for G
    t.nostage = nostage ? 1 : 0;
    const int threads = ((G * c.z + 31) / 32) * 32;
    if (smem > (size_t)kMaxSmem) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: %zu B of shared memory", smem);
    const size_t per_cta = (size_t)t.E * threads * sizeof(float);
    if (per_cta > kScratchBytes)
        return fail(LDPC_ERR_UNSUPPORTED,
                    "ldpc_decode_f32_noalloc: one CTA needs %zu B of message scratch, the static scratch holds %zu B",
                    per_cta, kScratchBytes);

    const bool prod = cfg->variant == LDPC_F32_SP;
    ldpc::sp_fn k = nullptr;
    for (const NoallocKernel& v : kKernels)
        if (v.dmax == dmax && v.prod == prod) k = v.k;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, threads, smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "float decoder: launch does not fit an SM");

    ldpc::SpJob job;
    memset(&job, 0, sizeof(job));
    job.llr = llr;
    job.ncw = (long long)n;
    job.post_out = post_out;
    job.hard_out = hard_out;
    job.iters_out = iters_out;
    job.ref_period = 1;
    job.bucket_size = (long long)n;
    job.n_buckets = 1;
    job.num_par = c.num_par;
    job.max_iter = (int)cfg->max_iter;
    job.prod = prod;
    job.beta = cfg->beta;
    // decode_row's Max_row_simd (decode_functions.cpp:27-32) for a float build
    job.maxv = cfg->max_row_metric < 1e-6 ? (float)(1.0 - (double)cfg->max_row_metric) : cfg->max_row_metric;
    job.r_scratch = ds->scratch;
    const long long want = ((long long)n + G - 1) / G;
    const long long cap = std::min<long long>((long long)per_sm * ds->sms, (long long)(kScratchBytes / per_cta));
    const int grid = (int)std::min(want, cap);
    k<<<grid, threads, smem, (cudaStream_t)stream>>>(t, job);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}
