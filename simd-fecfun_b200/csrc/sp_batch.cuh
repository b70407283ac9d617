// Float decoders (sum-product or offset min-sum) over several codes in one
// persistent launch: the chunk list of the int8 batch (oms_rt.cuh), each
// chunk decoded by sp_decode_range with the code's tables copied into shared
// memory when the CTA changes code.
#pragma once
#include "sp_f32.cuh"
#include "tables.h"

namespace ldpc {

// One code of a float batch, in device memory.
struct alignas(16) SpCode {
    SpTables t;
    int max_iter, num_par;
    float beta, maxv;                // offset (min-sum) and decode_row's Max_val
};

struct SpBatchJob {
    const float* llr;                // [ncw][n]
    long long ncw;
    float* post_out;
    uint32_t* hard_out;
    uint8_t* iters_out;
    const uint32_t* ref_bits;
    long long ref_period;
    long long bucket_size;
    unsigned long long* counters;
    int n_buckets;
    int code;
};

struct SpBatchLaunch {
    const SpCode* codes;
    const SpBatchJob* jobs;
    const RtChunk* chunks;
    int n_chunks;
    unsigned int* claim;             // chunks claimed beyond the first grid (zeroed before each launch)
    float* r_scratch;                // per-CTA messages when they do not fit shared memory
    long long r_words_per_cta;
};

__host__ __device__ constexpr int sp_code_bytes() { return (int)((sizeof(SpCode) + 15) & ~(size_t)15); }

template <int DMAX, bool PROD, bool RSMEM>
__global__ void __maxnreg__(sp_max_regs(DMAX, PROD, RSMEM)) sp_batch_kernel(const __grid_constant__ SpBatchLaunch lp) {
    extern __shared__ __align__(16) unsigned char spb_smem[];
    __shared__ int s_code;
    const SpCode& C = *reinterpret_cast<const SpCode*>(spb_smem);
    float* sm_f = reinterpret_cast<float*>(spb_smem + sp_code_bytes());
    if (threadIdx.x == 0) s_code = -1;
    __shared__ int s_claim;
    // chunk b first, then the next unclaimed chunk: CTAs that drew cheap
    // chunks take more of them
    auto next_chunk = [&](int ci) -> int {
        if (!lp.claim) return ci + (int)gridDim.x;
        __syncthreads();
        if (threadIdx.x == 0) s_claim = (int)gridDim.x + (int)atomicAdd(lp.claim, 1u);
        __syncthreads();
        return s_claim;
    };
    for (int ci = blockIdx.x; ci < lp.n_chunks; ci = next_chunk(ci)) {
        const RtChunk ch = lp.chunks[ci];
        const SpBatchJob bj = lp.jobs[ch.job];
        __syncthreads();   // the previous chunk is finished with the shared tables and state
        if (s_code != bj.code) {
            const uint4* src = reinterpret_cast<const uint4*>(lp.codes + bj.code);
            uint4* dst = reinterpret_cast<uint4*>(spb_smem);
            for (int i = threadIdx.x; i < (int)(sizeof(SpCode) / 16); i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            if (threadIdx.x == 0) s_code = bj.code;
        }
        SpJob job;
        job.llr = bj.llr;
        job.ncw = bj.ncw;
        job.post_out = bj.post_out;
        job.hard_out = bj.hard_out;
        job.iters_out = bj.iters_out;
        job.ref_bits = bj.ref_bits;
        job.ref_period = bj.ref_period;
        job.bucket_size = bj.bucket_size;
        job.counters = bj.counters;
        job.n_buckets = bj.n_buckets;
        job.num_par = C.num_par;
        job.max_iter = C.max_iter;
        job.prod = PROD;
        job.beta = C.beta;
        job.maxv = C.maxv;
        job.r_scratch = nullptr;
        sp_decode_range<DMAX, PROD, RSMEM>(C.t, job, ch.lo, ch.hi, sm_f,
                                           RSMEM ? nullptr : lp.r_scratch + (long long)blockIdx.x * lp.r_words_per_cta);
    }
}

}  // namespace ldpc
