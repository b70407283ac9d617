// Layered int8 offset min-sum over run-time code tables: any code shape
// (802.11ay, 802.3ca, 5G NR base graphs 1 and 2, ...) and several codes in one
// launch.  Same arithmetic as oms_f16_kernel (packed f16x2 lanes, two
// codewords per 32-bit word, reference int8 semantics bit for bit:
// decode_functions.cpp:11-103, LDPCdecode.cpp:79-201), with
//   - the layer loop over tables in shared memory (row weights, edge columns
//     and shifts), unrolled to DMAX edge slots per layer;
//   - the offset beta8 per layer (a single beta is the reference's case; a
//     table of per-layer offsets serves learned offsets);
//   - the check messages in shared memory (RSMEM) or, for large codes, in a
//     per-CTA global scratch area (L2-resident at these sizes);
//   - work given as chunks (a job's codeword range): CTA b decodes chunks
//     b, b + grid, ...; within a chunk the persistent slot refill of
//     oms_f16_kernel keeps every slot busy.
#pragma once
#include <type_traits>

#include "oms_f16.cuh"

namespace ldpc {

// Offset (half2 bits) and beta = 0 quirk mask of layer l for the two
// codewords of a pair, at iterations it0 (low lane) and it1 (high lane).
__device__ __forceinline__ void rt_offsets(const RtCode& C, int l, int it0, int it1, uint32_t& beta2, uint32_t& quirk) {
    if (!C.beta_tab) {
        beta2 = C.beta2[l];
        quirk = C.quirk2[l];
        return;
    }
    const int last = C.tab_rows - 1;
    const uint32_t b0 = C.beta_tab[(it0 < last ? it0 : last) * C.L + l];
    const uint32_t b1 = C.beta_tab[(it1 < last ? it1 : last) * C.L + l];
    beta2 = b0 | (b1 << 16);
    quirk = (b0 ? 0u : 0x0000d800u) | (b1 ? 0u : 0xd8000000u);
}

template <int DMAX, bool QUIRK>
__device__ __forceinline__ void rt_layer(const RtCode& C, int l, uint32_t* Ps, uint32_t* Rt, int rstride, int t, int gbase,
                                         int z, uint32_t beta2, uint32_t quirk_l) {
    constexpr uint32_t SGN = 0x80008000u;
    const int d = C.rw[l], eb = C.ebase[l];
    const uint32_t quirk = QUIRK ? quirk_l : 0u;
    uint32_t q[DMAX];
    int addr[DMAX];
    uint32_t mn1 = H2_1024, mn2 = H2_1024;
    uint32_t sx = 0;
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
            const uint32_t ed = C.edge[eb + j];
            addr[j] = gbase + (int)(ed >> 9) + wrap_add(t, (int)(ed & 511u), z);
            uint32_t Q = hsub2(Ps[addr[j]], Rt[(eb + j) * rstride]);
            Q = hmin2(hmax2(Q, H2_M128), H2_P127);
            if (QUIRK) {
                uint32_t a = habs2(Q);
                a = hfma2(heq2(Q, H2_M128), quirk, a);
                mn2 = hmin2(mn2, hmax2(mn1, a));
                mn1 = hmin2(mn1, a);
                sx ^= Q;
            } else {
                mn2 = hmin2_xs(mn2, hmax2_xs(mn1, Q));   // as oms_layer: signs ride in mn1
                mn1 = hmin2_xs(mn1, Q);
            }
            q[j] = Q;
        }
    }
    if (!QUIRK) {
        sx = mn1;
        mn1 = habs2(mn1);
        mn2 = habs2(mn2);
    }
    const uint32_t c1 = hmin2(hmax2(hsub2(mn1, beta2), H2_ZERO), C.maxv2);
    const uint32_t c2 = hmin2(hmax2(hsub2(mn2, beta2), H2_ZERO), C.maxv2);
    const uint32_t X = c1 ^ c2;
    const uint32_t M1 = c1 ^ (sx & SGN);
#pragma unroll
    for (int j = 0; j < DMAX; ++j) {
        if (j < d) {
            uint32_t a = habs2(q[j]);
            if (QUIRK) a = hfma2(heq2(q[j], H2_M128), quirk, a);
            const uint32_t eq = heq2_mask(a, mn1);
            const uint32_t Rn = M1 ^ (q[j] & SGN) ^ (eq & X);
            const uint32_t Pn = hmin2(hmax2(hadd2(q[j], Rn), H2_M128), H2_P127);
            Ps[addr[j]] = Pn;
            Rt[(eb + j) * rstride] = Rn;
        }
    }
}

// Calls f(std::integral_constant<int, D>) with the smallest unrolled width D
// >= d among 4, 6, 8, 10, 12, 16, 20, 24 and DMAX: a layer of weight d runs
// d edge slots' worth of predicated instructions rounded up a little, not
// DMAX (d is the same for every thread of the CTA, so the branch is uniform).
template <int DMAX, class F>
__device__ __forceinline__ void rt_dispatch(int d, F&& f) {
#define RT_BUCKET(W)                                               \
    if constexpr (DMAX > W) {                                      \
        if (d <= W) {                                              \
            f(std::integral_constant<int, W>{});                   \
            return;                                                \
        }                                                          \
    }
    RT_BUCKET(4) RT_BUCKET(6) RT_BUCKET(8) RT_BUCKET(10) RT_BUCKET(12) RT_BUCKET(16) RT_BUCKET(20) RT_BUCKET(24)
#undef RT_BUCKET
    f(std::integral_constant<int, DMAX>{});
}

template <int D>
__device__ __forceinline__ uint32_t rt_row_parity(const RtCode& C, int d, int eb, const uint32_t* Ps, int t, int gbase, int z) {
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        if (j < d) {
            const uint32_t ed = C.edge[eb + j];
            x ^= Ps[gbase + (int)(ed >> 9) + wrap_add(t, (int)(ed & 511u), z)];
        }
    }
    return x;
}

// syndrome of this thread's check rows with early exit (as oms_syndrome)
template <int DMAX>
__device__ __forceinline__ void rt_syndrome(const RtCode& C, const uint32_t* Ps, int t, int gbase, int z, uint32_t* synd) {
    uint32_t seen = 0;
    for (int l = 0; l < C.L; ++l) {
        const int d = C.rw[l], eb = C.ebase[l];
        uint32_t x = 0;
        rt_dispatch<DMAX>(d, [&](auto D) { x = rt_row_parity<decltype(D)::value>(C, d, eb, Ps, t, gbase, z); });
        x &= 0x80008000u;
        if (x & ~seen) {
            atomicOr(synd, x);
            seen |= x;
        }
        if (((seen | *reinterpret_cast<volatile uint32_t*>(synd)) & 0x80008000u) == 0x80008000u) break;
    }
}

// Shared memory: [RtCode copy][posteriors G x stride words][LLR staging 2G x nstage bytes][messages (E | 1) x blockDim words if RSMEM]
__host__ __device__ constexpr int rt_code_bytes() { return (int)((sizeof(RtCode) + 15) & ~(size_t)15); }

// Slot phase with the whole CTA on each finished codeword (used when the CTA
// has more warps than codeword slots, where one warp per slot would leave the
// others idle: 5G NR and other long codes).  Every thread derives the same
// set of finished slots from shared state.  Element i of a codeword belongs to
// thread i mod blockDim: that thread reads its finished posterior (hard bit,
// error, posterior out) and then writes the next codeword's LLR there, so no
// element is read by one thread and overwritten by another; warp w's lanes
// hold elements 32 (w + m nwarps) + lane, one hard-decision word per ballot.
// Then, after a barrier, warp k mod nwarps does slot k's bookkeeping, claim
// and prefetch.  Entered after a barrier that follows every thread's
// cp.async wait; the caller commits the prefetches and ends with a barrier.
// it_rd / it_wr: the slots' iteration counts of this iteration parity and of
// the next (-1 = empty slot).
__device__ __forceinline__ void rt_slots_coop(const RtCode& C, const RtJob& job, uint32_t* Ps, int8_t* stage_base, int stride,
                                           int nstage, int nslots, long long hi, int par, long long* s_cur,
                                           long long* s_next, const int* it_rd, int* it_wr, uint32_t (*s_synd)[16],
                                           uint32_t (*s_zero_mask)[16], int* s_busy, unsigned long long& s_head,
                                           unsigned long long (*s_cnt)[4], unsigned* s_err_bits, unsigned* s_err_slots) {
    const int tid = threadIdx.x, nthr = blockDim.x, warp = tid >> 5, lane = tid & 31, nwarps = nthr >> 5;
    const int n = C.n, z = C.z;
    unsigned fin = 0;
    for (int k = 0; k < nslots; ++k) {
        if (s_cur[k] < 0) continue;
        const uint32_t bit = (k & 1) ? 0x80000000u : 0x00008000u;
        if (!(s_synd[par][k >> 1] & bit) || it_rd[k] + 1 >= C.max_iter) fin |= 1u << k;
    }
    for (unsigned f = fin; f; f &= f - 1) {
        const int k = __ffs(f) - 1;
        const long long cw = s_cur[k];
        __half* pk = reinterpret_cast<__half*>(Ps + (k >> 1) * stride) + (k & 1);
        const uint32_t* ref = job.ref_bits ? job.ref_bits + (cw % job.ref_period) * C.hard_words : nullptr;
        unsigned errw = 0, errslots = 0;
        for (int i0 = warp * 32; i0 < C.kbits; i0 += nthr) {
            const int i = i0 + lane;
            const bool b = (i < C.kbits) && __hlt(pk[2 * i], __float2half(0.0f));
            const uint32_t word = __ballot_sync(0xffffffffu, b);
            if (lane == 0 && job.hard_out) job.hard_out[cw * C.hard_words + (i0 >> 5)] = word;
            if (ref) {
                uint32_t e = word ^ ref[i0 >> 5];
                if (i0 + 32 > C.kbits) e &= (1u << (C.kbits - i0)) - 1u;
                errw += __popc(e);
                if (C.num_par == 1) {
                    if (e) errslots = 1u;
                } else if ((e >> lane) & 1u) {
                    errslots |= 1u << ((i % z) % C.num_par);
                }
            }
        }
        if (ref && job.counters) {
            errslots = __reduce_or_sync(0xffffffffu, errslots);
            if (lane == 0 && errw) {
                atomicAdd(&s_err_bits[k], errw);
                atomicOr(&s_err_slots[k], errslots);
            }
        }
        if (job.post_out) {
            int8_t* dst = job.post_out + cw * (long long)n;
            for (int i = tid; i < n; i += nthr) dst[i] = (int8_t)__half2int_rn(pk[2 * i]);
        }
        if (s_next[k] >= 0) {
            const int8_t* st = stage_base + k * nstage;
            for (int i = tid; i < n; i += nthr) pk[2 * i] = __int2half_rn((int)st[i]);
        }
    }
    // every thread has taken its decision from s_cur / it_rd / s_synd, summed
    // its errors and read the staging buffers before the bookkeeping changes them
    __syncthreads();
    for (int k = warp; k < nslots; k += nwarps) {
        const long long cw = s_cur[k];
        if (cw < 0) {
            if (lane == 0) it_wr[k] = -1;
            continue;
        }
        const int it = it_rd[k] + 1;
        if (!((fin >> k) & 1u)) {
            if (lane == 0) {
                it_wr[k] = it;
                s_busy[par] = 1;
            }
            continue;
        }
        const long long nxt = s_next[k];
        unsigned long long c = 0;
        if (lane == 0) {
            if (job.iters_out) job.iters_out[cw] = (uint8_t)it;
            if (job.counters) {
                int bk = (int)(cw / job.bucket_size);
                bk = bk < job.n_buckets ? bk : job.n_buckets - 1;
                atomicAdd(&s_cnt[bk][0], 1ull);
                atomicAdd(&s_cnt[bk][1], (unsigned long long)it);
                if (s_err_bits[k]) {
                    atomicAdd(&s_cnt[bk][2], (unsigned long long)s_err_bits[k]);
                    atomicAdd(&s_cnt[bk][3], (unsigned long long)__popc(s_err_slots[k]));
                    s_err_bits[k] = 0;
                    s_err_slots[k] = 0;
                }
            }
            if (nxt >= 0) c = atomicAdd(&s_head, 1ull);
        }
        if (nxt >= 0) {
            c = __shfl_sync(0xffffffffu, c, 0);
            const long long fresh = (long long)c < hi ? (long long)c : -1;
            if (fresh >= 0) prefetch_llr(stage_base + k * nstage, job.llr, fresh, n, lane);
            if (lane == 0) {
                s_next[k] = fresh;
                s_busy[par] = 1;
            }
        }
        if (lane == 0) {
            s_cur[k] = nxt;
            it_wr[k] = nxt >= 0 ? 0 : -1;
            atomicOr(&s_zero_mask[par][k >> 1], (k & 1) ? 0xffff0000u : 0x0000ffffu);
        }
    }
}

template <int DMAX, bool QUIRK, bool RSMEM>
__global__ void __launch_bounds__(512) oms_rt_kernel(const __grid_constant__ RtLaunch lp) {
    extern __shared__ __align__(16) unsigned char rt_smem[];
    __shared__ long long s_cur[32];
    __shared__ long long s_next[32];
    // iterations done by slot k (-1 = empty), one copy per iteration parity:
    // the slot phase of parity p reads s_it[p] and writes s_it[p ^ 1], so
    // every warp sees the same slot states while others update them
    __shared__ int s_it[2][32];
    __shared__ uint32_t s_synd[2][16];
    __shared__ uint32_t s_zero_mask[2][16];
    __shared__ int s_busy[2];
    __shared__ unsigned long long s_head;
    __shared__ unsigned long long s_cnt[OMS_MAX_BUCKETS][4];
    __shared__ int s_code_idx;
    __shared__ unsigned s_err_bits[32], s_err_slots[32];   // cooperative write-out: per slot error sums

    const RtCode& C = *reinterpret_cast<const RtCode*>(rt_smem);
    uint32_t* const Ps = reinterpret_cast<uint32_t*>(rt_smem + rt_code_bytes());
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nwarps = nthr >> 5;
    if (tid == 0) s_code_idx = -1;

    const int n_chunks = lp.jobs ? lp.n_chunks : (int)gridDim.x;
    __shared__ int s_claim;
    // chunk b first, then the next unclaimed chunk (batch plans) or chunk
    // b + grid: CTAs that drew cheap chunks take more of them
    auto next_chunk = [&](int ci) -> int {
        if (!lp.claim) return ci + (int)gridDim.x;
        __syncthreads();
        if (tid == 0) s_claim = (int)gridDim.x + (int)atomicAdd(lp.claim, 1u);
        __syncthreads();
        return s_claim;
    };
    for (int ci = blockIdx.x; ci < n_chunks; ci = next_chunk(ci)) {
        // ---------------- chunk set-up ----------------
        RtJob job;
        long long lo, hi;
        if (lp.jobs) {
            const RtChunk ch = lp.chunks[ci];
            job = lp.jobs[ch.job];
            lo = ch.lo;
            hi = ch.hi;
        } else {
            job = lp.job0;
            lo = job.ncw * ci / gridDim.x;
            hi = job.ncw * (ci + 1) / gridDim.x;
        }
        __syncthreads();   // the previous chunk is finished with the shared tables
        if (s_code_idx != job.code) {
            const uint4* src = reinterpret_cast<const uint4*>(lp.codes + job.code);
            uint4* dst = reinterpret_cast<uint4*>(rt_smem);
            for (int i = tid; i < (int)(sizeof(RtCode) / 16); i += nthr) dst[i] = src[i];
            __syncthreads();
            if (tid == 0) s_code_idx = job.code;
        }
        const int z = C.z, n = C.n, G = C.G, stride = C.stride, E = C.E;
        const int nslots = 2 * G;
        const int nstage = (n + 15) & ~15;
        int8_t* const stage_base = reinterpret_cast<int8_t*>(Ps) + ((G * stride * 4 + 15) & ~15);
        const int t = tid / G, g = tid - (tid / G) * G;
        const bool active = t < z;
        const int gbase = g * stride;
        // check messages: in shared memory each thread's E words are contiguous
        // at an odd stride (E | 1, so a warp's 32 lanes fall in 32 banks) and
        // edge j of a layer is the layer's base plus an immediate; the global
        // scratch keeps edge-major words (coalesced)
        const int rstride = RSMEM ? 1 : nthr;
        uint32_t* const Rt = RSMEM ? reinterpret_cast<uint32_t*>(stage_base + 2 * G * nstage) + tid * (E | 1)
                                   : lp.r_scratch + (long long)blockIdx.x * lp.r_words_per_cta + tid;

        for (int i = tid; i < OMS_MAX_BUCKETS * 4; i += nthr) (&s_cnt[0][0])[i] = 0;
        for (int i = tid; i < G * stride; i += nthr) Ps[i] = 0;
        for (int e = 0; e < E; ++e) Rt[e * rstride] = 0u;
        if (tid < 32) {
            const long long c0 = lo + tid, c1 = lo + nslots + tid;
            const bool ok = tid < nslots;
            s_cur[tid] = ok && c0 < hi ? c0 : -1;
            s_next[tid] = ok && c1 < hi ? c1 : -1;
            s_it[0][tid] = ok && c0 < hi ? 0 : -1;
            s_it[1][tid] = -1;
            s_err_bits[tid] = s_err_slots[tid] = 0;
            if (tid < 16) {
                s_synd[0][tid] = s_synd[1][tid] = 0;
                s_zero_mask[0][tid] = s_zero_mask[1][tid] = 0;
            }
            if (tid < 2) s_busy[tid] = 0;
        }
        if (tid == 0) s_head = (unsigned long long)(lo + 2 * nslots);
        __syncthreads();
        // first round through the staging buffers (16-byte copies), then the
        // prefetch of the second round (each warp its own slots)
        for (int k = warp; k < nslots; k += nwarps)
            if (s_cur[k] >= 0) prefetch_llr(stage_base + k * nstage, job.llr, s_cur[k], n, lane);
        cp_async_commit();
        cp_async_wait_all();
        __syncwarp();
        for (int k = warp; k < nslots; k += nwarps) {
            if (s_cur[k] >= 0) {
                __half* dst = reinterpret_cast<__half*>(Ps + (k >> 1) * stride) + (k & 1);
                const int8_t* st = stage_base + k * nstage;
                for (int i = lane; i < n; i += 32) dst[2 * i] = __int2half_rn((int)st[i]);
            }
            __syncwarp();
            if (s_next[k] >= 0) prefetch_llr(stage_base + k * nstage, job.llr, s_next[k], n, lane);
        }
        cp_async_commit();
        __syncthreads();

        for (int par = 0;; par ^= 1) {
            // ---------------- one layered iteration ----------------
            // iteration index of this thread's two codewords (offset tables)
            const int it0 = max(s_it[par][2 * g], 0), it1 = max(s_it[par][2 * g + 1], 0);
            for (int l = 0; l < C.L; ++l) {
                if (active) {
                    uint32_t beta2, quirk;
                    rt_offsets(C, l, it0, it1, beta2, quirk);
                    rt_dispatch<DMAX>(C.rw[l], [&](auto D) {
                        rt_layer<decltype(D)::value, QUIRK>(C, l, Ps, Rt, rstride, t, gbase, z, beta2, quirk);
                    });
                }
                __syncthreads();
            }
            if (tid < 16) {
                s_synd[par ^ 1][tid] = 0;
                s_zero_mask[par ^ 1][tid] = 0;
            }
            if (tid == 0) s_busy[par ^ 1] = 0;
            if (active) rt_syndrome<DMAX>(C, Ps, t, gbase, z, &s_synd[par][g]);
            cp_async_wait_all();   // this thread's prefetches (issued in an earlier slot phase)
            __syncthreads();       // syndrome bits final, every prefetched byte visible

            if (nslots < nwarps) {
                // ------- more warps than slots (large codes): the whole CTA writes each
                // finished codeword out and refills its slot -------
                rt_slots_coop(C, job, Ps, stage_base, stride, nstage, nslots, hi, par, s_cur, s_next, s_it[par],
                              s_it[par ^ 1], s_synd, s_zero_mask, s_busy, s_head, s_cnt, s_err_bits, s_err_slots);
            } else {
                // ------- per-warp slots: lane k of every warp evaluates slot k; the
                // finished slots are dealt out in slot order, the j-th to warp
                // j mod nwarps (two codewords finishing together go to different
                // warps) -------
                unsigned done_mask;
                {
                    const int itk = lane < nslots ? s_it[par][lane] : -1;
                    const bool live = itk >= 0;
                    const uint32_t bit = (lane & 1) ? 0x80000000u : 0x00008000u;
                    const bool dn = live && (!(s_synd[par][lane >> 1] & bit) || itk + 1 >= C.max_iter);
                    done_mask = __ballot_sync(0xffffffffu, dn);
                    if (warp == 0 && lane < nslots && !dn) {
                        s_it[par ^ 1][lane] = live ? itk + 1 : -1;
                        if (live) s_busy[par] = 1;
                    }
                }
                int j = 0;
                for (unsigned m = done_mask; m; m &= m - 1, ++j) {
                    if (j % nwarps != warp) continue;
                    const int k = __ffs(m) - 1;
                    const long long cw = s_cur[k];
                    const int gg = k >> 1, hsel = k & 1;
                    const int it = s_it[par][k] + 1;
                    __half* pk = reinterpret_cast<__half*>(Ps + gg * stride) + hsel;
                    const uint32_t* ref = job.ref_bits ? job.ref_bits + (cw % job.ref_period) * C.hard_words : nullptr;
                    unsigned errw, errslots;
                    warp_hard_decisions<false>([&](int i) { return __hlt(pk[2 * i], __float2half(0.0f)); }, C.kbits,
                                               C.hard_words, z, C.num_par,
                                               job.hard_out ? job.hard_out + cw * C.hard_words : nullptr, ref, lane, errw,
                                               errslots);
                    if (job.post_out) {
                        int8_t* dst = job.post_out + cw * (long long)n;
                        for (int i = lane; i < n; i += 32) dst[i] = (int8_t)__half2int_rn(pk[2 * i]);
                    }
                    if (lane == 0 && job.iters_out) job.iters_out[cw] = (uint8_t)it;
                    if (job.counters && lane == 0) {
                        int bk = (int)(cw / job.bucket_size);
                        bk = bk < job.n_buckets ? bk : job.n_buckets - 1;
                        atomicAdd(&s_cnt[bk][0], 1ull);
                        atomicAdd(&s_cnt[bk][1], (unsigned long long)it);
                        if (errw) {
                            atomicAdd(&s_cnt[bk][2], (unsigned long long)errw);
                            atomicAdd(&s_cnt[bk][3], (unsigned long long)__popc(errslots));
                        }
                    }
                    __syncwarp();
                    const long long nxt = s_next[k];
                    if (nxt >= 0) {
                        const int8_t* st = stage_base + k * nstage;
                        for (int i = lane; i < n; i += 32) pk[2 * i] = __int2half_rn((int)st[i]);
                        __syncwarp();
                        unsigned long long c = 0;
                        if (lane == 0) c = atomicAdd(&s_head, 1ull);
                        c = __shfl_sync(0xffffffffu, c, 0);
                        const long long fresh = (long long)c < hi ? (long long)c : -1;
                        if (fresh >= 0) prefetch_llr(stage_base + k * nstage, job.llr, fresh, n, lane);
                        if (lane == 0) {
                            s_next[k] = fresh;
                            s_busy[par] = 1;
                        }
                    }
                    if (lane == 0) {
                        s_cur[k] = nxt;
                        s_it[par ^ 1][k] = nxt >= 0 ? 0 : -1;
                        atomicOr(&s_zero_mask[par][gg], hsel ? 0xffff0000u : 0x0000ffffu);
                    }
                }
            }
            cp_async_commit();
            __syncthreads();
            if (active) {
                const uint32_t m = s_zero_mask[par][g];
                if (m)
                    for (int e = 0; e < E; ++e) Rt[e * rstride] &= ~m;
            }
            if (!s_busy[par]) break;
        }
        cp_async_wait_all();
        if (job.counters) {
            __syncthreads();
            for (int i = tid; i < job.n_buckets * 4; i += nthr) {
                const unsigned long long v = (&s_cnt[0][0])[i];
                if (v) atomicAdd(job.counters + i, v);
            }
        }
    }
}

}  // namespace ldpc
