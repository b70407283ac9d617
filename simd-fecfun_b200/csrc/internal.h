// Internal declarations shared by the translation units of libldpc_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "ldpc_b200.h"
#include "tables.h"

namespace ldpc {

int fail(int code, const char* fmt, ...);

#define CUDA_TRY(expr)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) return ::ldpc::fail(LDPC_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

typedef void (*oms_fn)(const OmsTables, const OmsJob);
typedef void (*sp_fn)(const SpTables, const SpJob);
typedef void (*sp64_fn)(const SpTables, const SpJobT<double>);
typedef void (*rt_fn)(const RtLaunch);

// The dynamic shared-memory limit is an attribute of the kernel function,
// shared by every context that launches it: set it to the most any launch of
// that kernel may use (never to one context's size, which a later context
// with a smaller size would lower under the first one's launches).
inline cudaError_t allow_dynamic_smem(const void* fn, int bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
constexpr int kOmsMaxSmem = 200 * 1024;     // int8 register-shape kernels
constexpr int kSpMaxSmem = 220 * 1024;      // float decoders (B200: 227 KB per CTA less static shared memory)

struct OmsLaunch {
    int max_threads, min_blocks;   // __launch_bounds__ of this compilation
    oms_fn k_beta, k_beta0;
};

struct CompiledCode {
    int z, L, E;
    int col[256], shift[256];
};

struct OmsInst {
    int L, D;            // layers, edge slots per layer (padded shapes)
    const int* rw;       // exact row weights (fixed shapes) or nullptr
    const CompiledCode* compiled;   // code compiled in completely, or nullptr
    int smem_edges;                 // edge slots whose messages live in shared memory
    int n_launch;
    OmsLaunch launch[4];
};

// Arguments of one decode launch (device pointers).
struct DecodeArgs {
    const void* llr = nullptr;
    size_t n = 0;
    void* post = nullptr;
    uint32_t* hard = nullptr;
    uint8_t* iters = nullptr;
    const uint32_t* ref_bits = nullptr;
    long long ref_period = 1;
    long long bucket_size = 0;
    unsigned long long* counters = nullptr;
    int n_buckets = 0;
    int queue = 0;
};

}  // namespace ldpc

struct ldpc_code {
    int z = 0, mrow = 0, mcol = 0, max_row_weight = 0;
    std::vector<int32_t> row_weights, row_cols, row_shifts;
    bool has_enc = false;
    int num_par = 1;
    std::vector<int32_t> par_cnts, par_colnum, par_offset, punc_list, fill_list;
    int fill_cnt = 0;
    // decoded encoder schedule: parity record i computes column sched_col[i] as the XOR of
    // columns term_col[k] rotated by term_shift[k], k in [sched_first[i], +sched_cnt[i])
    std::vector<int32_t> sched_col, sched_first, sched_cnt, term_col, term_shift;
    std::vector<uint8_t> punct, filler;   // [n] 0/1 masks
};

struct ldpc_ctx {
    ldpc_code code;
    ldpc_cfg cfg;
    int device = 0;
    int sms = 0;
    int n = 0, kbits = 0, hard_words = 0;
    // int8 offset min-sum
    const ldpc::OmsInst* inst = nullptr;
    const ldpc::OmsLaunch* oms_launch = nullptr;
    ldpc::OmsTables omst;
    int oms_threads = 0, oms_smem = 0, oms_ctas = 0;
    uint32_t beta2 = 0, maxv2 = 0;
    bool beta0 = false;
    std::vector<int> layer_beta8;               // per-layer int8 offsets (ldpc_ctx_set_layer_offsets), empty = cfg.beta
    std::vector<int> tab_beta8;                 // int8 offset table [tab_rows][mrow] (ldpc_ctx_set_offset_table)
    int tab_rows = 0;
    uint16_t* d_beta_tab = nullptr;             // the table as half bits, on the device
    int oms_synd_loop = 0;                      // syndrome as a table loop (tuning: LDPC_OMS_SYND_LOOP)
    // int8 offset min-sum over run-time tables (shapes without a compiled kernel)
    bool oms_rt = false;
    ldpc::RtCode* d_rt_code = nullptr;
    ldpc::rt_fn rt_kernel = nullptr;
    int rt_threads = 0, rt_smem = 0, rt_ctas = 0, rt_G = 0;
    uint32_t* d_rt_scratch = nullptr;           // check messages of large codes (global)
    long long rt_words_per_cta = 0;
    // float decoders
    ldpc::SpTables spt;
    ldpc::sp_fn sp_kernel = nullptr;
    ldpc::sp64_fn sp64_kernel = nullptr;        // double variants
    int sp_threads = 0, sp_smem = 0, sp_ctas = 0;
    float* d_sp_scratch = nullptr;              // check messages of large codes (global)
    float maxf = 0.f;
    double maxd = 0.0;                          // Max_val of the double variants
    // int16 / int32 decoders (tables in spt)
    void* int_kernel = nullptr;
    int int_threads = 0, int_smem = 0, int_ctas = 0;
    void* d_int_scratch = nullptr;
    int ibeta = 0, imaxv = 0;
    // generation
    ldpc::GenTables gent;
    bool gen_ok = false;                        // generator/encoder usable for this code
    std::string gen_err;
    uint8_t* d_masks = nullptr;                 // punct[n] then filler[n]
    int16_t* d_gen_terms = nullptr;             // encoder schedule terms beyond the parameter block's capacity
    void* d_sim_llr = nullptr;                  // ldpc_simulate scratch: LLRs of one chunk, all SNR points
    void* d_sim_data = nullptr;                 //   sent data bits of the chunk
    void* d_sim_hard = nullptr;
    size_t sim_cap = 0;                         //   codewords the LLR scratch holds
    // device scratch
    static constexpr int kQueues = 4;
    unsigned long long* d_queue = nullptr;      // work counters, one per concurrent launch
    unsigned int* d_status = nullptr;
    unsigned long long* d_counters = nullptr;   // [OMS_MAX_BUCKETS][4] decode counters + [OMS_MAX_BUCKETS] uncoded
    cudaStream_t streams[2] = {nullptr, nullptr};
    // host-buffer pipeline: per stream, device buffers for one chunk (grow-only)
    void* d_pipe[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
    size_t pipe_bytes[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
};

namespace ldpc {
int setup_oms(ldpc_ctx* x);
int launch_oms(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s);
int setup_oms_rt(ldpc_ctx* x);
int launch_oms_rt(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s);
// Fill `out` for one code: int8 offset beta8[l] per layer (nullptr: beta8_all on every
// layer), Max8 as half2 bits, G codeword pairs per CTA.
int make_rt_code(const ldpc_code& c, int max_iter, uint32_t maxv2, const int* beta8, int beta8_all, int G, RtCode* out);
// Largest row weight the run-time kernels unroll for (0: unsupported).
int rt_dmax(int max_row_weight);
// codeword pairs per CTA of the run-time-table kernel for a code of lift Z
// and length N: CTAs of at most 128 threads (256 for N > 2048), fewest idle lanes
int rt_default_G(int z, int n);
constexpr int kRtMaxThreads = 512;          // __launch_bounds__ of oms_rt_kernel
constexpr int kRtMaxSmem = 200 * 1024;      // dynamic shared memory the run-time kernels may use
rt_fn rt_kernel_for(int dmax, bool quirk, bool rsmem);
int rt_stride(int n, int G);
// dynamic shared memory of one CTA: tables, G pairs of posteriors and staging, messages if rsmem
size_t rt_smem_bytes(int n, int G, int E, int threads, bool rsmem);
int setup_int(ldpc_ctx* x);
int launch_int(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s);
// the decoder of the context's variant
int launch_decode(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s);
// bytes per LLR / posterior element of a variant
inline int llr_bytes(int variant) {
    return variant == LDPC_INT8_OMS ? 1 : variant == LDPC_INT16_OMS ? 2
           : (variant == LDPC_F64_SP || variant == LDPC_F64_OMS) ? 8 : 4;
}
int setup_sp(ldpc_ctx* x);
// float-decoder tables of a code for G codewords per CTA
void fill_sp_tables(const ldpc_code& c, int G, SpTables* t);
int launch_sp(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s);
int setup_gen(ldpc_ctx* x);
int launch_gen(ldpc_ctx* x, uint64_t seed, uint64_t cw_offset, const float* snr_db, size_t n_snr, size_t n_per_snr,
               void* llr_int, float* llr_f32, uint32_t* data_bits, unsigned long long* uncoded, cudaStream_t s);
void release_gen(ldpc_ctx* x);
uint32_t half2_bits(float v);
int8_t max_row_i8(float max_row_metric);   // decode_row's Max_row_simd, int8 build
}  // namespace ldpc
