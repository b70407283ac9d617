// Kernel parameter blocks shared by the host code and the kernels.
#pragma once
#include <stdint.h>

namespace ldpc {

constexpr int OMS_MAX_L = 48;
constexpr int OMS_MAX_SLOTS_E = 256;   // L*D edge slots carried in the kernel parameters
constexpr int OMS_MAX_BUCKETS = 32;

struct OmsTables {
    int z, mcol, n, stride, G;
    int L, D;
    int kbits;                       // data columns * Z (hard-decision bits per codeword)
    int hard_words;                  // ceil(kbits / 32)
    int16_t rw[OMS_MAX_L];
    int32_t colz[OMS_MAX_SLOTS_E];   // column * Z of edge slot l*D + j
    int16_t shift[OMS_MAX_SLOTS_E];  // circulant shift of edge slot l*D + j
};

struct OmsJob {
    const int8_t* llr;               // [ncw][n]
    long long ncw;
    int8_t* post_out;                // [ncw][n] or null
    uint32_t* hard_out;              // [ncw][hard_words] or null; bit i of codeword = data bit i, LSB first
    uint8_t* iters_out;              // [ncw] or null
    const uint32_t* ref_bits;        // [ref_period][hard_words] sent data bits, or null
    long long ref_period;
    long long bucket_size;           // codewords per counter bucket (e.g. per SNR point)
    unsigned long long* counters;    // [n_buckets][4]: codewords, iterations, bit errors, codeword errors
    int n_buckets;
    int num_par;                     // interleaved sub-codewords per codeword (codeword errors counted per slot t % num_par)
    int max_iter;
    uint32_t beta2;                  // half2 bits of beta8
    uint32_t maxv2;                  // half2 bits of Max8
    unsigned long long* queue;       // work counter, zero before launch
    unsigned int* status;            // error word (0 = ok)
    int synd_loop;                   // 1: syndrome as a loop over the parameter tables (smaller code)
};

// ---- float decoders (sum-product / offset min-sum), R in shared memory ----
constexpr int SP_MAX_L = 64;
constexpr int SP_MAX_E = 512;

struct SpTables {
    int z, mcol, n, L, G;            // G = codewords per CTA (one per group of Z threads)
    int stride;                      // posterior words per group in shared memory
    int kbits, hard_words;
    int E;                           // sum of row weights
    int nostage;                     // 1: no shared staging buffer; refill from global memory
    int16_t rw[SP_MAX_L];
    int16_t ebase[SP_MAX_L];         // first edge of layer l
    int32_t colz[SP_MAX_E];          // column * Z of edge e
    int16_t shift[SP_MAX_E];
};

template <class T>                   // T = float or double
struct SpJobT {
    const T* llr;
    long long ncw;
    T* post_out;
    uint32_t* hard_out;
    uint8_t* iters_out;
    const uint32_t* ref_bits;
    long long ref_period;
    long long bucket_size;
    unsigned long long* counters;
    int n_buckets;
    int num_par;
    int max_iter;
    int prod;                        // 1 = sum-product, 0 = offset min-sum
    T beta;
    T maxv;                          // Max_val as decode_row computes it
    T* r_scratch;                    // global check messages when they do not fit shared memory
};
using SpJob = SpJobT<float>;

// ---- int8 offset min-sum with run-time code tables (any shape; several codes per launch) ----
constexpr int RT_MAX_L = 64;
constexpr int RT_MAX_E = 1024;
constexpr int RT_MAX_Z = 511;        // shifts are packed in 9 bits

// One code of a launch, in device memory; a CTA copies it into shared memory
// when it starts work on that code.
struct alignas(16) RtCode {
    int z, n, L, E;
    int G;                           // codeword pairs per CTA (thread (t, g): check row t, pair g)
    int stride;                      // posterior words per pair in shared memory
    int kbits, hard_words, num_par, max_iter;
    uint32_t maxv2;                  // half2 bits of Max8
    uint32_t beta2[RT_MAX_L];        // half2 bits of beta8 per layer
    uint32_t quirk2[RT_MAX_L];       // -128.0 in both lanes where beta8 = 0 (abs8(-128) = -128), else 0
    const uint16_t* beta_tab;        // or null: half bits of beta8 per [row][layer]; a codeword's iteration i
    int tab_rows;                    //   (0-based) uses row min(i, tab_rows - 1), in place of beta2 / quirk2
    int16_t rw[RT_MAX_L];
    int16_t ebase[RT_MAX_L];         // first edge of layer l
    uint32_t edge[RT_MAX_E];         // (column * Z) << 9 | shift
};

// One batch of codewords of one code (device pointers).
struct RtJob {
    const int8_t* llr;               // [ncw][n]
    long long ncw;
    int8_t* post_out;
    uint32_t* hard_out;
    uint8_t* iters_out;
    const uint32_t* ref_bits;
    long long ref_period;
    long long bucket_size;
    unsigned long long* counters;    // [n_buckets][4] as OmsJob
    int n_buckets;
    int code;                        // index into the launch's code array
};

// Codewords [lo, hi) of job `job`, decoded by one CTA.
struct RtChunk {
    int job;
    int pad;
    long long lo, hi;
};

struct RtLaunch {
    const RtCode* codes;
    const RtJob* jobs;               // null: one job, job0, split evenly over the grid
    const RtChunk* chunks;           // CTA b takes chunk b first, then the next claimed one (or b + grid, ...)
    int n_chunks;
    unsigned int* claim;             // chunks claimed beyond the first grid (zeroed before each launch), or null
    RtJob job0;
    uint32_t* r_scratch;             // check messages in global memory (when not in shared memory)
    long long r_words_per_cta;
};

// ---- fused generation ----
constexpr int GEN_MAX_TERMS = 1024;
constexpr int GEN_MAX_PAR = 64;
constexpr int GEN_MAX_COLS = 128;
constexpr int GEN_MAX_SNR = 32;

struct GenTables {
    int z, mcol, mrow, n, kbits, hard_words, words_per_col;
    int n_par;                       // parity records in schedule order
    int16_t par_col[GEN_MAX_PAR];
    int16_t par_first[GEN_MAX_PAR];
    int16_t par_cnt[GEN_MAX_PAR];
    int16_t term_col[GEN_MAX_TERMS];
    int16_t term_shift[GEN_MAX_TERMS];
    // schedules of more than GEN_MAX_TERMS terms (802.3ca's dense inverse):
    // the terms in device memory, [n_terms] columns then [n_terms] shifts
    const int16_t* term_dev;
    int n_terms;
    const uint8_t* punct;            // [n] 0/1, device
    const uint8_t* filler;           // [n] 0/1, device
    int any_punct, any_filler;
};

struct GenJob {
    uint64_t seed;
    uint64_t cw_offset;
    long long n_per_snr;
    int n_snr;
    float sigma[GEN_MAX_SNR];
    float sigma_factor[GEN_MAX_SNR];
    float max_abs;
    int8_t* llr_i8;                  // [n_snr][n_per_snr][n] or null
    int16_t* llr_i16;                // int16 contexts (gen_metrics: roundi, then compress)
    int32_t* llr_i32;                // int32 contexts (gen_metrics: roundi)
    double* llr_f64;                 // double contexts (gen_metrics: to_double of the float LLR)
    float* llr_f32;                  // [n_snr][n_per_snr][n] or null
    uint32_t* data_bits;             // [n_per_snr][hard_words] or null
    unsigned long long* uncoded;     // [n_snr] or null
    uint32_t philox_rk[20];          // Philox round keys of `seed`: (lo, hi) + r * (0x9E3779B9, 0xBB67AE85), r = 0..9
    long long snr_stride;            // elements between SNR rows: n_per_snr * n
};

}  // namespace ldpc
