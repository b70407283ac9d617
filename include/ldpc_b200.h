/* ldpc_b200.h -- C ABI of the B200 QC-LDPC simulation engine.
 *
 * Drop-in boundary for the reference's hot path (tomt-1/simd-fecfun).  The
 * reference exposes C++-linkage free functions with vectorclass types in
 * their signatures (prototypes: src/Top/LDPCtop.cpp:26-39); this header
 * replaces them with plain C types, opaque handles and status codes.
 *
 * Conventions
 *   - Every call returns an int status (LDPC_OK = 0) and never exits the
 *     process; ldpc_last_error() gives a message for the calling thread.
 *   - "dev" pointers are CUDA device pointers, and the call is asynchronous on
 *     `stream` (a cudaStream_t passed as void*; NULL = legacy default stream).
 *     "_host" calls take host memory and return when the results are there.
 *   - Codeword bit and LLR order is the reference's: column-major blocks,
 *     element c*Z + t is bit t of base-matrix column c (N = Z*mcol elements).
 *   - Hard decisions / data bits are packed LSB-first into 32-bit words:
 *     bit i of a codeword (i < kbits = Z*(mcol-mrow)) is bit (i%32) of word
 *     i/32; each codeword takes hard_words = ceil(kbits/32) words.
 *   - A context is bound to one device and is not thread-safe; different
 *     contexts are independent.
 */
#ifndef LDPC_B200_H
#define LDPC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    LDPC_OK = 0,
    LDPC_ERR_INVALID_ARG = 1,
    LDPC_ERR_BAD_TABLE = 2,     /* malformed or truncated .dat table */
    LDPC_ERR_UNSUPPORTED = 3,   /* parameters outside what the kernels implement */
    LDPC_ERR_CUDA = 4,
    LDPC_ERR_TIMEOUT = 5,       /* a bounded device wait gave up */
    LDPC_ERR_IO = 6,
    LDPC_ERR_NOMEM = 7
};

enum {
    LDPC_INT8_OMS = 0,          /* int8 offset min-sum   (LDPCtop_Vec64c_min)  */
    LDPC_F32_SP = 1,            /* float sum-product     (LDPCtop_Vec16f_prod) */
    LDPC_F32_OMS = 2,           /* float offset min-sum  (LDPCtop_Vec16f_min)  */
    LDPC_INT16_OMS = 3,         /* int16 offset min-sum  (LDPCtop_Vec32s_min)  */
    LDPC_INT32_OMS = 4,         /* int32 offset min-sum  (LDPCtop_Vec16w_min)  */
    LDPC_F64_SP = 5,            /* double sum-product    (LDPCtop_Vec8d_prod)  */
    LDPC_F64_OMS = 6            /* double offset min-sum (LDPCtop_Vec8d_min)   */
};

typedef struct ldpc_code ldpc_code;
typedef struct ldpc_ctx ldpc_ctx;

typedef struct {
    int z, mrow, mcol;          /* lifting size and base-matrix shape */
    int n;                      /* Z*mcol codeword bits */
    int kbits;                  /* Z*(mcol-mrow) data bits (filler included) */
    int num_par;                /* interleaved sub-codewords per codeword */
    int fill_cnt;               /* filler bits */
    int edges;                  /* Z * sum(row weights) */
    int max_row_weight;
    int hard_words;             /* ceil(kbits/32) */
    int has_encoder;            /* encoder schedule present */
} ldpc_code_info;

/* Decoder configuration: the reference's run-time knobs
 * (sim_struct_LDPC.h:3-20) plus the variant, which the reference selects at
 * compile time (build/Makefile:9-14). */
typedef struct {
    int variant;                /* one of the LDPC_* variants above */
    unsigned max_iter;          /* maximum decoder iterations (1..255) */
    float max_row_metric;       /* min-sum clamp, or 1-clamp for sum-product */
    float beta;                 /* offset (truncated to the element type for the integer variants) */
    float llr_scale;            /* LLR_scaling_factor */
    float max_abs_llr;          /* max_abs_LLR */
} ldpc_cfg;

/* Message for the most recent failure on the calling thread ("" if none). */
const char *ldpc_last_error(void);

/* Number of CUDA devices visible (0 when none; never an error). */
int ldpc_device_count(int *count);

/* ---- codes -------------------------------------------------------------- */

/* Load the reference's two table files.  Replaces encode_matrix_allocate()
 * (src/LDPCEnc/encode_matrix_allocate.cpp:38-92) and decode_matrix_allocate()
 * (src/LDPCDec/decode_matrix_allocate.cpp:12-61); unlike those it checks
 * every read and returns LDPC_ERR_IO / LDPC_ERR_BAD_TABLE instead of exiting.
 * enc_path may be NULL (decoder only). */
int ldpc_code_load_dat(const char *enc_path, const char *dec_path, ldpc_code **out);

/* Same from in-memory images of the two files (int32 words, little endian). */
int ldpc_code_from_tables(const int32_t *dec_words, size_t n_dec_words, const int32_t *enc_words,
                          size_t n_enc_words, ldpc_code **out);

int ldpc_code_get_info(const ldpc_code *code, ldpc_code_info *info);
void ldpc_code_destroy(ldpc_code *code);

/* ---- contexts ------------------------------------------------------------- */

/* Binds a code and a configuration to a CUDA device and uploads the tables.
 * Validates the configuration against the chosen variant. */
int ldpc_ctx_create(const ldpc_code *code, const ldpc_cfg *cfg, int device, ldpc_ctx **out);
void ldpc_ctx_destroy(ldpc_ctx *ctx);

/* int8 contexts: one offset per layer (beta_per_layer[mrow], truncated to
 * int8 like cfg.beta) in place of cfg.beta on every layer, e.g. learned
 * offsets quantised to the int8 LLR scale.  NULL restores cfg.beta.  The
 * reference applies one offset to all layers (decode_functions.cpp:59-62).
 * Decoding then runs on the run-time-table kernel.  The call waits for the
 * device to be idle, so it is not for use between asynchronous launches in
 * flight. */
int ldpc_ctx_set_layer_offsets(ldpc_ctx *ctx, const float *beta_per_layer);

/* int8 contexts: an offset table beta[rows][mrow] (1 <= rows <= 255, values
 * truncated to int8 like cfg.beta): iteration i (0-based) of a codeword uses
 * row min(i, rows - 1) -- learned per-(iteration, layer) offsets quantised to
 * the int8 LLR scale.  NULL restores cfg.beta; a later
 * ldpc_ctx_set_layer_offsets replaces it.  The reference applies one offset
 * everywhere (decode_functions.cpp:59-62).  Decoding runs on the
 * run-time-table kernel; the call waits for the device to be idle. */
int ldpc_ctx_set_offset_table(ldpc_ctx *ctx, const float *beta, unsigned rows);

/* ---- decoding ------------------------------------------------------------- */

/* Decode n codewords of int8 LLRs (variant LDPC_INT8_OMS).  Replaces
 * LDPCdecode_set() (src/LDPCDec/LDPCdecode.cpp:203-245), which decodes in
 * place and returns only the sum of iterations; here the results go to
 * separate buffers, each optional (NULL = not wanted):
 *   post_out  [n][N] int8 final posteriors (the reference's decoded_metrics)
 *   hard_out  [n][hard_words] packed hard decisions of the data bits
 *   iters_out [n] iterations each codeword ran (LDPCdecode's return value)
 * dev pointers; asynchronous on stream. */
int ldpc_decode_int8(ldpc_ctx *ctx, const int8_t *llr, size_t n, int8_t *post_out, uint32_t *hard_out,
                     uint8_t *iters_out, void *stream);

/* Float decoders (LDPC_F32_SP, LDPC_F32_OMS): same contract, float LLRs and
 * posteriors. */
int ldpc_decode_f32(ldpc_ctx *ctx, const float *llr, size_t n, float *post_out, uint32_t *hard_out,
                    uint8_t *iters_out, void *stream);

/* Double decoders (LDPC_F64_SP, LDPC_F64_OMS): same contract, double LLRs
 * and posteriors.  The reference's double builds take the float LLRs of
 * gen_metrics widened to double (gen_metrics.cpp:91-93); beta and
 * max_row_metric convert to double as decode_row does (decode_functions.cpp:27-32,
 * 59-60). */
int ldpc_decode_f64(ldpc_ctx *ctx, const double *llr, size_t n, double *post_out, uint32_t *hard_out,
                    uint8_t *iters_out, void *stream);

/* int16 / int32 decoders (LDPC_INT16_OMS / LDPC_INT32_OMS): same contract,
 * LLRs and posteriors of the element type.  The reference's element
 * semantics hold: saturating add/sub, abs of the most negative value is
 * itself, beta and max_row_metric truncated to the element type. */
int ldpc_decode_int16(ldpc_ctx *ctx, const int16_t *llr, size_t n, int16_t *post_out, uint32_t *hard_out,
                      uint8_t *iters_out, void *stream);
int ldpc_decode_int32(ldpc_ctx *ctx, const int32_t *llr, size_t n, int32_t *post_out, uint32_t *hard_out,
                      uint8_t *iters_out, void *stream);

/* Decode with fused error counting (any variant; dev pointers, async).
 * Codeword i is compared with sent data bits data_bits[i % ref_period] and
 * counted in bucket min(i / bucket_size, n_buckets-1) of
 * counters[n_buckets][4] = {codewords, iterations, bit errors, codeword
 * errors per sub-codeword} (LDPC_count_errors.cpp:40-136 fused into the
 * decoder's write-out); counters accumulate, the caller zeroes them.
 * hard_out / iters_out are optional as in ldpc_decode_int8. */
int ldpc_decode_count(ldpc_ctx *ctx, const void *llr, size_t n, uint32_t *hard_out, uint8_t *iters_out,
                      const uint32_t *data_bits, size_t ref_period, size_t bucket_size, unsigned long long *counters,
                      int n_buckets, void *stream);

/* Host-memory versions: copy in, decode, copy out (chunked and overlapped);
 * return when the outputs are in host memory.  *tot_iter (optional) receives
 * the sum of iterations, LDPCdecode_set's return value. */
int ldpc_decode_int8_host(ldpc_ctx *ctx, const int8_t *llr, size_t n, int8_t *post_out, uint32_t *hard_out,
                          uint8_t *iters_out, uint64_t *tot_iter);
int ldpc_decode_f32_host(ldpc_ctx *ctx, const float *llr, size_t n, float *post_out, uint32_t *hard_out,
                         uint8_t *iters_out, uint64_t *tot_iter);
int ldpc_decode_f64_host(ldpc_ctx *ctx, const double *llr, size_t n, double *post_out, uint32_t *hard_out,
                         uint8_t *iters_out, uint64_t *tot_iter);
int ldpc_decode_int16_host(ldpc_ctx *ctx, const int16_t *llr, size_t n, int16_t *post_out, uint32_t *hard_out,
                           uint8_t *iters_out, uint64_t *tot_iter);
int ldpc_decode_int32_host(ldpc_ctx *ctx, const int32_t *llr, size_t n, int32_t *post_out, uint32_t *hard_out,
                           uint8_t *iters_out, uint64_t *tot_iter);

/* Literal drop-in for LDPCdecode_set (LDPCdecode.cpp:203-245): decodes, in
 * place, num_codeword codewords stored in the reference's padded host layout
 * -- per codeword mcol columns of (ceil(Z/simd_par)+2)*simd_par elements,
 * element t of column c at offset simd_par + t (decode_matrix_allocate.cpp:55)
 * -- with elements of the variant's type (int8, int16, int32 or float).
 * *tot_iter receives the sum of iterations. */
int ldpc_decode_set_compat(ldpc_ctx *ctx, void *decoded_metrics, unsigned num_codeword, unsigned simd_par,
                           uint64_t *tot_iter);

/* ---- batched decoding of several codes in one graph ------------------------
 *
 * No counterpart in the reference: it runs one code per process
 * (build/run_LDPCsim.pl:102-109) and one codeword at a time
 * (LDPCdecode.cpp:227-243).  A batch holds several codes, each with its own
 * configuration; all codes use the same variant (LDPC_INT8_OMS, LDPC_F32_SP or
 * LDPC_F32_OMS).  int8 batches also take offsets per layer or per
 * (iteration, layer) (learned offsets).  A plan fixes a list of jobs (device
 * buffers of one code each) and splits them into chunks of equal work.  A
 * plan's launch is one persistent kernel per geometry class (codes that
 * would run at the same occupancy share one; LDPC_BATCH_ONE_LAUNCH forces a
 * single kernel), and it can be replayed from a CUDA graph with one kernel
 * node per class, free to overlap.  CTAs claim chunks from a per-launch
 * counter, so launches of one plan on different streams must not overlap.
 * Per codeword, the results are exactly those of ldpc_decode_int8 /
 * ldpc_decode_count on that code. */
typedef struct ldpc_batch ldpc_batch;
typedef struct ldpc_batch_plan ldpc_batch_plan;

typedef struct {
    int code;                       /* index of the code in the batch */
    const void *llr;                /* dev [n][N_code], int8 or float by the batch's variant */
    size_t n;
    void *post_out;                 /* dev, optional (NULL); element type as llr */
    uint32_t *hard_out;             /* dev [n][hard_words], optional */
    uint8_t *iters_out;             /* dev [n], optional */
    const uint32_t *data_bits;      /* dev, optional: fused counting as ldpc_decode_count */
    size_t ref_period;
    size_t bucket_size;
    unsigned long long *counters;   /* dev [n_buckets][4], accumulated */
    int n_buckets;
} ldpc_batch_job;

int ldpc_batch_create(const ldpc_code *const *codes, const ldpc_cfg *cfgs, int n_codes, int device,
                      ldpc_batch **out);
/* One int8 offset per layer of code `code` (values truncated like beta;
 * 0..127).  NULL restores cfg.beta on every layer.  It affects plans
 * created afterwards. */
int ldpc_batch_set_offsets(ldpc_batch *b, int code, const float *beta_per_layer);
/* An offset table beta[rows][mrow] for code `code` (as
 * ldpc_ctx_set_offset_table); NULL restores cfg.beta.  It replaces the
 * code's per-layer offsets and affects plans created afterwards. */
int ldpc_batch_set_offset_table(ldpc_batch *b, int code, const float *beta, unsigned rows);
void ldpc_batch_destroy(ldpc_batch *b);

/* Plan over `jobs`.  threads = CTA width, for every class (0: the autotuned
 * shapes, else max(256, the class's largest Z)); chunks_per_cta = work
 * chunks per resident CTA (0: tuned or 2). */
int ldpc_batch_plan_create(ldpc_batch *b, const ldpc_batch_job *jobs, int n_jobs, int threads, int chunks_per_cta,
                           ldpc_batch_plan **out);
int ldpc_batch_plan_launch(ldpc_batch_plan *p, void *stream);
/* The first call captures the launch into a CUDA graph; every call replays
 * it, ordered after the work already on `stream`. */
int ldpc_batch_plan_graph_launch(ldpc_batch_plan *p, void *stream);
void ldpc_batch_plan_destroy(ldpc_batch_plan *p);
/* Kernels one launch of the plan runs (one per geometry class; 0 when it
 * has no work). */
int ldpc_batch_plan_kernels(const ldpc_batch_plan *p);

/* Project autotuner: times plans over the first `sample` codewords of each
 * job (outputs not written) for every CTA width in {128..512} that fits and
 * 1, 2, 4 or 8 chunks per CTA, and the plan that leaves every code at its
 * own width (the single-code context's) with the default chunks per CTA.
 * It keeps the fastest setting for later plans and reports it (any output
 * pointer may be NULL; threads = cpc = 0 reports the codes' own widths).
 * int8 jobs of several geometry classes: each class is tuned on its own
 * jobs, and that set is kept when it beats the best single shape and the
 * codes' own widths on the whole sample; the report is then the shape of
 * the slowest class and the whole sample's time. */
int ldpc_batch_autotune(ldpc_batch *b, const ldpc_batch_job *jobs, int n_jobs, size_t sample, int *threads,
                        int *chunks_per_cta, double *ms);

/* ---- learned offsets: differentiable unrolled float offset min-sum --------
 *
 * No counterpart in the reference, whose decode_row has one offset for every
 * layer and iteration (decode_functions.cpp:59-62).  The context must use
 * LDPC_F32_OMS; its max_row_metric is the row clamp.  beta is a device array
 * [iters][mrow] of offsets.  The decoder runs exactly `iters` iterations
 * (no early exit), so the loss is a fixed function of beta.
 *
 * ldpc_learned_forward writes per-iteration checkpoints:
 *   ckpt_p [iters+1][n][N]   posteriors at the start of each iteration,
 *                            plus the final ones;
 *   ckpt_r [iters][n][E]     check messages at the start of each iteration
 *                            (E = ldpc_code_info.edges).
 *
 * ldpc_learned_backward returns the gradient of
 *   L = sum_it loss_w[it] * inv_norm * sum_cw sum_v softplus(-(1 - 2 c_v) P_it+1[v])
 * (binary cross-entropy of the posteriors after every iteration; c = sent
 * code bits, cw_bits [n][N] 0/1).  For each iteration it recomputes the
 * layers from its checkpoint, then runs the adjoint in reverse.
 * gbeta_part [grid][iters*mrow] receives one partial sum per CTA (grid from
 * ldpc_learned_grid); their column sums are dL/dbeta, reduced in a fixed
 * order, so results are deterministic.  grad_llr [n][N] (optional) receives
 * dL/dLLR. */
int ldpc_learned_grid(ldpc_ctx *ctx, size_t n, int *bwd_grid);
int ldpc_learned_forward(ldpc_ctx *ctx, const float *llr, size_t n, int iters, const float *beta, float *ckpt_p,
                         float *ckpt_r, void *stream);
int ldpc_learned_backward(ldpc_ctx *ctx, size_t n, int iters, const float *beta, const float *ckpt_p,
                          const float *ckpt_r, const uint8_t *cw_bits, const float *loss_w, float inv_norm,
                          float *gbeta_part, float *grad_llr, void *stream);
/* Decoding with learned offsets: up to `iters` iterations with early exit on
 * the syndrome, as the float decoders do; outputs as ldpc_decode_f32. */
int ldpc_learned_decode(ldpc_ctx *ctx, const float *llr, size_t n, int iters, const float *beta, float *post_out,
                        uint32_t *hard_out, uint8_t *iters_out, void *stream);

/* ---- channel generation -------------------------------------------------- */

/* Fused generation: random data bits, QC encoding, BPSK, AWGN and LLR
 * quantisation in one kernel.  Replaces gen_rand_databits()
 * (src/Top/gen_rand_databits.cpp:11-40), LDPCencode()
 * (src/LDPCEnc/LDPCencode.cpp:40-100), normdist2()
 * (src/RNGfunc/prng_functions.cpp:148-186) and gen_metrics()
 * (src/Top/gen_metrics.cpp:18-121).  Codeword i of SNR point s uses data and
 * noise drawn from Philox4x32-10 keyed by `seed` at counter (cw_offset + i),
 * so every SNR point sees the same data and the same noise, scaled by its
 * sigma, as the reference's inner loop does (LDPCtop.cpp:89-97).
 * Outputs (dev):
 *   llr_int or llr_f32 [n_snr][n_per_snr][N]   (either or both: llr_int holds
 *                      elements of the context's type -- int8, int16, int32,
 *                      or double for the LDPC_F64_* variants, the float LLRs
 *                      widened; llr_f32 the float LLRs)
 *   data_bits          [n_per_snr][hard_words] sent data bits (optional)
 *   uncoded_err        [n_snr] sign errors before decoding (optional,
 *                      accumulated: caller zeroes)                         */
int ldpc_generate(ldpc_ctx *ctx, uint64_t seed, uint64_t cw_offset, const float *snr_db, size_t n_snr,
                  size_t n_per_snr, void *llr_int, float *llr_f32, uint32_t *data_bits,
                  unsigned long long *uncoded_err, void *stream);

/* LLR quantisation of given noise (dev): cw_bits [n][N] 0/1 bytes,
 * noise [n][N] float -> llr [n][N] (llr_int in the context's element type,
 * llr_f32 float; float contexts fill llr_f32 only) at one SNR.
 * Bit-exact restatement of gen_metrics(); used for parity checks. */
int ldpc_llr_from_noise(ldpc_ctx *ctx, const uint8_t *cw_bits, const float *noise, size_t n, float snr_db,
                        void *llr_int, float *llr_f32, unsigned long long *uncoded_err, void *stream);

/* QC encoding (dev): data_bits [n][hard_words] packed -> cw_bits [n][N]
 * 0/1 bytes.  Replaces LDPCencode() (LDPCencode.cpp:40-100). */
int ldpc_encode(ldpc_ctx *ctx, const uint32_t *data_bits, size_t n, uint8_t *cw_bits, void *stream);

/* ---- simulation ------------------------------------------------------------ */

/* Per-SNR counters of a simulation run, the reference's per-loop report
 * (LDPCtop.cpp:127-129). */
typedef struct {
    float snr_db;
    unsigned long long codewords;
    unsigned long long iterations;
    unsigned long long bit_errors;
    unsigned long long cw_errors;       /* counted per sub-codeword, LDPC_count_errors.cpp:124-131 */
    unsigned long long uncoded_errors;
    double decode_ms;                   /* device time of the decode kernel */
} ldpc_snr_stats;

/* One outer-loop pass of the reference's simulator (LDPCtop.cpp:86-139) for
 * n_per_snr codewords at each SNR: generate, decode, count errors, on the
 * device.  Codeword counters start at cw_offset, so consecutive calls (or
 * ranks of a multi-GPU run) with different offsets draw disjoint data. */
int ldpc_simulate(ldpc_ctx *ctx, uint64_t seed, uint64_t cw_offset, const float *snr_db, size_t n_snr,
                  size_t n_per_snr, ldpc_snr_stats *stats);

/* Count errors of decoded hard decisions (dev): hard [n][hard_words] against
 * sent data_bits [n % ref_period][hard_words], codeword errors per
 * sub-codeword.  Replaces LDPC_count_errors() (LDPC_count_errors.cpp:40-136).
 * Results accumulate into counters[0..1] = {cw_errors, bit_errors}. */
int ldpc_count_errors(ldpc_ctx *ctx, const uint32_t *hard, size_t n, const uint32_t *data_bits, size_t ref_period,
                      unsigned long long *counters, void *stream);

/* ---- decoding without allocation --------------------------------------------
 *
 * No counterpart in the reference: the reference's decoder runs on the host
 * and never touches device memory.
 *
 * Float decoding (LDPC_F32_SP / LDPC_F32_OMS) that allocates no device
 * memory: no context is needed and nothing is allocated or freed, whatever
 * the code.  It is for callers that cannot allocate at that point:
 *   - their device memory is reserved up front by another allocator;
 *   - cudaFree (and at times cudaMalloc) synchronising the device would stall
 *     their other streams;
 *   - they cannot handle an out-of-memory failure mid-run.
 * ldpc_ctx_create, by contrast, allocates counters and tables, plus a message
 * scratch of tens of MB for large codes.
 *
 * Check messages go to one static 32 MiB array per device, reserved when the
 * library's kernels load there.
 *   - The grid is capped at the number of CTAs the array holds.
 *   - A code that needs more than the whole array for one CTA (edges per
 *     lifted row block x CTA threads x 4 bytes) is rejected with
 *     LDPC_ERR_UNSUPPORTED.
 *   - Nothing in it needs to start at zero.
 *
 * Arguments and outputs are those of ldpc_decode_f32 (dev pointers, async on
 * `stream`), on the CURRENT device; cfg's llr_scale / max_abs_llr are unused.
 *
 * Shared memory and codes accepted are the context path's: any code that
 * ldpc_ctx_create takes for a float variant (5G NR base graph 1 at Z=384 and
 * 802.3ca run without the LLR staging buffer, as there).
 *
 * The first call on each device does the setup: symbol lookup and kernel
 * attributes.  Make it before any stream capture.  Later calls take no lock.
 * After cudaDeviceReset on a device that has used it, do not call it again in
 * that process.  Two calls whose kernels may overlap on the same device race
 * on the shared array: order them (one stream, or events). */
int ldpc_decode_f32_noalloc(const ldpc_code *code, const ldpc_cfg *cfg, const float *llr, size_t n,
                            float *post_out, uint32_t *hard_out, uint8_t *iters_out, void *stream);

/* ---- measurement ----------------------------------------------------------- */

/* Sustained 32-bit integer instruction rate of `device` (ops/s), from a
 * microbenchmark of independent lop3 / iadd chains: the peak against which
 * the decoder's integer-pipe roofline fraction is reported.  No counterpart
 * in the reference (which times with RDTSC only, LDPCtop.cpp:107-114). */
int ldpc_probe_int32_peak(int device, double *ops_per_s);

/* Sustained FP32 fused multiply-add rate and MUFU (ex2.approx) rate of
 * `device` (instructions per second, one per thread per op), from chains of
 * independent operations: the denominators of the float decoders' roofline.
 * No counterpart in the reference. */
int ldpc_probe_fp32_peak(int device, double *fma_per_s, double *mufu_per_s);

/* Thread-level throughput (operations per clock per SM, at the device's
 * reported maximum clock) of single operations on packed lanes: int8x4 and
 * int16x2 SIMD intrinsics, s16x2 / f16x2 / f32 instructions, prmt, lop3 --
 * the measurements behind the int8 decoder's choice of f16x2 arithmetic.
 * Fills the first min(n_ops, 17) entries; names[i] (optional) receives a
 * static string naming operation i.  No counterpart in the reference. */
int ldpc_probe_op_rates(int device, double *ops_per_clk_sm, int n_ops, const char **names);

#ifdef __cplusplus
}
#endif
#endif /* LDPC_B200_H */
