/* ldpc_oracle.h -- scalar CPU restatement of the reference's LDPC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the correctness oracle for the B200
 * kernels; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The shipped library never links or calls it.
 *
 * Each function restates one reference routine, lane by lane, with plain
 * circulant indexing (check t of a layer touches bit (t + s) mod Z of every
 * active column) in place of the reference's SIMD mirror copies:
 *   orc_decode_int8  src/LDPCDec/LDPCdecode.cpp:79-201 + decode_functions.cpp:11-137
 *                    (SIMD_ELEM_BW=8, USE_BETA_OFFSET=1, USE_SAT_ADD_SUB=1)
 *   orc_decode_f32   same, SIMD_ELEM_BW=-32 (min or prod tree, min_find.pl)
 *   orc_llr          src/Top/gen_metrics.cpp:18-121 for one element
 *   orc_encode       src/LDPCEnc/LDPCencode.cpp:40-100 (XOR of rotated columns)
 *   orc_count_errors src/Top/LDPC_count_errors.cpp:40-136
 */
#ifndef LDPC_ORACLE_H
#define LDPC_ORACLE_H
#include <stddef.h>
#include <stdint.h>

typedef struct {
    int z, mrow, mcol;
    const int32_t *row_weights;  /* [mrow] */
    const int32_t *row_cols;     /* [sum row_weights] */
    const int32_t *row_shifts;   /* [sum row_weights], 0 <= s < z */
} orc_code;

/* Tree programs for the float check update, indexed by row weight d:
 * prog + off[d] holds len[d] int32 quadruples (see ldpc_b200/trees.py). */
typedef struct {
    const int32_t *prog;
    const int32_t *off;
    const int32_t *len;
    int max_d;
} orc_trees;

/* orc_decode_int8 with an offset table beta_tab[rows][mrow] (int8):
 * iteration i of a codeword uses row min(i, rows - 1) */
int orc_decode_int8_table(const orc_code *c, const int8_t *llr, size_t n_cw, unsigned max_iter,
                          float max_row_metric, const int8_t *beta_tab, int rows, int8_t *post_out,
                          uint32_t *iters_out);
/* orc_decode_int8 with one offset per layer (beta_layer[mrow], int8) */
int orc_decode_int8_layers(const orc_code *c, const int8_t *llr, size_t n_cw, unsigned max_iter,
                           float max_row_metric, const int8_t *beta_layer, int8_t *post_out, uint32_t *iters_out);
int orc_decode_int8(const orc_code *c, const int8_t *llr, size_t n_cw, unsigned max_iter,
                    float max_row_metric, float beta, int8_t *post_out, uint32_t *iters_out);

/* same decoder, evaluating the reference's generated min tree (min_find.pl)
 * for the exclusive minimum instead of the direct formula */
int orc_decode_int8_tree(const orc_code *c, const orc_trees *t, const int8_t *llr, size_t n_cw,
                         unsigned max_iter, float max_row_metric, float beta, int8_t *post_out,
                         uint32_t *iters_out);

/* mode 0 = min-sum tree, 1 = sum-product (tanh/atanh) tree with the shared
 * ldpc_math.h functions (what the GPU runs), 2 = sum-product with the C
 * library's tanh/atanh evaluated in double and rounded to float: an
 * independent transcendental, for reporting how far the shared one moves the
 * decode (not bit parity) */
int orc_decode_f32(const orc_code *c, const orc_trees *t, int mode, const float *llr, size_t n_cw,
                   unsigned max_iter, float max_row_metric, float beta, float *post_out,
                   uint32_t *iters_out);

/* the same decoder in double precision (the reference's Vec8d builds);
 * mode 2 = the C library's double tanh/atanh */
int orc_decode_f64(const orc_code *c, const orc_trees *t, int mode, const double *llr, size_t n_cw,
                   unsigned max_iter, float max_row_metric, float beta, double *post_out,
                   uint32_t *iters_out);

/* the shared tanh / atanh (ldpc_math.h) elementwise over arrays */
void orc_lm_tanh_array(const float *x, float *y, size_t n);
void orc_lm_atanh_array(const float *x, float *y, size_t n);
void orc_lmd_tanh_array(const double *x, double *y, size_t n);
void orc_lmd_atanh_array(const double *x, double *y, size_t n);

/* largest ulp error of the shared float tanh (kind 0) / atanh (kind 1)
 * against long-double tanhl / atanhl over float bit patterns lo..hi, step stride */
double orc_ulp_scan_f32(int kind, uint32_t lo_bits, uint32_t hi_bits, uint32_t stride, float *argmax);

/* sigma and LLR factor exactly as gen_metrics.cpp:26-30 computes them */
void orc_sigma(float snr, float llr_scale, float *sigma, float *sigma_factor);

/* one gen_metrics element: bit (0/1), noise sample, flags -> LLR (float and int);
 * returns 1 when the received sign differs from the sent one */
int orc_llr(int bit, float noise, float sigma, float sigma_factor, float max_abs, int punct,
            int filler, float *llr_f, int32_t *llr_i);

/* orc_llr over [total] elements of codewords of n bits (masks indexed by
 * element % n, may be NULL); returns the uncoded error count */
int64_t orc_llr_array(const uint8_t *bits, const float *noise, size_t total, int n, const uint8_t *punct,
                      const uint8_t *filler, float snr, float llr_scale, float max_abs, float *llr_f, int8_t *llr_i8);

/* encode: info [n][K_cols*z] bits (0/1) -> cw [n][mcol*z] bits;
 * sched = (parity col, n terms, (col, shift) * n) records, n_par records */
void orc_encode(int z, int mcol, int mrow, const int32_t *sched, int n_par, const uint8_t *info,
                size_t n_cw, uint8_t *cw);

/* hard decisions (post < 0) on the data columns vs sent bits; codeword
 * errors counted per interleaved sub-codeword (slot = bit index mod num_par) */
void orc_count_errors_i8(int z, int mcol, int mrow, int num_par, const int8_t *post, const uint8_t *cw_bits,
                         size_t n_cw, uint64_t *cw_err, uint64_t *bit_err);
void orc_count_errors_f32(int z, int mcol, int mrow, int num_par, const float *post, const uint8_t *cw_bits,
                          size_t n_cw, uint64_t *cw_err, uint64_t *bit_err);

#endif
