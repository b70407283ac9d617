/* ref_shim.cpp -- extern "C" entry points over the reference's own C++
 * functions, for the oracle and the CPU baseline (test infrastructure).
 *
 * Linked with the reference's unmodified sources (src/LDPCDec, src/LDPCEnc,
 * src/RNGfunc, src/Top) compiled against oracle/vcl_compat.  Each wrapper
 * calls exactly one reference function; the prototypes are the ones in
 * src/Top/LDPCtop.cpp:26-39.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "vectorclass.h"
#include "simd_defs.h"
#include "enc_defs.h"
#include "dec_struct_LDPC.h"
#include "enc_struct_LDPC.h"

typedef void (*min_fn_ptr_type)(SIMD_CLASS *, SIMD_CLASS *, SIMD_CLASS, int);
extern min_fn_ptr_type *all_minprod_func_ary;

void init_randstate(uint64_t *inp);
void encode_matrix_allocate(const char *, struct Henc_struct *, unsigned);
void decode_matrix_allocate(const char *filename, struct Hdec_struct *H, unsigned num_cw);
void normdist2(Vec8f *result, int simd_count);
void gen_rand_databits(unsigned num_codeword, struct Henc_struct *Henc);
void LDPCencode(const int num_codewords, struct Henc_struct H);
unsigned gen_metrics(unsigned num_codeword, float SNR, unsigned char *enc_cw_byteptr, int z_value, int mcol,
                     Vec8f *wgn_fltptr, SIMD_CLASS *simd_metric_ptr, float LLR_scaling_factor, float max_abs_LLR,
                     ENC_CLASS *puncture_mask, ENC_CLASS *filler_mask);
unsigned LDPCdecode_set(unsigned num_codeword, unsigned max_iter, float max_row_metric, float beta_offset,
                        struct Hdec_struct *Hdec, min_fn_ptr_type *min_funcs);
void LDPC_count_errors(unsigned num_codeword, struct Henc_struct *Henc, struct Hdec_struct *Hdec,
                       unsigned *tot_cw_err, unsigned *tot_bit_err);

struct RefCtx {
    Henc_struct enc;
    Hdec_struct dec;
    unsigned num_cw;
};

extern "C" {

/* layout of this build: SIMD_PAR, element bytes (negative = float), bytes per SIMD word */
void ref_layout(int *simd_par, int *elem_bw, int *width_bytes, int *enc_bytes) {
    *simd_par = SIMD_PAR;
    *elem_bw = SIMD_ELEM_BW;
    *width_bytes = WIDTH / 8;
    *enc_bytes = ENC_BW / 8;
}

void *ref_open(const char *enc_path, const char *dec_path, unsigned num_cw) {
    RefCtx *c = (RefCtx *)calloc(1, sizeof(RefCtx));
    encode_matrix_allocate(enc_path, &c->enc, num_cw);
    decode_matrix_allocate(dec_path, &c->dec, num_cw);
    c->num_cw = num_cw;
    /* The reference's mirror copies (LDPCdecode.cpp:133-150) store whole SIMD
     * words at unaligned offsets, and the last one of the buffer can end past
     * the allocation of decode_matrix_allocate.cpp:55 (seen with the int16
     * build at Z=24: 2 bytes over).  Decode into a copy with two spare
     * columns behind it, so such a store lands in slack instead of the heap. */
    unsigned spz = (c->dec.z_value + SIMD_PAR - 1) / SIMD_PAR;
    const size_t bytes = (size_t)num_cw * c->dec.mcol * (spz + 2) * (WIDTH / 8);
    const size_t slack = (size_t)2 * (spz + 2) * (WIDTH / 8);
    _mm_free(c->dec.decoded_metrics);
    c->dec.decoded_metrics = (SIMD_CLASS *)_mm_malloc(bytes + slack, WIDTH / 8);
    /* zero the codeword and metric buffers (the reference leaves them uninitialised) */
    memset(c->dec.decoded_metrics, 0, bytes + slack);
    memset(c->enc.cw_bits, 0, (size_t)num_cw * c->enc.mcol * sizeof(ENC_CLASS));
    return c;
}

void ref_dims(void *h, unsigned *z, unsigned *mrow, unsigned *mcol, unsigned *num_par, unsigned *fill_cnt) {
    RefCtx *c = (RefCtx *)h;
    *z = c->dec.z_value;
    *mrow = c->dec.mrow;
    *mcol = c->dec.mcol;
    *num_par = c->enc.num_par_cw;
    *fill_cnt = c->enc.filler_cnt;
}

void *ref_metrics(void *h) { return ((RefCtx *)h)->dec.decoded_metrics; }
void *ref_cw_bits(void *h) { return ((RefCtx *)h)->enc.cw_bits; }

/* LDPCdecode_set over codewords [first, first+count) of the context buffer */
unsigned ref_decode_set(void *h, unsigned first, unsigned count, unsigned max_iter,
                        float max_row_metric, float beta) {
    RefCtx *c = (RefCtx *)h;
    unsigned spz = (c->dec.z_value + SIMD_PAR - 1) / SIMD_PAR;
    SIMD_CLASS *base = c->dec.decoded_metrics;
    c->dec.decoded_metrics = base + (size_t)first * c->dec.mcol * (spz + 2);
    unsigned it = LDPCdecode_set(count, max_iter, max_row_metric, beta, &c->dec, all_minprod_func_ary);
    c->dec.decoded_metrics = base;
    return it;
}

/* one LDPCdecode_set call per codeword, to expose per-codeword iteration counts */
unsigned ref_decode_each(void *h, unsigned count, unsigned max_iter, float max_row_metric, float beta,
                         uint32_t *iters_out) {
    unsigned tot = 0;
    for (unsigned i = 0; i < count; ++i) {
        unsigned it = ref_decode_set(h, i, 1, max_iter, max_row_metric, beta);
        if (iters_out) iters_out[i] = it;
        tot += it;
    }
    return tot;
}

void ref_init_randstate(uint64_t *seeds64) { init_randstate(seeds64); }
void ref_normdist2(float *out, int simd_count) { normdist2((Vec8f *)out, simd_count); }
void ref_gen_rand_databits(void *h, unsigned n) { gen_rand_databits(n, &((RefCtx *)h)->enc); }
void ref_encode(void *h, unsigned n) { LDPCencode((int)n, ((RefCtx *)h)->enc); }

unsigned ref_gen_metrics(void *h, unsigned n, float snr, const float *wgn, float scale, float max_abs) {
    RefCtx *c = (RefCtx *)h;
    return gen_metrics(n, snr, (unsigned char *)c->enc.cw_bits, c->enc.z_value, c->enc.mcol,
                       (Vec8f *)wgn, c->dec.decoded_metrics + 1, scale, max_abs,
                       c->enc.puncture_mask, c->enc.filler_mask);
}

void ref_count_errors(void *h, unsigned n, unsigned *cw_err, unsigned *bit_err) {
    RefCtx *c = (RefCtx *)h;
    LDPC_count_errors(n, &c->enc, &c->dec, cw_err, bit_err);
}

} /* extern "C" */
