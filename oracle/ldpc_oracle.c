/* ldpc_oracle.c -- scalar CPU restatement of the reference's LDPC hot path.
 * TEST INFRASTRUCTURE ONLY (see ldpc_oracle.h).  Parity pinned against the
 * reference's own decoder sources built in oracle/_ref (tests/test_oracle.py).
 */
#include "ldpc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ldpc_math.h"

/* ---- int8 element semantics of the reference's Vec64c operations ---- */
static int8_t sat8(int v) { return (int8_t)(v < -128 ? -128 : v > 127 ? 127 : v); }
static int8_t wrap8(int v) { return (int8_t)(uint8_t)(v & 0xff); }
/* vectorclass abs(): the most negative value maps to itself */
static int8_t abs8(int8_t q) { return q < 0 ? wrap8(-(int)q) : q; }

/* decode_row's Max_row_simd (decode_functions.cpp:27-32) for an int8 build */
static int8_t max_row_i8(float max_row_metric) {
    if (max_row_metric < 1e-6) return (int8_t)(1.0 - (double)(int8_t)max_row_metric);
    return (int8_t)max_row_metric;
}
static float max_row_f32(float max_row_metric) {
    if (max_row_metric < 1e-6) return (float)(1.0 - (double)max_row_metric);
    return max_row_metric;
}

static int total_edges(const orc_code *c) {
    int e = 0;
    for (int r = 0; r < c->mrow; ++r) e += c->row_weights[r];
    return e;
}

static int max_weight(const orc_code *c) {
    int m = 0;
    for (int r = 0; r < c->mrow; ++r) if (c->row_weights[r] > m) m = c->row_weights[r];
    return m;
}

/* Evaluate a tree program (trees.py flat format) on the row's inputs.
 * kind: 0 = int8 min, 1 = float min, 2 = float product.  */
static void run_tree_i8(const int32_t *prog, int len, int d, const int8_t *in, int8_t maxv, int8_t *node, int8_t *out) {
    for (int j = 0; j < d; ++j) node[j] = in[j];
    for (int k = 0; k < len; ++k) {
        const int32_t *q = prog + 4 * k;
        if (q[0] == 0) node[q[1]] = node[q[2]] < node[q[3]] ? node[q[2]] : node[q[3]];
        else if (q[0] == 1) node[q[1]] = maxv < node[q[1]] ? maxv : node[q[1]];
        else out[q[1]] = node[q[2]];
    }
}

static void run_tree_f32(const int32_t *prog, int len, int d, int prod, const float *in, float maxv, float *node, float *out) {
    for (int j = 0; j < d; ++j) node[j] = in[j];
    for (int k = 0; k < len; ++k) {
        const int32_t *q = prog + 4 * k;
        if (q[0] == 0) {
            float a = node[q[2]], b = node[q[3]];
            node[q[1]] = prod ? a * b : (a < b ? a : b);
        } else if (q[0] == 1) {
            node[q[1]] = maxv < node[q[1]] ? maxv : node[q[1]];
        } else {
            out[q[1]] = node[q[2]];
        }
    }
}

/* the int8 program for weight d: reuse the float program layout passed in by
 * the caller (same schedule) */
static const orc_trees *g_trees_i8 = 0;

/* int8 layered offset min-sum with offset beta8[r] on layer r (the
 * reference's decoder has one offset for every layer; per-layer offsets are
 * the learned-offset extension). */
/* int8 decoding with an offset table beta_tab[rows][mrow]: iteration i
 * (0-based) of a codeword uses row min(i, rows - 1).  One row is one offset
 * per layer; the reference's single beta is one row of equal values. */
int orc_decode_int8_table(const orc_code *c, const int8_t *llr, size_t n_cw, unsigned max_iter,
                          float max_row_metric, const int8_t *beta_tab, int rows, int8_t *post_out,
                          uint32_t *iters_out) {
    const int z = c->z, n = z * c->mcol, E = total_edges(c), dmax = max_weight(c);
    const int8_t maxv = max_row_i8(max_row_metric);
    int8_t *P = (int8_t *)malloc((size_t)n);
    int8_t *R = (int8_t *)malloc((size_t)E * z);
    int8_t *Q = (int8_t *)malloc((size_t)dmax), *m = (int8_t *)malloc((size_t)dmax);
    int8_t *f = (int8_t *)malloc((size_t)dmax), *node = (int8_t *)malloc((size_t)dmax * 8 + 64);
    int *v = (int *)malloc(sizeof(int) * (size_t)dmax);
    for (size_t cw = 0; cw < n_cw; ++cw) {
        memcpy(P, llr + cw * (size_t)n, (size_t)n);
        memset(R, 0, (size_t)E * z);
        unsigned iter = 0;
        int done = 0;
        while (!done) {
            int e0 = 0;
            for (int r = 0; r < c->mrow; ++r) {
                const int d = c->row_weights[r];
                const int row = (int)iter < rows ? (int)iter : rows - 1;
                const int8_t beta8 = beta_tab[(size_t)row * c->mrow + r];
                for (int t = 0; t < z; ++t) {
                    int8_t rx = 0;
                    for (int j = 0; j < d; ++j) {
                        const int col = c->row_cols[e0 + j], s = c->row_shifts[e0 + j];
                        v[j] = col * z + (s + t) % z;
                        Q[j] = sat8((int)P[v[j]] - (int)R[(size_t)(e0 + j) * z + t]);
                        int8_t a = wrap8((int)abs8(Q[j]) - (int)beta8);
                        m[j] = a > 0 ? a : 0;
                        rx ^= Q[j];
                    }
                    if (g_trees_i8) {
                        run_tree_i8(g_trees_i8->prog + 4 * g_trees_i8->off[d], g_trees_i8->len[d], d, m, maxv, node, f);
                    } else {
                        for (int j = 0; j < d; ++j) {
                            int8_t mn = maxv;
                            for (int k = 0; k < d; ++k) if (k != j && m[k] < mn) mn = m[k];
                            f[j] = mn;
                        }
                    }
                    for (int j = 0; j < d; ++j) {
                        int8_t s = (int8_t)(rx ^ Q[j]);
                        int8_t rn = s < 0 ? wrap8(-(int)f[j]) : f[j];
                        P[v[j]] = sat8((int)Q[j] + (int)rn);
                        R[(size_t)(e0 + j) * z + t] = rn;
                    }
                }
                e0 += d;
            }
            /* syndrome on the posteriors after the full iteration */
            int bad = 0;
            e0 = 0;
            for (int r = 0; r < c->mrow && !bad; ++r) {
                const int d = c->row_weights[r];
                for (int t = 0; t < z; ++t) {
                    int8_t x = 0;
                    for (int j = 0; j < d; ++j) x ^= P[c->row_cols[e0 + j] * z + (c->row_shifts[e0 + j] + t) % z];
                    if (x < 0) { bad = 1; break; }
                }
                e0 += d;
            }
            ++iter;
            done = !bad || iter == max_iter;
        }
        if (post_out) memcpy(post_out + cw * (size_t)n, P, (size_t)n);
        if (iters_out) iters_out[cw] = iter;
    }
    free(P); free(R); free(Q); free(m); free(f); free(node); free(v);
    return 0;
}

int orc_decode_int8_layers(const orc_code *c, const int8_t *llr, size_t n_cw, unsigned max_iter,
                           float max_row_metric, const int8_t *beta_layer, int8_t *post_out, uint32_t *iters_out) {
    return orc_decode_int8_table(c, llr, n_cw, max_iter, max_row_metric, beta_layer, 1, post_out, iters_out);
}

int orc_decode_int8(const orc_code *c, const int8_t *llr, size_t n_cw, unsigned max_iter,
                    float max_row_metric, float beta, int8_t *post_out, uint32_t *iters_out) {
    int8_t *b = (int8_t *)malloc((size_t)(c->mrow > 0 ? c->mrow : 1));
    for (int r = 0; r < c->mrow; ++r) b[r] = (int8_t)beta;   /* implicit float -> int truncation, decode_functions.cpp:60 */
    const int rc = orc_decode_int8_layers(c, llr, n_cw, max_iter, max_row_metric, b, post_out, iters_out);
    free(b);
    return rc;
}

static uint32_t fbits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static float bitsf(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

int orc_decode_f32(const orc_code *c, const orc_trees *tr, int mode, const float *llr, size_t n_cw,
                   unsigned max_iter, float max_row_metric, float beta, float *post_out, uint32_t *iters_out) {
    const int z = c->z, n = z * c->mcol, E = total_edges(c), dmax = max_weight(c);
    const float maxv = max_row_f32(max_row_metric);
    if (dmax > tr->max_d) return -1;
    float *P = (float *)malloc(sizeof(float) * (size_t)n);
    float *R = (float *)malloc(sizeof(float) * (size_t)E * z);
    float *Q = (float *)malloc(sizeof(float) * (size_t)dmax), *x = (float *)malloc(sizeof(float) * (size_t)dmax);
    float *f = (float *)malloc(sizeof(float) * (size_t)dmax), *node = (float *)malloc(sizeof(float) * ((size_t)dmax * 8 + 64));
    int *v = (int *)malloc(sizeof(int) * (size_t)dmax);
    for (size_t cw = 0; cw < n_cw; ++cw) {
        memcpy(P, llr + cw * (size_t)n, sizeof(float) * (size_t)n);
        memset(R, 0, sizeof(float) * (size_t)E * z);
        unsigned iter = 0;
        int done = 0;
        while (!done) {
            int e0 = 0;
            for (int r = 0; r < c->mrow; ++r) {
                const int d = c->row_weights[r];
                for (int t = 0; t < z; ++t) {
                    uint32_t rx = 0;
                    for (int j = 0; j < d; ++j) {
                        const int col = c->row_cols[e0 + j], s = c->row_shifts[e0 + j];
                        v[j] = col * z + (s + t) % z;
                        Q[j] = P[v[j]] - R[(size_t)(e0 + j) * z + t];
                        float a = fabsf(Q[j]) - beta;
                        a = a > 0.0f ? a : 0.0f;
                        x[j] = mode == 1 ? lm_tanh(a * 0.5f) : mode == 2 ? (float)tanh((double)(a * 0.5f)) : a;
                        rx ^= fbits(Q[j]);
                    }
                    run_tree_f32(tr->prog + 4 * tr->off[d], tr->len[d], d, mode != 0, x, maxv, node, f);
                    for (int j = 0; j < d; ++j) {
                        float fj = mode == 1 ? 2.0f * lm_atanh(f[j]) : mode == 2 ? 2.0f * (float)atanh((double)f[j]) : f[j];
                        uint32_t s = rx ^ fbits(Q[j]);
                        float rn = (s & 0x80000000u) ? bitsf(fbits(fj) ^ 0x80000000u) : fj;
                        P[v[j]] = Q[j] + rn;
                        R[(size_t)(e0 + j) * z + t] = rn;
                    }
                }
                e0 += d;
            }
            int bad = 0;
            e0 = 0;
            for (int r = 0; r < c->mrow && !bad; ++r) {
                const int d = c->row_weights[r];
                for (int t = 0; t < z; ++t) {
                    uint32_t xx = 0;
                    for (int j = 0; j < d; ++j) xx ^= fbits(P[c->row_cols[e0 + j] * z + (c->row_shifts[e0 + j] + t) % z]);
                    if (xx & 0x80000000u) { bad = 1; break; }
                }
                e0 += d;
            }
            ++iter;
            done = !bad || iter == max_iter;
        }
        if (post_out) memcpy(post_out + cw * (size_t)n, P, sizeof(float) * (size_t)n);
        if (iters_out) iters_out[cw] = iter;
    }
    free(P); free(R); free(Q); free(x); free(f); free(node); free(v);
    return 0;
}

/* The float decoder in double precision: the reference's SIMD_ELEM_BW=-64
 * builds (LDPCtop_Vec8d_prod / Vec8d_min).  decode_row's operations are
 * unchanged, on double lanes: Q = P - R, a = max(|Q| - (double)beta, 0)
 * (decode_functions.cpp:53-62), tanh(a * 0.5) (min_find.pl:38), the product
 * or min tree with the clamp min(Max_val, .) at Max_val = 1.0 -
 * (double)max_row_metric below 1e-6 else (double)max_row_metric
 * (decode_functions.cpp:27-32, min_find.pl:99-107), 2.0 * atanh(.)
 * (min_find.pl:44), sign_combine and P = Q + R' (:85-91).  tanh/atanh are the
 * shared lmd_tanh / lmd_atanh. */
static uint64_t dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static double bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

static void run_tree_f64(const int32_t *prog, int len, int d, int prod, const double *in, double maxv, double *node,
                         double *out) {
    for (int j = 0; j < d; ++j) node[j] = in[j];
    for (int k = 0; k < len; ++k) {
        const int32_t *q = prog + 4 * k;
        if (q[0] == 0) {
            double a = node[q[2]], b = node[q[3]];
            node[q[1]] = prod ? a * b : (a < b ? a : b);
        } else if (q[0] == 1) {
            node[q[1]] = maxv < node[q[1]] ? maxv : node[q[1]];
        } else {
            out[q[1]] = node[q[2]];
        }
    }
}

int orc_decode_f64(const orc_code *c, const orc_trees *tr, int mode, const double *llr, size_t n_cw,
                   unsigned max_iter, float max_row_metric, float beta, double *post_out, uint32_t *iters_out) {
    const int z = c->z, n = z * c->mcol, E = total_edges(c), dmax = max_weight(c);
    const double maxv = max_row_metric < 1e-6 ? 1.0 - (double)max_row_metric : (double)max_row_metric;
    const double b = (double)beta;
    if (dmax > tr->max_d) return -1;
    double *P = (double *)malloc(sizeof(double) * (size_t)n);
    double *R = (double *)malloc(sizeof(double) * (size_t)E * z);
    double *Q = (double *)malloc(sizeof(double) * (size_t)dmax), *x = (double *)malloc(sizeof(double) * (size_t)dmax);
    double *f = (double *)malloc(sizeof(double) * (size_t)dmax);
    double *node = (double *)malloc(sizeof(double) * ((size_t)dmax * 8 + 64));
    int *v = (int *)malloc(sizeof(int) * (size_t)dmax);
    for (size_t cw = 0; cw < n_cw; ++cw) {
        memcpy(P, llr + cw * (size_t)n, sizeof(double) * (size_t)n);
        memset(R, 0, sizeof(double) * (size_t)E * z);
        unsigned iter = 0;
        int done = 0;
        while (!done) {
            int e0 = 0;
            for (int r = 0; r < c->mrow; ++r) {
                const int d = c->row_weights[r];
                for (int t = 0; t < z; ++t) {
                    uint64_t rx = 0;
                    for (int j = 0; j < d; ++j) {
                        const int col = c->row_cols[e0 + j], s = c->row_shifts[e0 + j];
                        v[j] = col * z + (s + t) % z;
                        Q[j] = P[v[j]] - R[(size_t)(e0 + j) * z + t];
                        double a = fabs(Q[j]) - b;
                        a = a > 0.0 ? a : 0.0;
                        x[j] = mode == 1 ? lmd_tanh(a * 0.5) : mode == 2 ? tanh(a * 0.5) : a;
                        rx ^= dbits(Q[j]);
                    }
                    run_tree_f64(tr->prog + 4 * tr->off[d], tr->len[d], d, mode != 0, x, maxv, node, f);
                    for (int j = 0; j < d; ++j) {
                        double fj = mode == 1 ? 2.0 * lmd_atanh(f[j]) : mode == 2 ? 2.0 * atanh(f[j]) : f[j];
                        uint64_t s = (rx ^ dbits(Q[j])) & 0x8000000000000000ULL;
                        double rn = bitsd(dbits(fj) ^ s);
                        P[v[j]] = Q[j] + rn;
                        R[(size_t)(e0 + j) * z + t] = rn;
                    }
                }
                e0 += d;
            }
            int bad = 0;
            e0 = 0;
            for (int r = 0; r < c->mrow && !bad; ++r) {
                const int d = c->row_weights[r];
                for (int t = 0; t < z; ++t) {
                    uint64_t xx = 0;
                    for (int j = 0; j < d; ++j) xx ^= dbits(P[c->row_cols[e0 + j] * z + (c->row_shifts[e0 + j] + t) % z]);
                    if (xx & 0x8000000000000000ULL) { bad = 1; break; }
                }
                e0 += d;
            }
            ++iter;
            done = !bad || iter == max_iter;
        }
        if (post_out) memcpy(post_out + cw * (size_t)n, P, sizeof(double) * (size_t)n);
        if (iters_out) iters_out[cw] = iter;
    }
    free(P); free(R); free(Q); free(x); free(f); free(node); free(v);
    return 0;
}

/* int8 decoding through the generated min tree instead of the direct
 * exclusive minimum (identical by exactness of integer min; kept to check it) */
int orc_decode_int8_tree(const orc_code *c, const orc_trees *tr, const int8_t *llr, size_t n_cw,
                         unsigned max_iter, float max_row_metric, float beta, int8_t *post_out,
                         uint32_t *iters_out) {
    g_trees_i8 = tr;
    int rc = orc_decode_int8(c, llr, n_cw, max_iter, max_row_metric, beta, post_out, iters_out);
    g_trees_i8 = 0;
    return rc;
}

void orc_sigma(float snr, float llr_scale, float *sigma, float *sigma_factor) {
    float three_db = 10 * log10f(2.0);
    float s = powf(10.0, ((snr + three_db) / -20.0));
    *sigma = s;
    *sigma_factor = 2 * llr_scale / (s * s);
}

int orc_llr(int bit, float noise, float sigma, float sigma_factor, float max_abs, int punct, int filler,
            float *llr_f, int32_t *llr_i) {
    float orig = bit ? -1.0f : 1.0f;
    float rx = fmaf(noise, sigma, orig);
    int err = (int)((fbits(orig) ^ fbits(rx)) >> 31);
    float l = rx * sigma_factor;
    l = max_abs < l ? max_abs : l;
    l = -max_abs > l ? -max_abs : l;
    if (punct) l = 0.0f;
    if (filler) l = max_abs;
    if (llr_f) *llr_f = l;
    if (llr_i) *llr_i = (int32_t)nearbyintf(l);
    return err;
}

void orc_encode(int z, int mcol, int mrow, const int32_t *sched, int n_par, const uint8_t *info,
                size_t n_cw, uint8_t *cw) {
    const int kc = mcol - mrow, n = z * mcol;
    uint8_t *acc = (uint8_t *)malloc((size_t)z);
    for (size_t w = 0; w < n_cw; ++w) {
        uint8_t *x = cw + w * (size_t)n;
        memset(x, 0, (size_t)n);
        memcpy(x, info + w * (size_t)kc * z, (size_t)kc * z);
        const int32_t *p = sched;
        for (int k = 0; k < n_par; ++k) {
            int pc = p[0], cnt = p[1];
            memset(acc, 0, (size_t)z);
            for (int i = 0; i < cnt; ++i) {
                int col = p[2 + 2 * i], sh = p[3 + 2 * i];
                for (int t = 0; t < z; ++t) acc[t] ^= x[col * z + (t + sh) % z];
            }
            memcpy(x + pc * z, acc, (size_t)z);
            p += 2 + 2 * cnt;
        }
    }
    free(acc);
}

static void count_core(int z, int mcol, int mrow, int num_par, const uint8_t *hard, const uint8_t *sent,
                       uint64_t *cw_err, uint64_t *bit_err) {
    int slot_err[64];
    uint64_t bits = 0;
    memset(slot_err, 0, sizeof(slot_err));
    for (int c = 0; c < mcol - mrow; ++c)
        for (int t = 0; t < z; ++t)
            if (hard[c * z + t] != sent[c * z + t]) { ++bits; slot_err[t % num_par] = 1; }
    if (bits) {
        for (int p = 0; p < num_par; ++p) *cw_err += (uint64_t)slot_err[p];
        *bit_err += bits;
    }
}

void orc_count_errors_i8(int z, int mcol, int mrow, int num_par, const int8_t *post, const uint8_t *cw_bits,
                         size_t n_cw, uint64_t *cw_err, uint64_t *bit_err) {
    const int n = z * mcol;
    uint8_t *hard = (uint8_t *)malloc((size_t)n);
    *cw_err = 0; *bit_err = 0;
    for (size_t w = 0; w < n_cw; ++w) {
        for (int i = 0; i < n; ++i) hard[i] = post[w * (size_t)n + i] < 0;
        count_core(z, mcol, mrow, num_par, hard, cw_bits + w * (size_t)n, cw_err, bit_err);
    }
    free(hard);
}

void orc_count_errors_f32(int z, int mcol, int mrow, int num_par, const float *post, const uint8_t *cw_bits,
                          size_t n_cw, uint64_t *cw_err, uint64_t *bit_err) {
    const int n = z * mcol;
    uint8_t *hard = (uint8_t *)malloc((size_t)n);
    *cw_err = 0; *bit_err = 0;
    for (size_t w = 0; w < n_cw; ++w) {
        for (int i = 0; i < n; ++i) hard[i] = post[w * (size_t)n + i] < 0.0f;
        count_core(z, mcol, mrow, num_par, hard, cw_bits + w * (size_t)n, cw_err, bit_err);
    }
    free(hard);
}

int64_t orc_llr_array(const uint8_t *bits, const float *noise, size_t total, int n, const uint8_t *punct,
                      const uint8_t *filler, float snr, float llr_scale, float max_abs, float *llr_f, int8_t *llr_i8) {
    float sigma, sf;
    int64_t errs = 0;
    orc_sigma(snr, llr_scale, &sigma, &sf);
    for (size_t e = 0; e < total; ++e) {
        const int idx = (int)(e % (size_t)n);
        float l;
        int32_t li;
        errs += orc_llr(bits[e] & 1, noise[e], sigma, sf, max_abs, punct ? punct[idx] : 0, filler ? filler[idx] : 0, &l, &li);
        if (llr_f) llr_f[e] = l;
        if (llr_i8) llr_i8[e] = (int8_t)(int16_t)li;
    }
    return errs;
}

/* The shared tanh / atanh over arrays, so that tests can measure their error
 * against the C library's long-double functions. */
void orc_lm_tanh_array(const float *x, float *y, size_t n) { for (size_t i = 0; i < n; ++i) y[i] = lm_tanh(x[i]); }
void orc_lm_atanh_array(const float *x, float *y, size_t n) { for (size_t i = 0; i < n; ++i) y[i] = lm_atanh(x[i]); }
void orc_lmd_tanh_array(const double *x, double *y, size_t n) { for (size_t i = 0; i < n; ++i) y[i] = lmd_tanh(x[i]); }
void orc_lmd_atanh_array(const double *x, double *y, size_t n) { for (size_t i = 0; i < n; ++i) y[i] = lmd_atanh(x[i]); }

/* Largest error, in units in the last place of float, of the shared float
 * tanh (kind 0) or atanh (kind 1) against the C library's long-double
 * tanhl / atanhl, over the non-negative floats whose bit patterns run from
 * lo_bits to hi_bits (inclusive) in steps of `stride`.  The ulp of a true
 * value v is 2^(floor(log2 |v|) - 23).  Returns the input with the largest
 * error in *argmax. */
double orc_ulp_scan_f32(int kind, uint32_t lo_bits, uint32_t hi_bits, uint32_t stride, float *argmax) {
    double worst = 0.0;
    float wx = 0.0f;
    for (uint64_t b = lo_bits; b <= hi_bits; b += stride) {
        const float x = bitsf((uint32_t)b);
        const float y = kind ? lm_atanh(x) : lm_tanh(x);
        const long double v = kind ? atanhl((long double)x) : tanhl((long double)x);
        double u = 0.0;
        if (v != 0.0L) {
            int e;
            frexpl(v, &e);                               /* |v| in [2^(e-1), 2^e) */
            const long double ulp = ldexpl(1.0L, e - 1 - 23);
            u = (double)(fabsl((long double)y - v) / ulp);
        } else if (y != 0.0f) {
            u = INFINITY;
        }
        if (u > worst) { worst = u; wx = x; }
    }
    if (argmax) *argmax = wx;
    return worst;
}
