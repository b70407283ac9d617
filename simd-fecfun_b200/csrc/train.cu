// Host side of the learned-offset decoder: forward with checkpoints,
// adjoint, and evaluation with early exit.
#include <algorithm>
#include <cstring>

#include "internal.h"
#include "train.cuh"

using ldpc::fail;

namespace {

typedef void (*train_fn)(const ldpc::SpTables, const ldpc::TrainJob);

struct TrainKernels {
    int dmax;
    train_fn fwd, bwd;
};
const TrainKernels kTrain[] = {{8, ldpc::oms_train_fwd<8>, ldpc::oms_train_bwd<8>},
                               {16, ldpc::oms_train_fwd<16>, ldpc::oms_train_bwd<16>},
                               {32, ldpc::oms_train_fwd<32>, ldpc::oms_train_bwd<32>}};

constexpr int kTrainMaxSmem = 220 * 1024;

struct Geometry {
    train_fn k;
    int threads, smem, grid;
};

int geometry(ldpc_ctx* x, size_t n, bool backward, Geometry* g) {
    if (!x) return fail(LDPC_ERR_INVALID_ARG, "ctx is NULL");
    if (x->cfg.variant != LDPC_F32_OMS)
        return fail(LDPC_ERR_INVALID_ARG, "the learned-offset decoder needs a float offset min-sum context");
    const ldpc::SpTables& t = x->spt;
    const int d = x->code.max_row_weight;
    const TrainKernels* tk = nullptr;
    for (const TrainKernels& k : kTrain)
        if (d <= k.dmax) {
            tk = &k;
            break;
        }
    if (!tk) return fail(LDPC_ERR_UNSUPPORTED, "learned decoder: row weight %d > 32", d);
    const size_t n4 = (size_t)((t.n + 3) & ~3), ez4 = (size_t)((t.E * t.z + 3) & ~3);
    const size_t smem = backward ? 2 * (n4 + ez4) * 4 : (n4 + ez4) * 4;
    if (smem > (size_t)kTrainMaxSmem)
        return fail(LDPC_ERR_UNSUPPORTED, "learned decoder: %zu B of shared memory per codeword (N=%d, %d edges)", smem, t.n,
                    t.E * t.z);
    g->k = backward ? tk->bwd : tk->fwd;
    g->threads = ((t.z + 31) / 32) * 32;
    g->smem = (int)smem;
    CUDA_TRY(ldpc::allow_dynamic_smem((const void*)g->k, kTrainMaxSmem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)g->k, g->threads, g->smem));
    if (per_sm < 1) return fail(LDPC_ERR_UNSUPPORTED, "learned decoder: launch does not fit an SM");
    g->grid = (int)std::max<long long>(1, std::min<long long>((long long)n, (long long)per_sm * x->sms));
    return LDPC_OK;
}

int check_iters(int iters) {
    if (iters < 1 || iters > ldpc::TRAIN_MAX_ITERS)
        return fail(LDPC_ERR_INVALID_ARG, "iterations %d outside 1..%d", iters, ldpc::TRAIN_MAX_ITERS);
    return LDPC_OK;
}

}  // namespace

extern "C" {

int ldpc_learned_grid(ldpc_ctx* x, size_t n, int* bwd_grid) {
    Geometry g;
    if (int rc = geometry(x, n, true, &g)) return rc;
    if (bwd_grid) *bwd_grid = g.grid;
    return LDPC_OK;
}

int ldpc_learned_forward(ldpc_ctx* x, const float* llr, size_t n, int iters, const float* beta, float* ckpt_p,
                         float* ckpt_r, void* stream) {
    if (int rc = check_iters(iters)) return rc;
    if (n && (!llr || !beta || !ckpt_p || !ckpt_r)) return fail(LDPC_ERR_INVALID_ARG, "NULL buffer");
    Geometry g;
    if (int rc = geometry(x, n, false, &g)) return rc;
    if (n == 0) return LDPC_OK;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::TrainJob j;
    memset(&j, 0, sizeof(j));
    j.llr = llr;
    j.ncw = (long long)n;
    j.iters = iters;
    j.beta = beta;
    j.maxv = x->maxf;
    j.ckpt_p = ckpt_p;
    j.ckpt_r = ckpt_r;
    g.k<<<g.grid, g.threads, g.smem, (cudaStream_t)stream>>>(x->spt, j);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

int ldpc_learned_backward(ldpc_ctx* x, size_t n, int iters, const float* beta, const float* ckpt_p, const float* ckpt_r,
                          const uint8_t* cw_bits, const float* loss_w, float inv_norm, float* gbeta_part,
                          float* grad_llr, void* stream) {
    if (int rc = check_iters(iters)) return rc;
    if (n && (!beta || !ckpt_p || !ckpt_r || !cw_bits || !loss_w || !gbeta_part))
        return fail(LDPC_ERR_INVALID_ARG, "NULL buffer");
    Geometry g;
    if (int rc = geometry(x, n, true, &g)) return rc;
    if (n == 0) return LDPC_OK;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::TrainJob j;
    memset(&j, 0, sizeof(j));
    j.ncw = (long long)n;
    j.iters = iters;
    j.beta = beta;
    j.maxv = x->maxf;
    j.ckpt_p = const_cast<float*>(ckpt_p);
    j.ckpt_r = const_cast<float*>(ckpt_r);
    j.cw_bits = cw_bits;
    j.loss_w = loss_w;
    j.inv_norm = inv_norm;
    j.gbeta_part = gbeta_part;
    j.grad_llr = grad_llr;
    g.k<<<g.grid, g.threads, g.smem, (cudaStream_t)stream>>>(x->spt, j);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

int ldpc_learned_decode(ldpc_ctx* x, const float* llr, size_t n, int iters, const float* beta, float* post_out,
                        uint32_t* hard_out, uint8_t* iters_out, void* stream) {
    if (int rc = check_iters(iters)) return rc;
    if (n && (!llr || !beta)) return fail(LDPC_ERR_INVALID_ARG, "NULL buffer");
    Geometry g;
    if (int rc = geometry(x, n, false, &g)) return rc;
    if (n == 0) return LDPC_OK;
    CUDA_TRY(cudaSetDevice(x->device));
    ldpc::TrainJob j;
    memset(&j, 0, sizeof(j));
    j.llr = llr;
    j.ncw = (long long)n;
    j.iters = iters;
    j.beta = beta;
    j.maxv = x->maxf;
    j.early_exit = 1;
    j.post_out = post_out;
    j.hard_out = hard_out;
    j.iters_out = iters_out;
    g.k<<<g.grid, g.threads, g.smem, (cudaStream_t)stream>>>(x->spt, j);
    CUDA_TRY(cudaGetLastError());
    return LDPC_OK;
}

}  // extern "C"
