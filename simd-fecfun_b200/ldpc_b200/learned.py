"""Learned offsets for layered offset min-sum.

* :class:`LearnedOMSLoss` -- ``torch.autograd.Function`` over the CUDA
  forward (per-iteration checkpoints) and hand-written adjoint kernels
  (``ldpc_learned_forward`` / ``ldpc_learned_backward``).
* :func:`reference_loss` -- the same unrolled decoder and loss written with
  differentiable torch operations (any dtype, CPU or GPU): the reference
  gradient for the adjoint, and the function the finite-difference checks
  differentiate.
* :func:`train` / :func:`evaluate` -- training on codewords drawn by the
  library's own generator (Philox data bits, QC encoder, AWGN), and decoding
  with the learned offsets and early exit.  Under ``torch.distributed``
  training is data-parallel: every rank draws its own codewords and the
  offset gradients are averaged over the ranks (:func:`average_gradients`,
  one all-reduce of iters x layers floats per step).

The decoder is the reference's layered offset min-sum (decode_functions.cpp:
11-103, float variant) with the single offset ``beta_offset`` (sim_struct_
LDPC.h:13) replaced by one offset per iteration and layer.  Loss: binary
cross-entropy of the posteriors after every iteration,
``L = sum_it w[it] * mean_{cw, v} softplus(-(1 - 2 c_v) * P_it+1[v])``.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np
import torch
import torch.nn.functional as F

from . import capi


def _stream() -> Optional[int]:
    return torch.cuda.current_stream().cuda_stream or None


class LearnedOMSLoss(torch.autograd.Function):
    """loss = LearnedOMSLoss.apply(beta, llr, cw_bits, loss_w, ctx)

    beta [iters][mrow] float32 (cuda), llr [n][N] float32, cw_bits [n][N]
    uint8, loss_w [iters] float32; ctx a ``capi.Context`` of variant
    LDPC_F32_OMS.  The gradient flows to beta only."""

    @staticmethod
    def forward(fctx, beta, llr, cw_bits, loss_w, ctx):
        iters = beta.shape[0]
        n, N = llr.shape
        E = ctx.info.edges
        beta = beta.detach().contiguous().float()
        llr = llr.contiguous().float()
        ckpt_p = torch.empty((iters + 1, n, N), dtype=torch.float32, device=llr.device)
        ckpt_r = torch.empty((iters, n, E), dtype=torch.float32, device=llr.device)
        capi.check(capi.lib.ldpc_learned_forward(ctx.h, llr.data_ptr(), n, iters, beta.data_ptr(), ckpt_p.data_ptr(),
                                                 ckpt_r.data_ptr(), _stream()))
        s = 1.0 - 2.0 * cw_bits.float()
        per_it = F.softplus(-s.unsqueeze(0) * ckpt_p[1:]).sum(dim=(1, 2))
        loss = (loss_w.float() * per_it).sum() / float(n * N)
        fctx.save_for_backward(beta, ckpt_p, ckpt_r, cw_bits.contiguous(), loss_w.contiguous().float())
        fctx.ctx = ctx
        fctx.shape = (n, N)
        return loss

    @staticmethod
    def backward(fctx, g):
        beta, ckpt_p, ckpt_r, cw_bits, loss_w = fctx.saved_tensors
        ctx = fctx.ctx
        n, N = fctx.shape
        iters, L = beta.shape
        grid = C.c_int()
        capi.check(capi.lib.ldpc_learned_grid(ctx.h, n, C.byref(grid)))
        part = torch.empty((grid.value, iters * L), dtype=torch.float32, device=beta.device)
        capi.check(capi.lib.ldpc_learned_backward(ctx.h, n, iters, beta.data_ptr(), ckpt_p.data_ptr(), ckpt_r.data_ptr(),
                                                  cw_bits.data_ptr(), loss_w.data_ptr(), 1.0 / float(n * N),
                                                  part.data_ptr(), None, _stream()))
        gbeta = part.sum(dim=0).view(iters, L) * g
        return gbeta, None, None, None, None


def layer_tables(code):
    """Per layer: (index tensor [Z][d] into the posteriors, d)."""
    z = code.z
    d = code.dec
    out, e0 = [], 0
    t = np.arange(z)
    for w in d["row_weights"]:
        cols = np.array(d["row_cols"][e0:e0 + w])
        sh = np.array(d["row_shifts"][e0:e0 + w])
        v = cols[None, :] * z + (t[:, None] + sh[None, :]) % z
        out.append(torch.from_numpy(v.astype(np.int64)))
        e0 += w
    return out


def reference_loss(code, beta: torch.Tensor, llr: torch.Tensor, cw_bits: torch.Tensor, loss_w: torch.Tensor,
                   maxv: float, tables=None) -> torch.Tensor:
    """The unrolled decoder and loss in differentiable torch operations
    (dtype and device of ``llr``)."""
    tables = tables or layer_tables(code)
    P = llr
    n = P.shape[0]
    iters, L = beta.shape
    R = [torch.zeros((n,) + tuple(v.shape), dtype=P.dtype, device=P.device) for v in tables]
    s = 1.0 - 2.0 * cw_bits.to(P.dtype)
    total = torch.zeros((), dtype=P.dtype, device=P.device)
    for it in range(iters):
        for l, v in enumerate(tables):
            v = v.to(P.device)
            z, d = v.shape
            Q = P[:, v] - R[l]
            a = torch.relu(Q.abs() - beta[it, l])
            eye = torch.eye(d, dtype=torch.bool, device=P.device)
            A = a.unsqueeze(-2).expand(n, z, d, d).masked_fill(eye, float("inf"))
            f = torch.clamp(A.min(dim=-1).values, max=maxv)
            sg = torch.where(Q < 0, -1.0, 1.0).to(P.dtype)
            rn = sg.prod(dim=-1, keepdim=True) * sg * f
            P = P.scatter(1, v.reshape(1, -1).expand(n, -1), (Q + rn).reshape(n, -1))
            R[l] = rn
        total = total + loss_w[it] * F.softplus(-s * P).sum()
    return total / float(n * P.shape[1])


def snr_from_ebn0(ebn0_db: float, rate: float) -> float:
    """The reference's SNR (Es/N0 of real BPSK, gen_metrics.cpp:26-29) for a
    given Eb/N0: Es/N0 = Eb/N0 + 10 log10(R)."""
    return ebn0_db + 10.0 * math.log10(rate)


def draw(ctx, code, n: int, snr_db: Sequence[float], seed: int, offset: int):
    """n codewords split over the SNR points (each point its own codewords):
    float LLRs [n][N] and sent code bits [n][N] on the GPU."""
    k = len(snr_db)
    per = [n // k + (1 if i < n % k else 0) for i in range(k)]
    llrs, bits = [], []
    hw = ctx.info.hard_words
    for i, (m, snr) in enumerate(zip(per, snr_db)):
        if m == 0:
            continue
        llr = torch.empty((1, m, code.n), dtype=torch.float32, device="cuda")
        data = torch.empty((m, hw), dtype=torch.int32, device="cuda")
        ctx.generate(seed, offset + sum(per[:i]), [snr], m, llr_f32=llr, data_bits=data,
                     stream=_stream() or 0)
        cw = torch.empty((m, code.n), dtype=torch.uint8, device="cuda")
        ctx.encode(data, m, cw, stream=_stream() or 0)
        llrs.append(llr[0])
        bits.append(cw)
    return torch.cat(llrs), torch.cat(bits)


def average_gradients(params, group=None) -> None:
    """Data-parallel step: replace each gradient by its mean over the ranks
    of ``group`` (every rank decoded its own, equally sized batch, so this is
    the gradient of the loss over all ranks' codewords).  No-op without an
    initialised process group."""
    dist = torch.distributed
    if not (dist.is_available() and dist.is_initialized()):
        return
    world = dist.get_world_size(group)
    for p in params:
        if p.grad is not None:
            dist.all_reduce(p.grad, op=dist.ReduceOp.SUM, group=group)
            p.grad /= world


def _rank_world(group=None):
    dist = torch.distributed
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def train(ctx, code, iters: int = 10, batch: int = 65536, steps: int = 100, ebn0=(1.0, 2.5), lr: float = 0.01,
          init: float = 0.5, seed: int = 1, n_snr: int = 16, loss_w: Optional[Sequence[float]] = None, log=None,
          group=None, quant_step: Optional[float] = None):
    """Adam on beta [iters][mrow] (initialised to ``init``); every step draws
    a fresh batch at Eb/N0 points spread uniformly over ``ebn0``.  With a
    process group, ``batch`` is per rank: rank r draws codewords
    [(step * world + r) * batch, ...) of the generator's stream, the ranks
    share the Eb/N0 draw (same ``seed``) and average their gradients, so
    their offsets stay identical.

    ``quant_step``: quantisation-aware training for offsets that will be
    deployed on a grid (0.5 for the int8 decoder at LLR scale 2, whose
    offsets are integers in its own units): the decoder runs with beta
    rounded to the grid, the gradient passes the rounding unchanged
    (straight-through), and the returned offsets are on the grid."""
    rank, world = _rank_world(group)
    rate = code.k / (code.n - code.punc_cnt_bits - code.fill_cnt)
    beta = torch.full((iters, code.mrow), init, dtype=torch.float32, device="cuda", requires_grad=True)
    w = torch.tensor(loss_w if loss_w is not None else [1.0] * iters, dtype=torch.float32, device="cuda")
    opt = torch.optim.Adam([beta], lr=lr)
    rng = np.random.default_rng(seed)
    history = []
    for step in range(steps):
        eb = rng.uniform(ebn0[0], ebn0[1], n_snr)
        llr, bits = draw(ctx, code, batch, [snr_from_ebn0(e, rate) for e in eb], seed, (step * world + rank) * batch)
        opt.zero_grad()
        b_used = beta if quant_step is None else beta + (torch.round(beta / quant_step) * quant_step - beta).detach()
        loss = LearnedOMSLoss.apply(b_used, llr, bits, w, ctx)
        loss.backward()
        average_gradients([beta], group)
        opt.step()
        with torch.no_grad():
            beta.clamp_(min=0.0)
        history.append(float(loss))
        if log:
            log(step, float(loss))
    if quant_step is not None:
        return (torch.round(beta.detach() / quant_step) * quant_step), history
    return beta.detach(), history


def evaluate(ctx, code, beta: torch.Tensor, snr_db: float, n: int, seed: int = 99, offset: int = 1 << 40,
             chunk: int = 65536):
    """Decode n fresh codewords with offsets beta (early exit): returns
    (codeword error rate, bit error rate, average iterations)."""
    iters = beta.shape[0]
    beta = beta.contiguous().float()
    kb = ctx.info.kbits
    cw_err = bit_err = it_sum = 0
    done = 0
    while done < n:
        m = min(chunk, n - done)
        llr, bits = draw(ctx, code, m, [snr_db], seed, offset + done)
        hard = torch.empty((m, ctx.info.hard_words), dtype=torch.int32, device="cuda")
        its = torch.empty(m, dtype=torch.uint8, device="cuda")
        capi.check(capi.lib.ldpc_learned_decode(ctx.h, llr.data_ptr(), m, iters, beta.data_ptr(), None, hard.data_ptr(),
                                                its.data_ptr(), _stream()))
        dec = torch.stack([(hard >> b) & 1 for b in range(32)], dim=-1).reshape(m, -1)[:, :kb].to(torch.uint8)
        err = (dec != bits[:, :kb]).sum(dim=1)
        cw_err += int((err > 0).sum())
        bit_err += int(err.sum())
        it_sum += int(its.sum())
        done += m
    return cw_err / n, bit_err / (n * code.k), it_sum / n
