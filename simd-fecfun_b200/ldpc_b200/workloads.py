"""Measured workloads beyond the headline 802.11ad run (``bench.py
--workload ...``).  Each returns one JSON-ready dict.

* :func:`nr_mix` -- 5G NR base graph 1 (Z=384, K=8448, the full 46-row
  graph) and base graph 2 (Z=64/128/256, full 42-row graph), int8 offset
  min-sum with 20 iterations.  Uneven seeded codeword counts per code go
  through ONE persistent launch, autotuned and replayed from a CUDA graph.
  The same jobs decoded one code at a time are timed beside it.
* :func:`hetero_mix` -- every 802.11n code, 802.11ay 1/2..7/8 and 802.11ad
  13/16 in one launch, each at the SNR calibrated to codeword error rate
  near 1e-3: plain offsets vs learned per-(iteration, layer) offsets
  (trained in float, quantised to an int8 table).
* :func:`learned_run` -- training throughput of the learned-offset decoder
  (802.16e 1/2, Z=96, 10 iterations x 12 layers, batches of 65536
  codewords), then codeword error rate and average iterations of learned
  vs plain offsets.
* :func:`sp_sweep` -- float sum-product on 802.16e 1/2 for all 19 lifting
  sizes Z = 24..96.
* :func:`variants` -- the headline 802.11ad 1/2 simulation point decoded by
  every decoder variant of the reference's LDPCtop family (int8/int16/int32
  offset min-sum, float and double offset min-sum and sum-product), each
  with the Perl driver's parameters for that variant.

Inputs are synthetic, drawn on the device by the library's generator
(Philox data bits, QC encoding, AWGN); SNRs given as Eb/N0 are converted to
the reference's Es/N0 with the code rate."""
from __future__ import annotations

import math
import time
from typing import Dict, List

import numpy as np
import torch

from . import capi, codes, learned


def _events(n):
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def _rate(c) -> float:
    return c.k / (c.n - c.punc_cnt_bits - c.fill_cnt)


def _build_jobs(handles, objs, counts, snrs_per_code, seed, max_iter, beta=1.0):
    """LLR buffers, sent data and counters for every (code, SNR point) job."""
    specs, meta = [], []
    s = torch.cuda.current_stream().cuda_stream
    for ci, (h, c, m, snrs) in enumerate(zip(handles, objs, counts, snrs_per_code)):
        ctx = capi.Context(h, max_iter=max_iter, beta=beta)
        per = [m // len(snrs) + (1 if i < m % len(snrs) else 0) for i in range(len(snrs))]
        off = 0
        for snr, k in zip(snrs, per):
            llr = torch.empty((1, k, c.n), dtype=torch.int8, device="cuda")
            data = torch.empty((k, h.info.hard_words), dtype=torch.int32, device="cuda")
            ctx.generate(seed + ci, off, [snr], k, llr_i8=llr, data_bits=data, stream=s)
            cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
            specs.append(dict(code=ci, llr=llr, n=k, data_bits=data, ref_period=k, bucket_size=k, counters=cnt,
                              n_buckets=1))
            meta.append((ci, snr))
            off += k
        del ctx
    torch.cuda.synchronize()
    return specs, meta


def _quality(specs, meta, names, objs, steps) -> List[Dict]:
    out = []
    for s, (ci, snr) in zip(specs, meta):
        c = s["counters"].cpu().numpy()[0]
        n = int(c[0])
        out.append(dict(code=names[ci], snr_db=round(float(snr), 3), codewords=n,
                        avg_iter=float(c[1]) / max(1, n), cwer=float(c[3]) / max(1, n),
                        ber=float(c[2]) / max(1, n * objs[ci].k)))
    return out


# Roofline work units.
# int8 offset min-sum: 10 int8 lane-ops per edge and iteration (Q sub, abs,
# offset, clamp at 0, min1/min2 update (2), sign XOR, select, sign apply, P
# add), four lanes per 32-bit op: 2.5 packed int32 ops per edge-iteration,
# against the probed int32 issue rate.
INT8_OPS_PER_EDGE = 2.5
# float sum-product: FP32 operations per edge-iteration of the update as
# written (ldpc_math.h along its usual branches, a division counted once):
# tanh 23 (-2x, Cody-Waite e^y with a degree-8 Horner polynomial, -e/(2+e)),
# atanh 27 (2m/(1-m), log1p by exponent split, a degree-6 series in s^2 and
# the first-order correction), the rest of the edge 8 (P - R, |Q| - beta,
# max 0, x 0.5, ~2.3 tree products, 2 x atanh, Q + R'), against the probed
# FP32 fused multiply-add rate.
SP_FP32_OPS_PER_EDGE = 58.0


def _edge_iters_per_step(specs, quality, objs, steps) -> float:
    """Edge updates per timed step: codewords x average iterations x edges,
    summed over the jobs (quality holds the counters of ``steps`` steps)."""
    return sum(q["codewords"] * q["avg_iter"] * objs[sp["code"]].edges for sp, q in zip(specs, quality)) / steps


def _roofline(work_per_step: float, ms: float, peak: float, unit: str, definition: str, peak_source: str) -> Dict:
    achieved = work_per_step / (ms * 1e-3)
    return {"bound": unit.split()[0], "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "T%s/s" % unit,
            "frac": achieved / peak, "definition": definition, "peak_source": peak_source}


def _time_plan(plan, specs, steps, warmup, graph=True):
    s = torch.cuda.current_stream()
    for _ in range(warmup):
        (plan.graph_launch if graph else plan.launch)(s.cuda_stream)
    torch.cuda.synchronize()
    for sp in specs:
        sp["counters"].zero_()
    ev = _events(steps)
    for a, b in ev:
        a.record(s)
        (plan.graph_launch if graph else plan.launch)(s.cuda_stream)
        b.record(s)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def nr_mix(steps: int = 3, warmup: int = 1, seed: int = 7, llr_budget: float = 40e9, ebn0=(0.5, 1.0, 1.5),
           autotune: bool = True) -> Dict:
    names = ["5GNR_n25344_k8448", "5GNR_n3136_k576", "5GNR_n6400_k1280", "5GNR_n12800_k2560"]
    objs = [codes.code_by_name(n) for n in names]
    rng = np.random.default_rng(seed)
    drawn = rng.integers(100_000, 4_000_001, len(names))
    need = float(sum(int(m) * c.n for m, c in zip(drawn, objs)))
    scale = min(1.0, llr_budget / need)
    counts = [max(len(ebn0), int(m * scale)) for m in drawn]
    handles = [capi.Code.from_tables(c) for c in objs]
    snrs = [[learned.snr_from_ebn0(e, _rate(c)) for e in ebn0] for c in objs]
    specs, meta = _build_jobs(handles, objs, counts, snrs, seed, 20)
    batch = capi.Batch(handles, [dict(max_iter=20)] * len(objs))
    t0 = time.time()
    tuned = batch.autotune(specs, sample=16384) if autotune else (0, 0, 0.0)
    tune_s = time.time() - t0
    plan = batch.plan(specs)
    ms = _time_plan(plan, specs, steps, warmup)
    quality = _quality(specs, meta, names, objs, steps)
    total = sum(counts)
    info_bits = sum(m * c.k for m, c in zip(counts, objs))
    avg_ms = sum(ms) / len(ms)
    roofline = _roofline(_edge_iters_per_step(specs, quality, objs, steps) * INT8_OPS_PER_EDGE, avg_ms,
                         capi.probe_int32_peak(torch.cuda.current_device()), "int32 ops",
                         "sum over jobs of codewords x iterations x edges x 2.5 packed int32 ops (10 int8 lane-ops "
                         "per edge-iteration, 4 lanes per 32-bit op), per step, over the step's graph time",
                         "own microbenchmark of 32-bit lop3/iadd chains (ldpc_probe_int32_peak)")
    # the same jobs, one code at a time through the per-code entry point
    s = torch.cuda.current_stream()
    ctxs = [capi.Context(h, max_iter=20) for h in handles]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for sp in specs:
        ctxs[sp["code"]].decode_count(sp["llr"], sp["n"], data_bits=sp["data_bits"], ref_period=sp["n"],
                                      bucket_size=sp["n"], counters=sp["counters"], n_buckets=1, stream=s.cuda_stream)
    torch.cuda.synchronize()
    e0.record(s)
    for sp in specs:
        ctxs[sp["code"]].decode_count(sp["llr"], sp["n"], data_bits=sp["data_bits"], ref_period=sp["n"],
                                      bucket_size=sp["n"], counters=sp["counters"], n_buckets=1, stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    return {
        "metric": "codewords/s decoded, 5G NR BG1 Z=384 + BG2 Z=64/128/256 mix, int8 offset min-sum, 20 max iterations",
        "value": total / (avg_ms * 1e-3), "unit": "codewords/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": avg_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: Philox data bits, QC encoding, AWGN from the fused generator, resident in HBM",
        "config": {"workload": "5G NR: %s; codewords per code %s (seeded draw in [1e5, 4e6]%s); Eb/N0 %s dB "
                               "(Es/N0 = Eb/N0 + 10 log10 R); beta=1, max_row_metric=31, LLR scale 2, max|LLR| 24"
                               % (", ".join(names), counts,
                                  "" if scale >= 1 else ", scaled by %.3f to fit %.0f GB of LLRs" % (scale, llr_budget / 1e9),
                                  list(ebn0)),
                   "launch": "%d persistent kernels (one per geometry class) over %d jobs, in one CUDA graph"
                             % (plan.kernels, len(specs)),
                   "autotuned": {"threads": tuned[0], "chunks_per_cta": tuned[1], "sample_ms": tuned[2],
                                 "tuning_s": round(tune_s, 2)},
                   "l2": "inputs larger than L2 (%.1f GB of LLRs)" % (sum(m * c.n for m, c in zip(counts, objs)) / 1e9)},
        "info_gbps": info_bits / (avg_ms * 1e-3) / 1e9,
        "per_code_sequential": {"value": total / (seq_ms * 1e-3), "unit": "codewords/s",
                                "note": "same jobs, one ldpc_decode_count launch per job"},
        "roofline": roofline,
        "gpu_launches": steps * plan.kernels,
        "quality": quality,
    }


def _calibrate(h, c, target=1e-3, n=100_000, seed=5, max_iter=10):
    """SNR (reference convention) where the codeword error rate is near
    ``target``: bisection over ldpc_simulate runs, then log-linear
    interpolation between the bracketing points."""
    ctx = capi.Context(h, max_iter=max_iter)
    r = _rate(c)
    lo, hi = learned.snr_from_ebn0(0.0, r), learned.snr_from_ebn0(7.0, r)

    def cwer(snr):
        st = ctx.simulate(seed=seed, cw_offset=0, snr_db=[snr], n_per_snr=n)[0]
        return max(st["cw_errors"], 0.5) / n

    f_lo, f_hi = cwer(lo), cwer(hi)
    for _ in range(7):
        mid = 0.5 * (lo + hi)
        f = cwer(mid)
        if f > target:
            lo, f_lo = mid, f
        else:
            hi, f_hi = mid, f
    a, b = math.log(f_lo), math.log(f_hi)
    snr = lo + (hi - lo) * (a - math.log(target)) / (a - b) if a != b else hi
    return float(snr)


def hetero_mix(steps: int = 3, warmup: int = 1, total: int = 10_000_000, seed: int = 11, train_steps: int = 40) -> Dict:
    names = ["11n %s z%d" % (r, z) for z in (27, 54, 81) for r in ("1/2", "2/3", "3/4", "5/6")]
    names += ["11ay 1/2", "11ay 5/8", "11ay 3/4", "11ay 13/16", "11ay 7/8", "11ad 13/16"]
    objs = [codes.make_code(n) for n in names]
    handles = [capi.Code.from_tables(c) for c in objs]
    t0 = time.time()
    snr = [_calibrate(h, c) for h, c in zip(handles, objs)]
    cal_s = time.time() - t0
    counts = [total // len(objs) + (1 if i < total % len(objs) else 0) for i in range(len(objs))]
    specs, meta = _build_jobs(handles, objs, counts, [[s] for s in snr], seed, 10)
    batch = capi.Batch(handles, [dict(max_iter=10)] * len(objs))
    tuned = batch.autotune(specs, sample=32768)
    plan = batch.plan(specs)
    ms_plain = _time_plan(plan, specs, steps, warmup)
    q_plain = _quality(specs, meta, names, objs, steps)
    # learned offsets: float offset min-sum trained at the code's SNR,
    # converted to int8 LLR units (scale 2), rounded, and decoded as an int8
    # [iteration][layer] table
    t0 = time.time()
    offsets, kept = [], []
    for ci, (h, c) in enumerate(zip(handles, objs)):
        fctx = capi.Context(h, variant=capi.LDPC_F32_OMS, max_iter=10, max_row_metric=31.0, beta=0.5,
                            llr_scale=1.0, max_abs_llr=1e9)
        eb = snr[ci] - 10.0 * math.log10(_rate(c))
        beta, _ = learned.train(fctx, c, iters=10, batch=8192, steps=train_steps, ebn0=(eb - 0.25, eb + 0.25), lr=0.02,
                                init=0.5, seed=seed + ci, n_snr=4, quant_step=0.5)
        b8 = np.clip(np.rint(2.0 * beta.cpu().numpy()), 0, 127).astype(np.float32)   # [iters][layers]
        # deploy the table only when it beats the plain offset on fresh codewords: fewer
        # iterations, codeword errors within two standard deviations of the plain count
        vctx = capi.Context(h, max_iter=10)
        plain_v = vctx.simulate(seed=seed + 1000 + ci, cw_offset=1 << 40, snr_db=[snr[ci]], n_per_snr=200_000)[0]
        vctx.set_offset_table(b8)
        tab_v = vctx.simulate(seed=seed + 1000 + ci, cw_offset=1 << 40, snr_db=[snr[ci]], n_per_snr=200_000)[0]
        keep = (tab_v["iterations"] < plain_v["iterations"] and
                tab_v["cw_errors"] <= plain_v["cw_errors"] + 2.0 * math.sqrt(max(plain_v["cw_errors"], 1)))
        if keep:
            batch.set_offset_table(ci, b8)
        kept.append(bool(keep))
        offsets.append(b8.astype(int).tolist())
    train_s = time.time() - t0
    plan_l = batch.plan(specs)
    ms_learned = _time_plan(plan_l, specs, steps, warmup)
    q_learned = _quality(specs, meta, names, objs, steps)
    avg_plain, avg_learned = sum(ms_plain) / steps, sum(ms_learned) / steps
    it_p = sum(q["avg_iter"] * q["codewords"] for q in q_plain) / sum(q["codewords"] for q in q_plain)
    it_l = sum(q["avg_iter"] * q["codewords"] for q in q_learned) / sum(q["codewords"] for q in q_learned)
    return {
        "metric": "codewords/s decoded, 18-code 802.11n/ay/ad mix at CWER near 1e-3, int8 offset min-sum, 10 max iterations",
        "value": total / (avg_plain * 1e-3), "unit": "codewords/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": avg_plain, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: Philox data bits, QC encoding, AWGN from the fused generator, resident in HBM",
        "config": {"workload": "%d codes (%s), %d codewords in one CUDA graph (equal split), per-code SNR "
                               "calibrated to CWER 1e-3 (bisection over ldpc_simulate, 1e5 codewords per point, %.1f s)"
                               % (len(names), ", ".join(names), total, cal_s),
                   "autotuned": {"threads": tuned[0], "chunks_per_cta": tuned[1]},
                   "launch": "%d persistent kernels (one per geometry class) in one CUDA graph" % plan.kernels,
                   "snr_db": dict(zip(names, [round(s, 3) for s in snr]))},
        "info_gbps": sum(m * c.k for m, c in zip(counts, objs)) / (avg_plain * 1e-3) / 1e9,
        "learned": {"value": total / (avg_learned * 1e-3), "unit": "codewords/s", "avg_iter": it_l,
                    "offsets_int8": dict(zip(names, offsets)), "training_s": round(train_s, 1),
                    "deployed": dict(zip(names, kept)),
                    "deploy_rule": "a code keeps its learned table only when, on 2e5 fresh codewords at its SNR, it "
                                   "needs fewer iterations than the plain offset with codeword errors within two "
                                   "standard deviations; otherwise the plain offset stays",
                    "training": "float offset min-sum, 10 iterations, %d Adam steps of 8192 codewords at the "
                                "calibrated SNR +-0.25 dB, quantisation-aware (offsets rounded to multiples of 0.5, "
                                "straight-through gradient); offsets x2 (int8 LLR scale) deployed as an int8 "
                                "[iteration][layer] table" % train_steps},
        "plain_avg_iter": it_p,
        "gpu_launches": steps * plan.kernels,
        "quality_plain": q_plain, "quality_learned": q_learned,
    }


def learned_run(train_steps: int = 30, batch: int = 65536, eval_n: int = 200_000, seed: int = 3,
                weights: str = "uniform") -> Dict:
    """``weights``: "uniform" (every iteration's BCE counts once), "early"
    (iteration it weighted 1/(it+1), rewarding codewords that are right
    sooner) or "steep" (weight 2^-it: the first iterations dominate)."""
    code = codes.make_code("16e 1/2", z_over=96)
    h = capi.Code.from_tables(code)
    ctx = capi.Context(h, variant=capi.LDPC_F32_OMS, max_iter=10, max_row_metric=31.0, beta=0.5, llr_scale=1.0,
                       max_abs_llr=1e9)
    # warm-up step (allocations, module load), then timed training
    learned.train(ctx, code, iters=10, batch=batch, steps=1, seed=seed)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    lw = ([1.0 / (i + 1) for i in range(10)] if weights == "early" else
          [0.5 ** i for i in range(10)] if weights == "steep" else None)
    beta, hist = learned.train(ctx, code, iters=10, batch=batch, steps=train_steps, ebn0=(1.0, 2.5), lr=0.01,
                               init=0.5, seed=seed, loss_w=lw)
    e1.record()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1)
    # forward + adjoint alone on one batch
    llr, bits = learned.draw(ctx, code, batch, [learned.snr_from_ebn0(1.75, 0.5)], seed, 1 << 32)
    w = torch.ones(10, dtype=torch.float32, device="cuda")
    b = beta.clone().requires_grad_(True)
    for _ in range(2):
        learned.LearnedOMSLoss.apply(b, llr, bits, w, ctx).backward()
    ev = _events(5)
    for a, c in ev:
        a.record()
        learned.LearnedOMSLoss.apply(b, llr, bits, w, ctx).backward()
        c.record()
    torch.cuda.synchronize()
    fb_ms = sorted(a.elapsed_time(c) for a, c in ev)[2]
    plain = torch.full_like(beta, 0.5)
    evals = []
    # Eb/N0 points; 3.01 dB is the reference's SNR (Es/N0) of 0 dB at rate 1/2
    for eb in (0.0, 1.0, 1.5, 2.0, 2.5, 3.01):
        snr = learned.snr_from_ebn0(eb, 0.5)
        cp, bp, ip = learned.evaluate(ctx, code, plain, snr, eval_n)
        cl, bl, il = learned.evaluate(ctx, code, beta, snr, eval_n)
        evals.append(dict(ebn0_db=eb, plain=dict(cwer=cp, ber=bp, avg_iter=ip), learned=dict(cwer=cl, ber=bl, avg_iter=il),
                          iter_reduction=1.0 - il / ip))
    return {
        "metric": "codewords/s trained, learned-offset float offset min-sum, 802.16e 1/2 Z=96, 10 iterations x 12 layers",
        "value": batch * train_steps / (train_ms * 1e-3), "unit": "codewords/s", "n_gpus": 1, "steps": train_steps,
        "warmup": 1, "ms_per_step": train_ms / train_steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: codewords drawn on the device by the library's generator every step",
        "config": {"workload": "802.16e 1/2 Z=96 (N=2304), batches of %d codewords, Eb/N0 uniform in [1.0, 2.5] dB "
                               "(16 points per batch), 120 offsets from 0.5, Adam lr 0.01, BCE over all iterations "
                               "(%s weights)" % (batch, weights),
                   "step": "generation + encoding + forward with checkpoints + adjoint + Adam"},
        "forward_adjoint_ms": fb_ms,
        "forward_adjoint_cw_s": batch / (fb_ms * 1e-3),
        "loss_first_last": [hist[0], hist[-1]],
        "offsets": [[round(float(v), 3) for v in row] for row in beta.cpu()],
        "evaluation": evals,
        "gpu_launches": None,
    }


def sp_sweep(cw_per_z: int = 1 << 20, ebn0=(0.5, 1.0, 1.5, 2.0), seed: int = 5, max_iter: int = 10,
             llr_budget: float = 60e9, steps: int = 1, warmup: int = 1, autotune: bool = True) -> Dict:
    """802.16e rate 1/2 for every Z = 24, 28, ..., 96 (N = 576..2304), float
    sum-product (clamp 1 - 6e-8, LLR = 2y/sigma^2, no LLR limit), 10
    iterations.  All 19 codes, their codewords spread over the Eb/N0 points,
    are decoded by ONE persistent launch (a float batch plan replayed from a
    CUDA graph); the same jobs decoded one launch per (Z, Eb/N0) are timed
    beside it."""
    zs = list(range(24, 97, 4))
    objs = [codes.make_code("16e 1/2", z_over=z) for z in zs]
    need = float(sum(c.n * 4 for c in objs)) * cw_per_z
    scale = min(1.0, llr_budget / need)
    per_z = max(len(ebn0), int(cw_per_z * scale))
    handles = [capi.Code.from_tables(c) for c in objs]
    kw = dict(variant=capi.LDPC_F32_SP, max_iter=max_iter, max_row_metric=6e-8, beta=0.0, llr_scale=1.0,
              max_abs_llr=1e9)
    s = torch.cuda.current_stream()
    specs, meta, ctxs = [], [], []
    for ci, (c, h) in enumerate(zip(objs, handles)):
        ctx = capi.Context(h, **kw)
        ctxs.append(ctx)
        k = len(ebn0)
        per = per_z // k
        for i, e in enumerate(ebn0):
            llr = torch.empty((1, per, c.n), dtype=torch.float32, device="cuda")
            data = torch.empty((per, h.info.hard_words), dtype=torch.int32, device="cuda")
            ctx.generate(seed + zs[ci], i * per, [learned.snr_from_ebn0(e, 0.5)], per, llr_f32=llr, data_bits=data,
                         stream=s.cuda_stream)
            cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
            specs.append(dict(code=ci, llr=llr, n=per, data_bits=data, ref_period=per, bucket_size=per, counters=cnt,
                              n_buckets=1))
            meta.append((ci, e))
    torch.cuda.synchronize()
    batch = capi.Batch(handles, [kw] * len(objs))
    t0 = time.time()
    tuned = batch.autotune(specs, sample=8192) if autotune else (0, 0, 0.0)
    tune_s = time.time() - t0
    plan = batch.plan(specs)
    ms = _time_plan(plan, specs, steps, warmup)
    names = ["16e 1/2 Z=%d" % z for z in zs]
    quality = _quality(specs, meta, names, objs, steps)
    for q in quality:
        q["ebn0_db"] = q.pop("snr_db")
    total = sum(sp["n"] for sp in specs)
    info_bits = sum(sp["n"] * objs[sp["code"]].k for sp in specs)
    avg_ms = sum(ms) / len(ms)
    fma_peak, mufu_peak = capi.probe_fp32_peak(torch.cuda.current_device())
    roofline = _roofline(_edge_iters_per_step(specs, quality, objs, steps) * SP_FP32_OPS_PER_EDGE, avg_ms, fma_peak,
                         "fp32 ops",
                         "sum over jobs of codewords x iterations x edges x 58 FP32 operations per edge-iteration "
                         "(tanh 23, atanh 27, the rest of the update 8), per step, over the step's graph time",
                         "own microbenchmark of FP32 fma chains (ldpc_probe_fp32_peak)")
    roofline["mufu_peak"] = mufu_peak / 1e12
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for sp in specs:
        ctxs[sp["code"]].decode_count(sp["llr"], sp["n"], data_bits=sp["data_bits"], ref_period=sp["n"],
                                      bucket_size=sp["n"], counters=sp["counters"], n_buckets=1, stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    return {
        "metric": "codewords/s decoded, 802.16e 1/2 Z=24..96 (19 sizes) in one launch, float32 layered sum-product, "
                  "10 max iterations",
        "value": total / (avg_ms * 1e-3), "unit": "codewords/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": avg_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: Philox data bits, QC encoding, AWGN from the fused generator, resident in HBM",
        "config": {"workload": "802.16e 1/2, Z in 24..96 step 4 (shifts mod Z), %d codewords per Z%s over Eb/N0 %s dB "
                               "(Es/N0 = Eb/N0 - 3.01 dB), sum-product clamp 1-6e-8, LLR scale 1, no LLR limit"
                               % (per_z, "" if scale >= 1 else " (2^20 scaled by %.3f to fit %.0f GB of float LLRs)"
                                  % (scale, llr_budget / 1e9), list(ebn0)),
                   "launch": "%d persistent float batch kernels (one per geometry class) over %d jobs, in one "
                             "CUDA graph" % (plan.kernels, len(specs)),
                   "autotuned": {"threads": tuned[0], "chunks_per_cta": tuned[1], "sample_ms": tuned[2],
                                 "tuning_s": round(tune_s, 2)},
                   "l2": "inputs larger than L2 (%.1f GB of LLRs)" % (sum(sp["n"] * objs[sp["code"]].n * 4
                                                                          for sp in specs) / 1e9)},
        "info_gbps": info_bits / (avg_ms * 1e-3) / 1e9,
        "per_launch_sequential": {"value": total / (seq_ms * 1e-3), "unit": "codewords/s",
                                  "note": "same jobs, one ldpc_decode_count launch per (Z, Eb/N0)"},
        "roofline": roofline,
        "gpu_launches": steps * plan.kernels,
        "quality": quality,
    }


# (label, variant, reference build, max_row_metric, beta, LLR scale, max |LLR|):
# the Perl driver's defaults (run_LDPCsim.pl:29-32), and for sum-product its
# overrides (run_LDPCsim.pl:56-63: clamp 1-6e-8 float, 1-1e-16 double)
VARIANT_RUNS = [
    ("int8 offset min-sum", capi.LDPC_INT8_OMS, "Vec64c_min", 31.0, 1.0, 2.0, 24.0),
    ("int16 offset min-sum", capi.LDPC_INT16_OMS, "Vec32s_min", 31.0, 1.0, 2.0, 24.0),
    ("int32 offset min-sum", capi.LDPC_INT32_OMS, "Vec16w_min", 31.0, 1.0, 2.0, 24.0),
    ("float offset min-sum", capi.LDPC_F32_OMS, "Vec16f_min", 31.0, 1.0, 2.0, 24.0),
    ("float sum-product", capi.LDPC_F32_SP, "Vec16f_prod", 6e-8, 0.0, 1.0, 1e9),
    ("double offset min-sum", capi.LDPC_F64_OMS, "Vec8d_min", 31.0, 1.0, 2.0, 24.0),
    ("double sum-product", capi.LDPC_F64_SP, "Vec8d_prod", 1e-16, 0.0, 1.0, 1e9),
]


def variants(n_per_snr: int = 200_000, snrs=(-1.0, -0.75, -0.5, -0.25, 0.0), seed: int = 17,
             max_iter: int = 10) -> List[Dict]:
    """802.11ad 1/2 at the headline SNR points through ldpc_simulate for each
    variant: the generator writes LLRs of the variant's element type, the
    decoder runs with fused counting, and only the decoder's device time
    (CUDA events around each launch) counts.  One untimed pass first."""
    code = codes.make_code("11ad 1/2")
    h = capi.Code.from_tables(code)
    out = []
    for label, variant, ref, mrm, beta, scale, max_abs in VARIANT_RUNS:
        ctx = capi.Context(h, variant=variant, max_iter=max_iter, max_row_metric=mrm, beta=beta, llr_scale=scale,
                           max_abs_llr=max_abs)
        ctx.simulate(seed=seed, cw_offset=1 << 40, snr_db=list(snrs), n_per_snr=min(n_per_snr, 20_000))
        st = ctx.simulate(seed=seed, cw_offset=0, snr_db=list(snrs), n_per_snr=n_per_snr)
        cw = sum(x["codewords"] for x in st)
        ms = sum(x["decode_ms"] for x in st)
        out.append({
            "variant": label, "reference_build": "LDPCtop_" + ref, "codewords": cw, "decode_ms": ms,
            "value": cw / (ms * 1e-3), "unit": "codewords/s",
            "params": {"max_row_metric": mrm, "beta": beta, "llr_scale": scale, "max_abs_llr": max_abs},
            "avg_iter": sum(x["iterations"] for x in st) / cw,
            "quality": [{"snr_db": x["snr_db"], "cwer": x["cw_errors"] / x["codewords"],
                         "ber": x["bit_errors"] / (x["codewords"] * code.k)} for x in st],
        })
    return out


def _cwer_ci(err: int, n: int):
    """95 % Wilson interval of a codeword error rate."""
    if n == 0:
        return (0.0, 1.0)
    p, z = err / n, 1.96
    den = 1 + z * z / n
    c = (p + z * z / (2 * n)) / den
    h = z * math.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / den
    return (max(0.0, c - h), min(1.0, c + h))


def _coord_search(run, S, base, values, sweeps, limit, it0):
    """Coordinate descent over an offset table: minimise the average
    iterations ``run(table, S)[0]`` subject to codeword errors
    ``run(table, S)[1] <= limit``; first whole rows (one offset per
    iteration), then single entries.  Returns (table, avg_iter, trace)."""
    best, best_it = base.copy(), it0
    trace = []
    rows, cols = best.shape

    def consider(tab):
        nonlocal best, best_it
        it, e = run(tab, S)
        if e <= limit and it < best_it - 1e-9:
            best, best_it = tab.copy(), it

    for _ in range(sweeps):
        for i in range(rows):
            for v in values:
                if np.all(best[i] == v):
                    continue
                tab = best.copy()
                tab[i, :] = v
                consider(tab)
        trace.append(round(best_it, 5))
    for _ in range(sweeps):
        for i in range(rows):
            for l in range(cols):
                for v in values:
                    if v == best[i, l]:
                        continue
                    tab = best.copy()
                    tab[i, l] = v
                    consider(tab)
        trace.append(round(best_it, 5))
    return best, best_it, trace


def _search_point(run, S, V, base, values, sweeps, label, n_search, n_valid):
    it0, e0 = run(None, S)
    limit = e0 + 2.0 * math.sqrt(max(e0, 1))
    best, best_it, trace = _coord_search(run, S, base, values, sweeps, limit, it0)
    itp, ep = run(None, V)
    itb, eb = run(best, V)
    return {
        "point": label,
        "search": {"codewords": n_search, "plain_avg_iter": it0, "plain_cw_errors": e0, "best_avg_iter": best_it,
                   "feasible_cw_errors_max": limit, "trace_avg_iter": trace},
        "validation": {"codewords": n_valid,
                       "plain": {"avg_iter": itp, "cw_errors": ep, "cwer": ep / n_valid, "cwer_ci95": _cwer_ci(ep, n_valid)},
                       "best": {"avg_iter": itb, "cw_errors": eb, "cwer": eb / n_valid, "cwer_ci95": _cwer_ci(eb, n_valid)},
                       "iter_reduction": 1.0 - itb / itp},
        "best_table": best.tolist(),
    }


def offset_search(snr_db=(0.0, -0.5), n_search: int = 4_000_000, n_valid: int = 20_000_000,
                  values=(0, 1, 2, 3, 4), sweeps: int = 2, max_iter: int = 10, seed: int = 21,
                  f_ebn0=(3.0103, 2.0), f_search: int = 400_000, f_valid: int = 2_000_000,
                  f_values=(0.0, 0.25, 0.5, 0.75, 1.0, 1.5)) -> Dict:
    """Empirical ceiling of the iteration saving that offsets alone can buy:
    a coordinate search over offset tables beta[iteration][layer], run with
    the GPU decoders themselves.

    int8 (the headline code, 802.11ad 1/2, Es/N0 ``snr_db``): integer offsets
    in ``values`` (the reference truncates its one offset to an integer for
    the int8 build, decode_functions.cpp:59-62), the plain decoder being
    beta = 1 everywhere (the Perl driver's default).  Float offset min-sum
    (802.16e 1/2 Z=96, the learned decoder's code, Eb/N0 ``f_ebn0``; 3.01 dB
    is the reference's SNR of 0 dB at rate 1/2): offsets in ``f_values``,
    plain beta = 0.5.

    Per point, LLRs of a search set and of a fresh validation set are drawn
    once and stay in HBM.  The plain table's codeword errors e0 on the
    search set set the constraint: a table is feasible when its errors are
    at most e0 + 2 sqrt(e0).  The search minimises the average iterations over
    feasible tables (whole rows first, then single entries, ``sweeps`` passes
    each); the best table and the plain one are then decoded on the
    validation set and reported with 95 % intervals."""
    t_start = time.time()
    n_evals = 0
    s = torch.cuda.current_stream().cuda_stream
    cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
    points = []

    # ---- int8, 802.11ad rate 1/2 ----
    code = codes.make_code("11ad 1/2")
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=max_iter, max_row_metric=31.0, beta=1.0, llr_scale=2.0,
                       max_abs_llr=24.0)
    N, HW = code.n, ctx.info.hard_words

    def make8(n, snr, off):
        llr = torch.empty((1, n, N), dtype=torch.int8, device="cuda")
        data = torch.empty((n, HW), dtype=torch.int32, device="cuda")
        ctx.generate(seed, off, [snr], n, llr_i8=llr, data_bits=data, stream=s)
        return llr, data, n

    def run8(table, st):
        nonlocal n_evals
        llr, data, n = st
        ctx.set_offset_table(None if table is None else np.asarray(table, np.float32))
        cnt.zero_()
        ctx.decode_count(llr, n, data_bits=data, ref_period=n, bucket_size=n, counters=cnt, n_buckets=1, stream=s)
        c = cnt.cpu().numpy()[0]
        n_evals += 1
        return float(c[1]) / n, int(c[3])

    for snr in snr_db:
        S, V = make8(n_search, snr, 0), make8(n_valid, snr, 1 << 36)
        r = _search_point(run8, S, V, np.ones((max_iter, code.mrow), np.float32), values, sweeps,
                          "802.11ad 1/2 int8, Es/N0 %.2f dB" % snr, n_search, n_valid)
        r["best_table"] = np.asarray(r["best_table"]).astype(int).tolist()
        points.append(r)
        del S, V
    ctx.set_offset_table(None)

    # ---- float offset min-sum, 802.16e rate 1/2 Z=96 (the learned decoder's code) ----
    fcode = codes.make_code("16e 1/2", z_over=96)
    fctx = capi.Context(capi.Code.from_tables(fcode), variant=capi.LDPC_F32_OMS, max_iter=max_iter,
                        max_row_metric=31.0, beta=0.5, llr_scale=1.0, max_abs_llr=1e9)
    kb, fhw = fctx.info.kbits, fctx.info.hard_words
    pw = (2 ** torch.arange(32, dtype=torch.int64, device="cuda"))

    def makef(n, snr, off):
        llr, bits = learned.draw(fctx, fcode, n, [snr], seed, off)
        ref = torch.zeros((n, fhw * 32), dtype=torch.int64, device="cuda")
        ref[:, :kb] = bits[:, :kb].to(torch.int64)
        ref = (ref.view(n, fhw, 32) * pw).sum(dim=2).to(torch.uint32).view(torch.int32)
        del bits
        return llr, ref, n

    hard = torch.empty((f_valid, fhw), dtype=torch.int32, device="cuda")
    its = torch.empty(f_valid, dtype=torch.uint8, device="cuda")

    def runf(table, st):
        nonlocal n_evals
        llr, ref, n = st
        beta = torch.as_tensor(np.full((max_iter, fcode.mrow), 0.5, np.float32) if table is None else
                               np.asarray(table, np.float32), device="cuda").contiguous()
        capi.check(capi.lib.ldpc_learned_decode(fctx.h, llr.data_ptr(), n, max_iter, beta.data_ptr(), None,
                                                hard.data_ptr(), its.data_ptr(), s or None))
        e = int((hard[:n] != ref).any(dim=1).sum())
        n_evals += 1
        return float(its[:n].sum()) / n, e

    for eb in f_ebn0:
        snr = learned.snr_from_ebn0(eb, 0.5)
        S, V = makef(f_search, snr, 0), makef(f_valid, snr, 1 << 36)
        r = _search_point(runf, S, V, np.full((max_iter, fcode.mrow), 0.5, np.float32), f_values, sweeps,
                          "802.16e 1/2 Z=96 float, Eb/N0 %.2f dB (Es/N0 %.2f dB)" % (eb, snr), f_search, f_valid)
        points.append(r)
        del S, V
    return {
        "metric": "average iterations at matched codeword error rate, offset min-sum with searched offset tables "
                  "beta[iteration][layer] vs the plain offset",
        "value": max(p["validation"]["iter_reduction"] for p in points), "unit": "fraction of iterations saved",
        "n_gpus": 1, "higher_is_better": True, "vs_baseline": None, "dtype": "int8 and f32",
        "data": "synthetic: Philox data bits, QC encoding, AWGN from the fused generator, resident in HBM",
        "config": {"workload": "int8: 802.11ad 1/2, LLR scale 2, max|LLR| 24, Max 31, offsets %s, plain 1; float: "
                               "802.16e 1/2 Z=96, Max 31, offsets %s, plain 0.5; %d max iterations; coordinate search, "
                               "%d sweeps per stage (rows, then entries); feasible = codeword errors on the search set "
                               "<= e0 + 2 sqrt(e0)" % (list(values), list(f_values), max_iter, sweeps),
                   "evaluations": n_evals, "search_s": round(time.time() - t_start, 1)},
        "points": points,
        "gpu_launches": n_evals,
    }


def kernel_choice(max_n: int = 1_000_000, llr_bytes: float = 4e8, seed: int = 5, reps: int = 3) -> Dict:
    """int8 decode rate of every named code (802.3ca aside: one decode of it
    outlasts the rest) with the library's kernel choice and with the padded
    register shapes (``LDPC_OMS_PADDED``, the choice for codes without a
    compiled shape before the run-time-table kernel replaced them), at Es/N0
    calibrated to CWER ~1e-3; ldpc_decode_count, best of ``reps`` launches."""
    import os
    s = torch.cuda.current_stream()
    per_code = {}
    for name in [k for k in codes.ENCODE_METHOD if k != "802.3ca"]:
        c = codes.make_code(name)
        h = capi.Code.from_tables(c)
        snr = _calibrate(h, c, n=20_000)
        n = max(20_000, min(max_n, int(llr_bytes // c.n)))
        specs, _ = _build_jobs([h], [c], [n], [[snr]], seed, 10)
        sp = specs[0]
        rates = {}
        for tag, padded in (("default", False), ("padded", True)):
            saved = os.environ.get("LDPC_OMS_PADDED")
            if padded:
                os.environ["LDPC_OMS_PADDED"] = "1"
            else:
                os.environ.pop("LDPC_OMS_PADDED", None)
            try:
                ctx = capi.Context(h, max_iter=10)
            finally:
                if saved is None:
                    os.environ.pop("LDPC_OMS_PADDED", None)
                else:
                    os.environ["LDPC_OMS_PADDED"] = saved
            best = float("inf")
            for _ in range(reps):
                (a, b), = _events(1)
                a.record(s)
                ctx.decode_count(sp["llr"], n, data_bits=sp["data_bits"], ref_period=n, bucket_size=n,
                                 counters=sp["counters"], n_buckets=1, stream=s.cuda_stream)
                b.record(s)
                torch.cuda.synchronize()
                best = min(best, a.elapsed_time(b))
            rates[tag] = n / (best * 1e-3)
            ctx.close()
        per_code[name] = {"snr_db": round(snr, 3), "codewords": n, "default": rates["default"],
                          "padded": rates["padded"], "default_over_padded": rates["default"] / rates["padded"]}
    ratios = [v["default_over_padded"] for v in per_code.values()]
    return {
        "metric": "codewords/s decoded per named code, int8 offset min-sum, 10 max iterations: the library's "
                  "kernel choice against the padded register shapes",
        "value": None, "unit": "codewords/s", "n_gpus": 1, "higher_is_better": True, "dtype": "int8",
        "data": "synthetic: Philox data bits, QC encoding, AWGN from the fused generator, resident in HBM",
        "config": {"workload": "every named MatrixSet but 802.3ca; Es/N0 calibrated to CWER ~1e-3 (2e4 codewords per "
                               "bisection point); min(%d, %.0e / N) codewords per code; best of %d launches"
                               % (max_n, llr_bytes, reps)},
        "default_over_padded_min_max": [min(ratios), max(ratios)],
        "per_code": per_code,
        "gpu_launches": None,
    }
