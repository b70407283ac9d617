#!/usr/bin/env python
"""Headline benchmark: layered int8 offset min-sum decoding of 802.11ad
rate-1/2 codewords (Z=42, N=672, K=336) on B200, codewords per second.

Workload (one step): the reference's default simulation point
(build/run_LDPCsim.pl:8-36, README.md:41-47) -- SNR -1.00..0.00 dB in 0.25 dB
steps, 1e6 codewords per SNR point (5e6 per step per GPU), beta=1,
max_row_metric=31, LLR scale 2, max |LLR| 24, 10 max iterations with
early termination on the syndrome.  Inputs are synthetic: data bits and AWGN
from Philox4x32-10 through the fused generator, resident in HBM before the
timed region (3.36 GB of int8 LLRs per step per GPU, larger than L2).  A
step decodes every codeword with error counting fused (BER/CWER per SNR).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); each rank decodes its own 5e6
codewords (disjoint Philox counters), so scaling is weak and there is no
data-path collective; the timed region is bracketed by barriers and the
slowest rank's device time is reported.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "simd-fecfun_b200"))

CODE = "11ad 1/2"
SNRS = [-1.0, -0.75, -0.5, -0.25, 0.0]
MAX_ITER, MRM, BETA, SCALE, MAX_ABS = 10, 31.0, 1.0, 2.0, 24.0
PUBLISHED_CW_S = 9.0e7   # README.md:5, all processes of a dual-socket Ice Lake server
METRIC = "codewords/s decoded, 802.11ad rate-1/2, int8 offset min-sum, 10 max iterations"
WORKLOAD = ("802.11ad rate 1/2 (Z=42, N=672, K=336); SNR -1.00..0.00 dB step 0.25, 1e6 codewords per SNR; "
            "int8 layered offset min-sum beta=1, max_row_metric=31, LLR scale 2, max|LLR| 24, 10 max iterations, "
            "early termination on the syndrome")


def _clock_sampler(dev_index):
    """nvidia-smi clocks/throttle sampling during the timed region."""
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", "-i", str(dev_index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                              "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None
    return p


def _clock_summary(p):
    if p is None:
        return None
    p.terminate()
    try:
        out, _ = p.communicate(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
        out, _ = p.communicate()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx.append(float(f[2]))
        except ValueError:
            continue
        for nm, v in zip(names, f[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class _quiet_stdout:
    """Silence fd 1 (the reference's loaders print 'Matrix Params' lines;
    bench.py must print exactly one JSON line)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def cpu_reference_rate(llr_sample, threads, per_thread_cw, reps):
    """The reference's own LDPCdecode_set (oracle/_ref build, AVX-512) on host
    threads, one context per thread, decode-only time as the reference's RDTSC
    bracket (LDPCtop.cpp:107-110); the sample is decoded `reps` times (inputs
    restored in between).  Returns (cw/s, iterations of one pass, wall seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refbind as rb
    from ldpc_b200 import codes
    lib = rb.RefLib("Vec64c_min")
    code = codes.make_code(CODE)
    with _quiet_stdout():
        ctxs = [rb.RefCtx(lib, code, per_thread_cw) for _ in range(threads)]
    saved = []
    for k, c in enumerate(ctxs):
        c.set_llr(llr_sample[k * per_thread_cw:(k + 1) * per_thread_cw])
        saved.append(c.metrics.copy())
    iters = [0] * threads
    busy = [0.0] * threads
    wall = 0.0
    for rep in range(reps):
        for c, m in zip(ctxs, saved):
            c.metrics[...] = m
        t0 = [0.0] * threads
        t1 = [0.0] * threads

        def work(k):
            t0[k] = time.perf_counter()
            iters[k] = ctxs[k].decode_set(MAX_ITER, MRM, BETA)
            t1[k] = time.perf_counter()

        th = [threading.Thread(target=work, args=(k,)) for k in range(threads)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall += max(t1) - min(t0)
        for k in range(threads):
            busy[k] += t1[k] - t0[k]
    return reps * threads * per_thread_cw / wall, sum(iters), wall, sum(busy)


def _ref_thread_inputs(rb, lib, code, per, snrs, seed, scale, max_abs):
    """One host thread's sample for a reference build: `per` codewords split
    evenly over every SNR point (one reference context per point), each made by
    the reference's own pipeline (normdist2, gen_rand_databits, LDPCencode,
    gen_metrics) from the thread's seeds.  Every thread decodes the same SNR
    mix as the GPU step."""
    import numpy as np
    each = max(1, per // len(snrs))
    out = []
    for i, snr in enumerate(snrs):
        with _quiet_stdout():
            c = rb.RefCtx(lib, code, each)
        seeds = (np.arange(64, dtype=np.uint64) + np.uint64(seed + 97 * i)) * np.uint64(0x9E3779B97F4A7C15) | np.uint64(1)
        rb.ref_init_randstate(lib, seeds)
        wgn = rb.ref_normdist2(lib, c.wgn_count())
        c.gen_rand_databits()
        c.encode()
        c.gen_metrics(snr, wgn, scale, max_abs)
        out.append(c)
    return out


def run_reference(args):
    """--impl reference: the reference's own CPU path on this box's host cores."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import refbind as rb
    from ldpc_b200 import codes
    if not rb.ref_available("Vec64c_min"):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libref_Vec64c_min.so absent"}))
        return 0
    threads = os.cpu_count() or 1
    lib = rb.RefLib("Vec64c_min")
    code = codes.make_code(CODE)
    # untimed inputs: every thread's sample split evenly over the five SNR points
    ctxs = [_ref_thread_inputs(rb, lib, code, int(args.ref_sample), SNRS, 1000 + 1000 * k, SCALE, MAX_ABS)
            for k in range(threads)]
    for cs in ctxs:
        for c in cs:
            c.saved = c.metrics.copy()
    per = sum(c.num_cw for c in ctxs[0])
    rates = []
    tot_iter = 0
    for step in range(args.warmup + args.steps):
        for cs in ctxs:
            for c in cs:
                c.metrics[...] = c.saved
        t0 = [0.0] * threads
        t1 = [0.0] * threads
        its = [0] * threads

        def work(k):
            t0[k] = time.perf_counter()
            its[k] = sum(c.decode_set(MAX_ITER, MRM, BETA) for c in ctxs[k])
            t1[k] = time.perf_counter()

        th = [threading.Thread(target=work, args=(k,)) for k in range(threads)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if step >= args.warmup:
            rates.append(threads * per / (max(t1) - min(t0)))
            tot_iter += sum(its)
    value = threads * per * len(rates) / sum(threads * per / r for r in rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "codewords/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * threads * per / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_CW_S, "dtype": "int8",
        "data": "synthetic (the reference's own sfc64/xoshiro generators, gen_rand_databits, LDPCencode, gen_metrics)",
        "config": {"workload": WORKLOAD, "sample_per_step": threads * per,
                   "note": "each step decodes a bounded sample of the workload: %d codewords per host thread, "
                           "split evenly over the five SNR points" % per},
        "cpu_baseline": {"value": value, "unit": "codewords/s", "cores": threads, "kind": "reference",
                         "sample": "%d codewords per thread x %d threads per step" % (per, threads)},
        "e2e": {"value": value, "unit": "codewords/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "avg_iterations": tot_iter / (threads * per * len(rates)),
    }
    print(json.dumps(line))
    return 0


def ref_variant_rate(build, mrm, beta, scale, max_abs, threads, per, snrs, max_iter=10):
    """One reference build (oracle/_ref/libref_<build>.so) on host threads:
    inputs through the reference's own pipeline (normdist2,
    gen_rand_databits, LDPCencode, gen_metrics), every thread's sample split
    evenly over the SNR points, untimed; then LDPCdecode_set on every thread at
    once, timed.  Returns (codewords/s, average iterations) or None when the
    build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import refbind as rb
    from ldpc_b200 import codes
    if not rb.ref_available(build):
        return None
    lib = rb.RefLib(build)
    code = codes.make_code(CODE, elem_size=abs(lib.elem_bw))
    ctxs = [_ref_thread_inputs(rb, lib, code, per, snrs, 2000 + 1000 * k, scale, max_abs) for k in range(threads)]
    per = sum(c.num_cw for c in ctxs[0])
    t0 = [0.0] * threads
    t1 = [0.0] * threads
    its = [0] * threads

    def work(k):
        t0[k] = time.perf_counter()
        its[k] = sum(c.decode_set(max_iter, mrm, beta) for c in ctxs[k])
        t1[k] = time.perf_counter()

    th = [threading.Thread(target=work, args=(k,)) for k in range(threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return threads * per / (max(t1) - min(t0)), sum(its) / (threads * per)


def run_variants(args, clk):
    """--workload variants: every decoder variant on the headline 802.11ad
    simulation point, GPU device time beside the reference build of the same
    variant on this box's host cores."""
    from ldpc_b200 import workloads
    rows = workloads.variants(n_per_snr=args.variant_n)
    threads = os.cpu_count() or 1
    for r, run in zip(rows, workloads.VARIANT_RUNS):
        _, _, build, mrm, beta, scale, max_abs = run
        # a bounded CPU sample: fewer codewords for the slower element types
        per = max(64, int(args.variant_ref_sample * {"c": 1.0, "s": 0.5, "w": 0.25, "f": 0.25, "d": 0.1}[build.split("_")[0][-1]]))
        rr = ref_variant_rate(build, mrm, beta, scale, max_abs, threads, per, SNRS)
        if rr is not None:
            r["cpu_reference"] = {"value": rr[0], "unit": "codewords/s", "cores": threads, "kind": "reference",
                                  "avg_iter": rr[1], "sample": "%d codewords x %d threads" % (per, threads)}
            r["speedup_vs_cpu_reference"] = r["value"] / rr[0]
    dsp = rows[-1]
    return {
        "metric": "codewords/s decoded, 802.11ad rate-1/2, each decoder variant, 10 max iterations",
        "value": dsp["value"], "value_is": "double sum-product (the slowest variant); every variant under 'variants'",
        "unit": "codewords/s", "n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "per variant",
        "data": "synthetic: Philox data bits + AWGN from the fused generator, LLRs of each variant's element type",
        "config": {"workload": "802.11ad rate 1/2, SNR -1.00..0.00 dB step 0.25, %d codewords per SNR per variant; "
                               "the Perl driver's parameters per variant" % args.variant_n,
                   "timing": "decoder device time only (CUDA events around each launch in ldpc_simulate)"},
        "gpu_launches": 2 * len(rows) * len(SNRS),
        "variants": rows,
    }


def run_sim(args):
    """--workload sim: the process-level drop-in against the reference's own
    simulator.  ldpc_sim (linked as LDPCtop_Vec64c_min_b200) and the
    reference's LDPCtop_Vec64c_min (built from its sources in oracle/_ref) get
    the same stdin blob parameters (802.11ad 1/2, the Perl driver's defaults,
    SNR -1.00..0.00 dB step 0.25, given seeds); the reference runs one process
    per host core, as its Perl driver does.  Wall-clock time from process
    start to exit covers everything a simulation does: noise and data
    generation, encoding, decoding, error counting and start-up."""
    import tempfile
    from ldpc_b200 import codes, simproto
    code = codes.make_code(CODE)
    seeds = [(0x2545F4914F6CDD1D * (i + 1)) & ((1 << 56) - 1) for i in range(64)]
    n_snr = len(SNRS)
    sim = os.path.join(ROOT, "simd-fecfun_b200", "ldpc_b200", "ldpc_sim")
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "LDPCtop_Vec64c_min")
    out = {}
    with tempfile.TemporaryDirectory() as d:
        code.write_dat(os.path.join(d, "e.dat"), os.path.join(d, "d.dat"))
        exe = os.path.join(d, "LDPCtop_Vec64c_min_b200")
        os.symlink(sim, exe)

        def run(path, per_snr, inner, procs=1):
            data = simproto.blob(1, inner, per_snr // inner, MAX_ITER, MRM, SCALE, MAX_ABS, BETA, SNRS[0], SNRS[-1],
                                 0.25, seeds, "e.dat", "d.dat")
            t0 = time.perf_counter()
            ps = [subprocess.Popen([path], stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                   cwd=d) for _ in range(procs)]
            for p in ps:   # every process gets its blob at once (820 bytes fit the pipe), then all run together
                p.stdin.write(data)
                p.stdin.close()
            outs = [(p.stdout.read(), p.stderr.read()) for p in ps]
            for p in ps:
                p.wait(timeout=900)
            wall = time.perf_counter() - t0
            loops = []
            for p, (o, e) in zip(ps, outs):
                if p.returncode != 0:
                    raise RuntimeError("%s exited %d: %s" % (path, p.returncode, (o + e).decode()[-500:]))
                loops += simproto.parse(o.decode())["loops"]
            cw = procs * (per_snr // inner) * inner * n_snr
            cwe = sum(v[4] for v in loops)
            return {"codewords": cw, "wall_s": wall, "value": cw / wall, "unit": "codewords/s",
                    "cw_errors": cwe, "iterations": sum(v[2] for v in loops)}

        run(exe, 10_000, 10)                       # warm: first-touch of the binary and the CUDA cache
        out["gpu_startup"] = run(exe, 10, 1)        # one tiny run: the fixed cost (process, CUDA, tables), for context
        gpu = run(exe, args.sim_n, 10)
        ref = None
        if os.path.exists(ref_exe):
            threads = os.cpu_count() or 1
            ref = run(ref_exe, args.sim_ref_n, 10, procs=threads)
            ref.update({"cores": threads, "kind": "reference", "sample": "%d processes x %d codewords per SNR"
                        % (threads, args.sim_ref_n)})
    return {
        "metric": "codewords/s simulated by the process-level drop-in (stdin blob to result lines), "
                  "802.11ad rate-1/2, int8 offset min-sum, 10 max iterations",
        "value": gpu["value"], "unit": "codewords/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: each program's own generator (Philox on the GPU; the reference's sfc64/xoshiro and "
                "normdist2 on the host)",
        "config": {"workload": "802.11ad 1/2, SNR -1.00..0.00 dB step 0.25, %d codewords per SNR (GPU), beta=1, "
                               "max_row_metric=31, LLR scale 2, max|LLR| 24, 10 max iterations" % args.sim_n,
                   "timing": "wall clock from process start to exit, start-up included"},
        "ldpc_sim": gpu, "gpu_startup": out["gpu_startup"],
        "cpu_baseline": ref,
        "speedup_vs_reference_processes": gpu["value"] / ref["value"] if ref else None,
        "gpu_launches": None,
    }


def run_workload(args):
    """The other measured workloads (ldpc_b200.workloads), on one GPU; under
    torchrun only rank 0 runs."""
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    import torch
    from ldpc_b200 import workloads
    torch.cuda.set_device(local)
    clk = _clock_sampler(local)
    if args.workload == "nr-mix":
        out = workloads.nr_mix(steps=args.steps, warmup=args.warmup, llr_budget=args.llr_budget_gb * 1e9,
                               autotune=not args.no_autotune)
    elif args.workload == "hetero-mix":
        out = workloads.hetero_mix(steps=args.steps, warmup=args.warmup)
    elif args.workload == "sp-sweep":
        out = workloads.sp_sweep(cw_per_z=args.sp_cw, steps=args.steps, warmup=args.warmup,
                                 autotune=not args.no_autotune)
    elif args.workload == "variants":
        out = run_variants(args, clk)
    elif args.workload == "sim":
        out = run_sim(args)
    elif args.workload == "op-rates":
        from ldpc_b200 import capi
        rates = capi.probe_op_rates(local)
        fma, mufu = capi.probe_fp32_peak(local)
        out = {"metric": "thread-level operations per clock per SM (eight independent chains per thread)",
               "value": None, "unit": "ops/clk/SM", "n_gpus": 1, "dtype": "packed int8/int16/f16 and f32",
               "rates": {k: round(v, 2) for k, v in rates},
               "int32_ops_per_s": capi.probe_int32_peak(local), "fp32_fma_per_s": fma, "mufu_per_s": mufu,
               "gpu_launches": None}
    elif args.workload == "kernel-choice":
        out = workloads.kernel_choice()
    elif args.workload == "offset-search":
        out = workloads.offset_search(n_search=args.search_n, n_valid=args.search_valid_n)
    else:
        out = workloads.learned_run(train_steps=max(args.steps, 2), batch=args.learned_batch,
                                    weights=args.learned_weights)
    out["clocks"] = _clock_summary(clk)
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-per-snr", type=int, default=1_000_000)
    ap.add_argument("--ref-sample", type=int, default=20000, help="codewords per host thread per reference step")
    ap.add_argument("--cpu-sample", type=int, default=30000, help="codewords per host thread for the CPU baseline")
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--variant-n", type=int, default=200_000, help="codewords per SNR per variant (--workload variants)")
    ap.add_argument("--sim-n", type=int, default=100_000_000, help="codewords per SNR for ldpc_sim (--workload sim)")
    ap.add_argument("--sim-ref-n", type=int, default=100_000,
                    help="codewords per SNR per reference process (--workload sim)")
    ap.add_argument("--variant-ref-sample", type=int, default=4000,
                    help="int8 codewords per host thread for the reference builds (--workload variants)")
    ap.add_argument("--workload", default="11ad",
                    choices=["11ad", "nr-mix", "hetero-mix", "learned", "sp-sweep", "variants", "sim", "offset-search",
                             "op-rates", "kernel-choice"],
                    help="11ad: the headline run; others: the batched 5G NR mix, the 18-code 802.11 mix "
                         "(plain vs learned offsets), learned-offset training, the float sum-product Z sweep, "
                         "every decoder variant on the headline point, the process-level drop-in against the "
                         "reference's own simulator (one GPU)")
    ap.add_argument("--llr-budget-gb", type=float, default=40.0, help="nr-mix: LLR bytes the codeword counts are scaled to")
    ap.add_argument("--no-autotune", action="store_true", help="nr-mix: default launch shape")
    ap.add_argument("--learned-batch", type=int, default=65536)
    ap.add_argument("--search-n", type=int, default=4_000_000, help="offset-search: codewords of the search set")
    ap.add_argument("--search-valid-n", type=int, default=20_000_000,
                    help="offset-search: fresh codewords that validate the best table")
    ap.add_argument("--learned-weights", default="uniform", choices=["uniform", "early", "steep"])
    ap.add_argument("--sp-cw", type=int, default=1 << 20, help="sp-sweep: codewords per Z")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "11ad":
        return run_workload(args)

    import numpy as np
    import torch
    from ldpc_b200 import capi, codes, sharding

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    code = codes.make_code(CODE)
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=MAX_ITER, max_row_metric=MRM, beta=BETA,
                       llr_scale=SCALE, max_abs_llr=MAX_ABS, device=local)
    N, HW = ctx.info.n, ctx.info.hard_words
    nps = args.n_per_snr
    nsnr = len(SNRS)
    total = nsnr * nps
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    # ---- inputs, resident in HBM (untimed): Philox data + AWGN, all SNR points share the noise
    llr = torch.empty((nsnr, nps, N), dtype=torch.int8, device="cuda")
    data = torch.empty((nps, HW), dtype=torch.int32, device="cuda")
    unc = torch.zeros(nsnr, dtype=torch.int64, device="cuda")
    # this rank's share of the global codeword range (disjoint Philox counters)
    cw_start, _ = sharding.weak_shard(nps, rank, ws)
    ctx.generate(seed=2024, cw_offset=cw_start, snr_db=SNRS, n_per_snr=nps, llr_i8=llr, data_bits=data,
                 uncoded=unc, stream=sptr)
    # the generator itself (untimed for the headline): the same call again, timed by events;
    # algorithmic bytes = the int8 LLRs of every SNR point + the packed data bits
    gen_ms = []
    for _ in range(3):
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        ctx.generate(seed=2024, cw_offset=cw_start, snr_db=SNRS, n_per_snr=nps, llr_i8=llr, data_bits=data,
                     uncoded=unc, stream=sptr)
        g1.record(stream)
        torch.cuda.synchronize()
        gen_ms.append(g0.elapsed_time(g1))
    gen_bytes = total * N + nps * HW * 4
    generation = {"kernel": "gen_kernel", "ms": statistics.median(gen_ms), "bytes": gen_bytes,
                  "achieved_gbs": gen_bytes / (statistics.median(gen_ms) * 1e-3) / 1e9,
                  "what": "%d codewords: data bits, QC encoding, one AWGN draw per bit, int8 LLRs at %d SNR points"
                          % (nps, nsnr)}
    hard = torch.empty((total, HW), dtype=torch.int32, device="cuda")
    iters = torch.empty(total, dtype=torch.uint8, device="cuda")
    counters = torch.zeros((nsnr, 4), dtype=torch.int64, device="cuda")

    def step():
        ctx.decode_count(llr, total, hard=hard, iters=iters, data_bits=data, ref_period=nps, bucket_size=nps,
                         counters=counters, n_buckets=nsnr, stream=sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    counters.zero_()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = _clock_sampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_stop = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    t_stop.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = _clock_summary(clk)
    elapsed_ms = t_start.elapsed_time(t_stop)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    c_all, elapsed_ms = sharding.finish_run(counters, elapsed_ms)
    cnt = c_all.cpu().numpy()
    value = ws * total * args.steps / (elapsed_ms * 1e-3)
    ms_per_step = elapsed_ms / args.steps

    quality = []
    kbits = ctx.info.kbits
    for s_i, snr in enumerate(SNRS):
        cw, it, be, ce = (int(v) for v in cnt[s_i])
        quality.append({"snr_db": snr, "codewords": cw, "avg_iter": it / max(cw, 1), "ber": be / max(cw * kbits, 1),
                        "cwer": ce / max(cw, 1)})

    # ---- roofline of the decode kernel (the only kernel of a step)
    E = ctx.info.edges
    iters_per_launch = float(cnt[:, 1].sum()) / args.steps / ws
    avg_launch_s = statistics.mean(launch_ms) * 1e-3
    ops_per_launch = iters_per_launch * E * 2.5           # 10 int8 lane-ops per edge-iteration, 4 lanes per int32 op
    peak = capi.probe_int32_peak(local)
    bytes_per_cw = N + 4 * HW + 1
    traffic = None
    pipe = None
    prof = os.path.join(ROOT, "profiles", "decode_11ad_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            p = json.load(f)
        traffic = p["dram_bytes_per_codeword"] * total
        if "alu_pipe_pct" in p:
            # what the hardware executes, beside the 2.5-op-per-edge definition of "achieved"
            pipe = {"alu_pipe_active": p["alu_pipe_pct"] / 100, "issue_active": p["issue_active_pct"] / 100,
                    "thread_instructions_per_edge_per_codeword": p["warp_instructions"] * 32.0
                    / (p["codeword_iterations"] * p["edges_per_codeword"]),
                    "source": "ncu --set full of this kernel (profiles/oms_f16_11ad_small_ncu.md)"}
    roofline = {
        "bound": "alu", "achieved": ops_per_launch / avg_launch_s / 1e12, "peak": peak / 1e12, "unit": "Tops/s (int32)",
        "frac": ops_per_launch / avg_launch_s / peak, "traffic": traffic,
        "peak_source": "own microbenchmark of independent 32-bit lop3/iadd chains on this GPU (ldpc_probe_int32_peak)",
        "ops_definition": "sum over codewords of edges(2184) x iterations x 2.5 packed int32 ops (10 int8 lane-ops per "
                          "edge-iteration, 4 lanes per 32-bit op)",
        "hbm": {"achieved_gbs": bytes_per_cw * total / avg_launch_s / 1e9, "bytes_per_codeword": bytes_per_cw},
    }
    if pipe:
        roofline["pipe"] = pipe
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hbm_peak = json.load(f)["hbm_gbs"]
        roofline["hbm"]["peak_gbs"] = hbm_peak
        roofline["hbm"]["frac"] = roofline["hbm"]["achieved_gbs"] / hbm_peak
        roofline["hbm"]["peak_source"] = "MEASURED_PEAKS.json (measured)"
        generation["frac_of_hbm"] = generation["achieved_gbs"] / hbm_peak
    except (OSError, KeyError, ValueError):
        pass

    # ---- end to end through the host-memory C-ABI (pinned in, results out)
    e2e = None
    if not args.no_e2e:
        h_llr = torch.empty((total, N), dtype=torch.int8, pin_memory=True)
        h_llr.copy_(llr.view(total, N))
        h_hard = torch.empty((total, HW), dtype=torch.int32, pin_memory=True)
        h_it = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        a_llr, a_hard, a_it = h_llr.numpy(), h_hard.numpy().view(np.uint32), h_it.numpy()
        import ctypes as C
        tot = C.c_uint64()

        def e2e_step():
            capi.check(capi.lib.ldpc_decode_int8_host(ctx.h, a_llr.ctypes.data, total, None, a_hard.ctypes.data,
                                                      a_it.ctypes.data, C.byref(tot)))

        e2e_step()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        t1 = time.perf_counter()
        e2e_s = t1 - t0
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": ws * total * args.steps / e2e_s, "unit": "codewords/s", "h2d_bytes_per_step": total * N,
               "d2h_bytes_per_step": total * (4 * HW + 1),
               "path": "ldpc_decode_int8_host: pinned host LLRs -> chunked H2D / decode / D2H of hard bits and "
                       "iteration counts on two streams"}
        del h_llr, h_hard, h_it

    # ---- CPU baseline: the reference's own decoder on this box's host cores (rank 0, N=1)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import refbind as rb
        if rb.ref_available("Vec64c_min"):
            threads = os.cpu_count() or 1
            per = int(args.cpu_sample)
            take = -(-threads * per // nsnr)
            take = min(take, nps)
            per = min(per, take * nsnr // threads)
            sample = torch.cat([llr[s_i, :take] for s_i in range(nsnr)]).cpu().numpy()
            gpu_it = torch.cat([iters[s_i * nps:s_i * nps + take] for s_i in range(nsnr)]).cpu().numpy()
            rate, ref_iters, wall, busy = cpu_reference_rate(sample, threads, per, args.cpu_reps)
            cpu = {"value": rate, "unit": "codewords/s", "cores": threads, "kind": "reference",
                   "sample": "%d threads x %d codewords x %d passes, taken from the first %d codewords of each SNR "
                             "point of this step's inputs; decode-only time of the reference's LDPCdecode_set "
                             "built from its own sources (AVX-512)" % (threads, per, args.cpu_reps, take),
                   "cpu_seconds": busy}
            # the same inputs on both sides: iteration totals must agree
            cpu["same_inputs_total_iterations_equal"] = int(ref_iters) == int(
                gpu_it[:threads * per].astype(np.int64).sum())

    line = {
        "metric": METRIC, "value": value, "unit": "codewords/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_CW_S, "dtype": "int8",
        "data": "synthetic: Philox4x32-10 data bits + Box-Muller AWGN from the fused generator, resident in HBM",
        "config": {"workload": WORKLOAD, "codewords_per_step_per_gpu": total, "parallelism": "dp%d (codeword shards)" % ws,
                   "l2": "inputs larger than L2 (%.2f GB of LLRs per step per GPU)" % (total * N / 1e9),
                   "info_gbps": value * 336 / 1e9},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps, "clocks": clocks,
        "quality": quality, "generation": generation,
    }
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
