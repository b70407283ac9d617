"""Statistical parity of the whole chain (data bits, QC encoding, AWGN, LLR
quantisation, int8 offset min-sum, error counting): codeword error rates of
ldpc_simulate (Philox noise, GPU) against the reference's own pipeline
(its sfc64/xoshiro generators, normdist2, gen_rand_databits, LDPCencode,
gen_metrics, LDPCdecode_set, LDPC_count_errors; built from its sources, run
on the host), at the reference's default 802.11ad 1/2 point (README.md:41-47).
The two draw different noise, so they must agree within sampling error:
|z| < 4 for the two-proportion test on codeword errors.  Average iterations
and bit error rates are compared with looser bounds (bit errors cluster
within codewords)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SNRS = [-1.0, -0.5]
MAX_ITER, MRM, BETA, SCALE, MAX_ABS = 10, 31.0, 1.0, 2.0, 24.0


def _reference(code, n_per_snr, chunk=20000):
    import refbind as rb
    if not rb.ref_available("Vec64c_min"):
        pytest.skip("reference build absent")
    lib = rb.RefLib("Vec64c_min")
    ctx = rb.RefCtx(lib, code, chunk)
    seeds = (np.arange(64, dtype=np.uint64) + np.uint64(77)) * np.uint64(0x9E3779B97F4A7C15) | np.uint64(1)
    rb.ref_init_randstate(lib, seeds)
    acc = {s: [0, 0, 0, 0] for s in SNRS}      # codewords, cw errors, bit errors, iterations
    for _ in range(n_per_snr // chunk):
        wgn = rb.ref_normdist2(lib, ctx.wgn_count())
        ctx.gen_rand_databits()
        ctx.encode()
        for s in SNRS:                          # the same noise at every SNR point (LDPCtop.cpp:89-97)
            ctx.gen_metrics(s, wgn, SCALE, MAX_ABS)
            it = ctx.decode_set(MAX_ITER, MRM, BETA)
            cwe, be = ctx.count_errors()
            a = acc[s]
            a[0] += chunk
            a[1] += cwe
            a[2] += be
            a[3] += it
    return acc


def test_error_rates_agree_with_reference_pipeline(capi):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    ref = _reference(code, 200_000)
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=MAX_ITER, max_row_metric=MRM, beta=BETA,
                       llr_scale=SCALE, max_abs_llr=MAX_ABS)
    gpu = ctx.simulate(seed=12345, cw_offset=0, snr_db=SNRS, n_per_snr=2_000_000)
    for s, g in zip(SNRS, gpu):
        n1, e1, b1, i1 = ref[s]
        n2, e2 = g["codewords"], g["cw_errors"]
        p1, p2 = e1 / n1, e2 / n2
        p = (e1 + e2) / (n1 + n2)
        z = (p1 - p2) / math.sqrt(p * (1 - p) * (1 / n1 + 1 / n2))
        ber1, ber2 = b1 / (n1 * code.k), g["bit_errors"] / (n2 * code.k)
        it1, it2 = i1 / n1, g["iterations"] / n2
        print("SNR %.2f: CWER ref %.4e gpu %.4e (z=%.2f)  BER ref %.4e gpu %.4e  iters ref %.4f gpu %.4f"
              % (s, p1, p2, z, ber1, ber2, it1, it2))
        assert abs(z) < 4.0
        assert abs(ber1 - ber2) <= 0.15 * ber2
        assert abs(it1 - it2) <= 0.02 * it2
