"""Golden vectors from the reference's own code (oracle/_ref build).

Runs the reference's decoders (LDPCdecode_set, int8 min-sum / float
and double sum-product / float and double min-sum), encoder (LDPCencode) and LLR generator
(gen_metrics) -- all built from its unmodified sources by
``make -C oracle ref`` -- on seeded inputs and stores inputs and outputs in
``ref_vectors.npz``.  The CPU tests check the oracle against these without
needing the reference tree.

    make -C oracle ref && python tests/golden/make_ref_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "simd-fecfun_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import refbind as rb  # noqa: E402
from ldpc_b200 import codes  # noqa: E402


def ref_pipeline(lib, code, n, snr, scale, max_abs, seed):
    ctx = rb.RefCtx(lib, code, n)
    seeds = (np.arange(64, dtype=np.uint64) + np.uint64(seed)) * np.uint64(0x9E3779B97F4A7C15) | np.uint64(1)
    rb.ref_init_randstate(lib, seeds)
    wgn = rb.ref_normdist2(lib, ctx.wgn_count())
    ctx.gen_rand_databits()
    ctx.encode()
    unc = ctx.gen_metrics(snr, wgn, scale, max_abs)
    return ctx, wgn, unc


def main():
    out = {}
    # int8 offset min-sum (LDPCtop_Vec64c_min defaults) on three codes
    lib = rb.RefLib("Vec64c_min")
    for tag, name, snr, n in (("i8_11ad", "11ad 1/2", -0.5, 96), ("i8_16e", "16e 1/2", 1.0, 32),
                              ("i8_11n81", "11n 1/2 z81", 1.5, 16)):
        code = codes.make_code(name)
        ctx, wgn, unc = ref_pipeline(lib, code, n, snr, 2.0, 24.0, 5)
        llr = ctx.posteriors()
        cw = ctx.codeword_bits()
        it = ctx.decode_each(10, 31.0, 1.0)
        out[tag + "_llr"] = llr
        out[tag + "_post"] = ctx.posteriors()
        out[tag + "_iters"] = it
        out[tag + "_cw"] = cw
        if tag == "i8_11ad":
            # gen_metrics check: noise and LLRs of the first 8 codewords
            # (8 noise floats per byte of Z, per column: gen_metrics.cpp:35-60)
            zb = (code.z + 7) // 8 * 8
            out[tag + "_wgn8"] = wgn[:8 * code.mcol * zb].reshape(8, code.mcol, zb)[:, :, :code.z].reshape(8, code.n)
        out[tag + "_snr"] = np.array([snr], np.float32)
    # float sum-product and float min-sum (16-lane tables)
    for variant, tag, mode, mrm, beta in (("Vec16f_prod", "f32sp", 1, 6e-8, 0.0), ("Vec16f_min", "f32ms", 0, 31.0, 0.5)):
        lib = rb.RefLib(variant)
        for ctag, name, snr, n in (("11ad", "11ad 1/2", -0.5, 16), ("16e", "16e 1/2", 1.0, 8)):
            code = codes.make_code(name, elem_size=32)
            ctx, wgn, unc = ref_pipeline(lib, code, n, snr, 1.0, 1e9, 9)
            llr = ctx.posteriors()
            it = ctx.decode_each(10, mrm, beta)
            out["%s_%s_llr" % (tag, ctag)] = llr
            out["%s_%s_post" % (tag, ctag)] = ctx.posteriors()
            out["%s_%s_iters" % (tag, ctag)] = it
    # double sum-product (the Perl driver's clamp for d_prod, run_LDPCsim.pl:59)
    # and double min-sum (8-lane tables); gen_metrics widens the float LLRs to
    # double (gen_metrics.cpp:91-93)
    for variant, tag, mode, mrm, beta in (("Vec8d_prod", "f64sp", 1, 1e-16, 0.0), ("Vec8d_min", "f64ms", 0, 31.0, 0.5)):
        lib = rb.RefLib(variant)
        for ctag, name, snr, n in (("11ad", "11ad 1/2", -0.5, 16), ("16e", "16e 1/2", 1.0, 8)):
            code = codes.make_code(name, elem_size=64)
            ctx, wgn, unc = ref_pipeline(lib, code, n, snr, 1.0, 1e9, 9)
            llr = ctx.posteriors()
            it = ctx.decode_each(10, mrm, beta)
            out["%s_%s_llr" % (tag, ctag)] = llr
            out["%s_%s_post" % (tag, ctag)] = ctx.posteriors()
            out["%s_%s_iters" % (tag, ctag)] = it
    np.savez_compressed(os.path.join(HERE, "ref_vectors.npz"), **out)


if __name__ == "__main__":
    main()
