"""The oracle (scalar C restatement) pinned against the reference's own code:
committed golden vectors from the reference build (tests/golden/ref_vectors.npz),
and live comparisons where the reference build (oracle/_ref) is present."""
import os

import numpy as np
import pytest

from conftest import ROOT

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "ref_vectors.npz"))


@pytest.mark.parametrize("tag,name", [("i8_11ad", "11ad 1/2"), ("i8_16e", "16e 1/2"), ("i8_11n81", "11n 1/2 z81")])
def test_int8_decoder_matches_reference_golden(oracle, tag, name):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    post, it = oracle.decode_int8(code, GOLD[tag + "_llr"], 10, 31.0, 1.0)
    assert np.array_equal(it, GOLD[tag + "_iters"])
    assert np.array_equal(post, GOLD[tag + "_post"])
    post_t, it_t = oracle.decode_int8(code, GOLD[tag + "_llr"], 10, 31.0, 1.0, use_tree=True)
    assert np.array_equal(post_t, post) and np.array_equal(it_t, it)


@pytest.mark.parametrize("tag,mode,mrm,beta", [("f32sp", 1, 6e-8, 0.0), ("f32ms", 0, 31.0, 0.5)])
@pytest.mark.parametrize("ctag,name", [("11ad", "11ad 1/2"), ("16e", "16e 1/2")])
def test_float_decoders_match_reference_golden(oracle, tag, mode, mrm, beta, ctag, name):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    post, it = oracle.decode_f32(code, GOLD["%s_%s_llr" % (tag, ctag)], mode, 10, mrm, beta)
    assert np.array_equal(it, GOLD["%s_%s_iters" % (tag, ctag)])
    assert np.array_equal(post.view(np.uint32), GOLD["%s_%s_post" % (tag, ctag)].view(np.uint32))


@pytest.mark.parametrize("tag,mode,mrm,beta", [("f64sp", 1, 1e-16, 0.0), ("f64ms", 0, 31.0, 0.5)])
@pytest.mark.parametrize("ctag,name", [("11ad", "11ad 1/2"), ("16e", "16e 1/2")])
def test_double_decoders_match_reference_golden(oracle, tag, mode, mrm, beta, ctag, name):
    """LDPCtop_Vec8d_prod / Vec8d_min: double posteriors bit for bit; the
    reference's double LLRs are its float LLRs widened."""
    from ldpc_b200 import codes
    code = codes.make_code(name)
    llr = GOLD["%s_%s_llr" % (tag, ctag)]
    assert llr.dtype == np.float64 and np.array_equal(llr.astype(np.float32).astype(np.float64), llr)
    post, it = oracle.decode_f64(code, llr, mode, 10, mrm, beta)
    assert np.array_equal(it, GOLD["%s_%s_iters" % (tag, ctag)])
    assert np.array_equal(post.view(np.uint64), GOLD["%s_%s_post" % (tag, ctag)].view(np.uint64))


@pytest.mark.parametrize("tag,name", [("i8_11ad", "11ad 1/2"), ("i8_16e", "16e 1/2"), ("i8_11n81", "11n 1/2 z81")])
def test_encoder_matches_reference_golden(oracle, tag, name):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    cw = GOLD[tag + "_cw"]
    kb = code.z * (code.mcol - code.mrow)
    assert np.array_equal(oracle.encode(code, cw[:, :kb]), cw)
    H = code.full_h().astype(np.int64)
    assert not ((cw.astype(np.int64) @ H.T) % 2).any()


def test_llr_quantiser_matches_reference_golden(oracle):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    noise = GOLD["i8_11ad_wgn8"]
    bits = GOLD["i8_11ad_cw"][:8]
    snr = float(GOLD["i8_11ad_snr"][0])
    _, li, _ = oracle.llr_array(code, bits, noise, snr, 2.0, 24.0)
    assert np.array_equal(li, GOLD["i8_11ad_llr"][:8])


def test_oracle_matches_live_reference_build(oracle):
    """Extra codes and parameters against the reference build itself."""
    import refbind as rb
    from ldpc_b200 import codes
    if not rb.ref_available("Vec64c_min"):
        pytest.skip("reference build oracle/_ref absent")
    lib = rb.RefLib("Vec64c_min")
    rng = np.random.default_rng(0)
    for name in ("11ad 13/16", "16e 5/6", "11n 2/3 z54", "11ay 1/2", "ITU G.hn 1/2 z14", "5GNR_n1000_k500"):
        code = codes.code_by_name(name)
        ctx = rb.RefCtx(lib, code, 24)
        llr = rng.integers(-30, 31, (24, code.n)).astype(np.int8) + \
            np.where(rng.random((24, code.n)) < 0.5, 8, -8).astype(np.int8)
        for beta, mrm in ((1.0, 31.0), (0.0, 31.0), (3.0, 15.0)):
            ctx.set_llr(llr)
            it = ctx.decode_each(8, mrm, beta)
            post_o, it_o = oracle.decode_int8(code, llr, 8, mrm, beta)
            assert np.array_equal(it, it_o), (name, beta)
            assert np.array_equal(ctx.posteriors(), post_o), (name, beta)


def test_error_counter_matches_reference_semantics(oracle):
    """LDPC_count_errors: bits compared on data columns, codeword errors per
    interleaved sub-codeword (LDPC_count_errors.cpp:108-130)."""
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2", num_par=3)
    rng = np.random.default_rng(2)
    n = 5
    cw = rng.integers(0, 2, (n, code.n), dtype=np.uint8)
    post = np.where(cw == 1, -5, 5).astype(np.int8)
    post[1, 7] = -post[1, 7]           # one error in sub-codeword 7 % 3 = 1
    post[2, 3] = -post[2, 3]           # two errors in sub-codewords 0 and 2 (positions 3, 5)
    post[2, 5] = -post[2, 5]
    post[3, code.z * (code.mcol - code.mrow) + 1] *= -1   # parity bit: not counted
    cwe, be = oracle.count_errors(code, post, cw)
    assert be == 3 and cwe == 3
