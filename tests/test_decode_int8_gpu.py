"""int8 offset min-sum decoder on the GPU vs the oracle: bit-exact posteriors,
hard decisions and per-codeword iteration counts (the reference's
LDPCdecode_set semantics, src/LDPCDec/LDPCdecode.cpp:79-245)."""
import numpy as np
import pytest

from conftest import make_llr_int8, pack_bits

pytestmark = pytest.mark.gpu


def _ctx(capi, code, **kw):
    return capi.Context(capi.Code.from_tables(code), **kw)


def _check(capi, oracle, code, llr, max_iter=10, mrm=31.0, beta=1.0):
    ctx = _ctx(capi, code, max_iter=max_iter, max_row_metric=mrm, beta=beta)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, max_iter, mrm, beta)
    assert np.array_equal(iters, it_o.astype(np.uint8))
    assert np.array_equal(post, post_o)
    kb = ctx.info.kbits
    assert np.array_equal(hard, pack_bits((post_o[:, :kb] < 0).astype(np.uint8)))
    assert tot == int(it_o.sum())


@pytest.mark.parametrize("snr", [-1.0, -0.5, 0.0, 2.0])
def test_11ad_half_matches_oracle(capi, oracle, snr):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr, _, _ = make_llr_int8(code, 3000, snr, seed=11 + int(snr * 4), oracle=oracle)
    _check(capi, oracle, code, llr)


@pytest.mark.parametrize("name,snr", [("16e 1/2", 1.0), ("11n 1/2 z27", 1.0), ("11n 1/2 z81", 1.5),
                                      ("ITU G.hn 1/2 z14", 1.0), ("11ad 5/8", 1.0), ("11ad 3/4", 2.5),
                                      ("11ad 13/16", 3.5), ("16e 2/3A", 2.0), ("16e 3/4B", 3.0),
                                      ("16e 5/6", 4.0), ("11n 5/6 z81", 4.5)])
def test_other_codes_match_oracle(capi, oracle, name, snr):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    llr, _, _ = make_llr_int8(code, 600, snr, seed=5, oracle=oracle)
    _check(capi, oracle, code, llr)


def test_saturation_and_random_llrs(capi, oracle):
    """Full-range int8 LLRs: saturating Q and P paths, non-converging words."""
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    rng = np.random.default_rng(3)
    llr = rng.integers(-128, 128, (500, code.n)).astype(np.int8)
    _check(capi, oracle, code, llr)
    big = np.where(rng.random((500, code.n)) < 0.5, -128, 127).astype(np.int8)
    _check(capi, oracle, code, big)


@pytest.mark.parametrize("beta,mrm,max_iter", [(0.0, 31.0, 10), (2.0, 20.0, 10), (1.0, 127.0, 5), (1.0, 31.0, 1),
                                               (1.0, 31.0, 20), (0.0, 5e-8, 10)])
def test_parameters(capi, oracle, beta, mrm, max_iter):
    """beta = 0 (int8 abs(-128) quirk), other clamps, max_iter edge cases."""
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr, _, _ = make_llr_int8(code, 800, -0.5, seed=21, max_abs=100.0, scale=8.0, oracle=oracle)
    _check(capi, oracle, code, llr, max_iter=max_iter, mrm=mrm, beta=beta)


@pytest.mark.parametrize("n", [0, 1, 29, 30, 31, 61, 4441])
def test_ragged_counts(capi, oracle, n):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr, _, _ = make_llr_int8(code, max(n, 1), -1.0, seed=n, oracle=oracle)
    llr = llr[:n]
    if n == 0:
        ctx = _ctx(capi, code)
        post, hard, iters, tot = ctx.decode_host(np.zeros((0, code.n), np.int8))
        assert tot == 0 and iters.size == 0
        return
    _check(capi, oracle, code, llr)


def test_device_api_and_num_par(capi, oracle):
    """Device-pointer entry point (torch buffers) and a num_par=2 super-code."""
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2", num_par=2, elem_size=8)
    llr, _, _ = make_llr_int8(code, 700, -0.5, seed=9, oracle=oracle)
    ctx = _ctx(capi, code)
    d_llr = torch.from_numpy(llr).cuda()
    post = torch.empty_like(d_llr)
    hard = torch.empty((llr.shape[0], ctx.info.hard_words), dtype=torch.int32, device="cuda")
    iters = torch.empty(llr.shape[0], dtype=torch.uint8, device="cuda")
    ctx.decode_int8(d_llr, llr.shape[0], post, hard, iters)
    torch.cuda.synchronize()
    post_o, it_o = oracle.decode_int8(code, llr, 10, 31.0, 1.0)
    assert np.array_equal(post.cpu().numpy(), post_o)
    assert np.array_equal(iters.cpu().numpy(), it_o.astype(np.uint8))


def test_compat_reference_layout(capi, oracle):
    """ldpc_decode_set_compat: the reference's padded in-place layout."""
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    n, P = 300, 64
    llr, _, _ = make_llr_int8(code, n, -0.75, seed=2, oracle=oracle)
    spz = (code.z + P - 1) // P
    buf = np.zeros((n, code.mcol, (spz + 2) * P), np.int8)
    buf[:, :, P:P + code.z] = llr.reshape(n, code.mcol, code.z)
    ctx = _ctx(capi, code)
    tot = ctx.decode_set_compat(buf, n, P)
    post_o, it_o = oracle.decode_int8(code, llr, 10, 31.0, 1.0)
    assert tot == int(it_o.sum())
    assert np.array_equal(buf[:, :, P:P + code.z].reshape(n, code.n), post_o)


def test_unaligned_llr_pointer(capi, oracle):
    """Device LLRs starting at an odd address take the byte-copy prefetch path."""
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr, _, _ = make_llr_int8(code, 200, -0.5, seed=13, oracle=oracle)
    ctx = _ctx(capi, code)
    buf = torch.zeros(llr.size + 1, dtype=torch.int8, device="cuda")
    buf[1:] = torch.from_numpy(llr.ravel()).cuda()
    iters = torch.empty(llr.shape[0], dtype=torch.uint8, device="cuda")
    post = torch.empty(llr.shape, dtype=torch.int8, device="cuda")
    ctx.decode_int8(buf.data_ptr() + 1, llr.shape[0], post, None, iters)
    torch.cuda.synchronize()
    post_o, it_o = oracle.decode_int8(code, llr, 10, 31.0, 1.0)
    assert np.array_equal(post.cpu().numpy(), post_o)
    assert np.array_equal(iters.cpu().numpy(), it_o.astype(np.uint8))


def test_fused_error_counting(capi, oracle):
    """ldpc_decode_count: per-bucket codewords/iterations/bit and codeword errors."""
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    n = 1500
    llr, info, _ = make_llr_int8(code, n, -1.0, seed=17, oracle=oracle)
    ctx = _ctx(capi, code)
    data = torch.from_numpy(pack_bits(info).view(np.int32)).cuda()
    cnt = torch.zeros((3, 4), dtype=torch.int64, device="cuda")
    ctx.decode_count(torch.from_numpy(llr).cuda(), n, data_bits=data, ref_period=n, bucket_size=500, counters=cnt,
                     n_buckets=3)
    torch.cuda.synchronize()
    post_o, it_o = oracle.decode_int8(code, llr, 10, 31.0, 1.0)
    c = cnt.cpu().numpy()
    for b in range(3):
        sl = slice(500 * b, 500 * (b + 1))
        cw_err, bit_err = oracle.count_errors(code, post_o[sl], np.concatenate(
            [info[sl], np.zeros((500, code.n - info.shape[1]), np.uint8)], axis=1))
        assert c[b, 0] == 500 and c[b, 1] == int(it_o[sl].sum())
        assert c[b, 2] == bit_err and c[b, 3] == cw_err
