"""Float decoders on the GPU (sum-product and offset min-sum) vs the oracle:
bit-identical posteriors and iteration counts (tolerance 1e-4 relative on
posteriors is the requirement; the shared tanh/atanh and tree order give 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _float_llr(code, n, snr, seed, oracle):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    cw = oracle.encode(code, info)
    noise = rng.standard_normal(cw.shape, dtype=np.float32)
    lf, _, _ = oracle.llr_array(code, cw, noise, snr, 1.0, 1e9)
    return lf


def _check(capi, oracle, code, llr, mode, mrm, beta, max_iter=10):
    variant = capi.LDPC_F32_SP if mode == 1 else capi.LDPC_F32_OMS
    ctx = capi.Context(capi.Code.from_tables(code), variant=variant, max_iter=max_iter, max_row_metric=mrm,
                       beta=beta, llr_scale=1.0, max_abs_llr=1e9)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_f32(code, llr, mode, max_iter, mrm, beta)
    assert np.array_equal(iters, it_o.astype(np.uint8))
    rel = np.abs(post - post_o) / np.maximum(np.abs(post_o), 1e-30)
    assert rel.max() <= 1e-4
    assert np.array_equal(post.view(np.uint32), post_o.view(np.uint32))
    assert np.array_equal((post < 0), (post_o < 0))


@pytest.mark.parametrize("name,snr,n", [("11ad 1/2", -0.5, 300), ("16e 1/2", 1.0, 200), ("11n 1/2 z81", 1.5, 60),
                                        ("11ay 1/2", -0.25, 100), ("16e 5/6", 4.0, 100), ("ITU G.hn 1/2 z14", 1.0, 300)])
def test_sum_product_matches_oracle(capi, oracle, name, snr, n):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    _check(capi, oracle, code, _float_llr(code, n, snr, 3, oracle), 1, 6e-8, 0.0)


@pytest.mark.parametrize("z", [24, 52, 96])
def test_sum_product_16e_z_sweep(capi, oracle, z):
    from ldpc_b200 import codes
    code = codes.make_code("16e 1/2", z_over=z)
    _check(capi, oracle, code, _float_llr(code, 120, 1.25, z, oracle), 1, 6e-8, 0.0)


@pytest.mark.parametrize("name,snr", [("11ad 1/2", -0.5), ("16e 1/2", 1.0), ("11n 5/6 z81", 4.5)])
def test_float_min_sum_matches_oracle(capi, oracle, name, snr):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    _check(capi, oracle, code, _float_llr(code, 200, snr, 5, oracle), 0, 31.0, 0.5)


@pytest.mark.parametrize("env", ["LDPC_SP_RSMEM", "LDPC_SP_RGLOBAL"])
@pytest.mark.parametrize("mode", [1, 0])
def test_message_placements(capi, oracle, env, mode):
    """Check messages in shared memory and in global scratch (the context
    picks by occupancy; the switches force each placement)."""
    import os
    from ldpc_b200 import codes
    for name, snr in (("16e 1/2", 1.0), ("11ad 1/2", -0.5)):
        code = codes.make_code(name)
        os.environ[env] = "1"
        try:
            llr = _float_llr(code, 150, snr, 7, oracle)
            mrm, beta = (6e-8, 0.0) if mode == 1 else (31.0, 0.5)
            _check(capi, oracle, code, llr, mode, mrm, beta)
        finally:
            os.environ.pop(env, None)


def test_large_code_messages_in_global_memory(capi, oracle):
    """802.3ca (Z=256, 12 x 69): messages exceed shared memory."""
    from ldpc_b200 import codes
    code = codes.make_code("802.3ca")
    _check(capi, oracle, code, _float_llr(code, 6, 3.0, 1, oracle), 1, 6e-8, 0.0, max_iter=4)


def test_float_decode_count_and_generate(capi, oracle):
    """Generator (float LLRs) -> decoder with fused counting agrees with the
    oracle decoding the same LLRs."""
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("16e 1/2", z_over=48)
    ctx = capi.Context(capi.Code.from_tables(code), variant=capi.LDPC_F32_SP, max_row_metric=6e-8, beta=0.0,
                       llr_scale=1.0, max_abs_llr=1e9)
    n = 400
    llr = torch.empty((1, n, code.n), dtype=torch.float32, device="cuda")
    data = torch.empty((n, ctx.info.hard_words), dtype=torch.int32, device="cuda")
    ctx.generate(9, 0, [1.0], n, llr_f32=llr, data_bits=data)
    cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
    ctx.decode_count(llr, n, data_bits=data, ref_period=n, bucket_size=n, counters=cnt, n_buckets=1)
    torch.cuda.synchronize()
    L = llr[0].cpu().numpy()
    post_o, it_o = oracle.decode_f32(code, L, 1, 10, 6e-8, 0.0)
    info = np.unpackbits(data.cpu().numpy().view(np.uint8), axis=1, bitorder="little")[:, :ctx.info.kbits]
    cw = np.concatenate([info, np.zeros((n, code.n - info.shape[1]), np.uint8)], axis=1)
    cwe, be = oracle.count_errors(code, post_o, cw)
    c = cnt.cpu().numpy()[0]
    assert c[0] == n and c[1] == int(it_o.sum()) and c[2] == be and c[3] == cwe


def test_contexts_sharing_a_kernel_keep_their_shared_memory(capi, oracle):
    """Two live contexts whose codes run the same kernel with different
    shared-memory sizes: creating the smaller one must not break launches of
    the larger one (the limit belongs to the kernel, not to a context)."""
    from ldpc_b200 import codes
    big = codes.make_code("16e 1/2", z_over=96)
    small = codes.make_code("16e 1/2", z_over=24)
    kw = dict(variant=capi.LDPC_F32_SP, max_iter=10, max_row_metric=6e-8, beta=0.0, llr_scale=1.0, max_abs_llr=1e9)
    ctx_big = capi.Context(capi.Code.from_tables(big), **kw)
    ctx_small = capi.Context(capi.Code.from_tables(small), **kw)
    for code, ctx in ((big, ctx_big), (small, ctx_small), (big, ctx_big)):
        llr = _float_llr(code, 40, 1.25, 4, oracle)
        post, hard, iters, tot = ctx.decode_host(llr)
        post_o, it_o = oracle.decode_f32(code, llr, 1, 10, 6e-8, 0.0)
        assert np.array_equal(post.view(np.uint32), post_o.view(np.uint32))
    i8 = [codes.code_by_name("5GNR_n3136_k576"), codes.code_by_name("5GNR_n1000_k500")]
    ctxs = [capi.Context(capi.Code.from_tables(c), max_iter=10) for c in i8]
    from conftest import make_llr_int8
    for c, ctx in zip(i8 + i8[:1], ctxs + ctxs[:1]):
        llr, _, _ = make_llr_int8(c, 30, -3.0, seed=2, oracle=oracle)
        post, hard, iters, tot = ctx.decode_host(llr)
        post_o, it_o = oracle.decode_int8(c, llr, 10, 31.0, 1.0)
        assert np.array_equal(post, post_o)
