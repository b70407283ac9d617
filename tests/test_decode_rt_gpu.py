"""int8 offset min-sum over run-time code tables on the GPU vs the oracle:
codes without a compiled register shape (802.11ay, 802.3ca, 5G NR base
graphs 1 and 2) and, forced, codes that have one; bit-exact posteriors, hard
decisions and iteration counts.  5G NR also through the float decoders and
the generator (encoder with direct parity columns, puncture and filler
masks)."""
import os

import numpy as np
import pytest

from conftest import make_llr_int8, pack_bits

pytestmark = pytest.mark.gpu


def _ctx_env(capi, code, env=None, **kw):
    """Context created with tuning variables set (they are read at creation)."""
    saved = {k: os.environ.get(k) for k in (env or {})}
    os.environ.update(env or {})
    try:
        return capi.Context(capi.Code.from_tables(code), **kw)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _check(capi, oracle, code, llr, max_iter=10, mrm=31.0, beta=1.0, env=None):
    ctx = _ctx_env(capi, code, env, max_iter=max_iter, max_row_metric=mrm, beta=beta)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, max_iter, mrm, beta)
    assert np.array_equal(iters, it_o.astype(np.uint8))
    assert np.array_equal(post, post_o)
    kb = ctx.info.kbits
    assert np.array_equal(hard, pack_bits((post_o[:, :kb] < 0).astype(np.uint8)))
    assert tot == int(it_o.sum())
    return it_o


@pytest.mark.parametrize("name,snr,n,max_iter", [
    ("11ay 1/2", -0.25, 600, 10), ("11ay 5/8", 1.0, 400, 10), ("802.3ca", 3.0, 16, 10),
    ("5GNR_n25344_k8448", -4.2, 12, 20),      # base graph 1, Z=384, full 46 rows
    ("5GNR_n3136_k576", -6.0, 200, 20),       # base graph 2, Z=64, fillers
    ("5GNR_n6400_k1280", -6.3, 80, 20),       # base graph 2, Z=128
    ("5GNR_n12800_k2560", -6.5, 30, 20),      # base graph 2, Z=256
    ("5GNR_n1000_k500", -1.0, 300, 20), ("5GNR_n300_k100", -3.0, 600, 20),
    ("5GNR_n10000_k8000", 2.5, 40, 20),
])
def test_runtime_tables_match_oracle(capi, oracle, name, snr, n, max_iter):
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    llr, _, _ = make_llr_int8(code, n, snr, seed=3, oracle=oracle)
    it = _check(capi, oracle, code, llr, max_iter=max_iter)
    assert it.max() > 1     # not all trivially converged


@pytest.mark.parametrize("env", [{"LDPC_OMS_RT": "1"}, {"LDPC_OMS_RT": "1", "LDPC_OMS_RT_GLOBAL": "1"}],
                         ids=["smem", "global"])
@pytest.mark.parametrize("name,snr", [("11ad 1/2", -0.5), ("16e 1/2", 1.0), ("11n 5/6 z81", 4.5),
                                      ("ITU G.hn 1/2 z14", 1.0)])
def test_forced_runtime_kernel(capi, oracle, env, name, snr):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    llr, _, _ = make_llr_int8(code, 700, snr, seed=8, oracle=oracle)
    _check(capi, oracle, code, llr, env=env)


@pytest.mark.parametrize("name,snr", [("16e 1/2", 1.0), ("11n 5/6 z81", 4.5), ("ITU G.hn 1/2 z14", 1.0),
                                      ("11ad 13/16", 3.4)])
def test_padded_register_shapes(capi, oracle, name, snr):
    """The padded register shapes (PaddedShape<L, D>), which run only when
    LDPC_OMS_PADDED asks for them (the run-time-table kernel is the faster
    default for these codes)."""
    from ldpc_b200 import codes
    code = codes.make_code(name)
    llr, _, _ = make_llr_int8(code, 500, snr, seed=9, oracle=oracle)
    _check(capi, oracle, code, llr, env={"LDPC_OMS_PADDED": "1"})


@pytest.mark.parametrize("env", [None, {"LDPC_OMS_RT": "1", "LDPC_OMS_RT_GLOBAL": "1"}], ids=["default", "rt_global"])
@pytest.mark.parametrize("beta,mrm,max_iter", [(0.0, 31.0, 10), (2.0, 20.0, 7), (1.0, 127.0, 1), (0.0, 5e-8, 10)])
def test_runtime_parameters_and_saturation(capi, oracle, beta, mrm, max_iter, env):
    """beta = 0 (the abs8(-128) quirk), clamps, max_iter = 1, full-range LLRs;
    the default kernel and the run-time-table kernel with global messages."""
    from ldpc_b200 import codes
    code = codes.code_by_name("5GNR_n1000_k500")
    llr, _, _ = make_llr_int8(code, 300, -1.0, seed=21, max_abs=100.0, scale=8.0, oracle=oracle)
    _check(capi, oracle, code, llr, max_iter=max_iter, mrm=mrm, beta=beta, env=env)
    rng = np.random.default_rng(4)
    big = np.where(rng.random((200, code.n)) < 0.5, -128, 127).astype(np.int8)
    _check(capi, oracle, code, big, max_iter=max_iter, mrm=mrm, beta=beta, env=env)


@pytest.mark.parametrize("n", [1, 5, 33, 1001])
def test_runtime_ragged_counts(capi, oracle, n):
    from ldpc_b200 import codes
    code = codes.make_code("11ay 1/2")
    llr, _, _ = make_llr_int8(code, n, -0.5, seed=n, oracle=oracle)
    _check(capi, oracle, code, llr)


def test_runtime_fused_error_counting(capi, oracle):
    import torch
    from ldpc_b200 import codes
    code = codes.code_by_name("5GNR_n3136_k576")
    n = 600
    llr, info, _ = make_llr_int8(code, n, -6.2, seed=17, oracle=oracle)
    ctx = _ctx_env(capi, code, max_iter=20)
    data = torch.from_numpy(pack_bits(info).view(np.int32)).cuda()
    cnt = torch.zeros((2, 4), dtype=torch.int64, device="cuda")
    ctx.decode_count(torch.from_numpy(llr).cuda(), n, data_bits=data, ref_period=n, bucket_size=300, counters=cnt,
                     n_buckets=2)
    torch.cuda.synchronize()
    post_o, it_o = oracle.decode_int8(code, llr, 20, 31.0, 1.0)
    c = cnt.cpu().numpy()
    for b in range(2):
        sl = slice(300 * b, 300 * (b + 1))
        cw_err, bit_err = oracle.count_errors(code, post_o[sl], np.concatenate(
            [info[sl], np.zeros((300, code.n - info.shape[1]), np.uint8)], axis=1))
        assert c[b, 0] == 300 and c[b, 1] == int(it_o[sl].sum())
        assert c[b, 2] == bit_err and c[b, 3] == cw_err


def _float_llr(oracle, code, n, snr, seed):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    cw = oracle.encode(code, info)
    noise = rng.standard_normal(cw.shape, dtype=np.float32)
    lf, _, _ = oracle.llr_array(code, cw, noise, snr, 1.0, 1e9)
    return lf


@pytest.mark.parametrize("name,snr,n,mode", [("5GNR_n3136_k576", -6.0, 60, 1), ("5GNR_n1000_k500", -1.0, 100, 1),
                                             ("5GNR_n1000_k500", -1.0, 100, 0), ("5GNR_n25344_k8448", -4.2, 4, 1)])
def test_nr_float_decoders_match_oracle(capi, oracle, name, snr, n, mode):
    """5G NR through the float decoders (tolerance 1e-4 relative; 0 observed)."""
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    llr = _float_llr(oracle, code, n, snr, 5)
    variant = capi.LDPC_F32_SP if mode == 1 else capi.LDPC_F32_OMS
    mrm, beta = (6e-8, 0.0) if mode == 1 else (31.0, 0.5)
    ctx = capi.Context(capi.Code.from_tables(code), variant=variant, max_iter=12, max_row_metric=mrm, beta=beta,
                       llr_scale=1.0, max_abs_llr=1e9)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_f32(code, llr, mode, 12, mrm, beta)
    assert np.array_equal(iters, it_o.astype(np.uint8))
    rel = np.abs(post - post_o) / np.maximum(np.abs(post_o), 1e-30)
    assert rel.max() <= 1e-4
    assert np.array_equal(post.view(np.uint32), post_o.view(np.uint32))


@pytest.mark.parametrize("name", ["5GNR_n25344_k8448", "5GNR_n3136_k576", "5GNR_n1000_k500", "5GNR_n10000_k8000"])
def test_nr_generator_matches_oracle(capi, oracle, name):
    """Encoder (direct parity columns 1 and 3 + substitution rows) and the LLR
    quantiser with puncture (LLR 0) and filler (+max) masks."""
    import torch
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=20)
    rng = np.random.default_rng(6)
    n = 40
    info = rng.integers(0, 2, (n, code.z * (code.mcol - code.mrow)), dtype=np.uint8)
    for s, e in zip(code.fill_list[0::2], code.fill_list[1::2]):
        info[:, s:e + 1] = 0
    d = torch.from_numpy(pack_bits(info).view(np.int32)).cuda()
    out = torch.empty((n, code.n), dtype=torch.uint8, device="cuda")
    ctx.encode(d, n, out)
    torch.cuda.synchronize()
    cw = out.cpu().numpy()
    assert np.array_equal(cw, oracle.encode(code, info))
    assert not code.syndrome(cw[:4]).any()
    noise = rng.standard_normal((n, code.n), dtype=np.float32)
    lf, li, errs = oracle.llr_array(code, cw, noise, -2.0, 2.0, 24.0)
    d_i8 = torch.empty((n, code.n), dtype=torch.int8, device="cuda")
    unc = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.llr_from_noise(torch.from_numpy(cw).cuda(), torch.from_numpy(noise).cuda(), n, -2.0, d_i8, None, unc)
    torch.cuda.synchronize()
    assert np.array_equal(d_i8.cpu().numpy(), li)
    assert int(unc.item()) == errs


def test_nr_generate_and_simulate(capi):
    """Fused generation on 5G NR: filler data bits are zero, punctured LLRs are
    0, filler LLRs +max; a short simulation decodes at a working SNR."""
    import torch
    from ldpc_b200 import codes
    code = codes.code_by_name("5GNR_n3136_k576")
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=20)
    n = 256
    llr = torch.empty((1, n, code.n), dtype=torch.int8, device="cuda")
    data = torch.empty((n, ctx.info.hard_words), dtype=torch.int32, device="cuda")
    ctx.generate(7, 0, [-3.0], n, llr_i8=llr, data_bits=data)
    torch.cuda.synchronize()
    l = llr.cpu().numpy()[0]
    fs, fe = code.fill_list
    ps, pe = code.punc_list[:2]
    assert (l[:, ps:pe + 1] == 0).all() and (l[:, fs:fe + 1] == 24).all()
    bits = np.unpackbits(data.cpu().numpy().view(np.uint8), axis=1, bitorder="little")
    assert not bits[:, fs:fe + 1].any()
    st = ctx.simulate(seed=3, cw_offset=0, snr_db=[-3.0], n_per_snr=2000)[0]
    assert st["codewords"] == 2000 and st["cw_errors"] == 0 and st["iterations"] >= 2000


@pytest.mark.parametrize("name,snr", [("11ad 1/2", -0.5), ("5GNR_n1000_k500", -1.0)])
def test_context_layer_offsets(capi, oracle, name, snr):
    """ldpc_ctx_set_layer_offsets: one int8 offset per layer (0 included),
    then back to cfg.beta (for 11ad, back onto the compiled kernel)."""
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    llr, _, _ = make_llr_int8(code, 400, snr, seed=31, oracle=oracle)
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=12, beta=1.0)
    b = np.arange(code.mrow, dtype=np.float32) % 4 + np.float32(0.5)      # truncated to 0..3
    ctx.set_layer_offsets(b)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, 12, 31.0, beta_layers=b.astype(np.int8))
    assert np.array_equal(post, post_o) and np.array_equal(iters, it_o.astype(np.uint8))
    ctx.set_layer_offsets(None)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, 12, 31.0, 1.0)
    assert np.array_equal(post, post_o) and np.array_equal(iters, it_o.astype(np.uint8))
    with pytest.raises(capi.LdpcError):
        ctx.set_layer_offsets(np.full(code.mrow, 300.0, np.float32))


@pytest.mark.parametrize("name,snr,rows", [("11ad 1/2", -0.5, 12), ("11ad 1/2", -0.5, 3), ("5GNR_n1000_k500", -1.0, 20)])
def test_context_offset_table(capi, oracle, name, snr, rows):
    """ldpc_ctx_set_offset_table: iteration i uses row min(i, rows-1) (rows
    shorter than max_iter included), offsets 0..3 with zeros (the abs8(-128)
    quirk); then the per-layer form replaces it, and None restores beta."""
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    max_iter = 12 if rows != 20 else 20
    llr, _, _ = make_llr_int8(code, 500, snr, seed=41, oracle=oracle)
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=max_iter, beta=1.0)
    rng = np.random.default_rng(rows)
    tab = rng.integers(0, 4, (rows, code.mrow)).astype(np.float32) + np.float32(0.25)
    tab[0, 0] = 0.0
    ctx.set_offset_table(tab)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, max_iter, 31.0, beta_table=tab.astype(np.int8))
    assert np.array_equal(iters, it_o.astype(np.uint8)) and np.array_equal(post, post_o)
    kb = ctx.info.kbits
    assert np.array_equal(hard, pack_bits((post_o[:, :kb] < 0).astype(np.uint8)))
    ctx.set_layer_offsets(tab[1])
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, max_iter, 31.0, beta_layers=tab[1].astype(np.int8))
    assert np.array_equal(iters, it_o.astype(np.uint8)) and np.array_equal(post, post_o)
    ctx.set_offset_table(None)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_int8(code, llr, max_iter, 31.0, 1.0)
    assert np.array_equal(iters, it_o.astype(np.uint8)) and np.array_equal(post, post_o)
    with pytest.raises(capi.LdpcError):
        ctx.set_offset_table(np.full((2, code.mrow), 128.0, np.float32))
