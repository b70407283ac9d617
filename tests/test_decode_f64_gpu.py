"""Double sum-product and double offset min-sum (the reference's
LDPCtop_Vec8d_prod / LDPCtop_Vec8d_min) on the GPU: bit-exact posteriors,
hard decisions and per-codeword iteration counts against the oracle's double
decoder, the committed golden vectors of the reference build, and the
reference build itself where oracle/_ref is present; large codes whose
double posteriors leave no room for the staging buffer; the generator's
double LLRs (the float LLRs widened, gen_metrics.cpp:91-93)."""
import os

import numpy as np
import pytest

from conftest import ROOT, pack_bits

pytestmark = pytest.mark.gpu

# the Perl driver's parameters: clamp 1 - 1e-16 for d_prod (run_LDPCsim.pl:56-63)
MODES = {1: ("Vec8d_prod", 1e-16, 0.0), 0: ("Vec8d_min", 31.0, 0.5)}


def _llr(oracle, code, n, snr, seed):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    for s, e in zip(code.fill_list[0::2], code.fill_list[1::2]):
        info[:, s:e + 1] = 0
    cw = oracle.encode(code, info)
    noise = rng.standard_normal(cw.shape, dtype=np.float32)
    lf, _, _ = oracle.llr_array(code, cw, noise, snr, 1.0, 1e9)
    return lf.astype(np.float64), info


def _ctx(capi, code, mode, max_iter=10, mrm=None, beta=None):
    _, m, b = MODES[mode]
    return capi.Context(capi.Code.from_tables(code), variant=capi.LDPC_F64_SP if mode == 1 else capi.LDPC_F64_OMS,
                        max_iter=max_iter, max_row_metric=m if mrm is None else mrm, beta=b if beta is None else beta,
                        llr_scale=1.0, max_abs_llr=1e9)


def _check(capi, oracle, code, llr, mode, max_iter=10, mrm=None, beta=None):
    _, m, b = MODES[mode]
    m = m if mrm is None else mrm
    b = b if beta is None else beta
    ctx = _ctx(capi, code, mode, max_iter, m, b)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_o, it_o = oracle.decode_f64(code, llr, mode, max_iter, m, b)
    assert np.array_equal(iters, it_o.astype(np.uint8))
    assert np.array_equal(post.view(np.uint64), post_o.view(np.uint64))
    kb = ctx.info.kbits
    assert np.array_equal(hard, pack_bits((post_o[:, :kb] < 0).astype(np.uint8)))
    assert tot == int(it_o.sum())
    return it_o


@pytest.mark.parametrize("mode", [1, 0])
@pytest.mark.parametrize("name,snr,n", [("11ad 1/2", -0.5, 300), ("16e 1/2", 1.0, 300), ("11n 5/6 z81", 3.0, 120),
                                        ("11ay 1/2", -0.25, 200), ("ITU G.hn 1/2 z14", 1.0, 400),
                                        ("5GNR_n3136_k576", -6.0, 40)])
def test_matches_oracle(capi, oracle, mode, name, snr, n):
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    llr, _ = _llr(oracle, code, n, snr, 11)
    it = _check(capi, oracle, code, llr, mode)
    assert it.max() > 1


@pytest.mark.parametrize("mode", [1, 0])
@pytest.mark.parametrize("ctag,name", [("11ad", "11ad 1/2"), ("16e", "16e 1/2")])
def test_matches_reference_golden(capi, mode, ctag, name):
    """Inputs and outputs of the reference's own double build (committed)."""
    from ldpc_b200 import codes
    g = np.load(os.path.join(ROOT, "tests", "golden", "ref_vectors.npz"))
    tag = "f64sp" if mode == 1 else "f64ms"
    code = codes.make_code(name)
    ctx = _ctx(capi, code, mode)
    post, hard, iters, tot = ctx.decode_host(g["%s_%s_llr" % (tag, ctag)])
    assert np.array_equal(iters, g["%s_%s_iters" % (tag, ctag)].astype(np.uint8))
    assert np.array_equal(post.view(np.uint64), g["%s_%s_post" % (tag, ctag)].view(np.uint64))


@pytest.mark.parametrize("mode", [1, 0])
def test_matches_live_reference_build(capi, oracle, mode):
    import refbind as rb
    from ldpc_b200 import codes
    variant, mrm, beta = MODES[mode]
    if not rb.ref_available(variant):
        pytest.skip("reference build %s absent" % variant)
    lib = rb.RefLib(variant)
    for name, snr in (("11n 2/3 z54", 2.5), ("11ay 5/8", 1.0), ("16e 3/4A", 2.0), ("5GNR_n1000_k500", -1.0)):
        code = codes.code_by_name(name, elem_size=64)
        llr, _ = _llr(oracle, code, 24, snr, 4)
        ref = rb.RefCtx(lib, code, 24)
        ref.set_llr(llr)
        it_r = ref.decode_each(10, mrm, beta)
        post, hard, iters, tot = _ctx(capi, code, mode).decode_host(llr)
        assert np.array_equal(iters, it_r.astype(np.uint8)), name
        assert np.array_equal(post.view(np.uint64), ref.posteriors().view(np.uint64)), name


@pytest.mark.parametrize("mode", [1, 0])
@pytest.mark.parametrize("name,snr,n", [("5GNR_n25344_k8448", -4.2, 4), ("802.3ca", 3.0, 4)])
def test_large_codes_without_staging(capi, oracle, mode, name, snr, n):
    """5G NR base graph 1 at Z=384 and 802.3ca: the double posteriors fill the
    CTA's shared memory, so a codeword slot is refilled from global memory."""
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    llr, _ = _llr(oracle, code, n, snr, 7)
    _check(capi, oracle, code, llr, mode, max_iter=6)


@pytest.mark.parametrize("beta,mrm,max_iter", [(0.0, 6e-8, 10), (0.75, 1e-9, 1), (0.0, 0.9999, 20)])
def test_parameters(capi, oracle, beta, mrm, max_iter):
    """Sum-product with an offset, the clamp above and below 1e-6, one iteration."""
    from ldpc_b200 import codes
    code = codes.make_code("16e 1/2")
    llr, _ = _llr(oracle, code, 200, 0.8, 3)
    _check(capi, oracle, code, llr, 1, max_iter=max_iter, mrm=mrm, beta=beta)


@pytest.mark.parametrize("n", [1, 7, 129])
def test_ragged_counts_device_api_and_counting(capi, oracle, n):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr, info = _llr(oracle, code, n, -0.5, n)
    ctx = _ctx(capi, code, 1)
    d = torch.from_numpy(llr).cuda()
    post = torch.empty_like(d)
    iters = torch.empty(n, dtype=torch.uint8, device="cuda")
    ctx.decode_f64(d, n, post=post, iters=iters)
    cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
    data = torch.from_numpy(pack_bits(info).view(np.int32)).cuda()
    ctx.decode_count(d, n, data_bits=data, ref_period=n, bucket_size=n, counters=cnt, n_buckets=1)
    torch.cuda.synchronize()
    post_o, it_o = oracle.decode_f64(code, llr, 1, 10, 1e-16, 0.0)
    assert np.array_equal(post.cpu().numpy().view(np.uint64), post_o.view(np.uint64))
    assert np.array_equal(iters.cpu().numpy(), it_o.astype(np.uint8))
    cw_err, bit_err = oracle.count_errors(code, post_o, np.concatenate(
        [info, np.zeros((n, code.n - info.shape[1]), np.uint8)], axis=1))
    assert cnt.cpu().numpy()[0].tolist() == [n, int(it_o.sum()), bit_err, cw_err]


def test_generator_writes_widened_float_llrs(capi):
    import torch
    from ldpc_b200 import codes
    code = codes.code_by_name("5GNR_n1000_k500")
    ctx = _ctx(capi, code, 1)
    n, snr = 64, [-1.0, 0.5]
    l64 = torch.empty((2, n, code.n), dtype=torch.float64, device="cuda")
    l32 = torch.empty((2, n, code.n), dtype=torch.float32, device="cuda")
    ctx.generate(seed=5, cw_offset=0, snr_db=snr, n_per_snr=n, llr_int=l64, llr_f32=l32)
    torch.cuda.synchronize()
    assert torch.equal(l64, l32.double())
    st = ctx.simulate(seed=5, cw_offset=0, snr_db=snr, n_per_snr=2000)
    assert [s["codewords"] for s in st] == [2000, 2000] and st[0]["cw_errors"] >= st[1]["cw_errors"]


def test_wrong_element_type_and_batches_are_refused(capi):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    ctx = _ctx(capi, code, 1)
    with pytest.raises(capi.LdpcError):
        ctx.decode_host(np.zeros((2, code.n), np.float32))
    h = capi.Code.from_tables(code)
    with pytest.raises(capi.LdpcError):
        capi.Batch([h], [dict(variant=capi.LDPC_F64_SP, max_row_metric=1e-16, beta=0.0)])
