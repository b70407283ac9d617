"""int16 and int32 offset min-sum on the GPU against the reference's own
LDPCtop_Vec32s_min / LDPCtop_Vec16w_min decoders (built from its sources in
oracle/_ref): bit-exact posteriors, hard decisions and per-codeword iteration
counts, including saturated inputs at the element limits and beta = 0 (abs
of the most negative value is itself)."""
import numpy as np
import pytest

from conftest import pack_bits

pytestmark = pytest.mark.gpu

VARIANTS = {16: ("Vec32s_min", np.int16, 3), 32: ("Vec16w_min", np.int32, 4)}


def _reference(bits, code, llr, max_iter, mrm, beta):
    import refbind as rb
    name, dt, _ = VARIANTS[bits]
    if not rb.ref_available(name):
        pytest.skip("reference build %s absent" % name)
    lib = rb.RefLib(name)
    ctx = rb.RefCtx(lib, code, llr.shape[0])
    ctx.set_llr(llr)
    it = ctx.decode_each(max_iter, mrm, beta)
    return ctx.posteriors(), it


def _llr(code, n, bits, scale, lim, seed, oracle):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    cw = oracle.encode(code, info)
    y = (1.0 - 2.0 * cw) + 0.9 * rng.standard_normal(cw.shape)
    return np.clip(np.rint(y * scale), -lim, lim).astype(VARIANTS[bits][1])


def _check(capi, code, llr, bits, max_iter=10, mrm=31.0, beta=1.0):
    ctx = capi.Context(capi.Code.from_tables(code), variant=VARIANTS[bits][2], max_iter=max_iter,
                       max_row_metric=mrm, beta=beta)
    post, hard, iters, tot = ctx.decode_host(llr)
    post_r, it_r = _reference(bits, code, llr, max_iter, mrm, beta)
    assert np.array_equal(iters, it_r.astype(np.uint8))
    assert np.array_equal(post, post_r)
    kb = ctx.info.kbits
    assert np.array_equal(hard, pack_bits((post_r[:, :kb] < 0).astype(np.uint8)))
    assert tot == int(it_r.sum())


@pytest.mark.parametrize("bits", [16, 32])
@pytest.mark.parametrize("name", ["11ad 1/2", "16e 1/2", "11n 5/6 z81", "ITU G.hn 1/2 z14", "5GNR_n1000_k500",
                                  "5GNR_n3136_k576"])
def test_matches_reference_decoder(capi, oracle, bits, name):
    from ldpc_b200 import codes
    code = codes.code_by_name(name, elem_size=bits)  # the reference build's SIMD layout
    llr = _llr(code, 150, bits, 40.0, 1000, 3, oracle)
    _check(capi, code, llr, bits, mrm=400.0, beta=7.0)


@pytest.mark.parametrize("bits", [16, 32])
@pytest.mark.parametrize("beta,mrm,max_iter", [(0.0, 31.0, 10), (3.0, 5e-8, 10), (1.0, 1e4, 1), (0.0, 1e4, 20)])
def test_limits_and_parameters(capi, oracle, bits, beta, mrm, max_iter):
    """Inputs at the element limits (saturating add/sub, the abs quirk)."""
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2", elem_size=bits)
    info = np.iinfo(VARIANTS[bits][1])
    rng = np.random.default_rng(bits + max_iter)
    big = np.where(rng.random((120, code.n)) < 0.5, info.min, info.max).astype(VARIANTS[bits][1])
    _check(capi, code, big, bits, max_iter=max_iter, mrm=mrm, beta=beta)
    llr = _llr(code, 120, bits, 3000.0, info.max, 5, oracle)
    _check(capi, code, llr, bits, max_iter=max_iter, mrm=mrm, beta=beta)


def test_large_code_and_device_api(capi, oracle):
    """802.3ca (messages in global scratch) through the device entry point."""
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("802.3ca", elem_size=16)
    llr = _llr(code, 6, 16, 30.0, 500, 9, oracle)
    ctx = capi.Context(capi.Code.from_tables(code), variant=capi.LDPC_INT16_OMS, max_iter=5, max_row_metric=200.0,
                       beta=2.0)
    d = torch.from_numpy(llr).cuda()
    post = torch.empty_like(d)
    iters = torch.empty(llr.shape[0], dtype=torch.uint8, device="cuda")
    ctx.decode_int16(d, llr.shape[0], post, None, iters)
    torch.cuda.synchronize()
    post_r, it_r = _reference(16, code, llr, 5, 200.0, 2.0)
    assert np.array_equal(post.cpu().numpy(), post_r)
    assert np.array_equal(iters.cpu().numpy(), it_r.astype(np.uint8))
