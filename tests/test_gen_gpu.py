"""Generation path on the GPU: QC encoder and LLR quantiser bit-exact with
the oracle (and, where its build is present, with the reference's own
LDPCencode/gen_metrics); Philox/Box-Muller noise checked statistically."""
import numpy as np
import pytest

from conftest import pack_bits

pytestmark = pytest.mark.gpu

# 802.3ca: 22355 schedule terms (its dense inverse), read from device memory
CODES = ["11ad 1/2", "11ad 13/16", "11ay 13/16", "16e 1/2", "16e 5/6", "11n 1/2 z27", "11n 3/4 z81",
         "ITU G.hn 1/2 z14", "802.3ca"]


def _ctx(capi, code, **kw):
    return capi.Context(capi.Code.from_tables(code), **kw)


@pytest.mark.parametrize("name", CODES)
def test_encode_matches_oracle(capi, oracle, name):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code(name)
    try:
        ctx = _ctx(capi, code)
    except capi.LdpcError as e:
        if e.code != capi.LDPC_ERR_UNSUPPORTED:
            raise
        ctx = _ctx(capi, code, variant=capi.LDPC_F32_SP, max_row_metric=6e-8, beta=0.0, llr_scale=1.0,
                   max_abs_llr=1e9)
    rng = np.random.default_rng(4)
    n = 257
    info = rng.integers(0, 2, (n, code.z * (code.mcol - code.mrow)), dtype=np.uint8)
    d = torch.from_numpy(pack_bits(info).view(np.int32)).cuda()
    out = torch.empty((n, code.n), dtype=torch.uint8, device="cuda")
    ctx.encode(d, n, out)
    torch.cuda.synchronize()
    cw = out.cpu().numpy()
    assert np.array_equal(cw, oracle.encode(code, info))
    H = code.full_h().astype(np.int64)
    assert not ((cw[:8].astype(np.int64) @ H.T) % 2).any()


@pytest.mark.parametrize("snr,scale,max_abs", [(-1.0, 2.0, 24.0), (0.5, 2.0, 24.0), (3.0, 4.0, 100.0), (1.0, 1.0, 1e9)])
def test_llr_from_noise_matches_oracle(capi, oracle, snr, scale, max_abs):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    ctx = _ctx(capi, code, llr_scale=scale, max_abs_llr=max_abs)
    rng = np.random.default_rng(7)
    n = 400
    bits = rng.integers(0, 2, (n, code.n), dtype=np.uint8)
    noise = rng.standard_normal((n, code.n), dtype=np.float32) * np.float32(1.5)
    lf, li, errs = oracle.llr_array(code, bits, noise, snr, scale, max_abs)
    d_i8 = torch.empty((n, code.n), dtype=torch.int8, device="cuda")
    d_f = torch.empty((n, code.n), dtype=torch.float32, device="cuda")
    unc = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.llr_from_noise(torch.from_numpy(bits).cuda(), torch.from_numpy(noise).cuda(), n, snr, d_i8, d_f, unc)
    torch.cuda.synchronize()
    if max_abs <= 127:
        assert np.array_equal(d_i8.cpu().numpy(), li)
    assert np.array_equal(d_f.cpu().numpy().view(np.uint32), lf.view(np.uint32))
    assert int(unc.item()) == errs


def test_llr_matches_reference_gen_metrics(capi):
    """The reference's own gen_metrics (oracle/_ref build) on the same noise."""
    import torch
    import refbind as rb
    from ldpc_b200 import codes
    if not rb.ref_available("Vec64c_min"):
        pytest.skip("reference build absent")
    lib = rb.RefLib("Vec64c_min")
    code = codes.make_code("11ad 1/2")
    n = 64
    ref = rb.RefCtx(lib, code, n)
    rng = np.random.default_rng(1)
    info = rng.integers(0, 2, (n, code.z * 8), dtype=np.uint8)
    ref.set_info_bits(info)
    ref.encode()
    cw = ref.codeword_bits()
    zb = (code.z + 7) // 8 * 8                       # gen_metrics reads 8 noise floats per byte
    wgn = np.zeros((n, code.mcol, zb), np.float32)
    wgn[:, :, :code.z] = rng.standard_normal((n, code.mcol, code.z), dtype=np.float32)
    flat_wgn = np.zeros(ref.wgn_count() * 8, np.float32)
    flat_wgn[:wgn.size] = wgn.ravel()
    unc_ref = ref.gen_metrics(-0.5, flat_wgn, 2.0, 24.0)
    llr_ref = ref.posteriors()
    ctx = _ctx(capi, code)
    d_i8 = torch.empty((n, code.n), dtype=torch.int8, device="cuda")
    unc = torch.zeros(1, dtype=torch.int64, device="cuda")
    noise = np.ascontiguousarray(wgn[:, :, :code.z].reshape(n, code.n))
    ctx.llr_from_noise(torch.from_numpy(cw).cuda(), torch.from_numpy(noise).cuda(), n, -0.5, d_i8, None, unc)
    torch.cuda.synchronize()
    assert np.array_equal(d_i8.cpu().numpy(), llr_ref)
    assert int(unc.item()) == unc_ref


def test_generate_consistency_and_noise_statistics(capi, oracle):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    snrs = np.array([-1.0, 0.0, 2.0], np.float32)
    ctx = _ctx(capi, code, llr_scale=1.0, max_abs_llr=1e30)
    n = 20000
    llr = torch.empty((len(snrs), n, code.n), dtype=torch.float32, device="cuda")
    data = torch.empty((n, ctx.info.hard_words), dtype=torch.int32, device="cuda")
    unc = torch.zeros(len(snrs), dtype=torch.int64, device="cuda")
    ctx.generate(123, 1000, snrs, n, llr_f32=llr, data_bits=data, uncoded=unc)
    torch.cuda.synchronize()
    L = llr.cpu().numpy()
    dbits = data.cpu().numpy().view(np.uint32)
    info = np.unpackbits(dbits.view(np.uint8), axis=1, bitorder="little")[:, :ctx.info.kbits]
    cw = oracle.encode(code, info)
    orig = 1.0 - 2.0 * cw
    for k, snr in enumerate(snrs):
        sigma, sf = oracle.sigma(float(snr), 1.0)
        noise = (L[k] / sf - orig) / sigma
        assert abs(noise.mean()) < 5e-3
        assert abs(noise.var() - 1.0) < 5e-3
        frac_tail = np.mean(np.abs(noise) > 3.0)
        assert abs(frac_tail - 2.6998e-3) < 3e-4
        assert int(unc[k].item()) == int(((L[k] < 0) != (orig < 0)).sum())
    # the same noise at every SNR point
    n0 = (L[0] / oracle.sigma(-1.0, 1.0)[1] - orig) / oracle.sigma(-1.0, 1.0)[0]
    n2 = (L[2] / oracle.sigma(2.0, 1.0)[1] - orig) / oracle.sigma(2.0, 1.0)[0]
    assert np.abs(n0 - n2).max() < 1e-3
    # data bits are uniform
    assert abs(info.mean() - 0.5) < 2e-3
    # counter-based: a different offset gives different data, the same offset the same
    data2 = torch.empty_like(data)
    ctx.generate(123, 1000 + 7, snrs[:1], 16, llr_f32=llr[0], data_bits=data2)
    torch.cuda.synchronize()
    assert np.array_equal(data2.cpu().numpy()[:9], data.cpu().numpy()[7:16])


@pytest.mark.parametrize("variant,bits,scale,max_abs", [("Vec32s_min", 16, 40.0, 1000.0), ("Vec16w_min", 32, 4000.0, 1e6)])
def test_integer_llrs_match_reference_gen_metrics(capi, variant, bits, scale, max_abs):
    """int16 / int32 LLRs (roundi, then compress for int16) against the
    reference's gen_metrics of the matching build, on the same noise."""
    import torch
    import refbind as rb
    from ldpc_b200 import codes
    if not rb.ref_available(variant):
        pytest.skip("reference build absent")
    lib = rb.RefLib(variant)
    code = codes.make_code("11ad 1/2", elem_size=bits)
    n = 48
    ref = rb.RefCtx(lib, code, n)
    rng = np.random.default_rng(2)
    ref.set_info_bits(rng.integers(0, 2, (n, code.z * 8), dtype=np.uint8))
    ref.encode()
    cw = ref.codeword_bits()
    zb = (code.z + 7) // 8 * 8
    wgn = np.zeros((n, code.mcol, zb), np.float32)
    wgn[:, :, :code.z] = rng.standard_normal((n, code.mcol, code.z), dtype=np.float32)
    flat = np.zeros(ref.wgn_count() * 8, np.float32)
    flat[:wgn.size] = wgn.ravel()
    unc_ref = ref.gen_metrics(0.25, flat, scale, max_abs)
    llr_ref = ref.posteriors()
    ctx = capi.Context(capi.Code.from_tables(code), variant=capi.LDPC_INT16_OMS if bits == 16 else capi.LDPC_INT32_OMS,
                       llr_scale=scale, max_abs_llr=max_abs)
    dt = torch.int16 if bits == 16 else torch.int32
    out = torch.empty((n, code.n), dtype=dt, device="cuda")
    unc = torch.zeros(1, dtype=torch.int64, device="cuda")
    noise = np.ascontiguousarray(wgn[:, :, :code.z].reshape(n, code.n))
    ctx.llr_from_noise(torch.from_numpy(cw).cuda(), torch.from_numpy(noise).cuda(), n, 0.25, llr_int=out, uncoded=unc)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), llr_ref)
    assert int(unc.item()) == unc_ref
    # the fused generator quantises the same way: its int16/int32 LLRs decode in simulate
    st = ctx.simulate(seed=5, cw_offset=0, snr_db=[1.0], n_per_snr=5000)[0]
    assert st["codewords"] == 5000 and st["iterations"] >= 5000


@pytest.mark.parametrize("name,n", [("11ad 1/2", 3000), ("16e 1/2", 2000), ("11n 5/6 z81", 1500),
                                    ("5GNR_n3136_k576", 1000), ("5GNR_n1000_k500", 1000), ("5GNR_n25344_k8448", 120),
                                    ("5GNR_n2048_k704 bg1 z32", 1000), ("802.3ca", 64)])
def test_generate_int8_path_matches_float_path(capi, name, n):
    """The generator's int8-only path (four LLRs rounded and packed per word,
    uncoded errors from sign masks) against its general path on the same
    seed: identical data bits and uncoded counts, and int8 LLRs equal to the
    float LLRs rounded half-even.  Covers the per-thread encoder (Z <= 64, no
    filler bits), the warp encoder (larger Z or filler bits, and 802.3ca's
    schedule in device memory), puncturing and filler LLRs."""
    import torch
    from ldpc_b200 import codes
    if name.endswith("bg1 z32"):   # Z = 32 without filler bits: the per-thread encoder with puncturing
        code = codes.code_by_name(name.split()[0], bg=1, z=32)
    else:
        code = codes.code_by_name(name)
    ctx = capi.Context(capi.Code.from_tables(code), max_iter=10, max_row_metric=31.0, beta=1.0, llr_scale=2.0,
                       max_abs_llr=24.0)
    snrs = np.array([-1.0, 0.5, 3.0], np.float32)
    hw = ctx.info.hard_words
    lf = torch.empty((len(snrs), n, code.n), dtype=torch.float32, device="cuda")
    li = torch.empty((len(snrs), n, code.n), dtype=torch.int8, device="cuda")
    d1 = torch.empty((n, hw), dtype=torch.int32, device="cuda")
    d2 = torch.empty_like(d1)
    u1 = torch.zeros(len(snrs), dtype=torch.int64, device="cuda")
    u2 = torch.zeros_like(u1)
    ctx.generate(77, 5000, snrs, n, llr_f32=lf, data_bits=d1, uncoded=u1)
    ctx.generate(77, 5000, snrs, n, llr_i8=li, data_bits=d2, uncoded=u2)
    torch.cuda.synchronize()
    assert torch.equal(d1, d2)
    assert torch.equal(u1, u2)
    F = lf.cpu().numpy()
    assert np.array_equal(li.cpu().numpy(), np.rint(F).astype(np.int16).astype(np.int8))
    if code.punc_list:
        assert np.all(F[:, :, code.punc_list[0]:code.punc_list[1] + 1] == 0)
