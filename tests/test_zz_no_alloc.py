"""ldpc_decode_f32_noalloc (static device scratch, no context) against the
context path ldpc_decode_f32 on the same inputs, through the C ABI.

Tolerance: posteriors within 1e-4 relative (the float decoders' stated
tolerance); hard decisions and iteration counts identical.  Both paths run
the same kernel arithmetic, so the posteriors are expected to agree bit for
bit.  Each case calls the no-alloc entry point twice in a row, so the second
call reuses a scratch array the first one left dirty."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _llr(o, code, n, snr, seed):
    """BPSK + AWGN float LLRs of random codewords at `snr` dB ([n][N]); the
    oracle encodes and quantises them."""
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    cw = o.encode(code, info)
    noise = rng.standard_normal(cw.shape, dtype=np.float32)
    lf, _, _ = o.llr_array(code, cw, noise, snr, 1.0, 1e9)
    return lf


def _noalloc(capi, torch, code_h, cfg, llr_d, n, N, hw):
    post = torch.full((n, N), float("nan"), dtype=torch.float32, device="cuda")
    hard = torch.full((n, hw), -1, dtype=torch.int32, device="cuda")
    iters = torch.full((n,), 255, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    capi.check(capi.lib.ldpc_decode_f32_noalloc(code_h.h, C.byref(cfg), llr_d.data_ptr(), n, post.data_ptr(),
                                                hard.data_ptr(), iters.data_ptr(), s or None))
    torch.cuda.synchronize()
    return post.cpu().numpy(), hard.cpu().numpy().view(np.uint32), iters.cpu().numpy()


@pytest.mark.parametrize("name,variant,snr,n,mrm,beta,max_iter", [
    ("802.3ca", "sp", 3.0, 240, 6e-8, 0.0, 4),          # messages beyond shared memory; grid capped by the scratch
    ("11ad 1/2", "sp", -0.5, 3000, 6e-8, 0.0, 10),
    ("11n 5/6 z81", "oms", 4.5, 1000, 31.0, 0.5, 10),
])
def test_noalloc_matches_context_path(capi, oracle, name, variant, snr, n, mrm, beta, max_iter):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code(name)
    ch = capi.Code.from_tables(code)
    v = capi.LDPC_F32_SP if variant == "sp" else capi.LDPC_F32_OMS
    ctx = capi.Context(ch, variant=v, max_iter=max_iter, max_row_metric=mrm, beta=beta, llr_scale=1.0,
                       max_abs_llr=1e9)
    N, hw = ch.info.n, ch.info.hard_words
    llr = _llr(oracle, code, n, snr, 11)
    llr_d = torch.from_numpy(llr).cuda()

    post_r = torch.empty((n, N), dtype=torch.float32, device="cuda")
    hard_r = torch.empty((n, hw), dtype=torch.int32, device="cuda")
    iters_r = torch.empty((n,), dtype=torch.uint8, device="cuda")
    ctx.decode_f32(llr_d.data_ptr(), n, post_r.data_ptr(), hard_r.data_ptr(), iters_r.data_ptr(),
                   torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    post_r, hard_r, iters_r = post_r.cpu().numpy(), hard_r.cpu().numpy().view(np.uint32), iters_r.cpu().numpy()
    assert iters_r.min() >= 1

    cfg = capi.Cfg(v, max_iter, mrm, beta, 1.0, 1e9)
    for _ in range(2):
        post, hard, iters = _noalloc(capi, torch, ch, cfg, llr_d, n, N, hw)
        assert np.array_equal(iters, iters_r)
        assert np.array_equal(hard, hard_r)
        np.testing.assert_allclose(post, post_r, rtol=1e-4, atol=0)
        assert np.array_equal(post.view(np.uint32), post_r.view(np.uint32))


def test_noalloc_rejects_int8_and_bad_config(capi):
    from ldpc_b200 import codes
    ch = capi.Code.from_tables(codes.make_code("11ad 1/2"))
    for cfg in (capi.Cfg(capi.LDPC_INT8_OMS, 10, 31.0, 1.0, 2.0, 24.0), capi.Cfg(capi.LDPC_F32_SP, 0, 6e-8, 0.0, 1.0, 1e9)):
        rc = capi.lib.ldpc_decode_f32_noalloc(ch.h, C.byref(cfg), None, 0, None, None, None, None)
        assert rc != capi.LDPC_OK
        assert capi.lib.ldpc_last_error().decode()
