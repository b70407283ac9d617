"""ldpc_decode_f32_noalloc (static device scratch, no context) through the C
ABI, against the context path ldpc_decode_f32 and against the oracle.

Callers such as a framework that reserved the device's memory in its own
pool, or a process that must not let cudaFree synchronise the device, use
this entry point; it keeps its check messages in a fixed per-device array.

Tolerance: posteriors within 1e-4 relative (the float decoders' stated
tolerance); hard decisions and iteration counts identical.  Both paths and
the oracle run the same arithmetic, so the posteriors are expected to agree
bit for bit.  Each case calls the no-alloc entry point twice in a row, so the
second call reuses a scratch array the first one left dirty, and checks that
neither call changed the device's free memory.

The 5G NR base graph 1 (Z=384) case comes first: its float context sets the
kernel's shared-memory limit to the most any launch uses (one codeword needs
209 KB with its staging buffer); a no-alloc call in between must not lower it
under the context's next launch."""
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


class _Outputs:
    def __init__(self, torch, n, N, hw):
        self.post = torch.full((n, N), float("nan"), dtype=torch.float32, device="cuda")
        self.hard = torch.full((n, hw), -1, dtype=torch.int32, device="cuda")
        self.iters = torch.full((n,), 255, dtype=torch.uint8, device="cuda")

    def host(self):
        return (self.post.cpu().numpy(), self.hard.cpu().numpy().view(np.uint32), self.iters.cpu().numpy())


def _noalloc(capi, torch, code_h, cfg, llr_d, n, out):
    s = torch.cuda.current_stream().cuda_stream
    capi.check(capi.lib.ldpc_decode_f32_noalloc(code_h.h, C.byref(cfg), llr_d.data_ptr(), n, out.post.data_ptr(),
                                                out.hard.data_ptr(), out.iters.data_ptr(), s or None))


def _same(a, b):
    post, hard, iters = a
    post_r, hard_r, iters_r = b
    assert np.array_equal(iters, iters_r)
    assert np.array_equal(hard, hard_r)
    np.testing.assert_allclose(post, post_r, rtol=1e-4, atol=0)
    assert np.array_equal(post.view(np.uint32), post_r.view(np.uint32))


@pytest.mark.parametrize("name,variant,snr,n,mrm,beta,max_iter", [
    ("5GNR_n25344_k8448", "sp", -4.2, 6, 6e-8, 0.0, 6),   # 209 KB per codeword with staging: runs without it
    ("802.3ca", "sp", 3.0, 240, 6e-8, 0.0, 4),          # messages beyond shared memory; grid capped by the scratch
    ("11ad 1/2", "sp", -0.5, 3000, 6e-8, 0.0, 10),
    ("11n 5/6 z81", "oms", 4.5, 1000, 31.0, 0.5, 10),
])
def test_noalloc_matches_context_path_and_oracle(capi, oracle, name, variant, snr, n, mrm, beta, max_iter):
    import torch
    from ldpc_b200 import codes
    code = codes.code_by_name(name)
    ch = capi.Code.from_tables(code)
    v = capi.LDPC_F32_SP if variant == "sp" else capi.LDPC_F32_OMS
    ctx = capi.Context(ch, variant=v, max_iter=max_iter, max_row_metric=mrm, beta=beta, llr_scale=1.0,
                       max_abs_llr=1e9)
    N, hw = ch.info.n, ch.info.hard_words
    llr = _llr(oracle, code, n, snr, 11)
    llr_d = torch.from_numpy(llr).cuda()
    cfg = capi.Cfg(v, max_iter, mrm, beta, 1.0, 1e9)

    # one no-alloc call between the context's creation and its first launch
    warm = _Outputs(torch, n, N, hw)
    _noalloc(capi, torch, ch, cfg, llr_d, n, warm)
    torch.cuda.synchronize()

    ref = _Outputs(torch, n, N, hw)
    ctx.decode_f32(llr_d.data_ptr(), n, ref.post.data_ptr(), ref.hard.data_ptr(), ref.iters.data_ptr(),
                   torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref_h = ref.host()
    assert ref_h[2].min() >= 1
    _same(warm.host(), ref_h)

    # the oracle on the same LLRs
    post_o, it_o = oracle.decode_f32(code, llr, 1 if variant == "sp" else 0, max_iter, mrm, beta)
    assert np.array_equal(ref_h[2], it_o.astype(np.uint8))
    np.testing.assert_allclose(ref_h[0], post_o, rtol=1e-4, atol=0)
    assert np.array_equal(ref_h[0].view(np.uint32), post_o.view(np.uint32))

    # two calls in a row on preallocated outputs: same results, no device memory taken
    outs = [_Outputs(torch, n, N, hw) for _ in range(2)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for o in outs:
        _noalloc(capi, torch, ch, cfg, llr_d, n, o)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, "free device memory moved by %d bytes across two no-alloc calls" % (free0 - free1)
    for o in outs:
        _same(o.host(), ref_h)


def test_noalloc_rejects_int8_and_bad_config(capi):
    from ldpc_b200 import codes
    ch = capi.Code.from_tables(codes.make_code("11ad 1/2"))
    for cfg in (capi.Cfg(capi.LDPC_INT8_OMS, 10, 31.0, 1.0, 2.0, 24.0), capi.Cfg(capi.LDPC_F32_SP, 0, 6e-8, 0.0, 1.0, 1e9)):
        rc = capi.lib.ldpc_decode_f32_noalloc(ch.h, C.byref(cfg), None, 0, None, None, None, None)
        assert rc != capi.LDPC_OK
        assert capi.lib.ldpc_last_error().decode()
