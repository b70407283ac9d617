"""Learned-offset decoder on the GPU: the forward equals the float offset
min-sum decoder bit for bit when the offsets are constant; the loss matches
the float64 torch restatement; the hand-written adjoint matches the float64
autograd gradient and FP64 central finite differences (h = 1e-4); gradients
are deterministic; a few training steps lower the loss."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# fp32 kernels against the fp64 restatement: relative to the largest gradient component
GRAD_TOL = 2e-3
# finite differences against the fp64 autograd gradient, on components without a kink within h
FD_TOL = 1e-4


def _ctx(capi, code, mrm=20.0):
    return capi.Context(capi.Code.from_tables(code), variant=capi.LDPC_F32_OMS, max_iter=10, max_row_metric=mrm,
                        beta=0.5, llr_scale=1.0, max_abs_llr=1e9)


def _data(oracle, code, n, sigma, seed):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, code.z * (code.mcol - code.mrow)), dtype=np.uint8)
    cw = oracle.encode(code, info)
    llr = ((2.0 / sigma ** 2) * ((1.0 - 2.0 * cw) + sigma * rng.standard_normal(cw.shape))).astype(np.float32)
    return llr, cw


@pytest.mark.parametrize("name,zo,sigma", [("16e 1/2", 24, 0.85), ("16e 1/2", 96, 0.8), ("11n 2/3 z27", None, 0.7)])
def test_constant_offsets_equal_float_min_sum(capi, oracle, name, zo, sigma):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code(name, z_over=zo) if zo else codes.make_code(name)
    ctx = _ctx(capi, code, mrm=31.0)
    llr, _ = _data(oracle, code, 300, sigma, 1)
    d = torch.from_numpy(llr).cuda()
    n = llr.shape[0]
    post_a = torch.empty_like(d)
    it_a = torch.empty(n, dtype=torch.uint8, device="cuda")
    ctx.decode_f32(d, n, post_a, None, it_a)
    beta = torch.full((10, code.mrow), 0.5, dtype=torch.float32, device="cuda")
    post_b = torch.empty_like(d)
    it_b = torch.empty(n, dtype=torch.uint8, device="cuda")
    capi.check(capi.lib.ldpc_learned_decode(ctx.h, d.data_ptr(), n, 10, beta.data_ptr(), post_b.data_ptr(), None,
                                            it_b.data_ptr(), None))
    torch.cuda.synchronize()
    assert np.array_equal(it_a.cpu().numpy(), it_b.cpu().numpy())
    assert np.array_equal(post_a.cpu().numpy().view(np.uint32), post_b.cpu().numpy().view(np.uint32))


def _grads(capi, oracle, code, n, iters, sigma, seed):
    import torch
    from ldpc_b200 import learned
    ctx = _ctx(capi, code)
    llr, cw = _data(oracle, code, n, sigma, seed)
    rng = np.random.default_rng(seed + 1)
    b0 = rng.uniform(0.2, 0.9, (iters, code.mrow))
    w = np.linspace(0.5, 1.5, iters)
    beta = torch.tensor(b0, dtype=torch.float32, device="cuda", requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float32, device="cuda")
    loss = learned.LearnedOMSLoss.apply(beta, torch.from_numpy(llr).cuda(), torch.from_numpy(cw).cuda(), wt, ctx)
    loss.backward()
    g_cuda = beta.grad.cpu().numpy().astype(np.float64)
    # float64 autograd of the restatement
    b64 = torch.tensor(b0, dtype=torch.float64, requires_grad=True)
    tables = learned.layer_tables(code)
    ref = learned.reference_loss(code, b64, torch.from_numpy(llr.astype(np.float64)), torch.from_numpy(cw),
                                 torch.tensor(w), 20.0, tables)
    ref.backward()
    return ctx, llr, cw, b0, w, float(loss.detach()), g_cuda, float(ref.detach()), b64.grad.numpy(), tables


def test_adjoint_matches_fp64_autograd_and_finite_differences(capi, oracle):
    import torch
    from ldpc_b200 import codes, learned
    code = codes.make_code("16e 1/2", z_over=24)
    # a small case: the loss is piecewise smooth, and the fewer pieces, the
    # fewer central differences straddle a kink
    ctx, llr, cw, b0, w, loss, g_cuda, ref, g_ref, tables = _grads(capi, oracle, code, 4, 3, 0.85, 3)
    assert abs(loss - ref) <= 1e-4 * abs(ref)
    scale = np.abs(g_ref).max()
    assert scale > 1e-5
    assert np.abs(g_cuda - g_ref).max() <= GRAD_TOL * scale
    # FP64 central finite differences of the same loss.  min-sum is piecewise
    # linear: where a kink (|Q| = beta, an argmin change downstream) falls
    # inside [beta - h, beta + h] the central difference is not the
    # derivative.  With h = 1e-6 no window holds one here, and every
    # component must agree; with h = 1e-4 a minority of windows do, and the
    # others must agree.
    llr64 = torch.from_numpy(llr.astype(np.float64))
    bits = torch.from_numpy(cw)
    wt = torch.tensor(w)

    def central(h):
        fd = np.zeros_like(g_ref)
        with torch.no_grad():
            for i in range(b0.shape[0]):
                for l in range(b0.shape[1]):
                    b = torch.tensor(b0)
                    b[i, l] += h
                    lp = float(learned.reference_loss(code, b, llr64, bits, wt, 20.0, tables))
                    b[i, l] -= 2 * h
                    lm = float(learned.reference_loss(code, b, llr64, bits, wt, 20.0, tables))
                    fd[i, l] = (lp - lm) / (2 * h)
        return fd

    fd6 = central(1e-6)
    assert np.abs(fd6 - g_ref).max() <= 1e-6 * scale
    assert np.abs(g_cuda - fd6).max() <= GRAD_TOL * scale
    fd4 = central(1e-4)
    smooth = np.abs(fd4 - g_ref) <= FD_TOL * scale
    assert smooth.mean() >= 0.6
    assert np.abs(g_cuda - fd4)[smooth].max() <= GRAD_TOL * scale + FD_TOL * scale


@pytest.mark.parametrize("n,iters,zo", [(16, 5, 24), (16, 10, 96)])
def test_adjoint_matches_fp64_autograd(capi, oracle, n, iters, zo):
    """Larger cases against the fp64 autograd gradient; Z=96 (N=2304) with
    10 iterations x 12 layers = 120 offsets."""
    from ldpc_b200 import codes
    code = codes.make_code("16e 1/2", z_over=zo)
    ctx, llr, cw, b0, w, loss, g_cuda, ref, g_ref, tables = _grads(capi, oracle, code, n, iters, 0.8, 5)
    assert abs(loss - ref) <= 1e-4 * abs(ref)
    assert np.abs(g_cuda - g_ref).max() <= GRAD_TOL * np.abs(g_ref).max()


def test_gradient_is_deterministic(capi, oracle):
    import torch
    from ldpc_b200 import codes, learned
    code = codes.make_code("16e 1/2", z_over=96)
    ctx = _ctx(capi, code)
    llr, cw = _data(oracle, code, 700, 0.8, 7)
    d, bits = torch.from_numpy(llr).cuda(), torch.from_numpy(cw).cuda()
    w = torch.ones(6, dtype=torch.float32, device="cuda")
    gs = []
    for _ in range(2):
        beta = torch.full((6, code.mrow), 0.5, dtype=torch.float32, device="cuda", requires_grad=True)
        learned.LearnedOMSLoss.apply(beta, d, bits, w, ctx).backward()
        gs.append(beta.grad.cpu().numpy())
    assert np.array_equal(gs[0].view(np.uint32), gs[1].view(np.uint32))


def test_training_lowers_the_loss(capi):
    """Offsets trained from 0 lower the loss on a fixed held-out batch."""
    import torch
    from ldpc_b200 import codes, learned
    code = codes.make_code("16e 1/2", z_over=96)
    ctx = _ctx(capi, code)
    beta, hist = learned.train(ctx, code, iters=6, batch=2048, steps=30, lr=0.05, init=0.0, seed=2)
    assert beta.shape == (6, code.mrow) and float(beta.min()) >= 0.0
    snr = [learned.snr_from_ebn0(e, 0.5) for e in (1.25, 1.75, 2.25)]
    llr, bits = learned.draw(ctx, code, 4096, snr, seed=77, offset=1 << 30)
    w = torch.ones(6, dtype=torch.float32, device="cuda")
    l0 = float(learned.LearnedOMSLoss.apply(torch.zeros_like(beta), llr, bits, w, ctx))
    l1 = float(learned.LearnedOMSLoss.apply(beta, llr, bits, w, ctx))
    assert l1 < 0.98 * l0
    cwer, ber, avg_it = learned.evaluate(ctx, code, beta, learned.snr_from_ebn0(2.0, 0.5), 4096)
    assert 0.0 <= cwer < 0.5 and 1.0 <= avg_it <= 6.0
