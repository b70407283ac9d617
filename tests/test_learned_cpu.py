"""The float64 torch restatement of the learned-offset decoder and loss (the
reference gradient for the CUDA adjoint): its autograd gradient agrees with
FP64 central finite differences (h = 1e-4)."""
import numpy as np
import pytest
import torch


def test_reference_gradient_matches_finite_differences(oracle):
    from ldpc_b200 import codes, learned
    code = codes.make_code("16e 1/2", z_over=24)
    rng = np.random.default_rng(0)
    n, iters = 6, 3
    info = rng.integers(0, 2, (n, code.z * (code.mcol - code.mrow)), dtype=np.uint8)
    cw = oracle.encode(code, info)
    sigma = 0.8
    llr = (2.0 / sigma ** 2) * ((1.0 - 2.0 * cw) + sigma * rng.standard_normal(cw.shape))
    llr_t = torch.from_numpy(llr)
    bits = torch.from_numpy(cw)
    w = torch.tensor([0.5, 1.0, 2.0], dtype=torch.float64)
    beta = torch.from_numpy(rng.uniform(0.2, 0.9, (iters, code.mrow))).requires_grad_(True)
    tables = learned.layer_tables(code)
    loss = learned.reference_loss(code, beta, llr_t, bits, w, 20.0, tables)
    loss.backward()
    g = beta.grad.numpy()
    scale = np.abs(g).max()
    assert scale > 1e-4

    def central(h):
        fd = np.zeros_like(g)
        with torch.no_grad():
            for i in range(iters):
                for l in range(code.mrow):
                    b = beta.detach().clone()
                    b[i, l] += h
                    lp = float(learned.reference_loss(code, b, llr_t, bits, w, 20.0, tables))
                    b[i, l] -= 2 * h
                    lm = float(learned.reference_loss(code, b, llr_t, bits, w, 20.0, tables))
                    fd[i, l] = (lp - lm) / (2 * h)
        return fd

    # min-sum is piecewise linear in beta: with h = 1e-6 no difference window
    # holds a kink and all components agree; with h = 1e-4 the windows
    # without one agree (a kink inside a window makes it an average slope)
    assert np.abs(central(1e-6) - g).max() <= 1e-6 * scale
    fd4 = central(1e-4)
    smooth = np.abs(fd4 - g) <= 1e-4 * scale
    assert smooth.mean() >= 0.6
