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


def _dp_worker(rank, world, port, path, out):
    import os
    import sys
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "simd-fecfun_b200"))
    import torch.distributed as dist
    from ldpc_b200 import codes, learned
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    d = np.load(path)
    code = codes.make_code("16e 1/2", z_over=24)
    n = d["llr"].shape[0] // world
    sl = slice(rank * n, (rank + 1) * n)
    beta = torch.from_numpy(d["beta"]).requires_grad_(True)
    opt = torch.optim.Adam([beta], lr=0.05)
    for _ in range(2):
        opt.zero_grad()
        loss = learned.reference_loss(code, beta, torch.from_numpy(d["llr"][sl]), torch.from_numpy(d["cw"][sl]),
                                      torch.ones(2, dtype=torch.float64), 20.0)
        loss.backward()
        learned.average_gradients([beta])
        opt.step()
    np.save(out % rank, beta.detach().numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_data_parallel_step_equals_one_process(oracle, tmp_path):
    """Two gloo ranks, each on half of a batch, with averaged gradients: the
    offsets after two Adam steps equal one process on the whole batch, and
    both ranks hold the same offsets."""
    import socket
    import torch.multiprocessing as mp
    from ldpc_b200 import codes, learned
    code = codes.make_code("16e 1/2", z_over=24)
    rng = np.random.default_rng(3)
    n = 8
    info = rng.integers(0, 2, (n, code.z * (code.mcol - code.mrow)), dtype=np.uint8)
    cw = oracle.encode(code, info)
    llr = (2.0 / 0.64) * ((1.0 - 2.0 * cw) + 0.8 * rng.standard_normal(cw.shape))
    beta0 = rng.uniform(0.2, 0.9, (2, code.mrow))
    path = str(tmp_path / "batch.npz")
    np.savez(path, llr=llr, cw=cw, beta=beta0)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = str(tmp_path / "beta_%d.npy")
    mp.start_processes(_dp_worker, args=(2, port, path, out), nprocs=2, join=True, start_method="spawn")
    beta = torch.from_numpy(beta0.copy()).requires_grad_(True)
    opt = torch.optim.Adam([beta], lr=0.05)
    for _ in range(2):
        opt.zero_grad()
        learned.reference_loss(code, beta, torch.from_numpy(llr), torch.from_numpy(cw),
                               torch.ones(2, dtype=torch.float64), 20.0).backward()
        opt.step()
    b0, b1 = np.load(out % 0), np.load(out % 1)
    assert np.array_equal(b0, b1)
    assert np.allclose(b0, beta.detach().numpy(), rtol=0, atol=1e-12)
    assert not np.allclose(b0, beta0)
