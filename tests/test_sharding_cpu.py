"""Multi-rank path on CPU: two gloo ranks decode their codeword shards with
the oracle and sum counters; the result equals one process doing all.  The
second test runs the bench's own exchange (weak_shard for the rank's Philox
counter range, per-SNR counters [n_snr][4] in the decode kernel's layout,
finish_run for the counter sum and the max-over-ranks time)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT, make_llr_int8


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _counters(oracle, code, llr, info):
    post, it = oracle.decode_int8(code, llr, 10, 31.0, 1.0)
    cw = np.concatenate([info, np.zeros((info.shape[0], code.n - info.shape[1]), np.uint8)], axis=1)
    cwe, be = oracle.count_errors(code, post, cw)
    return np.array([llr.shape[0], int(it.sum()), be, cwe], np.int64)


def _worker(rank, world, port, path, out):
    import sys
    for p in (os.path.join(ROOT, "simd-fecfun_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import refbind
    from ldpc_b200 import codes, sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    d = np.load(path)
    llr, info = d["llr"], d["info"]
    start, count = sharding.shard_range(llr.shape[0], rank, world)
    code = codes.make_code("11ad 1/2")
    c = torch.from_numpy(_counters(refbind.Oracle(), code, llr[start:start + count], info[start:start + count]))
    sharding.reduce_counters(c)
    if rank == 0:
        np.save(out, c.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_shard_ranges_partition():
    from ldpc_b200 import sharding
    for total in (0, 1, 7, 1000, 12345):
        for world in (1, 2, 3, 8):
            parts = [sharding.shard_range(total, r, world) for r in range(world)]
            assert sum(c for _, c in parts) == total
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(world - 1))
    with pytest.raises(ValueError):
        sharding.shard_range(10, 2, 2)


def test_two_rank_counters_equal_single_process(oracle, tmp_path):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr, info, _ = make_llr_int8(code, 301, -1.0, seed=3, oracle=oracle)
    path = str(tmp_path / "in.npz")
    np.savez(path, llr=llr, info=info)
    out = str(tmp_path / "out.npy")
    mp.start_processes(_worker, args=(2, _free_port(), path, out), nprocs=2, join=True, start_method="spawn")
    assert np.array_equal(np.load(out), _counters(oracle, code, llr, info))


SNRS2 = (-1.0, -0.5)


def _bench_counters(oracle, code, llr_snr, info):
    """[n_snr][4] = codewords, iterations, bit errors, codeword errors: the
    layout ldpc_decode_count fills per SNR bucket."""
    return np.stack([_counters(oracle, code, l, info) for l in llr_snr])


def _bench_worker(rank, world, port, path, out):
    import sys
    for p in (os.path.join(ROOT, "simd-fecfun_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    import refbind
    from ldpc_b200 import codes, sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    d = np.load(path)
    llr, info, nps = d["llr"], d["info"], int(d["nps"])
    start, count = sharding.weak_shard(nps, rank, world)
    assert count == nps
    code = codes.make_code("11ad 1/2")
    c = torch.from_numpy(_bench_counters(refbind.Oracle(), code, llr[:, start:start + count], info[start:start + count]))
    mine = c.clone()
    total, elapsed = sharding.finish_run(c, 10.0 + rank)   # rank 1 is the slow one
    assert torch.equal(c, mine)                            # the rank's own counters untouched
    if rank == 0:
        np.savez(out, total=total.numpy(), elapsed=np.float64(elapsed))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_exchange_two_ranks_equal_single_process(oracle, tmp_path):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    world, nps = 2, 120
    rng = np.random.default_rng(5)
    info = rng.integers(0, 2, (world * nps, code.k), dtype=np.uint8)
    cw = oracle.encode(code, info)
    noise = rng.standard_normal(cw.shape, dtype=np.float32)
    # one noise draw per global codeword index, scaled per SNR point (as the generator does)
    llr = np.stack([oracle.llr_array(code, cw, noise, s, 2.0, 24.0)[1] for s in SNRS2])
    path = str(tmp_path / "in.npz")
    np.savez(path, llr=llr, info=info, nps=nps)
    out = str(tmp_path / "out.npz")
    mp.start_processes(_bench_worker, args=(world, _free_port(), path, out), nprocs=world, join=True,
                       start_method="spawn")
    r = np.load(out)
    assert np.array_equal(r["total"], _bench_counters(oracle, code, llr, info))
    assert float(r["elapsed"]) == 11.0
