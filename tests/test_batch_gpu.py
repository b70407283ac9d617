"""Batched decoding (ldpc_batch_*): one persistent launch over jobs of
different codes and Z sizes, each codeword bit-exact with the oracle on its
own code; CUDA-graph replay; per-layer int8 offsets; fused counting per
job; the autotuner."""
import numpy as np
import pytest

from conftest import make_llr_int8, pack_bits

pytestmark = pytest.mark.gpu

MIX = [  # (code, kwargs for the code, snr, codewords, max_iter, beta)
    ("11ad 1/2", {}, -0.5, 700, 10, 1.0),
    ("16e 1/2", {"z_over": 24}, 1.5, 1300, 10, 1.0),
    ("16e 1/2", {}, 1.2, 210, 10, 2.0),
    ("11n 2/3 z54", {}, 2.5, 450, 10, 1.0),
    ("5GNR_n3136_k576", {}, -6.0, 333, 20, 1.0),
    ("11ay 1/2", {}, -0.25, 999, 10, 1.0),
]


def _mix(capi, oracle):
    import torch
    from ldpc_b200 import codes
    objs, handles, cfgs, data = [], [], [], []
    for i, (name, kw, snr, n, it, beta) in enumerate(MIX):
        c = codes.code_by_name(name, **kw)
        objs.append(c)
        handles.append(capi.Code.from_tables(c))
        cfgs.append(dict(max_iter=it, beta=beta))
        llr, info, _ = make_llr_int8(c, n, snr, seed=40 + i, oracle=oracle)
        data.append((llr, info))
    batch = capi.Batch(handles, cfgs)
    specs, bufs = [], []
    for i, (c, h, (llr, info)) in enumerate(zip(objs, handles, data)):
        n = llr.shape[0]
        b = dict(llr=torch.from_numpy(llr).cuda(), post=torch.empty((n, c.n), dtype=torch.int8, device="cuda"),
                 hard=torch.empty((n, h.info.hard_words), dtype=torch.int32, device="cuda"),
                 iters=torch.empty(n, dtype=torch.uint8, device="cuda"))
        bufs.append(b)
        specs.append(dict(code=i, n=n, **b))
    return batch, objs, handles, data, specs, bufs


def _verify(oracle, objs, handles, data, bufs, betas=None):
    for i, (name, kw, snr, n, it, beta) in enumerate(MIX):
        llr, _ = data[i]
        if betas is not None and betas[i] is not None and betas[i].ndim == 2:
            post_o, it_o = oracle.decode_int8(objs[i], llr, it, 31.0, beta_table=betas[i])
        elif betas is not None and betas[i] is not None:
            post_o, it_o = oracle.decode_int8(objs[i], llr, it, 31.0, beta_layers=betas[i])
        else:
            post_o, it_o = oracle.decode_int8(objs[i], llr, it, 31.0, beta)
        b = bufs[i]
        assert np.array_equal(b["iters"].cpu().numpy(), it_o.astype(np.uint8)), name
        assert np.array_equal(b["post"].cpu().numpy(), post_o), name
        kb = handles[i].info.kbits
        hard = b["hard"].cpu().numpy().view(np.uint32)
        assert np.array_equal(hard, pack_bits((post_o[:, :kb] < 0).astype(np.uint8))), name


def _clear(bufs):
    for b in bufs:
        b["post"].zero_()
        b["hard"].zero_()
        b["iters"].fill_(255)


@pytest.mark.parametrize("threads,cpc", [(0, 0), (128, 1), (384, 4), (512, 2)])
def test_mixed_batch_matches_oracle(capi, oracle, threads, cpc):
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    plan = batch.plan(specs, threads=threads, chunks_per_cta=cpc)
    _clear(bufs)
    plan.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _verify(oracle, objs, handles, data, bufs)


def test_graph_replay(capi, oracle):
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    plan = batch.plan(specs)
    s = torch.cuda.Stream()
    for _ in range(3):
        _clear(bufs)
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            plan.graph_launch(s.cuda_stream)
        s.synchronize()
        _verify(oracle, objs, handles, data, bufs)


def test_per_layer_offsets(capi, oracle):
    """Learned offsets, quantised to int8 per layer (0 included: the abs8(-128) quirk)."""
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    rng = np.random.default_rng(9)
    betas = []
    for i, c in enumerate(objs):
        if i % 2 == 0:
            b = rng.integers(0, 4, c.mrow).astype(np.float32) + np.float32(0.7)   # truncated to 0..3
            b[0] = 0.2
            batch.set_offsets(i, b)
            betas.append(b.astype(np.int8))
        else:
            betas.append(None)
    plan = batch.plan(specs)
    _clear(bufs)
    plan.launch()
    torch.cuda.synchronize()
    _verify(oracle, objs, handles, data, bufs, betas)


def test_offset_tables(capi, oracle):
    """Learned per-(iteration, layer) offsets quantised to int8: a table for
    some codes (rows = max_iter, or fewer: the last row repeats), per-layer
    offsets for one, plain beta for the rest; the two codewords of a pair
    run at different iterations, each with its own row."""
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    rng = np.random.default_rng(12)
    betas = [None] * len(objs)
    for i, c in enumerate(objs):
        rows = MIX[i][4] if i % 3 == 0 else 4
        if i % 3 == 2:
            b = rng.integers(0, 4, c.mrow).astype(np.float32) + np.float32(0.5)
            batch.set_offsets(i, b)
            betas[i] = b.astype(np.int8)
        else:
            t = rng.integers(0, 4, (rows, c.mrow)).astype(np.float32) + np.float32(0.5)
            t[rows - 1, 0] = 0.0
            batch.set_offset_table(i, t)
            betas[i] = t.astype(np.int8)
    plan = batch.plan(specs)
    _clear(bufs)
    plan.graph_launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _verify(oracle, objs, handles, data, bufs, betas)


def test_fused_counting_per_job(capi, oracle):
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    cnts = []
    for i, s in enumerate(specs):
        llr, info = data[i]
        s["data_bits"] = torch.from_numpy(pack_bits(info).view(np.int32)).cuda()
        s["ref_period"] = llr.shape[0]
        s["bucket_size"] = (llr.shape[0] + 1) // 2
        s["n_buckets"] = 2
        s["counters"] = torch.zeros((2, 4), dtype=torch.int64, device="cuda")
        cnts.append(s["counters"])
    plan = batch.plan(specs)
    plan.launch()
    torch.cuda.synchronize()
    for i, (name, kw, snr, n, it, beta) in enumerate(MIX):
        llr, info = data[i]
        post_o, it_o = oracle.decode_int8(objs[i], llr, it, 31.0, beta)
        c = cnts[i].cpu().numpy()
        half = (n + 1) // 2
        for bk, sl in enumerate([slice(0, half), slice(half, n)]):
            m = sl.stop - sl.start
            cw_err, bit_err = oracle.count_errors(objs[i], post_o[sl], np.concatenate(
                [info[sl], np.zeros((m, objs[i].n - info.shape[1]), np.uint8)], axis=1))
            assert c[bk, 0] == m and c[bk, 1] == int(it_o[sl].sum()), name
            assert c[bk, 2] == bit_err and c[bk, 3] == cw_err, name


def test_autotune_then_plan(capi, oracle):
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    t, c, ms = batch.autotune(specs, sample=256)
    assert t in (128, 192, 256, 320, 384, 448, 512) and c in (1, 2, 4, 8) and ms > 0
    plan = batch.plan(specs)      # uses the tuned shape
    _clear(bufs)
    plan.launch()
    torch.cuda.synchronize()
    _verify(oracle, objs, handles, data, bufs)


def test_empty_and_invalid_jobs(capi):
    import torch
    from ldpc_b200 import codes
    h = capi.Code.from_tables(codes.make_code("11ad 1/2"))
    batch = capi.Batch([h], [dict()])
    llr = torch.zeros((4, 672), dtype=torch.int8, device="cuda")
    batch.plan([dict(code=0, llr=llr, n=0)]).launch()
    with pytest.raises(capi.LdpcError):
        batch.plan([dict(code=1, llr=llr, n=4)])
    with pytest.raises(capi.LdpcError):
        capi.Batch([h], [dict(beta=200.0)])


def _float_llr(oracle, code, n, snr, seed):
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    cw = oracle.encode(code, info)
    noise = rng.standard_normal(cw.shape, dtype=np.float32)
    lf, _, _ = oracle.llr_array(code, cw, noise, snr, 1.0, 1e9)
    return lf


@pytest.mark.parametrize("mode", [1, 0])
def test_float_batch_mixed_lifting_sizes(capi, oracle, mode):
    """802.16e 1/2 at Z = 24, 52, 76, 96 in one float launch (sum-product or
    offset min-sum), plus 802.11ad 1/2; each codeword bit-exact with the
    oracle on its own code; then replayed from a CUDA graph."""
    import torch
    from ldpc_b200 import codes
    variant = capi.LDPC_F32_SP if mode == 1 else capi.LDPC_F32_OMS
    mrm, beta = (6e-8, 0.0) if mode == 1 else (31.0, 0.5)
    objs = [codes.make_code("16e 1/2", z_over=z) for z in (24, 52, 76, 96)] + [codes.make_code("11ad 1/2")]
    counts = [300, 170, 90, 257, 333]
    handles = [capi.Code.from_tables(c) for c in objs]
    batch = capi.Batch(handles, [dict(variant=variant, max_iter=10, max_row_metric=mrm, beta=beta)] * len(objs))
    specs, data = [], []
    for i, (c, h, n) in enumerate(zip(objs, handles, counts)):
        llr = _float_llr(oracle, c, n, 1.25 if i < 4 else -0.5, 10 + i)
        b = dict(llr=torch.from_numpy(llr).cuda(), post=torch.empty((n, c.n), dtype=torch.float32, device="cuda"),
                 iters=torch.empty(n, dtype=torch.uint8, device="cuda"))
        specs.append(dict(code=i, n=n, **b))
        data.append(llr)
    plan = batch.plan(specs)
    for launch in (plan.launch, plan.graph_launch, plan.graph_launch):
        for sp in specs:
            sp["post"].zero_()
            sp["iters"].fill_(255)
        torch.cuda.synchronize()
        launch(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for c, sp, llr in zip(objs, specs, data):
            post_o, it_o = oracle.decode_f32(c, llr, mode, 10, mrm, beta)
            assert np.array_equal(sp["iters"].cpu().numpy(), it_o.astype(np.uint8))
            assert np.array_equal(sp["post"].cpu().numpy().view(np.uint32), post_o.view(np.uint32))


def test_batch_variants_must_agree(capi):
    from ldpc_b200 import codes
    h = capi.Code.from_tables(codes.make_code("11ad 1/2"))
    with pytest.raises(capi.LdpcError):
        capi.Batch([h, h], [dict(), dict(variant=capi.LDPC_F32_SP, max_row_metric=6e-8, beta=0.0)])
    fb = capi.Batch([h], [dict(variant=capi.LDPC_F32_OMS)])
    with pytest.raises(capi.LdpcError):
        fb.set_offsets(0, np.ones(8, np.float32))


def test_geometry_classes_and_single_launch(capi, oracle):
    """Codes of different occupancy classes get one kernel each (graph nodes
    free to overlap); LDPC_BATCH_ONE_LAUNCH keeps one kernel; the results are
    the same either way."""
    import os
    import torch
    batch, objs, handles, data, specs, bufs = _mix(capi, oracle)
    plan = batch.plan(specs)
    assert plan.kernels >= 2
    os.environ["LDPC_BATCH_ONE_LAUNCH"] = "1"
    try:
        one = batch.plan(specs)
    finally:
        os.environ.pop("LDPC_BATCH_ONE_LAUNCH", None)
    assert one.kernels == 1
    for p in (plan, one):
        _clear(bufs)
        torch.cuda.synchronize()
        p.graph_launch(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        _verify(oracle, objs, handles, data, bufs)
