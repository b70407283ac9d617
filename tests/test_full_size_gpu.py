"""Properties that hold at the headline's full size (802.11ad 1/2, 5e6
codewords per launch, int8, 10 iterations, inputs from the fused
generator), where the oracle would take hours:
  - noiseless round trip: every codeword decodes in one iteration, zero errors;
  - codewords are independent: one launch over 5e6 equals two launches over
    the halves, codeword for codeword;
  - early termination is consistent: a codeword that stopped before the
    10th iteration satisfies every parity check, and one that fails a check
    ran all 10;
  - the encoder is linear over GF(2)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_FULL = 5_000_000


def _ctx(capi, code):
    return capi.Context(capi.Code.from_tables(code), max_iter=10, max_row_metric=31.0, beta=1.0, llr_scale=2.0,
                        max_abs_llr=24.0)


def _check_index(code):
    """[rows][max weight] posterior indexes of every parity check, padded
    with index N (a column of zeros appended to the signs)."""
    z, d = code.z, code.dec
    rows = []
    e0 = 0
    for l in range(code.mrow):
        w = d["row_weights"][l]
        cols, sh = d["row_cols"][e0:e0 + w], d["row_shifts"][e0:e0 + w]
        for t in range(z):
            rows.append([c * z + (s + t) % z for c, s in zip(cols, sh)])
        e0 += w
    dm = max(len(r) for r in rows)
    return np.array([r + [code.n] * (dm - len(r)) for r in rows], np.int64)


def test_noiseless_round_trip_full_size(capi):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    ctx = _ctx(capi, code)
    llr = torch.empty((1, N_FULL, code.n), dtype=torch.int8, device="cuda")
    data = torch.empty((N_FULL, ctx.info.hard_words), dtype=torch.int32, device="cuda")
    unc = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.generate(seed=2024, cw_offset=0, snr_db=[40.0], n_per_snr=N_FULL, llr_int=llr, data_bits=data, uncoded=unc)
    cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
    ctx.decode_count(llr[0], N_FULL, data_bits=data, ref_period=N_FULL, bucket_size=N_FULL, counters=cnt, n_buckets=1)
    torch.cuda.synchronize()
    assert int(unc[0]) == 0
    assert cnt.cpu().numpy()[0].tolist() == [N_FULL, N_FULL, 0, 0]
    assert int(llr.abs().min()) == 24     # every LLR at the clip: no noise got through


@pytest.mark.parametrize("name,variant,n", [("5GNR_n25344_k8448", "LDPC_INT8_OMS", 200_000),
                                            ("5GNR_n3136_k576", "LDPC_INT8_OMS", 1_000_000),
                                            ("16e 1/2", "LDPC_F32_SP", 1_000_000)])
def test_noiseless_round_trip_other_codes(capi, name, variant, n):
    """Punctured columns (LLR 0) and filler bits (LLR +max) of 5G NR, and the
    float sum-product decoder: zero errors on every codeword."""
    import torch
    from ldpc_b200 import codes
    code = codes.code_by_name(name) if name.startswith("5G") else codes.make_code(name, z_over=96)
    v = getattr(capi, variant)
    fl = v != capi.LDPC_INT8_OMS
    ctx = capi.Context(capi.Code.from_tables(code), variant=v, max_iter=20, max_row_metric=6e-8 if fl else 31.0,
                       beta=0.0 if fl else 1.0, llr_scale=1.0 if fl else 2.0, max_abs_llr=1e9 if fl else 24.0)
    llr = torch.empty((1, n, code.n), dtype=torch.float32 if fl else torch.int8, device="cuda")
    data = torch.empty((n, ctx.info.hard_words), dtype=torch.int32, device="cuda")
    if fl:
        ctx.generate(seed=11, cw_offset=0, snr_db=[40.0], n_per_snr=n, llr_f32=llr, data_bits=data)
    else:
        ctx.generate(seed=11, cw_offset=0, snr_db=[40.0], n_per_snr=n, llr_int=llr, data_bits=data)
    cnt = torch.zeros((1, 4), dtype=torch.int64, device="cuda")
    iters = torch.empty(n, dtype=torch.uint8, device="cuda")
    ctx.decode_count(llr[0], n, iters=iters, data_bits=data, ref_period=n, bucket_size=n, counters=cnt, n_buckets=1)
    torch.cuda.synchronize()
    c = cnt.cpu().numpy()[0].tolist()
    assert c[0] == n and c[2] == 0 and c[3] == 0
    assert int(iters.max()) < 20 and c[1] == int(iters.sum())


def test_launch_split_and_early_exit_full_size(capi):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    ctx = _ctx(capi, code)
    llr = torch.empty((1, N_FULL, code.n), dtype=torch.int8, device="cuda")
    ctx.generate(seed=7, cw_offset=0, snr_db=[-0.5], n_per_snr=N_FULL, llr_int=llr)
    hw = ctx.info.hard_words
    post = torch.empty((N_FULL, code.n), dtype=torch.int8, device="cuda")
    hard = torch.empty((N_FULL, hw), dtype=torch.int32, device="cuda")
    iters = torch.empty(N_FULL, dtype=torch.uint8, device="cuda")
    ctx.decode_int8(llr[0], N_FULL, post=post, hard=hard, iters=iters)
    half = N_FULL // 2 + 12345
    hard2 = torch.empty_like(hard)
    iters2 = torch.empty_like(iters)
    ctx.decode_int8(llr[0, :half], half, hard=hard2[:half], iters=iters2[:half])
    ctx.decode_int8(llr[0, half:], N_FULL - half, hard=hard2[half:], iters=iters2[half:])
    torch.cuda.synchronize()
    assert torch.equal(hard, hard2) and torch.equal(iters, iters2)
    assert int(iters.min()) >= 1 and int(iters.max()) == 10
    # parity of every check on the final posteriors, in chunks
    idx = torch.from_numpy(_check_index(code)).cuda()
    failing = torch.empty(N_FULL, dtype=torch.bool, device="cuda")
    step = 250_000
    for a in range(0, N_FULL, step):
        b = min(N_FULL, a + step)
        sign = (post[a:b] < 0).to(torch.uint8)
        sign = torch.cat([sign, torch.zeros((b - a, 1), dtype=torch.uint8, device="cuda")], dim=1)
        par = sign[:, idx].sum(dim=2) & 1
        failing[a:b] = par.any(dim=1)
    early = iters < 10
    # stopped early => every check satisfied (so a failing check => all 10 iterations)
    assert not bool((failing & early).any())
    assert int(early.sum()) > 0.9 * N_FULL and int(failing.sum()) > 0    # both cases occur


def test_encoder_linearity(capi):
    import torch
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    ctx = _ctx(capi, code)
    hw = ctx.info.hard_words
    n = 1_000_000
    g = torch.Generator(device="cuda").manual_seed(5)
    mask = torch.full((hw,), -1, dtype=torch.int32, device="cuda")
    kb = ctx.info.kbits
    if kb % 32:
        mask[-1] = (1 << (kb % 32)) - 1
    a = torch.randint(-2 ** 31, 2 ** 31 - 1, (n, hw), dtype=torch.int32, device="cuda", generator=g) & mask
    b = torch.randint(-2 ** 31, 2 ** 31 - 1, (n, hw), dtype=torch.int32, device="cuda", generator=g) & mask
    ca, cb, cx = (torch.empty((n, code.n), dtype=torch.uint8, device="cuda") for _ in range(3))
    ctx.encode(a, n, ca)
    ctx.encode(b, n, cb)
    ctx.encode(a ^ b, n, cx)
    torch.cuda.synchronize()
    assert torch.equal(ca ^ cb, cx)
    assert torch.equal(ca[:, :kb].to(torch.int32), ((a[:, :, None] >> torch.arange(32, device="cuda")) & 1)
                       .reshape(n, -1)[:, :kb].to(torch.int32))
