"""ldpc_sim on the GPU: the lines it prints for the reference's stdin blob
carry exactly the counters of ldpc_simulate with the same generator key and
codeword offsets (one outer loop = loop_count * num_codeword codewords per
SNR point), for the int8, int16, float and double sum-product variants."""
import os
import subprocess

import pytest

from conftest import ROOT
from ldpc_b200.simproto import blob, fold_seeds, parse

pytestmark = pytest.mark.gpu
SIM = os.path.join(ROOT, "simd-fecfun_b200", "ldpc_b200", "ldpc_sim")


@pytest.mark.parametrize("exe,name,params", [
    ("LDPCtop_Vec64c_min_b200", "11ad 1/2", dict(mrm=31.0, scale=2.0, max_abs=24.0, beta=1.0, snr=(-1.0, 0.0, 0.5))),
    ("LDPCtop_Vec16f_prod_b200", "16e 1/2", dict(mrm=6e-8, scale=1.0, max_abs=1e9, beta=0.0, snr=(0.5, 1.5, 0.5))),
    ("LDPCtop_Vec32s_min_b200", "11n 1/2 z27", dict(mrm=400.0, scale=20.0, max_abs=800.0, beta=5.0, snr=(0.5, 1.5, 1.0))),
    ("LDPCtop_Vec8d_prod_b200", "11ad 1/2", dict(mrm=1e-16, scale=1.0, max_abs=1e9, beta=0.0, snr=(-0.5, 0.5, 1.0))),
])
def test_lines_match_simulate(capi, tmp_path, exe, name, params):
    from ldpc_b200 import codes
    code = codes.make_code(name)
    code.write_dat(str(tmp_path / "e.dat"), str(tmp_path / "d.dat"))
    seeds = [(0x1234567 * (i + 1)) & ((1 << 56) - 1) for i in range(64)]
    outer, inner, ncw = 2, 3, 4000
    s0, s1, st = params["snr"]
    data = blob(outer, inner, ncw, 10, params["mrm"], params["scale"], params["max_abs"], params["beta"], s0, s1, st,
                seeds, "e.dat", "d.dat")
    os.symlink(SIM, tmp_path / exe)
    r = subprocess.run([str(tmp_path / exe)], input=data, capture_output=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout.decode()[-2000:]
    out = parse(r.stdout.decode())
    assert out["cw_count"] == inner * ncw and out["matrix"][:3] == (code.z, code.mcol, code.mrow)
    snrs = [s0 + k * st for k in range(int((s1 - s0 + 1e-6) / st) + 1)]
    assert len(out["loops"]) == outer * len(snrs)
    variant = {"64c": capi.LDPC_INT8_OMS, "32s": capi.LDPC_INT16_OMS, "8d_": capi.LDPC_F64_SP}.get(exe[11:14],
                                                                                             capi.LDPC_F32_SP)
    ctx = capi.Context(capi.Code.from_tables(code), variant=variant, max_iter=10, max_row_metric=params["mrm"],
                       beta=params["beta"], llr_scale=params["scale"], max_abs_llr=params["max_abs"])
    key = fold_seeds(seeds)
    for o in range(outer):
        ref = ctx.simulate(seed=key, cw_offset=o * inner * ncw, snr_db=snrs, n_per_snr=inner * ncw)
        for k, st_ in enumerate(ref):
            snr, inp, it, be, cwe, ticks = out["loops"][o * len(snrs) + k]
            assert abs(snr - snrs[k]) < 1e-5
            assert (inp, it, be, cwe) == (st_["uncoded_errors"], st_["iterations"], st_["bit_errors"], st_["cw_errors"])
            assert ticks > 0


def test_resumed_run_equals_uninterrupted(tmp_path):
    """A run stopped after two outer loops (its state file saved) and resumed
    with four prints, loop for loop, the counters of one uninterrupted
    four-loop run: the resumed loops continue at the saved codeword offset."""
    from ldpc_b200 import codes
    codes.make_code("11ad 1/2").write_dat(str(tmp_path / "e.dat"), str(tmp_path / "d.dat"))
    seeds = [(0x9E3779B9 * (i + 3)) & ((1 << 56) - 1) for i in range(64)]
    mk = lambda outer: blob(outer, 2, 3000, 10, 31.0, 2.0, 24.0, 1.0, -1.0, 0.0, 0.5, seeds, "e.dat", "d.dat")  # noqa: E731
    exe = tmp_path / "LDPCtop_Vec64c_min_b200"
    os.symlink(SIM, exe)

    def run(outer, state=None):
        env = dict(os.environ)
        env.pop("LDPC_SIM_STATE", None)
        if state:
            env["LDPC_SIM_STATE"] = str(state)
        r = subprocess.run([str(exe)], input=mk(outer), capture_output=True, timeout=300, cwd=tmp_path, env=env)
        assert r.returncode == 0, r.stdout.decode()[-2000:]
        return [l[:5] for l in parse(r.stdout.decode())["loops"]]

    st = tmp_path / "run.state"
    first = run(2, st)
    assert st.exists() and len(first) == 2 * 3
    resumed = run(4, st)
    whole = run(4)
    assert resumed[:6] == first
    assert resumed == whole
