"""Host-side robustness of the simulation driver, without a GPU.

* ldpc_b200.simrun sums the "loop" lines of N simulator processes as the
  reference's run_LDPCsim.pl:156-178 does.  When one process is killed
  mid-run, the survivors' counts and the dead process's completed loops are
  reported, and the dead process is listed with its exit status.  The
  processes here are stand-ins that speak the protocol
  (tests/fake_ldpc_sim.py); the failure is made on the host (SIGKILL).
* ldpc_sim's state file (LDPC_SIM_STATE): a saved run that covers every outer
  loop is replayed without a device; a state of other parameters is reported
  and ignored; a partial state is replayed before the decoder is created.
  The GPU side (a resumed run continues with the counters of an uninterrupted
  one) is in test_ldpc_sim_gpu.py."""
import os
import signal
import subprocess
import sys

import pytest

from conftest import ROOT
from ldpc_b200 import simrun
from ldpc_b200.simproto import blob, parse, state_text

FAKE = [sys.executable, os.path.join(ROOT, "tests", "fake_ldpc_sim.py")]
SIM = os.path.join(ROOT, "simd-fecfun_b200", "ldpc_b200", "ldpc_sim")
INT8 = 0   # LDPC_INT8_OMS, the variant of LDPCtop_Vec64c_min_b200


def _blob(outer, seed0):
    return blob(outer, 2, 100, 10, 31.0, 2.0, 24.0, 1.0, -1.0, 0.0, 0.5, [seed0] + list(range(1, 64)),
                "LDPCencode.raw.dat", "LDPCdecode.raw.dat")


def _fake_counts(outer, seeds, n_snr=3):
    """Per SNR index: (uncoded, iterations, bit errors, cw errors) the stand-in prints in total."""
    tot = {}
    for s0 in seeds:
        for o in range(outer):
            for k in range(n_snr):
                v = (s0 + 7 * o + k) % 97
                t = tot.setdefault(k, [0, 0, 0, 0])
                for j, x in enumerate((1000 + v, 600 + v, v, v // 10)):
                    t[j] += x
    return tot


def _counts(t):
    return [t["uncoded_bit_errors"], t["iterations"], t["bit_errors"], t["cw_errors"]]


def test_sums_like_the_perl_driver():
    r = simrun.run(FAKE, [_blob(3, s) for s in (5, 6, 7)])
    assert r["failed"] == [] and r["processes"] == 3 and r["loops_received"] == 3 * 3 * 3
    exp = _fake_counts(3, (5, 6, 7))
    assert len(r["snr"]) == 3
    for k, t in enumerate(r["snr"].values()):
        assert _counts(t) == exp[k]
        assert t["codewords"] == 3 * 3 * 200


def test_killed_process_leaves_a_partial_result():
    """Process 1 is killed right after it reports its first outer loop; the
    other two finish all six.  The result is the survivors' counts plus the
    dead process's delivered loops, and the dead process is listed."""
    killed = []

    def on_line(i, p, line):
        if i == 1 and not killed and line.startswith("loop 0:") and "SNR=0.000000" in line:
            p.send_signal(signal.SIGKILL)
            killed.append(p.pid)

    r = simrun.run(FAKE, [_blob(6, s) for s in (5, 6, 7)], on_line=on_line)
    assert killed
    assert len(r["failed"]) == 1
    f = r["failed"][0]
    assert f["process"] == 1 and f["returncode"] == -signal.SIGKILL
    got_loops = f["loops_received"]
    assert 3 <= got_loops < 6 * 3 and got_loops % 3 == 0
    assert r["loops_received"] == 2 * 6 * 3 + got_loops
    # survivors in full, plus the dead process's first got_loops / 3 outer loops
    exp = _fake_counts(6, (5, 7))
    dead = _fake_counts(got_loops // 3, (6,))
    for k, t in enumerate(r["snr"].values()):
        assert _counts(t) == [a + b for a, b in zip(exp[k], dead[k])]
        assert t["codewords"] == (2 * 6 + got_loops // 3) * 200


def _sim(tmp_path, data, state):
    exe = tmp_path / "LDPCtop_Vec64c_min_b200"
    if not exe.exists():
        os.symlink(SIM, exe)
    env = dict(os.environ, LDPC_SIM_STATE=str(state))
    return subprocess.run([str(exe)], input=data, capture_output=True, timeout=120, cwd=tmp_path, env=env)


def _lines(outer, n_snr=3):
    return ["loop %d: SNR=%f  inp_bit_err=%d tot_iter=%d tot_bit_err=%d tot_cw_err=%d tot_dec_ticks=%d"
            % (o, -1.0 + 0.5 * k, 10 + o, 600 + k, 3, 1, 99) for o in range(outer) for k in range(n_snr)]


@pytest.fixture
def tables(tmp_path):
    if not os.path.exists(SIM):
        pytest.fail("ldpc_sim is not built")
    from ldpc_b200 import codes
    codes.make_code("11ad 1/2").write_dat(str(tmp_path / "LDPCencode.raw.dat"), str(tmp_path / "LDPCdecode.raw.dat"))
    return tmp_path


def test_complete_state_is_replayed_without_a_device(tables):
    data = _blob(2, 11)
    st = tables / "run.state"
    st.write_text(state_text(data, INT8, 0x1234, _lines(2)))
    r = _sim(tables, data, st)
    assert r.returncode == 0, r.stdout
    out = parse(r.stdout.decode())
    assert out["matrix"] == (42, 16, 8, 1, 0)
    assert [l[2] for l in out["loops"]] == [600, 601, 602] * 2
    # a state covering more loops than asked: only the first outer loops are printed
    r = _sim(tables, _blob(1, 11), st)
    assert r.returncode == 0 and len(parse(r.stdout.decode())["loops"]) == 3


def test_foreign_or_partial_state(tables):
    data = _blob(3, 11)
    st = tables / "run.state"
    # other parameters (another seed): reported, ignored
    st.write_text(state_text(_blob(3, 12), INT8, 0x1234, _lines(3)))
    r = _sim(tables, data, st)
    assert b"belongs to another run" in r.stdout
    if r.returncode != 0:                       # no device here: nothing replayed, then the device error
        assert parse(r.stdout.decode())["loops"] == []
        assert b"ERROR: creating the decoder" in r.stdout
    # a partial state (one of three loops, plus half a loop): the whole loop is replayed first
    st.write_text(state_text(data, INT8, 0x1234, _lines(1) + _lines(2)[3:4]))
    r = _sim(tables, data, st)
    out = parse(r.stdout.decode())
    if r.returncode != 0:
        assert len(out["loops"]) == 3 and b"ERROR: creating the decoder" in r.stdout
    else:
        assert len(out["loops"]) == 9
