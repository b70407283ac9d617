"""ldpc_sim, the process-level drop-in for LDPCtop_<variant>: it reads the
reference's 820-byte stdin blob and prints the lines run_LDPCsim.pl parses.
Without a GPU it must get as far as the matrix parameters and then fail
with a message (never hang)."""
import os
import subprocess

import pytest

from conftest import ROOT
from ldpc_b200.simproto import blob, parse

SIM = os.path.join(ROOT, "simd-fecfun_b200", "ldpc_b200", "ldpc_sim")


def _run(tmp_path, data, name="LDPCtop_Vec64c_min_b200"):
    exe = tmp_path / name
    if not exe.exists():
        os.symlink(SIM, exe)
    return subprocess.run([str(exe)], input=data, capture_output=True, timeout=120, cwd=tmp_path)


def test_protocol_up_to_the_device(tmp_path):
    from ldpc_b200 import codes
    if not os.path.exists(SIM):
        pytest.fail("ldpc_sim is not built")
    code = codes.make_code("11ad 1/2")
    code.write_dat(str(tmp_path / "LDPCencode.raw.dat"), str(tmp_path / "LDPCdecode.raw.dat"))
    data = blob(2, 3, 1000, 10, 31.0, 2.0, 24.0, 1.0, -1.0, 0.0, 0.25, list(range(1, 65)), "LDPCencode.raw.dat",
                "LDPCdecode.raw.dat")
    assert len(data) == 820
    r = _run(tmp_path, data)
    out = parse(r.stdout.decode())
    assert out["cw_count"] == 3000
    assert out["matrix"] == (42, 16, 8, 1, 0)
    if r.returncode != 0:
        assert b"ERROR: creating the decoder" in r.stdout
    else:
        assert len(out["loops"]) == 2 * 5


def test_short_blob_and_missing_tables(tmp_path):
    r = _run(tmp_path, b"\0" * 100)
    assert r.returncode == 1 and b"Error in reading sim parameters" in r.stdout
    data = blob(1, 1, 10, 10, 31.0, 2.0, 24.0, 1.0, 0.0, 0.0, 0.25, [0] * 64, "nope.enc", "nope.dec")
    r = _run(tmp_path, data)
    assert r.returncode == 1 and b"ERROR: loading the .dat tables" in r.stdout
