"""The C-ABI library without a GPU: it loads, exports every entry point the
header declares, parses and validates tables, and fails loudly (status codes,
never exit) on bad input."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def test_exports_every_declared_entry_point(capi):
    with open(os.path.join(ROOT, "include", "ldpc_b200.h")) as f:
        hdr = f.read()
    declared = set(re.findall(r"\b(ldpc_[a-z0-9_]+)\s*\(", hdr))
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(capi.lib, s)]
    assert not missing, missing


def test_code_from_tables_info(capi):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    c = capi.Code.from_tables(code)
    i = c.info
    assert (i.z, i.mrow, i.mcol, i.n, i.kbits, i.edges, i.max_row_weight, i.hard_words, i.has_encoder) == \
        (42, 8, 16, 672, 336, 2184, 8, 11, 1)


def test_load_dat_files(capi, tmp_path):
    from ldpc_b200 import codes
    code = codes.make_code("16e 1/2", z_over=96)
    e, d = str(tmp_path / "enc.dat"), str(tmp_path / "dec.dat")
    code.write_dat(e, d)
    c = capi.Code.from_dat(e, d)
    assert c.info.z == 96 and c.info.n == 2304
    c2 = capi.Code.from_dat(None, d)
    assert c2.info.has_encoder == 0


def _expect(capi, code, fn):
    with pytest.raises(capi.LdpcError) as ei:
        fn()
    assert ei.value.code == code
    return str(ei.value)


def test_bad_tables_are_rejected(capi, tmp_path):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    dec = np.frombuffer(code.dec_dat_bytes(), "<i4").copy()
    enc = code.enc_dat_bytes()
    B = capi.LDPC_ERR_BAD_TABLE
    _expect(capi, B, lambda: capi.Code.from_bytes(dec[:5].tobytes()))                  # short header
    _expect(capi, B, lambda: capi.Code.from_bytes(dec[:-10].tobytes()))               # truncated
    bad = dec.copy(); bad[7 + 8] = 99                                                   # column out of range
    assert "column" in _expect(capi, B, lambda: capi.Code.from_bytes(bad.tobytes()))
    bad = dec.copy(); bad[7 + 8 + 52] = 42                                              # shift == Z
    assert "shift" in _expect(capi, B, lambda: capi.Code.from_bytes(bad.tobytes()))
    bad = dec.copy(); bad[7 + 8 + 1] = bad[7 + 8]                                       # column repeated in a row
    assert "twice" in _expect(capi, B, lambda: capi.Code.from_bytes(bad.tobytes()))
    bad = dec.copy(); bad[7] = 1                                                        # row weight 1
    _expect(capi, B, lambda: capi.Code.from_bytes(bad.tobytes()))
    e2 = np.frombuffer(enc, "<i4").copy(); e2[0] = 43                                   # Z mismatch
    assert "match" in _expect(capi, B, lambda: capi.Code.from_bytes(dec.tobytes(), e2.tobytes()))
    e3 = np.frombuffer(enc, "<i4").copy(); e3[6 + 16] = 99999                           # work-area address
    _expect(capi, B, lambda: capi.Code.from_bytes(dec.tobytes(), e3.tobytes()))
    _expect(capi, capi.LDPC_ERR_IO, lambda: capi.Code.from_dat(None, str(tmp_path / "missing.dat")))


def test_context_without_gpu_fails_loudly(capi):
    from ldpc_b200 import codes
    code = capi.Code.from_tables(codes.make_code("11ad 1/2"))
    if capi.device_count() > 0:
        pytest.skip("a GPU is present")
    msg = _expect(capi, capi.LDPC_ERR_CUDA, lambda: capi.Context(code))
    assert "device" in msg


def test_invalid_configurations(capi):
    from ldpc_b200 import codes
    code = capi.Code.from_tables(codes.make_code("11ad 1/2"))
    _expect(capi, capi.LDPC_ERR_UNSUPPORTED, lambda: capi.Context(code, max_iter=0))
    _expect(capi, capi.LDPC_ERR_UNSUPPORTED, lambda: capi.Context(code, max_iter=300))
    _expect(capi, capi.LDPC_ERR_INVALID_ARG, lambda: capi.Context(code, variant=7))
