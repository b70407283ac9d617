import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "simd-fecfun_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import refbind
    return refbind.Oracle()


@pytest.fixture(scope="session")
def capi():
    from ldpc_b200 import capi as c
    return c


def make_llr_int8(code, n, snr_db, seed, scale=2.0, max_abs=24.0, oracle=None):
    """Seeded synthetic int8 LLRs: random data, QC-encoded by the oracle,
    BPSK over AWGN, quantised like gen_metrics (numpy float32 arithmetic)."""
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, (n, (code.mcol - code.mrow) * code.z), dtype=np.uint8)
    cw = oracle.encode(code, info)
    sigma = np.float32(10.0 ** (-(snr_db + 10 * np.log10(2.0)) / 20.0))
    y = (1.0 - 2.0 * cw.astype(np.float32)) + sigma * rng.standard_normal(cw.shape, dtype=np.float32)
    llr = np.clip(np.rint(y * np.float32(2 * scale / sigma ** 2)), -max_abs, max_abs).astype(np.int8)
    return llr, info, cw


def pack_bits(bits):
    """[n][k] 0/1 -> [n][ceil(k/32)] uint32, bit i -> word i//32 bit i%32."""
    n, k = bits.shape
    w = (k + 31) // 32
    padded = np.zeros((n, w * 32), np.uint8)
    padded[:, :k] = bits
    return np.packbits(padded, axis=1, bitorder="little").view("<u4").reshape(n, w)
