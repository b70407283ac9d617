"""The oracle's sum-product with the shared tanh/atanh (mode 1, what the GPU
runs bit for bit) against the same decoder with the C library's tanh/atanh
(mode 2), float and double: decisions and iteration counts agree, posteriors
differ near the clamp (see test_sp_libm_gpu.py for the GPU side)."""
import numpy as np
import pytest

from test_sp_libm_gpu import _float_llr, compare


@pytest.mark.parametrize("name,z,snr,n", [("11ad 1/2", None, -0.5, 400), ("16e 1/2", 96, -1.76, 150)])
def test_float_shared_vs_libm(oracle, name, z, snr, n):
    from ldpc_b200 import codes
    code = codes.make_code(name, z_over=z) if z else codes.make_code(name)
    llr = _float_llr(code, n, snr, 5, oracle)
    p1, i1 = oracle.decode_f32(code, llr, 1, 10, 6e-8, 0.0)
    p2, i2 = oracle.decode_f32(code, llr, 2, 10, 6e-8, 0.0)
    st = compare(p1, i1, p2, i2, 10)
    assert st["hard_equal_converged"] == 1.0
    assert st["iter_equal"] >= 0.99
    assert st["rel_median"] < 1e-4
    assert not np.array_equal(p1, p2)      # the two transcendentals really differ


def test_double_shared_vs_libm(oracle):
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    llr = _float_llr(code, 300, -0.5, 6, oracle).astype(np.float64)
    p1, i1 = oracle.decode_f64(code, llr, 1, 10, 1e-16, 0.0)
    p2, i2 = oracle.decode_f64(code, llr, 2, 10, 1e-16, 0.0)
    st = compare(p1, i1, p2, i2, 10)
    assert st["hard_equal_converged"] == 1.0
    assert st["iter_equal"] >= 0.99
    assert st["rel_median"] < 1e-9
