"""Error bounds of the shared tanh / atanh (simd-fecfun_b200/csrc/ldpc_math.h)
against the C library's long-double functions.

The sum-product check update is tanh(|Q|/2) -> product tree -> 2*atanh
(src/LDPCDec/min_find.pl:37-45).  The reference takes tanh/atanh from the
absent vectorclass library, so the decoder, the oracle and the reference
build all run ldpc_math.h; these tests pin that function to an independent
one.

Bounds, in units in the last place of the result's type (float: 2^(e-23),
double: 2^(e-52), for a true value in [2^e, 2^(e+1))):
  float tanh  on [0, 40]      4.07 ulp  (exhaustive over every float once: 4.067 at x = 0.12554)
  float atanh on [0, 1)       4.45 ulp  (exhaustive: 4.443 at x = 0.12366)
  double tanh on [0, 40]      4.3  ulp  (4.20 at x = 0.12562 in 4e7 samples)
  double atanh on [0, 1)      4.6  ulp  (4.48 at x = 0.12428 in 4e7 samples)
The float tests scan a strided subset of all float bit patterns plus every
float around the worst points; the double tests sample uniformly, densely
near 1 for atanh and over many binades near 0."""
import ctypes as C
import struct

import numpy as np
import pytest

F_TANH_MAX = 4.07
F_ATANH_MAX = 4.45
D_TANH_MAX = 4.3
D_ATANH_MAX = 4.6


def _bits(v):
    return struct.unpack("<I", struct.pack("<f", v))[0]


def _scan(oracle, kind, lo, hi, stride):
    f = oracle.lib.orc_ulp_scan_f32
    f.restype = C.c_double
    f.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]
    x = C.c_float()
    w = f(kind, lo, hi, stride, C.byref(x))
    return w, x.value


def test_float_tanh_ulp(oracle):
    worst, at = _scan(oracle, 0, 0, _bits(40.0), 97)
    assert worst <= F_TANH_MAX, (worst, at)
    # every float around the worst region (the expm1 branch switch at 2x = 1/4)
    worst, at = _scan(oracle, 0, _bits(0.12), _bits(0.13), 1)
    assert 3.5 < worst <= F_TANH_MAX, (worst, at)
    # tanh(0) = 0 and saturation
    assert oracle.shared_math("tanh", np.array([0.0, 10.0, 40.0], np.float32)).tolist() == [0.0, 1.0, 1.0]


def test_float_atanh_ulp(oracle):
    worst, at = _scan(oracle, 1, 0, _bits(1.0) - 1, 97)
    assert worst <= F_ATANH_MAX, (worst, at)
    worst, at = _scan(oracle, 1, _bits(0.118), _bits(0.13), 1)
    assert 3.5 < worst <= F_ATANH_MAX, (worst, at)
    # every float in the last binades below 1, where 2*atanh carries the decoder's largest messages
    worst, at = _scan(oracle, 1, _bits(1.0) - (1 << 16), _bits(1.0) - 1, 1)
    assert worst <= F_ATANH_MAX, (worst, at)


def _ulp_d(y, x, ref):
    v = ref.astype(np.longdouble)
    e = np.floor(np.log2(np.abs(v).astype(np.float64)))
    ulp = np.ldexp(np.longdouble(1.0), (e - 52).astype(np.int64))
    return np.abs(y.astype(np.longdouble) - v) / ulp


@pytest.mark.parametrize("name", ["tanh", "atanh"])
def test_double_ulp(oracle, name):
    if np.finfo(np.longdouble).nmant < 63:
        pytest.skip("long double is not wider than double here")
    rng = np.random.default_rng(17)
    if name == "tanh":
        x = np.concatenate([rng.uniform(0, 40, 2_000_000), rng.uniform(0.1, 0.15, 1_000_000),
                            2.0 ** -np.arange(1, 1000, 0.01)])
        ref = np.tanh(x.astype(np.longdouble))
        bound = D_TANH_MAX
    else:
        x = np.concatenate([rng.uniform(0, 1, 2_000_000), rng.uniform(0.1, 0.15, 1_000_000),
                            1 - 2.0 ** -np.arange(1, 53, 0.0005), 2.0 ** -np.arange(1, 1000, 0.01)])
        x = x[x < 1]
        ref = np.arctanh(x.astype(np.longdouble))
        bound = D_ATANH_MAX
    y = oracle.shared_math(name, x)
    u = _ulp_d(y, x, ref)
    i = int(np.argmax(u))
    assert u[i] <= bound, (float(u[i]), float(x[i]))
