"""ctypes bindings for the oracle libraries (test infrastructure only).

* :class:`RefLib` drives the reference's own C++ sources built by
  ``make -C oracle ref`` (``oracle/_ref/libref_<variant>.so``) through the
  ``extern "C"`` shim in ``oracle/ref_shim.cpp``.  Buffers use the
  reference's layouts: decoder metrics per codeword are ``mcol`` columns of
  ``(ceil(Z/P)+2)`` SIMD words, element ``j`` of column ``c`` at word
  ``1 + c*(spz+2)`` (src/LDPCDec/decode_matrix_allocate.cpp:55,
  src/Top/gen_metrics.cpp:37-39); codeword bits are one 512-bit word per
  column, bit ``t`` = LSB-first (src/Top/gen_rand_databits.cpp:24-38).
* :class:`Oracle` is the scalar C restatement (``oracle/liboracle.so``).

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` may use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_u32p = C.POINTER(C.c_uint32)


def _aligned(n: int, dtype, align: int = 64) -> np.ndarray:
    """A zeroed 1-D array whose data starts on an `align`-byte boundary: the
    reference's vector types are 32/64-byte aligned, and their stores may
    assume it (its own buffers come from _mm_malloc)."""
    itemsize = np.dtype(dtype).itemsize
    raw = np.zeros(n * itemsize + align, np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * itemsize].view(dtype)


def ref_available(variant: str = "Vec64c_min") -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % variant))


class RefLib:
    """One reference build variant (e.g. ``Vec64c_min``, ``Vec16f_prod``)."""

    def __init__(self, variant: str = "Vec64c_min"):
        path = os.path.join(REF_DIR, "libref_%s.so" % variant)
        # RTLD_LOCAL: every variant defines the same C++ symbols
        self.lib = C.CDLL(path, mode=os.RTLD_LOCAL)
        L = self.lib
        L.ref_layout.argtypes = [C.POINTER(C.c_int)] * 4
        L.ref_open.restype = C.c_void_p
        L.ref_open.argtypes = [C.c_char_p, C.c_char_p, C.c_uint]
        L.ref_dims.argtypes = [C.c_void_p] + [C.POINTER(C.c_uint)] * 5
        L.ref_metrics.restype = C.c_void_p
        L.ref_metrics.argtypes = [C.c_void_p]
        L.ref_cw_bits.restype = C.c_void_p
        L.ref_cw_bits.argtypes = [C.c_void_p]
        L.ref_decode_set.restype = C.c_uint
        L.ref_decode_set.argtypes = [C.c_void_p, C.c_uint, C.c_uint, C.c_uint, C.c_float, C.c_float]
        L.ref_decode_each.restype = C.c_uint
        L.ref_decode_each.argtypes = [C.c_void_p, C.c_uint, C.c_uint, C.c_float, C.c_float, _u32p]
        L.ref_init_randstate.argtypes = [C.POINTER(C.c_uint64)]
        L.ref_normdist2.argtypes = [C.POINTER(C.c_float), C.c_int]
        L.ref_gen_rand_databits.argtypes = [C.c_void_p, C.c_uint]
        L.ref_encode.argtypes = [C.c_void_p, C.c_uint]
        L.ref_gen_metrics.restype = C.c_uint
        L.ref_gen_metrics.argtypes = [C.c_void_p, C.c_uint, C.c_float, C.POINTER(C.c_float), C.c_float, C.c_float]
        L.ref_count_errors.argtypes = [C.c_void_p, C.c_uint, _u32p, _u32p]
        p, e, w, eb = (C.c_int(), C.c_int(), C.c_int(), C.c_int())
        L.ref_layout(C.byref(p), C.byref(e), C.byref(w), C.byref(eb))
        self.simd_par, self.elem_bw, self.width_bytes, self.enc_bytes = p.value, e.value, w.value, eb.value
        self.dtype = {8: np.int8, 16: np.int16, 32: np.int32, -32: np.float32, -64: np.float64}[self.elem_bw]


class RefCtx:
    """Reference encoder+decoder state for one code and ``num_cw`` codewords."""

    def __init__(self, lib: RefLib, code, num_cw: int):
        self.lib, self.code, self.num_cw = lib, code, num_cw
        self._tmp = tempfile.TemporaryDirectory()
        enc = os.path.join(self._tmp.name, "LDPCencode.raw.dat")
        dec = os.path.join(self._tmp.name, "LDPCdecode.raw.dat")
        code.write_dat(enc, dec)
        self.h = lib.lib.ref_open(enc.encode(), dec.encode(), num_cw)
        z, mr, mc, npar, fc = (C.c_uint(), C.c_uint(), C.c_uint(), C.c_uint(), C.c_uint())
        lib.lib.ref_dims(self.h, C.byref(z), C.byref(mr), C.byref(mc), C.byref(npar), C.byref(fc))
        self.z, self.mrow, self.mcol = z.value, mr.value, mc.value
        P = lib.simd_par
        self.spz = (self.z + P - 1) // P
        self.col_elems = (self.spz + 2) * P
        itemsize = np.dtype(lib.dtype).itemsize
        nelem = num_cw * self.mcol * self.col_elems
        self.metrics = np.ctypeslib.as_array(
            C.cast(lib.lib.ref_metrics(self.h), C.POINTER(C.c_uint8)), shape=(nelem * itemsize,)
        ).view(lib.dtype).reshape(num_cw, self.mcol, self.col_elems)
        self.cw_bits = np.ctypeslib.as_array(
            C.cast(lib.lib.ref_cw_bits(self.h), C.POINTER(C.c_uint8)),
            shape=(num_cw * self.mcol * lib.enc_bytes,)).reshape(num_cw, self.mcol, lib.enc_bytes)

    # -- decoder input/output in the flat [cw][col*Z + t] view
    def set_llr(self, llr: np.ndarray) -> None:
        P = self.lib.simd_par
        llr = np.asarray(llr).reshape(self.num_cw, self.mcol, self.z)
        self.metrics[...] = 0
        self.metrics[:, :, P:P + self.z] = llr

    def posteriors(self) -> np.ndarray:
        P = self.lib.simd_par
        return self.metrics[:, :, P:P + self.z].reshape(self.num_cw, self.mcol * self.z).copy()

    def decode_each(self, max_iter: int, max_row_metric: float, beta: float) -> np.ndarray:
        it = np.zeros(self.num_cw, dtype=np.uint32)
        self.lib.lib.ref_decode_each(self.h, self.num_cw, max_iter, max_row_metric, beta,
                                     it.ctypes.data_as(_u32p))
        return it

    def decode_set(self, max_iter: int, max_row_metric: float, beta: float, first=0, count=None) -> int:
        count = self.num_cw if count is None else count
        return int(self.lib.lib.ref_decode_set(self.h, first, count, max_iter, max_row_metric, beta))

    # -- encoder
    def set_info_bits(self, bits: np.ndarray) -> None:
        """bits: [num_cw][K_cols*Z] uint8 0/1 (data columns only)."""
        kc = self.mcol - self.mrow
        bits = np.asarray(bits, dtype=np.uint8).reshape(self.num_cw, kc, self.z)
        self.cw_bits[...] = 0
        packed = np.packbits(bits, axis=2, bitorder="little")
        self.cw_bits[:, :kc, :packed.shape[2]] = packed

    def codeword_bits(self) -> np.ndarray:
        unp = np.unpackbits(self.cw_bits, axis=2, bitorder="little")[:, :, :self.z]
        return unp.reshape(self.num_cw, self.mcol * self.z)

    def encode(self) -> None:
        self.lib.lib.ref_encode(self.h, self.num_cw)

    def gen_rand_databits(self) -> None:
        self.lib.lib.ref_gen_rand_databits(self.h, self.num_cw)

    def gen_metrics(self, snr: float, wgn: np.ndarray, scale: float, max_abs: float) -> int:
        src = np.asarray(wgn, dtype=np.float32).ravel()
        wgn = _aligned(src.size, np.float32)
        wgn[:] = src
        return int(self.lib.lib.ref_gen_metrics(self.h, self.num_cw, snr,
                                                 wgn.ctypes.data_as(C.POINTER(C.c_float)), scale, max_abs))

    def count_errors(self):
        cw, bit = C.c_uint32(), C.c_uint32()
        self.lib.lib.ref_count_errors(self.h, self.num_cw, C.byref(cw), C.byref(bit))
        return cw.value, bit.value

    def wgn_count(self) -> int:
        """Number of Vec8f words of noise LDPCtop allocates per inner loop (LDPCtop.cpp:60-64)."""
        n = self.num_cw * self.mcol * ((self.z + 7) // 8)
        return n + (n & 1)


def ref_init_randstate(lib: RefLib, seeds64) -> None:
    s = np.ascontiguousarray(seeds64, dtype=np.uint64)
    assert s.size == 64
    lib.lib.ref_init_randstate(s.ctypes.data_as(C.POINTER(C.c_uint64)))


def ref_normdist2(lib: RefLib, simd_count: int) -> np.ndarray:
    out = _aligned(simd_count * 8, np.float32)
    lib.lib.ref_normdist2(out.ctypes.data_as(C.POINTER(C.c_float)), simd_count)
    return out


class Oracle:
    """The scalar C restatement (``oracle/liboracle.so``)."""

    def __init__(self):
        self.lib = C.CDLL(os.path.join(HERE, "liboracle.so"))
        self._trees = None

    class _Code(C.Structure):
        _fields_ = [("z", C.c_int), ("mrow", C.c_int), ("mcol", C.c_int),
                    ("row_weights", C.POINTER(C.c_int32)), ("row_cols", C.POINTER(C.c_int32)),
                    ("row_shifts", C.POINTER(C.c_int32))]

    class _Trees(C.Structure):
        _fields_ = [("prog", C.POINTER(C.c_int32)), ("off", C.POINTER(C.c_int32)),
                    ("len", C.POINTER(C.c_int32)), ("max_d", C.c_int)]

    def _code(self, code):
        d = code.dec
        keep = [np.ascontiguousarray(d[k], dtype=np.int32) for k in ("row_weights", "row_cols", "row_shifts")]
        p = C.POINTER(C.c_int32)
        s = self._Code(code.z, code.mrow, code.mcol, *(a.ctypes.data_as(p) for a in keep))
        return s, keep

    def _tree_struct(self):
        if self._trees is None:
            import sys
            sys.path.insert(0, os.path.join(os.path.dirname(HERE), "simd-fecfun_b200"))
            from ldpc_b200 import trees
            prog, off, ln = [], [0] * 54, [0] * 54
            for d in range(2, 54):
                fp = trees.flat_program(d)
                off[d] = len(prog) // 4
                ln[d] = len(fp) // 4
                prog += fp
            keep = [np.array(prog, np.int32), np.array(off, np.int32), np.array(ln, np.int32)]
            p = C.POINTER(C.c_int32)
            self._trees = (self._Trees(keep[0].ctypes.data_as(p), keep[1].ctypes.data_as(p),
                                       keep[2].ctypes.data_as(p), 53), keep)
        return self._trees[0]

    def shared_math(self, name, x):
        """The shared tanh / atanh (ldpc_math.h) elementwise: name in
        {"tanh", "atanh"}; float32 input runs the float functions, float64 the
        double ones."""
        x = np.ascontiguousarray(x)
        if x.dtype == np.float32:
            fn = {"tanh": self.lib.orc_lm_tanh_array, "atanh": self.lib.orc_lm_atanh_array}[name]
        elif x.dtype == np.float64:
            fn = {"tanh": self.lib.orc_lmd_tanh_array, "atanh": self.lib.orc_lmd_atanh_array}[name]
        else:
            raise TypeError("float32 or float64 input")
        y = np.empty_like(x)
        fn(x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), C.c_size_t(x.size))
        return y

    def decode_int8(self, code, llr, max_iter=10, max_row_metric=31.0, beta=1.0, use_tree=False, beta_layers=None,
                    beta_table=None):
        """int8 layered offset min-sum; ``beta_layers`` (one int8 offset per
        layer) or ``beta_table`` ([rows][layers] int8, iteration i uses row
        min(i, rows-1)) replaces the single ``beta``."""
        llr = np.ascontiguousarray(llr, dtype=np.int8).reshape(-1, code.n)
        n = llr.shape[0]
        post = np.zeros_like(llr)
        it = np.zeros(n, np.uint32)
        cs, keep = self._code(code)
        if beta_table is not None:
            b = np.ascontiguousarray(beta_table, dtype=np.int8)
            assert b.ndim == 2 and b.shape[1] == code.mrow
            self.lib.orc_decode_int8_table(C.byref(cs), llr.ctypes.data_as(C.c_void_p), C.c_size_t(n),
                                           C.c_uint(max_iter), C.c_float(max_row_metric), b.ctypes.data_as(C.c_void_p),
                                           C.c_int(b.shape[0]), post.ctypes.data_as(C.c_void_p),
                                           it.ctypes.data_as(C.c_void_p))
            return post, it
        if beta_layers is not None:
            b = np.ascontiguousarray(beta_layers, dtype=np.int8)
            assert b.size == code.mrow
            self.lib.orc_decode_int8_layers(C.byref(cs), llr.ctypes.data_as(C.c_void_p), C.c_size_t(n),
                                            C.c_uint(max_iter), C.c_float(max_row_metric), b.ctypes.data_as(C.c_void_p),
                                            post.ctypes.data_as(C.c_void_p), it.ctypes.data_as(C.c_void_p))
            return post, it
        if use_tree:
            self.lib.orc_decode_int8_tree(C.byref(cs), C.byref(self._tree_struct()), llr.ctypes.data_as(C.c_void_p),
                                          C.c_size_t(n), C.c_uint(max_iter), C.c_float(max_row_metric), C.c_float(beta),
                                          post.ctypes.data_as(C.c_void_p), it.ctypes.data_as(C.c_void_p))
        else:
            self.lib.orc_decode_int8(C.byref(cs), llr.ctypes.data_as(C.c_void_p), C.c_size_t(n), C.c_uint(max_iter),
                                     C.c_float(max_row_metric), C.c_float(beta), post.ctypes.data_as(C.c_void_p),
                                     it.ctypes.data_as(C.c_void_p))
        return post, it

    def decode_f32(self, code, llr, mode=1, max_iter=10, max_row_metric=6e-8, beta=0.0):
        llr = np.ascontiguousarray(llr, dtype=np.float32).reshape(-1, code.n)
        n = llr.shape[0]
        post = np.zeros_like(llr)
        it = np.zeros(n, np.uint32)
        cs, keep = self._code(code)
        rc = self.lib.orc_decode_f32(C.byref(cs), C.byref(self._tree_struct()), C.c_int(mode),
                                     llr.ctypes.data_as(C.c_void_p), C.c_size_t(n), C.c_uint(max_iter),
                                     C.c_float(max_row_metric), C.c_float(beta), post.ctypes.data_as(C.c_void_p),
                                     it.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("orc_decode_f32 failed (row weight above the tree table)")
        return post, it

    def decode_f64(self, code, llr, mode=1, max_iter=10, max_row_metric=6e-8, beta=0.0):
        llr = np.ascontiguousarray(llr, dtype=np.float64).reshape(-1, code.n)
        n = llr.shape[0]
        post = np.zeros_like(llr)
        it = np.zeros(n, np.uint32)
        cs, keep = self._code(code)
        rc = self.lib.orc_decode_f64(C.byref(cs), C.byref(self._tree_struct()), C.c_int(mode),
                                     llr.ctypes.data_as(C.c_void_p), C.c_size_t(n), C.c_uint(max_iter),
                                     C.c_float(max_row_metric), C.c_float(beta), post.ctypes.data_as(C.c_void_p),
                                     it.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("orc_decode_f64 failed (row weight above the tree table)")
        return post, it

    def sigma(self, snr, llr_scale):
        s, f = C.c_float(), C.c_float()
        self.lib.orc_sigma(C.c_float(snr), C.c_float(llr_scale), C.byref(s), C.byref(f))
        return s.value, f.value

    def llr(self, bits, noise, snr, llr_scale, max_abs, punct=None, filler=None):
        """Element-wise gen_metrics over flat arrays; returns (llr_f32, llr_i32, uncoded_errors)."""
        sigma, sf = self.sigma(snr, llr_scale)
        bits = np.asarray(bits, np.uint8).ravel()
        noise = np.asarray(noise, np.float32).ravel()
        pn = np.zeros(bits.size, np.uint8) if punct is None else np.asarray(punct, np.uint8).ravel()
        fl = np.zeros(bits.size, np.uint8) if filler is None else np.asarray(filler, np.uint8).ravel()
        lf = np.zeros(bits.size, np.float32)
        li = np.zeros(bits.size, np.int32)
        f = self.lib.orc_llr
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int,
                      C.POINTER(C.c_float), C.POINTER(C.c_int32)]
        errs = 0
        pf = lf.ctypes.data_as(C.POINTER(C.c_float))
        pi = li.ctypes.data_as(C.POINTER(C.c_int32))
        for i in range(bits.size):
            errs += f(int(bits[i]), float(noise[i]), sigma, sf, max_abs, int(pn[i]), int(fl[i]),
                      C.cast(C.byref(pf.contents, 4 * i), C.POINTER(C.c_float)),
                      C.cast(C.byref(pi.contents, 4 * i), C.POINTER(C.c_int32)))
        return lf, li, errs

    def llr_array(self, code, bits, noise, snr, llr_scale, max_abs):
        """gen_metrics over [n][N] bits and noise: (float LLRs, int8 LLRs, uncoded errors)."""
        bits = np.ascontiguousarray(bits, dtype=np.uint8)
        noise = np.ascontiguousarray(noise, dtype=np.float32)
        lf = np.empty(bits.shape, np.float32)
        li = np.empty(bits.shape, np.int8)
        f = self.lib.orc_llr_array
        f.restype = C.c_int64
        pn = np.zeros(code.n, np.uint8)
        fl = np.zeros(code.n, np.uint8)
        for s, e in zip(code.punc_list[0::2], code.punc_list[1::2]):
            pn[s:e + 1] ^= 1
        for s, e in zip(code.fill_list[0::2], code.fill_list[1::2]):
            fl[s:e + 1] ^= 1
        errs = f(bits.ctypes.data_as(C.c_void_p), noise.ctypes.data_as(C.c_void_p), C.c_size_t(bits.size),
                 C.c_int(code.n), pn.ctypes.data_as(C.c_void_p), fl.ctypes.data_as(C.c_void_p), C.c_float(snr),
                 C.c_float(llr_scale), C.c_float(max_abs), lf.ctypes.data_as(C.c_void_p), li.ctypes.data_as(C.c_void_p))
        return lf, li, int(errs)

    def encode(self, code, info):
        info = np.ascontiguousarray(info, dtype=np.uint8).reshape(-1, (code.mcol - code.mrow) * code.z)
        n = info.shape[0]
        sched = []
        recs = code.enc_schedule()
        for pc, terms in recs:
            sched += [pc, len(terms)]
            for col, sh in terms:
                sched += [col, sh]
        sched = np.array(sched, np.int32)
        cw = np.zeros((n, code.n), np.uint8)
        self.lib.orc_encode(C.c_int(code.z), C.c_int(code.mcol), C.c_int(code.mrow), sched.ctypes.data_as(C.c_void_p),
                            C.c_int(len(recs)), info.ctypes.data_as(C.c_void_p), C.c_size_t(n), cw.ctypes.data_as(C.c_void_p))
        return cw

    def count_errors(self, code, post, cw_bits):
        post = np.ascontiguousarray(post)
        if post.dtype in (np.float64, np.int16, np.int32):
            post = np.where(post < 0, -1, 1).astype(np.int8)     # only the signs are counted
        cw_bits = np.ascontiguousarray(cw_bits, dtype=np.uint8)
        n = post.shape[0]
        a, b = C.c_uint64(), C.c_uint64()
        fn = self.lib.orc_count_errors_i8 if post.dtype == np.int8 else self.lib.orc_count_errors_f32
        if post.dtype not in (np.int8, np.float32):
            raise TypeError(post.dtype)
        fn(C.c_int(code.z), C.c_int(code.mcol), C.c_int(code.mrow), C.c_int(code.num_par),
           post.ctypes.data_as(C.c_void_p), cw_bits.ctypes.data_as(C.c_void_p), C.c_size_t(n), C.byref(a), C.byref(b))
        return a.value, b.value
