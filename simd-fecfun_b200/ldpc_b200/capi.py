"""ctypes binding of libldpc_b200.so (declarations: include/ldpc_b200.h).

The library must have been built (``python simd-fecfun_b200/build.py``);
importing this module without it raises ``ImportError`` -- there is no CPU
fallback.  Device buffers are passed as raw pointers (``tensor.data_ptr()``);
host buffers as numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libldpc_b200.so")

LDPC_OK = 0
LDPC_ERR_INVALID_ARG = 1
LDPC_ERR_BAD_TABLE = 2
LDPC_ERR_UNSUPPORTED = 3
LDPC_ERR_CUDA = 4
LDPC_ERR_TIMEOUT = 5
LDPC_ERR_IO = 6
LDPC_ERR_NOMEM = 7

LDPC_INT8_OMS = 0
LDPC_F32_SP = 1
LDPC_F32_OMS = 2
LDPC_INT16_OMS = 3
LDPC_INT32_OMS = 4
LDPC_F64_SP = 5
LDPC_F64_OMS = 6

ERROR_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "BAD_TABLE", 3: "UNSUPPORTED", 4: "CUDA", 5: "TIMEOUT", 6: "IO",
               7: "NOMEM"}


class LdpcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s: %s" % (ERROR_NAMES.get(code, code), msg))
        self.code = code


class CodeInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("z", "mrow", "mcol", "n", "kbits", "num_par", "fill_cnt", "edges",
                                       "max_row_weight", "hard_words", "has_encoder")]


class Cfg(C.Structure):
    _fields_ = [("variant", C.c_int), ("max_iter", C.c_uint), ("max_row_metric", C.c_float), ("beta", C.c_float),
                ("llr_scale", C.c_float), ("max_abs_llr", C.c_float)]


class SnrStats(C.Structure):
    _fields_ = [("snr_db", C.c_float), ("codewords", C.c_ulonglong), ("iterations", C.c_ulonglong),
                ("bit_errors", C.c_ulonglong), ("cw_errors", C.c_ulonglong), ("uncoded_errors", C.c_ulonglong),
                ("decode_ms", C.c_double)]


_vp = C.c_void_p
_sz = C.c_size_t


class BatchJob(C.Structure):
    _fields_ = [("code", C.c_int), ("llr", _vp), ("n", _sz), ("post_out", _vp), ("hard_out", _vp), ("iters_out", _vp),
                ("data_bits", _vp), ("ref_period", _sz), ("bucket_size", _sz), ("counters", _vp), ("n_buckets", C.c_int)]


_PROTOS = {
    "ldpc_last_error": (C.c_char_p, []),
    "ldpc_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "ldpc_code_load_dat": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_vp)]),
    "ldpc_code_from_tables": (C.c_int, [_vp, _sz, _vp, _sz, C.POINTER(_vp)]),
    "ldpc_code_get_info": (C.c_int, [_vp, C.POINTER(CodeInfo)]),
    "ldpc_code_destroy": (None, [_vp]),
    "ldpc_ctx_create": (C.c_int, [_vp, C.POINTER(Cfg), C.c_int, C.POINTER(_vp)]),
    "ldpc_ctx_destroy": (None, [_vp]),
    "ldpc_ctx_set_layer_offsets": (C.c_int, [_vp, _vp]),
    "ldpc_ctx_set_offset_table": (C.c_int, [_vp, _vp, C.c_uint]),
    "ldpc_batch_set_offset_table": (C.c_int, [_vp, C.c_int, _vp, C.c_uint]),
    "ldpc_decode_int8": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp]),
    "ldpc_decode_f32": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp]),
    "ldpc_decode_int16": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp]),
    "ldpc_decode_int32": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp]),
    "ldpc_decode_f64": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp]),
    "ldpc_decode_f64_host": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "ldpc_decode_int16_host": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "ldpc_decode_int32_host": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "ldpc_decode_int8_host": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "ldpc_decode_f32_host": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "ldpc_decode_set_compat": (C.c_int, [_vp, _vp, C.c_uint, C.c_uint, C.POINTER(C.c_uint64)]),
    "ldpc_generate": (C.c_int, [_vp, C.c_uint64, C.c_uint64, _vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp]),
    "ldpc_llr_from_noise": (C.c_int, [_vp, _vp, _vp, _sz, C.c_float, _vp, _vp, _vp, _vp]),
    "ldpc_encode": (C.c_int, [_vp, _vp, _sz, _vp, _vp]),
    "ldpc_simulate": (C.c_int, [_vp, C.c_uint64, C.c_uint64, _vp, _sz, _sz, C.POINTER(SnrStats)]),
    "ldpc_count_errors": (C.c_int, [_vp, _vp, _sz, _vp, _sz, _vp, _vp]),
    "ldpc_decode_count": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _sz, _sz, _vp, C.c_int, _vp]),
    "ldpc_probe_int32_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "ldpc_probe_fp32_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ldpc_probe_op_rates": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_char_p)]),
    "ldpc_decode_f32_noalloc": (C.c_int, [_vp, C.POINTER(Cfg), _vp, _sz, _vp, _vp, _vp, _vp]),
    "ldpc_batch_create": (C.c_int, [C.POINTER(_vp), C.POINTER(Cfg), C.c_int, C.c_int, C.POINTER(_vp)]),
    "ldpc_batch_set_offsets": (C.c_int, [_vp, C.c_int, _vp]),
    "ldpc_batch_destroy": (None, [_vp]),
    "ldpc_batch_plan_create": (C.c_int, [_vp, C.POINTER(BatchJob), C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "ldpc_batch_plan_launch": (C.c_int, [_vp, _vp]),
    "ldpc_batch_plan_graph_launch": (C.c_int, [_vp, _vp]),
    "ldpc_batch_plan_destroy": (None, [_vp]),
    "ldpc_batch_plan_kernels": (C.c_int, [_vp]),
    "ldpc_learned_grid": (C.c_int, [_vp, _sz, C.POINTER(C.c_int)]),
    "ldpc_learned_forward": (C.c_int, [_vp, _vp, _sz, C.c_int, _vp, _vp, _vp, _vp]),
    "ldpc_learned_backward": (C.c_int, [_vp, _sz, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_float, _vp, _vp, _vp]),
    "ldpc_learned_decode": (C.c_int, [_vp, _vp, _sz, C.c_int, _vp, _vp, _vp, _vp, _vp]),
    "ldpc_batch_autotune": (C.c_int, [_vp, C.POINTER(BatchJob), C.c_int, _sz, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double)]),
}

if not os.path.exists(LIB_PATH):
    raise ImportError("libldpc_b200.so is not built (run python simd-fecfun_b200/build.py)")
lib = C.CDLL(LIB_PATH)
for _name, (_res, _args) in _PROTOS.items():
    if hasattr(lib, _name):
        _f = getattr(lib, _name)
        _f.restype = _res
        _f.argtypes = _args


def exported_symbols():
    return [n for n in _PROTOS if hasattr(lib, n)]


def check(rc: int) -> None:
    if rc != LDPC_OK:
        raise LdpcError(rc, lib.ldpc_last_error().decode())


def device_count() -> int:
    n = C.c_int()
    check(lib.ldpc_device_count(C.byref(n)))
    return n.value


def probe_int32_peak(device: int = 0) -> float:
    v = C.c_double()
    check(lib.ldpc_probe_int32_peak(device, C.byref(v)))
    return v.value


def probe_fp32_peak(device: int = 0):
    """(FP32 fused multiply-adds per second, MUFU ops per second) of the device."""
    f, m = C.c_double(), C.c_double()
    check(lib.ldpc_probe_fp32_peak(device, C.byref(f), C.byref(m)))
    return f.value, m.value


def probe_op_rates(device: int = 0):
    """[(operation, thread-level ops per clock per SM)] of the packed-lane probe."""
    n = 17
    v = (C.c_double * n)()
    names = (C.c_char_p * n)()
    check(lib.ldpc_probe_op_rates(device, v, n, names))
    return [(names[i].decode(), v[i]) for i in range(n)]


def _ptr(x) -> Optional[int]:
    """Device pointer of a torch tensor, address of a numpy array, or None."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, int):
        return x
    raise TypeError(type(x))


class Code:
    """An LDPC code loaded into the library (the two .dat tables)."""

    def __init__(self, handle):
        self.h = handle
        info = CodeInfo()
        check(lib.ldpc_code_get_info(self.h, C.byref(info)))
        self.info = info

    @classmethod
    def from_dat(cls, enc_path: Optional[str], dec_path: str) -> "Code":
        h = _vp()
        check(lib.ldpc_code_load_dat(enc_path.encode() if enc_path else None, dec_path.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_bytes(cls, dec_bytes: bytes, enc_bytes: Optional[bytes] = None) -> "Code":
        d = np.frombuffer(dec_bytes, dtype="<i4").copy()
        e = np.frombuffer(enc_bytes, dtype="<i4").copy() if enc_bytes is not None else None
        h = _vp()
        check(lib.ldpc_code_from_tables(d.ctypes.data, d.size, e.ctypes.data if e is not None else None,
                                        e.size if e is not None else 0, C.byref(h)))
        return cls(h)

    @classmethod
    def from_tables(cls, code) -> "Code":
        """From an ``ldpc_b200.codes.Code`` (generated tables)."""
        return cls.from_bytes(code.dec_dat_bytes(), code.enc_dat_bytes())

    def close(self):
        if self.h:
            lib.ldpc_code_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """Decoder / generator context on one device (ldpc_ctx_create)."""

    def __init__(self, code: Code, variant: int = LDPC_INT8_OMS, max_iter: int = 10, max_row_metric: float = 31.0,
                 beta: float = 1.0, llr_scale: float = 2.0, max_abs_llr: float = 24.0, device: int = 0):
        self.code = code
        self.cfg = Cfg(variant, max_iter, max_row_metric, beta, llr_scale, max_abs_llr)
        h = _vp()
        check(lib.ldpc_ctx_create(code.h, C.byref(self.cfg), device, C.byref(h)))
        self.h = h
        self.info = code.info

    def close(self):
        if getattr(self, "h", None):
            lib.ldpc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_layer_offsets(self, beta_per_layer=None):
        """int8 contexts: one offset per layer (None restores cfg.beta)."""
        if beta_per_layer is None:
            check(lib.ldpc_ctx_set_layer_offsets(self.h, None))
            return
        b = np.ascontiguousarray(beta_per_layer, dtype=np.float32)
        check(lib.ldpc_ctx_set_layer_offsets(self.h, b.ctypes.data))

    def set_offset_table(self, beta=None):
        """int8 contexts: offsets beta[rows][layers]; iteration i uses row
        min(i, rows-1) (None restores cfg.beta)."""
        if beta is None:
            check(lib.ldpc_ctx_set_offset_table(self.h, None, 0))
            return
        b = np.ascontiguousarray(beta, dtype=np.float32)
        check(lib.ldpc_ctx_set_offset_table(self.h, b.ctypes.data, b.shape[0]))

    # ---- device-pointer API (torch tensors) ----
    def decode_int8(self, llr, n, post=None, hard=None, iters=None, stream=0):
        check(lib.ldpc_decode_int8(self.h, _ptr(llr), n, _ptr(post), _ptr(hard), _ptr(iters), stream or None))

    def decode_f32(self, llr, n, post=None, hard=None, iters=None, stream=0):
        check(lib.ldpc_decode_f32(self.h, _ptr(llr), n, _ptr(post), _ptr(hard), _ptr(iters), stream or None))

    def decode_int16(self, llr, n, post=None, hard=None, iters=None, stream=0):
        check(lib.ldpc_decode_int16(self.h, _ptr(llr), n, _ptr(post), _ptr(hard), _ptr(iters), stream or None))

    def decode_int32(self, llr, n, post=None, hard=None, iters=None, stream=0):
        check(lib.ldpc_decode_int32(self.h, _ptr(llr), n, _ptr(post), _ptr(hard), _ptr(iters), stream or None))

    def decode_f64(self, llr, n, post=None, hard=None, iters=None, stream=0):
        check(lib.ldpc_decode_f64(self.h, _ptr(llr), n, _ptr(post), _ptr(hard), _ptr(iters), stream or None))

    def decode_count(self, llr, n, hard=None, iters=None, data_bits=None, ref_period=1, bucket_size=0, counters=None,
                     n_buckets=1, stream=0):
        check(lib.ldpc_decode_count(self.h, _ptr(llr), n, _ptr(hard), _ptr(iters), _ptr(data_bits), ref_period,
                                    bucket_size, _ptr(counters), n_buckets, stream or None))

    def generate(self, seed, cw_offset, snr_db, n_per_snr, llr_i8=None, llr_f32=None, data_bits=None, uncoded=None,
                 stream=0, llr_int=None):
        """llr_int (alias llr_i8): LLRs of the context's element type (int8,
        int16, int32, or double for the double variants)."""
        llr_i8 = llr_int if llr_int is not None else llr_i8
        snr = np.ascontiguousarray(snr_db, dtype=np.float32)
        check(lib.ldpc_generate(self.h, seed, cw_offset, snr.ctypes.data, snr.size, n_per_snr, _ptr(llr_i8),
                                _ptr(llr_f32), _ptr(data_bits), _ptr(uncoded), stream or None))

    def llr_from_noise(self, cw_bits, noise, n, snr_db, llr_i8=None, llr_f32=None, uncoded=None, stream=0,
                       llr_int=None):
        llr_i8 = llr_int if llr_int is not None else llr_i8
        check(lib.ldpc_llr_from_noise(self.h, _ptr(cw_bits), _ptr(noise), n, snr_db, _ptr(llr_i8), _ptr(llr_f32),
                                      _ptr(uncoded), stream or None))

    def encode(self, data_bits, n, cw_bits, stream=0):
        check(lib.ldpc_encode(self.h, _ptr(data_bits), n, _ptr(cw_bits), stream or None))

    def count_errors(self, hard, n, data_bits, ref_period, counters, stream=0):
        check(lib.ldpc_count_errors(self.h, _ptr(hard), n, _ptr(data_bits), ref_period, _ptr(counters), stream or None))

    def simulate(self, seed, cw_offset, snr_db, n_per_snr):
        snr = np.ascontiguousarray(snr_db, dtype=np.float32)
        st = (SnrStats * snr.size)()
        check(lib.ldpc_simulate(self.h, seed, cw_offset, snr.ctypes.data, snr.size, n_per_snr, st))
        return [dict(snr_db=s.snr_db, codewords=s.codewords, iterations=s.iterations, bit_errors=s.bit_errors,
                     cw_errors=s.cw_errors, uncoded_errors=s.uncoded_errors, decode_ms=s.decode_ms) for s in st]

    # ---- host-memory API (numpy) ----
    def decode_host(self, llr: np.ndarray, want_post=True, want_hard=True, want_iters=True):
        llr = np.ascontiguousarray(llr)
        n = llr.shape[0]
        N = self.info.n
        if llr.size != n * N:
            raise ValueError("llr must be [n][%d]" % N)
        post = np.empty_like(llr) if want_post else None
        hard = np.empty((n, self.info.hard_words), np.uint32) if want_hard else None
        iters = np.empty(n, np.uint8) if want_iters else None
        tot = C.c_uint64()
        fns = {np.dtype(np.int8): lib.ldpc_decode_int8_host, np.dtype(np.float32): lib.ldpc_decode_f32_host,
               np.dtype(np.int16): lib.ldpc_decode_int16_host, np.dtype(np.int32): lib.ldpc_decode_int32_host,
               np.dtype(np.float64): lib.ldpc_decode_f64_host}
        if llr.dtype not in fns:
            raise TypeError(llr.dtype)
        fn = fns[llr.dtype]
        check(fn(self.h, llr.ctypes.data, n, _ptr(post), _ptr(hard), _ptr(iters), C.byref(tot)))
        return post, hard, iters, tot.value

    def decode_set_compat(self, metrics: np.ndarray, num_codeword: int, simd_par: int) -> int:
        tot = C.c_uint64()
        check(lib.ldpc_decode_set_compat(self.h, metrics.ctypes.data, num_codeword, simd_par, C.byref(tot)))
        return tot.value


class Batch:
    """Several codes decoded by one persistent launch (ldpc_batch_*).
    ``cfgs`` holds one dict of Context keyword arguments (variant, max_iter,
    max_row_metric, beta) per code; every code of a batch uses the same
    variant (int8 offset min-sum, or one of the float decoders)."""

    def __init__(self, codes: Sequence["Code"], cfgs: Sequence[dict], device: int = 0):
        if len(codes) != len(cfgs):
            raise ValueError("one configuration per code")
        self.codes = list(codes)
        arr = (_vp * len(codes))(*[c.h for c in codes])
        cf = (Cfg * len(codes))()
        for i, k in enumerate(cfgs):
            cf[i] = Cfg(k.get("variant", LDPC_INT8_OMS), k.get("max_iter", 10), k.get("max_row_metric", 31.0),
                        k.get("beta", 1.0), k.get("llr_scale", 2.0), k.get("max_abs_llr", 24.0))
        h = _vp()
        check(lib.ldpc_batch_create(arr, cf, len(codes), device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.ldpc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_offsets(self, code: int, beta_per_layer=None):
        if beta_per_layer is None:
            check(lib.ldpc_batch_set_offsets(self.h, code, None))
            return
        b = np.ascontiguousarray(beta_per_layer, dtype=np.float32)
        check(lib.ldpc_batch_set_offsets(self.h, code, b.ctypes.data))

    def set_offset_table(self, code: int, beta=None):
        """int8 batches: offsets beta[rows][layers] for one code; iteration i
        uses row min(i, rows-1) (None restores cfg.beta)."""
        if beta is None:
            check(lib.ldpc_batch_set_offset_table(self.h, code, None, 0))
            return
        b = np.ascontiguousarray(beta, dtype=np.float32)
        check(lib.ldpc_batch_set_offset_table(self.h, code, b.ctypes.data, b.shape[0]))

    @staticmethod
    def _jobs(specs):
        arr = (BatchJob * max(1, len(specs)))()
        for i, s in enumerate(specs):
            arr[i] = BatchJob(s["code"], _ptr(s["llr"]), s["n"], _ptr(s.get("post")), _ptr(s.get("hard")),
                              _ptr(s.get("iters")), _ptr(s.get("data_bits")), s.get("ref_period", 0),
                              s.get("bucket_size", 0), _ptr(s.get("counters")), s.get("n_buckets", 1))
        return arr

    def plan(self, specs, threads: int = 0, chunks_per_cta: int = 0) -> "BatchPlan":
        """specs: dicts with code, llr, n and optional post/hard/iters/data_bits/
        ref_period/bucket_size/counters/n_buckets (torch tensors or pointers)."""
        arr = self._jobs(specs)
        h = _vp()
        check(lib.ldpc_batch_plan_create(self.h, arr, len(specs), threads, chunks_per_cta, C.byref(h)))
        return BatchPlan(h, self)

    def autotune(self, specs, sample: int = 8192):
        arr = self._jobs(specs)
        t, c, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib.ldpc_batch_autotune(self.h, arr, len(specs), sample, C.byref(t), C.byref(c), C.byref(ms)))
        return t.value, c.value, ms.value


class BatchPlan:
    def __init__(self, h, batch: Batch):
        self.h = h
        self.batch = batch

    def launch(self, stream=0):
        check(lib.ldpc_batch_plan_launch(self.h, stream or None))

    def graph_launch(self, stream=0):
        check(lib.ldpc_batch_plan_graph_launch(self.h, stream or None))

    @property
    def kernels(self) -> int:
        """Kernels one launch runs (one per geometry class)."""
        return int(lib.ldpc_batch_plan_kernels(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib.ldpc_batch_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
