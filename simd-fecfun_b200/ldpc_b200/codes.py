"""QC-LDPC code tables: base matrices, encoder schedule, decoder tables.

This module restates the reference's table generation (MATLAB, not runnable
here) in Python:

* ``GetHMatrix``   matlab/LDPC/GetHMatrix.m:27-436  -> :func:`base_matrix`
* ``lift_matrix``  matlab/LDPC/lift_matrix.m:1-20   -> :func:`_lift`
* ``encode_method`` matlab/LDPC/encode_method.m:1-194 -> :data:`ENCODE_METHOD`
* ``gen_encode``   matlab/LDPC/gen_encode.m:1-85     -> :func:`_gen_encode`
* ``decode_method`` matlab/LDPC/decode_method.m:1-52 -> :func:`_decode_method`
* ``gen_decode``   matlab/LDPC/gen_decode.m:1-68     -> :func:`_gen_decode`
* ``gen_structs``  build/gen_structs.m:28-64          -> :func:`make_code`

The two ``.dat`` writers produce the int32 file layouts that the reference's
loaders read (src/LDPCDec/decode_matrix_allocate.cpp:22-50 and
src/LDPCEnc/encode_matrix_allocate.cpp:51-86), so a code built here can be
handed to the reference's own C++ simulator unchanged.

All shifts follow the reference's rule "shift mod Z" (ExpandH.m:14 uses
``circshift(eye(Z), -s)``): check ``t`` of a layer touches bit
``(t + s) mod Z`` of each active column.
"""
from __future__ import annotations

import json
import re
import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

_DATA = os.path.join(os.path.dirname(__file__), "data", "base_matrices.json")
_TABLES: Optional[dict] = None


def _tables() -> dict:
    global _TABLES
    if _TABLES is None:
        with open(_DATA) as f:
            _TABLES = json.load(f)
    return _TABLES


# encode_method.m:12-397 -- (direct parity columns, substitution rows,
# substitution columns, inverse method, default Z).  1-based like MATLAB.
def _seq(a, b):
    return list(range(a, b + 1))


_R11 = (_seq(1, 11), _seq(2, 12))
_R7 = (_seq(1, 7), _seq(2, 8))
_R5 = (_seq(1, 5), _seq(2, 6))
_R3 = (_seq(1, 3), _seq(2, 4))
ENCODE_METHOD: Dict[str, Tuple[List[int], List[int], List[int], int, int]] = {
    "11ad 1/2": ([], _seq(1, 8), _seq(1, 8), 0, 42),
    "11ad 5/8": ([], _seq(1, 6), _seq(1, 6), 0, 42),
    "11ad 3/4": ([], _seq(1, 4), _seq(1, 4), 0, 42),
    "11ad 13/16": ([], _seq(1, 3), _seq(1, 3), 0, 42),
    "11ay 1/2": ([], _seq(1, 16), _seq(1, 16), 0, 42),
    "11ay 5/8": ([], _seq(1, 12), _seq(1, 12), 0, 42),
    "11ay 3/4": ([], _seq(1, 8), _seq(1, 8), 0, 42),
    "11ay 13/16": ([], _seq(1, 6), _seq(1, 6), 0, 42),
    "11ay 7/8": ([], _seq(1, 4), [2, 1, 3, 4], 0, 42),
    "16e 1/2": ([1], *_R11, 0, 24),
    "ITU G.hn 1/2 z14": ([1], *_R11, 0, 14),
    "802.3ca": ([8, 11, 12], [2, 6, 12, 1, 4, 5, 7, 11, 8], [4, 2, 3, 10, 7, 1, 9, 6, 5], 1, 256),
    "16e 2/3A": ([1], *_R7, 0, 24),
    "16e 2/3B": ([1], *_R7, 0, 24),
    "16e 3/4A": ([1], *_R5, 0, 24),
    "16e 3/4B": ([1], *_R5, 0, 24),
    "16e 5/6": ([1], *_R3, 0, 24),
}
for _z in (27, 54, 81):
    ENCODE_METHOD["11n 1/2 z%d" % _z] = ([1], *_R11, 0, _z)
    ENCODE_METHOD["11n 2/3 z%d" % _z] = ([1], *_R7, 0, _z)
    ENCODE_METHOD["11n 3/4 z%d" % _z] = ([1], *_R5, 0, _z)
    ENCODE_METHOD["11n 5/6 z%d" % _z] = ([1], *_R3, 0, _z)

MATRIX_SETS = list(ENCODE_METHOD.keys())

# The reference encoder works on one 512-bit word per column
# (include/enc_defs.h:3-4, gen_encode.m:6).
ENC_BW = 512
_BYTE_PER_SIMD = ENC_BW // 8


def _lift(hc: np.ndarray, liftr: Sequence[int], liftc: Sequence[int]) -> np.ndarray:
    """lift_matrix.m: each entry becomes a 2x2 diagonal block; listed blocks
    (1-based row/col of the base matrix) become anti-diagonal."""
    r, c = hc.shape
    out = -np.ones((2 * r, 2 * c), dtype=np.int64)
    out[0::2, 0::2] = hc
    out[1::2, 1::2] = hc
    for lr, lc in zip(liftr, liftc):
        row, col = 2 * (lr - 1), 2 * (lc - 1)
        top = out[row, col:col + 2].copy()
        out[row, col:col + 2] = out[row + 1, col:col + 2]
        out[row + 1, col:col + 2] = top
    return out


def base_matrix(name: str) -> Tuple[np.ndarray, int]:
    """GetHMatrix(MatrixSet): the base matrix (-1 = zero block) and its Z."""
    t = _tables()
    if name not in t:
        raise KeyError("unknown MatrixSet %r" % name)
    e = t[name]
    if "lift_of" in e:
        h, z = base_matrix(e["lift_of"])
        return _lift(h, e["liftr"], e["liftc"]), z
    h = np.array(e["H"], dtype=np.int64)
    if e.get("listed_transposed"):
        h = h.T.copy()
    return h, int(e["Z"])


def nr_base_graph(bg: int, ils: int) -> np.ndarray:
    """Hbg_matrix(Hbg_idx, Lifting_idx): 5G NR base graph ``bg`` (1 or 2)
    with the shift column of lifting-set index ``ils`` (0..7)."""
    e = _tables()["5G_BG%d" % bg]
    h = -np.ones((e["rows"], e["cols"]), dtype=np.int64)
    for r, c, vals in e["entries"]:
        h[r, c] = vals[ils]
    return h


# ----------------------------------------------------------------------------
# GF(2) helpers (bit-packed rows)
# ----------------------------------------------------------------------------

def expand_h(hc: np.ndarray, z: int) -> np.ndarray:
    """ExpandH.m: full binary H; block (r,c) = circshift(eye(Z), -s)."""
    mrow, mcol = hc.shape
    h = np.zeros((mrow * z, mcol * z), dtype=np.uint8)
    t = np.arange(z)
    for r in range(mrow):
        for c in range(mcol):
            s = hc[r, c]
            if s >= 0:
                h[r * z + t, c * z + (t + s) % z] = 1
    return h


def _gf2_solve_rows(m2: np.ndarray, rows: Sequence[int]) -> np.ndarray:
    """Rows ``rows`` of inv(M2) over GF(2), by Gauss-Jordan on [M2 | I]."""
    n = m2.shape[0]
    if m2.shape != (n, n):
        raise ValueError("M2 must be square")
    nw = (2 * n + 63) // 64
    aug = np.zeros((n, 2 * n), dtype=np.uint8)
    aug[:, :n] = m2
    aug[np.arange(n), n + np.arange(n)] = 1
    packed = np.packbits(aug, axis=1, bitorder="little")
    pad = nw * 8 - packed.shape[1]
    if pad:
        packed = np.concatenate([packed, np.zeros((n, pad), np.uint8)], axis=1)
    w = packed.view(np.uint64).copy()
    for col in range(n):
        word, bit = divmod(col, 64)
        colbits = (w[:, word] >> np.uint64(bit)) & np.uint64(1)
        cand = np.nonzero(colbits[col:])[0]
        if cand.size == 0:
            raise np.linalg.LinAlgError("M2 is singular over GF(2)")
        p = col + int(cand[0])
        if p != col:
            w[[col, p]] = w[[p, col]]
            colbits = (w[:, word] >> np.uint64(bit)) & np.uint64(1)
        hit = np.nonzero(colbits)[0]
        hit = hit[hit != col]
        if hit.size:
            w[hit] ^= w[col]
    inv = np.unpackbits(w.view(np.uint8), axis=1, bitorder="little")[:, n:2 * n]
    return inv[list(rows)]


# ----------------------------------------------------------------------------
# Encoder schedule (gen_encode.m)
# ----------------------------------------------------------------------------

def _wa_addr(col0: np.ndarray, shift: np.ndarray) -> np.ndarray:
    """gen_encode.m:42-44,61-63: byte address into the encoder work area
    (16 SIMD words per column; word 2*(shift%8) holds the 2Z copy at that bit
    offset, read at byte ``shift//8``)."""
    return col0 * 16 * _BYTE_PER_SIMD + (shift & 7) * 2 * _BYTE_PER_SIMD + (shift >> 3)


def _gen_encode(hc, z, direct_cols, subst_row, subst_col, punc_list, fill_list):
    mrow, mcol = hc.shape
    hlog = hc >= 0
    col_cnts: List[int] = []
    par_offset: List[int] = []
    if direct_cols:
        # Rows z*(d-1) of inv(M2) M1.  When the parity part is block lower
        # triangular, M2 = [[A, 0], [C, D]] with A the leading m0 x m0 base
        # blocks (5G NR: the 4 x 4 core), those rows of inv(M2) are rows of
        # inv(A) padded with zeros, so only A and the first m0 block rows of
        # M1 are expanded.
        kb = mcol - mrow
        par = hc[:, kb:]
        m0 = max(direct_cols)
        while m0 < mrow and (par[:m0, m0:] >= 0).any():
            m0 += 1
        a = expand_h(par[:m0, :m0], z)
        m1 = expand_h(hc[:m0, :kb], z)
        want = [z * (d - 1) for d in direct_cols]
        inv_rows = _gf2_solve_rows(a, want)
        row1_direct = (inv_rows.astype(np.int64) @ m1.astype(np.int64)) % 2
        for ii in range(len(direct_cols)):
            idx = np.nonzero(row1_direct[ii])[0]
            cols = idx // z
            sh = idx - cols * z
            addr = _wa_addr(cols, sh)
            par_offset.extend(int(a) for a in addr)
            col_cnts.append(len(addr))
    for r1, c1 in zip(subst_row, subst_col):
        r = r1 - 1
        target = c1 + mcol - mrow - 1           # 0-based parity column
        tmp = [c for c in np.nonzero(hlog[r])[0] if c != target]
        col_cnts.append(len(tmp))
        rot = hc[r, target]
        off = np.mod(z - rot + hc[r, tmp], z)
        par_offset.extend(int(a) for a in _wa_addr(np.array(tmp, dtype=np.int64), off))
    par_colnum = [d - 1 for d in direct_cols] + [c - 1 for c in subst_col]
    return col_cnts, par_colnum, par_offset


# ----------------------------------------------------------------------------
# Decoder tables (decode_method.m + gen_decode.m)
# ----------------------------------------------------------------------------

def _simd_offsets(v: np.ndarray, z: int, eps: int) -> np.ndarray:
    zrem = z % eps
    out = v.copy()
    m = out >= zrem
    out[m] = np.mod(out[m] - z, eps)
    return out


def _decode_method(name, hc, z, eps):
    hc = hc.copy()
    if name == "802.3ca":
        hc[[0, 1]] = hc[[1, 0]]
    mrow, mcol = hc.shape
    hlog = hc >= 0
    prev_all = np.zeros(mcol, dtype=np.int64)
    for r in range(mrow):
        cols = np.nonzero(hlog[r])[0]
        prev = prev_all[cols]
        best, best_off, best_row = -1, None, None
        base = hc[r, cols]
        for i in range(z):
            new_row = np.mod(base + i, z)
            off = _simd_offsets(new_row, z, eps)
            cnt = int(np.sum(off == prev))
            if cnt > best:
                best, best_off, best_row = cnt, off, new_row
        hc[r, cols] = best_row
        prev_all[cols] = best_off
    return hc


def _gen_decode(hc, z, eps):
    mrow, mcol = hc.shape
    hlog = hc >= 0
    zrem = z % eps
    perfect = zrem == 0
    row_weights, row_cols, row_off = [], [], []
    for r in range(mrow):
        cols = np.nonzero(hlog[r])[0]
        row_cols.extend(int(c) for c in cols)
        row_weights.append(len(cols))
        row_off.extend(int(v) for v in hc[r, cols])
    f2b_cnt, b2f_cnt, f2b_off, b2f_off, f2b_cols, b2f_cols = [], [], [], [], [], []
    prev_all = np.zeros(mcol, dtype=np.int64)
    for r in range(mrow):
        cols = np.nonzero(hlog[r])[0]
        offs = hc[r, cols].astype(np.int64)
        prev = prev_all[cols]
        offs = np.mod(offs, eps) if perfect else _simd_offsets(offs, z, eps)
        delta = offs - prev
        pos, neg = delta > 0, delta < 0
        f2b_cnt.append(int(pos.sum()))
        b2f_cnt.append(int(neg.sum()))
        f2b_off.extend(int(v) for v in prev[pos])
        b2f_off.extend(int(v) for v in prev[neg])
        f2b_cols.extend(int(c) for c in cols[pos])
        b2f_cols.extend(int(c) for c in cols[neg])
        prev_all[cols] = offs
    neg = prev_all > 0
    b2f_cnt.append(int(neg.sum()))
    b2f_off.extend(int(v) for v in prev_all[neg])
    b2f_cols.extend(int(c) for c in np.nonzero(neg)[0])
    return dict(row_weights=row_weights, row_cols=row_cols, row_shifts=row_off,
                f2b_cnt=f2b_cnt, f2b_cols=f2b_cols, f2b_off=f2b_off,
                b2f_cnt=b2f_cnt, b2f_cols=b2f_cols, b2f_off=b2f_off,
                max_row_weight=max(row_weights))


# ----------------------------------------------------------------------------
# The code object
# ----------------------------------------------------------------------------

@dataclass
class Code:
    """One QC-LDPC code with the reference's encoder and decoder tables."""
    name: str
    z: int
    mrow: int
    mcol: int
    num_par: int
    hc: np.ndarray                  # scaled base matrix before the row relabel (encoder view)
    hc_dec: np.ndarray              # base matrix after decode_method's relabel (decoder view)
    dec: dict
    par_cnts: List[int]
    par_colnum: List[int]
    par_offset: List[int]
    punc_list: List[int] = field(default_factory=list)
    fill_list: List[int] = field(default_factory=list)

    @property
    def n(self) -> int:
        return self.z * self.mcol

    @property
    def fill_cnt(self) -> int:
        return sum(e - s + 1 for s, e in zip(self.fill_list[0::2], self.fill_list[1::2]))

    @property
    def punc_cnt_bits(self) -> int:
        return sum(e - s + 1 for s, e in zip(self.punc_list[0::2], self.punc_list[1::2]))

    @property
    def k(self) -> int:
        """Information bits per (super-)codeword: Z*(mcol-mrow) - fill."""
        return self.z * (self.mcol - self.mrow) - self.fill_cnt

    @property
    def edges(self) -> int:
        return self.z * int(sum(self.dec["row_weights"]))

    def enc_schedule(self) -> List[Tuple[int, List[Tuple[int, int]]]]:
        """Decode par_offset into (parity column, [(source column, shift)])."""
        out, idx = [], 0
        for pc, cnt in zip(self.par_colnum, self.par_cnts):
            terms = []
            for a in self.par_offset[idx:idx + cnt]:
                col, rem = divmod(a, 16 * _BYTE_PER_SIMD)
                mod8, off = divmod(rem, 2 * _BYTE_PER_SIMD)
                terms.append((col, off * 8 + mod8))
            idx += cnt
            out.append((self.mcol - self.mrow + pc, terms))
        return out

    def dec_dat_bytes(self) -> bytes:
        d = self.dec
        head = [self.mrow, self.mcol, self.z, len(d["row_cols"]), d["max_row_weight"],
                len(d["f2b_cols"]), len(d["b2f_cols"])]
        body = (d["row_weights"] + d["row_cols"] + d["row_shifts"] + d["f2b_cnt"] + d["f2b_cols"]
                + d["f2b_off"] + d["b2f_cnt"] + d["b2f_cols"] + d["b2f_off"])
        return struct.pack("<%di" % (len(head) + len(body)), *(head + body))

    def enc_dat_bytes(self) -> bytes:
        vals = ([self.z, len(self.punc_list), len(self.fill_list), self.num_par, self.mrow, self.mcol]
                + self.par_cnts + self.par_colnum + self.par_offset + self.punc_list + self.fill_list)
        return struct.pack("<%di" % len(vals), *vals)

    def write_dat(self, enc_path: str, dec_path: str) -> None:
        with open(enc_path, "wb") as f:
            f.write(self.enc_dat_bytes())
        with open(dec_path, "wb") as f:
            f.write(self.dec_dat_bytes())

    def full_h(self) -> np.ndarray:
        return expand_h(self.hc, self.z)

    def syndrome(self, cw: np.ndarray) -> np.ndarray:
        """H c over GF(2) for codewords cw [n][N] (0/1), without expanding H:
        check t of row block r sums bit (t + s) % Z of every column block c
        with shift s = hc[r, c] (ExpandH.m's circulant).  Returns [n][mrow*Z]."""
        cw = np.asarray(cw, dtype=np.uint8).reshape(-1, self.n)
        z = self.z
        out = np.zeros((cw.shape[0], self.mrow * z), np.uint8)
        idx = np.arange(z)
        for r in range(self.mrow):
            acc = out[:, r * z:(r + 1) * z]
            for c in np.nonzero(self.hc[r] >= 0)[0]:
                acc ^= cw[:, c * z + (idx + int(self.hc[r, c])) % z]
        return out


def make_code(name: str, num_par: int = 1, z_over: Optional[int] = None,
              simd_size: int = 512, elem_size: int = 8) -> Code:
    """gen_structs.m:28-64 for a named MatrixSet (5G NR is built by
    :func:`make_nr_code`)."""
    if name not in ENCODE_METHOD:
        raise KeyError("unknown MatrixSet %r" % name)
    hc, _ = base_matrix(name)
    direct, srow, scol, _inv, z = ENCODE_METHOD[name]
    z = z * num_par
    hc = hc * num_par
    hc[hc < 0] = -1
    if z_over is not None:
        z = int(z_over)
    return _build(name, hc, z, num_par, direct, srow, scol, [], [], simd_size // elem_size)


# ----------------------------------------------------------------------------
# 5G NR codes (GetHMatrix.m:398-434 for '5GNR_n<#>_k<#>', with the lifting
# size rules of 3GPP TS 38.212 restated for Hbg_fill_puncture(n, k), which the
# reference calls but does not ship)
# ----------------------------------------------------------------------------

# TS 38.212 Table 5.3.2-1: set index iLS holds the lifting sizes a * 2^j <= 384
NR_LIFT_A = (2, 3, 5, 7, 9, 11, 13, 15)
NR_INFO_COLS = {1: 22, 2: 10}          # systematic base columns (2 of them punctured)
NR_ROWS = {1: 46, 2: 42}
NR_MAX_K = {1: 22 * 384, 2: 10 * 384}


def nr_lifting_sizes() -> Dict[int, int]:
    """Every 5G NR lifting size Z with its set index iLS."""
    out = {}
    for ils, a in enumerate(NR_LIFT_A):
        z = a
        while z <= 384:
            out[z] = ils
            z *= 2
    return dict(sorted(out.items()))


def nr_select(n: int, k: int) -> Tuple[int, int, int]:
    """(base graph, Z, iLS) for k information bits sent as n code bits.
    Base graph per TS 38.212 7.2.2 (graph 2 if k <= 292, or k <= 3824 and
    k/n <= 0.67, or k/n <= 0.25); Kb = 22 for graph 1, else 10/9/8/6 for
    k > 640 / > 560 / > 192 / otherwise (5.2.2); Z = the smallest lifting size
    with Kb * Z >= k."""
    if not (0 < k < n):
        raise ValueError("need 0 < k < n")
    r = k / n
    bg = 2 if (k <= 292 or (k <= 3824 and r <= 0.67) or r <= 0.25) else 1
    kb = 22 if bg == 1 else (10 if k > 640 else 9 if k > 560 else 8 if k > 192 else 6)
    sizes = nr_lifting_sizes()
    cand = [z for z in sizes if kb * z >= k]
    if not cand or k > NR_MAX_K[bg]:
        raise ValueError("k=%d needs code block segmentation (base graph %d holds %d)" % (k, bg, NR_MAX_K[bg]))
    z = cand[0]
    return bg, z, sizes[z]


def make_nr_code(n: int, k: int, num_par: int = 1, bg: Optional[int] = None, z: Optional[int] = None,
                 simd_size: int = 512, elem_size: int = 8) -> Code:
    """The reference's '5GNR_n<n>_k<k>' MatrixSet (GetHMatrix.m:398-434,
    encode_method.m:185-190, gen_structs.m:29-39).  The first 2Z systematic
    bits are punctured, parity bits beyond n are punctured at the end, and the
    Z*Kb - k filler bits end the systematic part.  ``bg``/``z`` override the
    TS 38.212 selection (e.g. to pick one lifting size of a set)."""
    sel_bg, sel_z, _ = nr_select(n, k)
    bg = sel_bg if bg is None else bg
    z = sel_z if z is None else z
    sizes = nr_lifting_sizes()
    if z not in sizes:
        raise ValueError("Z=%d is not a 5G NR lifting size" % z)
    ils = sizes[z]
    info_mcol = NR_INFO_COLS[bg]
    if k > info_mcol * z:
        raise ValueError("k=%d exceeds %d systematic columns of Z=%d" % (k, info_mcol, z))
    start_punc = 2
    p_mcol = -(-(n - k) // z) + start_punc
    if not 4 <= p_mcol <= NR_ROWS[bg]:
        raise ValueError("n=%d, k=%d needs %d parity columns (4..%d)" % (n, k, p_mcol, NR_ROWS[bg]))
    h = nr_base_graph(bg, ils)[:p_mcol, :p_mcol + info_mcol]
    h = np.where(h >= 0, h % z, -1)
    mcol = p_mcol + info_mcol
    punc_parity = z * (p_mcol - start_punc) - (n - k)
    punc = [1, start_punc * z]
    if punc_parity > 0:
        punc += [z * mcol - punc_parity + 1, z * mcol]
    fill_cnt = z * info_mcol - k
    fill = [z * info_mcol - fill_cnt + 1, z * info_mcol] if fill_cnt > 0 else []
    # gen_structs.m:33-37: scale the inclusive 1-based pairs by num_par, make them 0-based
    scale = lambda lst: [((v - 1) * num_par + 1 if i % 2 == 0 else v * num_par) - 1 for i, v in enumerate(lst)]
    srow = ([2, 4] + list(range(5, 100)))[:p_mcol - 2]
    direct = [1, 3]
    zz = z * num_par
    hc = np.where(h >= 0, h * num_par, -1)
    return _build("5GNR_n%d_k%d" % (n, k), hc, zz, num_par, direct, srow, list(srow), scale(punc), scale(fill),
                  simd_size // elem_size)


def code_by_name(name: str, **kw) -> Code:
    """make_code for the named MatrixSets, make_nr_code for '5GNR_n<n>_k<k>'."""
    if name.startswith("5GNR_"):
        m = re.fullmatch(r"5GNR_n(\d+)_k(\d+)", name)
        if not m:
            raise KeyError("bad 5G NR MatrixSet %r (want 5GNR_n<n>_k<k>)" % name)
        return make_nr_code(int(m.group(1)), int(m.group(2)), **kw)
    return make_code(name, **kw)


def _build(name, hc, z, num_par, direct, srow, scol, punc_list, fill_list, eps):
    if z > ENC_BW:
        raise ValueError("Z=%d exceeds the %d-bit encoder column" % (z, ENC_BW))
    par_cnts, par_colnum, par_offset = _gen_encode(hc, z, direct, srow, scol, punc_list, fill_list)
    hc_dec = _decode_method(name, hc, z, eps)
    dec = _gen_decode(hc_dec, z, eps)
    mrow, mcol = hc.shape
    return Code(name=name, z=z, mrow=mrow, mcol=mcol, num_par=num_par, hc=hc, hc_dec=hc_dec,
                dec=dec, par_cnts=par_cnts, par_colnum=par_colnum, par_offset=par_offset,
                punc_list=list(punc_list), fill_list=list(fill_list))


def read_dec_dat(data: bytes) -> dict:
    """Parse an ``LDPCdecode.raw.dat`` image (decode_matrix_allocate.cpp:22-50)."""
    v = np.frombuffer(data, dtype="<i4")
    mrow, mcol, z, ones, maxrow, nf, nb = (int(x) for x in v[:7])
    p = 7
    def take(n):
        nonlocal p
        out = [int(x) for x in v[p:p + n]]
        if len(out) != n:
            raise ValueError("truncated decoder table")
        p += n
        return out
    d = dict(mrow=mrow, mcol=mcol, z=z, max_row_weight=maxrow)
    d["row_weights"] = take(mrow)
    d["row_cols"] = take(ones)
    d["row_shifts"] = take(ones)
    d["f2b_cnt"] = take(mrow)
    d["f2b_cols"] = take(nf)
    d["f2b_off"] = take(nf)
    d["b2f_cnt"] = take(mrow + 1)
    d["b2f_cols"] = take(nb)
    d["b2f_off"] = take(nb)
    return d
