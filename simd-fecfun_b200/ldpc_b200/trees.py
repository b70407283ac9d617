"""Exclusive-combination trees of the check-node update.

For a check of weight ``d`` the reference computes, for every edge ``j``,
the combination (min for min-sum, product of tanh for sum-product) of the
other ``d-1`` edges with a fixed balanced tree generated by
src/LDPCDec/min_find.pl:24-164 (table of functions min_find_wrap.pl:6,42-60).
Integer min is exact in any order, but the float product is not, so the GPU
sum-product kernel and the CPU oracle evaluate *this* schedule to agree with
the reference bit for bit.

This module restates the generator's algorithm and returns the schedule as a
small program over node ids:

* nodes ``0..d-1`` are the edge inputs (tanh(|Q|/2), or |Q|-beta clamped at 0);
* ``("op", dst, a, b)``   node[dst] = combine(node[a], node[b]);
* ``("clamp", n)``        node[n] = min(Max_val, node[n])   (min_find.pl:99-107);
* ``outputs[j]``          the node holding the combination excluding edge j.

Nodes are identified in the generator by the bit mask of the inputs they
combine; the masks are kept here for checking against the generator.
"""
from __future__ import annotations

from functools import lru_cache
from typing import List, Tuple

MAX_ROW_WEIGHT = 53      # min_find_wrap.pl:6 (limit from the double mantissa used for masks)


@lru_cache(maxsize=None)
def tree_program(d: int) -> Tuple[Tuple[tuple, ...], Tuple[int, ...], Tuple[int, ...]]:
    """Return (ops, outputs, masks) for row weight ``d`` (2 <= d <= 53)."""
    if not 2 <= d <= MAX_ROW_WEIGHT:
        raise ValueError("row weight %d outside 2..%d" % (d, MAX_ROW_WEIGHT))
    ids = {}
    masks: List[int] = []

    def node(mask):
        if mask not in ids:
            ids[mask] = len(masks)
            masks.append(mask)
        return ids[mask]

    ops: List[tuple] = []
    for i in range(d):
        node(1 << i)
    levels_m = [[1 << i for i in range(d)]]
    levels_c = [[1] * d]
    # step 1: reduce pairwise down to two nodes
    lvl = 1
    while True:
        prev_m, prev_c = levels_m[lvl - 1], levels_c[lvl - 1]
        nprev = len(prev_m)
        half = nprev >> 1
        cur_m, cur_c = [], []
        for i in range(half):
            m1, m2 = prev_m[2 * i], prev_m[2 * i + 1]
            cur_m.append(m1 | m2)
            cur_c.append(prev_c[2 * i] + prev_c[2 * i + 1])
            if d != 2:
                ops.append(("op", node(m1 | m2), ids[m1], ids[m2]))
        if nprev & 1:
            half += 1
            cur_m.append(prev_m[-1])
            cur_c.append(prev_c[-1])
        order = sorted(range(len(cur_m)), key=lambda k: cur_c[k])   # stable, like Perl's mergesort
        levels_m.append([cur_m[k] for k in order])
        levels_c.append([cur_c[k] for k in order])
        lvl += 1
        if not half > 2:
            break
    lvl -= 1
    comb = lvl - 1
    cur_m, cur_c = list(levels_m[lvl]), list(levels_c[lvl])
    for i in range(2):
        ops.append(("clamp", ids[1 << i] if d == 2 else ids[cur_m[i]]))
    # step 2: combine back up until every exclusive set exists
    end_cnt = 0
    seen = set()
    while True:
        next_m, next_c, used = [], [], set()
        pm, pc = levels_m[comb], levels_c[comb]        # comb == -1 reads the last level, as Perl does
        for i in range(len(cur_m)):
            for j in range(len(pm)):
                t1, t2 = pc[j], cur_c[i]
                m1, m2 = pm[j], cur_m[i]
                m = m1 | m2
                if m1 & m2 or t1 + t2 == d or m in seen:
                    continue
                if t1 + t2 == d - 1:
                    end_cnt += 1
                ops.append(("op", node(m), ids[m1], ids[m2]))
                seen.add(m)
                used.add(m2)
                if t1 + t2 != d - 1:
                    next_m.append(m)
                    next_c.append(t1 + t2)
        for i in range(len(cur_m)):
            if cur_m[i] not in used:
                next_m.append(cur_m[i])
                next_c.append(cur_c[i])
        comb -= 1
        cur_m, cur_c = next_m, next_c
        if not end_cnt < d or comb < -1:
            break
    full = (1 << d) - 1
    outputs = tuple(ids[full ^ (1 << j)] for j in range(d))
    return tuple(ops), outputs, tuple(masks)


def flat_program(d: int) -> List[int]:
    """Program as int quadruples: (0, dst, a, b) combine, (1, n, 0, 0) clamp,
    followed by d quadruples (2, j, node, 0) naming the outputs."""
    ops, outs, _ = tree_program(d)
    flat: List[int] = []
    for op in ops:
        if op[0] == "op":
            flat += [0, op[1], op[2], op[3]]
        else:
            flat += [1, op[1], 0, 0]
    for j, n in enumerate(outs):
        flat += [2, j, n, 0]
    return flat


def num_nodes(d: int) -> int:
    return len(tree_program(d)[2])
