"""Generate csrc/gen_trees.cuh: the exclusive-combination trees of the check
update (ldpc_b200/trees.py, the schedule of the reference's min_find.pl) as
straight-line device code, one function per row weight.

    tree_<d>(T* x, T* out, comb, clamp)   T = float or double

with comb(a, b) and clamp(v) supplied by the including kernel.  Run by
build.py before compiling; the output is a build product (git-ignored).
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from ldpc_b200 import trees  # noqa: E402

MAX_D = 32


def generate(path):
    out = ["// generated by simd-fecfun_b200/gen_trees.py from ldpc_b200/trees.py -- do not edit",
           "#pragma once", "namespace ldpc {", ""]
    for d in range(2, MAX_D + 1):
        ops, outs, masks = trees.tree_program(d)
        nn = len(masks)
        out.append("template <class T, class Comb, class Clamp>")
        out.append("__device__ __forceinline__ void tree_%d(T* x, T* out, Comb comb, Clamp clamp) {" % d)
        out.append("    T n[%d];" % nn)
        out.append("#pragma unroll")
        out.append("    for (int i = 0; i < %d; ++i) n[i] = x[i];" % d)
        for op in ops:
            if op[0] == "op":
                out.append("    n[%d] = comb(n[%d], n[%d]);" % (op[1], op[2], op[3]))
            else:
                out.append("    n[%d] = clamp(n[%d]);" % (op[1], op[1]))
        for j, k in enumerate(outs):
            out.append("    out[%d] = n[%d];" % (j, k))
        out.append("}")
        out.append("")
    out.append("template <int DMAX, class T, class Comb, class Clamp>")
    out.append("__device__ __forceinline__ void run_tree(int d, T* x, T* out, Comb comb, Clamp clamp) {")
    out.append("    switch (d) {")
    for d in range(2, MAX_D + 1):
        out.append("        case %d: if constexpr (DMAX >= %d) tree_%d(x, out, comb, clamp); break;" % (d, d, d))
    out.append("        default: break;")
    out.append("    }")
    out.append("}")
    out.append("}  // namespace ldpc")
    text = "\n".join(out) + "\n"
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)


if __name__ == "__main__":
    generate(os.path.join(HERE, "csrc", "gen_trees.cuh"))
