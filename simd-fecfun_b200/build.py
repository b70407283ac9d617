"""Build libldpc_b200.so (the C-ABI library with the sm_100a kernels).

    python simd-fecfun_b200/build.py [--force] [-j N]

Each csrc/*.cu is compiled to csrc/_build/*.o with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and the
objects are linked into ldpc_b200/libldpc_b200.so.  A unit is rebuilt when it
or any csrc header is newer than its object.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
INC = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "ldpc_b200", "libldpc_b200.so")
SIM = os.path.join(HERE, "ldpc_b200", "ldpc_sim")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
         "--expt-relaxed-constexpr", "-I" + INC, "-I" + CSRC]


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INC, "*.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, force: bool, hdr_time: float, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    sys.path.insert(0, HERE)
    import gen_trees
    gen_trees.generate(os.path.join(CSRC, "gen_trees.cuh"))
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _newest_header()
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    # the process-level drop-in (ldpc_sim), linked against the library next to it
    src = os.path.join(HERE, "sim", "ldpc_sim.cpp")
    if force or not os.path.exists(SIM) or os.path.getmtime(SIM) < max(os.path.getmtime(src), os.path.getmtime(LIB)):
        cmd = ["g++", "-O2", "-std=c++17", "-I" + INC, src, "-o", SIM, "-L" + os.path.dirname(LIB), "-lldpc_b200",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("ldpc_sim build failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true", help="print ptxas register/spill usage")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
