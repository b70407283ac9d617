"""Run N simulator processes and sum what they report, as the reference's
experiment driver does (build/run_LDPCsim.pl:98-128 spawns ``num_proc``
copies of the LDPCtop_* binary, writes the 820-byte blob to each, and
parse_line at :156-178 sums every "loop" line per SNR point).

Differences, by design:
  * a process that dies (a signal, a non-zero exit, output cut short) does
    not stop the run: its completed "loop" lines still count, and the result
    lists it under ``failed`` with its exit status and the number of loop
    lines it delivered (the Perl driver sums whatever its children print and
    cannot tell a dead child from a finished one);
  * every process may get its own blob (for example its own seeds).

Works with ldpc_sim (linked as LDPCtop_<variant>_b200) or with the
reference's own binaries; nothing here touches a GPU.
"""
from __future__ import annotations

import os
import selectors
import subprocess
from typing import Callable, Dict, List, Optional, Sequence

from .simproto import LOOP_RE, MATRIX_RE


def run(exe, blobs: Sequence[bytes], cwd: Optional[str] = None, env: Optional[Dict[str, str]] = None,
        on_line: Optional[Callable[[int, subprocess.Popen, str], None]] = None, timeout: float = 3600.0) -> Dict:
    """Start one process of ``exe`` (a path, or a command as a list) per
    blob, feed it the blob on stdin and read its output until every process
    has ended.

    Returns ``{"snr": {snr: {...sums...}}, "cw_per_loop": n, "processes": k,
    "failed": [...], "loops_received": m}``; the per-SNR sums are
    uncoded bit errors, iterations, bit errors, codeword errors, decoder
    ticks and codewords (``cw_per_loop`` times the number of loop lines), as
    run_LDPCsim.pl accumulates them.  ``on_line(proc_index, popen, line)`` is
    called for every line read (a test uses it to kill a process mid-run)."""
    sel = selectors.DefaultSelector()
    procs: List[subprocess.Popen] = []
    bufs: List[bytes] = []
    loops = [0] * len(blobs)
    cw_count = [None] * len(blobs)
    num_par = [1] * len(blobs)
    totals: Dict[float, Dict[str, int]] = {}
    for i, b in enumerate(blobs):
        p = subprocess.Popen([exe] if isinstance(exe, str) else list(exe), stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                             cwd=cwd, env=env)
        try:
            p.stdin.write(b)
            p.stdin.close()
        except BrokenPipeError:
            pass
        procs.append(p)
        bufs.append(b"")
        sel.register(p.stdout, selectors.EVENT_READ, i)

    def handle(i: int, line: str) -> None:
        if line.startswith("CW Count"):
            cw_count[i] = int(line.split()[2])
        elif line.startswith("Matrix Params"):
            m = MATRIX_RE.search(line)
            if m:
                num_par[i] = int(m.group(4))
        elif line.startswith("loop"):
            m = LOOP_RE.search(line)
            if not m:
                return
            snr = float(m.group(1))
            t = totals.setdefault(snr, {"uncoded_bit_errors": 0, "iterations": 0, "bit_errors": 0, "cw_errors": 0,
                                        "dec_ticks": 0, "codewords": 0})
            t["uncoded_bit_errors"] += int(m.group(2))
            t["iterations"] += int(m.group(3))
            t["bit_errors"] += int(m.group(4))
            t["cw_errors"] += int(m.group(5))
            t["dec_ticks"] += int(m.group(6))
            t["codewords"] += (cw_count[i] or 0) * num_par[i]
            loops[i] += 1
        if on_line:
            on_line(i, procs[i], line)

    open_count = len(procs)
    while open_count:
        events = sel.select(timeout)
        if not events:
            for p in procs:
                if p.poll() is None:
                    p.kill()
            raise TimeoutError("no output from the simulator processes for %.0f s" % timeout)
        for key, _ in events:
            i = key.data
            chunk = os.read(key.fileobj.fileno(), 65536)
            if not chunk:
                sel.unregister(key.fileobj)
                open_count -= 1
                if bufs[i]:
                    handle(i, bufs[i].decode(errors="replace"))   # a last line without its newline
                    bufs[i] = b""
                continue
            bufs[i] += chunk
            *lines, bufs[i] = bufs[i].split(b"\n")
            for ln in lines:
                handle(i, ln.decode(errors="replace"))
    failed = []
    for i, p in enumerate(procs):
        rc = p.wait()
        if rc != 0:
            failed.append({"process": i, "returncode": rc, "loops_received": loops[i]})
    return {"snr": dict(sorted(totals.items())), "cw_per_loop": cw_count[0], "processes": len(procs),
            "failed": failed, "loops_received": sum(loops)}
