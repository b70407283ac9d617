"""Extract the standard QC-LDPC base matrices into ``base_matrices.json``.

The numbers are the published base matrices of IEEE 802.11ad/ay, 802.16e,
802.11n, ITU-T G.hn, IEEE 802.3ca and 3GPP TS 38.212 (5G NR base graphs 1
and 2).  The reference keeps them as MATLAB source in
``matlab/LDPC/GetHMatrix.m:27-436`` and ``matlab/LDPC/Hbg_matrix.m:3-525``;
this script parses those two files once and writes the tables in a neutral
JSON form.  Lifted codes (11ay) and the transposed 802.3ca listing are
stored exactly as listed in the source; ``ldpc_b200.codes`` applies the
lifting and the transposition.

Run it from a checkout that has the reference tree:

    python extract_base_matrices.py <reference root> base_matrices.json
"""
import json
import re
import sys


def _parse_matrix(body):
    rows = []
    for line in body.replace(";", "\n").splitlines():
        vals = [int(v) for v in re.findall(r"-?\d+", line)]
        if vals:
            rows.append(vals)
    return rows


def parse_gethmatrix(text):
    out = {}
    # split on "case '<name>'" markers
    parts = re.split(r"\n\s*case\s+'([^']+)'", text)
    for name, body in zip(parts[1::2], parts[2::2]):
        body = body.split("\n\totherwise")[0]
        entry = {}
        mz = re.search(r"\bZ\s*=\s*(\d+)\s*;", body)
        if mz:
            entry["Z"] = int(mz.group(1))
        mh = re.search(r"\bH\s*=\s*\[(.*?)\]\s*;", body, re.S)
        if mh and "GetHMatrix" not in mh.group(1):
            entry["H"] = _parse_matrix(mh.group(1))
        mb = re.search(r"GetHMatrix\('([^']+)'\)", body)
        if mb:
            entry["lift_of"] = mb.group(1)
            entry["liftr"] = [int(v) for v in re.findall(r"-?\d+", re.search(r"liftr\s*=\s*\[(.*?)\]", body).group(1))]
            entry["liftc"] = [int(v) for v in re.findall(r"-?\d+", re.search(r"liftc\s*=\s*\[(.*?)\]", body).group(1))]
        if re.search(r"H\s*=\s*transpose\(H\)", body):
            entry["listed_transposed"] = True
        out[name] = entry
    return out


def parse_hbg(text):
    out = {}
    for bg, nr, nc in ((1, 46, 68), (2, 42, 52)):
        ents = re.findall(r"Hbg%d\((\d+)\+1,(\d+)\+1,:\)\s*=\s*\[([^\]]*)\]" % bg, text)
        out["5G_BG%d" % bg] = {
            "rows": nr, "cols": nc,
            "entries": [[int(r), int(c), [int(v) for v in vals.split()]] for r, c, vals in ents],
        }
    return out


def main():
    root, dst = sys.argv[1], sys.argv[2]
    with open(root + "/matlab/LDPC/GetHMatrix.m") as f:
        tables = parse_gethmatrix(f.read())
    with open(root + "/matlab/LDPC/Hbg_matrix.m") as f:
        tables.update(parse_hbg(f.read()))
    with open(dst, "w") as f:
        json.dump(tables, f, separators=(",", ":"))
        f.write("\n")


if __name__ == "__main__":
    main()
