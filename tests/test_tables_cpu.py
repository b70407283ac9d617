"""Code tables: encoder schedules produce codewords of the code (H c = 0,
the reference's own encoder check, build/LDPCenc_test.m:40-43), the .dat
images round-trip, and the tree schedule restates min_find.pl exactly."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT


@pytest.mark.parametrize("num_par", [1, 2])
def test_every_matrix_set_encodes_to_codewords(oracle, num_par):
    from ldpc_b200 import codes
    rng = np.random.default_rng(num_par)
    for name in codes.MATRIX_SETS:
        if name == "802.3ca":
            continue   # 3072-bit GF(2) inverse: covered by test_8023ca_direct_columns
        code = codes.make_code(name, num_par=num_par)
        info = rng.integers(0, 2, (3, code.z * (code.mcol - code.mrow)), dtype=np.uint8)
        cw = oracle.encode(code, info)
        H = code.full_h().astype(np.int64)
        assert not ((cw.astype(np.int64) @ H.T) % 2).any(), name


@pytest.mark.parametrize("z", [24, 28, 52, 76, 96])
def test_16e_z_sweep(oracle, z):
    """The reference's 16e rule: shifts of the Z=96 table taken mod Z (z_over)."""
    from ldpc_b200 import codes
    code = codes.make_code("16e 1/2", z_over=z)
    assert code.z == z and max(code.dec["row_shifts"]) < z
    info = np.random.default_rng(z).integers(0, 2, (2, 12 * z), dtype=np.uint8)
    cw = oracle.encode(code, info)
    assert not ((cw.astype(np.int64) @ code.full_h().astype(np.int64).T) % 2).any()


def test_dat_roundtrip_and_layout():
    from ldpc_b200 import codes
    code = codes.make_code("11ad 1/2")
    d = codes.read_dec_dat(code.dec_dat_bytes())
    assert (d["mrow"], d["mcol"], d["z"]) == (8, 16, 42)
    assert d["row_weights"] == [5, 6, 6, 6, 7, 7, 7, 8]
    assert sum(d["row_weights"]) == 52 and len(d["row_cols"]) == 52
    assert d["row_cols"][:5] == [0, 2, 4, 6, 8]
    enc = np.frombuffer(code.enc_dat_bytes(), "<i4")
    assert list(enc[:6]) == [42, 0, 0, 1, 8, 16]
    # decode_method's relabel: each layer's shifts = base shifts + one constant
    hc, _ = codes.base_matrix("11ad 1/2")
    e0 = 0
    for r, w in enumerate(d["row_weights"]):
        cols = d["row_cols"][e0:e0 + w]
        rot = {(d["row_shifts"][e0 + j] - hc[r, c]) % 42 for j, c in enumerate(cols)}
        assert len(rot) == 1
        e0 += w


def test_lifted_and_transposed_tables():
    from ldpc_b200 import codes
    h, z = codes.base_matrix("11ay 1/2")
    assert h.shape == (16, 32) and z == 42
    base, _ = codes.base_matrix("11ad 1/2")
    assert (h >= 0).sum() == 2 * (base >= 0).sum()
    h3, z3 = codes.base_matrix("802.3ca")
    assert h3.shape == (12, 69) and z3 == 256
    bg1 = codes.nr_base_graph(1, 1)
    assert bg1.shape == (46, 68) and (bg1 >= 0).sum() == 316
    bg2 = codes.nr_base_graph(2, 0)
    assert bg2.shape == (42, 52) and (bg2 >= 0).sum() == 197


def test_tree_schedule_matches_generator_golden():
    from ldpc_b200 import trees
    with open(os.path.join(ROOT, "tests", "golden", "min_find_trees.json")) as f:
        gold = json.load(f)
    for d in range(2, 54):
        ops, outs, masks = trees.tree_program(d)
        hx = lambda m: format(m, "x").zfill(int((d - 0.1) / 4) + 1)  # noqa: E731
        st = [["in", hx(1 << i), i] for i in range(d)]
        for op in ops:
            if op[0] == "op":
                st.append(["op", hx(masks[op[1]]), hx(masks[op[2]]), hx(masks[op[3]])])
            else:
                st.append(["clamp", hx(masks[op[1]])])
        st += [["out", j, hx(masks[n])] for j, n in enumerate(outs)]
        if str(d) in gold["full"]:
            assert st == gold["full"][str(d)], d
        assert hashlib.sha256(json.dumps(st).encode()).hexdigest() == gold["sha256"][str(d)], d


def test_tree_min_equals_exclusive_minimum():
    """Every output of the min tree is min(Max, min over the other inputs)."""
    from ldpc_b200 import trees
    rng = np.random.default_rng(1)
    for d in range(2, 30):
        ops, outs, _ = trees.tree_program(d)
        for _ in range(20):
            x = list(rng.integers(0, 40, d))
            mx = 31
            node = x + [0] * (trees.num_nodes(d) - d)
            for op in ops:
                if op[0] == "op":
                    node[op[1]] = min(node[op[2]], node[op[3]])
                else:
                    node[op[1]] = min(mx, node[op[1]])
            for j in range(d):
                assert node[outs[j]] == min([mx] + [x[k] for k in range(d) if k != j])


def test_nr_lifting_size_selection():
    """TS 38.212 lifting sets (51 sizes) and the base-graph / Z choice for the
    5G NR workloads: graph 1 Z=384 (k=8448) and graph 2 Z=64/128/256."""
    from ldpc_b200 import codes
    sizes = codes.nr_lifting_sizes()
    assert len(sizes) == 51 and max(sizes) == 384 and sizes[384] == 1 and sizes[256] == 0 and sizes[15] == 7
    assert codes.nr_select(25344, 8448) == (1, 384, 1)
    assert codes.nr_select(6400, 1280) == (2, 128, 0)
    assert codes.nr_select(12800, 2560) == (2, 256, 0)
    assert codes.nr_select(3136, 576) == (2, 64, 0)     # Kb = 9: 9*60 < 576 <= 9*64
    assert codes.nr_select(300, 100) == (2, 18, 4)      # Kb = 6
    with pytest.raises(ValueError):
        codes.nr_select(30000, 9000)                     # needs code block segmentation


@pytest.mark.parametrize("name,mrow,mcol,punc,fill", [
    ("5GNR_n25344_k8448", 46, 68, [0, 767], []),
    ("5GNR_n3136_k576", 42, 52, [0, 127], [576, 639]),
    ("5GNR_n1000_k500", 10, 20, [0, 127, 1268, 1279], [500, 639]),
    ("5GNR_n10000_k8000", 8, 30, [0, 767, 11216, 11519], [8000, 8447]),
])
def test_nr_codes_encode_to_codewords(oracle, name, mrow, mcol, punc, fill):
    """GetHMatrix's 5GNR_n<n>_k<k>: shape, puncture/filler lists, and H c = 0
    for the encoder schedule (direct parity columns 1 and 3, then substitution)."""
    from ldpc_b200 import codes
    c = codes.code_by_name(name)
    assert (c.mrow, c.mcol, c.punc_list, c.fill_list) == (mrow, mcol, punc, fill)
    sent = c.n - c.punc_cnt_bits - c.fill_cnt          # punctured and filler bits are not sent
    n_req, k_req = (int(v) for v in name[6:].split("_k"))
    assert sent == n_req and c.k == k_req
    rng = np.random.default_rng(2)
    info = rng.integers(0, 2, (6, (c.mcol - c.mrow) * c.z), dtype=np.uint8)
    for s, e in zip(c.fill_list[0::2], c.fill_list[1::2]):
        info[:, s:e + 1] = 0
    cw = oracle.encode(c, info)
    assert np.array_equal(cw[:, :info.shape[1]], info)
    assert not c.syndrome(cw).any()


def test_nr_num_par_scales_lists():
    """gen_structs.m:33-37: each puncture/filler pair scales by num_par."""
    from ldpc_b200 import codes
    a = codes.make_nr_code(1000, 500)
    b = codes.make_nr_code(1000, 500, num_par=2)
    assert b.z == 2 * a.z
    assert b.punc_list == [a.punc_list[0] * 2, (a.punc_list[1] + 1) * 2 - 1, a.punc_list[2] * 2, (a.punc_list[3] + 1) * 2 - 1]
    assert b.fill_list == [a.fill_list[0] * 2, (a.fill_list[1] + 1) * 2 - 1]


def test_syndrome_matches_expanded_h(oracle):
    from ldpc_b200 import codes
    c = codes.make_code("16e 1/2")
    rng = np.random.default_rng(5)
    x = rng.integers(0, 2, (3, c.n), dtype=np.uint8)
    want = (x.astype(np.int64) @ c.full_h().astype(np.int64).T) % 2
    assert np.array_equal(c.syndrome(x), want.astype(np.uint8))
