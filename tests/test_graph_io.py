"""Host graph substrate: .gr format (FileGraph.cpp:44-53), the reference's
graph-convert fixtures, seeded generators and host transpose.  CPU only."""
import hashlib
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from galois_b200 import (GbError, HostCSR, assign_weights_f32, assign_weights_u32, csr_to_edgelist, edgelist_to_csr,
                         erdos_renyi, grid2d, read_gr, rmat, transpose, write_gr)
from galois_b200 import _lib

GOLD = Path(__file__).resolve().parent / "golden"


def small_graph():
    return HostCSR.from_edges(5, [0, 0, 1, 3, 3, 3, 4], [1, 2, 2, 0, 1, 4, 4],
                              w_u32=[10, 20, 30, 40, 50, 60, 70])


@pytest.mark.parametrize("edge_bytes", [0, 4, -4])
def test_gr_roundtrip(tmp_path, edge_bytes):
    g = small_graph()
    g.w_f32 = np.linspace(0.1, 0.7, g.m).astype(np.float32)
    p = tmp_path / "g.gr"
    write_gr(p, g, edge_bytes)
    h = read_gr(p, edge_bytes)
    assert np.array_equal(h.end_offs, g.end_offs) and np.array_equal(h.col, g.col)
    if edge_bytes == 4:
        assert np.array_equal(h.w_u32, g.w_u32)
    if edge_bytes == -4:
        assert np.array_equal(h.w_f32, g.w_f32)


def test_gr_layout_bytes(tmp_path):
    """Header {ver, sizeofEdge, n, m}, end offsets, uint32 dsts, 4-byte pad for
    odd m, then edge data (FileGraph.cpp:44-53)."""
    g = small_graph()  # m = 7 (odd)
    p = tmp_path / "g.gr"
    write_gr(p, g, 4)
    raw = p.read_bytes()
    ver, szedge, n, m = struct.unpack_from("<4Q", raw, 0)
    assert (ver, szedge, n, m) == (1, 4, 5, 7)
    ends = struct.unpack_from("<5Q", raw, 32)
    assert list(ends) == g.end_offs.tolist()
    dst = struct.unpack_from("<7I", raw, 32 + 40)
    assert list(dst) == g.col.tolist()
    pad_off = 32 + 40 + 28
    assert struct.unpack_from("<I", raw, pad_off)[0] == 0
    assert list(struct.unpack_from("<7I", raw, pad_off + 4)) == g.w_u32.tolist()
    assert len(raw) == pad_off + 4 + 28


def test_gr_version2_reader(tmp_path):
    g = small_graph()
    p = tmp_path / "v2.gr"
    with open(p, "wb") as f:
        f.write(struct.pack("<4Q", 2, 4, g.n, g.m))
        f.write(g.end_offs.astype("<u8").tobytes())
        f.write(g.col.astype("<u8").tobytes())
        f.write(b"\0" * 8)  # odd m: v2 pads one 8-byte slot (FileGraph.cpp:127-134)
        f.write(g.w_u32.astype("<u4").tobytes())
    h = read_gr(p, 4)
    assert np.array_equal(h.col, g.col) and np.array_equal(h.w_u32, g.w_u32)


def test_gr_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.gr"
    p.write_bytes(struct.pack("<4Q", 3, 0, 1, 0) + b"\0" * 8)
    with pytest.raises(GbError) as e:
        read_gr(p)
    assert e.value.status == _lib.GB_ERR_FORMAT
    p.write_bytes(struct.pack("<4Q", 1, 0, 4, 10))  # truncated
    with pytest.raises(GbError):
        read_gr(p)
    g = small_graph()
    g.col = g.col.copy()
    g.col[2] = 9  # destination >= n
    write_gr(p, g, 0)
    with pytest.raises(GbError):
        read_gr(p)
    with pytest.raises(GbError) as e:
        read_gr(tmp_path / "missing.gr")
    assert e.value.status == _lib.GB_ERR_FILE
    write_gr(p, small_graph(), 0)  # sizeofEdge 0
    with pytest.raises(GbError) as e:
        read_gr(p, 4)  # asks for 4-byte edge data
    assert e.value.status == _lib.GB_ERR_FORMAT


@pytest.mark.parametrize("inp,skip,delim,expected", [
    ("with-blank-lines.edgelist", False, "", "with-blank-lines.edgelist.expected"),
    ("sample.csv", True, ",", "with-blank-lines.edgelist.expected"),
    ("with-comments.edgelist", False, "", "with-comments.edgelist.expected"),
])
def test_graph_convert_fixtures(tmp_path, inp, skip, delim, expected):
    """tools/graph-convert/CMakeLists.txt:29-31: edgelist2gr / csv2gr then
    gr2edgelist must reproduce the .expected file byte for byte."""
    src = GOLD / "graph_convert" / inp
    g = edgelist_to_csr(src, skip, delim)
    gr = tmp_path / "t.gr"
    write_gr(gr, g, 0)
    back = read_gr(gr, 0)
    out = tmp_path / "t.edgelist"
    csr_to_edgelist(out, back)
    assert out.read_bytes() == (GOLD / "graph_convert" / expected).read_bytes()


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        if a is not None:
            h.update(a.tobytes())
    return h.hexdigest()[:32]


def test_generators_match_committed_digests():
    gold = json.loads((GOLD / "generators.json").read_text())
    g, perm = rmat(12, 16, seed=20, symmetrize=True)
    assert _digest(g.end_offs, g.col, perm) == gold["rmat12_sym_seed20"]["digest"]
    g, perm = rmat(11, 16, seed=22, symmetrize=False)
    assign_weights_u32(g, 1, 255, seed=22)
    assert _digest(g.end_offs, g.col, g.w_u32, perm) == gold["rmat11_dir_seed22_w"]["digest"]
    g = grid2d(33, 47)
    assert _digest(g.end_offs, g.col) == gold["grid33x47"]["digest"]
    g = erdos_renyi(5000, 8.0, seed=3)
    assign_weights_f32(g, seed=3)
    assert _digest(g.end_offs, g.col, g.w_f32) == gold["er5000_seed3_wf"]["digest"]


def test_rmat_properties():
    g, perm = rmat(11, 16, seed=7, symmetrize=True)
    offs = g.offs
    src = np.repeat(np.arange(g.n), g.degrees())
    assert (src != g.col).all()  # no self-loops
    for v in range(0, g.n, 97):  # sorted, unique adjacency
        row = g.col[offs[v]:offs[v + 1]]
        assert (np.diff(row.astype(np.int64)) > 0).all()
    fwd = set(zip(src.tolist(), g.col.tolist()))
    assert all((b, a) in fwd for a, b in list(fwd)[:5000])  # symmetric
    assert sorted(perm.tolist()) == list(range(g.n))
    g2, _ = rmat(11, 16, seed=7, symmetrize=True)
    assert np.array_equal(g.col, g2.col)  # deterministic
    g3, _ = rmat(11, 16, seed=8, symmetrize=True)
    assert not np.array_equal(g.col[:1000], g3.col[:1000])


def test_grid_and_er_and_weights():
    g = grid2d(64, 50)
    assert g.m == 2 * 64 * 49 + 2 * 50 * 63
    assert g.degrees().max() == 4 and g.degrees().min() == 2
    e = erdos_renyi(20000, 8.0, seed=1)
    assert 7.5 < e.m / e.n < 8.1
    assign_weights_u32(e, 1, 255, seed=2)
    assert e.w_u32.min() >= 1 and e.w_u32.max() <= 255 and len(np.unique(e.w_u32)) == 255
    assign_weights_f32(e, seed=2)
    assert e.w_f32.min() > 0 and e.w_f32.max() <= 1.0


def test_host_transpose():
    g, _ = rmat(10, 8, seed=3, symmetrize=False)
    assign_weights_u32(g, 1, 9, seed=1)
    t, emap = transpose(g)
    src = np.repeat(np.arange(g.n), g.degrees())
    tsrc = np.repeat(np.arange(t.n), t.degrees())
    assert np.array_equal(g.col[emap], tsrc)  # arc emap[k] of g points at the row of k
    assert np.array_equal(src[emap], t.col)
    assert np.array_equal(g.w_u32[emap], t.w_u32)
    tt, _ = transpose(t)
    assert np.array_equal(tt.col, g.col) and np.array_equal(tt.end_offs, g.end_offs)


def test_mt19937_known_answer():
    """The oracle's generator is the standard's: the 10000th output of a
    default-constructed std::mt19937 is 4123659995 ([rand.predef])."""
    import oracle

    assert int(oracle.mt19937_raw(10000)[-1]) == 4123659995


@pytest.mark.parametrize("dtype,lo,hi", [("u32", 1, 100), ("u32", 1, 255), ("f32", 1, 100)])
def test_reference_random_weights_gr(tmp_path, dtype, lo, hi):
    """gr2randomweightgr (graph-convert.cpp:1145-1190): a .gr written with
    assign_weights_reference carries, in arc order, the draws of a default
    std::mt19937 through the uniform distribution the converter uses."""
    import oracle
    from galois_b200 import assign_weights_reference

    g, _ = rmat(9, 8, seed=3, symmetrize=False)
    assign_weights_reference(g, lo, hi, dtype)
    eb = 4 if dtype == "u32" else -4
    p = tmp_path / "w.gr"
    write_gr(p, g, eb)
    raw = p.read_bytes()
    ver, szedge, n, m = struct.unpack_from("<4Q", raw, 0)
    assert (ver, szedge, n, m) == (1, 4, g.n, g.m)
    data_off = 32 + 8 * n + 4 * m + (4 if m % 2 else 0)
    got = np.frombuffer(raw, dtype=np.uint32, count=m, offset=data_off)
    want = oracle.gr2randomweight(m, lo, hi, dtype)
    assert np.array_equal(got, want.view(np.uint32))
    if dtype == "u32":
        assert got.min() >= lo and got.max() <= hi
    else:
        f = got.view(np.float32)
        assert f.min() >= lo and f.max() < hi
    h = read_gr(p, eb)
    assert np.array_equal(h.w_u32 if dtype == "u32" else h.w_f32.view(np.uint32), want.view(np.uint32))


def test_reference_random_weights_rejects_bad_arguments():
    from galois_b200 import assign_weights_reference

    g = small_graph()
    with pytest.raises(GbError):
        assign_weights_reference(g, 5, 1)
    with pytest.raises(GbError):
        assign_weights_reference(g, -3, 5, "u32")
