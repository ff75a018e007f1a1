"""Reference CSR directory format: layout, round trips, malformed inputs."""
import json
import os
import shutil

import numpy as np
import pytest

import matrixgraph_b200 as mg
from matrixgraph_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ARRAYS = ("globalid", "indeg", "outdeg", "in_off", "out_off", "in_edges", "out_edges")


def expected():
    with open(os.path.join(GOLDEN, "expected.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["toy_graph", "docs_example"])
def test_golden_layout(name):
    g = mg.CSRGraph.Read(os.path.join(GOLDEN, name) + "/")
    want = expected()[name]["arrays"]
    for a in ARRAYS:
        assert g.array(a).tolist() == want[a], a


def test_golden_bytes_follow_layout():
    """graphs/0.bin is the concatenation of the arrays in the reference order."""
    d = os.path.join(GOLDEN, "toy_graph")
    raw = np.fromfile(os.path.join(d, "graphs", "0.bin"), dtype=np.uint32)
    want = expected()["toy_graph"]["arrays"]
    n = expected()["toy_graph"]["n"]
    flat = sum((want[a] for a in ARRAYS), []) + list(range(n)) * 2
    assert raw.tolist() == flat
    lab = np.fromfile(os.path.join(d, "label", "0.bin"), dtype=np.uint32)
    assert lab.tolist() == [0] * n


def test_round_trip_bytes(tmp_path):
    for name in ("toy_graph", "docs_example"):
        src = os.path.join(GOLDEN, name) + "/"
        g = mg.CSRGraph.Read(src)
        dst = str(tmp_path / name) + "/"
        g.Write(dst)
        for f in ("graphs/0.bin", "label/0.bin", "meta.yaml"):
            assert open(src + f, "rb").read() == open(dst + f, "rb").read(), f


def test_round_trip_generated(tmp_path):
    g = mg.chung_lu(500, avg_deg=6, n_labels=5)
    g.Write(str(tmp_path) + "/")
    h = mg.CSRGraph.Read(str(tmp_path) + "/")
    for a in ARRAYS + ("labels",):
        assert np.array_equal(g.array(a), h.array(a))


def test_meta_yaml_num_edges_wraps():
    """num_edges is the uint32 sum m_in + m_out, as ImmutableCSR::Write stores it."""
    meta = open(os.path.join(GOLDEN, "toy_graph", "meta.yaml")).read()
    assert "num_edges: 50" in meta


def test_flow_style_meta_accepted(tmp_path):
    src = os.path.join(GOLDEN, "docs_example")
    dst = tmp_path / "g"
    shutil.copytree(src, dst)
    (dst / "meta.yaml").write_text(
        "GraphMetadata: \n  num_vertices: 5\n  num_edges: 24\n  max_vid: 4\n  min_vid: 0\n"
        "  count_border_vertices: 0\n  num_subgraphs: 1\n"
        "  subgraphs: [{gid: 0, num_vertices: 5, num_incoming_edges: 12, "
        "num_outgoing_edges: 12, max_vid: 4, min_vid: 0}]\n")
    g = mg.CSRGraph.Read(str(dst) + "/")
    assert g.n == 5 and g.m_out == 12


def _broken(tmp_path, meta=None, truncate_bin=None, drop=None):
    src = os.path.join(GOLDEN, "toy_graph")
    dst = tmp_path / "bad"
    shutil.copytree(src, dst)
    if meta is not None:
        (dst / "meta.yaml").write_text(meta)
    if truncate_bin is not None:
        b = (dst / "graphs" / "0.bin").read_bytes()
        (dst / "graphs" / "0.bin").write_bytes(b[:truncate_bin])
    if drop:
        os.remove(dst / drop)
    return str(dst) + "/"


def test_missing_dir_is_io_error(tmp_path):
    with pytest.raises(L.MGError) as e:
        mg.CSRGraph.Read(str(tmp_path / "nope") + "/")
    assert e.value.code == L.MG_E_IO


def test_missing_label_file(tmp_path):
    with pytest.raises(L.MGError) as e:
        mg.CSRGraph.Read(_broken(tmp_path, drop="label/0.bin"))
    assert e.value.code == L.MG_E_IO


def test_malformed_meta(tmp_path):
    for meta in ("GraphMetadata:\n  num_subgraphs: 2\n",
                 "GraphMetadata:\n  num_vertices: 16\n  num_edges: 50\n  max_vid: 15\n"
                 "  min_vid: 0\n  num_subgraphs: 1\n  subgraphs:\n    - gid: 0\n"
                 "      num_vertices: -3\n",
                 "not yaml at all"):
        with pytest.raises(L.MGError) as e:
            mg.CSRGraph.Read(_broken(tmp_path / str(abs(hash(meta))), meta=meta))
        assert e.value.code == L.MG_E_FORMAT


def test_truncated_bin(tmp_path):
    with pytest.raises(L.MGError) as e:
        mg.CSRGraph.Read(_broken(tmp_path, truncate_bin=100))
    assert e.value.code == L.MG_E_FORMAT


def test_inconsistent_offsets(tmp_path):
    d = _broken(tmp_path)
    b = bytearray(open(d + "graphs/0.bin", "rb").read())
    n = 16
    off = 4 * (3 * n + (n + 1))  # out_off[0]
    b[off:off + 4] = (7).to_bytes(4, "little")
    open(d + "graphs/0.bin", "wb").write(bytes(b))
    with pytest.raises(L.MGError) as e:
        mg.CSRGraph.Read(d)
    assert e.value.code == L.MG_E_FORMAT


def test_csv_converter_semantics(tmp_path):
    """First-appearance id compaction and labels vid % range (edgelist.cu:262-290,425)."""
    p = tmp_path / "e.csv"
    p.write_text("10,20\n20,30\n30,10\n10,10\n10,20\n")
    g = mg.CSRGraph.from_csv(str(p), 2)
    assert g.n == 3
    assert g.array("labels").tolist() == [0, 1, 0]
    assert g.array("out_off").tolist() == [0, 3, 4, 5]
    assert g.array("out_edges").tolist() == [0, 1, 1, 2, 0]  # duplicates + loop kept


def test_query_shapes_symmetric():
    for name, (k, e) in mg.SHAPES.items():
        qq = mg.CSRGraph.query(k, e, [0] * k)
        assert qq.m_out == 2 * len(e), name
        assert qq.array("in_off").tolist() == qq.array("out_off").tolist()
