"""Graph files straight to CSR (gvizCudaLoadEdgesFile / gvizCudaLoadObjFile /
gvizCudaLoadGexfFile)
against gviz's own loaders (src/utils/graphLoader.c, the reference compiled
from its sources) followed by its adjacency order: the same vertex numbering,
the same neighbour lists, the same failures."""
import numpy as np
import pytest

EDGES_CASES = {
    "plain_1based": "1 2\n2 3\n3 1\n",
    "zero_based_weights_comments": "% header comment\n0 5 0.5\n5 7 1\n\n  % indented comment\n7 0 2\n",
    "duplicates_selfloops": "4 4\n1 2\n2 1\n1 2\n9 4\n",
    "sparse_ids_crlf": "1000000 3\r\n3 77\r\n77 1000000\r\n4000000 3\r\n",
    "tabs_and_blanks": "\t10\t11\n\n11   12\t9.5\n",
    "header": "3 2\n1 2\n2 3\n",
}
EDGES_BAD = {
    "negative": "1 2\n-3 4\n",
    "one_column": "1 2\n3\n",
    "word": "a b\n",
    "empty": "",
    "only_comments": "% nothing\n%\n",
}
OBJ_CASES = {
    "quad_and_tri": "# mesh\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\nf 1 3 2\n",
    "slashes_negative": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\nf 1/1/1 2/1/1 3/1/1\n"
                        "v 1 1 0\nf -1//1 -2//1 -3//1\n",
    "shared_edges_isolated": "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 5 5 5\n"
                             "f 1 2 3\nf 3 2 4\nf 4 3 1\ng group\nusemtl m\ns off\n",
    "degenerate": "v 0 0 0\nv 1 0 0\nf 1 1 2\nf 2\nf 1 2\n",
}
OBJ_BAD = {"zero_index": "v 0 0 0\nf 0 1\n", "out_of_range": "v 0 0 0\nf 1 2\n",
           "no_vertices": "# empty\n", "bad_token": "v 0 0 0\nv 1 1 1\nf 1 x\n"}


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return p


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("case", sorted(EDGES_CASES))
def test_edges_file_matches_gviz(ref, tmp_path, case, directed):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".edges", EDGES_CASES[case])
    skip = case == "header"
    want = ref.load_edges_csr(p, directed, skip)
    row, col, ext = graphs.load_edges_file(p, directed, skip)
    assert want is not None
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])
    assert len(ext) == len(row) - 1


def test_edges_file_external_ids(ref, tmp_path):
    """Ids far apart: gviz's loader sizes its id map by max - min + 1 and
    cannot allocate it here; this loader maps only the ids present."""
    from grapher_b200 import graphs
    p = _write(tmp_path, "ids.edges", "1000000 3\n3 77\n77 1000000\n5000000000 3\n")
    row, col, ext = graphs.load_edges_file(p)
    assert ext.tolist() == [1000000, 3, 77, 5000000000]
    assert row.tolist() == [0, 2, 5, 7, 8]
    assert col.tolist() == [1, 2, 0, 2, 3, 1, 0, 1]


@pytest.mark.parametrize("case", sorted(EDGES_BAD))
def test_edges_file_failures_match_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".edges", EDGES_BAD[case])
    assert ref.load_edges_csr(p) is None
    with pytest.raises(OSError):
        graphs.load_edges_file(p)


def test_missing_file(tmp_path):
    from grapher_b200 import graphs
    with pytest.raises(OSError):
        graphs.load_edges_file(tmp_path / "absent.edges")
    with pytest.raises(OSError):
        graphs.load_obj_file(tmp_path / "absent.obj")
    with pytest.raises(OSError):
        graphs.load_gexf_file(tmp_path / "absent.gexf")


@pytest.mark.parametrize("case", sorted(OBJ_CASES))
def test_obj_file_matches_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".obj", OBJ_CASES[case])
    want = ref.load_obj_csr(p)
    row, col = graphs.load_obj_file(p)
    assert want is not None
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])


@pytest.mark.parametrize("case", sorted(OBJ_BAD))
def test_obj_file_failures_match_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".obj", OBJ_BAD[case])
    assert ref.load_obj_csr(p) is None
    with pytest.raises(OSError):
        graphs.load_obj_file(p)


def test_random_edges_file_matches_gviz(ref, tmp_path):
    """A seeded 200k-line file with duplicates, self-loops and scattered ids."""
    from grapher_b200 import graphs
    rng = np.random.default_rng(5)
    ids = rng.choice(10 ** 7, 30000, replace=False) + 1
    u = ids[rng.integers(0, len(ids), 200000)]
    v = ids[rng.integers(0, len(ids), 200000)]
    lines = "\n".join(f"{a} {b}" for a, b in zip(u, v))
    p = _write(tmp_path, "rand.edges", "% random\n" + lines + "\n")
    want = ref.load_edges_csr(p)
    row, col, ext = graphs.load_edges_file(p)
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])
    assert ext[0] == u[0]


GEXF_HEAD = '<?xml version="1.0" encoding="UTF-8"?>\n<gexf version="1.3">\n<graph defaultedgetype="undirected">\n'
GEXF_TAIL = '</graph>\n</gexf>\n'
GEXF_CASES = {
    "path_of_four": GEXF_HEAD + '<nodes>\n<node id="n1"/>\n<node id="n2" />\n<node id="n3"/>\n'
                    '<node id="n4"/>\n</nodes>\n<edges>\n<edge id="e1" source="n1" target="n2"/>\n'
                    '<edge id="e2" source="n3" target="n2"/>\n<edge id="e3" source="n3" target="n4"/>\n'
                    '</edges>\n' + GEXF_TAIL,
    "attribute_tables": GEXF_HEAD + '<attributes class="node">\n'
                        '<attribute id="w" title="weight" type="double"/>\n'
                        '<attribute id="k" title="kind"/>\n</attributes>\n'
                        '<attributes class="edge">\n<attribute title="no id here"/>\n</attributes>\n'
                        "<nodes>\n<node id='p' label='P'>\n<attvalues>\n"
                        '<attvalue for="w" value="2.5"/>\n<attvalue for="k" value="x &amp; y"/>\n'
                        '</attvalues>\n</node>\n<node id="q" label="Q"></node>\n<node id="r"/>\n'
                        '</nodes>\n<edges>\n<edge source="r" target="p" weight="3"/>\n'
                        "<edge source='q' target='p'/>\n</edges>\n" + GEXF_TAIL,
    "legacy_attvalue_id": GEXF_HEAD + '<nodes>\n<node id="0" label="zero">\n<attvalues>'
                          '<attvalue id="1" value="5"/></attvalues>\n</node>\n<node id="1"/>\n'
                          '</nodes>\n<edges><edge source="1" target="0"/></edges>\n' + GEXF_TAIL,
    "duplicates_selfloop_isolated": GEXF_HEAD + '<nodes>\n<node id="a"/>\n<node id="b"/>\n'
                                    '<node id="a" label="second a"/>\n<node id="c"/>\n'
                                    '<node id="lonely"/>\n</nodes>\n<edges>\n'
                                    '<edge source="a" target="b"/>\n<edge source="b" target="a"/>\n'
                                    '<edge source="a" target="b"/>\n<edge source="c" target="c"/>\n'
                                    '<edge source="c" target="a"/>\n</edges>\n' + GEXF_TAIL,
    "attribute_substring": GEXF_HEAD + '<nodes>\n<node pid="x" id="a"/>\n<node id="b"/>\n'
                           '</nodes>\n<edges>\n<edge source="x" target="b"/>\n</edges>\n' + GEXF_TAIL,
    "crlf_tabs_comment": (GEXF_HEAD + '<nodes>\r\n<node\tid="u"\t/>\r\n<!-- <node id="c1"/> -->\r\n'
                          '<node\nid="v"/>\r\n</nodes>\r\n<edges>\r\n<edge\tsource="u"\ttarget="v"/>\r\n'
                          '<edge source="c1" target="u">\r\n</edge>\r\n</edges>\r\n' + GEXF_TAIL),
    "edges_first": GEXF_HEAD + '<edges>\n<edge source="b" target="a"/>\n</edges>\n<nodes>\n'
                   '<node id="a"/>\n<node id="b"/>\n</nodes>\n' + GEXF_TAIL,
}
GEXF_BAD = {
    "no_nodes": GEXF_HEAD + '<nodes>\n</nodes>\n<edges>\n</edges>\n' + GEXF_TAIL,
    "node_without_id": GEXF_HEAD + '<nodes><node label="A"/></nodes>\n' + GEXF_TAIL,
    "unknown_target": GEXF_HEAD + '<nodes><node id="a"/></nodes><edges><edge source="a" '
                      'target="zz"/></edges>\n' + GEXF_TAIL,
    "edge_without_target": GEXF_HEAD + '<nodes><node id="a"/></nodes><edges><edge source="a"/>'
                           '</edges>\n' + GEXF_TAIL,
    "unterminated_node": GEXF_HEAD + '<nodes><node id="a"><attvalues></attvalues>\n' + GEXF_TAIL,
    "attvalue_without_value": GEXF_HEAD + '<nodes><node id="a"><attvalues><attvalue for="0"/>'
                              '</attvalues></node></nodes>\n' + GEXF_TAIL,
    "unterminated_attributes": GEXF_HEAD + '<attributes class="node">\n<nodes><node id="a"/>'
                               '</nodes>\n' + GEXF_TAIL,
    "attribute_without_id": GEXF_HEAD + '<attributes class="node"><attribute title="t"/>'
                            '</attributes><nodes><node id="a"/></nodes>\n' + GEXF_TAIL,
    "id_too_long": GEXF_HEAD + '<nodes><node id="' + "x" * 300 + '"/></nodes>\n' + GEXF_TAIL,
}


@pytest.mark.parametrize("case", sorted(GEXF_CASES))
def test_gexf_file_matches_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".gexf", GEXF_CASES[case])
    want = ref.load_gexf_csr(p)
    row, col = graphs.load_gexf_file(p)
    assert want is not None
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])


@pytest.mark.parametrize("case", sorted(GEXF_BAD))
def test_gexf_file_failures_match_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".gexf", GEXF_BAD[case])
    assert ref.load_gexf_csr(p) is None
    with pytest.raises(OSError):
        graphs.load_gexf_file(p)


def test_random_gexf_file_matches_gviz(ref, tmp_path):
    """A seeded 20,000-node, 60,000-edge file with string ids in shuffled
    order, duplicates and self-loops."""
    from grapher_b200 import graphs
    rng = np.random.default_rng(9)
    names = [f"node-{i:05d}" for i in rng.permutation(20000)]
    u = rng.integers(0, 20000, 60000)
    v = rng.integers(0, 20000, 60000)
    body = "".join(f'<node id="{n}" label="{n.upper()}"/>\n' for n in names)
    edges = "".join(f'<edge id="{i}" source="{names[a]}" target="{names[b]}"/>\n'
                    for i, (a, b) in enumerate(zip(u, v)))
    p = _write(tmp_path, "rand.gexf", GEXF_HEAD + "<nodes>\n" + body + "</nodes>\n<edges>\n"
               + edges + "</edges>\n" + GEXF_TAIL)
    want = ref.load_gexf_csr(p)
    row, col = graphs.load_gexf_file(p)
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])
    assert len(row) == 20001 and len(col) == 120000
