"""Lossless checkpoints (gvizCudaForceSaveCheckpoint / LoadCheckpoint):
a run stopped, saved, loaded into a fresh handle of the same graph and
continued matches the uninterrupted run bit for bit, in both precisions
and for batches; damaged or foreign files are refused. The text export
keeps every bit through gviz's own gvizEmbeddedGraphLoadEmbedding."""
import numpy as np
import pytest

from helpers import cfg, make_layout

pytestmark = pytest.mark.gpu


def _graph():
    from grapher_b200 import graphs
    a, b = graphs.barabasi_albert(3000, 3, 5)
    row, col = graphs.to_csr(3000, a, b)
    return 3000, row, col


def _state(lay):
    sf, sp, ef = lay.fa2_state()
    return lay.positions(), sf, sp, ef, lay.stat_history()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_resume_is_bit_exact(tmp_path, prec):
    from grapher_b200 import graphs
    V, row, col = _graph()
    c = cfg(model=1, theta=0.8, gravity=1.0, precision=prec)
    a = make_layout(row, col, c)
    a.begin(0, positions=graphs.randomize_positions(V, 100.0, 3))
    for _ in range(7):
        a.step()
    path = tmp_path / "run.gvzckpt"
    a.save_checkpoint(path, name="ba3000")
    for _ in range(6):
        a.step()
    b = make_layout(row, col, cfg(model=1))  # configuration comes from the file
    assert b.load_checkpoint(path, restore_params=True) == "ba3000"
    for _ in range(6):
        b.step()
    for x, y in zip(_state(a), _state(b)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.stat_history()[:7], b.stat_history()[:7])
    assert b.stat_history().shape == (13, 5)


def test_batch_resume_is_bit_exact(tmp_path):
    from grapher_b200 import graphs
    gs = []
    for i, V in enumerate([200, 57, 1000]):
        a, b = graphs.random_connected(V, 0.01, 40 + i)
        gs.append((V, a, b))
    row, col, offs = graphs.batch(gs)
    x0 = np.concatenate([graphs.randomize_positions(V, 30.0, 9 + i) for i, (V, _, _) in enumerate(gs)])
    c = cfg(model=0, theta=0.7)
    a = make_layout(row, col, c, graph_offsets=offs)
    a.begin(0, positions=x0)
    a.run(5, 1e-12)
    path = tmp_path / "batch.gvzckpt"
    a.save_checkpoint(path)
    a.run(9, 1e-12)
    b = make_layout(row, col, c, graph_offsets=offs)
    b.load_checkpoint(path)
    b.run(9, 1e-12)
    assert np.array_equal(a.positions(), b.positions())
    for g in range(3):
        assert np.array_equal(a.stat_history(g), b.stat_history(g))


def test_refuses_damaged_and_foreign_files(tmp_path):
    from grapher_b200 import graphs
    from grapher_b200._native import GvizCudaError
    V, row, col = _graph()
    a = make_layout(row, col, cfg(model=1))
    a.begin(0, positions=graphs.randomize_positions(V, 100.0, 3))
    a.step()
    path = tmp_path / "a.gvzckpt"
    a.save_checkpoint(path)
    raw = bytearray(path.read_bytes())
    x_before = a.positions()
    # one flipped bit in the positions
    bad = tmp_path / "bad.gvzckpt"
    raw2 = bytearray(raw)
    raw2[200] ^= 0x10
    bad.write_bytes(bytes(raw2))
    with pytest.raises(GvizCudaError):
        a.load_checkpoint(bad)
    # truncated, and one byte too many
    (tmp_path / "short.gvzckpt").write_bytes(bytes(raw[:-9]))
    (tmp_path / "long.gvzckpt").write_bytes(bytes(raw) + b"\0")
    for name in ("short.gvzckpt", "long.gvzckpt", "absent.gvzckpt"):
        with pytest.raises(GvizCudaError):
            a.load_checkpoint(tmp_path / name)
    # another graph
    a2, b2 = graphs.grid(20, 20)
    r2, c2 = graphs.to_csr(400, a2, b2)
    other = make_layout(r2, c2, cfg(model=1))
    with pytest.raises(GvizCudaError):
        other.load_checkpoint(path)
    assert np.array_equal(a.positions(), x_before)


def test_text_export_round_trips_through_gviz(ref, tmp_path):
    """gviz's loader reads the 17-digit export back bit for bit; gviz's own
    six-decimal save does not."""
    from grapher_b200 import graphs
    a, b = graphs.random_connected(500, 0.02, 8)
    row, col = graphs.to_csr(500, a, b)
    lay = make_layout(row, col, cfg(model=0, theta=0.7))
    lay.begin(0, positions=graphs.randomize_positions(500, 50.0, 4))
    for _ in range(4):
        lay.step()
    path = tmp_path / "emb.txt"
    lay.save_embedding_text(path, name="g500")
    r = ref.create_edges(500, a, b, 0)
    assert r.load_embedding(path) == 0
    assert np.array_equal(r.positions(), lay.positions())
    lossy = tmp_path / "lossy.txt"
    assert r.save_embedding(lossy) == 0
    r2 = ref.create_edges(500, a, b, 0)
    assert r2.load_embedding(lossy) == 0
    assert not np.array_equal(r2.positions(), lay.positions())
    r.close()
    r2.close()
