"""Host-side mirror of the reference interface: configuration semantics and result types."""
import numpy as np

import graphzeppelin_b200 as gz


def test_cc_alg_configuration_defaults_and_bounds(capsys):
    c = gz.CCAlgConfiguration()
    assert c.get_sketches_factor() == 1 and c.get_batch_factor() == 1
    c.sketches_factor(0).batch_factor(-2)
    assert c.get_sketches_factor() == 1 and c.get_batch_factor() == 1
    assert "out of bounds" in capsys.readouterr().out
    c.sketches_factor(1.5)
    assert "Num sketches factor   = 1.5" in str(c)


def test_driver_configuration():
    d = gz.DriverConfiguration().gutter_sys(gz.CACHETREE).worker_threads(0)
    assert d.get_worker_threads() == 1
    assert d.get_gutter_sys() == gz.CACHETREE


def test_connected_components_helpers():
    parent = np.array([3, 3, 5, 3, 9, 5, 9, 9, 8, 9], np.uint32)
    cc = gz.ConnectedComponents(parent, 4)
    assert cc.size() == 4
    sets = cc.get_component_sets()
    assert sets == [{0, 1, 3}, {2, 5}, {8}, {4, 6, 7, 9}]
    assert cc.is_connected(0, 3) and not cc.is_connected(0, 2)
    assert cc.canonical_labels().tolist() == [0, 0, 2, 0, 4, 2, 4, 4, 8, 4]


def test_graph_update_and_pairing():
    u = gz.GraphUpdate((5, 2), gz.UpdateType.DELETE)
    assert u.edge.src == 5 and u.type == 1
    assert gz.concat_pairing_fn(5, 2) == (2 << 32) | 5
    assert gz.inv_concat_pairing_fn((2 << 32) | 5) == (2, 5)


def test_binary_file_stream_breakpoints(tmp_path):
    from graphzeppelin_b200 import streams as S
    st = S.erdos_renyi_stream(50, 0.2, seed=1)
    p = str(tmp_path / "s.bin")
    st.write(p)
    bfs = gz.BinaryFileStream(p)
    assert bfs.vertices() == 50 and bfs.edges() == st.num_updates
    assert bfs.set_break_point(10)
    a = bfs.take_until_break()
    assert a.size == 10
    assert not bfs.set_break_point(5)
    assert bfs.set_break_point(gz.END_OF_STREAM)
    assert bfs.take_until_break().size == st.num_updates - 10
