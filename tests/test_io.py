"""CPU: the reference's mesher file formats (testcases/IMR26/README.md:137-145,
uniform2D.cpp / uniform3D.cpp :183-201): .bin point clouds and the
elems.txt / nodes.txt dumps, round trips and exact text layout."""
import numpy as np
import pytest

from stream_b200 import io as sio


@pytest.mark.parametrize("dim", [2, 3])
def test_point_cloud_round_trip(tmp_path, dim):
    rng = np.random.default_rng(dim)
    c = rng.random((257, dim)).astype(np.float32)
    a = rng.random(257).astype(np.float32)
    p = tmp_path / "cloud.bin"
    sio.write_point_cloud(p, c, a)
    assert p.stat().st_size == 257 * (dim + 1) * 4
    raw = np.fromfile(p, dtype=np.float32).reshape(-1, dim + 1)  # the reference's reader
    assert np.array_equal(raw[:, :dim], c) and np.array_equal(raw[:, dim], a)
    c2, a2 = sio.read_point_cloud(p, dim)
    assert np.array_equal(c2, c) and np.array_equal(a2, a)


def test_point_cloud_rejects_ragged(tmp_path):
    p = tmp_path / "bad.bin"
    np.arange(7, dtype=np.float32).tofile(p)
    with pytest.raises(ValueError):
        sio.read_point_cloud(p, 2)


def test_dump_text_layout(tmp_path):
    elems = np.array([[0, 5, 9], [4294967295, 1, 2]], np.uint32)
    nodes = np.array([[0.123456, 1.0], [-2.5, 3.000004]], np.float32)
    sio.write_elems_txt(tmp_path / "elems.txt", elems)
    sio.write_nodes_txt(tmp_path / "nodes.txt", nodes)
    assert (tmp_path / "elems.txt").read_text() == "0 5 9\n4294967295 1 2\n"
    want = "".join("%.5f %.5f\n" % (float(x), float(y)) for x, y in nodes)  # printf("%.5f") of the promoted float
    assert (tmp_path / "nodes.txt").read_text() == want
    assert np.array_equal(sio.read_elems_txt(tmp_path / "elems.txt", 2), elems)
    assert np.allclose(sio.read_nodes_txt(tmp_path / "nodes.txt", 2), nodes, atol=5e-6)


def test_tets_dump(tmp_path):
    e = np.array([[1, 2, 3, 4]], np.uint32)
    sio.write_elems_txt(tmp_path / "e.txt", e)
    assert (tmp_path / "e.txt").read_text() == "1 2 3 4\n"
    assert np.array_equal(sio.read_elems_txt(tmp_path / "e.txt", 3), e)
