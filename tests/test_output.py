"""VTU output: counts, polyhedron face lists and cell data read back (CPU)."""
import xml.etree.ElementTree as ET

import numpy as np

from flowsolversourcecode_b200 import mesh as fm
from flowsolversourcecode_b200.output import write_vtu


def test_vtu_round_trip(tmp_path):
    m = fm.box_mesh(3, 2, 2, jitter=0.1, seed=1)
    n = m.n_cells
    rng = np.random.default_rng(0)
    p = rng.standard_normal(n)
    g = rng.standard_normal(3 * n)
    path = str(tmp_path / "box.vtu")
    write_vtu(path, m, {"p": p, "grad": g})
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfCells")) == n
    assert int(piece.get("NumberOfPoints")) == m.points.reshape(-1, 3).shape[0]
    arrays = {a.get("Name"): np.array(a.text.split(), float) for a in piece.iter("DataArray") if a.get("Name")}
    assert np.array_equal(arrays["offsets"], 8 * np.arange(1, n + 1))          # hexahedra: 8 nodes
    assert np.all(arrays["types"] == 42)
    faces = arrays["faces"].astype(int)
    fo = arrays["faceoffsets"].astype(int)
    start = 0
    for c in range(n):
        assert faces[start] == 6 and fo[c] - start == 1 + 6 * 5   # 6 quads
        start = fo[c]
    assert np.array_equal(arrays["p"], p)
    assert np.array_equal(arrays["grad"].reshape(n, 3), g.reshape(3, n).T)
