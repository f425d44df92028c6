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


def test_tecplot_neutral_box(tmp_path):
    """Tecplot FEBLOCK output of a Gambit brick box: the zone, node blocks in
    first-appearance order, node values by the reference's inverse-distance
    interpolation (a constant stays constant, a linear field is exact at
    interior nodes of a uniform box) and the brick node order."""
    import oracle
    from flowsolversourcecode_b200 import case as cs
    from flowsolversourcecode_b200 import neutral
    from flowsolversourcecode_b200.output import _face_centroids, write_tecplot
    neu = neutral.neu_box(3, 3, 3, "hex")
    pm = neutral.to_polymesh(neu)
    _, case = cs.cavity(3)
    case.patches = {n: ("wall", (0.0, 0.0, 0.0)) for n in pm.patch_names}
    o = oracle.Oracle(pm, case)
    N = o.N
    xc = np.concatenate([o.get("xc"), o.get("yc"), o.get("zc")])
    bfc = _face_centroids(pm, np.arange(pm.n_internal, pm.n_faces))
    lin = lambda x, y, z: x + 2.0 * y + 3.0 * z
    f = {"u": lin(*xc.reshape(3, N)), "bu": lin(*bfc.T), "p": np.full(N, 5.0), "bp": np.full(bfc.shape[0], 5.0)}
    for k in ("v", "w"):
        f[k] = np.zeros(N)
        f["b" + k] = np.zeros(bfc.shape[0])
    path = str(tmp_path / "box.dat")
    write_tecplot(path, neu, pm, f, xc, mu=0.01)
    lines = open(path).read().splitlines()
    assert "Title" in lines[0] and lines[1].count('"') == 2 * 9
    assert lines[2].split() == ["Zone", "N=", "64", ",E=", "27", ",F=FEBLOCK,", "ET=BRICK"]
    vals = np.array([float(x) for x in lines[3:3 + 64 * 9]]).reshape(9, 64)
    conn = np.array([[int(t) for t in l.split()] for l in lines[3 + 64 * 9:]])
    assert conn.shape == (27, 8) and conn.min() == 1 and conn.max() == 64
    pts = np.asarray(pm.points).reshape(-1, 3)
    first = []
    for e in range(neu.n_elements):
        for nd in neu.nodes[neu.node_ptr[e]:neu.node_ptr[e + 1]]:
            if nd not in first:
                first.append(int(nd))
    assert np.array_equal(vals[0], pts[first, 0]) and np.array_equal(vals[2], pts[first, 2])
    np.testing.assert_allclose(vals[7], 5.0, rtol=1e-14)                 # pressure
    interior = np.array([all(0.0 < c < 1.0 for c in pts[n]) for n in first])
    np.testing.assert_allclose(vals[3][interior], lin(*pts[first].T)[interior], rtol=1e-12)
    e0 = neu.nodes[neu.node_ptr[0]:neu.node_ptr[1]]
    assert [first[q - 1] for q in conn[0]] == [int(e0[q]) for q in (4, 5, 1, 0, 6, 7, 3, 2)]
