"""Gambit neutral-file meshes: the record formats of ReadNeutralGrid, the
O(N) face connectivity against the literal O(N^2) GlobalConnectivity
restatement (GlobalGridConnectivity.for:4-345), and the solver on meshes
that keep the element-local face order (CPU oracle; GPU against it)."""

import ctypes as C

import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs
from flowsolversourcecode_b200 import neutral as nm

KINDS = ["hex", "wedge", "tet"]
ALL_KINDS = KINDS + ["pyramid", "mixed"]   # 'mixed': bricks and pyramids sharing faces


def _literal():
    import oracle
    return oracle.load().om_neu_connectivity_literal


@pytest.mark.parametrize("kind", ALL_KINDS)
def test_neu_write_read_roundtrip(kind, tmp_path):
    m = nm.neu_box(3, 4, 2, kind, jitter=0.3, seed=2)
    p = str(tmp_path / "m.neu")
    nm.write_neu(p, m)
    r = nm.read_neu(p)
    np.testing.assert_allclose(r.points, m.points, rtol=1e-10, atol=1e-12)
    for k in ("etype", "node_ptr", "nodes", "bc_size", "bc_element", "bc_face"):
        assert np.array_equal(getattr(r, k), getattr(m, k)), k
    assert r.bc_names == m.bc_names
    assert len(r.groups) == 1 and np.array_equal(r.groups[0][2], np.arange(m.n_elements))
    r2 = nm.read_neu(p, scale=(2.0, 1.0, 0.5))   # GridScalex/y/z
    np.testing.assert_allclose(r2.points, m.points * [2.0, 1.0, 0.5], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("kind", ALL_KINDS)
@pytest.mark.parametrize("shuffle", [False, True])
def test_connectivity_matches_literal_global_connectivity(kind, shuffle):
    """Every array -- interior face order, face nodes, owner/neighbour,
    boundary faces, each element's local face list -- equals the O(N^2)
    restatement's, also with the elements in a scrambled order."""
    m = nm.neu_box(4, 3, 3, kind, jitter=0.2, seed=1)
    if shuffle:
        rng = np.random.default_rng(0)
        perm = rng.permutation(m.n_elements)
        inv = np.empty_like(perm)
        inv[perm] = np.arange(perm.size)
        lists = [m.nodes[m.node_ptr[e]:m.node_ptr[e + 1]] for e in perm]
        m.etype = m.etype[perm]
        m.node_ptr = np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.int32)
        m.nodes = np.concatenate(lists).astype(np.int32)
        m.bc_element = inv[m.bc_element].astype(np.int32)
    a = nm.connectivity(m)
    b = nm.connectivity(m, _literal())
    assert a["n_internal"] == b["n_internal"] and a["n_faces"] == b["n_faces"]
    for k in ("face_ptr", "face_nodes", "owner", "neighbour", "cell_face_ptr", "cell_faces"):
        assert np.array_equal(a[k], b[k]), k
    # owner below neighbour, every element face used once
    assert np.all(a["owner"][:a["n_internal"]] < a["neighbour"])
    assert np.array_equal(np.sort(a["cell_faces"]),
                          np.sort(np.concatenate([np.arange(a["n_faces"]), np.arange(a["n_internal"])])))


def test_connectivity_rejects_bad_meshes():
    m = nm.neu_box(2, 2, 2, "hex")
    bad = nm.neu_box(2, 2, 2, "hex")
    bad.etype = bad.etype.copy()
    bad.etype[3] = 9                           # unknown NTypeGeometry
    with pytest.raises(RuntimeError):
        nm.connectivity(bad)
    open_side = nm.neu_box(2, 2, 2, "hex")      # a side without boundary records
    n0 = int(open_side.bc_size[0])
    open_side.bc_size = open_side.bc_size[1:]
    open_side.bc_names = open_side.bc_names[1:]
    open_side.bc_element = open_side.bc_element[n0:]
    open_side.bc_face = open_side.bc_face[n0:]
    with pytest.raises(RuntimeError):
        nm.connectivity(open_side)
    assert nm.connectivity(m)["n_faces"] == 36


def test_neu_hex_cavity_matches_polymesh_cavity():
    """The same box through the neutral-file path (element-local face order)
    and the polyMesh path: same geometry and iterates up to summation order."""
    import oracle
    kw = dict(solver_mom="bicgs", solver_cont="bicgs", krylov_tol=1e-12, krylov_maxit=300)
    pm_box, c = cs.cavity(6, nz=4, **kw)
    pm = nm.to_polymesh(nm.neu_box(6, 6, 4, "hex"))
    a, b = oracle.Oracle(pm, c), oracle.Oracle(pm_box, c)

    def order(o):
        x = np.round(np.stack([o.get("zc"), o.get("yc"), o.get("xc")]), 9)
        return np.lexsort(x)

    ia, ib = order(a), order(b)
    np.testing.assert_allclose(a.get("vol")[ia], b.get("vol")[ib], rtol=1e-13)
    for _ in range(3):
        sa, sb = a.simple_iteration(), b.simple_iteration()
        assert abs(sa - sb) <= 1e-9 * abs(sb)
    for k in ("u", "v", "w", "p"):
        assert np.abs(a.get(k)[ia] - b.get(k)[ib]).max() <= 1e-9 * np.abs(b.get(k)).max(), k


@pytest.mark.parametrize("kind", ["wedge", "tet", "pyramid", "mixed"])
def test_oracle_cavity_on_wedges_and_tetrahedra(kind):
    import oracle
    _, c = cs.cavity(5, nz=3, solver_mom="bicgs", solver_cont="bicgs", krylov_tol=1e-10, krylov_maxit=300)
    o = oracle.Oracle(nm.to_polymesh(nm.neu_box(5, 5, 3, kind, jitter=0.2, seed=3)), c)
    r = [o.simple_iteration() for _ in range(60)]
    assert np.all(np.isfinite(r)) and r[-1] < 1e-3 * r[1]
    # the element volumes fill the unit box
    assert abs(o.get("vol").sum() - 1.0) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_neu_mesh_gpu_matches_oracle(kind):
    """Geometry and the first momentum system bit for bit, four outer
    iterations to 1e-7, on a jittered neutral-file mesh in element-local
    face order."""
    import oracle
    from flowsolversourcecode_b200.solver import Solver
    _, c = cs.cavity(5, nz=4, conv_scheme="sou", niter_start_hr=1, solver_mom="bicgs", solver_cont="bicgs",
                     krylov_tol=1e-10, krylov_maxit=300)
    pm = nm.to_polymesh(nm.neu_box(5, 5, 4, kind, jitter=0.2, seed=4))
    g, o = Solver(pm, c), oracle.Oracle(pm, c)

    def rel(x, y):
        return float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))

    assert rel(g.get("volume"), o.get("vol")) <= 1e-14
    conn = g.connectivity()
    W = g.W
    cf = conn["cf"].reshape(W, -1)
    for i in (0, g.N // 2, g.N - 1):
        lst = pm.cell_faces[pm.cell_face_ptr[i]:pm.cell_face_ptr[i + 1]]
        assert np.array_equal(cf[:len(lst), i], lst)
    rng = np.random.default_rng(0)
    for k in ("u", "v", "w", "p"):
        x = 0.05 * rng.standard_normal(g.N)
        g.set(k, x)
        o.set(k, x)
    g.set_iteration(1)
    o.set_iter(1)
    g.assemble_momentum(0)
    o.assemble_momentum(0)
    for k in ("ac", "bc", "anb"):
        assert rel(g.get(k), o.get(k)) <= 1e-14, k
    g.set_iteration(0)
    o.set_iter(0)
    for _ in range(4):
        g.simple_iteration()
        o.simple_iteration()
    for k in ("u", "v", "w", "p", "mdot"):
        assert rel(g.get(k), o.get(k)) <= 1e-7, k
    g.close()
