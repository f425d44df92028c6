"""Mesh generator and polyMesh I/O (CPU)."""
import numpy as np

from flowsolversourcecode_b200.mesh import box_mesh, read_polymesh, splitmix64, uniform01, write_polymesh


def test_box_counts():
    m = box_mesh(4, 3, 2)
    assert m.n_cells == 24
    # interior faces: (nx-1)ny nz + nx(ny-1)nz + nx ny(nz-1)
    assert m.n_internal == 3 * 3 * 2 + 4 * 2 * 2 + 4 * 3 * 1
    assert m.n_faces - m.n_internal == 2 * (3 * 2 + 4 * 2 + 4 * 3)
    assert list(m.patch_size) == [6, 6, 8, 8, 12, 12]
    assert int(m.patch_start[0]) == m.n_internal


def test_upper_triangular_order():
    m = box_mesh(5, 4, 3)
    own, nb = m.owner[:m.n_internal], m.neighbour
    assert np.all(own < nb)
    key = own.astype(np.int64) * m.n_cells + nb
    assert np.all(np.diff(key) > 0)


def test_2d_has_no_z_interior_faces():
    m = box_mesh(8, 8, 1)
    assert m.n_internal == 7 * 8 * 2


def test_splitmix_reference_values():
    # splitmix64 from state 0: published first outputs (Vigna's reference implementation)
    z = splitmix64(0, 3)
    assert int(z[0]) == 0xE220A8397B1DCDAF
    assert int(z[1]) == 0x6E789E6AA1B965F4
    assert int(z[2]) == 0x06C45D188009454F
    u = uniform01(7, 1000)
    assert u.min() >= 0.0 and u.max() < 1.0


def test_jitter_keeps_boundary_nodes():
    a = box_mesh(6, 6, 6)
    b = box_mesh(6, 6, 6, jitter=0.2, seed=0)
    d = np.abs(a.points - b.points)
    h = 1.0 / 6
    assert d.max() <= 0.2 * h + 1e-15
    on_bnd = np.any((a.points == 0.0) | (a.points == 1.0), axis=1)
    assert np.all(d[on_bnd] == 0.0)
    assert np.count_nonzero(d[~on_bnd]) > 0


def test_polymesh_roundtrip(tmp_path):
    m = box_mesh(3, 2, 2, jitter=0.1, seed=3)
    write_polymesh(m, str(tmp_path))
    r = read_polymesh(str(tmp_path))
    assert np.array_equal(r.points, m.points)
    assert np.array_equal(r.face_ptr, m.face_ptr)
    assert np.array_equal(r.face_nodes, m.face_nodes)
    assert np.array_equal(r.owner, m.owner)
    assert np.array_equal(r.neighbour, m.neighbour)
    assert r.patch_names == m.patch_names
    assert np.array_equal(r.patch_start, m.patch_start)
