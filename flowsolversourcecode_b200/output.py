"""Headless solution output: VTK XML unstructured grid (.vtu) and Tecplot
ASCII (.dat).

The reference writes its fields for post-processing as Tecplot and VTU files
(ReadFoamMesh.f90:865 VTU writer; PrintingTecplotFile.for:4).  `write_vtu`
takes the polyMesh the solver was built from and cell-centred fields (the
arrays `Solver.get` returns) and writes every cell as a VTK_POLYHEDRON (type
42) with its faces, so any polyMesh cell shape is written without
special-casing hexahedra.  `write_tecplot` writes the Tecplot FEBLOCK zones of
a Gambit neutral-file mesh with node values interpolated from the cells and
boundary faces as the reference does.  ASCII, one file, no external libraries.
"""
from __future__ import annotations

import numpy as np

from .mesh import PolyMesh

VTK_POLYHEDRON = 42


def _cells_faces(mesh: PolyMesh):
    """Per cell: the list of its faces (global face ids) in face order."""
    n = mesh.n_cells
    own = np.asarray(mesh.owner, np.int64)
    nbr = np.asarray(mesh.neighbour, np.int64)
    nf = mesh.n_faces
    cell_of = np.concatenate([own, nbr])
    face_of = np.concatenate([np.arange(nf), np.arange(mesh.n_internal)])
    order = np.lexsort((face_of, cell_of))
    cell_of, face_of = cell_of[order], face_of[order]
    ptr = np.searchsorted(cell_of, np.arange(n + 1))
    return ptr, face_of


def write_vtu(path: str, mesh: PolyMesh, cell_data: dict | None = None) -> None:
    """Write `mesh` with the given cell fields (name -> array of n_cells, or
    of 3*n_cells in x, y, z blocks for a vector) to `path`."""
    cell_data = cell_data or {}
    n = mesh.n_cells
    pts = np.asarray(mesh.points, np.float64).reshape(-1, 3)
    fptr = np.asarray(mesh.face_ptr, np.int64)
    fnodes = np.asarray(mesh.face_nodes, np.int64)
    cptr, cfaces = _cells_faces(mesh)
    conn, offsets, faces, faceoffsets = [], [], [], []
    c_off = f_off = 0
    for c in range(n):
        fl = cfaces[cptr[c]:cptr[c + 1]]
        nodes = np.unique(np.concatenate([fnodes[fptr[f]:fptr[f + 1]] for f in fl]))
        conn.append(nodes)
        c_off += nodes.size
        offsets.append(c_off)
        rec = [len(fl)]
        for f in fl:
            fn = fnodes[fptr[f]:fptr[f + 1]]
            if f < mesh.n_internal and mesh.neighbour[f] == c:
                fn = fn[::-1]   # polyMesh faces point out of their owner: outward for every cell
            rec.append(fn.size)
            rec.extend(fn.tolist())
        faces.append(np.asarray(rec, np.int64))
        f_off += len(rec)
        faceoffsets.append(f_off)

    def arr(a, fmt):
        return " ".join(fmt % x for x in np.ravel(a))

    with open(path, "w") as out:
        out.write('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian">\n')
        out.write(f'<UnstructuredGrid>\n<Piece NumberOfPoints="{pts.shape[0]}" NumberOfCells="{n}">\n')
        out.write('<Points>\n<DataArray type="Float64" NumberOfComponents="3" format="ascii">\n')
        out.write(arr(pts, "%.17g") + "\n</DataArray>\n</Points>\n<Cells>\n")
        out.write('<DataArray type="Int64" Name="connectivity" format="ascii">\n' + arr(np.concatenate(conn), "%d") + "\n</DataArray>\n")
        out.write('<DataArray type="Int64" Name="offsets" format="ascii">\n' + arr(offsets, "%d") + "\n</DataArray>\n")
        out.write('<DataArray type="UInt8" Name="types" format="ascii">\n' + arr(np.full(n, VTK_POLYHEDRON), "%d") + "\n</DataArray>\n")
        out.write('<DataArray type="Int64" Name="faces" format="ascii">\n' + arr(np.concatenate(faces), "%d") + "\n</DataArray>\n")
        out.write('<DataArray type="Int64" Name="faceoffsets" format="ascii">\n' + arr(faceoffsets, "%d") + "\n</DataArray>\n")
        out.write("</Cells>\n<CellData>\n")
        for name, a in cell_data.items():
            a = np.asarray(a, np.float64)
            if a.size == 3 * n:
                v = a.reshape(3, n).T
                out.write(f'<DataArray type="Float64" Name="{name}" NumberOfComponents="3" format="ascii">\n')
                out.write(arr(v, "%.17g") + "\n</DataArray>\n")
            elif a.size == n:
                out.write(f'<DataArray type="Float64" Name="{name}" format="ascii">\n' + arr(a, "%.17g") + "\n</DataArray>\n")
            else:
                raise ValueError(f"{name}: {a.size} values for {n} cells")
        out.write("</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")


# ------------------------------------------------------------------ Tecplot
def _face_centroids(mesh: PolyMesh, faces) -> np.ndarray:
    """Face centroids of ProcessGeometry (ProcessGeometryRoutine.for): the
    area-weighted centroids of the triangles that fan out from the mean of
    the face's nodes."""
    pts = np.asarray(mesh.points, np.float64).reshape(-1, 3)
    out = np.zeros((len(faces), 3))
    for q, f in enumerate(faces):
        p = pts[mesh.face_nodes[mesh.face_ptr[f]:mesh.face_ptr[f + 1]]]
        c = p.sum(axis=0) / p.shape[0]
        a_sum, cx = 0.0, np.zeros(3)
        for k in range(p.shape[0]):
            p2, p3 = p[k], p[(k + 1) % p.shape[0]]
            s = 0.5 * np.cross(p2 - c, p3 - c)
            a = np.sqrt(s @ s)
            a_sum = a_sum + a
            cx = cx + (c + p2 + p3) / 3.0 * a
        out[q] = cx / a_sum
    return out


def node_values(neu, mesh: PolyMesh, cell: np.ndarray, bface: np.ndarray, xc: np.ndarray,
                bfc: np.ndarray | None = None) -> np.ndarray:
    """InterpolateFromElementsToNodes (InterpolateFromElementsToNodeForPlotting.for:815-900):
    a node on no boundary face takes the inverse-distance mean of the values
    of the elements that hold it (distances to their centroids); a node on a
    boundary face takes the inverse-distance mean of the values of the
    boundary faces that hold it.  Sums run in the reference's loop order."""
    n_nodes = np.asarray(mesh.points).reshape(-1, 3).shape[0]
    pts = np.asarray(mesh.points, np.float64).reshape(-1, 3)
    N = neu.n_elements
    xc = np.asarray(xc, np.float64).reshape(3, N).T
    bfaces = np.arange(mesh.n_internal, mesh.n_faces)
    if bfc is None:
        bfc = _face_centroids(mesh, bfaces)
    on_bnd = np.zeros(n_nodes, bool)
    for f in bfaces:
        on_bnd[mesh.face_nodes[mesh.face_ptr[f]:mesh.face_ptr[f + 1]]] = True
    s_inv = np.zeros(n_nodes)
    s_phi = np.zeros(n_nodes)
    el = np.repeat(np.arange(N), np.diff(neu.node_ptr))
    nd = np.asarray(neu.nodes, np.int64)
    m = ~on_bnd[nd]
    d = np.sqrt(((xc[el[m]] - pts[nd[m]]) ** 2).sum(axis=1))
    np.add.at(s_inv, nd[m], 1.0 / d)
    np.add.at(s_phi, nd[m], cell[el[m]] / d)
    bl, bn = [], []
    for q, f in enumerate(bfaces):
        fn = mesh.face_nodes[mesh.face_ptr[f]:mesh.face_ptr[f + 1]]
        bl.extend([q] * len(fn))
        bn.extend(fn.tolist())
    bl, bn = np.asarray(bl, np.int64), np.asarray(bn, np.int64)
    d = np.sqrt(((bfc[bl] - pts[bn]) ** 2).sum(axis=1))
    np.add.at(s_inv, bn, 1.0 / d)
    np.add.at(s_phi, bn, bface[bl] / d)
    out = np.zeros(n_nodes)
    used = s_inv > 0.0
    out[used] = s_phi[used] / s_inv[used]
    return out


# Tecplot node orders of Gambit elements (PrintingTecplotFile.for:1657-1690)
_TEC_BRICK = (4, 5, 1, 0, 6, 7, 3, 2)
_TEC_TETRA = (3, 0, 2, 1)


def write_tecplot(path: str, neu, mesh: PolyMesh, fields: dict, xc: np.ndarray, mu: float,
                  turbulence: bool = False) -> None:
    """Tecplot (PrintingTecplotFile.for:4-1706) for a neutral-file mesh
    (`neutral.read_neu` / `neu_box`, solved on `neutral.to_polymesh` of it):
    one FEBLOCK zone per element group, x y z and then the node values of
    u, v, w, the velocity magnitude, the pressure and the laminar viscosity,
    and with k-epsilon k, epsilon, the turbulent and effective viscosities,
    their ratio and the turbulence intensity -- the variables the reference
    writes for this configuration, in its order.  `fields` holds the cell and
    boundary arrays of `Solver.get` (u v w p bu bv bw bp; tke ted mut btke
    bted bmut with k-epsilon).  Groups whose elements are all bricks or all
    tetrahedra are written as BRICK / TETRAHEDRON zones; other element types
    are not written by the reference either."""
    N = neu.n_elements
    B = mesh.n_faces - mesh.n_internal
    u, v, w, p = (np.asarray(fields[k], np.float64) for k in ("u", "v", "w", "p"))
    bu, bv, bw, bp = (np.asarray(fields[k], np.float64) for k in ("bu", "bv", "bw", "bp"))
    var = [("u-Velocity (m/s)", u, bu), ("v-Velocity (m/s)", v, bv), ("w-Velocity (m/s)", w, bw),
           ("Velocity-Magnitude (m/s)", np.sqrt(u ** 2 + v ** 2 + w ** 2), np.sqrt(bu ** 2 + bv ** 2 + bw ** 2)),
           ("Pressure (Pa)", p, bp)]
    if turbulence:
        k, e, mt = (np.asarray(fields[q], np.float64) for q in ("tke", "ted", "mut"))
        bk, be, bmt = (np.asarray(fields[q], np.float64) for q in ("btke", "bted", "bmut"))
        two3 = float(np.float32(2.0 / 3.0))
        vm, bvm = var[3][1], var[3][2]
        var += [("Turbulent kinetic energy (m2/s2)", k, bk), ("Turbulent dissipation rate (m2/s3)", e, be),
                ("Laminar viscosity (Pa.s)", np.full(N, mu), np.full(B, mu)),
                ("Turbulent viscosity (Pa.s)", mt, bmt),
                ("Effective viscosity (Pa.s)", mu + mt, mu + bmt),
                ("Turbulent viscosity ratio", mt / mu, bmt / mu),
                ("Turbulent intensity (%)", 100.0 * np.sqrt(two3 * k) / np.maximum(vm, 1e-15),
                 100.0 * np.sqrt(two3 * bk) / np.maximum(bvm, 1e-15))]
    else:
        var.append(("Laminar viscosity (Pa.s)", np.full(N, mu), np.full(B, mu)))
    bfc = _face_centroids(mesh, np.arange(mesh.n_internal, mesh.n_faces))
    nodal = [node_values(neu, mesh, c, b, xc, bfc) for _, c, b in var]
    pts = np.asarray(mesh.points, np.float64).reshape(-1, 3)
    groups = neu.groups or [("all", 0, np.arange(N))]
    with open(path, "w") as out:
        out.write(' Title = "Example" \n')
        out.write(' Variables= "x (m)", "y (m)", "z (m)" ' + "".join(f',"{n}"' for n, _, _ in var) + "\n")
        for _, _, elems in groups:
            elems = np.asarray(elems, np.int64)
            types = {int(neu.etype[e]) for e in elems}
            if types == {4}:
                et, order = "BRICK", _TEC_BRICK
            elif types == {6}:
                et, order = "TETRAHEDRON", _TEC_TETRA
            else:
                continue
            local, nodes = {}, []
            for e in elems:   # nodes in order of first appearance (ComputeNumberOfNodesInGroups.for:20-50)
                for nd in neu.nodes[neu.node_ptr[e]:neu.node_ptr[e + 1]]:
                    if int(nd) not in local:
                        local[int(nd)] = len(nodes) + 1
                        nodes.append(int(nd))
            nodes = np.asarray(nodes, np.int64)
            out.write(f" Zone N= {len(nodes)}  ,E= {len(elems)} ,F=FEBLOCK,  ET={et}\n")
            for a in (pts[nodes, 0], pts[nodes, 1], pts[nodes, 2]) + tuple(nv[nodes] for nv in nodal):
                out.write("\n".join("%.17g" % x for x in a) + "\n")
            for e in elems:
                en = neu.nodes[neu.node_ptr[e]:neu.node_ptr[e + 1]]
                out.write(" ".join(str(local[int(en[q])]) for q in order) + "\n")
