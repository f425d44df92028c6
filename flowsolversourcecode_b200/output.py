"""Headless solution output: VTK XML unstructured grid (.vtu).

The reference writes its fields for post-processing as Tecplot and VTU files
(ReadFoamMesh.f90:865 VTU writer; PrintingTecplotFile.for:4).  This writer
takes the polyMesh the solver was built from and cell-centred fields (the
arrays `Solver.get` returns) and writes every cell as a VTK_POLYHEDRON (type
42) with its faces, so any polyMesh cell shape is written without
special-casing hexahedra.  ASCII, one file, no external libraries.
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
