"""Gambit neutral (.neu) meshes: reader, writer, box generators and the
conversion to the solver's mesh form.

The reference reads a neutral file with ReadNeutralGrid
(GridAndGeometry/ReadGridFromNeutralFile.for) and builds its face list with
GlobalConnectivity (GridAndGeometry/GlobalGridConnectivity.for:4-523), an
O(N^2) search.  `to_polymesh` calls the library's O(N) `fs_neu_connectivity`,
which returns the same faces in the same order, and keeps each element's
faces in its local face order and its nodes in file order (the order of the
reference's per-cell sums), so the solver reproduces the reference's
neutral-file path rather than its polyMesh path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .mesh import BOX_PATCHES, PolyMesh, uniform01

NODES_PER_TYPE = {4: 8, 5: 6, 6: 4, 7: 5}   # brick, wedge, tetrahedron, pyramid
FACES_PER_TYPE = {4: 6, 5: 5, 6: 4, 7: 5}
# GlobalConnectivity's element-local faces, 0-based element node positions
# (GlobalGridConnectivity.for:21-120)
LOCAL_FACES = {
    4: ((0, 1, 5, 4), (1, 3, 7, 5), (3, 2, 6, 7), (2, 0, 4, 6), (1, 0, 2, 3), (4, 5, 7, 6)),
    5: ((0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5), (0, 2, 1), (3, 4, 5)),
    6: ((1, 0, 2), (0, 1, 3), (1, 2, 3), (2, 0, 3)),
    7: ((0, 2, 3, 1), (0, 1, 4), (1, 3, 4), (3, 2, 4), (2, 0, 4)),
}


@dataclass
class NeuMesh:
    points: np.ndarray                     # (n_nodes, 3)
    etype: np.ndarray                      # (n_elements,) NTypeGeometry
    node_ptr: np.ndarray                   # (n_elements+1,)
    nodes: np.ndarray                      # 0-based element nodes in file order
    bc_names: list = field(default_factory=list)
    bc_size: np.ndarray = None             # records per set
    bc_element: np.ndarray = None          # 0-based, sets concatenated
    bc_face: np.ndarray = None             # 0-based element-local face
    groups: list = field(default_factory=list)   # (name, material, 0-based elements)
    title: str = "FlowSolver mesh"

    @property
    def n_elements(self) -> int:
        return int(self.etype.shape[0])


# ----------------------------------------------------------------- reading
def read_neu(path: str, scale=(1.0, 1.0, 1.0)) -> NeuMesh:
    """ReadNeutralGrid (ReadGridFromNeutralFile.for): the header counts, nodal
    coordinates (x GridScalex/y/z), elements, element groups and the
    element-face boundary records (NBCDataType 1; node records are skipped,
    GlobalConnectivity does not use them)."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = 0

    def nxt():
        nonlocal pos
        s = lines[pos]
        pos += 1
        return s

    def section(name):
        nonlocal pos
        while name not in lines[pos].upper():
            pos += 1
        pos += 1

    section("NUMNP")
    nn, ne, ng, nb = (int(x) for x in nxt().split()[:4])
    section("NODAL COORDINATES")
    pts = np.zeros((nn, 3))
    for _ in range(nn):
        t = nxt().split()
        pts[int(t[0]) - 1] = [float(t[1]), float(t[2]), float(t[3])]
    pts *= np.asarray(scale, np.float64)
    section("ELEMENTS/CELLS")
    etype = np.zeros(ne, np.int32)
    elem_nodes = [None] * ne
    for _ in range(ne):
        s = nxt()
        e, ty, k = int(s[0:8]), int(s[9:11]), int(s[12:14])
        vals = []
        rest = s[15:]
        while True:
            vals += [int(rest[q:q + 8]) for q in range(0, len(rest.rstrip()), 8)]
            if len(vals) >= k:
                break
            rest = nxt()[15:]
        etype[e - 1] = ty
        elem_nodes[e - 1] = [v - 1 for v in vals[:k]]
    groups = []
    for _ in range(ng):
        section("ELEMENT GROUP")
        h = nxt()
        t = h.replace(":", " ").split()
        count, material, nflags = int(t[3]), int(t[5]), int(t[7])
        name = nxt().strip()
        got = 0
        while got < nflags:
            got += len(nxt().split())
        els = []
        while len(els) < count:
            els += [int(x) - 1 for x in nxt().split()]
        groups.append((name, material, np.asarray(els, np.int32)))
    names, sizes, be, bf = [], [], [], []
    for _ in range(nb):
        section("BOUNDARY CONDITIONS")
        h = nxt()
        name, t = h[:32].strip(), h[32:].split()
        dtype, nrec = int(t[0]), int(t[1])
        if dtype == 1:
            names.append(name)
            sizes.append(nrec)
            for _ in range(nrec):
                r = nxt().split()
                be.append(int(r[0]) - 1)
                bf.append(int(r[2]) - 1)
        else:
            pos += nrec
    ptr = np.zeros(ne + 1, np.int32)
    ptr[1:] = np.cumsum([len(x) for x in elem_nodes])
    return NeuMesh(pts, etype, ptr, np.concatenate(elem_nodes).astype(np.int32), names,
                   np.asarray(sizes, np.int32), np.asarray(be, np.int32), np.asarray(bf, np.int32), groups)


# ----------------------------------------------------------------- writing
def write_neu(path: str, m: NeuMesh) -> None:
    """A neutral file in the record formats ReadNeutralGrid reads."""
    ne, nn = m.n_elements, m.points.shape[0]
    groups = m.groups or [("fluid", 2, np.arange(ne, dtype=np.int32))]
    out = ["        CONTROL INFO 2.4.6", "** GAMBIT NEUTRAL FILE", m.title,
           "PROGRAM:                Gambit     VERSION:  2.4.6", "",
           "     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL",
           "%10d%10d%10d%10d%10d%10d" % (nn, ne, len(groups), len(m.bc_names), 3, 3),
           "ENDOFSECTION", "   NODAL COORDINATES 2.4.6"]
    out += ["%10d%20.11e%20.11e%20.11e" % (i + 1, *m.points[i]) for i in range(nn)]
    out += ["ENDOFSECTION", "      ELEMENTS/CELLS 2.4.6"]
    for e in range(ne):
        nd = [int(x) + 1 for x in m.nodes[m.node_ptr[e]:m.node_ptr[e + 1]]]
        s = "%8d %2d %2d " % (e + 1, m.etype[e], len(nd)) + "".join("%8d" % x for x in nd[:7])
        out.append(s)
        for q in range(7, len(nd), 7):
            out.append(" " * 15 + "".join("%8d" % x for x in nd[q:q + 7]))
    out.append("ENDOFSECTION")
    for g, (name, material, els) in enumerate(groups):
        out += ["       ELEMENT GROUP 2.4.6",
                "GROUP:%11d ELEMENTS:%11d MATERIAL:%11d NFLAGS:%11d" % (g + 1, len(els), material, 1),
                "%32s" % name, "%8d" % 0]
        for q in range(0, len(els), 10):
            out.append("".join("%8d" % (x + 1) for x in els[q:q + 10]))
        out.append("ENDOFSECTION")
    r = 0
    for name, n in zip(m.bc_names, m.bc_size):
        out += [" BOUNDARY CONDITIONS 2.4.6", "%32s%8d%8d%8d%8d" % (name, 1, n, 0, 6)]
        for q in range(r, r + n):
            e = int(m.bc_element[q])
            out.append("%10d%5d%5d" % (e + 1, m.etype[e], m.bc_face[q] + 1))
        r += n
        out.append("ENDOFSECTION")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


# ----------------------------------------------------------------- generators
def neu_box(nx: int, ny: int, nz: int, kind: str = "hex", lx: float = 1.0, ly: float = 1.0, lz: float = 1.0,
            jitter: float = 0.0, seed: int = 0) -> NeuMesh:
    """A box of nx*ny*nz hexahedra ('hex'), each split into 2 wedges along
    the x-y diagonal ('wedge'), into 6 tetrahedra around its main diagonal
    ('tet', conforming across cells) or into 6 pyramids on its faces with
    the apex at its centre ('pyramid'; 'mixed' keeps every other hexahedron
    whole, so bricks and pyramids share faces), with the six sides as
    boundary sets named like the polyMesh box (xmin ... zmax).  Interior
    nodes move by up to jitter/2 of a cell (seeded)."""
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    idx = np.stack([I.ravel(), J.ravel(), K.ravel()], 1)       # node grid indices, node id = (i*(ny+1)+j)*(nz+1)+k
    h = np.array([lx / nx, ly / ny, lz / nz])
    pts = idx * h
    if jitter:
        inner = np.all((idx > 0) & (idx < [nx, ny, nz]), axis=1)
        r = uniform01(seed, 3 * idx.shape[0]).reshape(-1, 3) - 0.5
        pts[inner] += jitter * r[inner] * h

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    types, conn = [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                c = [nid(i + a, j + b, k + d) for d in (0, 1) for b in (0, 1) for a in (0, 1)]   # Gambit brick order
                if kind == "hex":
                    types.append(4)
                    conn.append(c)
                elif kind == "wedge":
                    p000, p100, p010, p110, p001, p101, p011, p111 = c
                    types += [5, 5]
                    conn += [[p000, p100, p110, p001, p101, p111], [p000, p110, p010, p001, p111, p011]]
                elif kind == "tet":
                    P = {(a, b, d): nid(i + a, j + b, k + d) for a in (0, 1) for b in (0, 1) for d in (0, 1)}
                    for ax in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
                        v = [0, 0, 0]
                        path = [P[tuple(v)]]
                        for a in ax[:2]:
                            v[a] = 1
                            path.append(P[tuple(v)])
                        path.append(P[(1, 1, 1)])
                        types.append(6)
                        conn.append(path)
                elif kind in ("pyramid", "mixed"):
                    if kind == "mixed" and (i + j + k) % 2 == 0:
                        types.append(4)
                        conn.append(c)
                        continue
                    # six pyramids on the hex faces with the apex at the cell centre
                    centre = len(pts)
                    pts = np.vstack([pts, pts[c].mean(axis=0)])
                    idx = np.vstack([idx, [i + 0.5, j + 0.5, k + 0.5]])
                    for f in LOCAL_FACES[4]:
                        q = [c[x] for x in f]               # a cycle: base nodes 1,2,4,3 in Gambit order
                        types.append(7)
                        conn.append([q[0], q[1], q[3], q[2], centre])
                else:
                    raise ValueError(kind)
    etype = np.asarray(types, np.int32)
    ptr = np.zeros(len(conn) + 1, np.int32)
    ptr[1:] = np.cumsum([len(x) for x in conn])
    nodes = np.asarray([x for c in conn for x in c], np.int32)
    # boundary records: element faces whose nodes all lie on one side
    sides = [(0, 0), (0, nx), (1, 0), (1, ny), (2, 0), (2, nz)]
    recs = [[] for _ in sides]
    for e in range(len(conn)):
        en = conn[e]
        for jf, lf in enumerate(LOCAL_FACES[int(etype[e])]):
            g = idx[[en[q] for q in lf]]
            for s, (ax, val) in enumerate(sides):
                if np.all(g[:, ax] == val):
                    recs[s].append((e, jf))
    be = np.asarray([e for r in recs for e, _ in r], np.int32)
    bf = np.asarray([f for r in recs for _, f in r], np.int32)
    return NeuMesh(pts, etype, ptr, nodes, list(BOX_PATCHES), np.asarray([len(r) for r in recs], np.int32), be, bf,
                   [("fluid", 2, np.arange(len(conn), dtype=np.int32))], title=f"{kind} box {nx}x{ny}x{nz}")


# ----------------------------------------------------------------- connectivity
def _neu_struct(m: NeuMesh):
    keep = [np.ascontiguousarray(a, np.int32) for a in (m.etype, m.node_ptr, m.nodes, m.bc_size, m.bc_element, m.bc_face)]
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    s = L.FsNeuIn(n_elements=m.n_elements, type=ip(keep[0]), node_ptr=ip(keep[1]), nodes=ip(keep[2]),
                  n_sets=len(m.bc_names), set_size=ip(keep[3]), bc_element=ip(keep[4]), bc_face=ip(keep[5]))
    return s, keep


def connectivity(m: NeuMesh, fn=None) -> dict:
    """GlobalConnectivity's face list: `fn` is fs_neu_connectivity (default)
    or any function with its signature (the oracle's literal restatement)."""
    s, keep = _neu_struct(m)
    fmax = int(sum(FACES_PER_TYPE.get(int(t), 6) for t in m.etype))   # the library rejects unknown types
    out = {"face_ptr": np.zeros(fmax + 1, np.int32), "face_nodes": np.zeros(4 * fmax, np.int32),
           "owner": np.zeros(fmax, np.int32), "neighbour": np.zeros(fmax, np.int32),
           "cell_face_ptr": np.zeros(m.n_elements + 1, np.int32), "cell_faces": np.zeros(fmax, np.int32)}
    ni, nf = C.c_int32(0), C.c_int32(0)
    if fn is None:
        fn = L.load().fs_neu_connectivity
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    rc = fn(C.byref(s), C.byref(ni), C.byref(nf), ip(out["face_ptr"]), ip(out["face_nodes"]), ip(out["owner"]),
            ip(out["neighbour"]), ip(out["cell_face_ptr"]), ip(out["cell_faces"]))
    if rc != 0:
        raise RuntimeError(f"neutral-file connectivity failed ({rc})")
    F, NF = ni.value, nf.value
    out["face_ptr"] = out["face_ptr"][:NF + 1]
    out["face_nodes"] = out["face_nodes"][:out["face_ptr"][-1]]
    out["owner"] = out["owner"][:NF]
    out["neighbour"] = out["neighbour"][:F]
    out["n_internal"], out["n_faces"] = F, NF
    return out


def to_polymesh(m: NeuMesh, fn=None) -> PolyMesh:
    """The solver's mesh form of a neutral-file mesh, with the element-local
    face order and the file's element node order attached."""
    c = connectivity(m, fn)
    F = c["n_internal"]
    starts = F + np.concatenate([[0], np.cumsum(m.bc_size)[:-1]]).astype(np.int32)
    pm = PolyMesh(np.ascontiguousarray(m.points, np.float64), c["face_ptr"], c["face_nodes"], c["owner"],
                  c["neighbour"], list(m.bc_names), starts, np.asarray(m.bc_size, np.int32))
    pm.cell_face_ptr, pm.cell_faces = c["cell_face_ptr"], c["cell_faces"]
    pm.cell_node_ptr, pm.cell_nodes = np.asarray(m.node_ptr, np.int32), np.asarray(m.nodes, np.int32)
    return pm
