"""Synthetic meshes in polyMesh form and an OpenFOAM polyMesh reader/writer.

The reference reads its meshes with ``Readit`` (SolveEquations/GridAndGeometry/
ReadFoamMesh.f90:31-297): ``points``, ``faces``, ``owner``, ``neighbour`` and
``boundary`` files, interior faces first (those that have a neighbour), then
the boundary faces patch by patch.  ``PolyMesh`` holds exactly that content,
0-based, and is what :func:`flowsolversourcecode_b200.solver.Solver` uploads.

``box_mesh`` generates the structured hex boxes of the benchmark cases as an
unstructured mesh, in OpenFOAM's upper-triangular face order (for each owner
cell in order, its faces to higher-numbered neighbours in increasing
neighbour order), so the same arrays written by :func:`write_polymesh` are a
valid input for the reference.  Interior nodes may be jittered by a seeded
splitmix64 stream.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

# patch order produced by box_mesh
BOX_PATCHES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """The first ``count`` outputs of splitmix64 started at state ``seed``.

    Output k uses state seed + (k+1)*0x9E3779B97F4A7C15 (the standard
    sequence), mixed with the published finaliser (Steele et al., 2014).
    """
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, count: int) -> np.ndarray:
    """Doubles in [0,1): the top 53 bits of each splitmix64 output times 2^-53."""
    return (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class PolyMesh:
    points: np.ndarray            # (n_nodes, 3) float64
    face_ptr: np.ndarray          # (n_faces+1,) int32
    face_nodes: np.ndarray        # int32
    owner: np.ndarray             # (n_faces,) int32
    neighbour: np.ndarray         # (n_internal,) int32
    patch_names: list = field(default_factory=list)
    patch_start: np.ndarray = None  # int32 face index of each patch's first face
    patch_size: np.ndarray = None

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])

    @property
    def n_internal(self) -> int:
        return int(self.neighbour.shape[0])

    @property
    def n_cells(self) -> int:
        return int(max(self.owner.max(), self.neighbour.max() if self.n_internal else -1)) + 1

    def patch(self, name: str) -> int:
        return self.patch_names.index(name)


def box_mesh(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0,
             jitter: float = 0.0, seed: int = 0) -> PolyMesh:
    """Structured nx*ny*nz hex box [0,lx]x[0,ly]x[0,lz] as a polyMesh.

    Cell (i,j,k) has index i + nx*(j + ny*k); node (i,j,k) has index
    i + (nx+1)*(j + (ny+1)*k).  ``jitter`` moves every node that is not on the
    boundary by U(-jitter*h, +jitter*h) per coordinate (h the spacing in that
    direction), drawing three splitmix64 values per node in node order.
    Patches: xmin, xmax, ymin, ymax, zmin, zmax.
    """
    nx, ny, nz = int(nx), int(ny), int(nz)
    px, py = nx + 1, ny + 1
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).copy()
    if jitter:
        nn = pts.shape[0]
        r = uniform01(seed, 3 * nn).reshape(nn, 3) * 2.0 - 1.0
        ii = np.arange(nn)
        ni, nj, nk = ii % px, (ii // px) % py, ii // (px * py)
        interior = (ni > 0) & (ni < nx) & (nj > 0) & (nj < ny) & (nk > 0) & (nk < nz)
        h = np.array([lx / nx, ly / ny, lz / nz])
        pts[interior] += jitter * r[interior] * h

    def node(i, j, k):
        return i + px * (j + py * k)

    # interior faces, owner-major, neighbours ascending: +x (c+1), +y (c+nx), +z (c+nx*ny)
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = ci.transpose(2, 1, 0).ravel(), cj.transpose(2, 1, 0).ravel(), ck.transpose(2, 1, 0).ravel()
    cell = ci + nx * (cj + ny * ck)
    faces, own, nbr = [], [], []
    blocks = []  # (mask, owner, nb, nodes) per direction, then merged owner-major
    # x faces between (i,j,k) and (i+1,j,k)
    mx = ci < nx - 1
    fx = np.stack([node(ci + 1, cj, ck), node(ci + 1, cj + 1, ck), node(ci + 1, cj + 1, ck + 1), node(ci + 1, cj, ck + 1)], 1)
    my = cj < ny - 1
    fy = np.stack([node(ci, cj + 1, ck), node(ci, cj + 1, ck + 1), node(ci + 1, cj + 1, ck + 1), node(ci + 1, cj + 1, ck)], 1)
    mz = ck < nz - 1
    fz = np.stack([node(ci, cj, ck + 1), node(ci + 1, cj, ck + 1), node(ci + 1, cj + 1, ck + 1), node(ci, cj + 1, ck + 1)], 1)
    # order: for each cell, x then y then z (neighbour c+1 < c+nx < c+nx*ny)
    n = cell.shape[0]
    fn = np.zeros((n, 3, 4), np.int64)
    fn[:, 0], fn[:, 1], fn[:, 2] = fx, fy, fz
    nb = np.stack([cell + 1, cell + nx, cell + nx * ny], 1)
    msk = np.stack([mx, my, mz], 1)
    order = np.argsort(cell, kind="stable")
    fn, nb, msk, cel = fn[order], nb[order], msk[order], cell[order]
    own_i = np.repeat(cel[:, None], 3, 1)[msk]
    nbr_i = nb[msk]
    nodes_i = fn[msk]
    # boundary patches, faces in cell order; node order gives an outward normal
    bnodes, bown, psz = [], [], []
    cs = cel  # cells sorted
    i_, j_, k_ = cs % nx, (cs // nx) % ny, cs // (nx * ny)
    for name in BOX_PATCHES:
        if name == "xmin":
            m = i_ == 0; q = np.stack([node(i_, j_, k_), node(i_, j_, k_ + 1), node(i_, j_ + 1, k_ + 1), node(i_, j_ + 1, k_)], 1)
        elif name == "xmax":
            m = i_ == nx - 1; q = np.stack([node(i_ + 1, j_, k_), node(i_ + 1, j_ + 1, k_), node(i_ + 1, j_ + 1, k_ + 1), node(i_ + 1, j_, k_ + 1)], 1)
        elif name == "ymin":
            m = j_ == 0; q = np.stack([node(i_, j_, k_), node(i_ + 1, j_, k_), node(i_ + 1, j_, k_ + 1), node(i_, j_, k_ + 1)], 1)
        elif name == "ymax":
            m = j_ == ny - 1; q = np.stack([node(i_, j_ + 1, k_), node(i_, j_ + 1, k_ + 1), node(i_ + 1, j_ + 1, k_ + 1), node(i_ + 1, j_ + 1, k_)], 1)
        elif name == "zmin":
            m = k_ == 0; q = np.stack([node(i_, j_, k_), node(i_, j_ + 1, k_), node(i_ + 1, j_ + 1, k_), node(i_ + 1, j_, k_)], 1)
        else:
            m = k_ == nz - 1; q = np.stack([node(i_, j_, k_ + 1), node(i_ + 1, j_, k_ + 1), node(i_ + 1, j_ + 1, k_ + 1), node(i_, j_ + 1, k_ + 1)], 1)
        bnodes.append(q[m]); bown.append(cs[m]); psz.append(int(m.sum()))
    all_nodes = np.concatenate([nodes_i] + bnodes, 0).astype(np.int32)
    owner = np.concatenate([own_i] + bown).astype(np.int32)
    nfaces = owner.shape[0]
    face_ptr = (np.arange(nfaces + 1, dtype=np.int64) * 4).astype(np.int32)
    n_int = own_i.shape[0]
    pstart = np.cumsum([n_int] + psz[:-1]).astype(np.int32)
    return PolyMesh(points=pts, face_ptr=face_ptr, face_nodes=all_nodes.ravel(), owner=owner,
                    neighbour=nbr_i.astype(np.int32), patch_names=list(BOX_PATCHES),
                    patch_start=pstart, patch_size=np.array(psz, np.int32))


BFS_PATCHES = ("inlet", "step", "xmax", "ymin", "ymax", "zmin", "zmax")


def bfs_mesh(nx: int, ny: int, nz: int, H: float = 1.0) -> PolyMesh:
    """Backward-facing-step channel 30H x 3H x 2H: the box of ``box_mesh``
    whose xmin patch is split into ``inlet`` (cells with y >= H) and ``step``
    (the wall of the step face, y < H), each in cell order.  ny must be a
    multiple of 3 so that y = H is a grid line.  Patches: inlet, step, xmax
    (the outlet), ymin, ymax, zmin, zmax."""
    if ny % 3:
        raise ValueError("ny must be a multiple of 3 (y = H on a grid line)")
    m = box_mesh(nx, ny, nz, 30.0 * H, 3.0 * H, 2.0 * H)
    s0, n0 = int(m.patch_start[0]), int(m.patch_size[0])
    own = m.owner[s0:s0 + n0]
    j = (own // nx) % ny
    up = np.nonzero(j >= ny // 3)[0]
    lo = np.nonzero(j < ny // 3)[0]
    order = np.concatenate([up, lo])
    fn = m.face_nodes.reshape(-1, 4).copy()
    fn[s0:s0 + n0] = fn[s0 + order]
    owner = m.owner.copy()
    owner[s0:s0 + n0] = own[order]
    psz = [len(up), len(lo)] + [int(x) for x in m.patch_size[1:]]
    pstart = np.cumsum([s0] + psz[:-1]).astype(np.int32)
    return PolyMesh(points=m.points, face_ptr=m.face_ptr, face_nodes=fn.ravel(), owner=owner,
                    neighbour=m.neighbour, patch_names=list(BFS_PATCHES),
                    patch_start=pstart, patch_size=np.array(psz, np.int32))


# --------------------------------------------------------------------------
# OpenFOAM ASCII polyMesh I/O (the files Readit parses)
# --------------------------------------------------------------------------
_HDR = """FoamFile
{{
    version     2.0;
    format      ascii;
    class       {cls};
    location    "constant/polyMesh";
    object      {obj};
}}
"""


def write_polymesh(mesh: PolyMesh, directory: str) -> None:
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "points"), "w") as f:
        f.write(_HDR.format(cls="vectorField", obj="points"))
        f.write(f"\n{mesh.points.shape[0]}\n(\n")
        for x, y, z in mesh.points:
            f.write(f"({float(x)!r} {float(y)!r} {float(z)!r})\n")
        f.write(")\n")
    with open(os.path.join(directory, "faces"), "w") as f:
        f.write(_HDR.format(cls="faceList", obj="faces"))
        f.write(f"\n{mesh.n_faces}\n(\n")
        for i in range(mesh.n_faces):
            nd = mesh.face_nodes[mesh.face_ptr[i]:mesh.face_ptr[i + 1]]
            f.write(f"{len(nd)}(" + " ".join(str(int(q)) for q in nd) + ")\n")
        f.write(")\n")
    for name, arr in (("owner", mesh.owner), ("neighbour", mesh.neighbour)):
        with open(os.path.join(directory, name), "w") as f:
            f.write(_HDR.format(cls="labelList", obj=name))
            f.write(f"\n{arr.shape[0]}\n(\n")
            f.write("\n".join(str(int(q)) for q in arr))
            f.write("\n)\n")
    with open(os.path.join(directory, "boundary"), "w") as f:
        f.write(_HDR.format(cls="polyBoundaryMesh", obj="boundary"))
        f.write(f"\n{len(mesh.patch_names)}\n(\n")
        for name, st, sz in zip(mesh.patch_names, mesh.patch_start, mesh.patch_size):
            f.write(f"    {name}\n    {{\n        type            patch;\n"
                    f"        nFaces          {int(sz)};\n        startFace       {int(st)};\n    }}\n")
        f.write(")\n")


def _list_body(path: str):
    with open(path) as f:
        txt = f.read()
    i = txt.index("FoamFile")
    j = txt.index("}", i)
    body = txt[j + 1:]
    k = body.index("(")
    n = int(body[:k].split()[-1])
    return n, body[k + 1:body.rindex(")")]


def read_polymesh(directory: str) -> PolyMesh:
    """Read an ASCII polyMesh the way Readit does (ReadFoamMesh.f90:52-270)."""
    n, body = _list_body(os.path.join(directory, "points"))
    pts = np.array(body.replace("(", " ").replace(")", " ").split(), np.float64).reshape(n, 3)
    n, body = _list_body(os.path.join(directory, "faces"))
    toks = body.replace("(", " ").replace(")", " ").split()
    ptr, nodes, q = [0], [], 0
    for _ in range(n):
        c = int(toks[q]); nodes.extend(int(t) for t in toks[q + 1:q + 1 + c]); q += 1 + c
        ptr.append(ptr[-1] + c)
    n, body = _list_body(os.path.join(directory, "owner"))
    owner = np.array(body.split(), np.int32)
    n, body = _list_body(os.path.join(directory, "neighbour"))
    nbr = np.array(body.split(), np.int32)
    with open(os.path.join(directory, "boundary")) as f:
        txt = f.read()
    body = txt[txt.index("}", txt.index("FoamFile")) + 1:]
    names, starts, sizes = [], [], []
    import re
    for m in re.finditer(r"(\w+)\s*\{([^}]*)\}", body):
        d = m.group(2)
        names.append(m.group(1))
        sizes.append(int(re.search(r"nFaces\s+(\d+)", d).group(1)))
        starts.append(int(re.search(r"startFace\s+(\d+)", d).group(1)))
    return PolyMesh(points=pts, face_ptr=np.array(ptr, np.int32), face_nodes=np.array(nodes, np.int32),
                    owner=owner, neighbour=nbr, patch_names=names,
                    patch_start=np.array(starts, np.int32), patch_size=np.array(sizes, np.int32))
