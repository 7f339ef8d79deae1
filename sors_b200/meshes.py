"""Synthetic meshes for the FEM workloads, and surface extraction.

Host-side set-up code (numpy), run once per mesh.  Node and element arrays use
the reference conventions: vertices (N,3) float64, elements (E,4) tets or (E,8)
hexes with the vertex order of IO::make_voxel_hex_grid
(cpp/src/io.cpp:931-988): bottom face 0-1-2-3, top face 4-5-6-7, i-edge 0->1.
"""
from __future__ import annotations

import numpy as np

# The six tetrahedra of the Kuhn (Freudenthal) split of a unit cell: each is
# the path c000 -> +e_a -> +e_a+e_b -> c111 for one permutation (a, b, c) of
# the axes.  Neighbouring cells split their shared faces the same way, so the
# resulting tet mesh is conforming.
_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def grid_nodes(nx: int, ny: int, nz: int, size) -> np.ndarray:
    """Nodes of an nx x ny x nz cell grid on [0,Lx]x[0,Ly]x[0,Lz]; vid = i + NX*(j + NY*k)."""
    Lx, Ly, Lz = size
    xs = np.linspace(0.0, Lx, nx + 1)
    ys = np.linspace(0.0, Ly, ny + 1)
    zs = np.linspace(0.0, Lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def _vid(i, j, k, NX, NY):
    return i + NX * (j + NY * k)


def hex_grid_elements(nx: int, ny: int, nz: int) -> np.ndarray:
    """Hexes in the vertex order of IO::make_voxel_hex_grid (cpp/src/io.cpp:967-984)."""
    NX, NY = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    e = np.stack([
        _vid(i, j, k, NX, NY), _vid(i + 1, j, k, NX, NY), _vid(i + 1, j + 1, k, NX, NY), _vid(i, j + 1, k, NX, NY),
        _vid(i, j, k + 1, NX, NY), _vid(i + 1, j, k + 1, NX, NY), _vid(i + 1, j + 1, k + 1, NX, NY),
        _vid(i, j + 1, k + 1, NX, NY)], axis=1)
    return e.astype(np.int32)


def kuhn_tet_elements(nx: int, ny: int, nz: int) -> np.ndarray:
    """6 tets per cell (Kuhn split), conforming across cells."""
    NX, NY = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)
    tets = []
    for (a, b, _c) in _PERMS:
        p0 = base
        p1 = base.copy(); p1[:, a] += 1
        p2 = p1.copy(); p2[:, b] += 1
        p3 = base + 1
        tets.append(np.stack([_vid(p[:, 0], p[:, 1], p[:, 2], NX, NY) for p in (p0, p1, p2, p3)], axis=1))
    # cell-major order: the 6 tets of one cell are consecutive
    t = np.stack(tets, axis=1).reshape(-1, 4)
    return t.astype(np.int32)


def jitter_interior(X: np.ndarray, h: float, frac: float, rng: np.random.Generator) -> np.ndarray:
    """Move interior nodes by U(-frac*h, +frac*h) per axis (boundary nodes stay)."""
    lo, hi = X.min(0), X.max(0)
    tol = 1e-9 * max(1.0, float(np.abs(X).max()))
    interior = np.all((X > lo + tol) & (X < hi - tol), axis=1)
    Xj = X.copy()
    Xj[interior] += rng.uniform(-frac * h, frac * h, size=(int(interior.sum()), 3))
    return Xj


def clamp_mask(X: np.ndarray, axis: int = 0, value: float | None = None, tol: float = 1e-9):
    """Neumann mask/value (3N) fixing every node with X[:,axis] == min (velocity 0)."""
    v = X[:, axis].min() if value is None else value
    fixed = np.abs(X[:, axis] - v) <= tol * max(1.0, abs(v)) + tol
    mask = np.repeat(fixed.astype(np.int32), 3)
    return mask, np.zeros(3 * X.shape[0])


# ---------------------------------------------------------------------------
# Workload meshes
# ---------------------------------------------------------------------------

def cantilever_tets(nx=20, ny=4, nz=4, size=(0.1, 0.02, 0.02)):
    """Structured beam split into 6 tets per cell (1920 tets, 525 nodes at 20x4x4)."""
    X = grid_nodes(nx, ny, nz, size)
    return X, kuhn_tet_elements(nx, ny, nz)


def jittered_block_tets(nx=200, ny=50, nz=50, size=(1.0, 0.25, 0.25), jitter=0.1, seed=0,
                        e_range=(5e4, 5e5)):
    """Jittered 6-tet block with per-element log-uniform Young's modulus."""
    rng = np.random.default_rng(seed)
    X = grid_nodes(nx, ny, nz, size)
    h = size[0] / nx
    X = jitter_interior(X, h, jitter, rng)
    T = kuhn_tet_elements(nx, ny, nz)
    E = np.exp(rng.uniform(np.log(e_range[0]), np.log(e_range[1]), size=T.shape[0]))
    return X, T, E


def hex_bar(nx=40, ny=8, nz=8, size=(0.2, 0.04, 0.04)):
    X = grid_nodes(nx, ny, nz, size)
    return X, hex_grid_elements(nx, ny, nz)


def voxel_cylinder(radius=0.02, length=0.2, h=1.25e-3, chamber_radius=0.004, chamber_offset=0.008,
                   chamber_angles_deg=(0.0, 120.0, 240.0), cap_layers=0):
    """Voxelised cylinder along z with cylindrical chambers (hexes, h-sized voxels).

    A voxel is solid when its centre lies inside the outer radius and outside
    every chamber; the first and last `cap_layers` voxel layers are solid
    everywhere, which closes the chambers so each becomes its own surface.
    Returns (X, hexes) with only the nodes used by solid voxels.
    """
    n_xy = int(np.ceil(2 * radius / h))
    nz = int(round(length / h))
    c = (np.arange(n_xy) + 0.5) * h - n_xy * h / 2.0
    cx, cy = np.meshgrid(c, c, indexing="ij")
    inside = cx ** 2 + cy ** 2 <= radius ** 2
    chambers = []
    for ang in chamber_angles_deg:
        a = np.deg2rad(ang)
        ox, oy = chamber_offset * np.cos(a), chamber_offset * np.sin(a)
        chambers.append((cx - ox) ** 2 + (cy - oy) ** 2 <= chamber_radius ** 2)
    solid2d = inside.copy()
    for ch in chambers:
        solid2d &= ~ch
    NX = NY = n_xy + 1
    ii, jj = np.nonzero(solid2d)
    ii_in, jj_in = np.nonzero(inside)
    hexes = []
    for k in range(nz):
        capped = k < cap_layers or k >= nz - cap_layers
        i, j = (ii_in, jj_in) if capped else (ii, jj)
        hexes.append(np.stack([
            _vid(i, j, k, NX, NY), _vid(i + 1, j, k, NX, NY), _vid(i + 1, j + 1, k, NX, NY),
            _vid(i, j + 1, k, NX, NY), _vid(i, j, k + 1, NX, NY), _vid(i + 1, j, k + 1, NX, NY),
            _vid(i + 1, j + 1, k + 1, NX, NY), _vid(i, j + 1, k + 1, NX, NY)], axis=1))
    H = np.concatenate(hexes, 0)
    used = np.unique(H)
    remap = -np.ones(NX * NY * (nz + 1), dtype=np.int64)
    remap[used] = np.arange(used.size)
    k_, r = np.divmod(used, NX * NY)
    j_, i_ = np.divmod(r, NX)
    X = np.stack([i_ * h - n_xy * h / 2.0, j_ * h - n_xy * h / 2.0, k_ * h], axis=1).astype(np.float64)
    return X, remap[H].astype(np.int32)


# ---------------------------------------------------------------------------
# Surface extraction (restates IO::extract_tet_surfaces / extract_hex_surfaces,
# cpp/src/io.cpp:570-781, with hashing instead of linear searches)
# ---------------------------------------------------------------------------
_TET_FACES = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])
_HEX_FACES = np.array([[0, 1, 2, 3], [4, 5, 6, 7], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7]])


def extract_surfaces(X: np.ndarray, elements: np.ndarray):
    """Boundary faces grouped by vertex-connectivity, oriented outwards.

    Returns (groups, face_elements): groups is a list of (F_g, nv) int arrays.
    Boundary faces are those that occur in exactly one element (io.cpp:580-612);
    a group grows by any face sharing a vertex with it (io.cpp:619-663); a face
    whose normal points towards its element's vertex mean is flipped (tets:
    (f0,f2,f1) on the sorted face, io.cpp:637-642; hexes: swap f1,f3, io.cpp:760).
    """
    elements = np.asarray(elements)
    nv = elements.shape[1]
    ftab = _TET_FACES if nv == 4 else _HEX_FACES
    E = elements.shape[0]
    faces = elements[:, ftab].reshape(-1, ftab.shape[1])           # (E*nf, fnv) in element order
    owner = np.repeat(np.arange(E), ftab.shape[0])
    key = np.sort(faces, axis=1)
    _, inv, counts = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    inv = inv.ravel()
    boundary = counts[inv] == 1
    bidx = np.nonzero(boundary)[0]                                 # first-insertion order
    if nv == 4:
        bfaces = key[bidx]                                         # sorted ascending, like the reference
    else:
        bfaces = faces[bidx]
    bown = owner[bidx]
    com = X[elements[bown]].mean(axis=1)
    # connected components through shared vertices (union-find on vertices)
    nverts = X.shape[0]
    parent = np.arange(nverts)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for f in bfaces:
        r0 = find(f[0])
        for v in f[1:]:
            r = find(v)
            if r != r0:
                parent[r] = r0
    roots = np.array([find(f[0]) for f in bfaces])
    order_roots = []
    seen = set()
    for r in roots:
        if r not in seen:
            seen.add(r); order_roots.append(r)
    groups, face_ele = [], []
    for r in order_roots:
        sel = np.nonzero(roots == r)[0]
        fs = bfaces[sel].copy()
        a = X[fs[:, 0]]; b = X[fs[:, 1]]; c = X[fs[:, 2]]
        n = np.cross(b - a, c - a)
        inward = np.einsum("ij,ij->i", n, com[sel] - a) > 0
        if nv == 4:
            fs[inward] = fs[inward][:, [0, 2, 1]]
        else:
            fs[inward] = fs[inward][:, [0, 3, 2, 1]]
        groups.append(fs.astype(np.int32))
        face_ele.append(bown[sel].astype(np.int32))
    return groups, face_ele
