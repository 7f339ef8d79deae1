"""Gmsh MSH reader for the mesh-load path (host side, numpy).

Restates what IO::read_tet_MSH / read_hex_MSH do (cpp/src/io.cpp:380-569)
through the mshio library: every node of every node block is kept in file
order, node tags are mapped to 0-based vertex indices, and only elements of
Gmsh type 4 (4-node tetrahedron) or 5 (8-node hexahedron) are returned, block
by block in file order.  Formats: MSH 4.1 and 2.2, ASCII and binary (the
layouts published in the Gmsh reference manual, "MSH file format").
"""
from __future__ import annotations

import numpy as np

_NODES_PER_TYPE = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5, 8: 3, 9: 6, 10: 9, 11: 10, 12: 27, 15: 1, 16: 8,
                   17: 20}


class _Cursor:
    def __init__(self, data: bytes):
        self.b = data
        self.i = 0

    def line(self) -> str:
        j = self.b.index(b"\n", self.i)
        s = self.b[self.i:j].decode("ascii", "replace").strip()
        self.i = j + 1
        return s

    def skip_ws(self):
        while self.i < len(self.b) and self.b[self.i] in b" \t\r\n":
            self.i += 1

    def take(self, dtype, count):
        n = np.dtype(dtype).itemsize * count
        out = np.frombuffer(self.b, dtype=dtype, count=count, offset=self.i)
        self.i += n
        return out

    def until(self, marker: bytes):
        j = self.b.index(marker, self.i)
        self.i = j + len(marker)
        self.skip_ws()


def _tokens_until(cur: _Cursor, marker: bytes):
    j = cur.b.index(marker, cur.i)
    toks = cur.b[cur.i:j].split()
    cur.i = j + len(marker)
    cur.skip_ws()
    return toks


def read_msh(filename):
    """Returns (vertices (N, 3) float64, {gmsh element type: (M, n) int32 vertex indices})."""
    with open(filename, "rb") as f:
        data = f.read()
    cur = _Cursor(data)
    cur.until(b"$MeshFormat")
    version, ftype, dsize = cur.line().split()[:3]
    binary = ftype == "1"
    if binary:
        one = cur.take("<i4", 1)[0]
        if one != 1:
            raise ValueError("big-endian MSH files are not supported")
        cur.skip_ws()
    cur.until(b"$EndMeshFormat")
    if version.startswith("4"):
        return _read_v4(cur, binary, int(dsize))
    if version.startswith("2"):
        return _read_v2(cur, binary)
    raise ValueError(f"unsupported MSH version {version}")


def _read_v4(cur, binary, dsize):
    st = "<u8" if dsize == 8 else "<u4"
    cur.until(b"$Nodes")
    if binary:
        nblocks, nnodes, _, _ = (int(v) for v in cur.take(st, 4))
        coords, tags = [], []
        for _ in range(nblocks):
            _, _, parametric = (int(v) for v in cur.take("<i4", 3))
            n = int(cur.take(st, 1)[0])
            if parametric:
                raise ValueError("parametric node blocks are not supported")
            tags.append(cur.take(st, n).astype(np.int64))
            coords.append(cur.take("<f8", 3 * n).reshape(n, 3))
        cur.skip_ws()
        cur.until(b"$EndNodes")
    else:
        toks = _tokens_until(cur, b"$EndNodes")
        p = 0
        nblocks, nnodes = int(toks[0]), int(toks[1])
        p = 4
        coords, tags = [], []
        for _ in range(nblocks):
            parametric, n = int(toks[p + 2]), int(toks[p + 3])
            if parametric:
                raise ValueError("parametric node blocks are not supported")
            p += 4
            tags.append(np.array(toks[p:p + n], dtype=np.int64)); p += n
            coords.append(np.array(toks[p:p + 3 * n], dtype=np.float64).reshape(n, 3)); p += 3 * n
    X = np.concatenate(coords) if coords else np.zeros((0, 3))
    T = np.concatenate(tags) if tags else np.zeros(0, np.int64)
    tag2idx = _tag_map(T)
    cur.until(b"$Elements")
    blocks = {}
    if binary:
        nblocks, _, _, _ = (int(v) for v in cur.take(st, 4))
        for _ in range(nblocks):
            _, _, etype = (int(v) for v in cur.take("<i4", 3))
            n = int(cur.take(st, 1)[0])
            nn = _NODES_PER_TYPE.get(etype)
            if nn is None:
                raise ValueError(f"unknown element type {etype}")
            rec = cur.take(st, n * (nn + 1)).reshape(n, nn + 1).astype(np.int64)
            blocks.setdefault(etype, []).append(rec[:, 1:])
    else:
        toks = _tokens_until(cur, b"$EndElements")
        nblocks = int(toks[0])
        p = 4
        for _ in range(nblocks):
            etype, n = int(toks[p + 2]), int(toks[p + 3])
            p += 4
            nn = _NODES_PER_TYPE.get(etype)
            if nn is None:
                raise ValueError(f"unknown element type {etype}")
            rec = np.array(toks[p:p + n * (nn + 1)], dtype=np.int64).reshape(n, nn + 1)
            p += n * (nn + 1)
            blocks.setdefault(etype, []).append(rec[:, 1:])
    return X, {t: tag2idx(np.concatenate(v)) for t, v in blocks.items()}


def _read_v2(cur, binary):
    cur.until(b"$Nodes")
    n = int(cur.line())
    if binary:
        rec = np.frombuffer(cur.b, dtype=np.dtype([("tag", "<i4"), ("xyz", "<f8", 3)]), count=n, offset=cur.i)
        cur.i += rec.nbytes
        cur.skip_ws()
        cur.until(b"$EndNodes")
        T = rec["tag"].astype(np.int64)
        X = np.array(rec["xyz"], dtype=np.float64)
    else:
        toks = _tokens_until(cur, b"$EndNodes")
        a = np.array(toks, dtype=np.float64).reshape(n, 4)
        T = a[:, 0].astype(np.int64)
        X = a[:, 1:4].copy()
    tag2idx = _tag_map(T)
    cur.until(b"$Elements")
    m = int(cur.line())
    blocks = {}
    if binary:
        done = 0
        while done < m:
            etype, count, ntags = (int(v) for v in cur.take("<i4", 3))
            nn = _NODES_PER_TYPE[etype]
            rec = cur.take("<i4", count * (1 + ntags + nn)).reshape(count, 1 + ntags + nn)
            blocks.setdefault(etype, []).append(rec[:, 1 + ntags:].astype(np.int64))
            done += count
    else:
        toks = _tokens_until(cur, b"$EndElements")
        p = 0
        rows = {}
        for _ in range(m):
            etype, ntags = int(toks[p + 1]), int(toks[p + 2])
            nn = _NODES_PER_TYPE[etype]
            s = p + 3 + ntags
            rows.setdefault(etype, []).append([int(t) for t in toks[s:s + nn]])
            p = s + nn
        for t, r in rows.items():
            blocks.setdefault(t, []).append(np.array(r, dtype=np.int64))
    return X, {t: tag2idx(np.concatenate(v)) for t, v in blocks.items()}


def _tag_map(tags):
    order = np.argsort(tags, kind="stable")
    sorted_tags = tags[order]

    def f(a):
        pos = np.searchsorted(sorted_tags, a)
        if pos.size and (pos.max() >= sorted_tags.size or not np.array_equal(sorted_tags[pos], a)):
            raise ValueError("element refers to an unknown node tag")
        return order[pos].astype(np.int32)
    return f


def read_tet_msh(filename):
    """IO::read_tet_MSH: (vertices, tets (E, 4)) - Gmsh type 4 elements only."""
    X, blocks = read_msh(filename)
    return X, blocks.get(4, np.zeros((0, 4), np.int32))


def read_hex_msh(filename):
    """IO::read_hex_MSH: (vertices, hexes (E, 8)) - Gmsh type 5 elements only."""
    X, blocks = read_msh(filename)
    return X, blocks.get(5, np.zeros((0, 8), np.int32))


def write_msh(filename, vertices, elements, version="4.1", binary=False):
    """Writes one node block and one element block (tets -> type 4, hexes -> type 5)."""
    X = np.asarray(vertices, np.float64)
    E = np.asarray(elements, np.int64)
    etype = 4 if E.shape[1] == 4 else 5
    n, m = X.shape[0], E.shape[0]
    tags = np.arange(1, n + 1, dtype=np.int64)
    with open(filename, "wb") as f:
        w = f.write
        w(f"$MeshFormat\n{version} {1 if binary else 0} 8\n".encode())
        if binary:
            w(np.array([1], "<i4").tobytes()); w(b"\n")
        w(b"$EndMeshFormat\n$Nodes\n")
        if version.startswith("4"):
            if binary:
                w(np.array([1, n, 1, n], "<u8").tobytes())
                w(np.array([3, 1, 0], "<i4").tobytes()); w(np.array([n], "<u8").tobytes())
                w(tags.astype("<u8").tobytes()); w(X.astype("<f8").tobytes()); w(b"\n")
            else:
                w(f"1 {n} 1 {n}\n3 1 0 {n}\n".encode())
                w("".join(f"{t}\n" for t in tags).encode())
                w("".join(f"{x:.17g} {y:.17g} {z:.17g}\n" for x, y, z in X).encode())
            w(b"$EndNodes\n$Elements\n")
            if binary:
                w(np.array([1, m, 1, m], "<u8").tobytes())
                w(np.array([3, 1, etype], "<i4").tobytes()); w(np.array([m], "<u8").tobytes())
                rec = np.concatenate([np.arange(1, m + 1)[:, None], E + 1], axis=1)
                w(rec.astype("<u8").tobytes()); w(b"\n")
            else:
                w(f"1 {m} 1 {m}\n3 1 {etype} {m}\n".encode())
                w("".join(" ".join(str(v) for v in [k + 1, *(E[k] + 1)]) + "\n" for k in range(m)).encode())
            w(b"$EndElements\n")
        else:
            w(f"{n}\n".encode())
            if binary:
                rec = np.zeros(n, dtype=np.dtype([("tag", "<i4"), ("xyz", "<f8", 3)]))
                rec["tag"] = tags; rec["xyz"] = X
                w(rec.tobytes()); w(b"\n")
            else:
                w("".join(f"{t} {x:.17g} {y:.17g} {z:.17g}\n" for t, (x, y, z) in zip(tags, X)).encode())
            w(f"$EndNodes\n$Elements\n{m}\n".encode())
            if binary:
                w(np.array([etype, m, 2], "<i4").tobytes())
                rec = np.concatenate([np.arange(1, m + 1)[:, None], np.zeros((m, 2), np.int64), E + 1], axis=1)
                w(rec.astype("<i4").tobytes()); w(b"\n")
            else:
                w("".join(" ".join(str(v) for v in [k + 1, etype, 2, 0, 0, *(E[k] + 1)]) + "\n"
                          for k in range(m)).encode())
            w(b"$EndElements\n")
