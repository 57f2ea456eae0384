"""CPU restatement of the reference's spatial hash grid (TEST INFRASTRUCTURE ONLY).

physgrad::sparse::SpatialHashGrid<float, uint32_t>
(src/sparse_data_structures.h:44-296) in numpy, used to check the GPU hash
grid of physgrad_b200 (pgmpm_hashgrid_*).  Pinned against the reference
class itself, compiled from its header into oracle/_ref/libref_hashgrid.so
(oracle/ref_shim/ref_hashgrid_shim.cpp), and against the golden fixture
tests/golden/hashgrid_small.npz generated from it.

Each function cites the lines it follows.  Arithmetic: single-precision
IEEE for the coordinates, uint32 wrap-around for the cell ids.
"""
import ctypes
import os

import numpy as np

U32 = np.uint64(0xFFFFFFFF)


def resolution(cell_size, dmin, dmax):
    """Constructor :80-85: ceil((max - min) / cell) per axis (single)."""
    cs = np.float32(cell_size)
    r = [int(np.ceil(np.float32(np.float32(dmax[a]) - np.float32(dmin[a])) / cs)) for a in range(3)]
    return r, (r[0] * r[1] * r[2]) & 0xFFFFFFFF


def expand_bits(v):
    """mortonEncode3D's expandBits :122-128 (uint32 arithmetic)."""
    v = np.asarray(v, np.uint64)
    v = (v * np.uint64(0x00010001)) & np.uint64(0xFF0000FF)
    v = (v * np.uint64(0x00000101)) & np.uint64(0x0F00F00F)
    v = (v * np.uint64(0x00000011)) & np.uint64(0xC30C30C3)
    v = (v * np.uint64(0x00000005)) & np.uint64(0x49249249)
    return v


def morton(x, y, z):
    """mortonEncode3D :121-131."""
    return (expand_bits(x) | (expand_bits(y) << np.uint64(1)) | (expand_bits(z) << np.uint64(2))) & U32


def grid_coords(p, cell_size, dmin):
    """getGridCoords :134-140: (uint32)((x - min) / cell) in single precision;
    the float -> uint32 conversion truncates toward zero to 64 bits and keeps
    the low 32 (x86-64)."""
    p = np.asarray(p, np.float32).reshape(-1, 3)
    t = (p - np.asarray(dmin, np.float32)) / np.float32(cell_size)
    return (np.trunc(t).astype(np.int64).astype(np.uint64)) & U32


def cell_ids(p, cell_size, dmin, res, total):
    """getCellID :143-151: coordinates clamped to resolution - 1."""
    c = grid_coords(p, cell_size, dmin)
    c = np.minimum(c, np.asarray(res, np.uint64) - np.uint64(1))
    return (morton(c[:, 0], c[:, 1], c[:, 2]) % np.uint64(total)).astype(np.uint32)


def build(p, cell_size, dmin, dmax):
    """buildHashTable :155-190: counts, exclusive scan, stable fill.
    Returns (counts, starts, particle_indices, cell_ids)."""
    res, total = resolution(cell_size, dmin, dmax)
    ids = cell_ids(p, cell_size, dmin, res, total)
    counts = np.bincount(ids, minlength=total).astype(np.uint32)
    starts = np.concatenate([[0], np.cumsum(counts, dtype=np.uint64)[:-1]]).astype(np.uint32)
    order = np.argsort(ids, kind="stable").astype(np.uint32)
    return counts, starts, order, ids


def neighbors(q, radius, cell_size, dmin, dmax, counts, starts, indices):
    """getNeighbors :206-240 for each query: (offsets, concatenated lists)."""
    res, total = resolution(cell_size, dmin, dmax)
    src = int(np.ceil(np.float32(radius) / np.float32(cell_size)))
    out, offs = [], [0]
    for c in grid_coords(q, cell_size, dmin):
        c = [int(v) for v in c]
        for dx in range(2 * src + 1):
            gx = (c[0] + dx - src) & 0xFFFFFFFF
            if gx >= res[0]:
                continue
            for dy in range(2 * src + 1):
                gy = (c[1] + dy - src) & 0xFFFFFFFF
                if gy >= res[1]:
                    continue
                for dz in range(2 * src + 1):
                    gz = (c[2] + dz - src) & 0xFFFFFFFF
                    if gz >= res[2]:
                        continue
                    cid = int(morton(gx, gy, gz)) % total
                    s, k = int(starts[cid]), int(counts[cid])
                    out.extend(indices[s:s + k].tolist())
        offs.append(len(out))
    return np.array(offs, np.int64), np.array(out, np.uint32)


# -- the reference class itself (oracle/_ref), when built
REF_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_hashgrid.so")


def reference_available():
    return os.path.exists(REF_LIB)


def reference_build_and_query(p, q, radius, cell_size, dmin, dmax):
    """Runs the reference SpatialHashGrid: (counts, starts, indices, offsets, lists)."""
    L = ctypes.CDLL(REF_LIB)
    L.ref_hashgrid_create.restype = ctypes.c_void_p
    L.ref_hashgrid_create.argtypes = [ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]
    L.ref_hashgrid_total_cells.restype = ctypes.c_uint32
    L.ref_hashgrid_total_cells.argtypes = [ctypes.c_void_p]
    L.ref_hashgrid_build.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32] + [ctypes.c_void_p] * 3
    L.ref_hashgrid_neighbors.restype = ctypes.c_int64
    L.ref_hashgrid_neighbors.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    L.ref_hashgrid_destroy.argtypes = [ctypes.c_void_p]
    p = np.ascontiguousarray(p, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    mn = np.asarray(dmin, np.float32)
    mx = np.asarray(dmax, np.float32)
    g = L.ref_hashgrid_create(np.float32(cell_size), mn.ctypes.data, mx.ctypes.data, max(len(p), 1))
    try:
        total = L.ref_hashgrid_total_cells(g)
        counts = np.zeros(total, np.uint32)
        starts = np.zeros(total, np.uint32)
        idx = np.zeros(max(len(p), 1), np.uint32)
        L.ref_hashgrid_build(g, p.ctypes.data, len(p), counts.ctypes.data, starts.ctypes.data, idx.ctypes.data)
        offs = np.zeros(len(q) + 1, np.int64)
        n = L.ref_hashgrid_neighbors(g, q.ctypes.data, len(q), np.float32(radius), offs.ctypes.data, None, 0)
        lists = np.zeros(max(n, 1), np.uint32)
        L.ref_hashgrid_neighbors(g, q.ctypes.data, len(q), np.float32(radius), offs.ctypes.data, lists.ctypes.data, n)
        return counts, starts, idx[: len(p)], offs, lists[:n]
    finally:
        L.ref_hashgrid_destroy(g)
