"""Spatial hash grid for particle neighbourhoods on the GPU.

Mirrors physgrad::sparse::SpatialHashGrid<float, uint32_t>
(src/sparse_data_structures.h:44-296, used by src/fsi_coupling.h:72): the
same constructor, buildHashTable, getNeighbors, getStats and table
accessors, over the C-ABI (pgmpm_hashgrid_*).  The table and the neighbour
lists equal the host class's bit for bit; getNeighbors returns, as there,
every particle of the cells within ceil(radius / cell_size) cells of the
query's cell, without a distance test.  ``neighbors`` answers many queries
in one call (offsets + indices).
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _capi as C
from ._capi import check, lib


def _f32(a, shape_last=3):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.reshape(-1, shape_last)


class SpatialHashGrid:
    def __init__(self, cell_size: float, domain_min: Sequence[float], domain_max: Sequence[float],
                 max_particles: int = 10_000_000, device: int = 0):
        dmin = (ctypes.c_float * 3)(*[float(v) for v in domain_min])
        dmax = (ctypes.c_float * 3)(*[float(v) for v in domain_max])
        h = ctypes.c_void_p()
        check(lib().pgmpm_hashgrid_create(float(cell_size), dmin, dmax, int(max_particles), int(device),
                                          ctypes.byref(h)))
        self._h = h
        self.cell_size = float(cell_size)
        self.n = 0
        info = self._info()
        self.total_cells = int(info.total_cells)
        self.resolution = tuple(int(r) for r in info.resolution)

    def _info(self):
        info = C.HashGridInfo()
        check(lib().pgmpm_hashgrid_stats(self._h, ctypes.byref(info)))
        return info

    def close(self):
        if getattr(self, "_h", None):
            lib().pgmpm_hashgrid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference API
    def buildHashTable(self, positions, num_particles: int | None = None):
        p = _f32(positions)
        n = len(p) if num_particles is None else int(num_particles)
        check(lib().pgmpm_hashgrid_build(self._h, p.ctypes.data, n, C.PTR_HOST, None))
        self.n = n

    def getNeighbors(self, x: float, y: float, z: float, radius: float) -> list:
        off, idx = self.neighbors(np.array([[x, y, z]], np.float32), radius)
        return idx.tolist()

    def getStats(self) -> dict:
        i = self._info()
        return {"average_particles_per_cell": i.average_particles_per_cell, "load_factor": i.load_factor,
                "max_particles_per_cell": i.max_particles_per_cell, "occupied_cells": i.occupied_cells,
                "memory_usage_mb": i.memory_usage_mb}

    def getCellSize(self) -> float:
        return self.cell_size

    def getTotalCells(self) -> int:
        return self.total_cells

    def getParticleIndices(self) -> np.ndarray:
        return self._table()[2]

    def getCellStartIndices(self) -> np.ndarray:
        return self._table()[1]

    def getCellParticleCounts(self) -> np.ndarray:
        return self._table()[0]

    def getParticleCellIds(self) -> np.ndarray:
        return self._table()[3]

    # -- batched queries
    def neighbors(self, queries, radius: float):
        """(offsets [nq + 1] int64, indices [offsets[-1]] uint32): query i's
        list is indices[offsets[i]:offsets[i + 1]]."""
        q = _f32(queries)
        nq = len(q)
        off = np.zeros(nq + 1, np.int64)
        total = ctypes.c_int64()
        check(lib().pgmpm_hashgrid_neighbors(self._h, q.ctypes.data, nq, float(radius), off.ctypes.data, None, 0,
                                             ctypes.byref(total), C.PTR_HOST, None))
        idx = np.zeros(max(int(total.value), 1), np.uint32)
        check(lib().pgmpm_hashgrid_neighbors(self._h, q.ctypes.data, nq, float(radius), off.ctypes.data,
                                             idx.ctypes.data, len(idx), ctypes.byref(total), C.PTR_HOST, None))
        return off, idx[: int(total.value)]

    def _table(self):
        c = np.zeros(self.total_cells, np.uint32)
        s = np.zeros(self.total_cells, np.uint32)
        ix = np.zeros(max(self.n, 1), np.uint32)
        cid = np.zeros(max(self.n, 1), np.uint32)
        check(lib().pgmpm_hashgrid_get_table(self._h, c.ctypes.data, s.ctypes.data, ix.ctypes.data, cid.ctypes.data,
                                             C.PTR_HOST, None))
        return c, s, ix[: self.n], cid[: self.n]
