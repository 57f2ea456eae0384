"""GPU spatial hash grid (pgmpm_hashgrid_*, physgrad_b200.SpatialHashGrid)
against the reference's SpatialHashGrid (src/sparse_data_structures.h):
integer work, so every array is compared bit for bit -- per-cell counts and
starts, particle indices sorted by cell, cell ids, and the getNeighbors
lists (offsets and concatenated indices) -- with the golden fixture made
from the reference class (tests/golden/make_hashgrid_golden.py)."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _case(g, k):
    prm = g[f"c{k}_param"]
    return float(prm[0]), prm[1:4], prm[4:7], float(prm[7])


@pytest.mark.parametrize("k", [0, 1, 2])
def test_hashgrid_matches_reference_golden(gpu, k):
    from oracle import hashgrid as H

    g = np.load(os.path.join(GOLDEN, "hashgrid_small.npz"))
    cs, mn, mx, r = _case(g, k)
    p, q = g[f"c{k}_p"], g[f"c{k}_q"]
    grid = gpu.SpatialHashGrid(cs, mn, mx, max_particles=len(p))
    for _ in range(2):  # a rebuild over the same grid gives the same table
        grid.buildHashTable(p)
        assert np.array_equal(grid.getCellParticleCounts(), g[f"c{k}_counts"])
        assert np.array_equal(grid.getCellStartIndices(), g[f"c{k}_starts"])
        assert np.array_equal(grid.getParticleIndices(), g[f"c{k}_indices"])
        res, total = H.resolution(cs, mn, mx)
        assert np.array_equal(grid.getParticleCellIds(), H.cell_ids(p, cs, mn, res, total))
        off, lists = grid.neighbors(q, r)
        assert np.array_equal(off, g[f"c{k}_offsets"]) and np.array_equal(lists, g[f"c{k}_lists"])
    i = 3
    assert grid.getNeighbors(*q[i], r) == g[f"c{k}_lists"][g[f"c{k}_offsets"][i]:g[f"c{k}_offsets"][i + 1]].tolist()
    st = grid.getStats()
    c = g[f"c{k}_counts"]
    assert st["occupied_cells"] == int((c > 0).sum()) and st["max_particles_per_cell"] == int(c.max())
    assert abs(st["load_factor"] - (c > 0).sum() / len(c)) < 1e-6


def test_hashgrid_device_pointers_capacity_and_errors(gpu):
    """Device arrays through the C-ABI give the host path's results; indices
    are written only when capacity covers the total; an empty build has empty
    cells and lists; more particles than max_particles is an error."""
    import torch

    from physgrad_b200 import _capi as C

    g = np.load(os.path.join(GOLDEN, "hashgrid_small.npz"))
    cs, mn, mx, r = _case(g, 0)
    p, q = g["c0_p"], g["c0_q"]
    grid = gpu.SpatialHashGrid(cs, mn, mx, max_particles=len(p))
    L = C.lib()
    pd = torch.tensor(p, device="cuda")
    qd = torch.tensor(q, device="cuda")
    assert L.pgmpm_hashgrid_build(grid._h, pd.data_ptr(), len(p), C.PTR_DEVICE, None) == 0
    grid.n = len(p)
    off = torch.zeros(len(q) + 1, dtype=torch.int64, device="cuda")
    tot = ctypes.c_int64()
    assert L.pgmpm_hashgrid_neighbors(grid._h, qd.data_ptr(), len(q), r, off.data_ptr(), None, 0, ctypes.byref(tot),
                                      C.PTR_DEVICE, None) == 0
    assert tot.value == len(g["c0_lists"])
    small = torch.full((5,), 7, dtype=torch.int32, device="cuda")
    assert L.pgmpm_hashgrid_neighbors(grid._h, qd.data_ptr(), len(q), r, off.data_ptr(), small.data_ptr(), 5,
                                      ctypes.byref(tot), C.PTR_DEVICE, None) == 0
    torch.cuda.synchronize()
    assert (small == 7).all().item()  # capacity too small: nothing written
    out = torch.zeros(tot.value, dtype=torch.int32, device="cuda")
    assert L.pgmpm_hashgrid_neighbors(grid._h, qd.data_ptr(), len(q), r, off.data_ptr(), out.data_ptr(), tot.value,
                                      ctypes.byref(tot), C.PTR_DEVICE, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(off.cpu().numpy(), g["c0_offsets"])
    assert np.array_equal(out.cpu().numpy().view(np.uint32), g["c0_lists"])
    grid.buildHashTable(np.zeros((0, 3), np.float32))
    assert int(grid.getCellParticleCounts().sum()) == 0
    o, lists = grid.neighbors(q[:4], r)
    assert lists.size == 0 and np.array_equal(o, np.zeros(5, np.int64))
    with pytest.raises(Exception, match="max_particles"):
        grid.buildHashTable(np.zeros((len(p) + 1, 3), np.float32))


def test_hashgrid_wide_radius_matches_oracle(gpu):
    """A radius of 5.5 cells visits 13^3 = 2197 cells per query, more than the
    fill's shared offset table holds (the offsets are then computed per
    cell): lists equal the restated reference's (oracle/hashgrid.py)."""
    from oracle import hashgrid as H

    rng = np.random.default_rng(11)
    cs, mn, mx = 0.05, np.zeros(3, np.float32), np.ones(3, np.float32)
    p = rng.random((4000, 3), dtype=np.float32)
    q = rng.random((24, 3), dtype=np.float32)
    r = 5.5 * cs
    grid = gpu.SpatialHashGrid(cs, mn, mx, max_particles=len(p))
    grid.buildHashTable(p)
    c, s, ix, _ = H.build(p, cs, mn, mx)
    o_ref, l_ref = H.neighbors(q, r, cs, mn, mx, c, s, ix)
    off, lists = grid.neighbors(q, r)
    assert np.array_equal(off, o_ref) and np.array_equal(lists, l_ref)
