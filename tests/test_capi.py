"""The C-ABI library loads, exports every entry point of include/pgmpm.h and
its structs match the ctypes mirror (CPU only: no compute calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pgmpm.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n.startswith(("pgmpm_", "launch_"))))


def test_library_exports_every_header_symbol(built_lib):
    names = header_functions()
    assert "pgmpm_create" in names and "launch_mpm_timestep_forward" in names
    L = ctypes.CDLL(built_lib)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert set(names) <= exported
    # nothing but the C entry points is exported
    extra = [e for e in exported if not e.startswith(("pgmpm_", "launch_")) and not e.startswith("_")]
    assert not extra, extra


def test_ctypes_mirror_covers_header(built_lib):
    from physgrad_b200 import _capi

    assert set(header_functions()) == set(_capi.SIGNATURES)


def test_struct_layout_matches_c(tmp_path):
    """sizeof/offsetof of the C structs == the ctypes mirror."""
    from physgrad_b200 import _capi as C

    prog = tmp_path / "layout.c"
    prog.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "pgmpm.h"
int main(void){
 printf("%zu %zu %zu %zu\n", sizeof(pgmpm_scene_desc), offsetof(pgmpm_scene_desc, dx), offsetof(pgmpm_scene_desc, gravity), offsetof(pgmpm_scene_desc, dt));
 printf("%zu %zu %zu\n", sizeof(pgmpm_material), offsetof(pgmpm_material, density), offsetof(pgmpm_material, viscosity));
 printf("%zu %zu %zu\n", sizeof(pgmpm_metrics), offsetof(pgmpm_metrics, p2g_block), offsetof(pgmpm_metrics, g2p_ms));
 printf("%zu %zu\n", sizeof(pgmpm_create_options), offsetof(pgmpm_create_options, max_tiles));
 return 0;}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(g) for g in got]
    exp = [ctypes.sizeof(C.SceneDesc), C.SceneDesc.dx.offset, C.SceneDesc.gravity.offset, C.SceneDesc.dt.offset,
           ctypes.sizeof(C.Material), C.Material.density.offset, C.Material.viscosity.offset,
           ctypes.sizeof(C.Metrics), C.Metrics.p2g_block.offset, C.Metrics.g2p_ms.offset,
           ctypes.sizeof(C.CreateOptions), C.CreateOptions.max_tiles.offset]
    assert got == exp


def test_header_compiles_as_c_and_cxx(tmp_path):
    for comp, ext in (("gcc", "c"), ("g++", "cpp")):
        f = tmp_path / f"h.{ext}"
        f.write_text('#include "pgmpm.h"\nint main(void){ return PGMPM_ABI_VERSION == 5 ? 0 : 1; }\n')
        subprocess.run([comp, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(f), "-o",
                        str(tmp_path / f"h_{ext}")], check=True)


def test_errors_without_gpu_are_reported_not_raised(built_lib):
    """On a machine without a GPU, create() fails with a status and message."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("machine has a GPU")
    except Exception:
        pass
    from physgrad_b200 import _capi as C
    from physgrad_b200.solver import Scene, Simulator, createElasticMaterial

    with pytest.raises(C.PGMPMError) as ei:
        Simulator([Scene()], [10], [createElasticMaterial(1000, 1e4, 0.3)])
    assert ei.value.code in (C.PGMPM_ERR_CUDA, C.PGMPM_ERR_ARG)
    assert "device" in str(ei.value).lower() or "cuda" in str(ei.value).lower()


def test_argument_validation_without_gpu(built_lib):
    from physgrad_b200 import _capi as C

    L = C.lib()
    h = ctypes.c_void_p()
    assert L.pgmpm_create(None, 0, None, None, 0, 0, ctypes.byref(h)) == C.PGMPM_ERR_ARG
    assert b"scene" in L.pgmpm_last_error()
    assert L.pgmpm_step(None, 1, None) == C.PGMPM_ERR_ARG
    assert L.pgmpm_radix_sort_pairs(None, None, None, None, 10, 8, None) == C.PGMPM_ERR_ARG
    assert L.pgmpm_abi_version() == 5
    # sparse grids: one MLS scene, at most 4091 nodes per axis (refused before any device work)
    sd = (C.SceneDesc * 2)()
    for d in sd:
        d.n[0] = d.n[1] = d.n[2] = 64
        d.dx, d.dt = 1.0 / 64, 1e-4
    cn = (ctypes.c_int64 * 2)(100, 100)
    md = (C.Material * 1)()
    md[0].type, md[0].model, md[0].youngs_modulus, md[0].poisson_ratio, md[0].density = 0, 0, 1e4, 0.3, 1000.0
    opt = C.CreateOptions(1, 0, 0)
    assert L.pgmpm_create_ex(sd, 2, cn, md, 1, 0, ctypes.byref(opt), ctypes.byref(h)) == C.PGMPM_ERR_UNSUPPORTED
    sd[0].n[0] = 4096
    assert L.pgmpm_create_ex(sd, 1, cn, md, 1, 0, ctypes.byref(opt), ctypes.byref(h)) == C.PGMPM_ERR_ARG
    assert b"nodes per axis" in L.pgmpm_last_error()


def test_workloads_are_seeded_and_shaped():
    from physgrad_b200 import workloads as W

    s1, c1, m1, st1, meta1 = W.config1(seed=0)
    s1b, _, _, st1b, _ = W.config1(seed=0)
    assert np.array_equal(st1["x"], st1b["x"])
    assert st1["x"].shape == (32768, 3) and c1 == [32768] and s1[0].n == (64, 64, 64)
    assert st1["x"].min() >= 0.3 and st1["x"].max() <= 0.6
    sc, counts, mats, st, meta = W.config4(seed=0)
    assert len(sc) == 64 and len(counts) == 64 and len(mats) == 64
    assert min(counts) >= 4096 and max(counts) <= 262144
    assert all(s.n[0] == (32 if c < 16384 else 64 if c < 131072 else 128) for s, c in zip(sc, counts))
    assert st["x"].shape[0] == sum(counts)
    assert np.array_equal(np.unique(st["mat"]), np.arange(64))


def test_vtk_writer_round_trip(built_lib, read_vtk, tmp_path):
    """pgmpm_vtk_write_particles (host arrays, no GPU): points, one vertex per
    particle, velocity, J = det F and material ids read back exactly."""
    import numpy as np

    from physgrad_b200 import _capi as C

    L = C.lib()
    rng = np.random.default_rng(0)
    n = 37
    x = rng.random((n, 3), dtype=np.float32)
    v = rng.standard_normal((n, 3)).astype(np.float32)
    F = (np.eye(3) + 0.1 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    mat = (np.arange(n) % 3).astype(np.int32)
    path = str(tmp_path / "p.vtk")
    ptr = lambda a: a.ctypes.data
    assert L.pgmpm_vtk_write_particles(path.encode(), n, ptr(x), ptr(v), ptr(F), ptr(mat), 0.25) == 0
    r = read_vtk(path)
    assert "t = 0.25" in r["header"]
    assert np.array_equal(r["x"], x) and np.array_equal(r["velocity"], v) and np.array_equal(r["material"], mat)
    assert np.array_equal(r["vertices"], np.stack([np.ones(n, np.int32), np.arange(n, dtype=np.int32)], 1))
    assert np.allclose(r["J"], np.linalg.det(F.astype(np.float64)), rtol=1e-5, atol=1e-6)
    # positions only; a bad path is an argument error with a message
    assert L.pgmpm_vtk_write_particles(path.encode(), n, ptr(x), None, None, None, 0.0) == 0
    r = read_vtk(path)
    assert r["velocity"] is None and r["J"] is None and np.array_equal(r["x"], x)
    assert L.pgmpm_vtk_write_particles(str(tmp_path / "no" / "dir.vtk").encode(), n, ptr(x), None, None, None,
                                       0.0) == C.PGMPM_ERR_ARG
    assert b"cannot open" in L.pgmpm_last_error()
