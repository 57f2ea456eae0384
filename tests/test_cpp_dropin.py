"""The C++ drop-in header (include/physgrad_b200/mpm_solver.h) compiles as the
reference's src/mpm_solver.h users would use it, links against libpgmpm.so,
and (on a GPU) runs."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "drop_in_solver.cpp")


def _build(built_lib, out):
    libdir = os.path.dirname(built_lib)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o",
                    out, "-L", libdir, "-lpgmpm", f"-Wl,-rpath,{libdir}"], check=True)


def test_dropin_header_compiles_and_links(built_lib, tmp_path):
    _build(built_lib, str(tmp_path / "drop_in"))


@pytest.mark.gpu
def test_dropin_header_runs_on_gpu(gpu, built_lib, tmp_path):
    exe = str(tmp_path / "drop_in")
    _build(built_lib, exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert '"steps": 15' in r.stdout


@pytest.mark.gpu
def test_dropin_run_writes_vtk_frames(gpu, built_lib, read_vtk, tmp_path):
    """enable_output: run() writes output_directory/frame_NNNNN.vtk whenever a
    step crosses a multiple of output_frequency (1e-3 s at 2.5e-4 s: 3 or 4
    frames, depending on float rounding of the time, as in the reference)."""
    exe = str(tmp_path / "drop_in")
    _build(built_lib, exe)
    out = tmp_path / "frames"
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert '"output_steps": 10' in r.stdout
    frames = sorted(os.listdir(out))
    assert 3 <= len(frames) <= 4 and frames[0] == "frame_00000.vtk", frames
    v = read_vtk(str(out / frames[-1]))
    assert v["x"].shape == (512, 3) and v["velocity"] is not None
