"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the reference's
own CPU solver built from its sources (oracle/_ref/libref_mpm.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_mpm.so")
REF_DIFF_PATH = os.path.join(HERE, "_ref", "libref_diff.so")
REF_COUPLING_PATH = os.path.join(HERE, "_ref", "libref_coupling.so")
REF_FSI_PATH = os.path.join(HERE, "_ref", "libref_fsi.so")

MLS, REF_COMPAT = 0, 1
BC_NONE, BC_STICKY, BC_SLIP, BC_SEPARATE = 0, 1, 2, 3
FIXED_COROTATED, NEO_HOOKEAN, EOS_FLUID = 0, 1, 2


class Scene(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32 * 3),
        ("physics", ctypes.c_int32),
        ("boundary", ctypes.c_int32),
        ("bthick", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
        ("pad1", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("origin", ctypes.c_double * 3),
        ("dt", ctypes.c_double),
        ("gravity", ctypes.c_double * 3),
    ]


class Material(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("E", ctypes.c_double),
        ("nu", ctypes.c_double),
        ("yield_stress", ctypes.c_double),
        ("viscosity", ctypes.c_double),
    ]


def reference_src() -> str | None:
    """The reference's ``src`` directory, or None when it is not on this machine.

    Taken from the environment variable PGMPM_REFERENCE_SRC, else from the
    ``reference_path`` field of the repository's BASELINE.json (its ``src``
    subdirectory).  The GPU hosts have no reference tree and use the files
    built beforehand into oracle/_ref."""
    env = os.environ.get("PGMPM_REFERENCE_SRC")
    if env:
        return env if os.path.isdir(env) else None
    meta = os.path.join(os.path.dirname(HERE), "BASELINE.json")
    try:
        import json

        with open(meta) as f:
            root = json.load(f).get("reference_path")
    except (OSError, ValueError):
        return None
    if not root:
        return None
    src = os.path.join(root, "src")
    return src if os.path.isdir(src) else None


def build(with_ref: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    targets = ["all"]
    src = reference_src() if with_ref else None
    if src:
        targets += ["ref", "REF_SRC=" + src]
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_ref=False)
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_run.argtypes = [ctypes.c_int, ctypes.POINTER(Scene), ctypes.POINTER(Material), ctypes.c_int,
                                 ctypes.c_int64, dp, dp, dp, dp, dp, dp, ctypes.c_void_p, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_keys.argtypes = [ctypes.POINTER(Scene), ctypes.c_int64, ctypes.c_void_p, ctypes.c_uint32,
                                  ctypes.c_void_p]
        L.oracle_stable_sort.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
        L.oracle_adjoint.argtypes = [ctypes.POINTER(Scene), ctypes.POINTER(Material), ctypes.c_int,
                                     ctypes.c_int64, dp, dp, dp, dp, dp, dp, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, dp, dp, dp, dp, dp]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_PATH)
        fp = ctypes.c_void_p
        R.ref_mpm_run.argtypes = [ctypes.c_int64, fp, fp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, fp, fp, fp, fp]
        _ref = R
    return _ref


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_scene(n, dx, dt, gravity=(0.0, -9.8, 0.0), origin=(0.0, 0.0, 0.0), physics=MLS,
               boundary=BC_STICKY, bthick=3) -> Scene:
    s = Scene()
    for a in range(3):
        s.n[a] = int(n[a] if hasattr(n, "__len__") else n)
        s.origin[a] = float(origin[a])
        s.gravity[a] = float(gravity[a])
    s.physics = physics
    s.boundary = boundary
    s.bthick = bthick
    s.dx = float(dx)
    s.dt = float(dt)
    return s


def make_materials(mats):
    """Tuples (model, E, nu[, yield_stress[, viscosity]]); model 0 fixed-
    corotated, 1 neo-Hookean, 2 EOS fluid (K in E), 3 von Mises
    (neo-Hookean predictor, yield_stress on the Cauchy stress)."""
    arr = (Material * len(mats))()
    for i, m in enumerate(mats):
        model, E, nu = m[:3]
        arr[i].model = int(model)
        arr[i].E = float(E)
        arr[i].nu = float(nu)
        arr[i].yield_stress = float(m[3]) if len(m) > 3 else 0.0
        arr[i].viscosity = float(m[4]) if len(m) > 4 else 0.0
    return arr


def run(scene: Scene, mats, state: dict, steps: int, prec: int = 64, nthreads: int = 0, want_grid=False):
    """Advance a copy of ``state`` (dict x,v,C,F,m,V0[,mat]) by ``steps`` steps."""
    n = state["x"].shape[0]
    x = np.ascontiguousarray(state["x"], dtype=np.float64).copy()
    v = np.ascontiguousarray(state["v"], dtype=np.float64).copy()
    C = np.ascontiguousarray(state["C"], dtype=np.float64).reshape(n, 9).copy()
    F = np.ascontiguousarray(state["F"], dtype=np.float64).reshape(n, 9).copy()
    m = np.ascontiguousarray(state["m"], dtype=np.float64)
    V0 = np.ascontiguousarray(state["V0"], dtype=np.float64)
    mat = state.get("mat")
    mat_p = None
    if mat is not None:
        mat = np.ascontiguousarray(mat, dtype=np.int32)
        mat_p = mat.ctypes.data
    nodes = scene.n[0] * scene.n[1] * scene.n[2]
    gm = np.zeros(nodes) if want_grid else None
    gv = np.zeros((nodes, 3)) if want_grid else None
    rc = lib().oracle_run(prec, ctypes.byref(scene), mats, len(mats), n, _dp(x), _dp(v), _dp(C), _dp(F),
                          _dp(m), _dp(V0), mat_p, steps, nthreads,
                          gm.ctypes.data if want_grid else None, gv.ctypes.data if want_grid else None)
    if rc != 0:
        raise RuntimeError(f"oracle_run failed: {rc}")
    out = {"x": x, "v": v, "C": C.reshape(n, 3, 3), "F": F.reshape(n, 3, 3)}
    if want_grid:
        out["grid_m"] = gm
        out["grid_v"] = gv
    return out


def keys(scene: Scene, x: np.ndarray, cell_base: int = 0) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.shape[0], dtype=np.uint32)
    lib().oracle_keys(ctypes.byref(scene), x.shape[0], x.ctypes.data, cell_base, out.ctypes.data)
    return out


def stable_sort(keys_in: np.ndarray, vals: np.ndarray | None = None):
    k = np.ascontiguousarray(keys_in, dtype=np.uint32)
    n = k.shape[0]
    ok = np.empty(n, dtype=np.uint32)
    ov = np.empty(n, dtype=np.uint32)
    vp = None
    if vals is not None:
        vals = np.ascontiguousarray(vals, dtype=np.uint32)
        vp = vals.ctypes.data
    lib().oracle_stable_sort(n, k.ctypes.data, vp, ok.ctypes.data, ov.ctypes.data)
    return ok, ov


def adjoint(scene: Scene, mats, state: dict, steps: int, grads_out: dict, nthreads: int = 0):
    """dL/d(initial state, E) given dL/d(final state) (FP64)."""
    n = state["x"].shape[0]
    f = lambda a, k: np.ascontiguousarray(a, dtype=np.float64).reshape(n, k).copy()
    x, v, C, F = f(state["x"], 3), f(state["v"], 3), f(state["C"], 9), f(state["F"], 9)
    m = np.ascontiguousarray(state["m"], dtype=np.float64)
    V0 = np.ascontiguousarray(state["V0"], dtype=np.float64)
    mat = state.get("mat")
    mat_p = None
    if mat is not None:
        mat = np.ascontiguousarray(mat, dtype=np.int32)
        mat_p = mat.ctypes.data
    gx, gv = f(grads_out.get("x", np.zeros((n, 3))), 3), f(grads_out.get("v", np.zeros((n, 3))), 3)
    gC, gF = f(grads_out.get("C", np.zeros((n, 9))), 9), f(grads_out.get("F", np.zeros((n, 9))), 9)
    gE = np.zeros(len(mats))
    rc = lib().oracle_adjoint(ctypes.byref(scene), mats, len(mats), n, _dp(x), _dp(v), _dp(C), _dp(F), _dp(m),
                              _dp(V0), mat_p, steps, nthreads, _dp(gx), _dp(gv), _dp(gC), _dp(gF), _dp(gE))
    if rc != 0:
        raise RuntimeError(f"oracle_adjoint failed: {rc}")
    return {"x": gx, "v": gv, "C": gC.reshape(n, 3, 3), "F": gF.reshape(n, 3, 3), "E": gE}


def com_loss(x, target=(0.5, 0.3, 0.5)) -> float:
    """||mean(x) - target||^2: the centre-of-mass loss of the differentiable
    configuration (equal particle masses, so the mean is the centre of mass)."""
    c = np.asarray(x, dtype=np.float64).mean(0) - np.asarray(target, dtype=np.float64)
    return float((c * c).sum())


def fd_v0_com(scene: Scene, mats, state: dict, steps: int, coords, eps: float = 1e-3, target=(0.5, 0.3, 0.5),
              workers: int = 0):
    """FP64 central differences of com_loss after ``steps`` steps with respect
    to the initial velocity coordinates ``coords`` ((particle, axis) pairs):
    (L(v0 + eps e) - L(v0 - eps e)) / (2 eps).  The 2 len(coords) forward runs
    go to concurrent host threads, one oracle worker each."""
    import concurrent.futures

    def one(c, sign):
        st = dict(state)
        v = np.array(state["v"], dtype=np.float64, copy=True)
        v[c[0], c[1]] += sign * eps
        st["v"] = v
        return com_loss(run(scene, mats, st, steps, prec=64, nthreads=1)["x"], target)

    jobs = [(c, s) for c in coords for s in (1.0, -1.0)]
    nw = workers or min(len(jobs), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(max_workers=nw) as ex:
        vals = list(ex.map(lambda a: one(*a), jobs))
    return np.array([(vals[2 * i] - vals[2 * i + 1]) / (2 * eps) for i in range(len(coords))])


def ref_diff_available() -> bool:
    return os.path.exists(REF_DIFF_PATH)


def ref_diff_run(x, v, m, n, dx, dt, steps):
    """The reference's own DifferentiableMPMSystem<float> (oracle/_ref): the
    forward with gradient recording on (simulationStep(dt), default gravity),
    then computeGradients().  Returns its final positions and the particle
    velocity and position gradients it reports."""
    R = ctypes.CDLL(REF_DIFF_PATH)
    fp = ctypes.c_void_p
    R.ref_diff_run.argtypes = [ctypes.c_int64, fp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                               ctypes.c_float, ctypes.c_int, fp, fp, fp]
    x = np.ascontiguousarray(x, dtype=np.float32)
    v = np.ascontiguousarray(v, dtype=np.float32)
    m = np.ascontiguousarray(m, dtype=np.float32)
    N = x.shape[0]
    xo, gv, gx = np.empty_like(x), np.empty_like(x), np.empty_like(x)
    rc = R.ref_diff_run(N, x.ctypes.data, v.ctypes.data, m.ctypes.data, n[0], n[1], n[2], dx, dt, steps,
                        xo.ctypes.data, gv.ctypes.data, gx.ctypes.data)
    if rc != 0:
        raise RuntimeError("ref_diff_run failed")
    return {"x": xo, "grad_v": gv, "grad_x": gx}


def ref_run(x, v, m, vol, n, dx, dt, gravity, steps, origin=(0.0, 0.0, 0.0), want_grid=False):
    """Run the reference's own MPMSolver<float,64> (oracle/_ref) in float."""
    R = ref_lib()
    x = np.ascontiguousarray(x, dtype=np.float32)
    v = np.ascontiguousarray(v, dtype=np.float32)
    m = np.ascontiguousarray(m, dtype=np.float32)
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    N = x.shape[0]
    xo = np.empty_like(x)
    vo = np.empty_like(v)
    nodes = n[0] * n[1] * n[2]
    gm = np.empty(nodes, dtype=np.float32) if want_grid else None
    gv = np.empty((nodes, 3), dtype=np.float32) if want_grid else None
    rc = R.ref_mpm_run(N, x.ctypes.data, v.ctypes.data, m.ctypes.data, vol.ctypes.data, n[0], n[1], n[2], dx,
                       origin[0], origin[1], origin[2], dt, gravity[0], gravity[1], gravity[2], steps,
                       xo.ctypes.data, vo.ctypes.data, gm.ctypes.data if want_grid else None,
                       gv.ctypes.data if want_grid else None)
    if rc != 0:
        raise RuntimeError("ref_mpm_run failed")
    out = {"x": xo, "v": vo}
    if want_grid:
        out["grid_m"] = gm
        out["grid_v"] = gv
    return out


# ------------------------------------------------------------ consumers
def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _coupling_call(fn, sph_x, sph_v, mpm_x, mpm_v, stiffness, damping, friction, radius, two_way):
    fp = ctypes.c_void_p
    fn.argtypes = [ctypes.c_int64, fp, fp, ctypes.c_int64, fp, fp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                   ctypes.c_float, ctypes.c_int, fp, fp, fp, fp]
    sx, sv, mx, mv = _f32(sph_x), _f32(sph_v), _f32(mpm_x), _f32(mpm_v)
    fs = np.empty_like(sx)
    fm = np.empty_like(mx)
    npairs = ctypes.c_int64()
    e = ctypes.c_float()
    rc = fn(sx.shape[0], sx.ctypes.data, sv.ctypes.data, mx.shape[0], mx.ctypes.data, mv.ctypes.data, stiffness,
            damping, friction, radius, int(two_way), fs.ctypes.data, fm.ctypes.data, ctypes.byref(npairs),
            ctypes.byref(e))
    if rc != 0:
        raise RuntimeError(f"coupling call failed: {rc}")
    return {"sph_force": fs, "mpm_force": fm, "n_pairs": npairs.value, "energy": e.value}


def sph_coupling(sph_x, sph_v, mpm_x, mpm_v, stiffness=1e5, damping=1e3, friction=0.3, radius=0.15, two_way=True):
    """The oracle's restatement of the SPH-MPM contact coupling (float, the
    reference's pair order): SPH forces (from zero), MPM solid-force sums,
    pair count, coupling energy."""
    return _coupling_call(lib().oracle_sph_coupling, sph_x, sph_v, mpm_x, mpm_v, stiffness, damping, friction,
                          radius, two_way)


def ref_coupling_available() -> bool:
    return os.path.exists(REF_COUPLING_PATH)


def ref_sph_coupling(sph_x, sph_v, mpm_x, mpm_v, stiffness=1e5, damping=1e3, friction=0.3, radius=0.15,
                     two_way=True):
    """The same through the reference's own SPHMPMCouplingSystem (oracle/_ref)."""
    return _coupling_call(ctypes.CDLL(REF_COUPLING_PATH).ref_sph_coupling, sph_x, sph_v, mpm_x, mpm_v, stiffness,
                          damping, friction, radius, two_way)


def kinetic_energy(v, m, mat=None, n_materials=1):
    """Kinetic energy per material id (FP64), the FSI energy monitor's sum."""
    L = lib()
    L.oracle_kinetic_energy.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_void_p]
    vv = np.ascontiguousarray(v, dtype=np.float64)
    mm = np.ascontiguousarray(m, dtype=np.float64)
    mt = None if mat is None else np.ascontiguousarray(mat, dtype=np.int32)
    out = np.zeros(n_materials)
    rc = L.oracle_kinetic_energy(vv.shape[0], vv.ctypes.data, mm.ctypes.data, None if mt is None else mt.ctypes.data,
                                 n_materials, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle_kinetic_energy failed: {rc}")
    return out


def ref_fsi_available() -> bool:
    return os.path.exists(REF_FSI_PATH)


def ref_fsi_energy(v_fluid, m_fluid, v_solid, m_solid) -> float:
    """FSISimulationManager's computeTotalEnergy of a fluid and a solid set
    (the reference's own code, oracle/_ref)."""
    R = ctypes.CDLL(REF_FSI_PATH)
    fp = ctypes.c_void_p
    R.ref_fsi_energy.argtypes = [ctypes.c_int64, fp, fp, ctypes.c_int64, fp, fp, fp]
    vf, mf, vs, ms = _f32(v_fluid), _f32(m_fluid), _f32(v_solid), _f32(m_solid)
    e = ctypes.c_float()
    rc = R.ref_fsi_energy(vf.shape[0], vf.ctypes.data, mf.ctypes.data, vs.shape[0], vs.ctypes.data, ms.ctypes.data,
                          ctypes.byref(e))
    if rc != 0:
        raise RuntimeError(f"ref_fsi_energy failed: {rc}")
    return e.value
