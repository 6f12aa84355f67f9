"""ctypes binding of the CPU oracle (oracle/build/liboracle.so).

Test infrastructure only: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _host_tag():
    """The oracle is compiled with -march=native, so each host CPU gets its own build."""
    import hashlib
    import platform

    info = platform.machine()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.startswith("flags"):
                    break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:10]


LIB_PATH = os.path.join(HERE, "build", f"liboracle-{_host_tag()}.so")

LR91, TT06 = 0, 1
FE, RL, BE, GRL1, GRL2 = 0, 1, 2, 3, 4
PC_NONE, PC_JACOBI, PC_BJACOBI = 0, 1, 2
STIM_NONE, STIM_SIMPLE, STIM_REGULAR = 0, 1, 2


class Stimulus(C.Structure):
    _fields_ = [("kind", C.c_int), ("magnitude", C.c_double), ("duration", C.c_double),
                ("start", C.c_double), ("period", C.c_double), ("stop", C.c_double)]


def simple(magnitude, duration, start=0.0):
    return Stimulus(STIM_SIMPLE, magnitude, duration, start, 0.0, 0.0)


def regular(magnitude, duration, period, start=0.0, stop=1.7976931348623157e308):
    return Stimulus(STIM_REGULAR, magnitude, duration, start, period, stop)


class Config(C.Structure):
    _fields_ = [("model", C.c_int), ("ode_method", C.c_int), ("dt_ode", C.c_double),
                ("dt_pde", C.c_double), ("am", C.c_double), ("cm", C.c_double),
                ("pc", C.c_int), ("use_abs_tol", C.c_int), ("tol", C.c_double),
                ("mass_lumping", C.c_int), ("max_iterations", C.c_int), ("solver", C.c_int),
                ("svi", C.c_int)]


class CableConfig(C.Structure):
    _fields_ = [("model", C.c_int), ("n_nodes", C.c_int), ("h", C.c_double), ("sigma", C.c_double),
                ("am", C.c_double), ("cm", C.c_double), ("dt", C.c_double), ("n_steps", C.c_int),
                ("n_regions", C.c_int), ("n_stim", C.c_int), ("stim_mag", C.c_double),
                ("stim_dur", C.c_double), ("rtol", C.c_double), ("max_iterations", C.c_int),
                ("checkpoint_every", C.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", HERE, f"OUT={LIB_PATH}"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.orc_num_states.restype = C.c_int
        L.orc_num_params.restype = C.c_int
        L.orc_stimulus_value.restype = C.c_double
        L.orc_stimulus_value.argtypes = [C.POINTER(Stimulus), C.c_double]
        L.orc_cell_compute.restype = C.c_int
        L.orc_cell_compute.argtypes = [C.c_int, C.c_int, dp, dp, C.POINTER(Stimulus), C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_double, dp, C.c_int]
        L.orc_cell_compute_except_voltage.restype = C.c_double
        L.orc_cell_compute_except_voltage.argtypes = [C.c_int, C.c_int, dp, dp, C.POINTER(Stimulus),
                                                      C.c_double, C.c_double, C.c_double, C.c_double,
                                                      C.c_double]
        L.orc_cell_iionic.restype = C.c_double
        L.orc_cell_iionic.argtypes = [C.c_int, dp, dp, C.c_double]
        L.orc_slab_mesh.restype = C.c_int
        L.orc_slab_mesh.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    ip, ip, ip, dp, ip]
        L.orc_tissue_create.restype = C.c_void_p
        L.orc_tissue_create.argtypes = [C.POINTER(Config), C.c_int, C.c_int, dp, C.c_int, ip, dp,
                                        ip, C.POINTER(Stimulus), C.c_int, ip, dp, C.c_int, dp]
        L.orc_tissue_destroy.argtypes = [C.c_void_p]
        L.orc_tissue_step.restype = C.c_int
        L.orc_tissue_step.argtypes = [C.c_void_p, C.c_int, ip]
        L.orc_tissue_time.restype = C.c_double
        L.orc_tissue_time.argtypes = [C.c_void_p]
        L.orc_tissue_get_voltage.argtypes = [C.c_void_p, dp]
        L.orc_tissue_get_states.argtypes = [C.c_void_p, dp]
        L.orc_tissue_get_caches.argtypes = [C.c_void_p, dp, dp]
        L.orc_tissue_matrix.restype = C.c_int
        L.orc_tissue_matrix.argtypes = [C.c_void_p, C.c_int, ip, ip, dp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_tissue_set_bidomain.restype = C.c_int
        L.orc_tissue_set_bidomain.argtypes = [C.c_void_p, dp, C.c_int, ip, dp, dp, ip, C.c_int]
        L.orc_tissue_get_extracellular.argtypes = [C.c_void_p, dp]
        L.orc_cable_run.restype = C.c_int
        L.orc_cable_run.argtypes = [C.POINTER(CableConfig), dp, ip, C.c_int, dp, dp, dp, dp]
        L.orc_cable_tangent_gradient.restype = C.c_int
        L.orc_cable_tangent_gradient.argtypes = [C.POINTER(CableConfig), dp, ip, C.c_int, dp, dp, C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


def num_states(model):
    return lib().orc_num_states(model)


def initial_states(model):
    y = np.zeros(num_states(model))
    lib().orc_initial_states(model, _dp(y))
    return y


def cell_compute(model, method, y, t0, t1, dt, tsamp=0.0, stim=None, params=None, cm=1.0):
    """Returns the (n_samples, n_states) trajectory; y is updated in place."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = y.size
    ts = max(tsamp, dt)
    max_s = int((t1 - t0) / ts + 2.5)
    out = np.zeros((max_s, n))
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    ns = lib().orc_cell_compute(model, method, _dp(y), _dp(p), C.byref(stim) if stim else None, cm,
                                t0, t1, dt, tsamp, _dp(out), max_s)
    return out[:ns], y


def cell_except_voltage(model, method, y, t0, t1, dt, stim=None, am=0.0, params=None, cm=1.0):
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    return lib().orc_cell_compute_except_voltage(model, method, _dp(y), _dp(p),
                                                 C.byref(stim) if stim else None, am, cm, t0, t1, dt)


def cell_iionic(model, y, params=None, cm=1.0):
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    return lib().orc_cell_iionic(model, _dp(np.ascontiguousarray(y, dtype=np.float64)), _dp(p), cm)


def slab_mesh(dim, h, width, height=0.0, depth=0.0):
    nn, ne = C.c_int(), C.c_int()
    grid = np.zeros(3, dtype=np.int32)
    rc = lib().orc_slab_mesh(dim, h, width, height, depth, C.byref(nn), C.byref(ne), _ip(grid), None, None)
    if rc != 0:
        raise ValueError("Space step does not divide the size of the mesh")
    xyz = np.zeros((nn.value, 3))
    conn = np.zeros((ne.value, dim + 1), dtype=np.int32)
    lib().orc_slab_mesh(dim, h, width, height, depth, C.byref(nn), C.byref(ne), _ip(grid), _dp(xyz), _ip(conn))
    return xyz, conn, grid


class Tissue:
    """Oracle monodomain tissue (MonodomainProblem restatement)."""

    def __init__(self, cfg: Config, dim, xyz, conn, sigma, stim_id=None, stims=(), param_id=None,
                 param_table=None, init_states=None):
        L = lib()
        self.n = xyz.shape[0]
        self.dim = dim
        self.ns = num_states(cfg.model)
        self._keep = []
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        sid = None if stim_id is None else np.ascontiguousarray(stim_id, dtype=np.int32)
        st = (Stimulus * max(1, len(stims)))(*stims)
        pid = None if param_id is None else np.ascontiguousarray(param_id, dtype=np.int32)
        pt = None if param_table is None else np.ascontiguousarray(param_table, dtype=np.float64)
        npset = 0 if pt is None else pt.shape[0]
        ini = None if init_states is None else np.ascontiguousarray(init_states, dtype=np.float64)
        self.cfg = cfg
        self.h = L.orc_tissue_create(C.byref(cfg), dim, self.n, _dp(xyz), conn.shape[0], _ip(conn),
                                     _dp(sigma), _ip(sid), st, len(stims), _ip(pid), _dp(pt), npset,
                                     _dp(ini))
        if not self.h:
            raise RuntimeError("orc_tissue_create failed")

    def step(self, n=1):
        its = np.zeros(n, dtype=np.int32)
        rc = lib().orc_tissue_step(self.h, n, _ip(its))
        if rc != 0:
            raise RuntimeError(f"oracle CG failed with code {rc}")
        return its

    @property
    def time(self):
        return lib().orc_tissue_time(self.h)

    def voltage(self):
        v = np.zeros(self.n)
        lib().orc_tissue_get_voltage(self.h, _dp(v))
        return v

    def set_bidomain(self, xyz, conn, sigma_i, sigma_e, fixed=None):
        """orc_tissue_set_bidomain: (V, phi_e) unknowns; fixed phi_e = 0 at `fixed` nodes, else the
        null space of constant phi_e."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        si = np.ascontiguousarray(sigma_i, dtype=np.float64)
        se = np.ascontiguousarray(sigma_e, dtype=np.float64)
        fx = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.int32)
        rc = lib().orc_tissue_set_bidomain(self.h, _dp(xyz), conn.shape[0], _ip(conn), _dp(si), _dp(se), _ip(fx),
                                           0 if fx is None else fx.size)
        if rc != 0:
            raise RuntimeError(f"orc_tissue_set_bidomain failed with code {rc}")

    def extracellular(self):
        phi = np.zeros(self.n)
        lib().orc_tissue_get_extracellular(self.h, _dp(phi))
        return phi

    def states(self):
        s = np.zeros((self.n, self.ns))
        lib().orc_tissue_get_states(self.h, _dp(s))
        return s

    def caches(self):
        a, b = np.zeros(self.n), np.zeros(self.n)
        lib().orc_tissue_get_caches(self.h, _dp(a), _dp(b))
        return a, b

    def matrix(self, which=0):
        nnz = lib().orc_tissue_matrix(self.h, which, None, None, None)
        rp = np.zeros(self.n + 1, dtype=np.int32)
        cols = np.zeros(nnz, dtype=np.int32)
        vals = np.zeros(nnz)
        lib().orc_tissue_matrix(self.h, which, _ip(rp), _ip(cols), _dp(vals))
        return rp, cols, vals

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_tissue_destroy(self.h)
            self.h = None


def cable_run(cfg: CableConfig, params, probes, targets=None, traces=False, gradient=False):
    """orc_cable_run: returns dict(loss, traces, grad) (None where not asked)."""
    params = np.ascontiguousarray(params, dtype=np.float64)
    probes = np.ascontiguousarray(probes, dtype=np.int32)
    tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.float64)
    loss = C.c_double(0.0)
    tr = np.zeros((cfg.n_steps, probes.size)) if traces else None
    g = np.zeros_like(params) if gradient else None
    rc = lib().orc_cable_run(C.byref(cfg), _dp(params), _ip(probes), probes.size, _dp(tg),
                             C.byref(loss) if tg is not None else None, _dp(tr), _dp(g))
    if rc != 0:
        raise RuntimeError(f"orc_cable_run failed with code {rc}")
    return dict(loss=loss.value if tg is not None else None, traces=tr, grad=g)


def cable_tangent_gradient(cfg: CableConfig, params, probes, targets, threads=None):
    """orc_cable_tangent_gradient: dL/dparams by forward mode, one tangent run per parameter."""
    params = np.ascontiguousarray(params, dtype=np.float64)
    probes = np.ascontiguousarray(probes, dtype=np.int32)
    tg = np.ascontiguousarray(targets, dtype=np.float64)
    g = np.zeros_like(params)
    rc = lib().orc_cable_tangent_gradient(C.byref(cfg), _dp(params), _ip(probes), probes.size, _dp(tg), _dp(g),
                                          int(threads or os.cpu_count() or 1))
    if rc != 0:
        raise RuntimeError(f"orc_cable_tangent_gradient failed with code {rc}")
    return g
