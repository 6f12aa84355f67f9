"""ctypes binding of libchastegpu.so (include/chaste_gpu.h).

The library is the only compute path: there is no CPU fallback.  Importing
works without a GPU (so the ABI can be inspected), but creating a tissue
raises :class:`ChasteGpuError` when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libchastegpu.so")

CG_OK = 0
CG_ERR_CG_MAXIT, CG_ERR_CG_DIVERGED, CG_ERR_NAN = 3, 4, 5
STATUS_NAMES = {
    0: "CG_OK", 1: "CG_ERR_ARG", 2: "CG_ERR_CUDA", 3: "CG_ERR_CG_MAXIT", 4: "CG_ERR_CG_DIVERGED",
    5: "CG_ERR_NAN", 6: "CG_ERR_STATE_RANGE", 7: "CG_ERR_ORDER", 8: "CG_ERR_TIMEOUT",
    9: "CG_ERR_NOMEM", 10: "CG_ERR_UNSUPPORTED",
}
MODEL_LR91, MODEL_TT06 = 0, 1
ODE_FORWARD_EULER, ODE_RUSH_LARSEN, ODE_BACKWARD_EULER, ODE_GRL1, ODE_GRL2 = 0, 1, 2, 3, 4
PC_NONE, PC_JACOBI, PC_BJACOBI = 0, 1, 2
PRECISION_FP64, PRECISION_MIXED = 0, 1
STIM_NONE, STIM_SIMPLE, STIM_REGULAR = 0, 1, 2
SOLVER_MONODOMAIN, SOLVER_OPERATOR_SPLITTING = 0, 1
INNER_PC_LINE, INNER_PC_JACOBI = 0, 1
BATCH_PER_BEAT, BATCH_PERSISTENT = 0, 1


class ChasteGpuError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        msg = f"{where}: {name}"
        try:
            msg += f" ({lib().cg_status_string(status).decode()})"
        except Exception:  # noqa: BLE001 - message decoration only
            pass
        super().__init__(msg)


class Config(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("ode_method", C.c_int), ("ode_time_step", C.c_double),
        ("pde_time_step", C.c_double), ("surface_area_to_volume_ratio", C.c_double),
        ("capacitance", C.c_double), ("ksp_preconditioner", C.c_int),
        ("use_absolute_tolerance", C.c_int), ("ksp_tolerance", C.c_double),
        ("use_mass_lumping", C.c_int), ("max_iterations", C.c_int), ("precision", C.c_int),
        ("device", C.c_int), ("check_state_ranges", C.c_int), ("activation_threshold", C.c_double),
        ("solver", C.c_int), ("use_state_variable_interpolation", C.c_int),
        ("mixed_inner_preconditioner", C.c_int),
    ]


class Stimulus(C.Structure):
    _fields_ = [("kind", C.c_int), ("magnitude", C.c_double), ("duration", C.c_double),
                ("start", C.c_double), ("period", C.c_double), ("stop", C.c_double)]


class Stats(C.Structure):
    _fields_ = [
        ("steps", C.c_longlong), ("time", C.c_double), ("last_cg_iterations", C.c_int),
        ("max_cg_iterations", C.c_int), ("total_cg_iterations", C.c_longlong),
        ("refinement_sweeps", C.c_int), ("operator_kind", C.c_int), ("status_bits", C.c_int),
        ("ms_last_call", C.c_double), ("pipelined_nodes_per_thread", C.c_int), ("cg_blocks", C.c_int),
        ("inner_preconditioner", C.c_int), ("inner_line_segment", C.c_int),
        ("step_graph", C.c_int), ("host_call_graph", C.c_int), ("capture_error", C.c_int),
    ]


class CableConfig(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("n_nodes", C.c_int), ("h", C.c_double), ("conductivity", C.c_double),
        ("surface_area_to_volume_ratio", C.c_double), ("capacitance", C.c_double),
        ("time_step", C.c_double), ("n_steps", C.c_int), ("n_regions", C.c_int),
        ("n_stimulated_nodes", C.c_int), ("stimulus_magnitude", C.c_double),
        ("stimulus_duration", C.c_double), ("ksp_tolerance", C.c_double), ("max_iterations", C.c_int),
        ("checkpoint_every", C.c_int),
    ]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p
# exported symbol -> (restype, argtypes); every name declared in include/chaste_gpu.h
SIGNATURES = {
    "cg_default_config": (None, [C.POINTER(Config)]),
    "cg_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "cg_set_mesh": (C.c_int, [_vp, C.c_int, C.c_int, _dp, C.c_int, _ip, _dp]),
    "cg_set_slab_mesh": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _ip]),
    "cg_set_cells": (C.c_int, [_vp, _dp, _ip, _dp, C.c_int]),
    "cg_set_bidomain_mesh": (C.c_int, [_vp, C.c_int, C.c_int, _dp, C.c_int, _ip, _dp, _dp]),
    "cg_set_fixed_extracellular_nodes": (C.c_int, [_vp, _ip, C.c_int]),
    "cg_get_extracellular_potential": (C.c_int, [_vp, _dp]),
    "cg_set_stimulus": (C.c_int, [_vp, _ip, C.POINTER(Stimulus), C.c_int]),
    "cg_step": (C.c_int, [_vp, C.c_int]),
    "cg_step_host": (C.c_int, [_vp, _dp, C.c_int, _dp, C.c_int]),
    "cg_step_profiled": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "cg_get_voltage": (C.c_int, [_vp, _dp]),
    "cg_set_voltage": (C.c_int, [_vp, _dp]),
    "cg_get_states": (C.c_int, [_vp, _dp]),
    "cg_get_cell_state": (C.c_int, [_vp, C.c_int, _dp]),
    "cg_get_caches": (C.c_int, [_vp, _dp, _dp]),
    "cg_get_activation_times": (C.c_int, [_vp, _dp]),
    "cg_get_stats": (C.c_int, [_vp, C.POINTER(Stats)]),
    "cg_get_iteration_history": (C.c_int, [_vp, C.c_int, _ip]),
    "cg_apply_inner_preconditioner": (C.c_int, [_vp, _dp, _dp]),
    "cg_num_nodes": (C.c_int, [_vp, _ip]),
    "cg_num_states": (C.c_int, [C.c_int, _ip]),
    "cg_slab_mesh": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _ip, _ip, _dp, _ip]),
    "cg_num_params": (C.c_int, [C.c_int, _ip]),
    "cg_snapshot_size": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "cg_snapshot": (C.c_int, [_vp, _vp, C.c_size_t]),
    "cg_restore": (C.c_int, [_vp, _vp, C.c_size_t]),
    "cg_destroy": (C.c_int, [_vp]),
    "cg_status_string": (C.c_char_p, [C.c_int]),
    "cg_batch_create": (C.c_int, [C.c_int, C.c_int, _ip, _dp, C.POINTER(Stimulus), C.c_double, C.c_double,
                                  C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "cg_batch_autotune": (C.c_int, [_vp, C.c_int, _ip]),
    "cg_batch_run": (C.c_int, [_vp, _dp]),
    "cg_batch_launch_shape": (C.c_int, [_vp, _ip, _ip]),
    "cg_batch_set_launch_shape": (C.c_int, [_vp, C.c_int, C.c_int]),
    "cg_batch_results": (C.c_int, [_vp, _dp, _dp, _ip, _ip, C.POINTER(C.c_float), _dp, _dp]),
    "cg_batch_destroy": (C.c_int, [_vp]),
    "cg_batch_set_engine": (C.c_int, [_vp, C.c_int]),
    "cg_batch_engine": (C.c_int, [_vp, _ip]),
    "cg_cable_default_config": (None, [C.POINTER(CableConfig)]),
    "cg_cable_create": (C.c_int, [C.POINTER(CableConfig), _ip, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "cg_cable_forward": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp]),
    "cg_cable_backward": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp]),
    "cg_cable_destroy": (C.c_int, [_vp]),
    "cg_runs_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "cg_runs_add_cell": (C.c_int, [_vp, C.c_int, _dp, C.POINTER(Stimulus), C.c_double, C.c_int, C.c_int, _ip]),
    "cg_runs_add_cable": (C.c_int, [_vp, C.POINTER(CableConfig), _dp, _ip, C.c_int, C.c_int, _ip]),
    "cg_runs_autotune": (C.c_int, [_vp, C.c_int, _ip, _ip]),
    "cg_runs_set_shape": (C.c_int, [_vp, C.c_int, C.c_int]),
    "cg_runs_shape": (C.c_int, [_vp, _ip, _ip]),
    "cg_runs_run": (C.c_int, [_vp, _dp]),
    "cg_runs_result": (C.c_int, [_vp, C.c_int, _dp, _dp, _ip, C.POINTER(C.c_longlong)]),
    "cg_runs_destroy": (C.c_int, [_vp]),
    "cg_selftest_barrier_timeout": (C.c_int, [C.c_int, C.c_double, _ip, _dp]),
    "cg_output_configure": (C.c_int, [_vp, C.c_int, C.c_int, _ip, C.c_int]),
    "cg_output_frames": (C.c_int, [_vp, _ip, _dp]),
    "cg_output_fetch": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "cg_output_activation": (C.c_int, [_vp, C.c_double]),
    "cg_output_get_activation": (C.c_int, [_vp, _dp]),
    "cg_output_cell_properties": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, _dp, _ip, _dp, _dp, _ip]),
    "cg_output_conduction_velocity": (C.c_int, [_vp, C.c_int, _dp, C.c_double, C.c_int, _dp, _ip]),
    "cg_part_create": (C.c_int, [C.POINTER(Config), C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp,
                                 C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "cg_part_rows": (C.c_int, [_vp, _ip, _ip, _ip, _ip]),
    "cg_part_set_cells": (C.c_int, [_vp, _dp, _ip, _dp, C.c_int]),
    "cg_part_set_stimulus": (C.c_int, [_vp, _ip, C.POINTER(Stimulus), C.c_int]),
    "cg_part_ode": (C.c_int, [_vp]),
    "cg_part_halo_pack": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "cg_part_halo_unpack": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "cg_part_cg_phase": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "cg_part_finish_step": (C.c_int, [_vp]),
    "cg_part_get_voltage": (C.c_int, [_vp, _dp]),
    "cg_part_config": (C.c_int, [_vp, C.POINTER(Config)]),
    "cg_part_destroy": (C.c_int, [_vp]),
    "cg_slab_solve_noalloc": (C.c_int, [C.POINTER(Config), C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.c_double, _dp, _vp, _vp, _vp, _ip]),
}

_lib = None


def lib():
    """Load libchastegpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ChasteGpuError(2, f"{LIB_PATH} not built (run chaste_b200.build.build_native())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, where):
    if status != CG_OK:
        raise ChasteGpuError(status, where)


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def iptr(a):
    return None if a is None else a.ctypes.data_as(_ip)


def default_config() -> Config:
    c = Config()
    lib().cg_default_config(C.byref(c))
    return c


def num_states(model):
    n = C.c_int()
    check(lib().cg_num_states(model, C.byref(n)), "cg_num_states")
    return n.value


def num_params(model):
    n = C.c_int()
    check(lib().cg_num_params(model, C.byref(n)), "cg_num_params")
    return n.value


def slab_mesh(dim, h, width, height=0.0, depth=0.0):
    """(xyz, conn) of the regular slab (cg_slab_mesh; host only, no GPU needed)."""
    nn, ne = C.c_int(), C.c_int()
    check(lib().cg_slab_mesh(dim, h, width, height, depth, C.byref(nn), C.byref(ne), None, None), "cg_slab_mesh")
    xyz = np.zeros((nn.value, 3))
    conn = np.zeros((ne.value, dim + 1), dtype=np.int32)
    check(lib().cg_slab_mesh(dim, h, width, height, depth, C.byref(nn), C.byref(ne), dptr(xyz), iptr(conn)),
          "cg_slab_mesh")
    return xyz, conn


def stimulus(kind, magnitude=0.0, duration=0.0, start=0.0, period=0.0, stop=1.7976931348623157e308):
    return Stimulus(kind, magnitude, duration, start, period, stop)


class Tissue:
    """One device-resident monodomain tissue (a cg_ctx)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        h = C.c_void_p()
        check(lib().cg_create(C.byref(cfg), C.byref(h)), "cg_create")
        self.h = h
        self.n = 0
        self.n_states = num_states(cfg.model)

    # -- set-up
    def set_mesh(self, xyz, conn, sigma):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        dim = conn.shape[1] - 1
        sigma = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma, dtype=np.float64),
                                                     (conn.shape[0], dim)))
        check(lib().cg_set_mesh(self.h, xyz.shape[0], dim, dptr(xyz), conn.shape[0], iptr(conn), dptr(sigma)),
              "cg_set_mesh")
        self.n = xyz.shape[0]

    def set_bidomain_mesh(self, xyz, conn, sigma_i, sigma_e):
        """cg_set_bidomain_mesh: the tissue solves for (V, phi_e); sigma_* per element (or broadcast)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        dim = conn.shape[1] - 1
        si, se = (np.ascontiguousarray(np.broadcast_to(np.asarray(s, dtype=np.float64), (conn.shape[0], dim)))
                  for s in (sigma_i, sigma_e))
        check(lib().cg_set_bidomain_mesh(self.h, xyz.shape[0], dim, dptr(xyz), conn.shape[0], iptr(conn), dptr(si),
                                         dptr(se)), "cg_set_bidomain_mesh")
        self.n = xyz.shape[0]

    def fix_extracellular_potential(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        check(lib().cg_set_fixed_extracellular_nodes(self.h, iptr(nodes), nodes.size),
              "cg_set_fixed_extracellular_nodes")

    def extracellular_potential(self):
        phi = np.empty(self.n)
        check(lib().cg_get_extracellular_potential(self.h, dptr(phi)), "cg_get_extracellular_potential")
        return phi

    def set_slab_mesh(self, dim, h, width, height=0.0, depth=0.0, sigma=(1.75, 1.75, 1.75)):
        sig = np.ascontiguousarray(np.asarray(sigma, dtype=np.float64)[:dim])
        n = C.c_int()
        check(lib().cg_set_slab_mesh(self.h, dim, h, width, height, depth, dptr(sig), C.byref(n)),
              "cg_set_slab_mesh")
        self.n = n.value

    def set_cells(self, init_states=None, param_set=None, param_table=None):
        ini = None if init_states is None else np.ascontiguousarray(init_states, dtype=np.float64)
        ps = None if param_set is None else np.ascontiguousarray(param_set, dtype=np.int32)
        pt = None if param_table is None else np.ascontiguousarray(param_table, dtype=np.float64)
        check(lib().cg_set_cells(self.h, dptr(ini), iptr(ps), dptr(pt), 0 if pt is None else pt.shape[0]),
              "cg_set_cells")

    def set_stimulus(self, stim_id, stims):
        sid = np.ascontiguousarray(stim_id, dtype=np.int32)
        arr = (Stimulus * max(1, len(stims)))(*stims)
        check(lib().cg_set_stimulus(self.h, iptr(sid), arr, len(stims)), "cg_set_stimulus")

    # -- stepping
    def step(self, n=1):
        check(lib().cg_step(self.h, int(n)), "cg_step")

    def step_host(self, v_in, n=1, v_out=None, keep_history=True):
        """n steps from the host voltage v_in (None: the device's), V after them into
        v_out (None: not read back); one synchronisation (cg_step_host)."""
        vi = None if v_in is None else np.ascontiguousarray(v_in, dtype=np.float64)
        if vi is not None and vi.size != self.n:
            raise ValueError("v_in must hold one value per node")
        if v_out is not None and (v_out.dtype != np.float64 or not v_out.flags.c_contiguous or v_out.size != self.n):
            raise ValueError("v_out must be a contiguous float64 array of one value per node")
        check(lib().cg_step_host(self.h, dptr(vi), int(n), dptr(v_out), 1 if keep_history else 0), "cg_step_host")
        return v_out

    def step_profiled(self, n=1):
        """Returns (ms in the ODE kernel, ms in the RHS+CG kernel) over n steps."""
        a, b = C.c_double(), C.c_double()
        check(lib().cg_step_profiled(self.h, int(n), C.byref(a), C.byref(b)), "cg_step_profiled")
        return a.value, b.value

    # -- views
    def voltage(self, out=None):
        """V (FP64, n values); `out` may be a caller buffer (e.g. page-locked) to fill."""
        v = np.empty(self.n) if out is None else out
        if v.dtype != np.float64 or v.size != self.n or not v.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of n values")
        check(lib().cg_get_voltage(self.h, dptr(v)), "cg_get_voltage")
        return v

    def set_voltage(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        check(lib().cg_set_voltage(self.h, dptr(v)), "cg_set_voltage")

    def states(self):
        s = np.empty((self.n, self.n_states))
        check(lib().cg_get_states(self.h, dptr(s)), "cg_get_states")
        return s

    def cell_state(self, node):
        s = np.empty(self.n_states)
        check(lib().cg_get_cell_state(self.h, int(node), dptr(s)), "cg_get_cell_state")
        return s

    def caches(self):
        a, b = np.empty(self.n), np.empty(self.n)
        check(lib().cg_get_caches(self.h, dptr(a), dptr(b)), "cg_get_caches")
        return a, b

    def activation_times(self):
        t = np.empty(self.n)
        check(lib().cg_get_activation_times(self.h, dptr(t)), "cg_get_activation_times")
        return t

    def stats(self) -> Stats:
        s = Stats()
        check(lib().cg_get_stats(self.h, C.byref(s)), "cg_get_stats")
        return s

    def iteration_history(self, n):
        it = np.zeros(n, dtype=np.int32)
        check(lib().cg_get_iteration_history(self.h, n, iptr(it)), "cg_get_iteration_history")
        return it

    def apply_inner_preconditioner(self, x):
        """B x for the mixed solve's x-line inner preconditioner (a diagnostic)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        check(lib().cg_apply_inner_preconditioner(self.h, dptr(x), dptr(y)), "cg_apply_inner_preconditioner")
        return y

    # -- printing-step output on the device
    def configure_output(self, printing_steps, max_frames, state_vars=()):
        sv = np.ascontiguousarray(state_vars, dtype=np.int32)
        check(lib().cg_output_configure(self.h, int(printing_steps), int(max_frames),
                                        iptr(sv) if sv.size else None, int(sv.size)), "cg_output_configure")
        self._out_nv = 1 + int(sv.size)

    def enable_activation_modifier(self, threshold):
        check(lib().cg_output_activation(self.h, float(threshold)), "cg_output_activation")

    def activation_modifier_times(self):
        """(n, 4): first activation, first recovery, second activation, second recovery."""
        t = np.zeros((self.n, 4))
        check(lib().cg_output_get_activation(self.h, dptr(t)), "cg_output_get_activation")
        return t

    def output_times(self):
        nf = C.c_int()
        check(lib().cg_output_frames(self.h, C.byref(nf), None), "cg_output_frames")
        t = np.zeros(nf.value)
        check(lib().cg_output_frames(self.h, C.byref(nf), dptr(t)), "cg_output_frames")
        return t

    def output_frames(self, first=0, count=None):
        """Frames as Hdf5DataWriter's Data dataset: (frames, nodes, variables), V first."""
        nf = C.c_int()
        check(lib().cg_output_frames(self.h, C.byref(nf), None), "cg_output_frames")
        count = nf.value - first if count is None else count
        out = np.zeros((count, self.n, getattr(self, "_out_nv", 1)))
        check(lib().cg_output_fetch(self.h, int(first), int(count), dptr(out)), "cg_output_fetch")
        return out

    @staticmethod
    def _rows(arr, counts):
        return [list(arr[i, :min(int(c), arr.shape[1])]) for i, c in enumerate(counts)]

    def cell_property_maps(self, percentage=90.0, threshold=-30.0, max_aps=16):
        """(APD map, upstroke-time map, max-upstroke-velocity map) as per-node lists, and
        the raw padded arrays with the list lengths."""
        n = self.n
        apd, ut, uv = (np.zeros((n, max_aps)) for _ in range(3))
        na, nu = np.zeros(n, np.int32), np.zeros(n, np.int32)
        check(lib().cg_output_cell_properties(self.h, float(percentage), float(threshold), int(max_aps), dptr(apd),
                                              iptr(na), dptr(ut), dptr(uv), iptr(nu)), "cg_output_cell_properties")
        return dict(apd=self._rows(apd, na), upstroke_time=self._rows(ut, nu), max_upstroke_velocity=self._rows(uv, nu),
                    apd_array=apd, upstroke_time_array=ut, max_upstroke_velocity_array=uv, n_apd=na, n_upstroke=nu)

    def conduction_velocity_map(self, origin, distances, threshold=-30.0, max_aps=16):
        d = np.ascontiguousarray(distances, dtype=np.float64)
        cv = np.zeros((self.n, max_aps))
        nc = np.zeros(self.n, np.int32)
        check(lib().cg_output_conduction_velocity(self.h, int(origin), dptr(d), float(threshold), int(max_aps),
                                                  dptr(cv), iptr(nc)), "cg_output_conduction_velocity")
        return self._rows(cv, nc)

    def snapshot(self) -> bytes:
        sz = C.c_size_t()
        check(lib().cg_snapshot_size(self.h, C.byref(sz)), "cg_snapshot_size")
        buf = C.create_string_buffer(sz.value)
        check(lib().cg_snapshot(self.h, buf, sz.value), "cg_snapshot")
        return buf.raw

    def restore(self, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        check(lib().cg_restore(self.h, buf, len(blob)), "cg_restore")

    def close(self):
        if getattr(self, "h", None):
            lib().cg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class CellBatch:
    """A population of single cells run in FP64 and FP32 side by side (cg_batch)."""

    def __init__(self, model, beats, params=None, stim=None, dt=0.01, beat_length=1000.0, max_aps=None, device=0):
        beats = np.ascontiguousarray(beats, dtype=np.int32)
        self.n = beats.size
        self.model = model
        self.n_states = num_states(model)
        self.max_beats = max(1, int(beats.max()))
        self.max_aps = int(max_aps or self.max_beats + 1)
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        st = stim if stim is not None else stimulus(STIM_REGULAR, -52.0, 1.0, 50.0, 1000.0)
        h = C.c_void_p()
        check(lib().cg_batch_create(model, self.n, iptr(beats), dptr(p), C.byref(st), dt, beat_length,
                                    self.max_aps, device, C.byref(h)), "cg_batch_create")
        self.h = h

    def autotune(self, steps=2000):
        """Pick threads per block and cells per thread; returns the threads per block."""
        tpb = C.c_int()
        check(lib().cg_batch_autotune(self.h, steps, C.byref(tpb)), "cg_batch_autotune")
        return tpb.value

    def set_launch_shape(self, threads_per_block, cells_per_thread):
        check(lib().cg_batch_set_launch_shape(self.h, threads_per_block, cells_per_thread),
              "cg_batch_set_launch_shape")

    def launch_shape(self):
        tpb, cpt = C.c_int(), C.c_int()
        check(lib().cg_batch_launch_shape(self.h, C.byref(tpb), C.byref(cpt)), "cg_batch_launch_shape")
        return tpb.value, cpt.value

    def set_engine(self, engine):
        check(lib().cg_batch_set_engine(self.h, int(engine)), "cg_batch_set_engine")

    def engine(self):
        e = C.c_int()
        check(lib().cg_batch_engine(self.h, C.byref(e)), "cg_batch_engine")
        return e.value

    def run(self):
        ms = C.c_double()
        check(lib().cg_batch_run(self.h, C.byref(ms)), "cg_batch_run")
        return ms.value

    def results(self):
        n, ma, mb, S = self.n, self.max_aps, self.max_beats, self.n_states
        a64, a32 = np.zeros((n, ma)), np.zeros((n, ma))
        k64, k32 = np.zeros(n, np.int32), np.zeros(n, np.int32)
        dv = np.zeros((n, mb), np.float32)
        s64, s32 = np.zeros((n, S)), np.zeros((n, S))
        check(lib().cg_batch_results(self.h, dptr(a64), dptr(a32), iptr(k64), iptr(k32),
                                     dv.ctypes.data_as(C.POINTER(C.c_float)), dptr(s64), dptr(s32)),
              "cg_batch_results")
        return dict(apd64=a64, apd32=a32, n_ap64=k64, n_ap32=k32, max_dv=dv, states64=s64, states32=s32)

    def close(self):
        if getattr(self, "h", None):
            lib().cg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class RunPopulation:
    """Single-cell and cable runs of one cell model in one persistent launch (cg_runs)."""

    def __init__(self, model, device=0):
        self.model = model
        self.n_states = num_states(model)
        self.n_params = num_params(model)
        self._cables = {}
        h = C.c_void_p()
        check(lib().cg_runs_create(model, device, C.byref(h)), "cg_runs_create")
        self.h = h

    def add_cell(self, method, n_steps, dt=0.01, sample_every=1, params=None, stim=None):
        """Returns the run id; params: n_params scale factors (None: all 1)."""
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
        i = C.c_int()
        check(lib().cg_runs_add_cell(self.h, method, dptr(p), C.byref(stim) if stim is not None else None, dt,
                                     int(n_steps), int(sample_every), C.byref(i)), "cg_runs_add_cell")
        return i.value

    def add_cable(self, cfg, params, probes, sample_every=1):
        """cfg: CableConfig; params: n_regions x (n_params + 1); probes: node indices."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        pr = np.ascontiguousarray(probes, dtype=np.int32)
        i = C.c_int()
        check(lib().cg_runs_add_cable(self.h, C.byref(cfg), dptr(p), iptr(pr), pr.size, int(sample_every),
                                      C.byref(i)), "cg_runs_add_cable")
        self._cables[i.value] = (cfg.n_nodes, pr.size)
        return i.value

    def autotune(self, steps=200):
        tpb, cpt = C.c_int(), C.c_int()
        check(lib().cg_runs_autotune(self.h, steps, C.byref(tpb), C.byref(cpt)), "cg_runs_autotune")
        return tpb.value, cpt.value

    def set_shape(self, threads_per_block, cells_per_thread):
        check(lib().cg_runs_set_shape(self.h, threads_per_block, cells_per_thread), "cg_runs_set_shape")

    def shape(self):
        tpb, cpt = C.c_int(), C.c_int()
        check(lib().cg_runs_shape(self.h, C.byref(tpb), C.byref(cpt)), "cg_runs_shape")
        return tpb.value, cpt.value

    def run(self):
        ms = C.c_double()
        check(lib().cg_runs_run(self.h, C.byref(ms)), "cg_runs_run")
        return ms.value

    def result(self, run_id):
        """Cell: (states (n_states,), trace (n_samples,)); cable: (states (n_nodes, n_states),
        trace (n_samples, n_probes), cg_iterations)."""
        ns = C.c_int()
        check(lib().cg_runs_result(self.h, run_id, None, None, C.byref(ns), None), "cg_runs_result")
        it = C.c_longlong()
        if run_id in self._cables:
            n, npr = self._cables[run_id]
            st, tr = np.zeros((n, self.n_states)), np.zeros((ns.value, npr))
            check(lib().cg_runs_result(self.h, run_id, dptr(st), dptr(tr), None, C.byref(it)), "cg_runs_result")
            return st, tr, it.value
        st, tr = np.zeros(self.n_states), np.zeros(ns.value)
        check(lib().cg_runs_result(self.h, run_id, dptr(st), dptr(tr), None, None), "cg_runs_result")
        return st, tr

    def close(self):
        if getattr(self, "h", None):
            lib().cg_runs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
