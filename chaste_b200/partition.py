"""Multi-GPU slab tissue: one process per GPU, rows owned in contiguous ranges.

Chaste distributes a tissue over MPI ranks by contiguous row ranges (PETSc's
PETSC_DECIDE split, global/src/parallel/DistributedVectorFactory.cpp:44-64): the
ionic ODEs stay local, and every operator application inside KSPSolve
(linalg/src/LinearSystem.cpp:1099) first exchanges the ghost rows the stencil
reaches, while each inner product is an all-reduce.  This module is that step for
libchastegpu: each rank holds its rows in a ``cg_part`` (chaste_b200/csrc/partition.cu),
and :class:`PartitionedSlabTissue` sequences one PDE step across the ranks --

    ODE (local) -> halo of V and z -> phase 0 (b = M z, r, B r) -> all-reduce
    -> per CG iteration: halo of B r -> phase 2 (A p, p.Ap) -> all-reduce
                         -> phase 3 (x, r, B r, norms) -> all-reduce

with PETSc's CG recurrence and KSPConvergedDefault test exactly as the single-GPU
kernel takes them (two all-reduces per iteration, as KSPSolve_CG makes).  Halos go
to the neighbouring ranks only (rank - 1 and rank + 1 in row order) through
torch.distributed point-to-point calls; the scalars through all_reduce.  Every
rank takes the same collective calls in the same order: all branch decisions are
made on all-reduced scalars, which every rank receives bitwise equal.

Backends: :class:`NativePartition` (the CUDA kernels); the tests add a CPU one
built on the oracle, so the decomposition itself is checked with gloo ranks
without a GPU.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N


def row_range(n, rank, world):
    """PETSc's PETSC_DECIDE split: rank r owns n/world rows, one more when r < n % world."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class NativePartition:
    """One rank's rows of a slab tissue on this process's GPU (the cg_part_* C-ABI)."""

    def __init__(self, cfg, dim, h, size, sigma, rank, world):
        L = N.lib()
        sig = np.ascontiguousarray(np.asarray(sigma, dtype=np.float64)[:dim])
        self.h = C.c_void_p()
        N.check(L.cg_part_create(C.byref(cfg), dim, h, *size, N.dptr(sig), rank, world, C.byref(self.h)),
                "cg_part_create")
        lo, hi, halo, n = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        N.check(L.cg_part_rows(self.h, C.byref(lo), C.byref(hi), C.byref(halo), C.byref(n)), "cg_part_rows")
        self.lo, self.hi, self.halo, self.n = lo.value, hi.value, halo.value, n.value
        self.cfg = cfg

    def set_cells(self, init_states=None, param_set=None, param_table=None):
        ini = None if init_states is None else np.ascontiguousarray(init_states, dtype=np.float64)
        ps = None if param_set is None else np.ascontiguousarray(param_set, dtype=np.int32)
        pt = None if param_table is None else np.ascontiguousarray(param_table, dtype=np.float64)
        N.check(N.lib().cg_part_set_cells(self.h, N.dptr(ini) if ini is not None else None,
                                          N.iptr(ps) if ps is not None else None,
                                          N.dptr(pt) if pt is not None else None,
                                          0 if pt is None else pt.shape[0]), "cg_part_set_cells")

    def set_stimulus(self, stim_id, stims):
        sid = np.ascontiguousarray(stim_id, dtype=np.int32)
        arr = (N.Stimulus * max(1, len(stims)))(*stims)
        N.check(N.lib().cg_part_set_stimulus(self.h, N.iptr(sid), arr, len(stims)), "cg_part_set_stimulus")

    def ode(self):
        N.check(N.lib().cg_part_ode(self.h), "cg_part_ode")

    def pack(self, which):
        lo, hi = np.empty(self.halo), np.empty(self.halo)
        N.check(N.lib().cg_part_halo_pack(self.h, which, N.dptr(lo), N.dptr(hi)), "cg_part_halo_pack")
        return lo, hi

    def unpack(self, which, lo, hi):
        N.check(N.lib().cg_part_halo_unpack(self.h, which, None if lo is None else N.dptr(lo),
                                            None if hi is None else N.dptr(hi)), "cg_part_halo_unpack")

    def phase(self, k, scalars=(0.0, 0.0)):
        s = np.ascontiguousarray(scalars, dtype=np.float64)
        out = np.zeros(4)
        N.check(N.lib().cg_part_cg_phase(self.h, k, N.dptr(s), N.dptr(out)), "cg_part_cg_phase")
        return out

    def finish_step(self):
        N.check(N.lib().cg_part_finish_step(self.h), "cg_part_finish_step")

    def voltage(self):
        v = np.empty(self.hi - self.lo)
        N.check(N.lib().cg_part_get_voltage(self.h, N.dptr(v)), "cg_part_get_voltage")
        return v

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            N.lib().cg_part_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


# halo vectors of a partition (cg_part_halo_pack's `which`)
HALO_V, HALO_Z, HALO_BR = 0, 1, 2


class PartitionedSlabTissue:
    """The monodomain step over the ranks of a torch.distributed process group.

    ``part`` is this rank's backend (:class:`NativePartition` on a GPU).  KSP
    settings come from its cg_config: relative or absolute tolerance as
    LinearSystem sets them (LinearSystem.cpp:584-602, 755-762), divergence at 1e5,
    max_iterations."""

    def __init__(self, part, group=None):
        import torch.distributed as dist

        self.part = part
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.world = self.dist.get_world_size(group) if self.dist else 1
        cfg = part.cfg
        self.rtol = 2.220446049250313e-16 if cfg.use_absolute_tolerance else cfg.ksp_tolerance
        self.abstol = cfg.ksp_tolerance if cfg.use_absolute_tolerance else 1e-50
        self.maxit = cfg.max_iterations if cfg.max_iterations > 0 else 10000
        self.iterations = []

    # -- communication
    def _allreduce(self, v):
        if self.world == 1:
            return v
        import torch

        t = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64))
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t.numpy()

    def _exchange(self, which):
        lo_blk, hi_blk = self.part.pack(which)
        if self.world == 1:
            return
        import torch

        ops, recv_lo, recv_hi = [], None, None
        # my first rows are the high halo of rank - 1, my last rows the low halo of rank + 1
        if self.rank > 0:
            recv_lo = torch.empty(self.part.halo, dtype=torch.float64)
            ops.append(self.dist.P2POp(self.dist.isend, torch.from_numpy(lo_blk), self.rank - 1, self.group))
            ops.append(self.dist.P2POp(self.dist.irecv, recv_lo, self.rank - 1, self.group))
        if self.rank < self.world - 1:
            recv_hi = torch.empty(self.part.halo, dtype=torch.float64)
            ops.append(self.dist.P2POp(self.dist.isend, torch.from_numpy(hi_blk), self.rank + 1, self.group))
            ops.append(self.dist.P2POp(self.dist.irecv, recv_hi, self.rank + 1, self.group))
        for req in self.dist.batch_isend_irecv(ops):
            req.wait()
        self.part.unpack(which, None if recv_lo is None else recv_lo.numpy(),
                         None if recv_hi is None else recv_hi.numpy())

    # -- one PDE step
    def _solve(self):
        """KSPSolve_CG with Jacobi and KSPConvergedDefault (as cg_fp64_kernel runs it)."""
        self._exchange(HALO_V)
        self._exchange(HALO_Z)
        s = self._allreduce(self.part.phase(0))
        rnorm0, dp, beta = math.sqrt(s[1]), math.sqrt(s[2]), s[3]
        if 0.0 < s[0] < 1e-15:     # LinearSystem.cpp:984-994: tiny RHS -> zero initial guess
            s2 = self._allreduce(self.part.phase(1))
            dp, beta = math.sqrt(s2[0]), s2[1]
            rnorm0 = dp
        if rnorm0 == 0.0:
            rnorm0 = dp
        ttol = max(self.rtol * rnorm0, self.abstol)
        if not math.isfinite(dp):
            raise N.ChasteGpuError(N.CG_ERR_NAN, "partitioned CG")
        if dp <= ttol:
            return 0
        if dp >= 1e5 * rnorm0:
            raise N.ChasteGpuError(N.CG_ERR_CG_DIVERGED, "partitioned CG")
        betaold = 0.0
        for it in range(self.maxit):
            if beta == 0.0:
                return it + 1
            bc = 0.0 if it == 0 else beta / betaold
            self._exchange(HALO_BR)
            dpi = self._allreduce(self.part.phase(2, (bc, 1.0 if it == 0 else 0.0)))[0]
            if not dpi > 0.0:
                raise N.ChasteGpuError(N.CG_ERR_CG_DIVERGED if math.isfinite(dpi) else N.CG_ERR_NAN,
                                       "partitioned CG")
            s = self._allreduce(self.part.phase(3, (beta / dpi, 0.0)))
            dp = math.sqrt(s[0])
            if not math.isfinite(dp):
                raise N.ChasteGpuError(N.CG_ERR_NAN, "partitioned CG")
            if dp <= ttol:
                return it + 1
            if dp >= 1e5 * rnorm0:
                raise N.ChasteGpuError(N.CG_ERR_CG_DIVERGED, "partitioned CG")
            betaold, beta = beta, s[1]
        raise N.ChasteGpuError(N.CG_ERR_CG_MAXIT, "partitioned CG")

    def step(self, n=1):
        for _ in range(n):
            self.part.ode()
            self.iterations.append(self._solve())
            self.part.finish_step()

    def voltage(self):
        """This rank's rows of V."""
        return self.part.voltage()

    def gather_voltage(self):
        """V of every row on every rank (all_gather of the row blocks)."""
        v = self.part.voltage()
        if self.world == 1:
            return v
        import torch

        sizes = [row_range(self.part.n, r, self.world) for r in range(self.world)]
        width = max(hi - lo for lo, hi in sizes)        # equal-sized blocks for all_gather
        mine = torch.zeros(width, dtype=torch.float64)
        mine[: v.size] = torch.from_numpy(v)
        bufs = [torch.empty(width, dtype=torch.float64) for _ in sizes]
        self.dist.all_gather(bufs, mine, group=self.group)
        return torch.cat([b[: hi - lo] for b, (lo, hi) in zip(bufs, sizes)]).numpy()
