"""A CPU backend for chaste_b200.partition.PartitionedSlabTissue, built on the
oracle: one rank's rows of the slab with the oracle's assembled A and M
(heart/src/solver/electrics/monodomain/MonodomainAssembler.cpp restated), its
cells stepped by the oracle's single-cell ComputeExceptVoltage, and the four
phases of the partitioned CG in numpy.  It lets the decomposition (row ranges,
halos, the order of the reductions) run on gloo ranks without a GPU; the GPU
backend is chaste_b200.partition.NativePartition."""
from __future__ import annotations

import ctypes as C

import numpy as np

from chaste_b200.partition import row_range


class OraclePartition:
    def __init__(self, O, case, rank, world, cfg):
        from tests import tissue_cases as TC

        self.O = O
        self.case = case
        self.cfg = cfg
        whole, xyz = TC.make_oracle(O, **case)         # matrices and initial states only
        self.n = xyz.shape[0]
        self.lo, self.hi = row_range(self.n, rank, world)
        rp, cols, a = whole.matrix(0)
        _, _, m = whole.matrix(1)
        self.rp, self.cols, self.a, self.m = rp, cols, a, m
        self.halo = int(max(np.abs(cols - np.repeat(np.arange(self.n), np.diff(rp))).max(), 1))
        self.diag = np.array([a[rp[i]:rp[i + 1]][cols[rp[i]:rp[i + 1]] == i][0] for i in range(self.n)])
        states = whole.states()
        self.y = states[self.lo:self.hi].copy()                # node-major
        self.x = np.zeros(self.n)                              # global-length, own rows + halos valid
        self.x[self.lo:self.hi] = self.y[:, 0]
        self.z = np.zeros(self.n)
        self.zp = np.zeros(self.n)
        nl = self.hi - self.lo
        self.r, self.p, self.q, self.b = np.zeros(nl), np.zeros(nl), np.zeros(nl), np.zeros(nl)
        self.sid = TC.slab_stim_ids(xyz, case["box_hi"])[self.lo:self.hi]
        self.stim = O.simple(*case["stim"])
        self.steps = 0

    def _rows(self, vals, vec):
        out = np.empty(self.hi - self.lo)
        for k, i in enumerate(range(self.lo, self.hi)):
            s, e = self.rp[i], self.rp[i + 1]
            out[k] = float(np.dot(vals[s:e], vec[self.cols[s:e]]))
        return out

    def ode(self):
        c = self.case
        dt = c["dt_pde"]
        t0, t1 = self.steps * dt, (self.steps + 1) * dt
        am, cm = c.get("am", 1400.0), c.get("cm", 1.0)
        for k in range(self.hi - self.lo):
            v = self.x[self.lo + k]
            y = self.y[k]
            y[0] = v
            st = self.stim if self.sid[k] >= 0 else None
            iion = self.O.cell_except_voltage(c["model"], c["method"], y, t0, t1, c["dt_ode"], stim=st, am=am, cm=cm)
            y[0] = v
            istim = self.O.lib().orc_stimulus_value(C.byref(st), t1) if st is not None else 0.0
            # z = Am*Cm*V/dt - Am*Iion - Istim (MonodomainSolver.cpp:92-101), the oracle's order
            self.z[self.lo + k] = am * cm * v * (1.0 / dt) + (-am * iion - istim)

    def _vec(self, which):
        return (self.x, self.z, self.zp)[which]

    def pack(self, which):
        v = self._vec(which)
        return v[self.lo:self.lo + self.halo].copy(), v[self.hi - self.halo:self.hi].copy()

    def unpack(self, which, lo, hi):
        v = self._vec(which)
        if lo is not None:
            v[self.lo - self.halo:self.lo] = lo
        if hi is not None:
            v[self.hi:self.hi + self.halo] = hi

    def phase(self, k, scalars=(0.0, 0.0)):
        own = slice(self.lo, self.hi)
        d = 1.0 / self.diag[own] if self.cfg.ksp_preconditioner == 1 else np.ones(self.hi - self.lo)
        s = np.zeros(4)
        if k == 0:
            self.b = self._rows(self.m, self.z)
            self.r = self.b - self._rows(self.a, self.x)
            w, zz = d * self.b, d * self.r
            self.zp[own] = zz
            s[:] = [np.abs(self.b).sum(), (w * w).sum(), (zz * zz).sum(), (self.r * zz).sum()]
        elif k == 1:
            zz = d * self.b
            self.x[own] = 0.0
            self.r = self.b.copy()
            self.zp[own] = zz
            s[:2] = [(zz * zz).sum(), (self.b * zz).sum()]
        elif k == 2:
            az = self._rows(self.a, self.zp)
            first = scalars[1] != 0.0
            self.q = az if first else az + scalars[0] * self.q
            self.p = self.zp[own].copy() if first else self.zp[own] + scalars[0] * self.p
            s[0] = (self.p * self.q).sum()
        else:
            self.x[own] += scalars[0] * self.p
            self.r = self.r - scalars[0] * self.q
            zz = d * self.r
            self.zp[own] = zz
            s[:2] = [(zz * zz).sum(), (zz * self.r).sum()]
        return s

    def finish_step(self):
        self.steps += 1

    def voltage(self):
        return self.x[self.lo:self.hi].copy()
