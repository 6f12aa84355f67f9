"""Paired oracle / GPU tissue set-ups shared by the parity tests and the benchmark."""
from __future__ import annotations

import numpy as np

LR91, TT06 = 0, 1
FE, RL = 0, 1


def slab_stim_ids(xyz, box_hi):
    """Nodes with every coordinate <= box_hi[d] (corner box from the origin)."""
    inside = np.ones(xyz.shape[0], bool)
    for d, hi in enumerate(box_hi):
        inside &= xyz[:, d] <= hi + 1e-12
    return np.where(inside, 0, -1).astype(np.int32)


def make_gpu(N, *, model, method, dt_ode, dt_pde, dim, h, size, sigma, stim, box_hi, am=1400.0, cm=1.0,
             abs_tol=None, rel_tol=1e-8, precision=0, use_csr=False, param_set=None, param_table=None,
             init_states=None, max_iterations=10000, solver=0, svi=0, inner_pc=0, lump=False, pc=1):
    """A GPU tissue on a regular slab (stencil operator, or CSR through cg_set_mesh when use_csr)."""
    from oracle import pyoracle as O  # mesh generator only: the same node/element order as the library

    cfg = N.default_config()
    cfg.model, cfg.ode_method = model, method
    cfg.ode_time_step, cfg.pde_time_step = dt_ode, dt_pde
    cfg.surface_area_to_volume_ratio, cfg.capacitance = am, cm
    cfg.ksp_preconditioner = pc
    if abs_tol is not None:
        cfg.use_absolute_tolerance, cfg.ksp_tolerance = 1, abs_tol
    else:
        cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, rel_tol
    cfg.precision = precision
    cfg.max_iterations = max_iterations
    cfg.solver = solver
    cfg.use_state_variable_interpolation = svi
    cfg.mixed_inner_preconditioner = inner_pc
    cfg.use_mass_lumping = 1 if lump else 0
    t = N.Tissue(cfg)
    xyz, conn, _ = O.slab_mesh(dim, h, *size)
    if use_csr:
        t.set_mesh(xyz, conn, np.asarray(sigma[:dim]))
    else:
        t.set_slab_mesh(dim, h, *size, sigma=sigma)
    t.set_cells(init_states=init_states, param_set=param_set, param_table=param_table)
    sid = slab_stim_ids(xyz, box_hi)
    t.set_stimulus(sid, [N.stimulus(N.STIM_SIMPLE, *stim)])
    return t, xyz


def make_oracle(O, *, model, method, dt_ode, dt_pde, dim, h, size, sigma, stim, box_hi, am=1400.0, cm=1.0,
                abs_tol=None, rel_tol=1e-8, param_set=None, param_table=None, init_states=None, solver=0, svi=0,
                pc=1, **_):
    xyz, conn, _ = O.slab_mesh(dim, h, *size)
    use_abs = abs_tol is not None
    cfg = O.Config(model, method, dt_ode, dt_pde, am, cm, pc, 1 if use_abs else 0,
                   abs_tol if use_abs else rel_tol, 0, 10000, solver, svi)
    sig = np.tile(np.asarray(sigma[:dim], float), (conn.shape[0], 1))
    sid = slab_stim_ids(xyz, box_hi)
    return O.Tissue(cfg, dim, xyz, conn, sig, sid, [O.simple(*stim)], param_id=param_set,
                    param_table=param_table, init_states=init_states), xyz


# Reduced versions of the benchmark configurations (same physics, smaller slabs)
LR91_2D = dict(model=LR91, method=FE, dt_ode=0.01, dt_pde=0.1, dim=2, h=0.01, size=(0.2, 0.2, 0.0),
               sigma=(1.75, 1.75, 1.75), stim=(-5e5, 0.5, 0.0), box_hi=(0.0199, 1e9))
TT06_3D = dict(model=TT06, method=RL, dt_ode=0.02, dt_pde=0.1, dim=3, h=0.01, size=(0.2, 0.07, 0.03),
               sigma=(1.75, 0.19, 0.19), stim=(-5e5, 1.0, 0.0), box_hi=(0.03, 0.03, 0.03))

# TestNiederer2011BenchmarkSimulation.hpp:82-157 at h = 0.05, dt = 0.01 (TestRunOnCoarsestMesh)
NIEDERER = dict(model=TT06, method=2, dt_ode=0.005, dt_pde=0.01, dim=3, h=0.05, size=(2.0, 0.7, 0.3),
                sigma=(0.17 * 0.62 / (0.17 + 0.62) * 10, 0.019 * 0.24 / (0.019 + 0.24) * 10,
                       0.019 * 0.24 / (0.019 + 0.24) * 10),
                stim=(-50000.0, 2.0, 0.0), box_hi=(0.15 + 1e-6,) * 3, am=1400.0, cm=1.0, abs_tol=2e-4, svi=1)


def niederer_activation(t, n, printing_steps=10, n_prints=400, printing_dt=0.1):
    """Activation times as TestNiederer2011BenchmarkSimulation.hpp:161-203 computes
    them from the printed voltages: linear interpolation to the first V > 0."""
    act = -np.ones(n)
    last = np.ones(n)
    for k in range(1, n_prints + 1):
        t.step(printing_steps)
        v = t.voltage()
        new = (v > 0) & (act < 0)
        act[new] = (k - v[new] / (v[new] - last[new])) * printing_dt
        last = np.where(v <= 0, v, last)
    return act


# The benchmark workloads at full size: the 2D LR91 sheet, the 3D TT06 slab and the 2.1M-node slab
LR91_SHEET_10201 = dict(model=LR91, method=FE, dt_ode=0.01, dt_pde=0.1, dim=2, h=0.01, size=(1.0, 1.0, 0.0),
                   sigma=(1.75, 1.75, 1.75), stim=(-5e5, 0.5, 0.0), box_hi=(0.0199, 1e9))
TT06_SLAB_442401 = dict(model=TT06, method=RL, dt_ode=0.02, dt_pde=0.1, dim=3, h=0.01, size=(2.0, 0.7, 0.3),
                  sigma=(1.75, 0.19, 0.19), stim=(-5e5, 1.0, 0.0), box_hi=(0.1, 0.1, 0.1))
TT06_SLAB_2099601 = dict(TT06_SLAB_442401, h=0.0125, size=(2.0, 2.0, 1.0))


def transmural(case):
    """The case with TT06 endo / mid / epi layers by thirds of z (param_set, param_table)."""
    from chaste_b200.heart import slab_coordinates, transmural_layers, transmural_param_table

    xyz = slab_coordinates(case["dim"], case["h"], *case["size"])
    return dict(case, param_set=transmural_layers(xyz[:, 2], case["size"][2]), param_table=transmural_param_table())
