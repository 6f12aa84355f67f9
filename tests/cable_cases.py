"""Cable set-ups shared by the fitting tests and the benchmark: the GPU cable
configuration, the same cable as an oracle tissue, and seeded parameter draws."""
from __future__ import annotations

import numpy as np

LR91 = 0


def cable_config(N, *, n_nodes, n_steps, n_regions, checkpoint_every=200, rtol=1e-8, h=0.01, dt=0.01,
                 sigma=1.75, n_stim=2, stim=(-5e5, 0.5)):
    from chaste_b200 import fitting

    cfg = fitting.default_cable_config()
    cfg.n_nodes, cfg.n_steps, cfg.n_regions = n_nodes, n_steps, n_regions
    cfg.checkpoint_every, cfg.ksp_tolerance = checkpoint_every, rtol
    cfg.h, cfg.time_step, cfg.conductivity = h, dt, sigma
    cfg.n_stimulated_nodes = n_stim
    cfg.stimulus_magnitude, cfg.stimulus_duration = stim
    return cfg


def oracle_config(O, cfg):
    """The oracle's description (orc_cable_config) of a GPU cable configuration."""
    return O.CableConfig(cfg.model, cfg.n_nodes, cfg.h, cfg.conductivity, cfg.surface_area_to_volume_ratio,
                         cfg.capacitance, cfg.time_step, cfg.n_steps, cfg.n_regions, cfg.n_stimulated_nodes,
                         cfg.stimulus_magnitude, cfg.stimulus_duration, cfg.ksp_tolerance, cfg.max_iterations,
                         cfg.checkpoint_every)


class PlainCableConfig:
    """The fields of cg_cable_config, for oracle-only (CPU) tests that do not load the GPU library."""

    def __init__(self, *, n_nodes, n_steps, n_regions, checkpoint_every=200, rtol=1e-8, h=0.01, dt=0.01,
                 sigma=1.75, n_stim=2, stim=(-5e5, 0.5), model=LR91):
        self.model, self.n_nodes, self.h, self.conductivity = model, n_nodes, h, sigma
        self.surface_area_to_volume_ratio, self.capacitance, self.time_step = 1400.0, 1.0, dt
        self.n_steps, self.n_regions, self.n_stimulated_nodes = n_steps, n_regions, n_stim
        self.stimulus_magnitude, self.stimulus_duration = stim
        self.ksp_tolerance, self.max_iterations, self.checkpoint_every = rtol, 10000, checkpoint_every


def node_regions(n, R):
    return np.minimum(R - 1, np.arange(n) * R // n)


def element_regions(n, R):
    return np.minimum(R - 1, np.arange(n - 1) * R // (n - 1))


def even_probes(n, k):
    return np.unique(np.round(np.linspace(0, n - 1, k)).astype(np.int32))


def lognormal_params(rng, n_sets, n_regions, stride, sd):
    """Scale factors exp(N(0, sd^2)) for every region and conductance."""
    return np.exp(rng.normal(0.0, sd, size=(n_sets, n_regions, stride)))


def oracle_cable(O, cfg, params):
    """The cable as an oracle monodomain tissue: params (R, P+1) scale factors."""
    n, R = cfg.n_nodes, cfg.n_regions
    xyz = np.zeros((n, 3))
    xyz[:, 0] = np.arange(n) * cfg.h
    conn = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).astype(np.int32)
    er = element_regions(n, R)
    sigma = (cfg.conductivity * params[er, -1]).reshape(-1, 1)
    stim_id = np.where(np.arange(n) < cfg.n_stimulated_nodes, 0, -1).astype(np.int32)
    ocfg = O.Config(cfg.model, 0, cfg.time_step, cfg.time_step, cfg.surface_area_to_volume_ratio,
                    cfg.capacitance, O.PC_JACOBI, 0, cfg.ksp_tolerance, 0, cfg.max_iterations)
    return O.Tissue(ocfg, 1, xyz, conn, sigma, stim_id, [O.simple(cfg.stimulus_magnitude, cfg.stimulus_duration)],
                    param_id=node_regions(n, R).astype(np.int32),
                    param_table=np.ascontiguousarray(params[:, :-1]))


def oracle_traces(O, cfg, params, probes):
    """Probe voltages after every step (n_steps x n_probes) of the oracle cable."""
    t = oracle_cable(O, cfg, params)
    out = np.zeros((cfg.n_steps, len(probes)))
    for k in range(cfg.n_steps):
        t.step(1)
        out[k] = t.voltage()[probes]
    return out


def oracle_loss(O, cfg, params, probes, targets):
    return float(np.mean((oracle_traces(O, cfg, params, probes) - targets) ** 2))
