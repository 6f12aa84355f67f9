"""Conductance fitting on a 1D monodomain cable: batched forward runs and the
discrete adjoint of the operator-split step behind ``torch.autograd.Function``.

The forward step is Chaste's monodomain step with the ODE step equal to the PDE
step (AbstractCardiacTissue::SolveCellSystems with ComputeExceptVoltage, then
MonodomainSolver::SetupLinearSystem, heart/src/solver/MonodomainSolver.cpp:92-101,
and the CG + Jacobi solve of (Am Cm/dt M + K) V = M z); the loss is the mean
squared mismatch of the voltage at probe nodes over every step.  Gradients with
respect to the per-region scale factors (the cell model's conductance scales
and the tissue conductivity scale) come from the adjoint kernel in
libchastegpu.so, which recomputes the forward run segment by segment from
checkpoints.  torch supplies device memory and the autograd plumbing only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def default_cable_config() -> N.CableConfig:
    """1000 nodes, h = 0.01 cm, LR91, dt 0.01 ms, 400 ms, 4 regions, checkpoints every 200 steps."""
    cfg = N.CableConfig()
    N.lib().cg_cable_default_config(C.byref(cfg))
    return cfg


def node_regions(n_nodes: int, n_regions: int) -> np.ndarray:
    """Region of every node: floor(i R / n), capped at R - 1."""
    i = np.arange(n_nodes)
    return np.minimum(n_regions - 1, i * n_regions // n_nodes)


def element_regions(n_nodes: int, n_regions: int) -> np.ndarray:
    """Region of every element (nodes e, e+1): floor(e R / (n - 1)), capped at R - 1."""
    e = np.arange(n_nodes - 1)
    return np.minimum(n_regions - 1, e * n_regions // (n_nodes - 1))


def even_probes(n_nodes: int, n_probes: int) -> np.ndarray:
    """n_probes evenly spaced node indices from the first node to the last."""
    return np.unique(np.round(np.linspace(0, n_nodes - 1, n_probes)).astype(np.int32))


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class Cable:
    """A cable of ``cfg.n_nodes`` nodes on one GPU (cg_cable_*).

    Parameter tensors are float64 on the cable's device, shaped
    (n_sets, n_regions, n_params + 1): per region the cell model's scale
    factors, then the conductivity scale.
    """

    def __init__(self, cfg: N.CableConfig, probes, device: int = 0):
        import torch

        self.cfg = cfg
        self.probes = np.ascontiguousarray(probes, dtype=np.int32)
        self.device = torch.device("cuda", device)
        npar = C.c_int()
        N.check(N.lib().cg_num_params(cfg.model, C.byref(npar)), "cg_num_params")
        self.n_params = npar.value
        self.stride = self.n_params + 1
        h = C.c_void_p()
        N.check(N.lib().cg_cable_create(C.byref(cfg), N.iptr(self.probes), self.probes.size, device, C.byref(h)),
                "cg_cable_create")
        self.h = h

    @property
    def shape(self):
        return (self.cfg.n_regions, self.stride)

    def _check_params(self, params):
        import torch

        if params.dtype != torch.float64 or params.device != self.device or params.dim() != 3 or \
                tuple(params.shape[1:]) != self.shape:
            raise ValueError(f"params must be float64 on {self.device} shaped (n_sets, {self.shape[0]}, "
                             f"{self.shape[1]})")
        return params.contiguous()

    def _check_targets(self, targets):
        import torch

        if targets is None:
            return None
        if targets.dtype != torch.float64 or targets.device != self.device or \
                tuple(targets.shape) != (self.cfg.n_steps, self.probes.size):
            raise ValueError(f"targets must be float64 on {self.device} shaped ({self.cfg.n_steps}, "
                             f"{self.probes.size})")
        return targets.contiguous()

    def forward(self, params, targets=None, traces=False, keep_checkpoints=False, iterations=False):
        """Run every parameter set; returns dict(loss, traces, iterations) (None where not asked)."""
        import torch

        params = self._check_params(params)
        targets = self._check_targets(targets)
        n_sets = params.shape[0]
        loss = torch.empty(n_sets, dtype=torch.float64, device=self.device) if targets is not None else None
        tr = torch.empty((n_sets, self.cfg.n_steps, self.probes.size), dtype=torch.float64,
                         device=self.device) if traces else None
        its = torch.empty(n_sets, dtype=torch.int32, device=self.device) if iterations else None
        stream = torch.cuda.current_stream(self.device).cuda_stream
        N.check(N.lib().cg_cable_forward(self.h, n_sets, _ptr(params), _ptr(targets), _ptr(loss), _ptr(tr),
                                         _ptr(its), 1 if keep_checkpoints else 0, C.c_void_p(stream)),
                "cg_cable_forward")
        return dict(loss=loss, traces=tr, iterations=its)

    def backward(self, params, targets):
        """dL/dparams of the last forward(keep_checkpoints=True) call (same params and targets)."""
        import torch

        params = self._check_params(params)
        targets = self._check_targets(targets)
        grad = torch.empty_like(params)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        N.check(N.lib().cg_cable_backward(self.h, params.shape[0], _ptr(params), _ptr(targets), _ptr(grad),
                                          C.c_void_p(stream)), "cg_cable_backward")
        return grad

    def close(self):
        if getattr(self, "h", None):
            N.lib().cg_cable_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def _function():
    import torch

    class CableMSELoss(torch.autograd.Function):
        """loss[s] = mean over steps and probes of (V_s - target)^2 for every parameter set s.

        backward runs the checkpointed adjoint; the targets get no gradient.
        """

        @staticmethod
        def forward(ctx, params, targets, cable):
            out = cable.forward(params, targets, keep_checkpoints=True)
            ctx.cable = cable
            ctx.save_for_backward(params, targets)
            return out["loss"]

        @staticmethod
        def backward(ctx, grad_loss):
            params, targets = ctx.saved_tensors
            g = ctx.cable.backward(params, targets)
            return g * grad_loss.reshape(-1, 1, 1), None, None

    return CableMSELoss


_CableMSELoss = None


def cable_mse_loss(params, targets, cable: Cable):
    """Differentiable per-set loss (shape (n_sets,)) of ``params`` on ``cable``."""
    global _CableMSELoss
    if _CableMSELoss is None:
        _CableMSELoss = _function()
    return _CableMSELoss.apply(params, targets, cable)
