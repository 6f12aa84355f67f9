"""Benchmark of the monodomain operator-split step on B200.

Workload (default): the 3D ten Tusscher 2006 epicardial slab, 2 x 0.7 x 0.3 cm
at h = 0.01 cm (ConstructRegularSlabMesh gives 201 x 71 x 31 = 442,401 nodes,
2.52M tetrahedra), Rush-Larsen dt_ode = 0.02 ms, PDE dt = 0.1 ms,
sigma = (1.75, 0.19, 0.19) mS/cm, corner stimulus -5e5 uA/cm^3 for 1 ms in a
0.1 cm cube, CG + Jacobi at rtol 1e-8.  A step is one PDE step of every node
(ODE -> RHS -> CG).  Metric: node-steps/s.  Every arm first advances the
simulation, untimed, to --t-start-ms (default 10 ms: the wavefront is inside the
slab), so the timed steps are the same window of the run for the GPU paths, the
CPU baseline and the reference arm.

The mixed-precision path (FP32 states, FP32 inner CG, FP64 residual
refinement) is the headline when its Vm stays within 0.5 mV of the FP64 path
run over the same steps in the same process; both are reported.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # the headline workload: the 3D TT06 slab of 442,401 nodes
    "tt06_slab_3d": dict(model=1, method=1, dt_ode=0.02, dt_pde=0.1, dim=3, h=0.01,
                         size=(2.0, 0.7, 0.3), sigma=(1.75, 0.19, 0.19), stim=(-5e5, 1.0, 0.0),
                         box_hi=(0.1, 0.1, 0.1), rel_tol=1e-8,
                         name="3D TT06-epi Rush-Larsen slab 2x0.7x0.3 cm h=0.01 (201x71x31 = 442,401 nodes)"),
    # the 2.1M-node TT06 slab: endo / mid / epi layers by thirds of z
    "tt06_slab_3d_large": dict(model=1, method=1, dt_ode=0.02, dt_pde=0.1, dim=3, h=0.0125,
                               size=(2.0, 2.0, 1.0), sigma=(1.75, 0.19, 0.19), stim=(-5e5, 1.0, 0.0),
                               box_hi=(0.1, 0.1, 0.1), rel_tol=1e-8, transmural=True,
                               name="3D TT06 Rush-Larsen slab 2x2x1 cm h=0.0125 (2,099,601 nodes), "
                                    "endo/mid/epi layers by z-thirds"),
    # the 2D LR91 forward-Euler sheet of 10,201 nodes
    "lr91_sheet_2d": dict(model=0, method=0, dt_ode=0.01, dt_pde=0.1, dim=2, h=0.01, size=(1.0, 1.0, 0.0),
                          sigma=(1.75, 1.75, 1.75), stim=(-5e5, 0.5, 0.0), box_hi=(0.0199, 1e9),
                          rel_tol=1e-8, name="2D LR91 forward-Euler sheet 1x1 cm h=0.01 (10,201 nodes)"),
}


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ode_bytes_per_node(model, w):
    s = 19 if model == 1 else 8
    # read+write S-1 states, read V (8) and the stimulus id (1), write Iion and z
    return 2 * (s - 1) * w + 8 + 1 + 2 * w


def csr_equivalent_bytes(model, mixed, its, sweeps, r=15):
    """The survey's algorithmic bytes per node-step of an assembled-CSR implementation
    (int32 columns, r entries per row): B_ode + B_rhs + k B_cg, with w = 8 (FP64) or 4
    (mixed inner iterations) and r*12 + 4 + 5*8 per FP64 refinement sweep.  The slab
    stencil moves far less (no matrix bytes); this is the figure to compare with a CSR
    solver's traffic, not this library's."""
    s = 19 if model == 1 else 8
    w = 4 if mixed else 8
    b_ode = (2 * (s - 1) + 2) * w
    b_rhs = r * (8 + 4) + 4 + 3 * 8
    b_cg = r * (w + 4) + 4 + 9 * w
    return b_ode + b_rhs + its * b_cg + (sweeps * (r * 12 + 4 + 5 * 8) if mixed else 0)


def cg_bytes(mixed, its, sweeps, pipelined=False):
    """Algorithmic bytes per node of one diffusion solve on the slab operator."""
    if mixed and pipelined:
        # residual pass: z32, V, class in; r64 and B r out.  per inner iteration only m = B w is
        # written and read back through the stencil (the other vectors stay in registers);
        # per sweep: e written and read, x and r64 read and written, B r written
        return (4 + 8 + 1 + 8 + 4) + its * (4 + 4) + sweeps * ((4 + 4) + 16 + 16 + 4)
    if not mixed:
        # phase 0: V, z, class in; r out.  per iteration: (r, p_old, cls) -> p_new ; (x, p_new, r, cls) -> (x, r)
        return (8 + 8 + 1 + 8) + its * ((8 + 8 + 1 + 8) + (8 + 8 + 8 + 1 + 16))
    per_sweep = (8 + 4 + 1 + 4 + 4) + (4 + 8 + 8)       # residual pass + x update
    per_it = (4 + 4 + 1 + 4) + (4 + 4 + 4 + 1 + 8)      # FP32 inner phases A and B
    return (8 + 4 + 1 + 4 + 4) + sweeps * per_sweep + its * per_it


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def transmural_cells(wl, xyz):
    """(param_set, param_table) of the workload's cells: the TT06 endo / mid / epi layers
    by thirds of z when the workload has them, else (None, None)."""
    if not wl.get("transmural"):
        return None, None
    from chaste_b200.heart import transmural_layers, transmural_param_table

    return transmural_layers(xyz[:, 2], wl["size"][2]), transmural_param_table()


def stimulated(wl, xyz):
    inside = np.ones(xyz.shape[0], bool)
    for d, hi in enumerate(wl["box_hi"][: wl["dim"]]):
        inside &= xyz[:, d] <= hi + 1e-12
    return np.where(inside, 0, -1).astype(np.int32)


def build_tissue(N, wl, precision, device, pc=None):
    from chaste_b200.heart import slab_coordinates

    cfg = N.default_config()
    cfg.model, cfg.ode_method = wl["model"], wl["method"]
    cfg.ode_time_step, cfg.pde_time_step = wl["dt_ode"], wl["dt_pde"]
    cfg.ksp_preconditioner = N.PC_JACOBI if pc is None else pc
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, wl["rel_tol"]
    cfg.precision = precision
    cfg.device = device
    t = N.Tissue(cfg)
    t.set_slab_mesh(wl["dim"], wl["h"], *wl["size"], sigma=wl["sigma"])
    xyz = slab_coordinates(wl["dim"], wl["h"], *wl["size"])
    pset, ptab = transmural_cells(wl, xyz)
    t.set_cells(param_set=pset, param_table=ptab)
    t.set_stimulus(stimulated(wl, xyz), [N.stimulus(N.STIM_SIMPLE, *wl["stim"])])
    return t


def start_steps(args, wl):
    return int(round(args.t_start_ms / wl["dt_pde"]))


def flush_l2(buf):
    buf.add_(1.0)


def run_ours(args, rank, world, device):
    import torch

    from chaste_b200 import _native as N
    from chaste_b200.build import build_native

    build_native()
    torch.cuda.set_device(device)
    wl = WORKLOADS[args.workload]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{device}")  # 256 MB > L2
    results = {}
    tissues = {label: build_tissue(N, wl, prec, device) for prec, label in ((0, "fp64"), (1, "mixed"))}
    for t in tissues.values():
        t.step(start_steps(args, wl))   # untimed: to the start of the timed window
        t.step(args.warmup)
    clk = ClockSampler(device)
    with clk:
        time.sleep(0.3)   # first nvidia-smi sample lands inside the timed region
        timed = {}
        for label, t in tissues.items():
            ms_total, its, sweeps = 0.0, 0, 0
            for _ in range(args.steps):
                flush_l2(flush)
                torch.cuda.synchronize()
                t.step(1)
                st = t.stats()
                ms_total += st.ms_last_call
                its += st.last_cg_iterations
                sweeps += st.refinement_sweeps
            timed[label] = (ms_total, its, sweeps)
    for label, t in tissues.items():
        ms_total, its, sweeps = timed[label]
        ms_ode = ms_cg = 0.0
        # per-phase device times on the same workload (kernel by kernel, no graph)
        k_prof = min(args.steps, 20)
        for _ in range(k_prof):
            flush_l2(flush)
            torch.cuda.synchronize()
            a, b = t.step_profiled(1)
            ms_ode += a
            ms_cg += b
        st = t.stats()
        results[label] = dict(tissue=t, ms_total=ms_total, its=its, sweeps=sweeps, ms_ode=ms_ode / k_prof,
                              ms_cg=ms_cg / k_prof, clocks=clk.summary(), steps_done=st.steps,
                              pipelined=st.pipelined_nodes_per_thread, cg_blocks=st.cg_blocks)
    n = results["fp64"]["tissue"].n
    # accuracy of the mixed path against FP64 at the same simulated time
    v64 = results["fp64"]["tissue"].voltage()
    v32 = results["mixed"]["tissue"].voltage()
    vm_err = float(np.abs(v64 - v32).max())
    # end-to-end through the C-ABI with host buffers: V in, step, V out every step, on a
    # fresh tissue advanced (untimed) to the same window the device-timed steps cover
    head = "mixed" if vm_err <= 0.5 else "fp64"
    te = build_tissue(N, wl, 1 if head == "mixed" else 0, device)
    te.step(start_steps(args, wl) + args.warmup)
    # page-locked host buffers (read by the ODE kernel through their device mapping;
    # the copy out is a DMA transfer)
    vin = torch.empty(te.n, dtype=torch.float64, pin_memory=True).numpy()
    vout = torch.empty(te.n, dtype=torch.float64, pin_memory=True).numpy()
    te.voltage(out=vin)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        # V in from the host, one step, V back to the host (cg_step_host: the step's ODE
        # reads V from the page-locked buffer as it computes; the caller passes back what
        # it got)
        te.step_host(vin, 1, vout, keep_history=True)
        vin, vout = vout, vin
    e2e_s = time.perf_counter() - t0
    out = {}
    for label, r in results.items():
        sec = r["ms_total"] / 1e3
        out[label] = dict(node_steps_per_s=n * args.steps / sec, ms_per_step=r["ms_total"] / args.steps,
                          mean_cg_iterations=r["its"] / args.steps, ms_ode=r["ms_ode"], ms_cg=r["ms_cg"],
                          sweeps=r["sweeps"] / args.steps, clocks=r["clocks"], pipelined=r["pipelined"],
                          cg_blocks=r["cg_blocks"])
    return dict(n=n, out=out, vm_err=vm_err, head=head, e2e_s=e2e_s, wl=wl)


# DRAM bytes (read + write) per launch of the dominant kernels from one ncu capture of
# the timed region's conditions (L2 flushed before the step, the window starting at
# --t-start-ms: `bench.py --profile mixed [--workload ...] --steps 1 --t-start-ms 0.5`,
# the 6th solve).  None where no such capture exists.
NCU_TRAFFIC = {
    ("tt06_slab_3d", "mixed", "cg_kernel"): 11.07e6,   # 10.21 MB read + 0.86 MB written, 163 us
    ("tt06_slab_3d_large", "mixed", "cg_kernel"): 124.7e6,   # 75.9 MB read + 48.8 MB written, 364 us
    ("lr91_sheet_2d", "mixed", "cg_kernel"): 0.296e6,   # 296 kB read + 256 B written, 99 us: all in L2
}


def roofline(res, args):
    peak, kind = hbm_peak()
    head = res["head"]
    o = res["out"][head]
    n = res["n"]
    mixed = head == "mixed"
    w = 4 if mixed else 8
    b_ode = ode_bytes_per_node(res["wl"]["model"], w) * n
    b_cg = cg_bytes(mixed, o["mean_cg_iterations"], o["sweeps"] if mixed else 0, o.get("pipelined", 0) > 0) * n
    ach_ode = b_ode / (o["ms_ode"] / 1e3) / 1e9
    ach_cg = b_cg / (o["ms_cg"] / 1e3) / 1e9
    dom = "ode" if o["ms_ode"] >= o["ms_cg"] else "cg"
    ach = ach_ode if dom == "ode" else ach_cg
    kern = "ode_kernel" if dom == "ode" else "cg_kernel"
    traffic = NCU_TRAFFIC.get((args.workload, head, kern))
    csr = csr_equivalent_bytes(res["wl"]["model"], mixed, o["mean_cg_iterations"], o["sweeps"] if mixed else 0,
                               r=15 if res["wl"]["dim"] == 3 else 7)
    return {"bound": "hbm", "kernel": kern, "achieved": round(ach, 1),
            "peak": peak, "peak_kind": kind, "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": traffic,
            "bytes_model": "matrix-free slab stencil: the bytes this kernel must move (states, vectors, "
                           "1-byte class per node; no matrix)",
            "csr_equivalent": {"bytes_per_node_step": csr,
                               "node_steps_per_s_at_peak": round(peak * 1e9 / csr, 1),
                               "note": "the survey's assembled-CSR byte model; a CSR solver at the HBM peak "
                                       "reaches this rate"},
            "per_kernel": {"ode_kernel": {"ms": round(o["ms_ode"], 4), "algorithmic_bytes": b_ode,
                                          "achieved_gbs": round(ach_ode, 1)},
                           "cg_kernel": {"ms": round(o["ms_cg"], 4), "algorithmic_bytes": int(b_cg),
                                         "achieved_gbs": round(ach_cg, 1)}}}


def cpu_baseline(wl, start_steps, seconds=15.0, threads=None):
    """The CPU oracle (a C++ restatement of Chaste's step) on the host cores: advanced
    untimed to the start of the timed window, then a bounded sample of steps."""
    from oracle import pyoracle as O

    threads = threads or os.cpu_count() or 1
    O.lib().orc_set_threads(threads)
    xyz, conn, _ = O.slab_mesh(wl["dim"], wl["h"], *wl["size"])
    cfg = O.Config(wl["model"], wl["method"], wl["dt_ode"], wl["dt_pde"], 1400.0, 1.0, O.PC_JACOBI, 0,
                   wl["rel_tol"], 0, 10000)
    sig = np.tile(np.asarray(wl["sigma"][: wl["dim"]]), (conn.shape[0], 1))
    pset, ptab = transmural_cells(wl, xyz)
    t = O.Tissue(cfg, wl["dim"], xyz, conn, sig, stimulated(wl, xyz), [O.simple(*wl["stim"])],
                 param_id=pset, param_table=ptab)
    ta = time.perf_counter()
    t.step(max(1, start_steps))
    t_adv = time.perf_counter() - ta
    k, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds and k < 200:
        t.step(1)
        k += 1
    dt = time.perf_counter() - t0
    t_ms = max(1, start_steps) * wl["dt_pde"]
    return {"value": xyz.shape[0] * k / dt, "unit": "node-steps/s", "cores": threads, "kind": "port",
            "sample": f"{k} PDE steps of the full {xyz.shape[0]}-node workload from t = {t_ms:g} ms "
                      f"(reached untimed in {t_adv:.1f} s), {dt:.1f} s, FP64, {threads} threads"}


def run_population(args):
    """Batched single cells: 8192 TT06 cells, six conductances scaled by lognormal(0, 0.2), 1-20 beats
    (uniform) at BCL 1000 ms, stimulus -52 uA/uF for 1 ms, Rush-Larsen dt 0.01 ms, FP64 and FP32 side by
    side, the engine the autotuner picks (one persistent launch in a CUDA graph, or one launch per beat).
    Metric: cell-steps/s over both precisions."""
    from chaste_b200 import _native as N
    from chaste_b200.build import build_native

    build_native()
    rng = np.random.default_rng(20261203)
    n = 8192
    params = np.ones((n, 9))
    params[:, :6] = np.exp(rng.normal(0.0, 0.2, size=(n, 6)))
    beats = rng.integers(1, 21, size=n).astype(np.int32)
    b = N.CellBatch(N.MODEL_TT06, beats, params)
    b.autotune(steps=2000)
    tpb, cpt = b.launch_shape()
    engine = "persistent" if b.engine() == N.BATCH_PERSISTENT else "per_beat"
    ms = b.run()
    r = b.results()
    steps = int(beats.sum()) * 100000
    k = r["n_ap64"]
    d_apd = [abs(r["apd64"][c, j] - r["apd32"][c, j]) for c in range(n) for j in range(min(k[c], r["apd64"].shape[1]))
             if r["apd64"][c, j] > 0 and r["apd32"][c, j] > 0]
    dv = [float(r["max_dv"][c, j]) for c in range(n) for j in range(int(beats[c]))]
    return {"metric": "single-cell population cell-steps/s (FP64 and FP32 copies of each cell in one launch)",
            "value": steps / (ms / 1e3), "unit": "cell-steps/s", "n_gpus": 1, "ms_total": ms,
            "higher_is_better": True, "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "8192 TT06-epi cells, lognormal(0,0.2) conductance scales, 1-20 beats at "
                                   "BCL 1000 ms, RL dt 0.01 ms", "cell_steps_per_precision": steps,
                       "engine": engine,
                       "threads_per_block": tpb if engine == "per_beat" else 128,
                       "cells_per_thread": cpt if engine == "per_beat" else 0.5,
                       "launch_shape": "autotuned over the per-beat kernel's threads per block x cells per "
                                       "thread and the persistent engine (one launch, work queue, two threads "
                                       "per cell)"},
            "apd90_fp32_vs_fp64_ms": {"max": max(d_apd), "mean": float(np.mean(d_apd)), "n": len(d_apd)},
            "per_beat_max_vm_error_mv": {"max": max(dv), "median": float(np.median(dv))}}


def run_cable(args):
    """Adjoint conductance fitting: LR91 cable of 1000 nodes, h 0.01 cm, dt 0.01 ms, 400 ms, stimulus at x = 0,
    20 evenly spaced probes, targets from scale factors drawn from lognormal(0, 0.3) over 4 regions x 7
    (six LR91 conductances + the region's tissue conductivity), loss = MSE of the probe traces, gradient by
    the adjoint with checkpoints every 200 steps; central differences (eps 1e-6) of all 28 parameters run
    as 56 cables in one launch.  Metric: gradient evaluations/s (forward with checkpoints + adjoint)."""
    import torch

    from chaste_b200 import fitting as F
    from chaste_b200.build import build_native

    build_native()
    cfg = F.default_cable_config()
    probes = F.even_probes(cfg.n_nodes, 20)
    cable = F.Cable(cfg, probes)
    rng = np.random.default_rng(20261203)
    truth = torch.tensor(np.exp(rng.normal(0.0, 0.3, size=(1, 4, cable.stride))), device="cuda")
    targets = cable.forward(truth, traces=True)["traces"][0].contiguous()
    p0 = torch.ones((1, 4, cable.stride), dtype=torch.float64, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    cable.forward(p0, targets, keep_checkpoints=True)   # warm-up
    torch.cuda.synchronize()
    ev[0].record()
    out = cable.forward(p0, targets, keep_checkpoints=True, iterations=True)
    ev[1].record()
    grad = cable.backward(p0, targets)
    ev[2].record()
    sets = np.repeat(np.ones((1, 4, cable.stride)), 2 * 4 * cable.stride, axis=0)
    for k in range(4 * cable.stride):
        sets[2 * k].flat[k] += 1e-6
        sets[2 * k + 1].flat[k] -= 1e-6
    d_sets = torch.tensor(sets, device="cuda")
    ev[3].record()
    fd_loss = cable.forward(d_sets, targets)["loss"]
    ev[4].record()
    torch.cuda.synchronize()
    t_fwd, t_adj, t_fd = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[3].elapsed_time(ev[4])
    g = grad.cpu().numpy()[0]
    fl = fd_loss.cpu().numpy()
    fd = ((fl[0::2] - fl[1::2]) / 2e-6).reshape(g.shape)
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())
    node_steps = cfg.n_nodes * cfg.n_steps
    line = {"metric": "cable gradient evaluations/s (forward with checkpoints + adjoint, 28 parameters)",
            "value": 1e3 / (t_fwd + t_adj), "unit": "gradients/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "LR91 cable 1000 nodes h=0.01 cm, dt 0.01 ms, 400 ms, 4 regions x 7 scales, "
                                   "20 probes, checkpoints every 200 steps, CG+Jacobi rtol 1e-8"},
            "ms_forward": t_fwd, "ms_adjoint": t_adj, "ms_fd_56_cables_one_launch": t_fd,
            "forward_node_steps_per_s": node_steps / (t_fwd / 1e3),
            "fd_cable_node_steps_per_s": 56 * node_steps / (t_fd / 1e3),
            "loss": float(out["loss"][0]), "cg_iterations_forward": int(out["iterations"][0]),
            "adjoint_vs_central_differences": {
                "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                "within_1e-4": int((rel <= 1e-4).sum()), "of": int(rel.size),
                "note": "LR91's h/j gate rates jump at V = -40 mV, so a 1e-6 change of a parameter that moves "
                        "activation times (g_Na, g_K1, g_b, sigma) crosses branch switches somewhere in the "
                        "cable; the forward-mode check of tests/test_gpu_cable.py covers those"}}
    if not args.no_cpu_baseline:
        from oracle import pyoracle as O

        from tests import cable_cases as CC

        # about one oracle forward of the whole cable (~8 s on one host core), fewer steps for a
        # smaller --cpu-seconds
        k = max(2000, min(cfg.n_steps, int(cfg.n_steps * args.cpu_seconds / 8.0)))
        cc = CC.PlainCableConfig(n_nodes=cfg.n_nodes, n_steps=k, n_regions=4)
        t0 = time.perf_counter()
        O.cable_run(CC.oracle_config(O, cc), np.ones((4, cable.stride)), probes, traces=True)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": cfg.n_nodes * k / dt, "unit": "node-steps/s (forward)", "cores": 1,
                                "kind": "port", "sample": f"{k} steps of the 1000-node cable forward, {dt:.1f} s"}
    return line


def mixed_population_runs(N, F, rng):
    """4096 LR91 single cells (Rush-Larsen dt 0.01 ms, 1-10 beats at BCL 500 ms, six conductances scaled by
    lognormal(0, 0.2), V sampled every 1 ms) and 64 LR91 cables (100-1000 nodes, 50-400 ms, 1-4 regions x 7
    lognormal(0, 0.2) scales, 5 probes sampled every 0.1 ms), every run of its own length."""
    cells, cables = [], []
    stim = N.stimulus(N.STIM_REGULAR, -25.5, 2.0, 5.0, 500.0)
    for _ in range(4096):
        cells.append((int(rng.integers(1, 11)) * 50000, np.exp(rng.normal(0.0, 0.2, size=6))))
    for _ in range(64):
        cfg = F.default_cable_config()
        cfg.n_nodes = int(rng.integers(100, 1001))
        cfg.n_steps = int(rng.integers(5, 41)) * 1000
        cfg.n_regions = int(rng.integers(1, 5))
        cables.append((cfg, np.exp(rng.normal(0.0, 0.2, size=(cfg.n_regions, 7))), F.even_probes(cfg.n_nodes, 5)))
    return stim, cells, cables


def run_mixed(args):
    """Single-cell and cable runs of LR91 with uneven lengths and their own parameters in ONE persistent
    launch (cg_runs_*), launch shape autotuned.  Metric: node-steps/s, a single cell counting as one node."""
    from chaste_b200 import _native as N
    from chaste_b200 import fitting as F
    from chaste_b200.build import build_native

    build_native()
    stim, cells, cables = mixed_population_runs(N, F, np.random.default_rng(20261204))
    pop = N.RunPopulation(N.MODEL_LR91)
    for steps, p in cells:
        pop.add_cell(N.ODE_RUSH_LARSEN, steps, 0.01, 100, p, stim)
    cids = [pop.add_cable(cfg, p, pr, 10) for cfg, p, pr in cables]
    tpb, cpt = pop.autotune(steps=2000)
    pop.run()                                   # warm-up
    ms = pop.run()
    cell_steps = sum(s for s, _ in cells)
    cable_steps = sum(cfg.n_nodes * cfg.n_steps for cfg, _, _ in cables)
    its = sum(pop.result(i)[2] for i in cids)
    line = {"metric": "mixed single-cell + cable population node-steps/s (one persistent launch)",
            "value": (cell_steps + cable_steps) / (ms / 1e3), "unit": "node-steps/s", "n_gpus": 1,
            "ms_total": ms, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "4096 LR91 cells RL dt 0.01 ms 1-10 beats of 500 ms + 64 LR91 cables of "
                                   "100-1000 nodes x 50-400 ms, dt 0.01 ms, CG+Jacobi rtol 1e-8",
                       "cell_steps": cell_steps, "cable_node_steps": cable_steps,
                       "cable_cg_iterations": int(its), "threads_per_block": tpb, "cells_per_thread": cpt}}
    if not args.no_cpu_baseline:
        from oracle import pyoracle as O

        from tests import cable_cases as CC

        # a bounded sample (about 10 s on one core): 150 cells for one beat each and the
        # first 10,000 steps of 4 cables
        t0 = time.perf_counter()
        n_cell = 0
        for steps, p in cells[:150]:
            y = O.initial_states(O.LR91)
            O.cell_compute(O.LR91, O.RL, y, 0.0, 500.0, 0.01, 1.0, O.regular(-25.5, 2.0, 500.0, 5.0), params=p)
            n_cell += 50000
        n_cab = 0
        for cfg, p, pr in cables[:4]:
            cc = CC.PlainCableConfig(n_nodes=cfg.n_nodes, n_steps=10000, n_regions=cfg.n_regions)
            O.cable_run(CC.oracle_config(O, cc), p, pr, traces=True)
            n_cab += cfg.n_nodes * 10000
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": (n_cell + n_cab) / dt, "unit": "node-steps/s", "cores": 1, "kind": "port",
                                "sample": f"150 cells x 1 beat and 4 cables x 10,000 steps of the population, {dt:.1f} s"}
    return line


def run_bidomain(args):
    """The bidomain step without a bath on the 2D LR91 sheet of 10,201 nodes (1 x 1 cm,
    h = 0.01 cm, 10,201 nodes, 20,402 unknowns), Chaste's default conductivities
    (intracellular 1.75 / 0.19, extracellular 7.0 / 2.365 mS/cm along x / y), forward Euler dt
    0.01 ms, PDE dt 0.1 ms, CG + Jacobi rtol 1e-8 with the null space of constant phi_e, FP64.
    Timed from t = --t-start-ms, L2 flushed before every step.  Metric: node-steps/s."""
    import torch

    from chaste_b200 import _native as N
    from chaste_b200.build import build_native

    build_native()
    dim, h, size = 2, 0.01, (1.0, 1.0, 0.0)
    xyz, conn = N.slab_mesh(dim, h, *size)
    si, se = (1.75, 0.19), (7.0, 2.365)
    cfg = N.default_config()
    cfg.model, cfg.ode_method = N.MODEL_LR91, N.ODE_FORWARD_EULER
    cfg.ode_time_step, cfg.pde_time_step = 0.01, 0.1
    cfg.ksp_preconditioner = N.PC_JACOBI
    cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, 1e-8
    sid = np.where(xyz[:, 0] <= 0.0199 + 1e-12, 0, -1).astype(np.int32)
    start = int(round(args.t_start_ms / 0.1))

    def tissue_at_window():
        tw = N.Tissue(cfg)
        tw.set_bidomain_mesh(xyz, conn, si, se)
        tw.set_cells()
        tw.set_stimulus(sid, [N.stimulus(N.STIM_SIMPLE, -5e5, 0.5, 0.0)])
        tw.step(start + args.warmup)
        return tw

    t = tissue_at_window()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda:0")
    ms, its = 0.0, 0
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        t.step(1)
        st = t.stats()
        ms += st.ms_last_call
        its += st.last_cg_iterations
    n = xyz.shape[0]
    # end to end on a fresh tissue at the same window
    te = tissue_at_window()
    vin = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    vout = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    te.voltage(out=vin)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        te.step_host(vin, 1, vout, keep_history=True)
        vin, vout = vout, vin
    e2e_s = time.perf_counter() - t0
    line = {"metric": "bidomain node-steps/s (FP64, null space of constant phi_e)",
            "value": n * args.steps / (ms / 1e3), "unit": "node-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "2D LR91 forward-Euler sheet 1x1 cm h=0.01 (10,201 nodes), bidomain, "
                                   "sigma_i (1.75, 0.19), sigma_e (7.0, 2.365)", "dt_ode_ms": 0.01,
                       "dt_pde_ms": 0.1, "solver": "CG+Jacobi rtol 1e-8, null space of constant phi_e",
                       "t_start_ms": args.t_start_ms, "l2": "flushed (256 MB write) before every timed step"},
            "mean_cg_iterations": its / args.steps,
            "e2e": {"value": n * args.steps / e2e_s, "unit": "node-steps/s", "h2d_bytes_per_step": 8 * n,
                    "d2h_bytes_per_step": 8 * n}}
    if not args.no_cpu_baseline:
        from oracle import pyoracle as O

        threads = os.cpu_count() or 1
        O.lib().orc_set_threads(threads)
        ocfg = O.Config(O.LR91, O.FE, 0.01, 0.1, 1400.0, 1.0, O.PC_JACOBI, 0, 1e-8, 0, 10000)
        sig_i = np.tile(np.asarray(si), (conn.shape[0], 1))
        o = O.Tissue(ocfg, dim, xyz, conn, sig_i, sid, [O.simple(-5e5, 0.5, 0.0)])
        o.set_bidomain(xyz, conn, sig_i, np.tile(np.asarray(se), (conn.shape[0], 1)))
        o.step(start)
        k, c0 = 0, time.perf_counter()
        while time.perf_counter() - c0 < args.cpu_seconds and k < 50:
            o.step(1)
            k += 1
        dt = time.perf_counter() - c0
        line["cpu_baseline"] = {"value": n * k / dt, "unit": "node-steps/s", "cores": threads, "kind": "port",
                                "sample": f"{k} PDE steps of the sheet from t = {args.t_start_ms:g} ms, {dt:.1f} s, "
                                          f"FP64, {threads} threads"}
    return line


def aggregate(dist, device, ms_step, e2e_s, n, steps, world):
    """Whole-job figures of N replicas: the max over ranks of the device step time and of
    the end-to-end time (a collective on `device`: cuda for NCCL, cpu for gloo), then
    throughput = all ranks' node-steps over that time."""
    if dist is not None and world > 1:
        import torch

        tt = torch.tensor([ms_step, e2e_s], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_step, e2e_s = tt.tolist()
    return {"ms_step": ms_step, "value": world * n / (ms_step / 1e3), "e2e_rate": world * n * steps / e2e_s}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tt06_slab_3d",
                    choices=sorted(WORKLOADS) + ["tt06_population", "lr91_cable_adjoint", "lr91_mixed_population",
                                                  "lr91_bidomain_sheet_2d"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--t-start-ms", type=float, default=10.0,
                    help="simulated time reached, untimed, before the warm-up and timed steps")
    ap.add_argument("--profile", choices=["fp64", "mixed", "fp64-bjacobi", "population", "runs"],
                    help="only build the workload's tissue in this precision (fp64-bjacobi: FP64 with Chaste's "
                         "default bjacobi preconditioner), advance it to --t-start-ms and take --steps steps "
                         "with an L2 flush before each (the program the ncu captures run)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.profile == "population":
        # the C3 population's launch shapes for --steps steps each (cg_batch_autotune), the
        # program the batch-kernel ncu capture runs
        from chaste_b200 import _native as N
        from chaste_b200.build import build_native

        build_native()
        rng = np.random.default_rng(20261203)
        params = np.ones((8192, 9))
        params[:, :6] = np.exp(rng.normal(0.0, 0.2, size=(8192, 6)))
        b = N.CellBatch(N.MODEL_TT06, rng.integers(1, 21, size=8192).astype(np.int32), params)
        tpb = b.autotune(steps=args.steps)
        print(json.dumps({"profile": "population", "threads_per_block": tpb, "shape": b.launch_shape()}), flush=True)
        return
    if args.profile == "runs":
        # the mixed population's launch shapes for --steps steps of every run (cg_runs_autotune),
        # the program the runs-kernel ncu capture runs
        from chaste_b200 import _native as N
        from chaste_b200 import fitting as F
        from chaste_b200.build import build_native

        build_native()
        stim, cells, cables = mixed_population_runs(N, F, np.random.default_rng(20261204))
        pop = N.RunPopulation(N.MODEL_LR91)
        for steps, p in cells:
            pop.add_cell(N.ODE_RUSH_LARSEN, steps, 0.01, 100, p, stim)
        for cfg, p, pr in cables:
            pop.add_cable(cfg, p, pr, 10)
        print(json.dumps({"profile": "runs", "shape": pop.autotune(steps=args.steps)}), flush=True)
        return
    if args.profile:
        import torch

        from chaste_b200 import _native as N
        from chaste_b200.build import build_native

        build_native()
        wl = WORKLOADS[args.workload]
        t = build_tissue(N, wl, 1 if args.profile == "mixed" else 0, 0,
                         pc=N.PC_BJACOBI if args.profile == "fp64-bjacobi" else None)
        t.step(start_steps(args, wl))
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda:0")
        ms = 0.0
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            t.step(1)
            ms += t.stats().ms_last_call
        torch.cuda.synchronize()
        st = t.stats()
        print(json.dumps({"profile": args.profile, "workload": args.workload, "steps": int(st.steps),
                          "last_cg_iterations": st.last_cg_iterations,
                          "ms_per_step": ms / max(1, args.steps)}), flush=True)
        return
    if args.workload == "tt06_population":
        print(json.dumps(run_population(args)), flush=True)
        return
    if args.workload == "lr91_cable_adjoint":
        print(json.dumps(run_cable(args)), flush=True)
        return
    if args.workload == "lr91_mixed_population":
        print(json.dumps(run_mixed(args)), flush=True)
        return
    if args.workload == "lr91_bidomain_sheet_2d":
        print(json.dumps(run_bidomain(args)), flush=True)
        return
    rank, world, local, dist = dist_setup(args)
    wl = WORKLOADS[args.workload]
    metric = "monodomain node-steps/s on 1 B200, mixed vs FP64 at <=0.5 mV Vm error"

    if args.impl == "reference":
        # Chaste's own CPU path (PETSc/MPI) cannot be built here; its restatement
        # (the oracle port) is timed on every host core, rank 0 only.
        if rank == 0:
            cb = cpu_baseline(wl, start_steps(args, wl), seconds=max(5.0, args.cpu_seconds))
            v = cb["value"]
            line = {"impl": "reference", "metric": metric, "value": v, "unit": "node-steps/s",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                    "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                    "config": {"workload": wl["name"], "t_start_ms": args.t_start_ms,
                               "window": "oracle port advanced untimed to t_start_ms, then timed"},
                    "cpu_baseline": cb,
                    "e2e": {"value": v, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch

    if dist:
        dist.barrier()
    res = run_ours(args, rank, world, local)
    head = res["head"]
    o = res["out"][head]
    agg = aggregate(dist, f"cuda:{local}", o["ms_per_step"], res["e2e_s"], res["n"], args.steps, world)
    ms_step, value, e2e_rate = agg["ms_step"], agg["value"], agg["e2e_rate"]
    if rank == 0:
        line = {
            "metric": metric, "value": value, "unit": "node-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 states+inner CG, f64 residual refinement" if head == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": wl["name"], "dt_ode_ms": wl["dt_ode"], "dt_pde_ms": wl["dt_pde"],
                       "solver": "CG+Jacobi rtol 1e-8 (PETSc convergence test)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "flushed (256 MB write) before every timed step",
                       "t_start_ms": args.t_start_ms,
                       "window": f"timed steps start at t = {args.t_start_ms + args.warmup * wl['dt_pde']:g} ms "
                                 f"(after {args.t_start_ms:g} ms untimed and {args.warmup} warm-up steps)",
                       "headline_precision": head},
            "fp64": res["out"]["fp64"], "mixed": res["out"]["mixed"],
            "mixed_vs_fp64": {"max_abs_vm_mv": res["vm_err"],
                              "speedup": res["out"]["fp64"]["ms_per_step"] / res["out"]["mixed"]["ms_per_step"]},
            "e2e": {"value": e2e_rate, "unit": "node-steps/s", "h2d_bytes_per_step": 8 * res["n"],
                    "d2h_bytes_per_step": 8 * res["n"],
                    "window": "the same steps as the device-timed ones, on a fresh tissue of the headline "
                              "precision; V read from a page-locked host buffer by the step's ODE kernel and "
                              "copied back to another every step (cg_step_host), L2 not flushed"},
            "gpu_launches": 2 * args.steps,
            "roofline": roofline(res, args),
            "clocks": o["clocks"],
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(wl, start_steps(args, wl), seconds=args.cpu_seconds)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
