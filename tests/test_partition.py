"""The multi-rank slab decomposition (chaste_b200/partition.py): rows in PETSc's
contiguous ranges, halo exchange before each operator application, all-reduced
inner products.  On CPU, gloo ranks with the oracle backend reproduce the
single-domain oracle solve (Vm within 1e-12 relative, the same CG iteration counts);
on a GPU, two ranks with the CUDA backend reproduce cg_step on the whole slab."""
import os
import socket
import types

import numpy as np
import pytest

from tests import tissue_cases as TC

CASES = {
    # 21 x 11 sheet: halo NX + 1 = 22 rows
    "lr91_2d": dict(TC.LR91_2D, size=(0.2, 0.1, 0.0), box_hi=(0.0199, 1e9)),
    # 11 x 6 x 4 slab: halo NX*NY + NX + 1 = 78 rows
    "tt06_3d": dict(TC.TT06_3D, size=(0.1, 0.05, 0.03), box_hi=(0.03, 0.03, 0.03)),
}
STEPS = {"lr91_2d": 20, "tt06_3d": 12}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_rank(rank, world, port, case_name, out):
    import datetime

    import torch.distributed as dist

    from chaste_b200.partition import PartitionedSlabTissue
    from oracle import pyoracle as O
    from tests.partition_cases import OraclePartition

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        case = CASES[case_name]
        cfg = types.SimpleNamespace(ksp_preconditioner=1, use_absolute_tolerance=0,
                                    ksp_tolerance=case.get("rel_tol", 1e-8), max_iterations=10000)
        t = PartitionedSlabTissue(OraclePartition(O, case, rank, world, cfg))
        t.step(STEPS[case_name])
        v = t.gather_voltage()
        if rank == 0:
            np.savez(out, v=v, its=np.asarray(t.iterations))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run_ranks(target, world, *args):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port) + args) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


def test_row_ranges_are_petsc_decide():
    from chaste_b200.partition import row_range

    for n, w in ((10, 3), (264, 2), (7, 7), (442401, 8)):
        ranges = [row_range(n, r, w) for r in range(w)]
        assert ranges[0][0] == 0 and ranges[-1][1] == n
        assert all(ranges[k][1] == ranges[k + 1][0] for k in range(w - 1))
        sizes = [hi - lo for lo, hi in ranges]
        assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


@pytest.mark.parametrize("case_name,world", [("lr91_2d", 2), ("tt06_3d", 2), ("tt06_3d", 3)])
def test_partitioned_oracle_solve_matches_single_domain(oracle, tmp_path, case_name, world):
    out = str(tmp_path / "v.npz")
    _run_ranks(_oracle_rank, world, case_name, out)
    got = np.load(out)
    o, _ = TC.make_oracle(oracle, **CASES[case_name])
    its = o.step(STEPS[case_name])
    ref = o.voltage()
    assert np.max(np.abs(got["v"] - ref) / np.maximum(np.abs(ref), 1.0)) <= 1e-12
    assert np.array_equal(got["its"], its)


def _gpu_rank(rank, world, port, case_name, out):
    import datetime

    import torch.distributed as dist

    from chaste_b200 import _native as N
    from chaste_b200.partition import NativePartition, PartitionedSlabTissue

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        case = CASES[case_name]
        cfg = N.default_config()
        cfg.model, cfg.ode_method = case["model"], case["method"]
        cfg.ode_time_step, cfg.pde_time_step = case["dt_ode"], case["dt_pde"]
        cfg.ksp_preconditioner = N.PC_JACOBI
        cfg.use_absolute_tolerance, cfg.ksp_tolerance = 0, 1e-8
        part = NativePartition(cfg, case["dim"], case["h"], case["size"], case["sigma"], rank, world)
        from oracle import pyoracle as O

        xyz, _, _ = O.slab_mesh(case["dim"], case["h"], *case["size"])
        part.set_cells()
        part.set_stimulus(TC.slab_stim_ids(xyz, case["box_hi"]), [N.stimulus(N.STIM_SIMPLE, *case["stim"])])
        t = PartitionedSlabTissue(part)
        t.step(STEPS[case_name])
        v = t.gather_voltage()
        if rank == 0:
            np.savez(out, v=v, its=np.asarray(t.iterations))
        dist.barrier()
        part.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("case_name,world", [("lr91_2d", 2), ("tt06_3d", 2), ("tt06_3d", 3)])
def test_partitioned_gpu_solve_matches_whole_slab(native, tmp_path, case_name, world):
    """Ranks as processes sharing the one GPU of this run: each rank's kernels are
    independent launches; the ranks meet only on the host (gloo), between kernels."""
    out = str(tmp_path / "v.npz")
    _run_ranks(_gpu_rank, world, case_name, out)
    got = np.load(out)
    g, _ = TC.make_gpu(native, **CASES[case_name])
    g.step(STEPS[case_name])
    ref = g.voltage()
    assert np.max(np.abs(got["v"] - ref) / np.maximum(np.abs(ref), 1.0)) <= 1e-12
    its = g.iteration_history(STEPS[case_name])
    assert np.abs(got["its"] - its).max() <= 1
