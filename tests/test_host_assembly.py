"""Host FE assembly of the library (compiled here with g++) against the oracle's matrices,
and the matrix-free slab stencil against the assembled rows."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("probe") / "libprobe.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", "-o", out,
                    os.path.join(ROOT, "tests", "cpp", "host_probe.cpp"),
                    os.path.join(ROOT, "chaste_b200", "csrc", "host", "assemble.cpp")], check=True)
    return C.CDLL(out)


def run_probe(L, dim, h, size, sigma, ms):
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    n, nnz = C.c_int(), C.c_int()
    sig = np.asarray(sigma, float)
    z = lambda a: a.ctypes.data_as(dp if a.dtype == np.float64 else ip)  # noqa: E731
    rc = L.probe_slab(dim, C.c_double(h), C.c_double(size[0]), C.c_double(size[1]), C.c_double(size[2]), z(sig),
                      C.c_double(ms), C.byref(n), C.byref(nnz), None, None, None, None, None, None, None, None,
                      None, None, None)
    assert rc == 0
    rp = np.zeros(n.value + 1, np.int32)
    cols = np.zeros(nnz.value, np.int32)
    a = np.zeros(nnz.value)
    m = np.zeros(nnz.value)
    ok, noff, ncls = C.c_int(), C.c_int(), C.c_int()
    offs = np.zeros(27, np.int32)
    at = np.zeros(27 * 27)
    mt = np.zeros(27 * 27)
    cls = np.zeros(n.value, np.int32)
    L.probe_slab(dim, C.c_double(h), C.c_double(size[0]), C.c_double(size[1]), C.c_double(size[2]), z(sig),
                 C.c_double(ms), C.byref(n), C.byref(nnz), z(rp), z(cols), z(a), z(m), C.byref(ok), C.byref(noff),
                 C.byref(ncls), z(offs), z(at), z(mt), z(cls))
    return dict(rp=rp, cols=cols, a=a, m=m, ok=ok.value, offs=offs[: noff.value],
                at=at[: ncls.value * noff.value].reshape(ncls.value, noff.value),
                mt=mt[: ncls.value * noff.value].reshape(ncls.value, noff.value), cls=cls)


CASES = [(1, 0.01, (0.1, 0.0, 0.0), (0.0005, 0, 0), 1.0 / 0.01),
         (2, 0.01, (0.3, 0.3, 0.0), (1.75, 1.75, 0), 1400.0 / 0.01),
         (3, 0.01, (0.1, 0.1, 0.1), (1.75, 1.75, 1.75), 1400.0 / 0.01),
         (3, 0.01, (0.2, 0.07, 0.03), (1.75, 0.19, 0.19), 1400.0 / 0.1)]


@pytest.mark.parametrize("dim,h,size,sigma,ms", CASES)
def test_library_assembly_matches_oracle(probe, oracle, dim, h, size, sigma, ms):
    O = oracle
    r = run_probe(probe, dim, h, size, sigma, ms)
    xyz, conn, _ = O.slab_mesh(dim, h, *size)
    dt = 1.0 / ms
    cfg = O.Config(O.LR91, O.FE, 0.01, dt, 1.0, 1.0, O.PC_JACOBI, 1, 2e-4, 0, 10000)
    t = O.Tissue(cfg, dim, xyz, conn, np.tile(np.asarray(sigma[:dim], float), (conn.shape[0], 1)))
    rp, cols, a = t.matrix(0)
    _, _, m = t.matrix(1)
    assert np.array_equal(rp, r["rp"]) and np.array_equal(cols, r["cols"])
    assert np.max(np.abs(a - r["a"])) <= 1e-13 * np.abs(a).max()
    assert np.max(np.abs(m - r["m"])) <= 1e-13 * np.abs(m).max()


@pytest.mark.parametrize("dim,h,size,sigma,ms", CASES)
def test_slab_stencil_reproduces_every_row(probe, dim, h, size, sigma, ms):
    r = run_probe(probe, dim, h, size, sigma, ms)
    assert r["ok"] == 1
    n = r["rp"].size - 1
    assert len(r["offs"]) == {1: 3, 2: 7, 3: 15}[dim] or (dim == 2 and len(r["offs"]) <= 9)
    for i in range(n):
        c = r["cls"][i]
        for k in range(r["rp"][i], r["rp"][i + 1]):
            o = list(r["offs"]).index(r["cols"][k] - i)
            assert abs(r["at"][c, o] - r["a"][k]) <= 1e-12 * np.abs(r["at"][c]).max()
            assert abs(r["mt"][c, o] - r["m"][k]) <= 1e-12 * np.abs(r["mt"][c]).max()
        # no coefficient outside the row's pattern
        nz = set(r["cols"][r["rp"][i]:r["rp"][i + 1]] - i)
        for o, off in enumerate(r["offs"]):
            if off not in nz:
                assert r["at"][c, o] == 0.0 and r["mt"][c, o] == 0.0


@pytest.mark.parametrize("dim,size", [(1, (0.1, 0.0, 0.0)), (2, (0.2, 0.1, 0.0)), (3, (0.1, 0.05, 0.03))])
def test_library_slab_mesh_matches_oracle(oracle, native, dim, size):
    """cg_slab_mesh (host only, loads the library without a GPU) gives the oracle's
    ConstructRegularSlabMesh node order and elements bit for bit."""
    xyz, conn = native.slab_mesh(dim, 0.01, *size)
    oxyz, oconn, _ = oracle.slab_mesh(dim, 0.01, *size)
    assert np.array_equal(xyz, oxyz)
    assert np.array_equal(conn, oconn)
