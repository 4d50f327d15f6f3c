"""The nested-dissection multifrontal analysis, checked on the CPU.

tests/mf_check.cpp runs the device solver's block algorithm in plain host
loops over the plan that erebus.jl_b200/csrc/mf_plan.h builds (the same
header the CUDA solver includes).  Its solutions of the oracle's assembled
systems, row-scaled as the device scales them, are compared with SuperLU on
the same matrices: the no-pivot multifrontal LU reaches a relative residual
of 1e-9 or better in one solve, and the unknowns agree with SuperLU to 1e-8
relative L2 per field.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def mf(tmp_path_factory):
    d = tmp_path_factory.mktemp("mf")
    so = str(d / "mf_check.so")
    subprocess.check_call(["g++", "-O3", "-std=c++17", "-shared", "-fPIC", "-o", so,
                           os.path.join(HERE, "mf_check.cpp")])
    L = ctypes.CDLL(so)
    P = ctypes.c_void_p
    L.mf_check_solve.argtypes = [ctypes.c_int] * 4 + [P, P, ctypes.c_longlong, ctypes.c_int,
                                                      P, P, ctypes.c_int]
    L.mf_check_stats.argtypes = [ctypes.c_int] * 4 + [P]
    L.mf_check_tasks.argtypes = [ctypes.c_int, ctypes.c_int]
    return L


def _a(x):
    return x.ctypes.data_as(ctypes.c_void_p)


def _ell(A):
    """Row-scaled ELL arrays (cols -1 padded) of a CSR matrix, and the scale."""
    A = sp.csr_matrix(A)
    rs = np.asarray(abs(A).sum(axis=1)).ravel()
    rs[rs == 0] = 1.0
    As = sp.diags(1.0 / rs) @ A
    As = sp.csr_matrix(As)
    n = As.shape[0]
    ell = int(np.diff(As.indptr).max())
    cols = -np.ones((n, ell), np.int32)
    vals = np.zeros((n, ell))
    for r in range(n):
        lo, hi = As.indptr[r], As.indptr[r + 1]
        cols[r, :hi - lo] = As.indices[lo:hi]
        vals[r, :hi - lo] = As.data[lo:hi]
    return As, cols, vals, 1.0 / rs, ell


def _solve(mf, d, ny, nx, leaf, A, b, inverted=0):
    As, cols, vals, sc, ell = _ell(A)
    bs = b * sc
    x = np.zeros(A.shape[0])
    rc = mf.mf_check_solve(d, ny, nx, leaf, _a(cols), _a(vals), A.shape[0], ell, _a(bs), _a(x),
                           inverted)
    assert rc == 0, rc
    res = np.linalg.norm(bs - As @ x) / np.linalg.norm(bs)
    return x, res, As, bs


@pytest.fixture(scope="module")
def stepped(pkg, oracle):
    """planetesimal_41 after one oracle timestep (non-trivial fields)."""
    st = pkg.make_state("planetesimal_41")
    o = oracle.Oracle(st)
    o.step(1)
    o.markers_to_nodes(st.timesum)
    o.gravity()
    oracle.lib().oracle_bulk_viscosity(o.pP, o.pG)
    return st, o


@pytest.mark.parametrize("leaf", [4, 16, 32, 64])
@pytest.mark.parametrize("inverted", [0, 1])
def test_hydromech_matches_superlu(mf, stepped, leaf, inverted):
    """Both forms of the sweeps: block substitution, and the inverted pivot
    blocks of the device's cooperative levels (here on every front; the top
    fronts at 41 x 41 have four 64-wide pivot blocks)."""
    st, o = stepped
    A, b = o.hydromech_system(st.dt)
    g = st.g
    x, res, As, bs = _solve(mf, 6, g.Ny1, g.Nx1, leaf, A, b, inverted)
    ref = spla.splu(sp.csc_matrix(As)).solve(bs)
    assert res < 1e-9, res
    for t in range(6):
        e = np.linalg.norm(x[t::6] - ref[t::6]) / np.linalg.norm(ref[t::6])
        assert e < 1e-8, (t, e)


def test_thermal_and_gravity(mf, stepped):
    st, o = stepped
    g = st.g
    for A, b in (o.thermal_system(st.dt), o.gravity_system()):
        for leaf in (16, 64):
            x, res, As, bs = _solve(mf, 1, g.Ny1, g.Nx1, leaf, A, b)
            ref = spla.spsolve(sp.csc_matrix(As), bs)
            assert res < 1e-12, (leaf, res)
            assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-10


@pytest.mark.parametrize("ny,nx,d,leaf", [(9, 13, 2, 4), (20, 7, 3, 6), (1, 30, 1, 4),
                                          (33, 33, 1, 1), (40, 44, 6, 16)])
@pytest.mark.parametrize("inverted", [0, 1])
def test_rectangles_random(mf, ny, nx, d, leaf, inverted):
    """Rectangular grids and other block sizes: a random diagonally dominant
    matrix with the 3 x 3 node coupling pattern."""
    rng = np.random.default_rng(ny * 1000 + nx)
    n = ny * nx * d
    rows, cols = [], []
    for j in range(nx):
        for i in range(ny):
            for dj in (-1, 0, 1):
                for di in (-1, 0, 1):
                    ii, jj = i + di, j + dj
                    if 0 <= ii < ny and 0 <= jj < nx:
                        for a in range(d):
                            for c in range(d):
                                rows.append((j * ny + i) * d + a)
                                cols.append((jj * ny + ii) * d + c)
    vals = rng.standard_normal(len(rows))
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A = A + sp.diags(np.asarray(abs(A).sum(axis=1)).ravel() + 1.0)
    b = rng.standard_normal(n)
    x, res, As, bs = _solve(mf, d, ny, nx, leaf, A, b, inverted)
    assert res < 1e-12, res


def test_stats_of_the_workloads(mf):
    """Tree sizes of the three grids the benchmarks use (the storage grows
    like N log N, not like the band's N^1.5)."""
    out = np.zeros(5, np.int64)
    sizes = {}
    for n1 in (42, 142, 402):
        assert mf.mf_check_stats(6, n1, n1, 16, _a(out)) == 0
        sizes[n1] = out.copy()
    assert sizes[142][2] * 8 < 2.5e9            # bytes of front storage at 141 x 141
    assert sizes[402][2] * 8 < 40e9             # and at 401 x 401


def test_cooperative_solve_task_maps(mf):
    """The task decoders of the cooperative solve levels (mf_tasks.h, compiled
    into the device solver as they are here): for every front shape up to
    Kt = 80 row blocks and 90 update row blocks, and every front of the three
    workloads' plans, each phase (F1, F2, B1, B2; F2 and B2 one task per row
    and in 8-tile chunks) covers its tiles exactly once, and every partial-sum
    slot is used once and lies inside the front's storage."""
    assert mf.mf_check_tasks(80, 90) == 0
