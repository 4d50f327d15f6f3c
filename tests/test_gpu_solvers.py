"""GPU: the direct solvers of the library against each other and against
the oracle.

The default solver is the nested-dissection multifrontal LU; the
block-banded LU in the reference's unknown order is the alternative
(ErebusSolverOptions.direct_solver).  Both factor the same row-scaled
matrix without pivoting and refine to a relative residual of 1e-13, so
their solutions agree to 1e-9 relative L2 per field, and each agrees with
the oracle's SuperLU solve to 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["vx", "vy", "pr", "pf", "qxD", "qyD"]


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


@pytest.fixture(scope="module")
def state41(pkg, oracle):
    st = pkg.make_state("planetesimal_41")
    o = oracle.Oracle(st)
    for ts in (1, 2):
        o.step(ts)
    return st


def _hydro_pass(pkg, st, solver, fp32=0):
    s = st.copy()
    sim = pkg.Simulation(s)
    sim.set_solver_options(direct_solver=solver, factor_fp32=fp32)
    sim.markers_to_nodes(s.timesum)
    sim.gravity()
    dt, conv, stats = sim.hydromech_pass(s.dt, 1)
    sim.download()
    sim.close()
    return s, stats


def test_multifrontal_matches_band_and_oracle(pkg, oracle, built_lib, state41):
    mf, st_mf = _hydro_pass(pkg, state41, 0)
    bd, st_bd = _hydro_pass(pkg, state41, 1)
    assert st_mf.converged and st_mf.rel_residual <= 1e-13, st_mf.rel_residual
    assert st_bd.converged and st_bd.rel_residual <= 1e-13
    so = state41.copy()
    o = oracle.Oracle(so)
    o.markers_to_nodes(so.timesum)
    o.gravity()
    o.hydromech_pass(so.dt, 1)
    for k in FIELDS:
        assert rel_l2(mf.grid[k], bd.grid[k]) < 1e-9, k
        assert rel_l2(mf.grid[k], so.grid[k]) < 1e-8, k


def test_multifrontal_steps_141(pkg, built_lib):
    """Three timesteps of the 141 x 141 workload with each solver: the
    marker positions agree to 1e-10 relative."""
    out = {}
    for solver in (0, 1):
        st = pkg.make_state("planetesimal_141")
        sim = pkg.Simulation(st)
        sim.set_solver_options(direct_solver=solver)
        for ts in (1, 2, 3):
            sim.step(ts)
        sim.download()
        sim.close()
        out[solver] = st
    a, b = out[0], out[1]
    assert a.marknum == b.marknum
    n = a.marknum
    for k in ("xm", "ym"):
        d = np.max(np.abs(a.m[k][:n] - b.m[k][:n])) / np.max(np.abs(b.m[k][:n]))
        assert d < 1e-10, (k, d)
    for k in ("tk2", "pr", "vx"):
        assert rel_l2(a.grid[k], b.grid[k]) < 1e-8, k


def test_mixed_precision_matches_fp64_and_oracle(pkg, oracle, built_lib, state41):
    """Mixed precision: FP32 multifrontal factors (tensor-core products with
    three TF32 terms) inside FP64 refinement reach the same 1e-13 residual;
    the solution agrees with the FP64 factors to 1e-9 and with the oracle to
    1e-8 per field."""
    mx, st_mx = _hydro_pass(pkg, state41, 0, fp32=1)
    fp, st_fp = _hydro_pass(pkg, state41, 0, fp32=0)
    assert st_mx.converged and st_mx.rel_residual <= 1e-13, st_mx.rel_residual
    assert st_mx.iterations >= st_fp.iterations
    so = state41.copy()
    o = oracle.Oracle(so)
    o.markers_to_nodes(so.timesum)
    o.gravity()
    o.hydromech_pass(so.dt, 1)
    for k in FIELDS:
        assert rel_l2(mx.grid[k], fp.grid[k]) < 1e-9, k
        assert rel_l2(mx.grid[k], so.grid[k]) < 1e-8, k


def test_mixed_precision_steps_141(pkg, built_lib):
    """Three timesteps of the 141 x 141 workload with FP32 and with FP64
    factors: marker positions agree to 1e-10 relative, fields to 1e-8."""
    out = {}
    for fp32 in (0, 1):
        st = pkg.make_state("planetesimal_141")
        sim = pkg.Simulation(st)
        sim.set_solver_options(factor_fp32=fp32)
        for ts in (1, 2, 3):
            sim.step(ts)
        sim.download()
        sim.close()
        out[fp32] = st
    a, b = out[1], out[0]
    assert a.marknum == b.marknum
    n = a.marknum
    for k in ("xm", "ym"):
        d = np.max(np.abs(a.m[k][:n] - b.m[k][:n])) / np.max(np.abs(b.m[k][:n]))
        assert d < 1e-10, (k, d)
    for k in ("tk2", "pr", "vx"):
        assert rel_l2(a.grid[k], b.grid[k]) < 1e-8, k


@pytest.mark.parametrize("mixed", [0, 1])
def test_inverted_pivot_blocks_match_block_substitution_141(pkg, built_lib, mixed):
    """The cooperative solve levels in their two forms: inverted pivot blocks
    (default; at 141 x 141 levels 5-9 run cooperatively) and the chained block
    substitution (mf_block_substitution = 1).  Both solve to the 1e-13
    residual target, so three timesteps end within the solve tolerance of
    each other, in the FP64 path and in the mixed-precision Krylov mode."""
    opt = dict(krylov=1, precond_fp32=1) if mixed else {}
    out = []
    for sub in (0, 1):
        st = pkg.make_state("planetesimal_141")
        sim = pkg.Simulation(st)
        sim.set_solver_options(mf_block_substitution=sub, **opt)
        stats = [sim.step(ts) for ts in (1, 2, 3)]
        fs = sim.factor_stats(0)
        sim.download()
        sim.close()
        out.append((st, stats, fs))
    (a, sa, fa), (b, sb, fb) = out
    assert fa.levels == fb.levels
    assert [s.titer for s in sa] == [s.titer for s in sb]
    assert max(s.worst_rel_residual for s in sa + sb) <= 1e-10
    assert a.marknum == b.marknum
    n = a.marknum
    for k in ("xm", "ym"):
        d = np.abs(a.m[k][:n] - b.m[k][:n]).max() / np.abs(b.m[k][:n]).max()
        assert d <= 1e-10, k
    for k in FIELDS + ["tk2"]:
        assert rel_l2(a.grid[k], b.grid[k]) <= 1e-8, k
