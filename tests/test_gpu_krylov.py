"""GPU: the mixed-precision Krylov mode of the solves.

With ErebusSolverOptions.krylov = 1 every solve is a flexible GMRES in FP64
preconditioned by the multifrontal LU of an earlier matrix of the same
system, applied from an FP32 copy of its FP64 factors (precond_fp32 = 1);
the factors are refreshed when a solve costs as much as the average solve
since the last factorisation, the factorisation included (its cost in
iterations modelled from the plan), or with refactor_iterations = n > 0
when a solve needed more than n iterations.  The solves meet the plain path's residual
target (1e-13), so the results agree with the oracle's SuperLU solves to the
same tolerances as the plain path (1e-8 relative L2 per field, marker
positions 1e-10), and with the plain FP64 GPU path to 1e-8.
"""
import numpy as np
import pytest

from parity_util import assert_step_parity, rel_l2, rel_linf

pytestmark = pytest.mark.gpu

MIXED = dict(krylov=1, precond_fp32=1)


@pytest.fixture(scope="module")
def state41(pkg, oracle):
    st = pkg.make_state("planetesimal_41")
    o = oracle.Oracle(st)
    for ts in (1, 2):
        o.step(ts)
    return st


def test_krylov_hydro_pass_matches_oracle(pkg, oracle, built_lib, state41):
    s = state41.copy()
    sim = pkg.Simulation(s)
    sim.set_solver_options(**MIXED)
    sim.markers_to_nodes(s.timesum)
    sim.gravity()
    dt, conv, stats = sim.hydromech_pass(s.dt, 1)
    sim.download()
    sim.close()
    assert stats.converged and stats.rel_residual <= 1e-13, stats.rel_residual
    so = state41.copy()
    o = oracle.Oracle(so)
    o.markers_to_nodes(so.timesum)
    o.gravity()
    o.hydromech_pass(so.dt, 1)
    for k in ["vx", "vy", "pr", "pf", "qxD", "qyD"]:
        assert rel_l2(s.grid[k], so.grid[k]) < 1e-8, k


def test_krylov_timesteps_match_oracle(pkg, oracle, built_lib):
    """Timesteps 1-4 of the 41 x 41 workload, device (mixed Krylov mode)
    against the oracle, each step compared on the same input state."""
    st = pkg.make_state("planetesimal_41")
    so = st.copy()
    o = oracle.Oracle(so)
    sg = st.copy()
    sim = pkg.Simulation(sg)
    sim.set_solver_options(**MIXED)
    for ts in (1, 2, 3, 4):
        ostats = o.step(ts)
        gs = sim.step(ts)
        sim.download()
        assert_step_parity(sg, so, gs, ostats, what="timestep %d" % ts)
        # continue both from the oracle's state, so each step is compared on
        # the same input
        for k in so.m:
            sg.m[k][...] = so.m[k]
        for k in so.grid:
            sg.grid[k][...] = so.grid[k]
        sg.marknum, sg.dt, sg.timesum = so.marknum, so.dt, so.timesum
        sim.upload()
    sim.close()


def _run(pkg, name, steps, **opt):
    st = pkg.make_state(name)
    sim = pkg.Simulation(st)
    sim.set_solver_options(**opt)
    stats = [sim.step(ts) for ts in range(1, steps + 1)]
    fs = sim.factor_stats(0)
    sim.download()
    sim.close()
    return st, stats, fs


def test_krylov_lagged_factors_141(pkg, built_lib):
    """Six timesteps of the 141 x 141 workload: the Krylov mode factors the
    Stokes-Darcy matrix fewer times than it solves, and ends where the plain
    FP64 path ends (positions 1e-10, fields 1e-8); two runs are identical."""
    a, sa, fa = _run(pkg, "planetesimal_141", 6, **MIXED)
    b, sb, fb = _run(pkg, "planetesimal_141", 6)
    c, _, _ = _run(pkg, "planetesimal_141", 6, **MIXED)
    assert fa.factorizations < sum(s.titer for s in sa), fa.factorizations
    assert fa.krylov_iterations > 0
    assert [s.titer for s in sa] == [s.titer for s in sb]
    assert a.marknum == b.marknum
    n = a.marknum
    for k in ("xm", "ym"):
        assert rel_linf(a.m[k][:n], b.m[k][:n]) < 1e-10, k
        np.testing.assert_array_equal(a.m[k][:n], c.m[k][:n])
    for k in ("tk2", "pr", "pf", "vx", "vy", "qxD", "qyD"):
        assert rel_l2(a.grid[k], b.grid[k]) < 1e-8, k
        np.testing.assert_array_equal(a.grid[k], c.grid[k])
    assert max(s.worst_rel_residual for s in sa) <= 1e-10


def test_krylov_fixed_refactor_threshold(pkg, built_lib):
    """The fixed-threshold rule (refactor_iterations = 4) on the 141 x 141
    workload: it factors at least as often as the cost rule and ends at the
    same state to the solve tolerance."""
    a, sa, fa = _run(pkg, "planetesimal_141", 4, **MIXED)
    b, sb, fb = _run(pkg, "planetesimal_141", 4, refactor_iterations=4, **MIXED)
    assert fb.factorizations >= fa.factorizations
    assert [s.titer for s in sa] == [s.titer for s in sb]
    n = a.marknum
    for k in ("xm", "ym"):
        assert rel_linf(a.m[k][:n], b.m[k][:n]) < 1e-10, k
    for k in ("tk2", "pr", "pf", "vx", "vy"):
        assert rel_l2(a.grid[k], b.grid[k]) < 1e-8, k
