"""GPU parity at the 401 x 401 workload (2,560,000 markers, rock viscosity
log-uniform 1e17-1e23 Pa s, a 1e6 contrast): timesteps 1 and 2 with the
plain FP64 solves and with the mixed-precision Krylov mode (whose second
timestep solves with the factors of the first: lagged preconditioner),
against the oracle.

The oracle needs about 10 minutes for the two timesteps, so its results are
a committed fixture (tests/golden/planetesimal_401_steps.npz, made by
tests/golden/make_planetesimal_401.py from the same seeded initial state):
every 7th P node of the solution fields and every 64th marker after each
timestep.  The device runs advance their own state (free-running) and must
match the fixture after each timestep within the library's parity bounds --
solution fields to 1e-8 relative L2 over the sample, marker positions to
1e-10 relative -- with the same thermochemical and plastic iteration counts
and dt, and every solve's scaled residual at most 1e-10.  The two device
runs are also compared with each other over the full fields.
"""
import os

import numpy as np
import pytest

from parity_util import rel_l2, rel_linf

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "planetesimal_401_steps.npz")
FIELDS = ["vx", "vy", "pr", "pf", "qxD", "qyD", "tk2"]


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(FIXTURE))


@pytest.fixture(scope="module")
def runs(pkg, built_lib):
    """Per mode: [(state copy, ErebusStepStats)] after timesteps 1 and 2, and
    the Stokes-Darcy factorisation count."""
    out = {}
    for mode, opt in (("fp64", {}), ("mixed", dict(krylov=1, precond_fp32=1))):
        st = pkg.make_state("planetesimal_401")
        sim = pkg.Simulation(st)
        if opt:
            sim.set_solver_options(**opt)
        steps = []
        for ts in (1, 2):
            gs = sim.step(ts)
            sim.download()
            steps.append((st.copy(), gs))
        nfac = sim.factor_stats(0).factorizations
        sim.close()
        out[mode] = (steps, nfac)
    return out


@pytest.mark.parametrize("ts", [1, 2])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_401_matches_oracle(golden, runs, mode, ts):
    st, gs = runs[mode][0][ts - 1]
    pre = "s%d_" % ts
    assert gs.titer == int(golden[pre + "titer"])
    assert gs.iplast_total == int(golden[pre + "iplast_total"])
    assert gs.marknum == int(golden[pre + "marknum"])
    assert abs(gs.dt - float(golden[pre + "dt"])) <= 1e-10 * float(golden[pre + "dt"])
    assert gs.worst_rel_residual <= 1e-10, gs.worst_rel_residual
    ns, ms = int(golden["node_stride"]), int(golden["marker_stride"])
    for k in FIELDS:
        got = np.asfortranarray(st.grid[k]).ravel(order="F")[::ns]
        e = rel_l2(got, golden[pre + "grid_" + k])
        assert e <= 1e-8, (mode, ts, k, e)
    n = st.marknum
    for k in ("xm", "ym"):
        e = rel_linf(st.m[k][:n][::ms], golden[pre + "m_" + k])
        assert e <= 1e-10, (mode, ts, k, e)
    for k in ("tkm", "phim", "XWsolidm0"):
        e = rel_linf(st.m[k][:n][::ms], golden[pre + "m_" + k])
        assert e <= 1e-8, (mode, ts, k, e)
    np.testing.assert_array_equal(st.m["tm"][:n][::ms], golden[pre + "m_tm"])


def test_401_mixed_matches_fp64_and_lags(runs):
    (steps_m, nfac_m), (steps_f, nfac_f) = runs["mixed"], runs["fp64"]
    for (a, _), (b, _) in zip(steps_m, steps_f):
        for k in FIELDS:
            assert rel_l2(a.grid[k], b.grid[k]) <= 1e-8, k
        n = b.marknum
        for k in ("xm", "ym"):
            assert rel_linf(a.m[k][:n], b.m[k][:n]) <= 1e-10, k
    # the plain path factors every new matrix (one per timestep here), the
    # Krylov mode keeps the first factors as the second timestep's
    # preconditioner unless they stop paying
    assert nfac_m <= nfac_f
