"""Ensemble of planetesimals of uneven sizes stepped concurrently (one host
thread and stream per body, solver kernels on one shared stream): every body
ends bit for bit where it ends when stepped alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_concurrent_bodies_equal_bodies_alone(pkg, built_lib):
    from erebus_b200.ensemble import Ensemble, ensemble_states
    kw = dict(seed=7, side_min=31, side_max=61)
    together = ensemble_states(4, **kw)
    alone = ensemble_states(4, **kw)
    assert len({st.p.Nx for st in together}) > 1        # uneven sizes
    ens = Ensemble(together)
    stats = ens.run(2)
    ens.download()
    ens.close()
    assert all(len(s) == 2 for s in stats)
    for a, b in zip(together, alone):
        sim = pkg.Simulation(b)
        for ts in (1, 2):
            sim.step(ts)
        sim.download()
        sim.close()
        assert (a.marknum, a.dt, a.timesum) == (b.marknum, b.dt, b.timesum)
        n = a.marknum
        for k in ("xm", "ym", "tkm", "phim", "sxxm"):
            np.testing.assert_array_equal(a.m[k][:n], b.m[k][:n], err_msg=k)
        for k in ("tk2", "vx", "vy", "pr", "pf", "FI"):
            np.testing.assert_array_equal(a.grid[k], b.grid[k], err_msg=k)
