"""erebus_step_host: a timestep on host arrays, with part of the copy-out
overlapping the timestep, gives bit for bit the state of upload + erebus_step
+ download, also when replenishment appends markers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hole(pkg):
    """planetesimal_41 with a band of cells emptied, so replenishment adds
    markers at the first timestep."""
    st = pkg.make_state("planetesimal_41")
    n, g = st.marknum, st.g
    keep = ~((st.m["xm"][:n] > 20 * g.dx) & (st.m["xm"][:n] < 21 * g.dx))
    for k in st.m:
        st.m[k][: keep.sum()] = st.m[k][:n][keep]
    st.marknum = int(keep.sum())
    return st


def test_step_host_equals_step_and_download(pkg, built_lib):
    a, b = _hole(pkg), _hole(pkg)
    n0 = a.marknum
    sa = pkg.Simulation(a)
    sb = pkg.Simulation(b)
    for ts in (1, 2):
        sa.step_host(ts)
        sb.step(ts)
    sb.download()
    sa.close()
    sb.close()
    assert a.marknum == b.marknum > n0          # markers were appended
    assert (a.dt, a.timesum) == (b.dt, b.timesum)
    n = a.marknum
    for k in a.m:
        if k == "etasolidm_m" and not a.p.per_marker_eta:
            continue
        np.testing.assert_array_equal(a.m[k][:n], b.m[k][:n], err_msg=k)
    for k in a.grid:
        np.testing.assert_array_equal(a.grid[k], b.grid[k], err_msg=k)


def test_step_host_rejects_bad_marker_types(pkg, built_lib):
    st = pkg.make_state("planetesimal_41")
    sim = pkg.Simulation(st)
    st.m["tm"][5] = 7
    with pytest.raises(pkg.ErebusError) as e:
        sim.step_host(1)
    assert e.value.code == 1
    st.m["tm"][5] = 1
    sim.step_host(1)                            # the state is still usable
    sim.close()


def test_host_syncs_are_counted(pkg, built_lib):
    """erebus_host_syncs counts the host's waits on the state's streams: a
    timestep waits where the reference decides (solve and iteration
    convergence, dt, the marker count), a few dozen times, not per kernel."""
    st = pkg.make_state("planetesimal_41")
    sim = pkg.Simulation(st)
    sim.step(1)
    y0, l0 = sim.host_syncs(), sim.kernel_launches()
    sim.step(2)
    dy, dl = sim.host_syncs() - y0, sim.kernel_launches() - l0
    sim.close()
    assert 0 < dy < dl, (dy, dl)
    assert dy < 200, dy
