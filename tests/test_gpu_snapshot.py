"""The asynchronous snapshot behind save_state (src/Erebus.jl:5718-5960,
E:7106): erebus_snapshot_begin stages the state in stream order and copies it
out while later timesteps run; the result equals a synchronous download taken
at the same point."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_snapshot_overlaps_next_step(pkg, built_lib):
    st = pkg.make_state("planetesimal_41")
    sim = pkg.Simulation(st)
    sim.step(1)
    want = sim.download().copy()
    buf = pkg.HostState(st.p, st.capacity, pinned=True)
    sim.snapshot_begin(buf)
    with pytest.raises(pkg.ErebusError):          # one snapshot at a time
        sim.snapshot_begin(pkg.HostState(st.p, st.capacity))
    sim.step(2)
    snap = sim.snapshot_wait()
    with pytest.raises(pkg.ErebusError):          # nothing pending any more
        sim.snapshot_wait()
    after = sim.download()
    sim.close()
    assert snap is buf
    assert (snap.marknum, snap.dt, snap.timesum) == (want.marknum, want.dt, want.timesum)
    n = want.marknum
    for k in want.m:
        if k == "etasolidm_m":
            continue
        np.testing.assert_array_equal(snap.m[k][:n], want.m[k][:n], err_msg=k)
    for k in want.grid:
        np.testing.assert_array_equal(snap.grid[k], want.grid[k], err_msg=k)
    # the second timestep moved on from the snapshot
    assert after.timesum > snap.timesum
    assert not np.array_equal(after.m["xm"][:n], snap.m["xm"][:n])


def test_run_simulation_writes_snapshots(pkg, built_lib, tmp_path):
    from erebus_b200.output import load_state, output_file
    st = pkg.make_state("planetesimal_41")
    ref = st.copy()
    stats = pkg.run_simulation(st, 4, output_path=str(tmp_path), savematstep=2)
    assert len(stats) == 4
    assert sorted(p.name for p in tmp_path.iterdir()) == ["output_00002.npz",
                                                          "output_00004.npz"]
    last = load_state(output_file(str(tmp_path), 4))
    assert last["timestep"] == 4 and last["marknum"] == st.marknum
    assert last["timesum"] == st.timesum and last["dt"] == st.dt
    np.testing.assert_array_equal(last["tk1"], st.grid["tk1"])
    np.testing.assert_array_equal(last["xm"], st.m["xm"][: st.marknum])
    # the same run without output ends in the same state
    pkg.run_simulation(ref, 4)
    np.testing.assert_array_equal(ref.grid["tk1"], st.grid["tk1"])
    first = load_state(output_file(str(tmp_path), 2))
    assert first["timesum"] < last["timesum"]


def test_snapshot_keeps_step_host_buffers(pkg, built_lib):
    """Growing the snapshot staging leaves the buffers of erebus_step_host
    alone: a run that snapshots between host timesteps ends bit for bit where
    the run without the snapshot ends."""
    a = pkg.make_state("planetesimal_41")
    b = a.copy()
    sa, sb = pkg.Simulation(a), pkg.Simulation(b)
    sa.step_host(1)
    sb.step_host(1)
    sa.snapshot_begin(pkg.HostState(a.p, a.capacity, pinned=True))
    sa.snapshot_wait()
    for ts in (2, 3):
        sa.step_host(ts)
        sb.step_host(ts)
    sa.close()
    sb.close()
    assert (a.marknum, a.dt, a.timesum) == (b.marknum, b.dt, b.timesum)
    n = a.marknum
    for k in a.m:
        if k == "etasolidm_m":
            continue
        np.testing.assert_array_equal(a.m[k][:n], b.m[k][:n], err_msg=k)
    for k in a.grid:
        np.testing.assert_array_equal(a.grid[k], b.grid[k], err_msg=k)
