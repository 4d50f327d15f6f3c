"""Device adjoint of the heat path (erebus_adjoint_heat) against the CPU
restatement (oracle/adjoint.py) and against central finite differences of
the oracle's timestep, for a state at mechanical rest (G = 0, reactions
off).  Objective: mean basic-node temperature inside the body after N
timesteps; parameters: per-marker porosity and the 26Al/27Al ratio."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_STEPS = 5


def _fresh(pkg, mode=9):
    import adjoint as AD
    st = pkg.make_state("planetesimal_41")
    st.p.marker_property_mode = mode
    return AD.at_rest(st)


@pytest.mark.parametrize("mode", [9, 1])
def test_device_adjoint_matches_cpu_adjoint(pkg, oracle, built_lib, mode):
    import adjoint as AD
    sg = _fresh(pkg, mode)
    sim = pkg.Simulation(sg)
    J, dphi, dratio, stats = sim.adjoint_heat(N_STEPS, checkpoint_every=2)
    sim.close()
    assert stats.steps == N_STEPS and stats.checkpoints == 3
    # constant laws: the transposed heat matrix is the same every step and is
    # factored once; temperature-dependent laws change it every step
    assert stats.factorizations == (1 if mode == 9 else N_STEPS)
    assert stats.markers == sg.marknum
    so = _fresh(pkg, mode)
    o, tape, W = AD.forward(so, N_STEPS)
    phib, rbar = AD.adjoint(o, so, tape, W)
    assert abs(J - AD.objective(so)) <= 1e-11 * abs(J)
    np.testing.assert_allclose(dphi, phib, rtol=1e-7, atol=1e-9 * np.abs(phib).max())
    assert abs(dratio - rbar) <= 1e-8 * abs(rbar)


def test_device_adjoint_matches_finite_differences(pkg, oracle, built_lib):
    import adjoint as AD
    sg = _fresh(pkg)
    n = sg.marknum
    phi0 = sg.m["phim"][:n].copy()
    sim = pkg.Simulation(sg)
    J, dphi, dratio, _ = sim.adjoint_heat(N_STEPS, checkpoint_every=5)
    sim.close()

    def J_of(scale=None, ratio=None):
        st = _fresh(pkg)
        if scale is not None:
            st.m["phim"][:n] *= scale
            st.m["phinewm"][:n] = st.m["phim"][:n]
        if ratio is not None:
            st.p.ratio_al = ratio
        AD.forward(st, N_STEPS)
        return AD.objective(st)

    h = 1e-6
    v = np.random.default_rng(3).uniform(0.5, 1.5, n)
    fd = (J_of(1 + h * v) - J_of(1 - h * v)) / (2 * h)
    assert abs(fd - np.dot(dphi, phi0 * v)) <= 1e-6 * abs(fd)
    r0 = sg.p.ratio_al
    fd = (J_of(ratio=r0 * (1 + h)) - J_of(ratio=r0 * (1 - h))) / (2 * h * r0)
    assert abs(fd - dratio) <= 1e-6 * abs(fd)


def test_checkpoint_interval_does_not_change_the_gradient(pkg, built_lib):
    out = []
    for k in (1, 3, N_STEPS):
        st = _fresh(pkg)
        sim = pkg.Simulation(st)
        out.append(sim.adjoint_heat(N_STEPS, checkpoint_every=k))
        sim.close()
    for J, dphi, dratio, st in out[1:]:
        assert J == out[0][0]
        np.testing.assert_allclose(dphi, out[0][1], rtol=1e-12,
                                   atol=1e-14 * np.abs(out[0][1]).max())
        assert abs(dratio - out[0][2]) <= 1e-12 * abs(out[0][2])


def test_states_not_at_rest_are_refused(pkg, built_lib):
    st = pkg.make_state("planetesimal_41")      # self-gravity on
    sim = pkg.Simulation(st)
    with pytest.raises(pkg.ErebusError) as e:
        sim.adjoint_heat(2)
    assert e.value.code == 1 and "rest" in str(e.value)
    # nothing ran: the first timestep still works as usual
    sim.step(1)
    sim.close()


def test_autograd_function(pkg, built_lib):
    """HeatObjective: J.backward() leaves the adjoint gradients in .grad."""
    import torch
    from erebus_b200.adjoint import HeatObjective, at_rest, heat_gradient
    st = at_rest(pkg.make_state("planetesimal_41"))
    n = st.marknum
    phim = torch.tensor(st.m["phim"][:n], dtype=torch.float64, requires_grad=True)
    ratio = torch.tensor(st.p.ratio_al, dtype=torch.float64, requires_grad=True)
    J = HeatObjective.apply(phim, ratio, st, 3, 2)
    J.backward()
    J0, g0, r0, _ = heat_gradient(st, 3, 2)
    assert J.item() == J0
    np.testing.assert_array_equal(phim.grad.numpy(), g0)
    assert ratio.grad.item() == r0
    # a perturbed porosity reaches the device through forward()
    J2 = HeatObjective.apply(phim.detach() * 1.01, ratio.detach(), st, 3, 2)
    assert J2.item() != J0


def test_device_adjoint_at_benchmark_size(pkg, oracle, built_lib):
    """The bench's adjoint workload (141x141, 4x4 markers per cell, porosity
    U(0.05, 0.25)) over two timesteps: device gradients equal the CPU
    restatement's."""
    import adjoint as AD
    from erebus_b200.adjoint import at_rest
    sg = at_rest(pkg.make_state("planetesimal_141_adjoint"))
    so = at_rest(pkg.make_state("planetesimal_141_adjoint"))
    sim = pkg.Simulation(sg)
    J, dphi, dratio, stats = sim.adjoint_heat(2, checkpoint_every=1)
    sim.close()
    o, tape, W = AD.forward(so, 2)
    phib, rbar = AD.adjoint(o, so, tape, W)
    assert stats.markers == so.marknum == 313600
    assert abs(J - AD.objective(so)) <= 1e-11 * abs(J)
    np.testing.assert_allclose(dphi, phib, rtol=1e-7, atol=1e-9 * np.abs(phib).max())
    assert abs(dratio - rbar) <= 1e-8 * abs(rbar)
