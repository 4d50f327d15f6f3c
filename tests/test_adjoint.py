"""The heat-path adjoint restated on the CPU (oracle/adjoint.py) against
central finite differences of the oracle's timestep: the objective is the
mean basic-node temperature inside the body after N timesteps, the
parameters the per-marker porosity and the 26Al/27Al ratio, for a state at
mechanical rest (G = 0, reactions off).  The device adjoint is compared with
this restatement and with finite differences in test_gpu_adjoint.py."""
import numpy as np
import pytest

N_STEPS = 4


def _fresh(pkg, mode):
    import adjoint as AD
    st = pkg.make_state("planetesimal_41")
    st.p.marker_property_mode = mode
    return AD.at_rest(st)


def _J(pkg, mode, phi_scale=None, ratio=None):
    import adjoint as AD
    st = _fresh(pkg, mode)
    n = st.marknum
    if phi_scale is not None:
        st.m["phim"][:n] *= phi_scale
        st.m["phinewm"][:n] = st.m["phim"][:n]
    if ratio is not None:
        st.p.ratio_al = ratio
    AD.forward(st, N_STEPS)
    return AD.objective(st)


@pytest.mark.parametrize("mode", [9, 1])
def test_cpu_adjoint_matches_finite_differences(pkg, oracle, mode):
    import adjoint as AD
    st = _fresh(pkg, mode)
    phi0 = st.m["phim"][: st.marknum].copy()
    o, tape, W = AD.forward(st, N_STEPS)
    assert [r["titer"] for r in tape] == [1] * N_STEPS      # no limiter acted
    phib, rbar = AD.adjoint(o, st, tape, W)
    n = st.marknum
    rng = np.random.default_rng(0)
    # a coherent direction: the relative error is that of the adjoint
    h = 1e-6
    v = rng.uniform(0.5, 1.5, n)
    fd = (_J(pkg, mode, 1 + h * v) - _J(pkg, mode, 1 - h * v)) / (2 * h)
    assert abs(fd - np.dot(phib, phi0 * v)) <= 1e-6 * abs(fd)
    # random signs resolve the per-marker gradient; a larger step keeps the
    # difference above the rounding of J (truncation error ~h^2)
    h = 1e-4
    v = rng.choice([-1.0, 1.0], n)
    fd = (_J(pkg, mode, 1 + h * v) - _J(pkg, mode, 1 - h * v)) / (2 * h)
    assert abs(fd - np.dot(phib, phi0 * v)) <= 1e-5 * abs(fd)
    # the 26Al/27Al ratio
    h = 1e-6
    r0 = st.p.ratio_al
    fd = (_J(pkg, mode, ratio=r0 * (1 + h)) - _J(pkg, mode, ratio=r0 * (1 - h))) / (2 * h * r0)
    assert abs(fd - rbar) <= 1e-6 * abs(fd)
