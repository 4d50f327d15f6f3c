"""save_state records (src/Erebus.jl:5718-5960): key names and order, array
layouts, and the file round trip; the asynchronous device snapshot behind
them is checked on the GPU in test_gpu_snapshot.py."""
import numpy as np

# jldsave's key list, src/Erebus.jl:5820-5955
REFERENCE_KEYS = (
    "timestep dt Δtreaction reaction_rate_coeff_mode marker_property_mode timesum marknum "
    "phim0 XWsolidm_init ratio_al t_half_al dsubgrids dsubgridt hr_al hr_fe rplanet rcrust "
    "psurface xsize ysize xcenter ycenter Nx Ny Nx1 Ny1 Nxm Nym dx dy dxm dym x y xvx yvx "
    "xvy yvy xp yp xxm yym ETA ETA0 GGG EXY SXY SXY0 wyx COH TEN FRI YNY RHOX RHOFX KX "
    "PHIX vx vxf RX qxD gx RHOY RHOFY KY PHIY vy vyf RY qyD gy RHO RHOCP ALPHA ALPHAF HR "
    "HA HS ETAP GGGP EXX SXX SXX0 tk1 tk2 vxp vyp vxpf vypf pr pf ps pr0 pf0 ps0 ETAPHI "
    "BETAPHI PHI APHI FI ETA5 ETA00 YNY5 YNY00 YNY_inv_ETA DSXY EII SII DSXX DMP DHP XWS "
    "XWsolidm0 xm ym tm tkm sxxm sxym etavpm phim rhototalm rhocptotalm etatotalm hrtotalm "
    "ktotalm tkm_rhocptotalm etafluidcur_inv_kphim inv_gggtotalm fricttotalm cohestotalm "
    "tenstotalm rhofluidcur alphasolidcur alphafluidcur").split()


def test_record_keys_follow_reference(pkg):
    from erebus_b200.output import state_record
    st = pkg.make_state("planetesimal_41")
    rec = state_record(10, st)
    assert list(rec) == REFERENCE_KEYS


def test_save_and_load_round_trip(pkg, tmp_path):
    from erebus_b200.output import load_state, output_file, save_state
    st = pkg.make_state("planetesimal_41")
    rng = np.random.default_rng(5)
    st.grid["vx"][:] = rng.random(st.grid["vx"].shape)
    st.grid["YNY"][:] = rng.integers(0, 2, st.grid["YNY"].shape)
    st.dt, st.timesum = 123.5, 4.25e12
    fid = save_state(str(tmp_path), 20, st)
    assert fid == output_file(str(tmp_path), 20)
    assert fid.endswith("output_00020.npz")
    rec = load_state(fid)
    assert list(rec) == REFERENCE_KEYS
    g = st.g
    assert rec["timestep"] == 20 and rec["marknum"] == st.marknum
    assert rec["dt"] == 123.5 and rec["timesum"] == 4.25e12
    assert rec["Δtreaction"] == st.p.dtreaction and rec["Nx1"] == g.Nx1
    np.testing.assert_array_equal(rec["vx"], st.grid["vx"])
    assert rec["vx"].shape == (g.Ny1, g.Nx1) and rec["vx"].flags.f_contiguous
    assert rec["YNY"].dtype == np.bool_
    np.testing.assert_array_equal(rec["YNY"], st.grid["YNY"].astype(bool))
    assert rec["xm"].shape == (st.marknum,)
    np.testing.assert_array_equal(rec["tm"], st.m["tm"][: st.marknum])
    # coordinates of src/constants.jl:40-47, 116-119
    np.testing.assert_allclose(rec["x"][-1], st.p.xsize, rtol=1e-14)
    np.testing.assert_allclose(rec["yp"][[0, -1]], [-g.dy / 2, st.p.ysize + g.dy / 2],
                               rtol=1e-14)
    np.testing.assert_allclose(rec["xxm"][[0, -1]], [g.dxm / 2, st.p.xsize - g.dxm / 2],
                               rtol=1e-14)
    assert rec["x"].size == g.Nx and rec["xvy"].size == g.Nx1 and rec["yym"].size == g.Nxm
