"""The allocation-free marker -> node pass (erebus_markers_to_nodes_noalloc).

It serves callers that own every device buffer themselves -- a host
framework with its own pool allocator, or an application held to a fixed
device-memory budget -- and therefore cannot let a library call cudaMalloc.
The test plays such a caller: it allocates the inputs and outputs itself
(with torch) and calls the entry point twice in a row through the C ABI,
checking each result against the state-based entry point
(erebus_markers_to_nodes).  Both run the same scatter in the reference's
summation order, so the comparison is exact, as in the other scatter
parity tests.  This file is collected last so that a failure here does not
hide the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.erebus_markers_to_nodes_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_double, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


NODE_FIELDS = ["ETA0", "ETA", "GGG", "SXY0", "COH", "TEN", "FRI", "YNY", "RHOX", "RHOFX",
               "KX", "PHIX", "RX", "RHOY", "RHOFY", "KY", "PHIY", "RY", "RHO", "RHOCP",
               "ALPHA", "ALPHAF", "HR", "GGGP", "SXX0", "tk1", "PHI", "BETAPHI"]
DERIVED = ["rhototalm", "rhocptotalm", "etatotalm", "hrtotalm", "ktotalm",
           "tkm_rhocptotalm", "etafluidcur_inv_kphim"]


def _device_views(pkg, st):
    """Caller-owned device copies of the host state, and the ABI structs
    holding their device addresses."""
    import torch
    n = st.marknum
    dm = {k: torch.from_numpy(np.ascontiguousarray(v[:n])).cuda() for k, v in st.m.items()}
    dg = {k: torch.from_numpy(np.asfortranarray(v).ravel(order="F")).cuda()
          for k, v in st.grid.items()}
    ms = pkg.ErebusMarkersHost()
    for name, ctype in ms._fields_:
        setattr(ms, name, ctypes.cast(ctypes.c_void_p(dm[name].data_ptr()), ctype))
    gs = pkg.ErebusGridHost()
    for name, ctype in gs._fields_:
        setattr(gs, name, ctypes.cast(ctypes.c_void_p(dg[name].data_ptr()), ctype))
    return dm, dg, ms, gs


def test_noalloc_matches_state_entry_point_twice(pkg, built_lib):
    import torch
    st = pkg.make_state("planetesimal_41")
    # the existing entry point
    ref = st.copy()
    sim = pkg.Simulation(ref)
    sim.markers_to_nodes(ref.timesum)
    sim.download()
    sim.close()
    f = _noalloc(built_lib)
    dm, dg, ms, gs = _device_views(pkg, st)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rc = f(ctypes.addressof(st.p), ctypes.addressof(ms), st.marknum,
               ctypes.addressof(gs), st.timesum, stream)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        for k in NODE_FIELDS:
            got = dg[k].cpu().numpy().reshape(ref.grid[k].shape, order="F")
            np.testing.assert_array_equal(got, ref.grid[k], err_msg="%s call %d" % (k, call))
        n = st.marknum
        for k in DERIVED:
            np.testing.assert_array_equal(dm[k].cpu().numpy(), ref.m[k][:n],
                                          err_msg="%s call %d" % (k, call))


def test_noalloc_rejects_oversize(pkg, built_lib):
    st = pkg.make_state("planetesimal_41")
    f = _noalloc(built_lib)
    dm, dg, ms, gs = _device_views(pkg, st)
    too_many = 131072 + 1
    assert f(ctypes.addressof(st.p), ctypes.addressof(ms), too_many,
             ctypes.addressof(gs), st.timesum, None) == 4   # EREBUS_ECAPACITY
    big = pkg.config_params("planetesimal_141")              # 142*142 > 16384 nodes
    assert f(ctypes.addressof(big), ctypes.addressof(ms), st.marknum,
             ctypes.addressof(gs), st.timesum, None) == 4
