"""The allocation-free marker -> node pass (erebus_markers_to_nodes_noalloc).

It serves callers that own every device buffer themselves -- a host
framework with its own pool allocator, or an application held to a fixed
device-memory budget -- and therefore cannot let a library call cudaMalloc.
The test plays such a caller: it allocates the inputs and outputs itself
(with torch) and calls the entry point twice in a row through the C ABI on
the same buffers, checking each result against the state-based entry point
(erebus_markers_to_nodes) on the same input.  The second call has fewer
markers, and moved ones, than the first, so counts, bucket starts or sums
left in the shared scratch by the first call would show up as differences.
Both entry points run the same scatter in the reference's summation order,
so the comparison is exact, as in the other scatter parity tests.  This file
is collected last so that a failure here does not hide the rest of the
suite.
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


def _state_entry_point(pkg, st):
    """Node fields and marker properties from erebus_markers_to_nodes."""
    ref = st.copy()
    sim = pkg.Simulation(ref)
    sim.markers_to_nodes(ref.timesum)
    sim.download()
    sim.close()
    return ref


def _second_input(pkg, st):
    """A smaller marker set than `st`'s, with every marker moved by up to
    0.4 cell widths (kept inside the box): the first 70% of the markers."""
    st2 = st.copy()
    n2 = int(st.marknum * 0.7)
    g = st.g
    k = np.arange(n2, dtype=np.uint64)
    xm, ym = st2.m["xm"], st2.m["ym"]
    xm[:n2] = np.clip(xm[:n2] + 0.4 * g.dx * (2 * pkg.host.u01(7, 1, k) - 1), 1.0,
                      st.p.xsize - 1.0)
    ym[:n2] = np.clip(ym[:n2] + 0.4 * g.dy * (2 * pkg.host.u01(7, 2, k) - 1), 1.0,
                      st.p.ysize - 1.0)
    st2.marknum = n2
    return st2


def _load(dm, dg, st):
    """Copies a host state into the caller's existing device buffers."""
    import torch
    n = st.marknum
    for k, v in st.m.items():
        dm[k][:n].copy_(torch.from_numpy(np.ascontiguousarray(v[:n])))
    for k, v in st.grid.items():
        dg[k].copy_(torch.from_numpy(np.asfortranarray(v).ravel(order="F")))


def _compare(dm, dg, ref, call):
    for k in NODE_FIELDS:
        got = dg[k].cpu().numpy().reshape(ref.grid[k].shape, order="F")
        np.testing.assert_array_equal(got, ref.grid[k], err_msg="%s call %d" % (k, call))
    n = ref.marknum
    for k in DERIVED:
        np.testing.assert_array_equal(dm[k][:n].cpu().numpy(), ref.m[k][:n],
                                      err_msg="%s call %d" % (k, call))


def test_noalloc_matches_state_entry_point_twice(pkg, built_lib):
    import torch
    st = pkg.make_state("planetesimal_41")
    st2 = _second_input(pkg, st)
    refs = [_state_entry_point(pkg, st), _state_entry_point(pkg, st2)]
    f = _noalloc(built_lib)
    dm, dg, ms, gs = _device_views(pkg, st)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (inp, ref) in enumerate(zip((st, st2), refs)):
        _load(dm, dg, inp)
        torch.cuda.synchronize()
        rc = f(ctypes.addressof(inp.p), ctypes.addressof(ms), inp.marknum,
               ctypes.addressof(gs), inp.timesum, stream)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        _compare(dm, dg, ref, call)


def test_noalloc_rejects_marker_type(pkg, built_lib):
    """A marker type outside 1..3 is reported as EREBUS_EINVAL (the kernel
    maps it to a valid table index and raises a flag; no access leaves the
    buffers)."""
    import torch
    st = pkg.make_state("planetesimal_41")
    f = _noalloc(built_lib)
    dm, dg, ms, gs = _device_views(pkg, st)
    dm["tm"][5] = 0
    torch.cuda.synchronize()
    assert f(ctypes.addressof(st.p), ctypes.addressof(ms), st.marknum,
             ctypes.addressof(gs), st.timesum, None) == 1      # EREBUS_EINVAL


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
