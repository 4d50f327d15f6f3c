"""Generates tests/golden/planetesimal_401_steps.npz: the oracle's first two
timesteps of the 401 x 401 workload (2,560,000 markers, rock viscosity
log-uniform 1e17-1e23 Pa s), sampled after each.

The oracle (C restatement of the reference's timestep plus SuperLU solves)
needs about 2 minutes for timestep 1 (one thermochemical iteration) and
about 8 for timestep 2 (three), with ~10 GB of host memory, which is too long
to repeat inside a test, so its results are stored once.  The state after
each timestep is kept on a fixed sample: every 7th P node of each
solution field (23,087 nodes) and every 64th marker (40,000 markers), which
suffices for the relative-error checks the GPU test makes (relative L2 of
the sampled fields, max relative error of the sampled positions).  The
initial state comes from the package's seeded generator, so the device run in
the test starts from the same arrays.

    python tests/golden/make_planetesimal_401.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

NODE_STRIDE = 7
MARKER_STRIDE = 64
FIELDS = ["vx", "vy", "pr", "pf", "qxD", "qyD", "tk2"]
MARKER_FIELDS = ["xm", "ym", "tkm", "phim", "XWsolidm0", "sxxm", "sxym"]


def main():
    import oracle as O
    pkg = O.load_package()
    st = pkg.make_state("planetesimal_401")
    o = O.Oracle(st)
    out = {"node_stride": NODE_STRIDE, "marker_stride": MARKER_STRIDE}
    for ts in (1, 2):
        t0 = time.time()
        stats = o.step(ts)
        el = time.time() - t0
        pre = "s%d_" % ts
        out.update({pre + "titer": stats["titer"], pre + "iplast_total": stats["iplast_total"],
                    pre + "dt": stats["dt"], pre + "marknum": stats["marknum"],
                    pre + "seconds": el})
        for k in FIELDS:
            out[pre + "grid_" + k] = np.array(
                np.asfortranarray(st.grid[k]).ravel(order="F")[::NODE_STRIDE], copy=True)
        n = st.marknum
        for k in MARKER_FIELDS:
            out[pre + "m_" + k] = st.m[k][:n][::MARKER_STRIDE].copy()
        out[pre + "m_tm"] = st.m["tm"][:n][::MARKER_STRIDE].astype(np.int8)
        print("timestep %d of planetesimal_401: titer %d, %.1f s" % (ts, stats["titer"], el),
              flush=True)
    np.savez_compressed(os.path.join(HERE, "planetesimal_401_steps.npz"), **out)


if __name__ == "__main__":
    main()
