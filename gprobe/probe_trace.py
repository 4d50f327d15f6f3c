import sys, os, ctypes, json
sys.path.insert(0, os.getcwd())
import numpy as np
import bench
pkg = bench.load_pkg()
L = pkg.device.load_library(os.path.join(os.getcwd(), 'gprobe/liberebus_trace.so'))
L.erebus_lu_trace.argtypes = [ctypes.c_void_p]; L.erebus_solve_trace.argtypes = [ctypes.c_void_p]
st = pkg.make_state('planetesimal_141')
sim = pkg.Simulation(st)
sim.step(1)
sim.markers_to_nodes(st.timesum); sim.gravity()
dt, conv, s = sim.hydromech_pass(1e11, 1)
tr = np.zeros((2, 128, 8), np.uint64); L.erebus_lu_trace(tr.ctypes.data)
sr = np.zeros((2, 128, 8), np.uint64); L.erebus_solve_trace(sr.ctypes.data)
out = {}
t = tr.astype(np.int64)
for cta in (0, 1):
    d = t[cta, 1:100]
    ph = {'B': d[:,1]-d[:,0], 'bar1': d[:,2]-d[:,1], 'C_gemm': d[:,3]-d[:,2], 'C_rest': d[:,4]-d[:,3], 'bar2': d[:,5]-d[:,4], 'step': t[cta,2:101,0]-t[cta,1:100,0]}
    out['factor_cta%d' % cta] = {k: float(np.median(v)) for k, v in ph.items()}
for sw in (0, 1):
    s2 = sr.astype(np.int64)[sw, 1:120]
    out['solve_sweep%d' % sw] = {'issue+dsmem': float(np.median(s2[:,1]-s2[:,0])), 'mbar_wait': float(np.median(s2[:,2]-s2[:,1])), 'gemv': float(np.median(s2[:,3]-s2[:,2])), 'cluster_sync': float(np.median(s2[:,4]-s2[:,3])), 'step': float(np.median(s2[1:,0]-s2[:-1,0]))}
print(json.dumps(out, indent=1))
