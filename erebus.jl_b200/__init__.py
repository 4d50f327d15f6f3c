"""erebus.jl_b200 -- B200-native marker-in-cell timestep of Erebus.jl.

Host-side mirror of the reference's timestep interface over the C-ABI
library `liberebus_b200.so` (built from csrc/ for sm_100a).  The device path
is the only compute path: when the library cannot be loaded or no CUDA
device is present, the calls raise; there is no CPU fallback.
"""
from .abi import (ErebusGridHost, ErebusMarkersHost, ErebusParams,  # noqa: F401
                  ErebusSolveStats, ErebusSolverOptions, ErebusStepStats,
                  ErebusSumsHost)
from .host import (Geometry, HostState, define_markers, make_state,  # noqa: F401
                   u01)
from .params import CONFIGS, config_params, default_params  # noqa: F401
from .device import (ErebusError, Simulation, load_library,  # noqa: F401,E402
                     run_simulation)
