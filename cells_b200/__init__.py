"""B200-native lattice Boltzmann wind-tunnel step engine: the slowernet/cells Solver / Solver3D
step API (src/solver.ts, src/solver3d.ts) over hand-written sm_100a CUDA in libcells.so."""
from .solver3d import Solver3D  # noqa: F401
from .solver2d import Batch2D, Solver  # noqa: F401
