"""B200-native Lagrangian DG time step (Lag2D curved-P2 path)."""
from .mesh import Mesh, Ctrl, quad_mesh, read_domn, write_domn, read_ctrl, write_ctrl  # noqa: F401
from .config import StepConfig, workload, WORKLOADS  # noqa: F401
