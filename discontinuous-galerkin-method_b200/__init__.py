"""B200-native engine for the 2D nodal DG elastic-wave time loop (P2, velocity-stress, central flux)."""
from . import build, meshgen, operators, workloads  # noqa: F401
from . import host  # noqa: F401
from . import engine  # noqa: F401  (loads libdg_gpu.so lazily, on first use)
from . import decompose  # noqa: F401
from . import sharding  # noqa: F401
