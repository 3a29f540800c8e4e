"""B200-native Peridigm hot path: LPS elastic material, critical-stretch damage,
velocity-Verlet explicit integration, short-range contact and quasi-static
Newton/CG, as sm_100a CUDA kernels behind the C ABI in include/pd_b200.h."""
from ._lib import PDError, load  # noqa: F401
from .context import Context, expr_eval  # noqa: F401

__all__ = ["Context", "PDError", "expr_eval", "load"]
