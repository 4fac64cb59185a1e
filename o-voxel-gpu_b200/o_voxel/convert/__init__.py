from .flexible_dual_grid import *  # noqa: F401,F403
