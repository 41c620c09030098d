"""mps3d_b200: B200-native geometric-multigrid / Krylov linear solve for the
7-point finite-volume operators of mps3d (mgridlib)."""
from .problem import Problem, BC_CODES, LEFT, RIGHT, BOTTOM, TOP, BACK, FRONT, ghosted  # noqa: F401
