"""B200-native multigrid solver for the 2-D mapped-grid Poisson operator of
MGPoisson2D (EdSantilli/MGPoisson2D), behind the reference's module interface.

``mgpoisson2d_b200.types`` and ``mgpoisson2d_b200.geometry`` need no GPU.  The
solver entry points (``vcycle``, ``fmg``, ``dc_vcycle``, ``Solver`` and the
operator-level calls) live in ``mgpoisson2d_b200.api`` and are loaded on first
use; they raise ImportError when the CUDA library has not been built.
"""
from .types import *  # noqa: F401,F403

_API_NAMES = {
    "vcycle", "fmg", "dc_vcycle", "Solver", "Batch", "Server", "map_geometry", "map_fourier_rhs", "MAP_IDENTITY", "MAP_WAVY_EXP",
    "MAP_SKEW_LAYER", "fill_ghosts", "extrapolate_ghosts", "compute_invdiags",
    "compute_laplacian", "compute_residual", "compute_pd", "compute_grad", "fill_boundary_fluxes",
    "compute_div", "relax_gs", "relax_jacobi", "solve_bicgstab2", "solve_bicgstab2_noalloc", "restrict", "prolong",
    "pnorm", "inner_prod", "estimate_maxdepth", "create_mgschedule", "MGPError", "library_path",
    "kernel_launch_count", "set_flags", "FLAG_DIRICHLET_COUPLED_DIAG", "FLAG_TIME_SMOOTHER", "FLAG_KRYLOV", "FLAG_MIXED",
    "FLAG_DIRECT_COARSE", "FLAG_GMRES", "FLAG_DIRECT_LARGE", "FLAG_LOCKSTEP", "FLAG_REPORT_MAXITER", "FLAG_BF16_COARSE",
    "NOALLOC_MAX_SIDE", "EXPORTS",
}


def __getattr__(name):
    if name in _API_NAMES:
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
