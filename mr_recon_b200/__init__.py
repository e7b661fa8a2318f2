"""mr_recon_b200 -- B200-native (sm_100a) Kaiser-Bessel NUFFT for MRI
reconstruction with the NUFFT / linop / CG API of mr_recon.

    from mr_recon_b200.fourier import triton_nufft      # drop-in NUFFT
    from mr_recon_b200.linops import sense_linop, batching_params
    from mr_recon_b200.recons import CG_SENSE_recon

Everything runs through libmrnufft.so (include/mrnufft.h); build it with
``python -m mr_recon_b200.build``. There is no CPU fallback.
"""

__version__ = "0.1.0"

from . import _lib  # noqa: F401
from .fourier import NUFFT, b200_nufft, triton_nufft, calc_toep_kernel_helper  # noqa: F401
from .linops import batching_params, linop, sense_linop, subspace_linop, subspace_linop_new  # noqa: F401
from .algs import conjugate_gradient, power_method_operator, FISTA, gradient_descent, SenseCG  # noqa: F401
from .recons import CG_SENSE_recon, FISTA_recon, min_norm_recon, coil_combine  # noqa: F401
from .plan import Plan  # noqa: F401
