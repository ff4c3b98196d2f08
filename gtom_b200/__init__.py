"""B200-native RELION-style Fourier projector, backprojector and gridding
reconstructor: a drop-in for gtom's d_rlnProject / d_rlnBackproject /
d_ReconstructGridding.  The compute lives in libgtomrln.so (CUDA, sm_100a);
this package binds its C ABI."""
from ._lib import GtomError, GtomLibraryMissing  # noqa: F401
from .relion import (  # noqa: F401
    d_BackprojectTomo,
    d_ReconstructGridding,
    d_rlnBackproject,
    d_rlnBackprojectShifted,
    d_rlnProject,
    d_rlnProjectShifted,
    elements_fft,
    gridding_weights,
    kaiser_bessel_table,
    matrices_from_angles,
    mlp_param_count,
    reconstruct_gridding_tol,
    reconstruct_gridding_warm,
    set_brick_tuning,
    set_path,
)
