"""steam_b200: the STEAM field-generation hot path on NVIDIA B200 (sm_100a).

World-keyed Philox noise, the extremal Levy transform, the turbulon kernel,
the circular-x/y linear-z convolution, the unit-mean flux cascade, the scalar
pattern and second convolution, the bounded add and the thermodynamic column
solve run as hand-written CUDA kernels behind the C ABI of
``include/steam_b200.h``.  The modules mirror the reference package:

    steam_b200.noise          keyed_uniforms, class_key, center_indices
    steam_b200.turbulons      SHAPES
    steam_b200.utils          convolve_fft_xy_oa_z, zoom_trilinear
    steam_b200.simulate       simulate, cascade_loop, simulate_flux_only, ...
    steam_b200.thermodynamics recover_diagnostics
    steam_b200.ledger         the realized-scalar records
"""

from . import _lib  # noqa: F401

__version__ = "0.1.0"

