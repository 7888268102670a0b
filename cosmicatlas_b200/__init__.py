"""cosmicatlas_b200: the CosmicAtlas/BAM per-iteration mesh hot path on B200.

Particle-to-mesh assignment (NGP/CIC/TSC), 3D r2c/c2r FFT, the binned power
spectrum and the T-web, as hand-written sm_100a kernels in libcam.so behind
the C ABI of include/cam.h.  This package holds the ctypes binding
(``_lib``), the host-side mirror of the reference interface (``api``), the
seeded input generators (``synth``) and the build script (``build``).
"""
from .api import (CIC, F32, F64, NGP, TSC, CamError, Context, Cwclass, Params, PowerSpectrumF,
                  default_context, do_fftw_c2r, do_fftw_r2c, getDensity_CIC, getDensity_NGP,
                  getDensity_TSC, make_grid)

__all__ = ["NGP", "CIC", "TSC", "F32", "F64", "CamError", "Context", "Cwclass", "Params", "PowerSpectrumF",
           "default_context", "do_fftw_r2c", "do_fftw_c2r", "getDensity_NGP", "getDensity_CIC",
           "getDensity_TSC", "make_grid"]
