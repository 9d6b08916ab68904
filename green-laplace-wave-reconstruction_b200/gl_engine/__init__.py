"""B200-native Green--Laplace (GL) bound-wave reconstruction engine.

Public API (mirrors the reference's calling patterns):

* :func:`gl_spectral_coefficients` / :func:`gl_spectral_surface` -- the
  MATLAB two-stage API (``src/gl_spectral_coefficients.m``,
  ``src/gl_spectral_surface.m``);
* :func:`surface_batch_device` -- the batched, device-resident variant;
* :class:`SurfaceStream` -- batches streamed to pinned host memory, each
  batch's device->host copy overlapping the next batch's evaluation;
* :func:`reconstruct_directional_field` -- the Python package entry
  (``python/src/green_laplace/spatial.py``).

The GL graphs run in ``_native/libgl_b200.so`` (hand-written sm_100a CUDA)
through its C ABI, ``include/gl_engine.h``.
"""

from .api import (DirectionalFieldResult, GLCoefficients, GLError, Plan, SurfaceBatch, SurfaceStream,
                  dimensionless_wavenumber_from_frequency, fft2_device, gauss_laguerre_rule,
                  get_plan, gl_spectral_coefficients, gl_spectral_surface,
                  reconstruct_directional_field, surface_batch_device)
from . import seastate

__all__ = [
    "DirectionalFieldResult", "GLCoefficients", "GLError", "Plan", "SurfaceBatch", "SurfaceStream",
    "dimensionless_wavenumber_from_frequency", "fft2_device", "gauss_laguerre_rule", "get_plan",
    "gl_spectral_coefficients", "gl_spectral_surface", "reconstruct_directional_field",
    "surface_batch_device", "seastate",
]
