"""
qpop_diffraction_b200: the kinematic-diffraction hot path of Q-POP-Diffraction
(per-cell structure-factor source, its 3-D FFT, |S Amp|^2 + fftshift), built for
NVIDIA B200 (sm_100a) as hand-written CUDA behind a C ABI (``libqpopdiff.so``,
declared in ``include/qpopdiff.h``).

``diffraction(params, atoms, oPhase, oStruc, u, region)`` is a drop-in for the
reference's standard-build compute call (src/python/diffraction.py:62-113).
"""

from .diffraction import diffraction, reciprocal_centre, q_axes, wavevectors, install  # noqa: F401
from .plan import Plan, Crystal, crystal_from  # noqa: F401
