"""pypomp_b200 -- pypomp's particle-filter hot path on NVIDIA B200 (sm_100a).

The per-observation loop behind ``Pomp.pfilter``, ``mop``, ``mif`` and
``train`` runs in hand-written CUDA (``pypomp_b200/csrc`` -> ``_lib/libppf.so``)
for the built-in models LG, SV and Ricker; the Python layer keeps the
reference's signatures and result tables.
"""

from . import _ffi  # noqa: F401  (loads libppf.so; fails loudly if it is missing)
from . import functional, maths, random  # noqa: F401
from .maths import logmeanexp, logmeanexp_se  # noqa: F401
from .models import LG, SV, Ricker  # noqa: F401
from .pomp import ParTrans, Pomp, PompParameters  # noqa: F401
from .autograd import mop_objective  # noqa: F401
from .panel import PanelParameters, PanelPomp  # noqa: F401
from .optim import (SGD, BFGS, Adam, FullMatrixAdam, LearningRate, Newton, RWSigma,  # noqa: F401
                    WeightedNewton)

__all__ = ["LG", "SV", "Ricker", "Pomp", "PompParameters", "functional", "random",
           "logmeanexp", "logmeanexp_se"]
from . import proposals  # noqa: F401
from .proposals import MVNDiagRW, MVNRWAdaptive, MVNRWFull  # noqa: F401
