"""slchannel_b200 -- slChannel's semi-Lagrangian BDF2 channel step on a B200.

A drop-in for the SL-BDF2 path of gmcavallazzi/SLchannel v1.0.1
(``slchannel.SLAdvector``, ``slchannel.SLChannelFlow.step_sl_bdf2`` and the
YAML config surface): the same Python entry points, executed by hand-written
sm_100a CUDA kernels in ``libslc_b200.so`` through the C ABI of
``include/slc_b200.h``.  One GPU; no CPU path.

Like the reference, importing the package sets torch's default dtype to
float64: the grid, fields and diagnostics are float64.
"""

import torch

torch.set_default_dtype(torch.float64)

__version__ = "0.1.0"

from .semilag import SLAdvector  # noqa: E402
from .solver import SLChannelFlow  # noqa: E402

__all__ = ["SLAdvector", "SLChannelFlow", "__version__"]
