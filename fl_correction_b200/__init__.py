"""fl_correction_b200: the self-absorption-corrected XRF tomography hot path
of FL_correction, rebuilt for NVIDIA B200 (sm_100a).

Module layout mirrors the reference package ``FL`` for the hot path:
``cuda_lib`` (native projector / cone / MLEM entry points), ``torch_functions``,
``torch_image_util``, ``detector_mask``, ``atten_util``, ``core`` and
``torch_recon``; the names are re-exported here as ``FL/__init__.py`` does.
All compute runs in ``libflc.so`` (C ABI: include/flc.h).
"""
from .detector_mask import *  # noqa: F401,F403
from .atten_util import *  # noqa: F401,F403
from .torch_image_util import *  # noqa: F401,F403
from .torch_functions import *  # noqa: F401,F403
from .core import *  # noqa: F401,F403
from .torch_recon import *  # noqa: F401,F403
from .cuda_lib import (cal_atten_cuda, forward_emission, forward_emission_batch,  # noqa: F401
                       backward_emission, backward_emission_batch, mlem_cuda, mlem_cuda_batch,
                       forward_emission_autograd, forward_emission_batch_autograd)

__version__ = "0.1.0"
