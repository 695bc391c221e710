"""The torch-operator composition of the corrected projection (autograd
reference of the gradient tests); it lives in the package because the
gradient benchmark times it as its plain-torch baseline."""
from fl_correction_b200.torch_composition import *  # noqa: F401,F403
from fl_correction_b200.torch_composition import (  # noqa: F401
    cone, exclusive_reverse_cumprod, project, rotate, xrf_project)
