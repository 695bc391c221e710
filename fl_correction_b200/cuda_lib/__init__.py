"""Drop-in for ``FL.cuda_lib`` (FL/cuda_lib/__init__.py:1-13)."""
from .atten_cuda import (cal_atten_cuda, forward_emission, forward_emission_batch,
                         backward_emission, backward_emission_batch, mlem_cuda, mlem_cuda_batch,
                         huber_grad, huber_grad_batch)
from .autograd import forward_emission_autograd, forward_emission_batch_autograd
