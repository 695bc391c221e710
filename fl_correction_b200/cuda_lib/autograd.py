"""autograd Functions over the native projector.

``forward_emission_autograd`` / ``forward_emission_batch_autograd`` keep the
reference's contract (FL/cuda_lib/autograd.py:5-77): forward is the
attenuated emission projection, backward applies its exact transpose to the
incoming gradient and returns a gradient for C only (atten, em_cs and theta
get None).
"""
import torch

from . import atten_cuda


class ForwardEmissionFunction(torch.autograd.Function):
    """Single slice: atten (A,H,W), C (R,H,W), em_cs (A,R), theta (A) -> (A,W)."""

    @staticmethod
    def forward(ctx, atten, C, em_cs, theta):
        ctx.save_for_backward(atten, em_cs, theta)
        return atten_cuda.forward_emission(atten, C, em_cs, theta)

    @staticmethod
    def backward(ctx, grad_output):
        atten, em_cs, theta = ctx.saved_tensors
        grad_C = atten_cuda.backward_emission(atten, grad_output.contiguous(), em_cs, theta)
        return None, grad_C, None, None


def forward_emission_autograd(atten, C, em_cs, theta):
    return ForwardEmissionFunction.apply(atten, C, em_cs, theta)


class ForwardEmissionBatchFunction(torch.autograd.Function):
    """Batched slices: atten (A,B,H,W), C (R,B,H,W) -> (A,B,W)."""

    @staticmethod
    def forward(ctx, atten, C, em_cs, theta):
        ctx.save_for_backward(atten, em_cs, theta)
        return atten_cuda.forward_emission_batch(atten, C, em_cs, theta)

    @staticmethod
    def backward(ctx, grad_output):
        atten, em_cs, theta = ctx.saved_tensors
        grad_C = atten_cuda.backward_emission_batch(atten, grad_output.contiguous(), em_cs, theta)
        return None, grad_C, None, None


def forward_emission_batch_autograd(atten, C, em_cs, theta):
    return ForwardEmissionBatchFunction.apply(atten, C, em_cs, theta)
