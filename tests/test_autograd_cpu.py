"""The torch.autograd operator fails loudly when no CUDA device is visible
(no CPU fallback exists on the product path)."""
import pytest
import torch

from owl_b200.autograd import SSGForward, ssg_forward


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-CUDA error path")
def test_autograd_without_cuda_raises():
    with pytest.raises(RuntimeError, match="CUDA"):
        ssg_forward(None, None, torch.ones(4, 3, requires_grad=True), torch.ones(4, 3))


def test_autograd_is_a_function():
    assert issubclass(SSGForward, torch.autograd.Function)
