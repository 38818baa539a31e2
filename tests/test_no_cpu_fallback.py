"""The library has no CPU path: on a host without a usable CUDA device,
creating a render context fails with the CUDA error status instead of
rendering some other way."""
import pytest


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a CUDA device is present")
def test_context_without_a_gpu_fails_with_the_cuda_status():
    from pcr_b200 import capi
    with pytest.raises(capi.PcrError) as e:
        capi.Context(device=0)
    assert e.value.status == 2 and "PCR_ERR_CUDA" in str(e.value)
