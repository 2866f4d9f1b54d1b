"""The SM-store device-to-host copy: bit-identical to a copy-engine copy,
for sizes that are and are not multiples of 16 bytes."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [4, 4096, 1 << 22, (1 << 20) + 3])
def test_copy_to_host_sm_matches_copy(gpu_lib, n):
    import torch
    from asohf_b200 import api
    a = api.Asohf(0)
    src = torch.randn(n, device="cuda:0")
    ref = src.cpu()
    dst = torch.full((n,), float("nan")).pin_memory()
    st = torch.cuda.Stream(device="cuda:0")
    st.wait_stream(torch.cuda.current_stream())
    a.copy_to_host_sm(dst, src, st)
    st.synchronize()
    assert torch.equal(dst.view(torch.int32), ref.view(torch.int32))
