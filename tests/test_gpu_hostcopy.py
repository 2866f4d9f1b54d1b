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


@pytest.mark.parametrize("sizes", [[4], [4096, (1 << 20) + 3], [(9 << 22) + 5, 1 << 22, 7]])
def test_copy_to_host_async_matches_copy(gpu_lib, sizes):
    """The chunked copy-engine copies (several in flight, one of more than
    one chunk): every byte arrives, after the work issued before them."""
    import torch
    from asohf_b200 import api
    a = api.Asohf(0)
    st = torch.cuda.current_stream()
    a.set_stream(st.cuda_stream)
    srcs = [torch.zeros(n, device="cuda:0") for n in sizes]
    for s in srcs:  # written on the context stream just before the copies are issued
        s.copy_(torch.randn(s.numel(), device="cuda:0"))
    dsts = [torch.full((n,), float("nan")).pin_memory() for n in sizes]
    for d, s in zip(dsts, srcs):
        a.copy_to_host_async(d, s)
    a.copy_wait()
    for d, s in zip(dsts, srcs):
        assert torch.equal(d.view(torch.int32), s.cpu().view(torch.int32))
    # a stream made to wait sees the copies done
    twice = srcs[0] * 2.0  # kept alive until the copy is done
    a.copy_to_host_async(dsts[0], twice)
    side = torch.cuda.Stream(device="cuda:0")
    a.copy_wait(side)
    side.synchronize()
    assert torch.equal(dsts[0], twice.cpu())
