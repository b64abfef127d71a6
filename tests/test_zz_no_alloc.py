"""The batch inversion that allocates no device memory, checked against the
allocating entry point (lxmfv_fe_op op 3), both through the C ABI.

lxmfv_fe_batch_invert_static is for callers that cannot call cudaMalloc: code
running while a CUDA graph is captured, or a host runtime that owns every
device allocation and hands the library buffers.  Such a caller passes device
buffers it already owns; the kernel's working storage is one static device
array of the library.  This file is collected last, so a run that stops at
its first failure has run every other test before this one; it passes both
alone in a fresh process (the first call sets up the array's address) and
after the other tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(rng, count):
    a = rng.integers(0, 2**32, size=(count, 8), dtype=np.uint64).astype(np.uint32)
    a[:3] = 0xFFFFFFFF  # values with bit 255 set, which the inversion drops
    a[5] = 0            # a zero zeroes its whole group, as in the walk
    return a


def test_static_scratch_matches_the_allocating_entry_point(lx):
    import torch

    rng = np.random.default_rng(2026)
    with lx.Backend(device=0, lanes=256) as b:
        torch.cuda.set_device(0)
        for count, group in ((4096, 64), (1000, 7)):  # two calls in a row
            a = _inputs(rng, count)
            expected = b.fe_op(3, a, group=group)
            d_a = torch.from_numpy(a.view(np.int32)).cuda()
            d_out = torch.zeros_like(d_a)
            torch.cuda.synchronize()
            lx.fe_batch_invert_static(d_a.data_ptr(), d_out.data_ptr(), count, group)
            torch.cuda.synchronize()
            got = d_out.cpu().numpy().view(np.uint32)
            assert got.shape == expected.shape
            assert (got == expected).all(), f"count {count}, group {group}"


def test_static_scratch_rejects_sizes_beyond_its_maximum(lx):
    import torch

    d = torch.zeros((2, 8), dtype=torch.int32, device="cuda:0")
    with pytest.raises(lx.LxmfvError) as e:
        lx.fe_batch_invert_static(d.data_ptr(), d.data_ptr(), lx.STATIC_SCRATCH_ELEMS + 1, 64)
    assert e.value.code == lx.ERR_ARG and "exceeds the static scratch" in str(e.value)
