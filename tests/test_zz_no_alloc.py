"""The batch inversion that allocates no device memory, checked against the
allocating entry point (lxmfv_fe_op op 3) and against the oracle, both
library calls through the C ABI.

lxmfv_fe_batch_invert_static is for callers that may not call cudaMalloc or
cudaFree: a host runtime that owns every device allocation and hands the
library its buffers, or a loop that cannot take cudaFree's implicit device
synchronisation.  Such a caller passes device buffers it already owns; the
kernel's working storage is one static device array of the library.  This
file is collected last, so a run that stops at its first failure has run
every other test before this one; it passes both alone in a fresh process
(the first call sets up the array's address) and after the other tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(rng, count):
    a = rng.integers(0, 2**32, size=(count, 8), dtype=np.uint64).astype(np.uint32)
    a[:3] = 0xFFFFFFFF  # values with bit 255 set, which the inversion drops
    a[5] = 0            # a zero zeroes its whole group, as in the walk
    return a


def test_static_scratch_matches_the_allocating_entry_point(lx, oracle):
    import torch

    rng = np.random.default_rng(2026)
    with lx.Backend(device=0, lanes=256) as b:
        torch.cuda.set_device(0)
        for count, group in ((4096, 64), (1000, 7)):  # two calls in a row
            a = _inputs(rng, count)
            expected = b.fe_op(3, a, group=group)
            assert (expected == oracle.fe_batch_invert(a, group)).all()
            d_a = torch.from_numpy(a.view(np.int32)).cuda()
            d_out = torch.zeros_like(d_a)
            torch.cuda.synchronize()
            lx.fe_batch_invert_static(d_a.data_ptr(), d_out.data_ptr(), count, group)
            torch.cuda.synchronize()
            got = d_out.cpu().numpy().view(np.uint32)
            assert got.shape == expected.shape
            assert (got == expected).all(), f"count {count}, group {group}"


def test_static_scratch_in_place_and_on_a_stream(lx, oracle):
    """d_out == d_a, on a stream of the caller's: the same results as the oracle."""
    import torch

    rng = np.random.default_rng(77)
    torch.cuda.set_device(0)
    s = torch.cuda.Stream(device=0)
    for count, group in ((lx.STATIC_SCRATCH_ELEMS, 256), (333, 64)):  # the maximum size, then a ragged one
        a = _inputs(rng, count)
        d = torch.from_numpy(a.view(np.int32).copy()).cuda()
        torch.cuda.synchronize()
        lx.fe_batch_invert_static(d.data_ptr(), d.data_ptr(), count, group, stream=s.cuda_stream)
        s.synchronize()
        got = d.cpu().numpy().view(np.uint32)
        assert (got == oracle.fe_batch_invert(a, group)).all(), f"in place, count {count}, group {group}"


def test_static_scratch_rejects_bad_calls(lx):
    import torch

    d = torch.zeros((16, 8), dtype=torch.int32, device="cuda:0")
    with pytest.raises(lx.LxmfvError) as e:
        lx.fe_batch_invert_static(d.data_ptr(), d.data_ptr(), lx.STATIC_SCRATCH_ELEMS + 1, 64)
    assert e.value.code == lx.ERR_ARG and "exceeds the static scratch" in str(e.value)
    with pytest.raises(lx.LxmfvError) as e:  # output one element past the input: overlapping, not in place
        lx.fe_batch_invert_static(d.data_ptr(), d.data_ptr() + 32, 8, 4)
    assert e.value.code == lx.ERR_ARG and "overlap" in str(e.value)
    torch.cuda.synchronize()
    assert int(d.abs().sum()) == 0  # nothing ran
