"""The allocation-free hash-grid insert (rtpg_hashgrid_insert_noalloc) against the handle-based
insert.

The entry point exists for callers that cannot allocate device memory: an application that
owns every allocation under a fixed budget, work enqueued while the stream is captured into a
CUDA graph, or a real-time loop that must not block in the allocator.  Its scratch is one
fixed device array shared by every call, so this test makes two calls in a row into the same
caller-owned table and checks that each gives exactly the slots and table contents of
rtpg_hashgrid_insert on a handle (integer results, compared bit for bit).  It lives in its
own file, collected last, and passes alone in a fresh process as well as after the other
tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(rng, n, mn, mx):
    pos = (rng.random((n, 3), dtype=np.float32) * (mx - mn) + mn).astype(np.float32)
    pos[: n // 4] = pos[: n // 16][rng.integers(0, n // 16, n // 4)]  # repeated cells
    return pos


@pytest.mark.parametrize("keying", [0, 1])
def test_noalloc_insert_matches_handle_insert(cuda, keying):
    import torch
    from rtlib_b200.hashgrid import NOALLOC_MAX_POINTS, HashGrid, insert_noalloc
    rng = np.random.default_rng(17 + keying)
    mn, mx = np.array([-2, -1, -3], np.float32), np.array([2, 3, 1], np.float32)
    bounds, nslots = [256, 128, 256], 1 << 14
    hg = HashGrid(mn, mx, bounds, nslots, keying=keying)
    table = torch.zeros(nslots, dtype=torch.int64, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    for call in range(2):
        pos = torch.from_numpy(_batch(rng, NOALLOC_MAX_POINTS, mn, mx)).to(cuda)
        want = torch.empty(pos.shape[0], dtype=torch.int32, device=cuda)
        got = torch.full((pos.shape[0],), -7, dtype=torch.int32, device=cuda)
        hg.insert(pos, want)
        insert_noalloc(mn, mx, bounds, table, pos, got, keying=keying, status=status)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())
        np.testing.assert_array_equal(table.cpu().numpy().view(np.uint64), hg.export())
    # the second call filled buckets past 32 entries: both report the full buckets
    assert (want.cpu().numpy().view(np.uint32) == 0xFFFFFFFF).any()
    assert int(status.item()) & 0x10 and hg.status() & 0x10


def test_noalloc_insert_rejects_oversized_batch(cuda):
    import torch
    from rtlib_b200._lib import RtpgError
    from rtlib_b200.hashgrid import NOALLOC_MAX_POINTS, insert_noalloc
    table = torch.zeros(1 << 10, dtype=torch.int64, device=cuda)
    pos = torch.zeros((NOALLOC_MAX_POINTS + 1, 3), dtype=torch.float32, device=cuda)
    out = torch.empty(NOALLOC_MAX_POINTS + 1, dtype=torch.int32, device=cuda)
    with pytest.raises(RtpgError, match="exceed the limit"):
        insert_noalloc((0, 0, 0), (1, 1, 1), (8, 8, 8), table, pos, out)
