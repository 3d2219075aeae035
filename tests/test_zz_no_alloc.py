"""The allocation-free commitment entry point (neo_gpu_commit_noalloc) gives
exactly the commitments of the standard entry point (neo_gpu_commit), on two
calls in a row that reuse the library's fixed device scratch.  Callers that
cannot allocate device memory (stream capture, framework-owned memory pools,
latency-critical provers) use it with buffers they already own."""
import numpy as np
import pytest

from nightstream_b200 import gpu

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu


def test_commit_noalloc_matches_commit_on_two_calls(ctx):
    import torch
    m = 4096
    rng = np.random.default_rng(2024)
    pp = rng.integers(0, Q, size=(16, m, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    for n_vec in (3, 12):  # two calls in a row share the scratch array
        Z = rng.integers(-1, 2, size=(n_vec, 54, m)).astype(np.int8)
        expect = ctx.commit(Z)
        d_z = torch.from_numpy(Z).cuda()
        d_out = torch.zeros((n_vec, 16, 54), dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        ctx.commit_noalloc(d_z.data_ptr(), n_vec, m, d_out.data_ptr())
        ctx.synchronize()
        got = d_out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, expect)


def test_commit_noalloc_rejects_too_many_vectors(ctx):
    import torch
    m = 64
    pp = np.random.default_rng(1).integers(0, Q, size=(16, m, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    dummy = torch.zeros(16, dtype=torch.int8, device="cuda")
    out = torch.zeros(16, dtype=torch.int64, device="cuda")
    with pytest.raises(gpu.NeoGpuError) as e:
        ctx.commit_noalloc(dummy.data_ptr(), 405, m, out.data_ptr())  # 405 * 16 * 81 > 524288
    assert e.value.code == 1


def _noalloc(ctx, Z, kappa):
    import torch
    n_vec, _, m = Z.shape
    d_z = torch.from_numpy(Z).cuda()
    d_out = torch.zeros((n_vec, kappa, 54), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.commit_noalloc(d_z.data_ptr(), n_vec, m, d_out.data_ptr())
    ctx.synchronize()
    return d_out.cpu().numpy().view(np.uint64)


def test_commit_noalloc_at_the_capacity_limit(ctx):
    # 404 vectors at kappa = 16: 404 * 16 * 81 = 523,584 of the 524,288 words
    m = 64
    rng = np.random.default_rng(404)
    pp = rng.integers(0, Q, size=(16, m, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    Z = rng.integers(-1, 2, size=(404, 54, m)).astype(np.int8)
    assert np.array_equal(_noalloc(ctx, Z, 16), ctx.commit(Z))


def test_commit_noalloc_other_kappa_and_odd_m(ctx):
    m = 1000
    rng = np.random.default_rng(8)
    pp = rng.integers(0, Q, size=(8, m, 54), dtype=np.uint64)
    ctx.pp_upload(pp)
    Z = rng.integers(-1, 2, size=(5, 54, m)).astype(np.int8)
    assert np.array_equal(_noalloc(ctx, Z, 8), ctx.commit(Z))


def test_commit_noalloc_without_pp_is_an_argument_error(ctx):
    import torch
    dummy = torch.zeros(16, dtype=torch.int8, device="cuda")
    out = torch.zeros(16, dtype=torch.int64, device="cuda")
    with pytest.raises(gpu.NeoGpuError) as e:
        ctx.commit_noalloc(dummy.data_ptr(), 1, 12345, out.data_ptr())  # no PP registered for m = 12345
    assert e.value.code == 1
