"""mpm_sort_particles_device_static: the Morton-key sort for hosts that cannot
allocate device memory (their memory belongs to another allocator, or their
frame loop must not block on cudaMalloc/cudaFree).  Its scratch is a fixed
array inside the library, shared by every call and never cleared, so the
check runs two calls in a row, the second smaller than the first, and
compares each with the allocating entry point, mpm_sort_particles_device.
Keys and permutation are integers: the tolerance is bit-exact, as in the
other sort tests.

This file sorts last (test_zz_*) so that a run stopping at the first failure
has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _positions(n, rng):
    """Uniform over a 128^3 grid plus a clustered part with many equal keys."""
    pos = rng.uniform(0, 128, (3, n)).astype(np.float32)
    k = n // 3
    pos[:, :k] = (rng.integers(0, 6, (3, k)) + rng.random((3, k)) * 0.999).astype(np.float32)
    return pos


def _sort_both(mpm, pos):
    import torch
    n = pos.shape[1]
    d = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for fn in (mpm.sort_particles_device, mpm.sort_particles_device_static):
        keys = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        perm = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        fn(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), n, keys.data_ptr(), perm.data_ptr(), stream)
        torch.cuda.synchronize()
        out.append((keys.cpu().numpy(), perm.cpu().numpy()))
    return out


def test_static_sort_matches_allocating_sort_twice(gpu_ok, mpm):
    rng = np.random.default_rng(2024)
    # The maximum size first, then a smaller one over the stale scratch.
    for n in (mpm.SORT_STATIC_MAX_PARTICLES, 100_003):
        (k_ref, p_ref), (k_st, p_st) = _sort_both(mpm, _positions(n, rng))
        assert np.array_equal(k_st, k_ref), f"keys differ at n={n}"
        assert np.array_equal(p_st, p_ref), f"permutation differs at n={n}"
        assert np.array_equal(np.sort(p_st), np.arange(n, dtype=np.int32))


def test_static_sort_allocates_nothing(gpu_ok, mpm):
    """After a first call (which may load the module), a static sort leaves
    the device's free memory unchanged."""
    import torch
    rng = np.random.default_rng(7)
    n = 300_000
    d = torch.from_numpy(np.ascontiguousarray(_positions(n, rng))).cuda()
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = (d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), n, keys.data_ptr(), perm.data_ptr(), stream)
    mpm.sort_particles_device_static(*args)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        mpm.sort_particles_device_static(*args)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_sort_rejects_oversize(gpu_ok, mpm):
    n = mpm.SORT_STATIC_MAX_PARTICLES + 1
    with pytest.raises(mpm.MpmError) as ei:
        mpm.sort_particles_device_static(1, 1, 1, n, 1, 1, 0)  # rejected before any pointer is used
    assert ei.value.name == "MPM_ERR_INVALID_ARGUMENT"
    assert "maximum" in str(ei.value)
