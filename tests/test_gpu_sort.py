"""Morton keys and the stable sort, bit-exact (setKeys kernels.cu:361-371,
thrust::sequence + sort_by_key engine.cu:98-99)."""
import numpy as np
import pytest

from parity import morton_reference, stable_sort_reference

pytestmark = pytest.mark.gpu


def _positions(kind, n, rng):
    if kind == "grid128":
        return rng.uniform(0, 128, (3, n)).astype(np.float32)
    if kind == "clustered":  # many ties: 8 particles per cell over a small block
        return (rng.integers(0, 6, (3, n)) + rng.random((3, n)) * 0.999).astype(np.float32)
    if kind == "edge":
        # negative, NaN, +/-inf, beyond 1024 (aliasing), huge, exact integers
        vals = np.array([-5.0, -0.0, 0.0, 0.99999994, 1.0, 1023.9999, 1024.0, 1500.5, 65535.0, 3.0e9, 5.0e9,
                         np.inf, -np.inf, np.nan, 127.5, 2.0 ** 31, 2.0 ** 32 - 256], np.float32)
        return rng.choice(vals, (3, n)).astype(np.float32)
    raise ValueError(kind)


def _sort_device(mpm, pos):
    import torch
    n = pos.shape[1]
    d = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    keys = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    perm = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    mpm.sort_particles_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), n, keys.data_ptr(),
                              perm.data_ptr(), s)
    torch.cuda.synchronize()
    return keys.cpu().numpy()[:n], perm.cpu().numpy()[:n]


@pytest.mark.parametrize("n", [1, 2, 31, 255, 256, 257, 2047, 2048, 2049, 100_003, 1_989_120])
@pytest.mark.parametrize("kind", ["grid128", "clustered"])
def test_sort_bitexact(gpu_ok, mpm, n, kind):
    rng = np.random.default_rng(n + len(kind))
    pos = _positions(kind, n, rng)
    keys, perm = _sort_device(mpm, pos)
    want_keys = morton_reference(pos)
    assert np.array_equal(keys, want_keys)
    assert np.array_equal(perm, stable_sort_reference(want_keys))


def test_sort_edge_values(gpu_ok, mpm):
    rng = np.random.default_rng(5)
    pos = _positions("edge", 50_000, rng)
    keys, perm = _sort_device(mpm, pos)
    want_keys = morton_reference(pos)
    assert np.array_equal(keys, want_keys)
    assert (want_keys < 0).any(), "edge set should produce keys with the sign bit set"
    assert np.array_equal(perm, stable_sort_reference(want_keys))


def test_sort_matches_oracle(gpu_ok, mpm, oracle64):
    rng = np.random.default_rng(9)
    pos = _positions("grid128", 70_000, rng)
    st = np.zeros((26, pos.shape[1]))
    st[0:3] = pos
    keys, perm = _sort_device(mpm, pos)
    ok = oracle64.morton_keys(st)
    assert np.array_equal(keys, ok)
    assert np.array_equal(perm, oracle64.sort_perm(ok))


def test_sort_empty(gpu_ok, mpm):
    keys, perm = _sort_device(mpm, np.zeros((3, 0), np.float32))
    assert keys.size == 0 and perm.size == 0


def test_engine_sort_each_substep(gpu_ok, mpm):
    """The engine's per-substep sort equals the stable sort of the keys of the
    state the substep started from, substep after substep."""
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(20_000, (32, 32, 32), seed=4)
    with mpm.Engine(cfg) as eng:
        eng.init(st)
        eng.init_sdf(tris)
        for _ in range(6):
            before = eng.get_buffer()
            eng.step(1)
            keys, perm = eng.get_sort()
            want = morton_reference(before[0:3])
            assert np.array_equal(keys, want)
            assert np.array_equal(perm, stable_sort_reference(want))
