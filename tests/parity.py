"""Comparison rules of the parity tests.

Tolerances (FP32 engine vs FP64 oracle, one substep, same inputs):
  * Morton keys and sort permutation: bit-exact.
  * velocity, F: max |got - want| <= RTOL * max |want| over the field
    (normwise relative error, RTOL = 1e-5).
  * C: the same, relative to max(max |C|, max |velocity|).  C = 4 sum w v
    (x_node - x_p)^T is a velocity over one cell; in uniform flow (a scene at
    rest under gravity) its terms cancel to near zero and what is left is the
    rounding of the velocity terms, so a velocity is its natural scale.
  * positions: the error of the DISPLACEMENT, max |got - want| <=
    RTOL * max |want - start| + 2 ulp(|position|) (a position near 100 cannot
    be stored closer than its float spacing).
  * grid mass / momentum / velocity: normwise relative, RTOL.
  * VOL and MASS: bit-identical (the engine never writes them).
"""
from __future__ import annotations

import numpy as np

RTOL = 1e-5


def normwise(got, want):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    err = float(np.max(np.abs(got - want))) if want.size else 0.0
    scale = float(np.max(np.abs(want))) if want.size else 0.0
    return err, scale


def assert_normwise(name, got, want, rtol=RTOL, floor=1e-12):
    err, scale = normwise(got, want)
    assert err <= rtol * max(scale, floor), f"{name}: max error {err:.3e} > {rtol:g} x {scale:.3e}"


def assert_state_close(got, want, start, rtol=RTOL):
    """got/want/start: (26, n) states; start is the input of the substep(s)."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    start = np.asarray(start, np.float64)
    if want.shape[1] == 0:
        return
    disp = np.max(np.abs(want[0:3] - start[0:3]))
    ulp = float(np.spacing(np.float32(np.max(np.abs(want[0:3])))))
    err = float(np.max(np.abs(got[0:3] - want[0:3])))
    assert err <= rtol * disp + 2 * ulp, f"position: max error {err:.3e} > {rtol:g} x {disp:.3e} + 2 ulp"
    assert_normwise("velocity", got[3:6], want[3:6], rtol)
    vmax = float(np.max(np.abs(want[3:6]))) if want.size else 0.0
    assert_normwise("C", got[6:15], want[6:15], rtol, floor=max(vmax, 1e-12))
    assert_normwise("F", got[15:24], want[15:24], rtol)
    assert np.array_equal(np.asarray(got[24:26], np.float32), np.asarray(want[24:26], np.float32)), "VOL/MASS changed"


def stable_sort_reference(keys):
    """thrust::sequence + sort_by_key on int keys: stable ascending."""
    return np.argsort(np.asarray(keys, np.int32), kind="stable").astype(np.int32)


def morton_reference(pos):
    """setKeys (kernels.cu:361-371) in numpy, for positions of shape (3, n)."""
    p = np.asarray(pos, np.float32)
    with np.errstate(invalid="ignore"):
        c = np.where(np.isnan(p), np.float32(0), np.maximum(np.float32(0), p))
        big = c >= np.float32(4294967296.0)
        u = np.where(big, np.uint64(0xFFFFFFFF), np.floor(np.where(big, 0, c)).astype(np.float64).astype(np.uint64))
    u = u.astype(np.uint64) & np.uint64(0xFFFFFFFF)

    def spread(v):
        v = v.astype(np.uint64)
        m = np.uint64(0xFFFFFFFF)
        v = (v * np.uint64(0x00010001) & m) & np.uint64(0xFF0000FF)
        v = (v * np.uint64(0x00000101) & m) & np.uint64(0x0F00F00F)
        v = (v * np.uint64(0x00000011) & m) & np.uint64(0xC30C30C3)
        v = (v * np.uint64(0x00000005) & m) & np.uint64(0x49249249)
        return v

    k = ((spread(u[2]) << np.uint64(2)) | (spread(u[1]) << np.uint64(1)) | spread(u[0])) & np.uint64(0xFFFFFFFF)
    return k.astype(np.uint32).view(np.int32)
