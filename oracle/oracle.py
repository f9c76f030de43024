"""ctypes wrappers of the CPU oracle and the reference engine.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py for the CPU-baseline leg and the reference arm.
The engine under test never calls into this module.

* `Oracle(64)` - FP64 restatement of the reference step (lib/libmpm_oracle64.so)
* `Oracle(32)` - FP32 OpenMP restatement, the timed CPU baseline
* `SceneOracle` - scene construction from OBJ models (lib/libscene_oracle.so)
* `RefEngine`  - the reference's own Engine compiled from its sources
                 (_ref/libref_engine.so); needs a GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_engine.so")


class _Params(ctypes.Structure):
    _fields_ = [("sx", ctypes.c_int32), ("sy", ctypes.c_int32), ("sz", ctypes.c_int32), ("padding", ctypes.c_int32),
                ("gravity", ctypes.c_float), ("dt", ctypes.c_float), ("gamma", ctypes.c_float),
                ("compression", ctypes.c_float), ("resolution", ctypes.c_float)]


def _params(cfg) -> _Params:
    return _Params(cfg.size_x, cfg.size_y, cfg.size_z, cfg.padding, cfg.gravity, cfg.dt, cfg.gamma,
                   cfg.compression, cfg.resolution)


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """CPU restatement of Engine::step / makeSDF at 64- or 32-bit precision."""

    def __init__(self, bits: int = 64):
        path = os.path.join(HERE, "lib", f"libmpm_oracle{bits}.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        self.lib = ctypes.CDLL(path)
        self.dtype = np.float64 if bits == 64 else np.float32
        P, L, V = ctypes.c_void_p, ctypes.c_long, None
        for name, res, args in [
            ("orc_init_particles", V, [P, P, L]), ("orc_morton_keys", V, [P, L, P]),
            ("orc_sort_perm", V, [P, L, P]), ("orc_p2g", V, [P, P, L, P, P, ctypes.c_int]),
            ("orc_grid_update", V, [P, P, P]), ("orc_g2p", V, [P, P, L, P, P, P]),
            ("orc_substep", V, [P, P, L, P, P, P, P, ctypes.c_int]), ("orc_positions", V, [P, L, P]),
            ("orc_make_sdf", V, [P, P, L, P, P]), ("orc_make_sdf_nodes", V, [P, P, L, P, L, P, P]),
            ("orc_real_bytes", ctypes.c_int, []),
            ("orc_threads", ctypes.c_int, []), ("orc_set_threads", V, [ctypes.c_int]),
        ]:
            f = getattr(self.lib, name)
            f.restype = res
            f.argtypes = args
        assert self.lib.orc_real_bytes() == np.dtype(self.dtype).itemsize

    def set_threads(self, n: int):
        self.lib.orc_set_threads(n)

    def threads(self) -> int:
        return self.lib.orc_threads()

    def _state(self, st):
        return np.ascontiguousarray(st, dtype=self.dtype).reshape(26, -1).copy()

    def init_particles(self, cfg, st):
        s = self._state(st)
        self.lib.orc_init_particles(ctypes.byref(_params(cfg)), _p(s), s.shape[1])
        return s

    def morton_keys(self, st):
        s = self._state(st)
        keys = np.empty(s.shape[1], np.int32)
        self.lib.orc_morton_keys(_p(s), s.shape[1], _p(keys))
        return keys

    def sort_perm(self, keys):
        k = np.ascontiguousarray(keys, np.int32)
        perm = np.empty(k.size, np.int32)
        self.lib.orc_sort_perm(_p(k), k.size, _p(perm))
        return perm

    def p2g(self, cfg, st, perm, tile_mode=1):
        s = self._state(st)
        grid = np.zeros((4, cfg.grid_number), self.dtype)
        self.lib.orc_p2g(ctypes.byref(_params(cfg)), _p(s), s.shape[1], _p(np.ascontiguousarray(perm, np.int32)),
                         _p(grid), tile_mode)
        return grid

    def grid_update(self, cfg, grid, sdf):
        g = np.ascontiguousarray(grid, self.dtype).copy()
        d = np.ascontiguousarray(sdf, self.dtype)
        self.lib.orc_grid_update(ctypes.byref(_params(cfg)), _p(g), _p(d))
        return g

    def g2p(self, cfg, st, perm, grid, sdf):
        s = self._state(st)
        g = np.ascontiguousarray(grid, self.dtype)
        d = np.ascontiguousarray(sdf, self.dtype)
        pp = None if perm is None else np.ascontiguousarray(perm, np.int32)
        self.lib.orc_g2p(ctypes.byref(_params(cfg)), _p(s), s.shape[1], _p(pp), _p(g), _p(d))
        return s

    def substep(self, cfg, st, sdf, tile_mode=1):
        """One Engine::step(): returns (state, grid, keys, perm)."""
        s = self._state(st)
        n = s.shape[1]
        grid = np.zeros((4, cfg.grid_number), self.dtype)
        keys = np.empty(n, np.int32)
        perm = np.empty(n, np.int32)
        d = np.ascontiguousarray(sdf, self.dtype)
        self.lib.orc_substep(ctypes.byref(_params(cfg)), _p(s), n, _p(grid), _p(d), _p(keys), _p(perm), tile_mode)
        return s, grid, keys, perm

    def make_sdf(self, cfg, tris):
        t = np.ascontiguousarray(tris, self.dtype).reshape(-1)
        sdf = np.empty(cfg.grid_number, self.dtype)
        wn = np.empty(cfg.grid_number, self.dtype)
        self.lib.orc_make_sdf(ctypes.byref(_params(cfg)), _p(t), t.size // 9, _p(sdf), _p(wn))
        return sdf, wn

    def make_sdf_nodes(self, cfg, tris, nodes):
        """(sdf, winding number) at the grid nodes `nodes` (flat indices)."""
        t = np.ascontiguousarray(tris, self.dtype).reshape(-1)
        idx = np.ascontiguousarray(nodes, np.int64)
        sdf = np.empty(idx.size, self.dtype)
        wn = np.empty(idx.size, self.dtype)
        self.lib.orc_make_sdf_nodes(ctypes.byref(_params(cfg)), _p(t), t.size // 9, _p(idx), idx.size, _p(sdf), _p(wn))
        return sdf, wn

    def empty_sdf(self, cfg):
        return np.full(cfg.grid_number, np.sqrt(np.float32(1e30)), self.dtype)


class RefEngine:
    """The reference's Engine (engine.cu) driven headless; one per process."""

    def __init__(self):
        if not os.path.exists(REF_LIB):
            raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference tree exists")
        self.lib = ctypes.CDLL(REF_LIB)
        P, L, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
        for name, res, args in [
            ("ref_config_reset", None, []), ("ref_config_load", None, [ctypes.c_char_p]),
            ("ref_config_has", I, [ctypes.c_char_p]), ("ref_config_get_int", I, [ctypes.c_char_p]),
            ("ref_config_get_float", ctypes.c_float, [ctypes.c_char_p]),
            ("ref_config_entries", I, [I, P, P, I, I]),
            ("ref_engine_create", I, [L, P]), ("ref_engine_init_sdf", I, [P, L]),
            ("ref_engine_set_state", I, [P]), ("ref_engine_step", I, [I]), ("ref_engine_time_steps", ctypes.c_float, [I]),
            ("ref_engine_get_state", I, [P]), ("ref_engine_get_grid", I, [P]), ("ref_engine_get_sdf", I, [P]),
            ("ref_engine_get_positions", I, [P]), ("ref_engine_get_perm", I, [P]), ("ref_engine_keys", I, [P]),
            ("ref_engine_sort_only", I, []), ("ref_engine_destroy", None, []),
            ("ref_engine_time_stages", I, [I, P]), ("ref_time_make_sdf", ctypes.c_float, [P, L]),
            ("ref_time_sort", ctypes.c_float, [I]),
        ]:
            f = getattr(self.lib, name)
            f.restype = res
            f.argtypes = args
        self.n = 0
        self.g = 0

    def load_config_text(self, text: str, path: str):
        with open(path, "w") as f:
            f.write(text)
        self.lib.ref_config_load(path.encode())

    def create(self, cfg, state26, tris, cfg_path: str):
        """Simulation's hand-off: config upload, Engine::init, Engine::initSDF."""
        self.load_config_text(cfg.to_text(), cfg_path)
        st = np.ascontiguousarray(state26, np.float32).reshape(26, -1)
        self.n = st.shape[1]
        self.g = cfg.grid_number
        rc = self.lib.ref_engine_create(self.n, _p(st))
        if rc != 0:
            raise RuntimeError(f"reference engine refused this scene (rc={rc}): grid nodes % 256 != 0 or n == 0")
        t = np.ascontiguousarray(tris, np.float32).reshape(-1)
        rc = self.lib.ref_engine_init_sdf(_p(t) if t.size else None, t.size // 9)
        if rc != 0:
            raise RuntimeError(f"reference initSDF failed (rc={rc})")

    def set_state(self, state26):
        """The particle buffer replaced by `state26` as it is (no initFMatrices)."""
        st = np.ascontiguousarray(state26, np.float32).reshape(26, -1)
        assert st.shape[1] == self.n
        assert self.lib.ref_engine_set_state(_p(st)) == 0

    def step(self, nsub=1):
        assert self.lib.ref_engine_step(nsub) == 0

    def time_steps(self, nsub) -> float:
        return float(self.lib.ref_engine_time_steps(nsub))

    def state(self):
        out = np.empty((26, self.n), np.float32)
        assert self.lib.ref_engine_get_state(_p(out)) == 0
        return out

    def grid(self):
        out = np.empty((4, self.g), np.float32)
        assert self.lib.ref_engine_get_grid(_p(out)) == 0
        return out

    def sdf(self):
        out = np.empty(self.g, np.float32)
        assert self.lib.ref_engine_get_sdf(_p(out)) == 0
        return out

    def positions(self):
        out = np.empty((self.n, 3), np.float32)
        assert self.lib.ref_engine_get_positions(_p(out)) == 0
        return out

    def perm(self):
        out = np.empty(self.n, np.int32)
        assert self.lib.ref_engine_get_perm(_p(out)) == 0
        return out

    def keys(self):
        out = np.empty(self.n, np.int32)
        assert self.lib.ref_engine_keys(_p(out)) == 0
        return out

    def sort_only(self):
        assert self.lib.ref_engine_sort_only() == 0

    def time_stages(self, nsub):
        """Per-stage device ms summed over nsub substeps: sort, clear, p2g, grid, g2p, export."""
        ms = np.zeros(6, np.float32)
        assert self.lib.ref_engine_time_stages(nsub, _p(ms)) == 0
        return dict(zip(("sort", "clear", "p2g", "grid", "g2p", "export"), ms.astype(float)))

    def time_make_sdf(self, tris) -> float:
        t = np.ascontiguousarray(tris, np.float32).reshape(-1)
        return float(self.lib.ref_time_make_sdf(_p(t) if t.size else None, t.size // 9))

    def time_sort(self, reps=10) -> float:
        return float(self.lib.ref_time_sort(reps))

    def destroy(self):
        self.lib.ref_engine_destroy()


class SceneOracle:
    """CPU restatement of the reference's OBJ -> particles / triangles path."""

    def __init__(self):
        path = os.path.join(HERE, "lib", "libscene_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        self.lib = ctypes.CDLL(path)
        P, L = ctypes.c_void_p, ctypes.c_long
        PP = ctypes.POINTER(ctypes.c_void_p)
        for name, res, args in [
            ("sco_free", None, [P]),
            ("sco_parse_obj", L, [ctypes.c_char_p, PP, ctypes.POINTER(L), PP, ctypes.POINTER(L)]),
            ("sco_voxelize", L, [P, L, P, L, ctypes.c_float, PP]),
            ("sco_normalize", L, [P, L, ctypes.c_float, ctypes.c_float, P, ctypes.c_int, PP]),
            ("sco_normalize_triangles", L, [P, L, ctypes.c_float, ctypes.c_float, P]),
        ]:
            f = getattr(self.lib, name)
            f.restype = res
            f.argtypes = args

    def _take(self, ptr, count, dtype):
        if not ptr:
            return np.zeros(0, dtype)
        buf = (ctypes.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr)
        out = np.frombuffer(bytes(buf), dtype=dtype).copy()
        self.lib.sco_free(ptr)
        return out

    def parse_obj(self, text: str):
        """(vertices (nv, 3) float32, faces (nt, 3) int32); raises on a malformed file."""
        v, f = ctypes.c_void_p(), ctypes.c_void_p()
        nv, nt = ctypes.c_long(), ctypes.c_long()
        line = self.lib.sco_parse_obj(text.encode(), ctypes.byref(v), ctypes.byref(nv), ctypes.byref(f),
                                      ctypes.byref(nt))
        if line:
            raise ValueError(f"OBJ line {line}")
        return (self._take(v.value, 3 * nv.value, np.float32).reshape(-1, 3),
                self._take(f.value, 3 * nt.value, np.int32).reshape(-1, 3))

    def voxelize(self, verts, faces, resolution: float = 100.0):
        v = np.ascontiguousarray(verts, np.float32)
        f = np.ascontiguousarray(faces, np.int32)
        out = ctypes.c_void_p()
        n = self.lib.sco_voxelize(_p(v), len(v), _p(f), len(f), resolution, ctypes.byref(out))
        if n < 0:
            raise ValueError("degenerate mesh")
        return self._take(out.value, 3 * n, np.float32).reshape(-1, 3)

    def normalize(self, pts, size: float, scale: float, disp, step: int):
        p = np.ascontiguousarray(pts, np.float32)
        d = np.ascontiguousarray(disp, np.float32)
        out = ctypes.c_void_p()
        n = self.lib.sco_normalize(_p(p), len(p), size, scale, _p(d), step, ctypes.byref(out))
        if n < 0:
            raise ValueError("lattice step below 1")
        return self._take(out.value, 3 * n, np.float32).reshape(-1, 3)

    def normalize_triangles(self, tris, size: float, scale: float, disp):
        t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9).copy()
        d = np.ascontiguousarray(disp, np.float32)
        k = self.lib.sco_normalize_triangles(_p(t), len(t), size, scale, _p(d))
        return t[:k]
