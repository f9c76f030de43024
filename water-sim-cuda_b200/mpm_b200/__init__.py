"""Python mirror of the B200 MLS-MPM engine's C ABI (include/mpm_b200.h).

The class `Engine` mirrors the reference's C++ `Engine` (engine.h:14-43):
`init(n, buffer)`, `step()`, `init_sdf(triangles)`, `get_buffer()`,
`get_positions()`, `get_grid()`, `get_number()`, and `sort_particles()`;
`parse_config_file` mirrors GameConfigData (game_configdata.cpp:22-90).
Every call goes through libmpm_b200.so.  There is no CPU fallback: the first
call into the library raises when it has not been built.  The library is
mapped on that first call, not at import, so that code which only needs the
pure-numpy parts (`Config`, `scenes`) maps no GPU code.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libmpm_b200.so")

PARTICLE_PLANES = 26
GRID_PLANES = 4
POS_X, VEL_X, C00, F00, VOL, MASS = 0, 3, 6, 15, 24, 25
STAGE_SORT, STAGE_P2G, STAGE_GRID, STAGE_G2P = 1, 2, 3, 4
HEALTH_NONFINITE, HEALTH_OUT_OF_GRID = 1, 2
FALLBACK_RULES = {"density_change": 0, "rest_density": 1, "rest_density_excess": 2}
WAIT_TEST_SDF_GIVE_UP, WAIT_TEST_SDF_EXPIRE, WAIT_TEST_MMA_GIVE_UP, WAIT_TEST_MMA_EXPIRE = 1, 2, 4, 8
SORT_STATIC_MAX_PARTICLES = 1 << 20  # MPM_SORT_STATIC_MAX_PARTICLES
CORRECTOR_PARAMS, CORRECTOR_FEATURES, CORRECTOR_OUTPUTS = 5478, 16, 3

STATUS = {
    0: "MPM_OK", 1: "MPM_ERR_INVALID_ARGUMENT", 2: "MPM_ERR_BAD_CONFIG", 3: "MPM_ERR_IO",
    4: "MPM_ERR_CUDA", 5: "MPM_ERR_OUT_OF_MEMORY", 6: "MPM_ERR_NOT_INITIALIZED",
    7: "MPM_ERR_NONFINITE_STATE", 8: "MPM_ERR_OUT_OF_GRID", 9: "MPM_ERR_TIMEOUT",
    10: "MPM_ERR_UNSUPPORTED", 11: "MPM_ERR_NO_DEVICE",
}


class MpmError(RuntimeError):
    """A non-zero mpm_status, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS.get(status, f"status {status}")
        super().__init__(f"{self.name}: {message}")


class _Config(ctypes.Structure):
    _fields_ = [
        ("size_x", ctypes.c_int32), ("size_y", ctypes.c_int32), ("size_z", ctypes.c_int32),
        ("padding", ctypes.c_int32), ("gravity", ctypes.c_float), ("dt", ctypes.c_float),
        ("gamma", ctypes.c_float), ("compression", ctypes.c_float), ("resolution", ctypes.c_float),
        ("substeps", ctypes.c_int32), ("sdf_resolution", ctypes.c_int32),
    ]


class _SceneEntry(ctypes.Structure):
    _fields_ = [("model_path", ctypes.c_char * 512), ("scale", ctypes.c_float),
                ("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class _LearnedStats(ctypes.Structure):
    _fields_ = [("large_steps", ctypes.c_int64), ("fallbacks", ctypes.c_int64),
                ("last_density_change", ctypes.c_double)]


class _Tuning(ctypes.Structure):
    _fields_ = [("p2g_ctas_per_sm", ctypes.c_int32), ("g2p_block", ctypes.c_int32), ("grid_block", ctypes.c_int32),
                ("p2g_ms", ctypes.c_float), ("g2p_ms", ctypes.c_float), ("grid_ms", ctypes.c_float),
                ("p2g_cell_cap", ctypes.c_int32)]


class _Stats(ctypes.Structure):
    _fields_ = [("substeps", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("sort_passes", ctypes.c_int64), ("health", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


@dataclass
class SceneEntry:
    """A WATER= or OBJECT= line: `path;scale;x;y;z` (struct ConfigObject)."""
    model_path: str
    scale: float
    x: float
    y: float
    z: float


@dataclass
class Config:
    """The config.txt keys of SimConfig (common.cuh:65-79)."""
    size_x: int = 128
    size_y: int = 128
    size_z: int = 128
    padding: int = 2
    gravity: float = 9.81
    dt: float = 0.01
    gamma: float = -2.0
    compression: float = 200.0
    resolution: float = 1.0
    substeps: int = 10
    sdf_resolution: int = 256
    waters: list = field(default_factory=list)
    objects: list = field(default_factory=list)

    @property
    def grid_number(self) -> int:
        return self.size_x * self.size_y * self.size_z

    def to_c(self) -> _Config:
        return _Config(self.size_x, self.size_y, self.size_z, self.padding, self.gravity, self.dt,
                       self.gamma, self.compression, self.resolution, self.substeps, self.sdf_resolution)

    def to_text(self) -> str:
        """config.txt text with float values that read back bit-identically."""
        f = lambda v: repr(float(np.float32(v)))
        lines = [f"SIZE_X={self.size_x}", f"SIZE_Y={self.size_y}", f"SIZE_Z={self.size_z}",
                 f"PADDING={self.padding}", f"GRAVITY={f(self.gravity)}", f"DT={f(self.dt)}",
                 f"GAMMA={f(self.gamma)}", f"COMPRESSION={f(self.compression)}",
                 f"RESOLUTION={f(self.resolution)}", f"SUBSTEPS={self.substeps}",
                 f"SDF_RESOLUTION={self.sdf_resolution}"]
        for tag, entries in (("WATER", self.waters), ("OBJECT", self.objects)):
            for e in entries:
                lines.append(f"{tag}={e.model_path};{f(e.scale)};{f(e.x)};{f(e.y)};{f(e.z)}")
        return "\n".join(lines) + "\n"


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C water-sim-cuda_b200` "
                           "(or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P, I32, I64, U32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
    sigs = {
        "mpm_abi_version": (I32, []),
        "mpm_status_string": (ctypes.c_char_p, [I32]),
        "mpm_config_parse_file": (I32, [ctypes.c_char_p, P, P, I32, P, P, I32, P, ctypes.c_char_p, I32]),
        "mpm_config_parse_string": (I32, [ctypes.c_char_p, P, P, I32, P, P, I32, P, ctypes.c_char_p, I32]),
        "mpm_create": (I32, [P, I32, P]),
        "mpm_destroy": (None, [P]),
        "mpm_init_particles": (I32, [P, I64, P]),
        "mpm_init_sdf": (I32, [P, P, I64]),
        "mpm_step": (I32, [P, I32]),
        "mpm_step_async": (I32, [P, I32]),
        "mpm_synchronize": (I32, [P]),
        "mpm_substep_partial": (I32, [P, I32]),
        "mpm_set_checks": (I32, [P, U32]),
        "mpm_set_wait_test": (I32, [P, U32]),
        "mpm_num_particles": (I64, [P]),
        "mpm_get_state": (I32, [P, P]),
        "mpm_set_state": (I32, [P, I64, P]),
        "mpm_positions_device": (P, [P]),
        "mpm_get_positions": (I32, [P, P]),
        "mpm_get_positions_async": (I32, [P, P]),
        "mpm_positions_wait": (I32, [P]),
        "mpm_get_grid": (I32, [P, P]),
        "mpm_get_sdf": (I32, [P, P]),
        "mpm_get_sort": (I32, [P, P, P]),
        "mpm_get_stats": (I32, [P, P, I32]),
        "mpm_set_stage_timing": (I32, [P, I32]),
        "mpm_get_stage_times": (I32, [P, P, P]),
        "mpm_stream": (P, [P]),
        "mpm_last_error": (ctypes.c_char_p, [P]),
        "mpm_global_last_error": (ctypes.c_char_p, []),
        "mpm_sort_particles_device": (I32, [P, P, P, I64, P, P, P]),
        "mpm_sort_particles_device_static": (I32, [P, P, P, I64, P, P, P]),
        "mpm_create_batch": (I32, [P, I32, I32, P]),
        "mpm_num_scenes": (I32, [P]),
        "mpm_init_particles_batch": (I32, [P, P, P]),
        "mpm_scene_init_sdf": (I32, [P, I32, P, I64]),
        "mpm_scene_num_particles": (I64, [P, I32]),
        "mpm_scene_get_state": (I32, [P, I32, P]),
        "mpm_scene_positions_device": (P, [P, I32]),
        "mpm_scene_get_positions": (I32, [P, I32, P]),
        "mpm_scene_get_grid": (I32, [P, I32, P]),
        "mpm_scene_get_sdf": (I32, [P, I32, P]),
        "mpm_scene_get_sort": (I32, [P, I32, P, P]),
        "mpm_scene_build": (I32, [ctypes.c_char_p, ctypes.c_char_p, I32, P]),
        "mpm_scene_data_free": (None, [P]),
        "mpm_scene_data_num_particles": (I64, [P]),
        "mpm_scene_data_num_triangles": (I64, [P]),
        "mpm_scene_data_state": (I32, [P, P]),
        "mpm_scene_data_triangles": (I32, [P, P]),
        "mpm_scene_data_log": (ctypes.c_char_p, [P]),
        "mpm_scene_last_error": (ctypes.c_char_p, []),
        "mpm_mesh_load_obj": (I32, [ctypes.c_char_p, P]),
        "mpm_mesh_from_obj_text": (I32, [ctypes.c_char_p, P]),
        "mpm_mesh_free": (None, [P]),
        "mpm_mesh_num_vertices": (I64, [P]),
        "mpm_mesh_num_triangles": (I64, [P]),
        "mpm_mesh_get": (I32, [P, P, P, P]),
        "mpm_voxelize": (I32, [P, ctypes.c_float, I32, P]),
        "mpm_points_create": (I32, [P, I64, P]),
        "mpm_points_count": (I64, [P]),
        "mpm_points_get": (I32, [P, P]),
        "mpm_points_free": (None, [P]),
        "mpm_points_normalize": (I32, [P, ctypes.c_float, ctypes.c_float, P, I32, I32]),
        "mpm_triangles_normalize": (I32, [P, P, ctypes.c_float, ctypes.c_float, P]),
        "mpm_checkpoint_save": (I32, [P, ctypes.c_char_p, ctypes.c_char_p]),
        "mpm_checkpoint_load": (I32, [ctypes.c_char_p, I32, P]),
        "mpm_checkpoint_info": (I32, [ctypes.c_char_p, P, P, P, ctypes.c_char_p, I32]),
        "mpm_render_params_default": (None, [P, I32, I32, I32]),
        "mpm_renderer_create": (I32, [P, I32, P]),
        "mpm_renderer_destroy": (None, [P]),
        "mpm_renderer_last_error": (ctypes.c_char_p, [P]),
        "mpm_renderer_set_background": (I32, [P, P]),
        "mpm_renderer_set_obstacles": (I32, [P, P, I64, P]),
        "mpm_renderer_get_background": (I32, [P, P, P]),
        "mpm_render_points": (I32, [P, P, I64, P]),
        "mpm_render_frame": (I32, [P, P]),
        "mpm_renderer_get_depth": (I32, [P, I32, P]),
        "mpm_renderer_get_image": (I32, [P, P, P]),
        "mpm_autotune": (I32, [P, I32, P]),
        "mpm_set_tuning": (I32, [P, P]),
        "mpm_get_tuning": (I32, [P, P]),
        "mpm_set_corrector": (I32, [P, P, I32, ctypes.c_float]),
        "mpm_step_learned": (I32, [P, I32, P]),
        "mpm_set_corrector_kernel": (I32, [P, I32]),
        "mpm_set_fallback_rule": (I32, [P, I32]),
        "mpm_set_fallback_on_device": (I32, [P, I32]),
        "mpm_learned_statistics": (I32, [P, P]),
        "mpm_corrector_create": (I32, [I32, I64, P]),
        "mpm_corrector_destroy": (None, [P]),
        "mpm_corrector_last_error": (ctypes.c_char_p, [P]),
        "mpm_corrector_size": (I64, [P]),
        "mpm_corrector_clear": (I32, [P]),
        "mpm_corrector_collect": (I32, [P, P, I64, ctypes.c_uint64]),
        "mpm_corrector_add_data": (I32, [P, I64, P, P]),
        "mpm_corrector_get_data": (I32, [P, I64, I64, P, P]),
        "mpm_corrector_init": (I32, [P, ctypes.c_uint64]),
        "mpm_corrector_train": (I32, [P, I32, I32, ctypes.c_float, ctypes.c_uint64, P]),
        "mpm_corrector_gradient": (I32, [P, I64, P, P, P]),
        "mpm_corrector_set_train_kernel": (I32, [P, I32]),
        "mpm_corrector_get_params": (I32, [P, P]),
        "mpm_corrector_set_params": (I32, [P, P]),
        "mpm_corrector_forward": (I32, [P, I64, P, P]),
        "mpm_corrector_forward_tc": (I32, [P, I64, P, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _LazyLib:
    """libmpm_b200.so, loaded (and its signatures set) on the first attribute
    access; raises RuntimeError there if the library is missing."""

    _cdll = None

    def __getattr__(self, name):
        if _LazyLib._cdll is None:
            _LazyLib._cdll = _load()
        return getattr(_LazyLib._cdll, name)

    @staticmethod
    def loaded() -> bool:
        return _LazyLib._cdll is not None


lib = _LazyLib()


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _parse(fn, arg, max_entries=64) -> Config:
    c = _Config()
    waters = (_SceneEntry * max_entries)()
    objects = (_SceneEntry * max_entries)()
    nw, no = ctypes.c_int32(0), ctypes.c_int32(0)
    err = ctypes.create_string_buffer(1024)
    st = fn(arg, ctypes.byref(c), waters, max_entries, ctypes.byref(nw), objects, max_entries,
            ctypes.byref(no), err, len(err))
    if st != 0:
        raise MpmError(st, err.value.decode(errors="replace"))
    cfg = Config(c.size_x, c.size_y, c.size_z, c.padding, c.gravity, c.dt, c.gamma, c.compression,
                 c.resolution, c.substeps, c.sdf_resolution)
    conv = lambda e: SceneEntry(e.model_path.decode(errors="replace"), e.scale, e.x, e.y, e.z)
    cfg.waters = [conv(waters[i]) for i in range(min(nw.value, max_entries))]
    cfg.objects = [conv(objects[i]) for i in range(min(no.value, max_entries))]
    return cfg


def parse_config_file(path: str) -> Config:
    """GameConfigData::setConfigDataFromFile + the key reads of initDeviceParams."""
    return _parse(lib.mpm_config_parse_file, path.encode())


def parse_config_string(text: str) -> Config:
    return _parse(lib.mpm_config_parse_string, text.encode())


class Engine:
    """One simulation on one GPU (the reference's `Engine`, engine.h:14-43)."""

    def __init__(self, cfg: Config, device: int = 0):
        self.cfg = cfg
        handle = ctypes.c_void_p()
        c = cfg.to_c()
        st = lib.mpm_create(ctypes.byref(c), device, ctypes.byref(handle))
        if st != 0:
            raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))
        self._h = handle
        self.n = 0

    def _check(self, st: int):
        if st != 0:
            raise MpmError(st, lib.mpm_last_error(self._h).decode(errors="replace"))

    def close(self):
        if getattr(self, "_h", None):
            lib.mpm_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- Engine::init / initSDF -------------------------------------------------
    def init(self, state26: np.ndarray):
        """Engine::init(n, buffer): state26 is (26, n) or flat 26*n float32 (copied)."""
        a = np.ascontiguousarray(state26, dtype=np.float32).reshape(-1)
        if a.size % PARTICLE_PLANES:
            raise ValueError("state size is not a multiple of 26")
        n = a.size // PARTICLE_PLANES
        self._check(lib.mpm_init_particles(self._h, n, _ptr(a)))
        self.n = n

    def init_sdf(self, triangles: np.ndarray):
        """Engine::initSDF(triangles): (t, 9) or (t, 3, 3) float32 in grid coordinates."""
        t = np.ascontiguousarray(triangles, dtype=np.float32).reshape(-1)
        if t.size % 9:
            raise ValueError("triangle array size is not a multiple of 9")
        self._check(lib.mpm_init_sdf(self._h, _ptr(t) if t.size else None, t.size // 9))

    def set_state(self, state26: np.ndarray):
        a = np.ascontiguousarray(state26, dtype=np.float32).reshape(-1)
        self._check(lib.mpm_set_state(self._h, a.size // PARTICLE_PLANES, _ptr(a)))

    # -- stepping -----------------------------------------------------------------
    def step(self, nsub: int = 1):
        """nsub calls of Engine::step() (one substep each), synchronous."""
        self._check(lib.mpm_step(self._h, int(nsub)))

    def step_async(self, nsub: int = 1):
        self._check(lib.mpm_step_async(self._h, int(nsub)))

    def synchronize(self):
        self._check(lib.mpm_synchronize(self._h))

    def substep_partial(self, upto: int):
        self._check(lib.mpm_substep_partial(self._h, int(upto)))

    def set_checks(self, flags: int):
        self._check(lib.mpm_set_checks(self._h, int(flags)))

    def set_wait_test(self, flags: int):
        """Test hooks of the bounded device waits (WAIT_TEST_* bits; 0 clears)."""
        self._check(lib.mpm_set_wait_test(self._h, int(flags)))

    # -- readback -----------------------------------------------------------------
    def get_number(self) -> int:
        return int(lib.mpm_num_particles(self._h))

    def get_buffer(self) -> np.ndarray:
        """Engine::getBuffer() copied to the host: (26, n) float32, original order."""
        out = np.empty((PARTICLE_PLANES, self.n), np.float32)
        self._check(lib.mpm_get_state(self._h, _ptr(out)))
        return out

    def get_positions(self, out: np.ndarray | None = None) -> np.ndarray:
        """Engine::getPositions() copied to the host: (n, 3) float32."""
        if out is None:
            out = np.empty((self.n, 3), np.float32)
        self._check(lib.mpm_get_positions(self._h, _ptr(out)))
        return out

    def get_positions_async(self, out: np.ndarray):
        """Start reading the current positions into `out` (pinned for overlap); see positions_wait."""
        self._check(lib.mpm_get_positions_async(self._h, _ptr(out)))

    def positions_wait(self):
        self._check(lib.mpm_positions_wait(self._h))

    def positions_device_ptr(self) -> int:
        return int(lib.mpm_positions_device(self._h) or 0)

    def get_grid(self) -> np.ndarray:
        """Engine::getGrid() planes copied to the host: (4, G) float32."""
        out = np.empty((GRID_PLANES, self.cfg.grid_number), np.float32)
        self._check(lib.mpm_get_grid(self._h, _ptr(out)))
        return out

    def get_sdf(self) -> np.ndarray:
        out = np.empty(self.cfg.grid_number, np.float32)
        self._check(lib.mpm_get_sdf(self._h, _ptr(out)))
        return out

    def get_sort(self):
        """(keys, perm) of the last substep's sortParticles (engine.cu:92-102)."""
        keys = np.empty(self.n, np.int32)
        perm = np.empty(self.n, np.int32)
        self._check(lib.mpm_get_sort(self._h, _ptr(keys), _ptr(perm)))
        return keys, perm

    def stats(self, reset_health: bool = False) -> dict:
        s = _Stats()
        self._check(lib.mpm_get_stats(self._h, ctypes.byref(s), int(reset_health)))
        return {"substeps": s.substeps, "kernel_launches": s.kernel_launches,
                "sort_passes": s.sort_passes, "health": s.health}

    def stream(self) -> int:
        return int(lib.mpm_stream(self._h) or 0)

    # -- launch shapes --------------------------------------------------------
    def autotune(self, repeats: int = 3) -> dict:
        """Time the candidate launch shapes on the current particles; keep the fastest."""
        t = _Tuning()
        self._check(lib.mpm_autotune(self._h, int(repeats), ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _Tuning._fields_}

    def tuning(self) -> dict:
        t = _Tuning()
        self._check(lib.mpm_get_tuning(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _Tuning._fields_}

    def set_tuning(self, p2g_ctas_per_sm: int = 12, g2p_block: int = 256, grid_block: int = 256,
                   p2g_cell_cap: int = 0):
        t = _Tuning(int(p2g_ctas_per_sm), int(g2p_block), int(grid_block), 0.0, 0.0, 0.0, int(p2g_cell_cap))
        self._check(lib.mpm_set_tuning(self._h, ctypes.byref(t)))

    # -- checkpoints ----------------------------------------------------------
    def save_checkpoint(self, path: str, note: str = ""):
        """State (original order), SDF, config and substep count to one file."""
        self._check(lib.mpm_checkpoint_save(self._h, path.encode(), note.encode()))

    @classmethod
    def load_checkpoint(cls, path: str, device: int = 0) -> "Engine":
        info = checkpoint_info(path)
        h = ctypes.c_void_p()
        st = lib.mpm_checkpoint_load(path.encode(), int(device), ctypes.byref(h))
        if st != 0:
            raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))
        e = cls.__new__(cls)
        e.cfg, e._h, e.n = info["config"], h, info["n"]
        return e

    # -- learned large step ---------------------------------------------------
    def set_corrector(self, params: np.ndarray | None, ratio: int = 4, max_density_change: float = 0.02):
        """The corrector's MPM_CORRECTOR_PARAMS floats (None: uncorrected large steps)."""
        if params is None:
            self._check(lib.mpm_set_corrector(self._h, None, int(ratio), float(max_density_change)))
            return
        w = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        if w.size != CORRECTOR_PARAMS:
            raise ValueError(f"expected {CORRECTOR_PARAMS} parameters, got {w.size}")
        self._check(lib.mpm_set_corrector(self._h, _ptr(w), int(ratio), float(max_density_change)))

    def set_corrector_kernel(self, tcgen05: bool = True):
        """The MLP inside the learned G2P: tcgen05 + TMEM (default) or mma.sync."""
        self._check(lib.mpm_set_corrector_kernel(self._h, 0 if tcgen05 else 1))

    def set_fallback_rule(self, rule: str = "density_change"):
        """The fallback statistic: "density_change" (default), "rest_density" or
        "rest_density_excess" (mpm_set_fallback_rule)."""
        self._check(lib.mpm_set_fallback_rule(self._h, FALLBACK_RULES[rule]))

    def set_fallback_on_device(self, on_device: bool = True):
        """Decide a checked large step's fallback on the device (a conditional
        graph node, the default) or on the host (a read-back per step)."""
        self._check(lib.mpm_set_fallback_on_device(self._h, 1 if on_device else 0))

    def learned_statistics(self) -> dict:
        """The three fallback means of the last checked large step."""
        out = np.zeros(3, np.float64)
        self._check(lib.mpm_learned_statistics(self._h, _ptr(out)))
        return {"density_change": float(out[0]), "rest_density": float(out[1]), "rest_density_before": float(out[2])}

    def step_learned(self, nlarge: int = 1) -> dict:
        """nlarge large steps of RATIO x DT; returns the running learned-step counters."""
        s = _LearnedStats()
        self._check(lib.mpm_step_learned(self._h, int(nlarge), ctypes.byref(s)))
        return {"large_steps": s.large_steps, "fallbacks": s.fallbacks,
                "last_density_change": s.last_density_change}

    def set_stage_timing(self, max_substeps: int):
        """Record CUDA events between the stages of the next max_substeps substeps."""
        self._check(lib.mpm_set_stage_timing(self._h, int(max_substeps)))

    def stage_times(self):
        """({'sort','p2g','grid','g2p'}: summed ms, substeps recorded); clears the record."""
        ms = (ctypes.c_double * 4)()
        cnt = ctypes.c_int32(0)
        self._check(lib.mpm_get_stage_times(self._h, ms, ctypes.byref(cnt)))
        return dict(zip(("sort", "p2g", "grid", "g2p"), list(ms))), cnt.value


def sort_particles_device(px: int, py: int, pz: int, n: int, keys: int, perm: int, stream: int = 0):
    """Engine::sortParticles on caller-owned device buffers (raw device pointers)."""
    st = lib.mpm_sort_particles_device(px, py, pz, n, keys, perm, stream or None)
    if st != 0:
        raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))


def sort_particles_device_static(px: int, py: int, pz: int, n: int, keys: int, perm: int, stream: int = 0):
    """sort_particles_device without any device allocation: the scratch is a
    fixed array inside the library (n <= SORT_STATIC_MAX_PARTICLES).  For hosts
    that cannot allocate device memory; calls that overlap on the GPU race."""
    st = lib.mpm_sort_particles_device_static(px, py, pz, n, keys, perm, stream or None)
    if st != 0:
        raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))


class Batch(Engine):
    """Independent scenes of their own sizes, physics and obstacles, stepped
    together on one device: every substep stage is one launch over all
    scenes.  No counterpart in the reference (one scene per process)."""

    def __init__(self, cfgs, device: int = 0):
        self.cfgs = list(cfgs)
        self.cfg = self.cfgs[0]
        arr = (_Config * len(self.cfgs))(*[c.to_c() for c in self.cfgs])
        handle = ctypes.c_void_p()
        st = lib.mpm_create_batch(arr, len(self.cfgs), device, ctypes.byref(handle))
        if st != 0:
            raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))
        self._h = handle
        self.n = 0
        self.counts = [0] * len(self.cfgs)

    @property
    def scenes(self) -> int:
        return int(lib.mpm_num_scenes(self._h))

    def init_all(self, states):
        """Engine::init for every scene: states[s] is (26, n_s) or flat 26*n_s float32."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1) for a in states]
        if len(arrs) != len(self.cfgs) or any(a.size % PARTICLE_PLANES for a in arrs):
            raise ValueError("one 26-plane state per scene expected")
        counts = (ctypes.c_int64 * len(arrs))(*[a.size // PARTICLE_PLANES for a in arrs])
        ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data if a.size else None for a in arrs])
        self._check(lib.mpm_init_particles_batch(self._h, counts, ptrs))
        self.counts = list(counts)
        self.n = sum(self.counts)

    def init_scene_sdf(self, scene: int, triangles):
        t = np.ascontiguousarray(triangles, dtype=np.float32).reshape(-1)
        self._check(lib.mpm_scene_init_sdf(self._h, scene, _ptr(t) if t.size else None, t.size // 9))

    def scene_buffer(self, scene: int) -> np.ndarray:
        out = np.empty((PARTICLE_PLANES, self.counts[scene]), np.float32)
        self._check(lib.mpm_scene_get_state(self._h, scene, _ptr(out)))
        return out

    def scene_positions(self, scene: int) -> np.ndarray:
        out = np.empty((self.counts[scene], 3), np.float32)
        self._check(lib.mpm_scene_get_positions(self._h, scene, _ptr(out)))
        return out

    def scene_grid(self, scene: int) -> np.ndarray:
        out = np.empty((GRID_PLANES, self.cfgs[scene].grid_number), np.float32)
        self._check(lib.mpm_scene_get_grid(self._h, scene, _ptr(out)))
        return out

    def scene_sdf(self, scene: int) -> np.ndarray:
        out = np.empty(self.cfgs[scene].grid_number, np.float32)
        self._check(lib.mpm_scene_get_sdf(self._h, scene, _ptr(out)))
        return out

    def scene_sort(self, scene: int):
        keys = np.empty(self.counts[scene], np.int32)
        perm = np.empty(self.counts[scene], np.int32)
        self._check(lib.mpm_scene_get_sort(self._h, scene, _ptr(keys), _ptr(perm)))
        return keys, perm


class Corrector:
    """Training data, parameters and Adam state of the learned corrector."""

    def __init__(self, capacity: int, device: int = 0):
        h = ctypes.c_void_p()
        st = lib.mpm_corrector_create(int(device), int(capacity), ctypes.byref(h))
        if st != 0:
            raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))
        self._h = h
        self.capacity = int(capacity)

    def _check(self, st: int):
        if st != 0:
            raise MpmError(st, lib.mpm_corrector_last_error(self._h).decode(errors="replace"))

    def close(self):
        if getattr(self, "_h", None):
            lib.mpm_corrector_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def size(self) -> int:
        return int(lib.mpm_corrector_size(self._h))

    def clear(self):
        self._check(lib.mpm_corrector_clear(self._h))

    def collect(self, engine: Engine, samples: int, seed: int):
        """The collection probe on the engine's current state (the engine advances RATIO substeps)."""
        st = lib.mpm_corrector_collect(self._h, engine._h, int(samples), int(seed))
        if st != 0:
            raise MpmError(st, lib.mpm_last_error(engine._h).decode(errors="replace"))

    def add_data(self, features: np.ndarray, targets: np.ndarray):
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, CORRECTOR_FEATURES)
        t = np.ascontiguousarray(targets, dtype=np.float32).reshape(-1, CORRECTOR_OUTPUTS)
        if len(f) != len(t):
            raise ValueError("features and targets differ in length")
        self._check(lib.mpm_corrector_add_data(self._h, len(f), _ptr(f), _ptr(t)))

    def get_data(self, first: int = 0, count: int | None = None):
        count = self.size - first if count is None else count
        f = np.empty((count, CORRECTOR_FEATURES), np.float32)
        t = np.empty((count, CORRECTOR_OUTPUTS), np.float32)
        self._check(lib.mpm_corrector_get_data(self._h, int(first), int(count), _ptr(f), _ptr(t)))
        return f, t

    def init(self, seed: int = 0):
        self._check(lib.mpm_corrector_init(self._h, int(seed)))

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> float:
        loss = ctypes.c_float(0.0)
        self._check(lib.mpm_corrector_train(self._h, int(steps), int(batch), float(lr), int(seed),
                                            ctypes.byref(loss)))
        return float(loss.value)

    def gradient(self, idx: np.ndarray):
        i = np.ascontiguousarray(idx, dtype=np.int64)
        g = np.empty(CORRECTOR_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(lib.mpm_corrector_gradient(self._h, len(i), _ptr(i), _ptr(g), _ptr(loss)))
        return g, float(loss[0])

    def set_train_kernel(self, kind: str):
        """'tcgen05' (every GEMM on the 5th-generation tensor cores, the default) or 'fp32'."""
        kinds = {"tcgen05": 0, "fp32": 1}
        if kind not in kinds:
            raise ValueError(f"unknown training kernel {kind!r}")
        self._check(lib.mpm_corrector_set_train_kernel(self._h, kinds[kind]))

    def get_params(self) -> np.ndarray:
        w = np.empty(CORRECTOR_PARAMS, np.float32)
        self._check(lib.mpm_corrector_get_params(self._h, _ptr(w)))
        return w

    def set_params(self, params: np.ndarray):
        w = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        if w.size != CORRECTOR_PARAMS:
            raise ValueError(f"expected {CORRECTOR_PARAMS} parameters")
        self._check(lib.mpm_corrector_set_params(self._h, _ptr(w)))

    def forward(self, features: np.ndarray, tcgen05: bool = False) -> np.ndarray:
        """The tensor-core inference of the learned G2P (mma.sync, or tcgen05 with TMEM)."""
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, CORRECTOR_FEATURES)
        out = np.empty((len(f), CORRECTOR_OUTPUTS), np.float32)
        fn = lib.mpm_corrector_forward_tc if tcgen05 else lib.mpm_corrector_forward
        self._check(fn(self._h, len(f), _ptr(f), _ptr(out)))
        return out


# -- scene construction (Simulation::Simulation's WATER= / OBJECT= path) ----------
def _scene_check(st: int):
    if st != 0:
        raise MpmError(st, lib.mpm_scene_last_error().decode(errors="replace"))


class Mesh:
    """An OBJ model: vertices and triangles (ObjLoader::loadObj + extractTriangles)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path: str) -> "Mesh":
        h = ctypes.c_void_p()
        _scene_check(lib.mpm_mesh_load_obj(path.encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_text(cls, text: str) -> "Mesh":
        h = ctypes.c_void_p()
        _scene_check(lib.mpm_mesh_from_obj_text(text.encode(), ctypes.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.mpm_mesh_free(self._h)
            self._h = None

    def arrays(self):
        """(vertices (nv, 3), faces (nt, 3) int32, triangles (nt, 9))."""
        nv, nt = lib.mpm_mesh_num_vertices(self._h), lib.mpm_mesh_num_triangles(self._h)
        v = np.empty((nv, 3), np.float32)
        f = np.empty((nt, 3), np.int32)
        t = np.empty((nt, 9), np.float32)
        _scene_check(lib.mpm_mesh_get(self._h, _ptr(v), _ptr(f), _ptr(t)))
        return v, f, t

    def voxelize(self, resolution: float = 100.0, device: int = 0) -> np.ndarray:
        """VoxelEngine::voxelize: (n, 3) voxel centres, z-major order."""
        h = ctypes.c_void_p()
        _scene_check(lib.mpm_voxelize(self._h, float(resolution), int(device), ctypes.byref(h)))
        try:
            return _points_array(h)
        finally:
            lib.mpm_points_free(h)


def _points_array(h) -> np.ndarray:
    n = lib.mpm_points_count(h)
    out = np.empty((n, 3), np.float32)
    _scene_check(lib.mpm_points_get(h, _ptr(out) if n else None))
    return out


def normalize_points(points: np.ndarray, normalize_size: float, scale: float, displacement, lattice_step: int,
                     device: int = 0) -> np.ndarray:
    """VoxelEngine::normalize(VoxelData&): centre, scale, displace, snap + 5^3 dilation."""
    p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(displacement, np.float32).reshape(3)
    h = ctypes.c_void_p()
    _scene_check(lib.mpm_points_create(_ptr(p) if len(p) else None, len(p), ctypes.byref(h)))
    try:
        _scene_check(lib.mpm_points_normalize(h, float(normalize_size), float(scale), _ptr(d), int(lattice_step),
                                              int(device)))
        return _points_array(h)
    finally:
        lib.mpm_points_free(h)


def normalize_triangles(tris: np.ndarray, normalize_size: float, scale: float, displacement) -> np.ndarray:
    """VoxelEngine::normalize(std::vector<Triangle>&): (t, 9) -> the kept, transformed triangles."""
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9).copy()
    d = np.ascontiguousarray(displacement, np.float32).reshape(3)
    n = ctypes.c_int64(len(t))
    _scene_check(lib.mpm_triangles_normalize(_ptr(t) if len(t) else None, ctypes.byref(n), float(normalize_size),
                                             float(scale), _ptr(d)))
    return t[:n.value]


def build_scene(config_text: str, base_dir: str = "", device: int = 0):
    """Simulation::Simulation's scene part: (Config, state (26, n), triangles (t, 9), log)."""
    cfg = parse_config_string(config_text)
    h = ctypes.c_void_p()
    _scene_check(lib.mpm_scene_build(config_text.encode(), base_dir.encode(), int(device), ctypes.byref(h)))
    try:
        n = lib.mpm_scene_data_num_particles(h)
        t = lib.mpm_scene_data_num_triangles(h)
        st = np.empty((PARTICLE_PLANES, n), np.float32)
        tris = np.empty((t, 9), np.float32)
        _scene_check(lib.mpm_scene_data_state(h, _ptr(st) if n else None))
        _scene_check(lib.mpm_scene_data_triangles(h, _ptr(tris) if t else None))
        log = lib.mpm_scene_data_log(h).decode(errors="replace")
    finally:
        lib.mpm_scene_data_free(h)
    return cfg, st, tris, log


def checkpoint_info(path: str) -> dict:
    c = _Config()
    n, sub = ctypes.c_int64(0), ctypes.c_int64(0)
    note = ctypes.create_string_buffer(1 << 16)
    st = lib.mpm_checkpoint_info(path.encode(), ctypes.byref(c), ctypes.byref(n), ctypes.byref(sub), note, len(note))
    if st != 0:
        raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))
    cfg = Config(c.size_x, c.size_y, c.size_z, c.padding, c.gravity, c.dt, c.gamma, c.compression,
                 c.resolution, c.substeps, c.sdf_resolution)
    return {"config": cfg, "n": n.value, "substeps": sub.value, "note": note.value.decode(errors="replace")}


# -- headless screen-space fluid rendering ----------------------------------------
class _RenderParams(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("grid", ctypes.c_int32 * 3),
                ("fov_y_degrees", ctypes.c_float), ("near_clip", ctypes.c_float), ("far_clip", ctypes.c_float),
                ("zoom_distance", ctypes.c_float), ("rotation", ctypes.c_float),
                ("rotation_vertical", ctypes.c_float), ("radius", ctypes.c_float), ("filter_size", ctypes.c_float),
                ("depth_falloff", ctypes.c_float), ("light_dir", ctypes.c_float * 3),
                ("clear_color", ctypes.c_float * 3)]


class Renderer:
    """The reference's SSF passes (depth splat, bilateral blur, composite) on the GPU."""

    def __init__(self, grid, width: int = 1920, height: int = 1600, device: int = 0, **overrides):
        p = _RenderParams()
        lib.mpm_render_params_default(ctypes.byref(p), int(grid[0]), int(grid[1]), int(grid[2]))
        p.width, p.height = int(width), int(height)
        for k, v in overrides.items():
            if k in ("light_dir", "clear_color"):
                getattr(p, k)[:] = [float(x) for x in v]
            else:
                setattr(p, k, v)
        h = ctypes.c_void_p()
        st = lib.mpm_renderer_create(ctypes.byref(p), int(device), ctypes.byref(h))
        if st != 0:
            raise MpmError(st, lib.mpm_global_last_error().decode(errors="replace"))
        self._h, self.width, self.height = h, p.width, p.height

    def _check(self, st):
        if st != 0:
            raise MpmError(st, lib.mpm_renderer_last_error(self._h).decode(errors="replace"))

    def close(self):
        if getattr(self, "_h", None):
            lib.mpm_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_background(self, rgb8: np.ndarray):
        a = np.ascontiguousarray(rgb8, np.uint8).reshape(self.height, self.width, 3)
        self._check(lib.mpm_renderer_set_background(self._h, _ptr(a)))

    def set_obstacles(self, triangles: np.ndarray, rgb=None):
        """The obstacle pass (dot.vert/dot.frag): (t, 9) triangles in grid coordinates."""
        t = np.ascontiguousarray(triangles, np.float32).reshape(-1, 9)
        c = None if rgb is None else np.ascontiguousarray(rgb, np.float32).reshape(3)
        self._check(lib.mpm_renderer_set_obstacles(self._h, _ptr(t) if len(t) else None, len(t),
                                                   _ptr(c) if c is not None else None))

    def background(self):
        """(background RGB8 (h, w, 3), obstacle window depth (h, w)), row 0 at the bottom."""
        b = np.empty((self.height, self.width, 3), np.uint8)
        d = np.empty((self.height, self.width), np.float32)
        self._check(lib.mpm_renderer_get_background(self._h, _ptr(b), _ptr(d)))
        return b, d

    def render_device(self, xyz_ptr: int, n: int, stream: int = 0):
        self._check(lib.mpm_render_points(self._h, ctypes.c_void_p(xyz_ptr), int(n), ctypes.c_void_p(stream)))

    def render_engine(self, engine: Engine):
        self._check(lib.mpm_render_frame(self._h, engine._h))

    def depth(self, which: int = 2) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        self._check(lib.mpm_renderer_get_depth(self._h, int(which), _ptr(out)))
        return out

    def image(self):
        """(float RGB (h, w, 3), 8-bit RGB), row 0 at the bottom."""
        f = np.empty((self.height, self.width, 3), np.float32)
        b = np.empty((self.height, self.width, 3), np.uint8)
        self._check(lib.mpm_renderer_get_image(self._h, _ptr(f), _ptr(b)))
        return f, b
