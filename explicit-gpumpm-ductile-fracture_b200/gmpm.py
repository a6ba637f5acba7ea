"""ctypes binding of the gmpm C-ABI (include/gmpm.h).

Loads libgmpm.so from this directory and raises if it is missing: there is no
CPU fallback.  Struct layouts mirror include/gmpm.h field for field.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libgmpm.so"

MAX_SLAB_BCS = 4
MAX_SPHERE_BCS = 2
MAX_MATERIALS = 8

# gmpm_status
OK, INVALID_ARG, OOM, TABLE_OVERFLOW, NONFINITE, OUT_OF_DOMAIN, CUDA_ERROR, NOT_SUPPORTED, NO_DEVICE, IO_ERROR = range(10)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "TABLE_OVERFLOW", 4: "NONFINITE", 5: "OUT_OF_DOMAIN",
                6: "CUDA_ERROR", 7: "NOT_SUPPORTED", 8: "NO_DEVICE", 9: "IO_ERROR"}

FLAG_OUT_OF_DOMAIN, FLAG_NONFINITE, FLAG_SVD_NOCONVERGE, FLAG_TABLE_OVERFLOW, FLAG_COPY_TIMEOUT = 1, 2, 4, 8, 16

PRECISION_FP32, PRECISION_FP64, PRECISION_FP32_FP64SVD = 0, 1, 2
HARDENING_EXPONENTIAL, HARDENING_LINEAR = 0, 1
PHASE_FIELD_OFF, PHASE_FIELD_EXPLICIT, PHASE_FIELD_IMPLICIT = 0, 1, 2

FIELD = dict(position=0, velocity=1, F=2, B=3, damage=4, alpha=5, psi_max=6, stress=7, volume=8, FP=9,
             pf_flux=10, mass=11, id=12)
FIELD_COMPONENTS = dict(position=3, velocity=3, F=9, B=9, damage=1, alpha=1, psi_max=1, stress=6, volume=1, FP=1,
                        pf_flux=3, mass=1, id=1)
ENERGY_VON_MISES_FRACTURE, ENERGY_FIXED_COROTATED, ENERGY_NEO_HOOKEAN_FRACTURE = 0, 1, 2
DTYPE_F64, DTYPE_F32, DTYPE_I32 = 0, 1, 2
ORDER_INTERNAL, ORDER_ORIGINAL = 0, 1
BIN = dict(counts=0, perm=1, keys=2, block_keys=3, block_start=4, cell_start=5, grid_keys=6, adj=7)
NOALLOC_MAX_PARTICLES = 1048576
NOALLOC_MAX_RES = 128


class Material(C.Structure):
    _fields_ = [("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double), ("density", C.c_double),
                ("yield_stress", C.c_double), ("hardening_law", C.c_int32), ("energy_model", C.c_int32),
                ("hardening", C.c_double), ("alpha_cap", C.c_double), ("dlambda_cap", C.c_double),
                ("strain_cap", C.c_double), ("psi_cap", C.c_double), ("fracture_energy", C.c_double),
                ("softening_onset", C.c_double), ("residual_fracture", C.c_double), ("theta", C.c_double),
                ("length_scale", C.c_double), ("mobility", C.c_double)]


class SlabBC(C.Structure):
    _fields_ = [("axis", C.c_int32), ("_pad0", C.c_int32), ("lo", C.c_double), ("hi", C.c_double),
                ("velocity", C.c_double * 3)]


class SphereBC(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("radius", C.c_double), ("velocity", C.c_double * 3)]


class SceneDesc(C.Structure):
    _fields_ = [("dx", C.c_double), ("grid_res", C.c_int32 * 3), ("_pad0", C.c_int32), ("dt", C.c_double),
                ("gravity", C.c_double * 3), ("particle_volume", C.c_double), ("n_materials", C.c_int32),
                ("_pad1", C.c_int32), ("materials", Material * MAX_MATERIALS), ("wall_bc", C.c_int32),
                ("wall_layers", C.c_int32), ("n_slab_bcs", C.c_int32), ("n_sphere_bcs", C.c_int32),
                ("slabs", SlabBC * MAX_SLAB_BCS), ("spheres", SphereBC * MAX_SPHERE_BCS),
                ("precision", C.c_int32), ("phase_field", C.c_int32), ("deterministic", C.c_int32),
                ("block_capacity", C.c_int32), ("svd_fallback_ratio", C.c_double),
                ("adaptive_dt", C.c_int32), ("_pad2", C.c_int32), ("cfl_number", C.c_double),
                ("pcg_max_iterations", C.c_int32), ("pcg_max_combine", C.c_int32), ("pcg_tolerance", C.c_double)]


class ParticleInit(C.Structure):
    _fields_ = [("count", C.c_int64), ("positions", C.POINTER(C.c_double)), ("velocities", C.POINTER(C.c_double)),
                ("masses", C.POINTER(C.c_double)), ("material_ids", C.POINTER(C.c_int32))]


class Diag(C.Structure):
    _fields_ = [("particle_mass", C.c_double), ("particle_momentum", C.c_double * 3), ("grid_mass", C.c_double),
                ("grid_momentum", C.c_double * 3), ("kinetic_energy", C.c_double), ("max_speed", C.c_double),
                ("min_damage", C.c_double), ("time", C.c_double), ("substeps", C.c_int64),
                ("n_particles", C.c_int64), ("n_blocks", C.c_int32), ("n_grid_blocks", C.c_int32),
                ("flags", C.c_uint32), ("_pad0", C.c_int32), ("kernel_launches", C.c_int64), ("dt", C.c_double),
                ("pcg_iterations", C.c_int32), ("_pad1", C.c_int32)]

    def as_dict(self) -> dict:
        return dict(particle_mass=self.particle_mass, particle_momentum=list(self.particle_momentum),
                    grid_mass=self.grid_mass, grid_momentum=list(self.grid_momentum),
                    kinetic_energy=self.kinetic_energy, max_speed=self.max_speed, min_damage=self.min_damage,
                    time=self.time, substeps=self.substeps, n_particles=self.n_particles, n_blocks=self.n_blocks,
                    n_grid_blocks=self.n_grid_blocks, flags=self.flags, kernel_launches=self.kernel_launches,
                    dt=self.dt, pcg_iterations=self.pcg_iterations)


class StageTimes(C.Structure):
    _fields_ = [("bin_ms", C.c_double), ("p2g_ms", C.c_double), ("grid_ms", C.c_double), ("g2p_ms", C.c_double),
                ("total_ms", C.c_double), ("substeps", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Geometry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("cells", C.c_int32 * 3), ("ppc", C.c_int32), ("n_plates", C.c_int32),
                ("gap_cells", C.c_int32), ("notch_width", C.c_int32), ("notch_depth", C.c_int32),
                ("_pad0", C.c_int32), ("dx", C.c_double), ("origin", C.c_double * 3), ("seed", C.c_uint64)]


class BatchOptions(C.Structure):
    _fields_ = [("autotune", C.c_int32), ("trial_substeps", C.c_int32), ("streams", C.c_int32),
                ("sm_share", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("n_scenes", C.c_int32), ("streams", C.c_int32), ("tuned", C.c_int32), ("n_candidates", C.c_int32),
                ("graph_nodes", C.c_int64), ("captures", C.c_int64), ("substeps", C.c_int64),
                ("best_ms_per_substep", C.c_double), ("sm_share_small", C.c_int32),
                ("sm_share_medium", C.c_int32), ("sm_share_large", C.c_int32), ("_pad0", C.c_int32),
                ("capture_seconds", C.c_double), ("kernel_nodes", C.c_int64), ("table_scenes", C.c_int32),
                ("_pad1", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("_")}


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_live", C.c_int32), ("autotune", C.c_int32)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("n_particles", C.c_int64),
                ("substeps_done", C.c_int64), ("horizon", C.c_int64), ("submit_time", C.c_double),
                ("admit_time", C.c_double), ("finish_time", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "admitted", "completed", "failed", "live", "queued",
                                          "substeps", "particle_substeps", "batches", "device_bytes_in_use",
                                          "capture_microseconds", "admit_microseconds", "retire_microseconds",
                                          "launch_microseconds")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


REQUEST_QUEUED, REQUEST_RUNNING, REQUEST_DONE, REQUEST_FAILED = 0, 1, 2, 3


# Exported entry points and their argument types, exactly as declared in include/gmpm.h.
SIGNATURES = {
    "gmpm_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "gmpm_context_destroy": (C.c_int, [C.c_void_p]),
    "gmpm_scene_desc_reference_defaults": (C.c_int, [C.POINTER(SceneDesc), C.c_double, C.c_int, C.c_int, C.c_int]),
    "gmpm_scene_create": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(ParticleInit),
                                    C.POINTER(C.c_void_p)]),
    "gmpm_scene_destroy": (C.c_int, [C.c_void_p]),
    "gmpm_substep": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "gmpm_substep_timed": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gmpm_set_dt": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "gmpm_set_velocity_conditions": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "gmpm_rebin": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gmpm_scene_sync": (C.c_int, [C.c_void_p]),
    "gmpm_read_particles": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    "gmpm_read_binning": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "gmpm_read_particles_async": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t,
                                            C.c_void_p]),
    "gmpm_read_wait": (C.c_int, [C.c_void_p]),
    "gmpm_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(Diag)]),
    "gmpm_status_string": (C.c_char_p, [C.c_int]),
    "gmpm_bin_positions_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_int, C.c_int, C.c_int,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gmpm_generate_particles": (C.c_int, [C.POINTER(Geometry), C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                          C.POINTER(C.c_int32), C.c_int64]),
    "gmpm_sample_obj": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int64]),
    "gmpm_sample_cube": (C.c_int, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int64]),
    "gmpm_sample_sdf": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_double, C.c_uint32,
                                  C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int64]),
    "gmpm_scene_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "gmpm_scene_load": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "gmpm_batch_options_defaults": (None, [C.POINTER(BatchOptions)]),
    "gmpm_batch_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.POINTER(BatchOptions),
                                    C.POINTER(C.c_void_p)]),
    "gmpm_batch_substep": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "gmpm_batch_get_info": (C.c_int, [C.c_void_p, C.POINTER(BatchInfo)]),
    "gmpm_batch_destroy": (C.c_int, [C.c_void_p]),
    "gmpm_server_options_defaults": (None, [C.POINTER(ServerOptions)]),
    "gmpm_server_create": (C.c_int, [C.c_void_p, C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "gmpm_server_submit": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(ParticleInit), C.c_int64,
                                     C.POINTER(C.c_int64)]),
    "gmpm_server_step": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "gmpm_server_poll": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(RequestStatus)]),
    "gmpm_server_read": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_size_t]),
    "gmpm_server_release": (C.c_int, [C.c_void_p, C.c_int64]),
    "gmpm_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "gmpm_server_destroy": (C.c_int, [C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libgmpm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing; build it with build.py (no CPU fallback exists)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class GmpmError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}")
        self.status = status


def check(status: int, what: str) -> None:
    if status != OK:
        raise GmpmError(status, what)


def _dptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def reference_defaults(dx: float, res) -> SceneDesc:
    d = SceneDesc()
    check(lib().gmpm_scene_desc_reference_defaults(C.byref(d), dx, int(res[0]), int(res[1]), int(res[2])),
          "reference_defaults")
    return d


def generate_particles(geom: Geometry) -> tuple[np.ndarray, np.ndarray]:
    L = lib()
    n = C.c_int64(0)
    check(L.gmpm_generate_particles(C.byref(geom), C.byref(n), None, None, 0), "generate_particles(count)")
    pos = np.empty((n.value, 3), dtype=np.float64)
    mat = np.empty(n.value, dtype=np.int32)
    check(L.gmpm_generate_particles(C.byref(geom), C.byref(n), _dptr(pos), _iptr(mat), n.value),
          "generate_particles")
    return pos, mat


def _sampled(call, what: str) -> np.ndarray:
    n = C.c_int64(0)
    check(call(C.byref(n), None, 0), f"{what}(count)")
    pos = np.empty((n.value, 3), dtype=np.float64)
    check(call(C.byref(n), _dptr(pos), n.value), what)
    return pos


def sample_obj(path) -> np.ndarray:
    """The reference's Sample::readObj: one particle per OBJ vertex record, y shifted by -0.2f."""
    p = str(path).encode()
    return _sampled(lambda n, out, cap: lib().gmpm_sample_obj(p, n, out, cap), "sample_obj")


def sample_cube(n_grid: int) -> np.ndarray:
    """The reference's Sample::Initialize_Data_cube on an n_grid^3 grid (27 particles per cell)."""
    return _sampled(lambda n, out, cap: lib().gmpm_sample_cube(int(n_grid), n, out, cap), "sample_cube")


def sample_sdf(path, center, res, dx: float, seed: int = 1) -> np.ndarray:
    """The reference's Sample::Initial_data: rejection samples of an SDF level set placed in the
    res[] grid cells around center[].  Draws from the C library's rand() after srand(seed), as the
    reference does (seed 1 reproduces the reference's run)."""
    p = str(path).encode()
    c = (C.c_uint32 * 3)(*[int(v) for v in center])
    r = (C.c_uint32 * 3)(*[int(v) for v in res])
    return _sampled(lambda n, out, cap: lib().gmpm_sample_sdf(p, c, r, float(dx), int(seed), n, out, cap),
                    "sample_sdf")


class Context:
    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        check(lib().gmpm_context_create(device, C.byref(self.h)), "context_create")

    def close(self) -> None:
        if self.h:
            lib().gmpm_context_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """One simulation scene on the device (gmpm_scene)."""

    def __init__(self, ctx: Context, desc: SceneDesc, positions: np.ndarray, masses: np.ndarray,
                 velocities: np.ndarray | None = None, material_ids: np.ndarray | None = None):
        self.ctx = ctx
        self.desc = desc
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1, 3)
        mid = None if material_ids is None else np.ascontiguousarray(material_ids, dtype=np.int32).reshape(-1)
        init = ParticleInit(len(pos), _dptr(pos), _dptr(v), _dptr(m), _iptr(mid))
        self.n = len(pos)
        self.h = C.c_void_p()
        check(lib().gmpm_scene_create(ctx.h, C.byref(desc), C.byref(init), C.byref(self.h)), "scene_create")

    def close(self) -> None:
        if self.h:
            lib().gmpm_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def substep(self, n: int = 1, stream: int | None = None) -> None:
        check(lib().gmpm_substep(self.h, int(n), C.c_void_p(stream) if stream else None), "substep")

    def save(self, path) -> None:
        check(lib().gmpm_scene_save(self.h, str(path).encode()), "scene_save")

    @classmethod
    def load(cls, ctx: Context, path) -> "Scene":
        """A scene restored from a checkpoint written by save()."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.h = C.c_void_p()
        check(lib().gmpm_scene_load(ctx.h, str(path).encode(), C.byref(self.h)), "scene_load")
        d = Diag()
        check(lib().gmpm_diagnostics(self.h, C.byref(d)), "diagnostics")
        self.n = int(d.n_particles)
        self.desc = None
        return self

    def substep_timed(self, n: int = 1, stream: int | None = None) -> dict:
        t = StageTimes()
        check(lib().gmpm_substep_timed(self.h, int(n), C.c_void_p(stream) if stream else None, C.byref(t)),
              "substep_timed")
        return t.as_dict()

    def set_dt(self, dt: float, stream: int | None = None) -> None:
        check(lib().gmpm_set_dt(self.h, float(dt), C.c_void_p(stream) if stream else None), "set_dt")

    def set_velocity_conditions(self, slabs=(), spheres=(), stream: int | None = None) -> None:
        """Replace the velocity conditions (sequences of SlabBC / SphereBC)."""
        arr_s = (SlabBC * max(1, len(slabs)))(*slabs)
        arr_p = (SphereBC * max(1, len(spheres)))(*spheres)
        self.set_velocity_conditions_raw(C.addressof(arr_s), len(slabs), C.addressof(arr_p), len(spheres), stream)

    def set_velocity_conditions_raw(self, slab_ptr: int, n_slabs: int, sphere_ptr: int, n_spheres: int,
                                    stream: int | None = None) -> None:
        """Same, from host pointers to packed gmpm_slab_bc / gmpm_sphere_bc arrays (e.g. pinned)."""
        check(lib().gmpm_set_velocity_conditions(self.h, C.c_void_p(slab_ptr), int(n_slabs), C.c_void_p(sphere_ptr),
                                                 int(n_spheres), C.c_void_p(stream) if stream else None),
              "set_velocity_conditions")

    def rebin(self, stream: int | None = None) -> None:
        check(lib().gmpm_rebin(self.h, C.c_void_p(stream) if stream else None), "rebin")

    def sync(self) -> int:
        return lib().gmpm_scene_sync(self.h)

    def read(self, field: str, order: int = ORDER_ORIGINAL, dtype: int = DTYPE_F64) -> np.ndarray:
        nc = FIELD_COMPONENTS[field]
        npdt = {DTYPE_F64: np.float64, DTYPE_F32: np.float32, DTYPE_I32: np.int32}[dtype]
        out = np.empty((self.n, nc), dtype=npdt)
        check(lib().gmpm_read_particles(self.h, FIELD[field], dtype, order, out.ctypes.data_as(C.c_void_p),
                                        out.nbytes, None), f"read_particles({field})")
        return out if nc > 1 else out.reshape(-1)

    def read_into(self, field: str, out_ptr: int, nbytes: int, order: int = ORDER_INTERNAL,
                  dtype: int = DTYPE_F32, stream: int | None = None) -> None:
        check(lib().gmpm_read_particles(self.h, FIELD[field], dtype, order, C.c_void_p(out_ptr), nbytes,
                                        C.c_void_p(stream) if stream else None), f"read_particles({field})")

    def read_into_async(self, field: str, out_ptr: int, nbytes: int, order: int = ORDER_INTERNAL,
                        dtype: int = DTYPE_F32, stream: int | None = None) -> None:
        """Overlapped read into (pinned) host memory; complete after read_wait()."""
        check(lib().gmpm_read_particles_async(self.h, FIELD[field], dtype, order, C.c_void_p(out_ptr), nbytes,
                                              C.c_void_p(stream) if stream else None), f"read_particles_async({field})")

    def read_wait(self) -> None:
        check(lib().gmpm_read_wait(self.h), "read_wait")

    def binning(self, array: str) -> np.ndarray:
        counts = np.zeros(4, dtype=np.int64)
        check(lib().gmpm_read_binning(self.h, BIN["counts"], counts.ctypes.data_as(C.c_void_p), counts.nbytes),
              "read_binning(counts)")
        if array == "counts":
            return counts
        n, nb, ng = int(counts[0]), int(counts[1]), int(counts[2])
        size = dict(perm=n, keys=n, block_keys=nb, block_start=nb + 1, cell_start=nb * 64 + 1, grid_keys=ng,
                    adj=nb * 8)[array]
        dt = np.uint32 if array in ("keys", "block_keys", "grid_keys") else np.int32
        out = np.empty(size, dtype=dt)
        check(lib().gmpm_read_binning(self.h, BIN[array], out.ctypes.data_as(C.c_void_p), out.nbytes),
              f"read_binning({array})")
        return out

    def diagnostics(self) -> dict:
        d = Diag()
        check(lib().gmpm_diagnostics(self.h, C.byref(d)), "diagnostics")
        return d.as_dict()


class Batch:
    """Independent scenes advanced together by one CUDA graph per substep (gmpm_batch)."""

    def __init__(self, ctx: Context, scenes, autotune: bool = True, trial_substeps: int = 2, streams: int = 0,
                 sm_share: int = 0):
        self.ctx = ctx
        self.scenes = list(scenes)  # keeps the scenes alive while the batch exists
        opt = BatchOptions()
        lib().gmpm_batch_options_defaults(C.byref(opt))
        opt.autotune, opt.trial_substeps, opt.streams, opt.sm_share = int(autotune), trial_substeps, streams, sm_share
        hs = (C.c_void_p * len(self.scenes))(*[sc.h for sc in self.scenes])
        self.h = C.c_void_p()
        check(lib().gmpm_batch_create(ctx.h, hs, len(self.scenes), C.byref(opt), C.byref(self.h)), "batch_create")

    def substep(self, n: int = 1, stream: int | None = None) -> None:
        check(lib().gmpm_batch_substep(self.h, int(n), C.c_void_p(stream) if stream else None), "batch_substep")

    def info(self) -> dict:
        i = BatchInfo()
        check(lib().gmpm_batch_get_info(self.h, C.byref(i)), "batch_get_info")
        return i.as_dict()

    def close(self) -> None:
        if self.h:
            lib().gmpm_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching serving loop (gmpm_server)."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int | None = None, max_live: int | None = None,
                 autotune: bool = True):
        self.ctx = ctx
        opt = ServerOptions()
        lib().gmpm_server_options_defaults(C.byref(opt))
        if hbm_budget_bytes is not None:
            opt.hbm_budget_bytes = int(hbm_budget_bytes)
        if max_live is not None:
            opt.max_live = int(max_live)
        opt.autotune = int(autotune)
        self.h = C.c_void_p()
        check(lib().gmpm_server_create(ctx.h, C.byref(opt), C.byref(self.h)), "server_create")

    def submit(self, desc: SceneDesc, positions: np.ndarray, masses: np.ndarray, velocities=None,
               material_ids=None, horizon: int = 1) -> int:
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1, 3)
        mid = None if material_ids is None else np.ascontiguousarray(material_ids, dtype=np.int32).reshape(-1)
        init = ParticleInit(len(pos), _dptr(pos), _dptr(v), _dptr(m), _iptr(mid))
        rid = C.c_int64()
        check(lib().gmpm_server_submit(self.h, C.byref(desc), C.byref(init), int(horizon), C.byref(rid)),
              "server_submit")
        return rid.value

    def submit_spec(self, spec, horizon: int) -> int:
        return self.submit(spec.desc, spec.positions, spec.masses, spec.velocities, spec.material_ids, horizon)

    def step(self, n: int = 1, stream: int | None = None) -> None:
        check(lib().gmpm_server_step(self.h, int(n), C.c_void_p(stream) if stream else None), "server_step")

    def poll(self, rid: int) -> dict:
        st = RequestStatus()
        check(lib().gmpm_server_poll(self.h, int(rid), C.byref(st)), "server_poll")
        return st.as_dict()

    def read(self, rid: int, field: str) -> np.ndarray:
        st = self.poll(rid)
        nc = FIELD_COMPONENTS[field]
        out = np.empty((st["n_particles"], nc), dtype=np.float32)
        check(lib().gmpm_server_read(self.h, int(rid), FIELD[field], out.ctypes.data_as(C.c_void_p), out.nbytes),
              f"server_read({field})")
        return out if nc > 1 else out.reshape(-1)

    def release(self, rid: int) -> None:
        check(lib().gmpm_server_release(self.h, int(rid)), "server_release")

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().gmpm_server_get_stats(self.h, C.byref(st)), "server_get_stats")
        return st.as_dict()

    def close(self) -> None:
        if self.h:
            lib().gmpm_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
