"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

ORACLE — test infrastructure only.  Loaded by tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline / reference arm; never by the product.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_KAT = HERE / "_ref" / "ref_kat"


def build(force: bool = False) -> Path:
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(
            p.stat().st_mtime for p in [HERE / "gmpm_oracle.cpp", HERE / "gmpm_oracle.h", HERE.parent / "include" / "gmpm.h"]):
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


_lib = None


def lib(desc_type=None, diag_type=None, material_type=None) -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
        L.orc_masks.argtypes = [C.POINTER(C.c_uint64)]
        L.orc_bit_spread.restype = C.c_uint64
        L.orc_bit_spread.argtypes = [C.c_uint64, C.c_int64]
        L.orc_linear_offset.restype = C.c_uint64
        L.orc_linear_offset.argtypes = [C.c_int, C.c_int, C.c_int]
        L.orc_packed_add.restype = C.c_uint64
        L.orc_packed_add.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_bit_pack.restype = C.c_int64
        L.orc_bit_pack.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_svd3.argtypes = [dp, dp, dp, dp]
        L.orc_lame.argtypes = [C.c_double, C.c_double, dp, dp, dp]
        L.orc_von_mises.argtypes = [vp, C.c_double, dp, dp]
        L.orc_constitutive.argtypes = [vp, C.c_double, C.c_double, dp, dp]
        L.orc_base_node.restype = C.c_int
        L.orc_base_node.argtypes = [C.c_double, ip, dp, ip]
        L.orc_grid_node.argtypes = [vp, C.c_double, ip, dp, dp]
        L.orc_scene_desc_reference_defaults.restype = C.c_int
        L.orc_scene_desc_reference_defaults.argtypes = [vp, C.c_double, C.c_int, C.c_int, C.c_int]
        L.orc_generate_particles.restype = C.c_int
        L.orc_generate_particles.argtypes = [vp, C.POINTER(C.c_int64), dp, ip, C.c_int64]
        L.orc_scene_create.restype = vp
        L.orc_scene_create.argtypes = [vp, C.c_int64, dp, dp, dp, ip]
        L.orc_scene_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        L.orc_substep.restype = C.c_uint32
        L.orc_substep.argtypes = [vp, C.c_int]
        L.orc_rebin.restype = C.c_uint32
        L.orc_rebin.argtypes = [vp]
        for f in ("orc_num_particles", "orc_num_blocks", "orc_num_grid_blocks"):
            getattr(L, f).restype = C.c_int64
            getattr(L, f).argtypes = [vp]
        L.orc_get_field.argtypes = [vp, C.c_int, dp]
        L.orc_get_binning.argtypes = [vp, C.c_int, vp]
        L.orc_diagnostics.argtypes = [vp, vp]
        _lib = L
    return _lib


def _dptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


FIELD_COMPONENTS = {0: 3, 1: 3, 2: 9, 3: 9, 4: 1, 5: 1, 6: 1, 7: 6, 8: 1, 9: 1, 10: 3, 11: 1, 12: 1}


class OracleScene:
    """FP64 CPU restatement of one scene; arrays in the oracle's sorted order."""

    def __init__(self, desc, positions, masses, velocities=None, material_ids=None):
        L = lib()
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1, 3)
        mid = None if material_ids is None else np.ascontiguousarray(material_ids, dtype=np.int32).reshape(-1)
        self.n = len(pos)
        self.h = L.orc_scene_create(C.byref(desc), self.n, _dptr(pos), _dptr(v), _dptr(m),
                                    None if mid is None else mid.ctypes.data_as(C.POINTER(C.c_int32)))
        if not self.h:
            raise RuntimeError("orc_scene_create failed")

    def __del__(self):
        try:
            if self.h:
                lib().orc_scene_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def substep(self, n: int = 1) -> int:
        return int(lib().orc_substep(self.h, n))

    def rebin(self) -> int:
        return int(lib().orc_rebin(self.h))

    def field(self, field_id: int) -> np.ndarray:
        nc = FIELD_COMPONENTS[field_id]
        out = np.empty(self.n * nc, dtype=np.float64)
        lib().orc_get_field(self.h, field_id, _dptr(out))
        return out.reshape(self.n, nc) if nc > 1 else out

    def field_by_id(self, field_id: int) -> np.ndarray:
        """Field in original particle order."""
        ids = self.field(12).astype(np.int64)
        f = self.field(field_id)
        out = np.empty_like(f)
        out[ids] = f
        return out

    def binning(self, array: int) -> np.ndarray:
        L = lib()
        nb, ng = int(L.orc_num_blocks(self.h)), int(L.orc_num_grid_blocks(self.h))
        if array == 0:
            out = np.zeros(4, dtype=np.int64)
        else:
            size = {1: self.n, 2: self.n, 3: nb, 4: nb + 1, 5: nb * 64 + 1, 6: ng, 7: nb * 8}[array]
            out = np.empty(size, dtype=np.uint32 if array in (2, 3, 6) else np.int32)
        L.orc_get_binning(self.h, array, out.ctypes.data_as(C.c_void_p))
        return out

    def diagnostics(self, diag_type):
        d = diag_type()
        lib().orc_diagnostics(self.h, C.byref(d))
        return d.as_dict()


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


class SceneSetup:
    """Scene set-up through the oracle instead of the product library, for the
    benchmark's CPU legs: the same ctypes structures (pure Python) filled by
    orc_scene_desc_reference_defaults and orc_generate_particles."""

    def __init__(self, G):
        self.G = G  # the package's gmpm module (its structure types only)

    def reference_defaults(self, dx: float, res):
        d = self.G.SceneDesc()
        if lib().orc_scene_desc_reference_defaults(C.byref(d), dx, int(res[0]), int(res[1]), int(res[2])) != 0:
            raise RuntimeError("orc_scene_desc_reference_defaults failed")
        return d

    def generate_particles(self, geom):
        L = lib()
        n = C.c_int64(0)
        if L.orc_generate_particles(C.byref(geom), C.byref(n), None, None, 0) != 0:
            raise RuntimeError("orc_generate_particles failed")
        pos = np.empty((n.value, 3), dtype=np.float64)
        mat = np.empty(n.value, dtype=np.int32)
        if L.orc_generate_particles(C.byref(geom), C.byref(n), _dptr(pos), mat.ctypes.data_as(C.POINTER(C.c_int32)),
                                    n.value) != 0:
            raise RuntimeError("orc_generate_particles failed")
        return pos, mat
