"""ctypes binding of the C++ host (lib/libmdn_host.so, md_nucleation_b200/host/).

The host reads the reference program's condition file and the ion / vapor
files it names (MD::readCondFile, src/initialization/setCondition.cpp:4-254;
Variables::readIonFile / readVaporFile), places the molecules, builds the
engine's replica descriptor and runs a batch with MD::run's cadence and
output files (src/run.cpp:17-74, src/output/output.cpp).  The command-line
form is bin/mdn_run.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from . import abi
from .build import BIN_DIR, HOST_LIB

MDN_RUN = os.path.join(BIN_DIR, "mdn_run")

_LIB = None


class Settings(C.Structure):
    _fields_ = [
        ("total_steps", C.c_longlong), ("relax_steps", C.c_longlong), ("observe", C.c_int),
        ("calc_number", C.c_int), ("pressure", C.c_double), ("n_gas", C.c_int), ("n_vapor", C.c_int),
        ("gas_kind", C.c_int), ("interactions", C.c_uint), ("nvt_mode", C.c_int),
        ("nvt_temperature", C.c_double), ("box", C.c_double),
    ]


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(HOST_LIB):
            raise FileNotFoundError(f"{HOST_LIB} is missing: build it with python -m md_nucleation_b200.build")
        L = C.CDLL(HOST_LIB)
        vp = C.c_void_p
        L.mdnh_load.argtypes = [C.c_char_p, C.c_int, C.c_ulonglong, C.c_int, C.POINTER(vp)]
        L.mdnh_load_ex.argtypes = [C.c_char_p, C.c_int, C.c_ulonglong, C.c_int, C.c_int, C.POINTER(vp)]
        L.mdnh_free.argtypes = [vp]
        L.mdnh_free.restype = None
        L.mdnh_last_error.restype = C.c_char_p
        L.mdnh_desc.argtypes = [vp]
        L.mdnh_desc.restype = C.POINTER(abi.ReplicaDesc)
        L.mdnh_get_settings.argtypes = [vp, C.POINTER(Settings)]
        L.mdnh_type_name.argtypes = [vp, C.c_int]
        L.mdnh_type_name.restype = C.c_char_p
        L.mdnh_dump_path.argtypes = [vp]
        L.mdnh_dump_path.restype = C.c_char_p
        L.mdnh_write_dump_frame.argtypes = [vp, C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p]
        L.mdnh_run.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(abi.Options), C.c_int]
        _LIB = L
    return _LIB


class HostError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _ck(rc):
    if rc != 0:
        raise HostError(rc, lib().mdnh_last_error().decode())


def _arr(ptr, n, dtype):
    if n <= 0 or not ptr:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy()


class HostSystem:
    """One system read from a condition file (and the files it names).
    place_device >= 0 places the molecules on that GPU (mdn_place), -1 on
    the CPU."""

    def __init__(self, condition_file: str, calc_number: int = 0, seed: int = 0, reference_masses: bool = False,
                 place_device: int = -1):
        self.L = lib()
        h = C.c_void_p()
        _ck(self.L.mdnh_load_ex(condition_file.encode(), calc_number, seed, 1 if reference_masses else 0,
                                place_device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.mdnh_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def desc(self) -> abi.ReplicaDesc:
        return self.L.mdnh_desc(self.h).contents

    def desc_ptr(self):
        return self.L.mdnh_desc(self.h)

    @property
    def settings(self) -> Settings:
        s = Settings()
        _ck(self.L.mdnh_get_settings(self.h, C.byref(s)))
        return s

    def type_name(self, t: int) -> str:
        return self.L.mdnh_type_name(self.h, t).decode()

    @property
    def dump_path(self) -> str:
        return self.L.mdnh_dump_path(self.h).decode()

    def topology(self, which: str) -> dict:
        """ion / gas / vapor topology of the descriptor as numpy arrays."""
        t = getattr(self.desc, which)
        n = t.n_atoms
        return {
            "type": _arr(t.type, n, np.int64), "charge": _arr(t.charge, n, float),
            "x": _arr(t.x, 3 * n, float).reshape(-1, 3),
            "bonds": _arr(t.bonds, 3 * t.n_bonds, np.int64).reshape(-1, 3),
            "rigid": _arr(t.rigid, 3 * t.n_rigid, np.int64).reshape(-1, 3),
            "angles": _arr(t.angles, 4 * t.n_angles, np.int64).reshape(-1, 4),
            "dihedrals": _arr(t.dihedrals, 5 * t.n_dihedrals, np.int64).reshape(-1, 5),
        }

    def write_dump_frame(self, path: str, timestep: int, type_: np.ndarray, x: np.ndarray, v: np.ndarray,
                         shift=None):
        type_ = np.ascontiguousarray(type_, np.int32)
        x = np.ascontiguousarray(x, float)
        v = np.ascontiguousarray(v, float)
        sh = None if shift is None else np.ascontiguousarray(shift, float)
        _ck(self.L.mdnh_write_dump_frame(self.h, path.encode(), int(timestep), len(type_),
                                         type_.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
                                         v.ctypes.data_as(C.c_void_p),
                                         None if sh is None else sh.ctypes.data_as(C.c_void_p)))


def run(systems: Sequence[HostSystem], verbose: bool = False, **options):
    """Runs the systems as one batch on one GPU (mdnh_run)."""
    from .engine import default_options
    opt = default_options(**options)
    arr = (C.c_void_p * len(systems))(*[s.h for s in systems])
    _ck(lib().mdnh_run(arr, len(systems), C.byref(opt), 1 if verbose else 0))
