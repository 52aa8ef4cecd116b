"""Python binding of the engine's C ABI (include/mdn.h), loaded from the
in-tree library md_nucleation_b200/lib/libmdn.so.

The binding fails loudly when the library is missing or no CUDA device is
present; there is no CPU fallback.  ``Engine`` drives a batch of replicas the
way ``MD::run`` drives one (reference src/run.cpp:17-74): ``step`` is n calls
of ``MD::verlet``, ``make_pair`` is ``MD::make_pair``, ``recenter`` the
re-centring between relaxation and production, ``set_nvt`` the thermostat
switches (``MD::setNVE``).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .system import ReplicaSpec, StateArrays, descs

_LIB = None
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libmdn.so")


class MdnError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mdn error {code}: {msg}")
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with python -m md_nucleation_b200.build")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.mdn_abi_version.restype = C.c_int
        L.mdn_last_error.restype = C.c_char_p
        L.mdn_default_options.argtypes = [C.POINTER(abi.Options)]
        L.mdn_device_count.argtypes = [C.POINTER(C.c_int)]
        L.mdn_create.argtypes = [C.POINTER(abi.ReplicaDesc), C.c_int, C.POINTER(abi.Options), C.POINTER(vp)]
        L.mdn_destroy.argtypes = [vp]
        L.mdn_step.argtypes = [vp, C.c_longlong, C.c_int]
        L.mdn_make_pair.argtypes = [vp]
        L.mdn_recenter.argtypes = [vp, C.c_int]
        L.mdn_set_nvt.argtypes = [vp, C.c_int, C.c_int, C.c_double]
        L.mdn_compute_forces.argtypes = [vp, C.c_uint]
        L.mdn_energies.argtypes = [vp, C.POINTER(C.c_double)]
        L.mdn_get_status.argtypes = [vp, C.POINTER(C.c_int)]
        L.mdn_clear_status.argtypes = [vp]
        L.mdn_replica_info_get.argtypes = [vp, C.c_int, C.POINTER(abi.ReplicaInfo)]
        L.mdn_download_state.argtypes = [vp, C.c_int, C.POINTER(abi.State)]
        L.mdn_upload_state.argtypes = [vp, C.c_int, C.POINTER(abi.State)]
        L.mdn_pair_list.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
        L.mdn_in_domain.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.mdn_events.argtypes = [vp, C.POINTER(abi.Event), C.c_int, C.POINTER(C.c_int)]
        L.mdn_kinetic.argtypes = [vp, C.POINTER(C.c_double)]
        L.mdn_last_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        L.mdn_set_launch.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.mdn_get_launch.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.mdn_tune_launch.argtypes = [vp, C.c_longlong, C.POINTER(C.c_int)]
        L.mdn_set_split.argtypes = [vp, C.c_int, C.c_int]
        L.mdn_get_split.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.mdn_adjoint_params.argtypes = [C.POINTER(abi.ReplicaDesc), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
        L.mdn_adjoint.argtypes = [vp, C.POINTER(abi.ReplicaDesc), C.POINTER(abi.AdjointSpec),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.mdn_snapshot.argtypes = [vp, C.POINTER(C.c_longlong), C.c_longlong, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.POINTER(C.c_double)]
        L.mdn_host_alloc.argtypes = [C.c_size_t, C.POINTER(C.c_void_p)]
        L.mdn_host_free.argtypes = [C.c_void_p]
        L.mdn_set_nvt_batch.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.mdn_profile.argtypes = [vp, C.c_int, C.POINTER(C.c_longlong)]
        dp = C.POINTER(C.c_double)
        L.mdn_place.argtypes = [C.c_int, C.POINTER(abi.PlaceDesc), dp, dp, dp, dp]
        if L.mdn_abi_version() != abi.ABI_VERSION:
            raise RuntimeError("libmdn.so ABI version mismatch")
        _LIB = L
    return _LIB


def _ck(rc):
    if rc != abi.OK:
        raise MdnError(rc, lib().mdn_last_error().decode())


def device_count() -> int:
    n = C.c_int(0)
    lib().mdn_device_count(C.byref(n))
    return n.value


def place(box, ion_x, n_gas, n_vapor, gas_sigma, vapor_sigma, seed, min_dist=10.0, device=0):
    """Initial centres and velocities of the gas and vapor molecules on the
    GPU (mdn_place): MD::initialization_gas / initialization_vapor
    (src/initialization/initializationGas.cpp:24-100,
    src/initialization/initializationVapor.cpp:14-76).  Returns
    (gas_x, gas_v, vapor_x, vapor_v), each [n, 3] float64."""
    ion = np.ascontiguousarray(ion_x, np.float64).reshape(-1, 3)
    d = abi.PlaceDesc(box=box, min_dist=min_dist, n_ion=len(ion), ion_x=abi.ptr(ion), n_gas=n_gas,
                      n_vapor=n_vapor, gas_sigma=gas_sigma, vapor_sigma=vapor_sigma, seed=seed)
    out = [np.zeros((n, 3)) for n in (n_gas, n_gas, n_vapor, n_vapor)]
    _ck(lib().mdn_place(device, C.byref(d), *[abi.ptr(a) for a in out]))
    return tuple(out)


def default_options(**kw) -> abi.Options:
    o = abi.Options()
    lib().mdn_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class PinnedArray:
    """A numpy view of page-locked host memory from mdn_host_alloc."""

    def __init__(self, shape, dtype):
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = C.c_void_p()
        _ck(lib().mdn_host_alloc(self.nbytes, C.byref(self.ptr)))
        buf = (C.c_byte * self.nbytes).from_address(self.ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            lib().mdn_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class SnapshotBuffer:
    """Host buffers of mdn_snapshot (page-locked when pinned=True)."""

    def __init__(self, n_replicas: int, capacity: int, pinned: bool = True):
        self.capacity = int(capacity)
        self.offset = np.zeros(n_replicas + 1, np.int64)
        if pinned:
            self._t = PinnedArray((capacity,), np.int32)
            self._x = PinnedArray((capacity, 3), np.float64)
            self._v = PinnedArray((capacity, 3), np.float64)
            self.type, self.x, self.v = self._t.array, self._x.array, self._v.array
        else:
            self.type = np.zeros(capacity, np.int32)
            self.x = np.zeros((capacity, 3))
            self.v = np.zeros((capacity, 3))
        self.type_ptr = self.type.ctypes.data_as(C.c_void_p)
        self.x_ptr = self.x.ctypes.data_as(C.c_void_p)
        self.v_ptr = self.v.ctypes.data_as(C.c_void_p)
        self.U = None

    def rows(self, r):
        a, b = self.offset[r], self.offset[r + 1]
        return self.type[a:b], self.x[a:b], self.v[a:b]

    @property
    def nbytes_used(self):
        n = int(self.offset[-1])
        return n * (4 + 48)


class Engine:
    """A batch of replicas resident on one GPU."""

    def __init__(self, specs: Sequence[ReplicaSpec], **options):
        self.specs = list(specs)
        self.L = lib()
        self._descs, self._keep = descs(self.specs)
        self.opt = default_options(**options)
        h = C.c_void_p()
        _ck(self.L.mdn_create(self._descs, len(self.specs), C.byref(self.opt), C.byref(h)))
        self.h = h

    @property
    def n(self):
        return len(self.specs)

    def close(self):
        if getattr(self, "h", None):
            self.L.mdn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- stepping -------------------------------------------------------------
    def step(self, n: int = 1, energy_mode: int = 0):
        _ck(self.L.mdn_step(self.h, n, energy_mode))

    def make_pair(self):
        _ck(self.L.mdn_make_pair(self.h))

    def recenter(self, compat: bool = True):
        _ck(self.L.mdn_recenter(self.h, 1 if compat else 0))

    def set_nvt(self, mode: int, temperature: float = 300.0, replica: int = -1):
        _ck(self.L.mdn_set_nvt(self.h, replica, mode, temperature))

    def set_nvt_batch(self, modes: np.ndarray, temperatures: np.ndarray):
        _ck(self.L.mdn_set_nvt_batch(self.h, abi.ptr(modes, C.c_int), abi.ptr(temperatures)))

    def compute_forces(self, term_mask: int = 0):
        _ck(self.L.mdn_compute_forces(self.h, term_mask))

    def get_launch(self):
        """(cluster size, threads per CTA, steps per launch) of mdn_step."""
        c, t, n = C.c_int(), C.c_int(), C.c_int()
        _ck(self.L.mdn_get_launch(self.h, C.byref(c), C.byref(t), C.byref(n)))
        return c.value, t.value, n.value

    def tune_launch(self, n_steps: int = 100) -> int:
        """Runs n_steps at each cluster size 1, 2, 4, 8 and keeps the fastest,
        then tries the split launch (mdn_tune_launch); returns the cluster
        size.  The steps advance the replicas."""
        best = C.c_int(0)
        _ck(self.L.mdn_tune_launch(self.h, n_steps, C.byref(best)))
        return best.value

    def set_split(self, n_largest: int, cluster_size: int = 0):
        """The n_largest replicas in a concurrent second launch on clusters of
        cluster_size CTAs (mdn_set_split); 0 turns it off."""
        _ck(self.L.mdn_set_split(self.h, n_largest, cluster_size))

    def get_split(self):
        """(n_largest, cluster_size) of the split launch, (0, 0) when off."""
        n, c = C.c_int(), C.c_int()
        _ck(self.L.mdn_get_split(self.h, C.byref(n), C.byref(c)))
        return n.value, c.value

    # ---- gradient harness ------------------------------------------------------
    def adjoint_params(self):
        """Rows (kind, type_a, type_b) of mdn_adjoint's gradient: kind 0 =
        gas-ion pair (eps at 2k, sigma at 2k+1), 1 = vapor-ion pair, 2 = the
        ion charge scale (the last parameter)."""
        n = C.c_int(0)
        _ck(self.L.mdn_adjoint_params(C.byref(self._descs[0]), C.byref(n), None, 0))
        rows = np.zeros((n.value // 2 + 1, 3), np.int32)
        _ck(self.L.mdn_adjoint_params(C.byref(self._descs[0]), C.byref(n), abi.ptr(rows, C.c_int), len(rows)))
        return rows, n.value

    def adjoint(self, n_steps: int, checkpoint_every: int = 100, count_radius: float = 10.0,
                count_width: float = 1.0, w_energy: float = 1.0, w_count: float = 1.0):
        """mdn_adjoint over the next n_steps of the (single) replica; returns
        (J, dJ/dtheta, (forward ms, adjoint ms)).  The replica advances."""
        spec = abi.AdjointSpec(n_steps, checkpoint_every, count_radius, count_width, w_energy, w_count)
        _, n = self.adjoint_params()
        J = C.c_double(0)
        grad = np.zeros(n)
        ms = np.zeros(2)
        _ck(self.L.mdn_adjoint(self.h, C.byref(self._descs[0]), C.byref(spec), C.byref(J), abi.ptr(grad),
                               abi.ptr(ms)))
        return J.value, grad, (float(ms[0]), float(ms[1]))

    def set_launch(self, cluster_size=0, threads=0, steps_per_launch=-1):
        _ck(self.L.mdn_set_launch(self.h, cluster_size, threads, steps_per_launch))

    # ---- results --------------------------------------------------------------
    def energies(self) -> np.ndarray:
        U = np.zeros((self.n, 8))
        _ck(self.L.mdn_energies(self.h, abi.ptr(U)))
        return U

    def status(self) -> np.ndarray:
        s = np.zeros(self.n, np.int32)
        _ck(self.L.mdn_get_status(self.h, abi.ptr(s, C.c_int)))
        return s

    def clear_status(self):
        _ck(self.L.mdn_clear_status(self.h))

    def info(self, r: int = 0) -> abi.ReplicaInfo:
        i = abi.ReplicaInfo()
        _ck(self.L.mdn_replica_info_get(self.h, r, C.byref(i)))
        return i

    def state(self, r: int = 0) -> StateArrays:
        s = StateArrays.for_spec(self.specs[r])
        st = s.to_c()
        _ck(self.L.mdn_download_state(self.h, r, C.byref(st)))
        s.pull_scalars(st)
        return s

    def upload(self, r: int, s: StateArrays):
        st = s.to_c()
        _ck(self.L.mdn_upload_state(self.h, r, C.byref(st)))

    def pair_list(self, r: int, kind: int) -> np.ndarray:
        cnt = C.c_int(0)
        _ck(self.L.mdn_pair_list(self.h, r, kind, None, 0, C.byref(cnt)))
        buf = np.zeros((max(cnt.value, 1), 2), np.int32)
        _ck(self.L.mdn_pair_list(self.h, r, kind, abi.ptr(buf, C.c_int), cnt.value, C.byref(cnt)))
        return buf[:cnt.value]

    def in_domain(self, r: int = 0):
        cnt = C.c_int(0)
        _ck(self.L.mdn_in_domain(self.h, r, 0, C.byref(cnt), None, None, None))
        n = cnt.value
        t = np.zeros(max(n, 1), np.int32)
        x = np.zeros((max(n, 1), 3))
        v = np.zeros((max(n, 1), 3))
        _ck(self.L.mdn_in_domain(self.h, r, n, C.byref(cnt), abi.ptr(t, C.c_int), abi.ptr(x), abi.ptr(v)))
        return t[:n], x[:n], v[:n]

    def events(self):
        cnt = C.c_int(0)
        cap = 65536
        buf = (abi.Event * cap)()
        _ck(self.L.mdn_events(self.h, buf, cap, C.byref(cnt)))
        return [buf[i] for i in range(min(cnt.value, cap))]

    def kinetic(self) -> np.ndarray:
        out = np.zeros((self.n, 4))
        _ck(self.L.mdn_kinetic(self.h, abi.ptr(out)))
        return out

    def snapshot(self, buf: "SnapshotBuffer", energies: bool = True):
        """All replicas' in-domain atoms (and energies) into `buf`; returns the
        row offsets per replica."""
        U = np.zeros((self.n, 8)) if energies else None
        _ck(self.L.mdn_snapshot(self.h, abi.ptr(buf.offset, C.c_longlong), buf.capacity, buf.type_ptr,
                                buf.x_ptr, buf.v_ptr, abi.ptr(U) if energies else None))
        buf.U = U
        return buf.offset

    PROFILE_PHASES = ("total", "core_integration", "gas_integration", "rebuild", "near_gas",
                      "core_bonded", "core_pairs", "core_reduce_kick")

    def profile(self, enable: bool = True):
        """Starts (enable) or stops the per-replica cycle accounting; returns the
        [n_replicas, 8] cycles accumulated so far."""
        out = np.zeros((self.n, 8), np.int64)
        _ck(self.L.mdn_profile(self.h, 1 if enable else 0, abi.ptr(out, C.c_longlong)))
        return out

    def last_timing(self):
        ms = C.c_double(0)
        n = C.c_longlong(0)
        _ck(self.L.mdn_last_timing(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value
