"""ctypes bindings of the oracle libraries -- TEST INFRASTRUCTURE ONLY.

  RefReplica   the reference program's own routines (oracle/_ref/libref_harness.so,
               built from the reference sources by oracle/Makefile)
  OracleReplica the FP64 CPU restatement (oracle/_build/libmdn_oracle.so)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module; nothing in the md_nucleation_b200 package does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from md_nucleation_b200 import abi
from md_nucleation_b200.system import ReplicaSpec, StateArrays

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_harness.so")
ORC_LIB = os.path.join(HERE, "_build", "libmdn_oracle.so")

_ref = None
_orc = None


# where oracle/Makefile reads the reference's sources: its REF variable from
# the environment, else the reference checkout beside the repository
REF_SRC = os.path.join(os.environ.get("REF", os.path.join(os.path.dirname(HERE), "..", "reference")), "src")


def reference_sources_present() -> bool:
    return os.path.isdir(REF_SRC)


def build(reference: bool = True):
    """Runs oracle/Makefile (the reference part only if its sources are present)."""
    target = "all" if reference else "restatement"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def have_reference() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle reference)")
        L = C.CDLL(REF_LIB)
        vp = C.c_void_p
        L.ref_create.restype = vp
        L.ref_create.argtypes = [C.POINTER(abi.ReplicaDesc), C.c_int]
        L.ref_destroy.argtypes = [vp]
        L.ref_info.argtypes = [vp, C.POINTER(C.c_int)]
        L.ref_get_state.argtypes = [vp, C.POINTER(abi.State)]
        L.ref_set_state.argtypes = [vp, C.POINTER(abi.State)]
        L.ref_verlet.argtypes = [vp, C.c_longlong, C.c_int, C.POINTER(C.c_double)]
        L.ref_verlet_shake.argtypes = [vp, C.c_longlong, C.c_int, C.POINTER(C.c_double)]
        L.ref_compute_forces.argtypes = [vp, C.c_uint, C.POINTER(C.c_double)]
        for n in ("ref_make_pair", "ref_update_in_centers", "ref_velocity_calculation",
                  "ref_update_position", "ref_update_position_shake", "ref_velocity_scaling",
                  "ref_nosehoover_zeta", "ref_nosehoover_ion", "ref_set_nve"):
            getattr(L, n).argtypes = [vp]
        L.ref_shake.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        L.ref_rotation.argtypes = [C.c_double] * 6 + [C.POINTER(C.c_double)]
        L.ref_kinetic.argtypes = [vp, C.POINTER(C.c_double)]
        L.ref_pair_list.restype = C.c_int
        L.ref_pair_list.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.ref_in_domain_atoms.restype = C.c_int
        L.ref_in_domain_atoms.argtypes = [vp]
        L.ref_export_dump.argtypes = [vp, C.c_char_p, C.c_double]
        L.ref_verlet_many.argtypes = [C.POINTER(vp), C.c_int, C.c_longlong, C.c_int]
        _ref = L
    return _ref


class RefReplica:
    """One replica driven by the reference's routines."""

    def __init__(self, spec: ReplicaSpec, make_pair: bool = True):
        self.spec = spec
        self.L = ref_lib()
        self._desc, self._keep = spec.to_desc()
        self.h = self.L.ref_create(C.byref(self._desc), 1 if make_pair else 0)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        out = (C.c_int * 8)()
        self.L.ref_info(self.h, out)
        keys = ("n_gas_in", "n_vapor_in", "loop_pair", "loop_update", "gi_pairs", "gv_pairs",
                "vv_pairs", "gg_pairs")
        return dict(zip(keys, list(out)))

    def get_state(self) -> StateArrays:
        s = StateArrays.for_spec(self.spec)
        st = s.to_c()
        self.L.ref_get_state(self.h, C.byref(st))
        s.pull_scalars(st)
        return s

    def set_state(self, s: StateArrays):
        st = s.to_c()
        self.L.ref_set_state(self.h, C.byref(st))

    def verlet(self, n=1, energy_mode=0, shake=False):
        U = np.zeros(8)
        f = self.L.ref_verlet_shake if shake else self.L.ref_verlet
        f(self.h, n, energy_mode, abi.ptr(U))
        return U

    def compute_forces(self, term_mask=0):
        U = np.zeros(8)
        self.L.ref_compute_forces(self.h, term_mask, abi.ptr(U))
        return U

    def call(self, name):
        getattr(self.L, "ref_" + name)(self.h)

    def shake(self, mol, old_x):
        old_x = np.ascontiguousarray(old_x, np.float64)
        self.L.ref_shake(self.h, mol, abi.ptr(old_x))

    def kinetic(self):
        out = np.zeros(6)
        self.L.ref_kinetic(self.h, abi.ptr(out))
        return out

    def pair_list(self, kind):
        n = self.L.ref_pair_list(self.h, kind, None, 0)
        buf = np.zeros((max(n, 1), 2), np.int32)
        self.L.ref_pair_list(self.h, kind, abi.ptr(buf, C.c_int), n)
        return buf[:n]

    def in_domain_atoms(self):
        return self.L.ref_in_domain_atoms(self.h)

    def export_dump(self, path, time_fs=0.0):
        self.L.ref_export_dump(self.h, path.encode(), time_fs)


def ref_rotation(A, B, C_, x, y, z):
    out = np.zeros(3)
    ref_lib().ref_rotation(A, B, C_, x, y, z, abi.ptr(out))
    return out


def ref_verlet_many(replicas, n_steps, threads=0):
    """Steps several RefReplica objects with the reference's own replica model:
    one replica per OpenMP thread (src/main.cpp:22-29)."""
    L = ref_lib()
    arr = (C.c_void_p * len(replicas))(*[r.h for r in replicas])
    L.ref_verlet_many(arr, len(replicas), n_steps, threads)


# ---------------------------------------------------------------------------
# the FP64 restatement
# ---------------------------------------------------------------------------
def orc_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_LIB):
            raise FileNotFoundError(f"{ORC_LIB} not built (make -C oracle restatement)")
        L = C.CDLL(ORC_LIB)
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(abi.ReplicaDesc), C.c_uint, C.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_step.argtypes = [vp, C.c_longlong, C.c_int]
        L.orc_make_pair.argtypes = [vp]
        L.orc_recenter.argtypes = [vp, C.c_int]
        L.orc_set_nvt.argtypes = [vp, C.c_int, C.c_double]
        L.orc_compute_forces.argtypes = [vp, C.c_uint]
        L.orc_energies.argtypes = [vp, C.POINTER(C.c_double)]
        L.orc_info.argtypes = [vp, C.POINTER(abi.ReplicaInfo)]
        L.orc_get_state.argtypes = [vp, C.POINTER(abi.State)]
        L.orc_set_state.argtypes = [vp, C.POINTER(abi.State)]
        L.orc_pair_list.restype = C.c_int
        L.orc_pair_list.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.orc_kinetic.argtypes = [vp, C.POINTER(C.c_double)]
        L.orc_status.restype = C.c_int
        L.orc_status.argtypes = [vp]
        L.orc_rotate.argtypes = [C.c_double] * 6 + [C.c_int, C.POINTER(C.c_double)]
        L.orc_philox.argtypes = [C.c_ulonglong, C.c_uint * 4, C.POINTER(C.c_uint)]
        L.orc_step_many.argtypes = [C.POINTER(vp), C.c_int, C.c_longlong, C.c_int]
        L.orc_objective.restype = C.c_double
        L.orc_objective.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_adjoint.restype = C.c_int
        L.orc_adjoint.argtypes = [vp, C.c_longlong, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
        L.orc_window.restype = C.c_double
        L.orc_window.argtypes = [vp, C.c_longlong, C.c_double, C.c_double, C.c_double, C.c_double]
        dp = C.POINTER(C.c_double)
        L.orc_place.restype = C.c_int
        L.orc_place.argtypes = [C.POINTER(abi.PlaceDesc), dp, dp, dp, dp]
        _orc = L
    return _orc


class OracleReplica:
    """One replica advanced by the FP64 restatement (same algorithm, same
    random streams and same reference behaviours as the CUDA engine)."""

    def __init__(self, spec: ReplicaSpec, quirks: int = abi.Q_ALL, force_mode: int = 0):
        self.spec = spec
        self.L = orc_lib()
        self._desc, self._keep = spec.to_desc()
        self.h = self.L.orc_create(C.byref(self._desc), quirks, force_mode)
        if not self.h:
            raise RuntimeError("orc_create failed")

    @classmethod
    def from_desc(cls, desc_ptr, quirks: int = abi.Q_ALL, force_mode: int = 0):
        """A replica from a descriptor built elsewhere (the C++ host's
        mdnh_desc); desc_ptr must outlive the replica."""
        from types import SimpleNamespace as NS
        d = desc_ptr.contents
        o = cls.__new__(cls)
        o.spec = NS(ion=NS(n=d.ion.n_atoms), gas=NS(n=d.gas.n_atoms), vapor=NS(n=d.vapor.n_atoms),
                    n_gas=d.n_gas, n_vapor=d.n_vapor)
        o.L = orc_lib()
        o._desc, o._keep = desc_ptr, None
        o.h = o.L.orc_create(desc_ptr, quirks, force_mode)
        if not o.h:
            raise RuntimeError("orc_create failed")
        return o

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1, energy_mode=0):
        self.L.orc_step(self.h, n, energy_mode)

    def make_pair(self):
        self.L.orc_make_pair(self.h)

    def recenter(self, compat=1):
        self.L.orc_recenter(self.h, compat)

    def set_nvt(self, mode, T=300.0):
        self.L.orc_set_nvt(self.h, mode, T)

    def compute_forces(self, term_mask=0):
        self.L.orc_compute_forces(self.h, term_mask)
        return self.energies()

    def energies(self):
        U = np.zeros(8)
        self.L.orc_energies(self.h, abi.ptr(U))
        return U

    def info(self):
        i = abi.ReplicaInfo()
        self.L.orc_info(self.h, C.byref(i))
        return i

    def status(self):
        return self.L.orc_status(self.h)

    def get_state(self) -> StateArrays:
        s = StateArrays.for_spec(self.spec)
        st = s.to_c()
        self.L.orc_get_state(self.h, C.byref(st))
        s.pull_scalars(st)
        return s

    def set_state(self, s: StateArrays):
        st = s.to_c()
        self.L.orc_set_state(self.h, C.byref(st))

    def pair_list(self, kind):
        n = self.L.orc_pair_list(self.h, kind, None, 0)
        buf = np.zeros((max(n, 1), 2), np.int32)
        self.L.orc_pair_list(self.h, kind, abi.ptr(buf, C.c_int), n)
        return buf[:n]

    def kinetic(self):
        out = np.zeros(4)
        self.L.orc_kinetic(self.h, abi.ptr(out))
        return out

    def objective(self, R0=10.0, W=1.0, w_energy=1.0, w_count=1.0):
        return self.L.orc_objective(self.h, R0, W, w_energy, w_count)

    def adjoint(self, n, theta, rows, R0=10.0, W=1.0, w_energy=1.0, w_count=1.0):
        """(J, dJ/dtheta) of the window over the next n steps by the FP64 CPU
        adjoint (oracle/adjoint_ad.h); the replica is not advanced.  theta,
        rows: as gradients.parameters (rows as mdn_adjoint_params)."""
        th = np.ascontiguousarray(theta, np.float64)
        rw = np.ascontiguousarray(rows, np.int32).reshape(-1, 3)
        J = C.c_double(0.0)
        g = np.zeros(len(th))
        rc = self.L.orc_adjoint(self.h, n, R0, W, w_energy, w_count, abi.ptr(th), abi.ptr(rw, C.c_int), len(rw),
                                C.byref(J), abi.ptr(g))
        if rc != 0:
            raise RuntimeError(f"orc_adjoint returned {rc}")
        return J.value, g

    def window(self, n, R0=10.0, W=1.0, w_energy=1.0, w_count=1.0):
        """Advances n steps; the window average of the objective."""
        return self.L.orc_window(self.h, n, R0, W, w_energy, w_count)


def orc_rotate(a, b, c, x, y, z, zy_quirk=0):
    out = np.zeros(3)
    orc_lib().orc_rotate(a, b, c, x, y, z, zy_quirk, abi.ptr(out))
    return out


def orc_philox(key, ctr):
    out = (C.c_uint * 4)()
    orc_lib().orc_philox(key, (C.c_uint * 4)(*ctr), out)
    return list(out)


def orc_place(box, ion_x, n_gas, n_vapor, gas_sigma, vapor_sigma, seed, min_dist=10.0):
    """The restated placement loop (orc_place): (gas_x, gas_v, vapor_x,
    vapor_v) as [n, 3] arrays, or RuntimeError when it does not converge."""
    ion = np.ascontiguousarray(ion_x, np.float64).reshape(-1, 3)
    d = abi.PlaceDesc(box=box, min_dist=min_dist, n_ion=len(ion), ion_x=abi.ptr(ion), n_gas=n_gas,
                      n_vapor=n_vapor, gas_sigma=gas_sigma, vapor_sigma=vapor_sigma, seed=seed)
    out = [np.zeros((n, 3)) for n in (n_gas, n_gas, n_vapor, n_vapor)]
    if orc_lib().orc_place(C.byref(d), *[abi.ptr(a) for a in out]) != 0:
        raise RuntimeError("placement did not converge")
    return tuple(out)


def orc_step_many(replicas, n_steps, threads=0):
    L = orc_lib()
    arr = (C.c_void_p * len(replicas))(*[r.h for r in replicas])
    L.orc_step_many(arr, len(replicas), n_steps, threads)
