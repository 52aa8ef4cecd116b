"""Replica descriptions: the Python mirror of ``mdn_replica_desc``.

A :class:`ReplicaSpec` holds everything ``MD::MD`` would have built for one
replica (reference ``src/initialization/md.cpp:8-40``): the type tables, the
ion (seed) topology and state, the gas and vapor molecule templates, the
molecule centres and the run parameters.  ``to_desc()`` packs it into the C
structure consumed by the engine (``mdn_create``), the CPU oracle and the
reference harness, so all three see byte-identical inputs.

Physical constants are the reference's (``src/constants.hpp:28-53``), kept
at their non-CODATA values on purpose.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi

# src/constants.hpp:28-53
NW = 6.02e23
KB = 1.38e-23
KB_REAL = KB * NW / 4184.0
E0 = 8.85e-12
E_CHARGE = 1.602e-19
QQRD2E = E_CHARGE * E_CHARGE / 4.0 / np.pi / E0 * NW * 1e10 / 4184.0
REAL_TO_KCALMOL = 10000 / 4.184
MN2, MHE, MAR = 28.0, 4.0026, 39.948
R_INTER, OVERLAP = 100.0, 10.0

# Gas species as readCondFile defines them (src/initialization/setCondition.cpp:43-118):
# atom mass, eps, sigma, template atoms, bond; and the molecule mass of
# Physical::setPhysicalProp (src/initialization/PhysicalProp.cpp:4-23) that
# divides the centre of mass and sets the Maxwell-Boltzmann width.
GAS_TABLE = {
    "He": dict(kind=abi.GAS_HE, mass=4.027, eps=0.0203, sigma=2.556,
               x=[[0.0, 0.0, 0.0]], bond=None, mol_mass=MHE),
    "N2": dict(kind=abi.GAS_N2, mass=14.01, eps=0.1098, sigma=3.27351824993,
               x=[[-0.549, 0.0, 0.0], [0.549, 0.0, 0.0]], bond=(1221.7, 1.098), mol_mass=MN2),
    "N2monoatomic": dict(kind=abi.GAS_N2MONO, mass=28.02, eps=0.14397, sigma=3.798,
                         x=[[0.0, 0.0, 0.0]], bond=None, mol_mass=MN2),
    "Ar": dict(kind=abi.GAS_AR, mass=28.02, eps=0.14397, sigma=3.798,
               x=[[0.0, 0.0, 0.0]], bond=None, mol_mass=MAR),
}
GAS_TABLE["N2mono"] = GAS_TABLE["N2monoatomic"]


@dataclass
class Topology:
    type: np.ndarray
    charge: np.ndarray
    x: np.ndarray  # [n,3]
    bonds: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    rigid: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    angles: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    dihedrals: np.ndarray = field(default_factory=lambda: np.zeros((0, 5), np.int32))

    def __post_init__(self):
        self.type = np.ascontiguousarray(self.type, np.int32)
        self.charge = np.ascontiguousarray(self.charge, np.float64)
        self.x = np.ascontiguousarray(np.asarray(self.x, np.float64).reshape(-1, 3))
        self.bonds = np.ascontiguousarray(np.asarray(self.bonds, np.int32).reshape(-1, 3))
        self.rigid = np.ascontiguousarray(np.asarray(self.rigid, np.int32).reshape(-1, 3))
        self.angles = np.ascontiguousarray(np.asarray(self.angles, np.int32).reshape(-1, 4))
        self.dihedrals = np.ascontiguousarray(np.asarray(self.dihedrals, np.int32).reshape(-1, 5))

    @property
    def n(self):
        return len(self.type)

    def to_c(self, keep):
        t = abi.Topology()
        t.n_atoms = self.n
        for name in ("type", "bonds", "rigid", "angles", "dihedrals"):
            a = getattr(self, name)
            keep.append(a)
            setattr(t, name, abi.ptr(a, C.c_int))
        for name in ("charge", "x"):
            a = getattr(self, name)
            keep.append(a)
            setattr(t, name, abi.ptr(a))
        t.n_bonds, t.n_rigid = len(self.bonds), len(self.rigid)
        t.n_angles, t.n_dihedrals = len(self.angles), len(self.dihedrals)
        return t


@dataclass
class ReplicaSpec:
    atom_mass: np.ndarray
    atom_eps: np.ndarray
    atom_sigma: np.ndarray
    atom_name: List[str]
    bond_coeff: np.ndarray      # [nb,2]
    angle_coeff: np.ndarray     # [na,2] (theta0 in rad)
    dihedral_multi: np.ndarray  # [nd]
    dihedral_coeff: np.ndarray  # [nd,15]
    ion: Topology
    ion_v: np.ndarray
    ion_bmh_type: np.ndarray
    gas: Topology
    gas_kind: int
    gas_com_mass: float
    gas_mb_mass: float
    vapor: Topology
    vapor_com_mass: float
    vapor_mb_mass: float
    gas_x: np.ndarray
    gas_v: np.ndarray
    vapor_x: np.ndarray
    vapor_v: np.ndarray
    dt: float = 1.0
    temperature: float = 300.0
    box: float = 400.0
    cutoff: float = 20.0
    margin: float = 10.0
    r_inter: float = R_INTER
    overlap: float = OVERLAP
    interactions: int = 0
    nvt_mode: int = abi.NVT_OFF
    nvt_temperature: float = 300.0
    efield: tuple = (0.0, 0.0, 0.0)
    seed: int = 1
    pressure: float = 1e5
    label: str = ""
    # optional per-type-pair LJ parameters [nt, nt] (symmetric) used instead
    # of Lorentz-Berthelot mixing; None = mixing
    pair_eps: Optional[np.ndarray] = None
    pair_sigma: Optional[np.ndarray] = None

    def __post_init__(self):
        f64 = lambda a, s=None: np.ascontiguousarray(np.asarray(a, np.float64).reshape(s) if s else np.asarray(a, np.float64))
        self.atom_mass = f64(self.atom_mass)
        self.atom_eps = f64(self.atom_eps)
        self.atom_sigma = f64(self.atom_sigma)
        self.bond_coeff = f64(self.bond_coeff, (-1, 2))
        self.angle_coeff = f64(self.angle_coeff, (-1, 2))
        self.dihedral_multi = np.ascontiguousarray(self.dihedral_multi, np.int32)
        self.dihedral_coeff = f64(self.dihedral_coeff, (-1, 15))
        self.ion_v = f64(self.ion_v, (-1, 3))
        self.ion_bmh_type = np.ascontiguousarray(self.ion_bmh_type, np.int32)
        self.gas_x = f64(self.gas_x, (-1, 3))
        self.gas_v = f64(self.gas_v, (-1, 3))
        self.vapor_x = f64(self.vapor_x, (-1, 3))
        self.vapor_v = f64(self.vapor_v, (-1, 3))

    # ---- sizes ---------------------------------------------------------------
    @property
    def n_gas(self):
        return len(self.gas_x)

    @property
    def n_vapor(self):
        return len(self.vapor_x)

    @property
    def n_mol(self):
        return 1 + self.n_gas + self.n_vapor

    def to_desc(self):
        """Returns (desc, keepalive).  keepalive must outlive every use of desc."""
        keep = []
        d = abi.ReplicaDesc()
        d.n_atom_types = len(self.atom_mass)
        for name in ("atom_mass", "atom_eps", "atom_sigma", "bond_coeff", "angle_coeff",
                     "dihedral_coeff", "ion_v", "gas_x", "gas_v", "vapor_x", "vapor_v"):
            a = getattr(self, name)
            keep.append(a)
            setattr(d, name, abi.ptr(a))
        for name in ("dihedral_multi", "ion_bmh_type"):
            a = getattr(self, name)
            keep.append(a)
            setattr(d, name, abi.ptr(a, C.c_int))
        d.n_bond_types = len(self.bond_coeff)
        d.n_angle_types = len(self.angle_coeff)
        d.n_dihedral_types = len(self.dihedral_multi)
        d.ion = self.ion.to_c(keep)
        d.gas = self.gas.to_c(keep)
        d.vapor = self.vapor.to_c(keep)
        d.gas_kind = self.gas_kind
        d.gas_com_mass = self.gas_com_mass
        d.gas_mb_mass = self.gas_mb_mass
        d.vapor_com_mass = self.vapor_com_mass
        d.vapor_mb_mass = self.vapor_mb_mass
        d.n_gas = self.n_gas
        d.n_vapor = self.n_vapor
        for name in ("dt", "temperature", "box", "cutoff", "margin", "r_inter", "overlap",
                     "nvt_temperature"):
            setattr(d, name, float(getattr(self, name)))
        d.interactions = int(self.interactions)
        d.nvt_mode = int(self.nvt_mode)
        for k in range(3):
            d.efield[k] = float(self.efield[k])
        d.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        if self.pair_eps is not None or self.pair_sigma is not None:
            eps, sig = self.pair_parameters()
            keep += [eps, sig]
            d.pair_eps, d.pair_sigma = abi.ptr(eps), abi.ptr(sig)
        return d, keep

    def pair_parameters(self):
        """(eps, sigma) per type pair [nt, nt]: the overrides, else mixing."""
        eps = np.sqrt(np.outer(self.atom_eps, self.atom_eps))
        sig = 0.5 * (self.atom_sigma[:, None] + self.atom_sigma[None, :])
        if self.pair_eps is not None:
            eps = np.ascontiguousarray(self.pair_eps, np.float64)
        if self.pair_sigma is not None:
            sig = np.ascontiguousarray(self.pair_sigma, np.float64)
        return np.ascontiguousarray(eps), np.ascontiguousarray(sig)

    # ---- derived quantities ------------------------------------------------
    def lj_table(self):
        """Lorentz-Berthelot table {48 eps s^12, 24 eps s^6}
        (Variables::setCrossPotentials, src/initialization/setCrossPotential.cpp:4-23)."""
        eps = np.sqrt(np.outer(self.atom_eps, self.atom_eps))
        sig = 0.5 * (self.atom_sigma[:, None] + self.atom_sigma[None, :])
        return 48 * eps * sig ** 12, 24 * eps * sig ** 6


def descs(specs):
    """Packs a list of specs into a ctypes array; returns (array, keepalive)."""
    arr = (abi.ReplicaDesc * len(specs))()
    keep = []
    for i, s in enumerate(specs):
        d, k = s.to_desc()
        arr[i] = d
        keep.append(k)
    return arr, keep


def mb_mass_kg(mol_mass):
    """pp->mgas = Mgas/Nw/1000 (src/initialization/PhysicalProp.cpp:23-24)."""
    return mol_mass / NW / 1000.0


def mb_sigma(T, m_kg):
    """Width of one velocity component in A/fs: sqrt(kT/m) * 1e-5 (updateGasIn.cpp:16)."""
    return np.sqrt(KB * T / m_kg) * 1e-5


def box_from_pressure(n_gas, T, p):
    """d_size = (N k T / p)^(1/3) * 1e10 (src/initialization/setCondition.cpp:247)."""
    return (n_gas * KB * T / p) ** (1 / 3.0) * 1e10


class StateArrays:
    """Host buffers for one replica in the mdn_state layout."""

    def __init__(self, n_ion, a_g, a_v, n_gas, n_vap):
        nm = 1 + n_gas + n_vap
        z = lambda *s: np.zeros(s, np.float64)
        self.ion_x, self.ion_v, self.ion_f = z(n_ion, 3), z(n_ion, 3), z(n_ion, 3)
        self.mol_x, self.mol_v = z(nm, 3), z(nm, 3)
        self.region = np.zeros(nm, np.uint8)
        self.gas_ax, self.gas_av, self.gas_af = z(n_gas, a_g, 3), z(n_gas, a_g, 3), z(n_gas, a_g, 3)
        self.vap_ax, self.vap_av, self.vap_af = z(n_vap, a_v, 3), z(n_vap, a_v, 3), z(n_vap, a_v, 3)
        self.vap_w = z(n_vap, a_v)
        self.loop_pair = 0
        self.loop_update = 0
        self.zeta = 0.0
        self.margin_length = 0.0
        self.dims = (n_ion, a_g, a_v, n_gas, n_vap)

    @classmethod
    def for_spec(cls, s: ReplicaSpec):
        return cls(s.ion.n, s.gas.n, s.vapor.n, s.n_gas, s.n_vapor)

    _arrays = ("ion_x", "ion_v", "ion_f", "mol_x", "mol_v", "gas_ax", "gas_av", "gas_af",
               "vap_ax", "vap_av", "vap_af", "vap_w")

    def to_c(self):
        st = abi.State()
        for n in self._arrays:
            setattr(st, n, abi.ptr(getattr(self, n)))
        st.region = abi.ptr(self.region, C.c_ubyte)
        st.loop_pair = int(self.loop_pair)
        st.loop_update = int(self.loop_update)
        st.zeta = float(self.zeta)
        st.margin_length = float(self.margin_length)
        return st

    def pull_scalars(self, st):
        self.loop_pair, self.loop_update = st.loop_pair, st.loop_update
        self.zeta, self.margin_length = st.zeta, st.margin_length

    def copy(self):
        o = StateArrays(*self.dims)
        for n in self._arrays + ("region",):
            setattr(o, n, getattr(self, n).copy())
        o.pull_scalars(self)
        return o
