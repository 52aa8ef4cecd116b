"""Seeded synthetic systems of the shapes the benchmark configurations name.

Every system is generated from one integer seed (0x4D444E55 + 1000*config +
replica).  The species follow the reference's own gas table and file
conventions: type tables are ordered ion, gas, vapor; angles are stored in
radians; dihedral types hold three (K, n, d) terms as in readIonFile
(src/initialization/readIonFile.cpp:85-104).

  config 0  Na4Cl3(+1) cluster (Born-Mayer-Huggins), 20 methanol, 2,000 He,
            1e5 Pa, 300 K, dt 1 fs, SHAKE on X-H bonds
  config 1  150-atom +1 chain (AMBER), 100 methanol, 100,000 N2 (rigid), 1e5 Pa
  config 2  batched replicas: gas in {He, Ar, N2, N2mono} with 5k-100k
            molecules, vapor in {methanol, 3-site water} with 10-300
            molecules, seed in {NaCl cluster, chain of 50-300 atoms}; the gas
            pressure of each replica is solved so that the expected number of
            in-domain atoms is drawn log-uniform in 500-20,000
  config 4  1,000,000 N2, 1,000 rigid water, 500-atom +2 chain
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import abi
from .system import (GAS_TABLE, KB, NW, R_INTER, OVERLAP, ReplicaSpec, Topology,
                     box_from_pressure, mb_mass_kg, mb_sigma)

SEED_BASE = 0x4D444E55
V_SPHERE = 4.0 / 3.0 * math.pi * (R_INTER + OVERLAP) ** 3
DEG = math.pi / 180.0


def seed_of(config: int, replica: int = 0) -> int:
    return SEED_BASE + 1000 * config + replica


# --------------------------------------------------------------------------
# molecule kinds: each returns a "species" dict with local type tables
# --------------------------------------------------------------------------
@dataclass
class Species:
    names: List[str]
    mass: List[float]
    eps: List[float]
    sigma: List[float]
    top: Topology            # type indices local to this species
    bond_coeff: np.ndarray   # [nb,2]
    angle_coeff: np.ndarray  # [na,2]
    dih_multi: np.ndarray
    dih_coeff: np.ndarray    # [nd,15]
    h_types: tuple = ()      # local types that count as hydrogen for "SHAKE H"
    bmh: Optional[np.ndarray] = None


def _dih_row(terms):
    """Three (K, n, d_deg) terms -> readIonFile's 15-column row."""
    row = []
    for k in range(3):
        K, n, d = terms[k] if k < len(terms) else (0.0, 0.0, 0.0)
        row += [K, n, d, math.cos(d * DEG), math.sin(d * DEG)]
    return row


def _rotmat(rng):
    """Uniform random rotation (quaternion method)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a*a+b*b-c*c-d*d, 2*(b*c-a*d), 2*(b*d+a*c)],
                     [2*(b*c+a*d), a*a-b*b+c*c-d*d, 2*(c*d-a*b)],
                     [2*(b*d-a*c), 2*(c*d+a*b), a*a-b*b-c*c+d*d]])


def _perp(u, rng):
    """A unit vector perpendicular to u."""
    u = u / np.linalg.norm(u)
    for _ in range(100):
        w = np.cross(u, rng.normal(size=3))
        if np.linalg.norm(w) > 1e-3:
            return w / np.linalg.norm(w)
    raise RuntimeError("no perpendicular found")


def _angle(a, b, c):
    u, v = a - b, c - b
    return math.acos(np.clip(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v), -1, 1))


def methanol() -> Species:
    """C, O, HO, 3 HC: bonds 1.43/0.96/1.09 A, angles 108-109.5 deg, one C-O
    torsion of periodicity 3, charges C +0.145, O -0.683, HO +0.418, HC +0.04."""
    bC, bO, bH = 1.43, 0.96, 1.09
    C0 = np.zeros(3)
    O = np.array([bC, 0.0, 0.0])
    th = 108.5 * DEG
    HO = O + bO * np.array([-math.cos(th), math.sin(th), 0.0])
    hs = []
    for phi in (60.0, 180.0, 300.0):
        t, p = 109.5 * DEG, phi * DEG
        hs.append(C0 + bH * np.array([math.cos(t), math.sin(t) * math.cos(p),
                                      math.sin(t) * math.sin(p)]))
    x = np.array([C0, O, HO] + hs)
    x -= x.mean(axis=0)
    types = [0, 1, 2, 3, 3, 3]
    bonds = [[0, 1, 0], [1, 2, 1], [0, 3, 2], [0, 4, 2], [0, 5, 2]]
    angles = []
    ang_coeff = []
    def add_angle(i, j, k, K):
        angles.append([i, j, k, len(ang_coeff)])
        ang_coeff.append([K, _angle(x[i], x[j], x[k])])
    add_angle(0, 1, 2, 55.0)
    for h in (3, 4, 5):
        add_angle(h, 0, 1, 50.0)
    add_angle(3, 0, 4, 35.0)
    add_angle(3, 0, 5, 35.0)
    add_angle(4, 0, 5, 35.0)
    dihedrals = [[3, 0, 1, 2, 0], [4, 0, 1, 2, 0], [5, 0, 1, 2, 0]]
    return Species(
        names=["C", "O", "HO", "HC"], mass=[12.011, 15.999, 1.008, 1.008],
        eps=[0.066, 0.170, 0.010, 0.030], sigma=[3.50, 3.12, 1.00, 2.50],
        top=Topology(type=types, charge=[0.145, -0.683, 0.418, 0.04, 0.04, 0.04], x=x,
                     bonds=bonds, angles=angles, dihedrals=dihedrals),
        bond_coeff=np.array([[320.0, bC], [553.0, bO], [340.0, bH]]),
        angle_coeff=np.array(ang_coeff),
        dih_multi=np.array([1], np.int32), dih_coeff=np.array([_dih_row([(0.18, 3, 0.0)])]),
        h_types=(2, 3))


def water() -> Species:
    """3-site water, O -0.834 e, H +0.417 e (TIP3P geometry); the O-H and H-H
    distances are bonds so that "SHAKE H" makes the molecule rigid."""
    r, th = 0.9572, 104.52 * DEG
    O = np.zeros(3)
    H1 = r * np.array([math.sin(th / 2), math.cos(th / 2), 0.0])
    H2 = r * np.array([-math.sin(th / 2), math.cos(th / 2), 0.0])
    x = np.array([O, H1, H2])
    x -= x.mean(axis=0)
    hh = float(np.linalg.norm(H1 - H2))
    return Species(
        names=["OW", "HW"], mass=[15.999, 1.008], eps=[0.1521, 0.010], sigma=[3.1507, 1.0],
        top=Topology(type=[0, 1, 1], charge=[-0.834, 0.417, 0.417], x=x,
                     bonds=[[0, 1, 0], [0, 2, 0], [1, 2, 1]], angles=[[1, 0, 2, 0]]),
        bond_coeff=np.array([[450.0, r], [0.0, hh]]),
        angle_coeff=np.array([[55.0, th]]),
        dih_multi=np.zeros(0, np.int32), dih_coeff=np.zeros((0, 15)),
        h_types=(1,))


def nacl_cluster() -> Species:
    """Na4Cl3(+1): a 2x2x2 rock-salt cube (a = 2.82 A) missing one Cl corner.
    Types: 0 = Na, 1 = Cl, which are also the Born-Mayer-Huggins rows."""
    a = 2.82
    xs, ts = [], []
    for i in (0, 1):
        for j in (0, 1):
            for k in (0, 1):
                if (i + j + k) % 2 == 0:
                    xs.append([i * a, j * a, k * a]); ts.append(0)
                elif (i, j, k) != (1, 1, 1):
                    xs.append([i * a, j * a, k * a]); ts.append(1)
    x = np.array(xs, float)
    q = [1.0 if t == 0 else -1.0 for t in ts]
    return Species(
        names=["Na", "Cl"], mass=[22.99, 35.45], eps=[0.10, 0.10], sigma=[2.35, 4.40],
        top=Topology(type=ts, charge=q, x=x),
        bond_coeff=np.zeros((0, 2)), angle_coeff=np.zeros((0, 2)),
        dih_multi=np.zeros(0, np.int32), dih_coeff=np.zeros((0, 15)),
        bmh=np.array(ts, np.int32))


def chain(n_atoms: int, charge: float, rng: np.random.Generator) -> Species:
    """A +q peptide-like chain: a self-avoiding heavy-atom backbone (bonds
    1.33-1.53 A, angles 110-120 deg, torsions of periodicity 1-3 with barriers
    0-2 kcal/mol) carrying hydrogens at 1.0-1.09 A; heavy-atom charges
    N(0, 0.3 e) shifted to the net charge, hydrogen charges |N(0.1, 0.04)| e
    (small and positive, so that no H-H pair attracts through the soft H core);
    LJ sigma 2.5-3.5 A, eps 0.02-0.2 (H: 2.5 A, 0.03).  Heavy atoms are
    tetravalent: two hydrogens on each interior atom, up to three on each
    end, placed at tetrahedral angles (the ends' cones turned for the largest
    clearance), so that no H-X-X equilibrium angle nears 180 deg, where the
    torsions through the hydrogen are singular.  A geometry is kept only if
    every pair outside the AMBER exclusions (1-2, 1-3, 1-4) is at least
    0.7 sigma apart."""
    n_heavy = max(3, n_atoms // 3)
    n_h = n_atoms - n_heavy
    n_heavy_types = 6
    # tetravalent heavy atoms: two hydrogens on each interior atom, the
    # remainder (at most three each) on the two chain ends
    if n_h > 2 * n_heavy + 2:
        raise ValueError(f"{n_atoms} atoms need more hydrogens than {n_heavy} heavy atoms carry")
    per = np.zeros(n_heavy, np.int64)
    left = n_h
    for i in [0, n_heavy - 1] + list(range(1, n_heavy - 1)):
        per[i] = min(left, 2)
        left -= per[i]
    for i in (0, n_heavy - 1):
        take = min(left, 1)
        per[i] += take
        left -= take
    hpar = [i for i in range(n_heavy) for _ in range(per[i])]
    mass = list(rng.choice([12.011, 14.007, 15.999], n_heavy_types)) + [1.008]
    eps = list(rng.uniform(0.02, 0.2, n_heavy_types)) + [0.03]
    sigma = list(rng.uniform(2.5, 3.5, n_heavy_types)) + [2.5]
    types = list(rng.integers(0, n_heavy_types, n_heavy)) + [n_heavy_types] * n_h
    sig = np.array([sigma[t] for t in types])
    n = n_heavy + n_h
    hs_of = [[] for _ in range(n_heavy)]
    for h, p_ in enumerate(hpar):
        hs_of[p_].append(n_heavy + h)
    # topology (independent of the geometry)
    bonds = [(i, i + 1) for i in range(n_heavy - 1)] + [(p_, n_heavy + h) for h, p_ in enumerate(hpar)]
    angles = [(i - 1, i, i + 1) for i in range(1, n_heavy - 1)]
    for i in range(n_heavy):
        for hh in hs_of[i]:
            for j in (i - 1, i + 1):
                if 0 <= j < n_heavy:
                    angles.append((hh, i, j))
        for a in range(len(hs_of[i])):
            for b in range(a + 1, len(hs_of[i])):
                angles.append((hs_of[i][a], i, hs_of[i][b]))
    dihed = [(i, i + 1, i + 2, i + 3) for i in range(n_heavy - 3)]
    hdih = []
    for i in range(n_heavy):
        for hh in hs_of[i]:
            if i + 2 < n_heavy:
                hdih.append((hh, i, i + 1, i + 2))
            if i - 2 >= 0:
                hdih.append((hh, i, i - 1, i - 2))
            if i + 1 < n_heavy:
                for h2 in hs_of[i + 1]:
                    hdih.append((hh, i, i + 1, h2))
    excl = set()
    for a, b in bonds:
        excl.add((min(a, b), max(a, b)))
    for a, _, c in angles:
        excl.add((min(a, c), max(a, c)))
    for a, _, _, d in dihed + hdih:
        excl.add((min(a, d), max(a, d)))

    def clearance_ok(xs):
        d = np.linalg.norm(xs[:, None] - xs[None], axis=2)
        lim = 0.7 * 0.5 * (sig[:, None] + sig[None, :])
        bad = d < lim
        for (a, b) in excl:
            bad[a, b] = bad[b, a] = False
        np.fill_diagonal(bad, False)
        return not bad.any()

    for _attempt in range(800):
        # heavy atoms three or more bonds apart stay 3.6 A apart; after 400
        # failed attempts (long chains, whose near-trans walks jam) the 1-4
        # neighbours, excluded from the non-bonded terms anyway, only need
        # 3.0 A (gauche or trans, not cis)
        skip = 2 if _attempt < 400 else 3
        bb = [np.zeros(3)]
        bl = rng.uniform(1.33, 1.53, n_heavy)
        ok = True
        for i in range(1, n_heavy):
            for _try in range(200):
                if i == 1:
                    d = rng.normal(size=3)
                    d /= np.linalg.norm(d)
                else:
                    prev = bb[-1] - bb[-2]
                    prev /= np.linalg.norm(prev)
                    th = rng.uniform(110, 120) * DEG
                    perp = _perp(prev, rng)
                    d = math.cos(math.pi - th) * prev + math.sin(math.pi - th) * perp
                cand = bb[-1] + bl[i] * d
                if all(np.linalg.norm(cand - p_) > 3.6 for p_ in bb[:-skip]) and (
                        skip == 2 or len(bb) < 3 or np.linalg.norm(cand - bb[-3]) > 3.0):
                    bb.append(cand)
                    break
            else:
                ok = False
                break
        if not ok:
            continue
        bb = np.array(bb)
        xs = np.zeros((n, 3))
        xs[:n_heavy] = bb
        for i in range(n_heavy):
            if not hs_of[i]:
                continue
            nb = [j for j in (i - 1, i + 1) if 0 <= j < n_heavy]
            u = -sum((bb[j] - bb[i]) / np.linalg.norm(bb[j] - bb[i]) for j in nb)
            u /= np.linalg.norm(u)
            nh = len(hs_of[i])
            others = np.concatenate([bb[[j for j in range(n_heavy) if abs(j - i) > 1]],
                                     xs[n_heavy:][[h for h in range(n_h) if hpar[h] < i]]])
            if len(nb) == 2:
                # interior atom: the hydrogens in the plane through the
                # bisector u normal to the backbone plane, 109.5 deg apart
                # (one hydrogen: along u), so every H-X-X angle is near
                # tetrahedral and none approaches 180 deg, where the torsions
                # through the hydrogen become singular
                n_pl = np.cross(bb[nb[0]] - bb[i], bb[nb[1]] - bb[i])
                n_pl /= np.linalg.norm(n_pl)
                if nh == 1:
                    dirs = [u]
                else:
                    a = 0.5 * 109.47 * DEG
                    dirs = [math.cos(a) * u + math.sin(a) * n_pl, math.cos(a) * u - math.sin(a) * n_pl]
                best_pos = np.array([bb[i] + 1.045 * d for d in dirs])
            else:
                # chain end: a cone at 109.5 deg from the one backbone bond,
                # turned about it for the largest clearance
                w0 = _perp(u, rng)
                best, best_pos = -1.0, None
                for k in range(24):
                    phi = 2 * math.pi * k / 24
                    pos = []
                    for hidx in range(nh):
                        ang = phi + 2 * math.pi * hidx / 3  # tetrahedral sites
                        v = w0 * math.cos(ang) + np.cross(u, w0) * math.sin(ang)
                        dirn = math.cos(70.53 * DEG) * u + math.sin(70.53 * DEG) * v
                        pos.append(bb[i] + 1.045 * dirn)
                    pos = np.array(pos)
                    m = np.linalg.norm(pos[:, None] - others[None], axis=2).min() if len(others) else 9.0
                    if m > best:
                        best, best_pos = m, pos
            for hidx, hh in enumerate(hs_of[i]):
                xs[hh] = best_pos[hidx]
        for h in range(n_h):  # bond lengths 1.0-1.09 A
            p_ = hpar[h]
            dv = xs[n_heavy + h] - xs[p_]
            xs[n_heavy + h] = xs[p_] + dv / np.linalg.norm(dv) * rng.uniform(1.0, 1.09)
        if clearance_ok(xs):
            break
    else:
        raise RuntimeError("could not grow a clash-free chain")
    # bonded parameters: one type per term, equilibrium values from the geometry
    bond_rows, bond_coeff = [], []
    for (i, j) in bonds:
        K = rng.uniform(250, 400) if j < n_heavy else 340.0
        bond_rows.append([i, j, len(bond_coeff)])
        bond_coeff.append([K, float(np.linalg.norm(xs[i] - xs[j]))])
    angle_rows, angle_coeff = [], []
    for (i, j, k) in angles:
        K = rng.uniform(40, 70) if (i < n_heavy and k < n_heavy) else (35.0 if (i >= n_heavy and k >= n_heavy) else 50.0)
        angle_rows.append([i, j, k, len(angle_coeff)])
        angle_coeff.append([K, _angle(xs[i], xs[j], xs[k])])
    dih_rows, dih_multi, dih_coeff = [], [], []
    for t in dihed:
        nt = int(rng.integers(1, 3))
        terms = [(rng.uniform(0, 2), int(rng.integers(1, 4)), float(rng.choice([0.0, 180.0]))) for _ in range(nt)]
        dih_rows.append(list(t) + [len(dih_multi)])
        dih_multi.append(nt)
        dih_coeff.append(_dih_row(terms))
    for t in hdih:
        dih_rows.append(list(t) + [len(dih_multi)])
        dih_multi.append(1)
        dih_coeff.append(_dih_row([(rng.uniform(0, 0.3), 3, 0.0)]))
    q = np.concatenate([rng.normal(0, 0.3, n_heavy), np.abs(rng.normal(0.1, 0.04, n_h))])
    q[:n_heavy] += (charge - q.sum()) / n_heavy
    xs = xs - xs.mean(axis=0)
    return Species(
        names=[f"X{k}" for k in range(n_heavy_types)] + ["H"],
        mass=mass, eps=eps, sigma=sigma,
        top=Topology(type=types, charge=q, x=xs, bonds=bond_rows, angles=angle_rows, dihedrals=dih_rows),
        bond_coeff=np.array(bond_coeff), angle_coeff=np.array(angle_coeff),
        dih_multi=np.array(dih_multi, np.int32), dih_coeff=np.array(dih_coeff),
        h_types=(n_heavy_types,))


def gas_species(name: str, rigid: bool = False) -> Species:
    g = GAS_TABLE[name]
    na = len(g["x"])
    bonds = [[0, 1, 0]] if g["bond"] else []
    return Species(names=[name], mass=[g["mass"]], eps=[g["eps"]], sigma=[g["sigma"]],
                   top=Topology(type=[0] * na, charge=[0.0] * na, x=g["x"],
                                bonds=[] if rigid else bonds, rigid=bonds if rigid else []),
                   bond_coeff=np.array([g["bond"]]) if g["bond"] else np.zeros((0, 2)),
                   angle_coeff=np.zeros((0, 2)), dih_multi=np.zeros(0, np.int32),
                   dih_coeff=np.zeros((0, 15)))


def _split_rigid(sp: Species, shake_h: bool):
    """readIonFile/readVaporFile: with "SHAKE H", bonds touching an H type go to
    rigid_pairs (src/initialization/readIonFile.cpp:131-137)."""
    if not shake_h or len(sp.top.bonds) == 0:
        return sp.top.bonds, sp.top.rigid
    keep, rig = [], list(sp.top.rigid)
    for b in sp.top.bonds:
        if sp.top.type[b[0]] in sp.h_types or sp.top.type[b[1]] in sp.h_types:
            rig.append(b)
        else:
            keep.append(b)
    return np.array(keep, np.int32).reshape(-1, 3), np.array(rig, np.int32).reshape(-1, 3)


# --------------------------------------------------------------------------
# assembling a replica
# --------------------------------------------------------------------------
def assemble(ion: Species, gas: Species, vap: Species, *, gas_name: str, n_gas: int,
             n_vap: int, T: float, p: float, dt: float, interactions: int, seed: int,
             shake_h: bool, rng: np.random.Generator, nvt_mode=abi.NVT_OFF,
             min_dist: float = 10.0, box: Optional[float] = None, label: str = "",
             reference_masses: bool = False, placer=None, gas_min_dist: float = 0.0) -> ReplicaSpec:
    """Concatenates the species' tables (ion, gas, vapor order), places the
    molecules uniformly in the cube and draws Maxwell-Boltzmann velocities.

    The gas molecule's COM mass is the sum of its atoms' masses, so that the
    centre-of-mass bookkeeping and the atom masses agree.  reference_masses=True
    takes the reference's molecular mass instead (src/constants.hpp:34,
    used by src/initialization/initializationGas.cpp:61): 4.0026 for He, whose
    atom is 4.027, and 39.948 for Ar, whose atom is 28.02
    (src/initialization/setCondition.cpp:50,104); the argon centre of mass
    then moves 30% off its atom.

    placer, when given, replaces the placement and the molecules' velocities:
    placer(box, ion_x, n_gas, n_vap, gas_sigma, vapor_sigma, seed) returns
    (gas_x, gas_v, vapor_x, vapor_v), e.g. engine.place (mdn_place on the GPU,
    the reference's placement rule)."""
    offs_t, offs_b, offs_a, offs_d = [0], [0], [0], [0]
    mass, eps, sig, names = [], [], [], []
    bc, ac, dm, dc = [], [], [], []
    tops = []
    for sp in (ion, gas, vap):
        t0, b0, a0, d0 = len(mass), len(bc), len(ac), len(dm)
        mass += list(sp.mass); eps += list(sp.eps); sig += list(sp.sigma); names += list(sp.names)
        bc += [list(r) for r in sp.bond_coeff]; ac += [list(r) for r in sp.angle_coeff]
        dm += list(sp.dih_multi); dc += [list(r) for r in sp.dih_coeff]
        bonds, rigid = _split_rigid(sp, shake_h)
        top = Topology(type=np.asarray(sp.top.type) + t0, charge=sp.top.charge, x=sp.top.x,
                       bonds=_shift(bonds, 3, 2, b0), rigid=_shift(rigid, 3, 2, b0),
                       angles=_shift(sp.top.angles, 4, 3, a0),
                       dihedrals=_shift(sp.top.dihedrals, 5, 4, d0))
        tops.append(top)
    ion_top, gas_top, vap_top = tops
    if box is None:
        box = box_from_pressure(n_gas, T, p)
    # ion: uniform random orientation, MB velocities per atom
    R = _rotmat(rng)
    ion_top.x = np.ascontiguousarray(ion_top.x @ R.T)
    m_ion = np.array([mass[t] for t in ion_top.type])
    ion_v = rng.normal(size=(ion_top.n, 3)) * mb_sigma(T, m_ion[:, None] * 1e-3 / NW)
    # vapor then gas centres, uniform in the cube, kept min_dist from the ion
    # atoms and from the vapor already placed
    half = box / 2
    ion_r = np.linalg.norm(ion_top.x, axis=1).max() if ion_top.n else 0.0
    if not np.all(np.isfinite(ion_top.x)):
        raise RuntimeError("non-finite ion coordinates")
    g = GAS_TABLE[gas_name]
    gas_com = g["mol_mass"] if reference_masses else float(sum(mass[t] for t in gas_top.type))
    gas_m = mb_mass_kg(gas_com)
    vap_com = float(sum(mass[t] for t in vap_top.type))
    vap_m = mb_mass_kg(vap_com)
    if placer is not None:
        gx, gv, vx, vv = placer(box, ion_top.x, n_gas, n_vap, mb_sigma(T, gas_m), mb_sigma(T, vap_m), seed)
    else:
        gx, gv, vx, vv = _place(rng, box, ion_top.x, n_gas, n_vap, min_dist, gas_min_dist, mb_sigma(T, gas_m),
                                mb_sigma(T, vap_m))
    bmh = ion.bmh if ion.bmh is not None else np.zeros(ion_top.n, np.int32)
    return ReplicaSpec(
        atom_mass=mass, atom_eps=eps, atom_sigma=sig, atom_name=names,
        bond_coeff=np.array(bc).reshape(-1, 2), angle_coeff=np.array(ac).reshape(-1, 2),
        dihedral_multi=np.array(dm, np.int32), dihedral_coeff=np.array(dc).reshape(-1, 15),
        ion=ion_top, ion_v=ion_v, ion_bmh_type=bmh,
        gas=gas_top, gas_kind=g["kind"], gas_com_mass=gas_com, gas_mb_mass=gas_m,
        vapor=vap_top, vapor_com_mass=vap_com, vapor_mb_mass=vap_m,
        gas_x=gx, gas_v=gv, vapor_x=vx, vapor_v=vv,
        dt=dt, temperature=T, box=box, interactions=interactions, nvt_mode=nvt_mode,
        seed=seed, pressure=p, label=label)


def _place(rng, box, ion_x, n_gas, n_vap, min_dist, gas_min_dist, gas_sigma, vap_sigma):
    """Centres uniform in the cube: vapor first, each min_dist from the ion
    atoms' bounding sphere and from the vapor already placed, then the gas
    (min_dist from the ion and the vapor, and gas_min_dist from each other
    when it is positive: systems with the gas-gas term need it);
    Maxwell-Boltzmann velocities."""
    half = box / 2
    ion_r = np.linalg.norm(ion_x, axis=1).max() if len(ion_x) else 0.0
    vx = []
    tries = 0
    while len(vx) < n_vap:
        tries += 1
        if tries > 1000 * (n_vap + 10):
            raise RuntimeError("vapor placement did not converge")
        c = rng.uniform(-half, half, 3)
        if np.linalg.norm(c) < ion_r + min_dist:
            continue
        if vx and np.min(np.linalg.norm(np.array(vx) - c, axis=1)) < min_dist:
            continue
        vx.append(c)
    vx = np.array(vx).reshape(-1, 3)
    gx = np.empty((0, 3))
    rounds = 0
    while len(gx) < n_gas:
        rounds += 1
        if rounds > 200:
            raise RuntimeError("gas placement did not converge")
        c = rng.uniform(-half, half, (2 * (n_gas - len(gx)) + 16, 3))
        ok = np.linalg.norm(c, axis=1) >= ion_r + min_dist
        if len(vx):
            for b in range(0, len(c), 4096):
                d = np.linalg.norm(c[b:b + 4096, None, :] - vx[None], axis=2).min(axis=1)
                ok[b:b + 4096] &= d >= min_dist
        c = c[ok]
        if gas_min_dist > 0:
            c = _thin(c, gx, gas_min_dist, box)
        gx = np.concatenate([gx, c])[:n_gas]
    gv = rng.normal(size=(n_gas, 3)) * gas_sigma
    vv = rng.normal(size=(n_vap, 3)) * vap_sigma
    return gx, gv, vx, vv


def _shift(arr, width, col, off):
    a = np.array(arr, np.int32).reshape(-1, width).copy()
    if len(a):
        a[:, col] += off
    return a


BASE_TERMS = abi.I_GI | abi.I_GV | abi.I_VI | abi.I_VV | abi.I_GAS_INTRA | abi.I_VAPOR_INTRA


def _thin(cand, placed, d, box):
    """The candidates, in order, that lie at least d from every placed centre
    and every earlier kept candidate (minimum image in the periodic cube)."""
    cells = {}
    n = max(1, int(box // d))
    w = box / n

    def key(p):
        return tuple(int(np.floor((p[k] + box / 2) / w)) % n for k in range(3))

    def clear(p):
        kx, ky, kz = key(p)
        for i in (-1, 0, 1):
            for j in (-1, 0, 1):
                for k in (-1, 0, 1):
                    for q in cells.get(((kx + i) % n, (ky + j) % n, (kz + k) % n), ()):
                        dv = p - q
                        dv -= box * np.round(dv / box)
                        if dv @ dv < d * d:
                            return False
        return True

    for p in placed:
        cells.setdefault(key(p), []).append(p)
    keep = []
    for p in cand:
        if clear(p):
            cells.setdefault(key(p), []).append(p)
            keep.append(p)
    return np.array(keep).reshape(-1, 3)


def config0(replica: int = 0, n_gas: int = 2000, n_vap: int = 20) -> ReplicaSpec:
    rng = np.random.default_rng(seed_of(0, replica))
    return assemble(nacl_cluster(), gas_species("He"), methanol(), gas_name="He", n_gas=n_gas,
                    n_vap=n_vap, T=300.0, p=1e5, dt=1.0,
                    interactions=BASE_TERMS | abi.I_BMH | abi.I_SHAKE,
                    seed=seed_of(0, replica), shake_h=True, rng=rng, label="config0")


def config1(replica: int = 0, n_gas: int = 100_000, n_vap: int = 100, chain_atoms: int = 150,
            rigid_n2: bool = True) -> ReplicaSpec:
    rng = np.random.default_rng(seed_of(1, replica))
    ion = chain(chain_atoms, 1.0, rng)
    return assemble(ion, gas_species("N2", rigid=rigid_n2), methanol(), gas_name="N2",
                    n_gas=n_gas, n_vap=n_vap, T=300.0, p=1e5, dt=1.0,
                    interactions=BASE_TERMS | abi.I_AMBER | abi.I_SHAKE,
                    seed=seed_of(1, replica), shake_h=True, rng=rng, label="config1")


def config3(replica: int = 0, n_near: int = 8, r_lo: float = 8.0, r_hi: float = 28.0, margin: float = 40.0,
            **kw) -> ReplicaSpec:
    """The adjoint window's system: configuration 1 with n_near of its
    methanol molecules moved to centres r_lo..r_hi A from the chain's
    centre (each at least 6 A from every chain atom and 8 A from each other),
    so that the window's ion-vapor energy and smooth count are not
    identically zero (at 1e5 Pa and 100 molecules in the 1,606 A box the
    domain holds 0.13 methanol on average).  The list margin is raised so
    that the window holds no effective-domain rebuild."""
    spec = config1(replica, **kw)
    rng = np.random.default_rng(seed_of(3, replica))
    ion_x = spec.ion.x
    placed = []
    tries = 0
    while len(placed) < n_near:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place the near methanol")
        d = rng.normal(size=3)
        c = d / np.linalg.norm(d) * rng.uniform(r_lo, r_hi)
        if np.linalg.norm(ion_x - c, axis=1).min() < 6.0:
            continue
        if placed and np.linalg.norm(np.array(placed) - c, axis=1).min() < 8.0:
            continue
        placed.append(c)
    spec.vapor_x[:n_near] = np.array(placed)
    spec.margin = margin
    spec.label = "config3"
    return spec


def config2_replica(replica: int, scale: float = 1.0) -> ReplicaSpec:
    """One replica of the batched configuration.  scale < 1 shrinks the
    molecule counts (tests use it); the density stays what the draw gives."""
    seed = seed_of(2, replica)
    rng = np.random.default_rng(seed)
    gas_name = ["He", "Ar", "N2", "N2monoatomic"][int(rng.integers(0, 4))]
    n_gas = int(round(math.exp(rng.uniform(math.log(5000), math.log(100_000))) * scale))
    use_water = bool(rng.integers(0, 2))
    n_vap = max(1, int(round(rng.uniform(10, 300) * scale)))
    target = math.exp(rng.uniform(math.log(500), math.log(20_000))) * scale
    if rng.integers(0, 2) == 0:
        ion = nacl_cluster()
        terms = BASE_TERMS | abi.I_BMH
    else:
        ion = chain(int(rng.integers(50, 301)), 1.0, rng)
        terms = BASE_TERMS | abi.I_AMBER
    vap = water() if use_water else methanol()
    gas = gas_species(gas_name)
    a_g = gas.top.n
    T = 300.0
    # in-domain gas molecules wanted -> number density -> box and pressure
    gas_atoms_in = max(target - ion.top.n, 50.0)
    n_dens = gas_atoms_in / a_g / V_SPHERE
    box = (n_gas / n_dens) ** (1 / 3)
    min_box = 2.2 * (R_INTER + OVERLAP)
    if box < min_box:  # keep the sphere inside the periodic cell
        n_gas = int(math.ceil(n_dens * min_box ** 3))
        box = (n_gas / n_dens) ** (1 / 3)
    p = n_dens * 1e30 * KB * T
    spacing = n_dens ** (-1 / 3)
    return assemble(ion, gas, vap, gas_name=gas_name, n_gas=n_gas, n_vap=n_vap, T=T, p=p,
                    dt=1.0, interactions=terms | abi.I_SHAKE, seed=seed, shake_h=True, rng=rng,
                    min_dist=min(10.0, 0.5 * spacing), box=box, label=f"config2[{replica}]")


def config2(n_replicas: int = 256, scale: float = 1.0) -> List[ReplicaSpec]:
    return [config2_replica(r, scale) for r in range(n_replicas)]


def config4_replica(replica: int = 0, n_gas: int = 1_000_000, n_vap: int = 1000, placer=None) -> ReplicaSpec:
    """placer: see assemble (the numpy placement of 1,000,000 molecules takes
    about 100 s; mdn_place does it in milliseconds)."""
    rng = np.random.default_rng(seed_of(4, replica))
    ion = chain(500, 2.0, rng)
    return assemble(ion, gas_species("N2"), water(), gas_name="N2", n_gas=n_gas, n_vap=n_vap,
                    T=300.0, p=1e5, dt=1.0,
                    interactions=BASE_TERMS | abi.I_AMBER | abi.I_SHAKE,
                    seed=seed_of(4, replica), shake_h=True, rng=rng, label="config4", placer=placer)


def small_system(seed: int = 7, gas: str = "N2", vapor: str = "methanol", ion: str = "nacl",
                 n_gas: int = 400, n_vap: int = 12, box: float = 260.0, interactions=None,
                 shake_h: bool = False, rigid_gas: bool = False, chain_atoms: int = 30,
                 nvt_mode=abi.NVT_OFF, dt: float = 1.0, gas_min_dist: float = 0.0) -> ReplicaSpec:
    """A small replica for parity tests: a dense gas in a small box so that
    the sphere holds many molecules (gas centres gas_min_dist apart when it
    is positive)."""
    rng = np.random.default_rng(seed)
    ion_sp = nacl_cluster() if ion == "nacl" else chain(chain_atoms, 1.0, rng)
    vap_sp = methanol() if vapor == "methanol" else water()
    if interactions is None:
        interactions = BASE_TERMS | (abi.I_BMH if ion == "nacl" else abi.I_AMBER)
        if shake_h:
            interactions |= abi.I_SHAKE
    n_dens = n_gas / box ** 3
    p = n_dens * 1e30 * KB * 300.0
    return assemble(ion_sp, gas_species(gas, rigid=rigid_gas), vap_sp, gas_name=gas,
                    n_gas=n_gas, n_vap=n_vap, T=300.0, p=p, dt=dt, interactions=interactions,
                    seed=seed, shake_h=shake_h, rng=rng, nvt_mode=nvt_mode,
                    min_dist=min(10.0, 0.5 * n_dens ** (-1 / 3)), box=box, label="small",
                    gas_min_dist=gas_min_dist)


# --------------------------------------------------------------------------
# input files in the reference's own format
# --------------------------------------------------------------------------
# type codes the reference's readers turn back into element names
# (src/initialization/readIonFile.cpp:49-67): C, N, O, H; Na stays "Na",
# "cl" becomes "Cl"
_CODE_BY_MASS = {12.011: "#c3", 14.007: "#n3", 15.999: "#os", 1.008: "#hc", 22.99: "Na", 35.45: "cl"}
_CODE_BY_NAME = {"Na": "Na", "Cl": "cl", "OW": "#ow", "O": "#oh", "HO": "#ho", "HW": "#hw", "HC": "#hc",
                 "H": "#hc", "C": "#c3", "N": "#n3"}


def _type_code(sp: Species, t: int) -> str:
    name = sp.names[t]
    if name in _CODE_BY_NAME:
        return _CODE_BY_NAME[name]
    if t in sp.h_types:
        return "#hc"
    return _CODE_BY_MASS.get(round(float(sp.mass[t]), 3), name)


def write_molecule_file(path: str, sp: Species) -> None:
    """One ion or vapor file as Variables::readIonFile / readVaporFile read
    it (src/initialization/readIonFile.cpp:30-156): tab-separated sections,
    1-based indices.  Angles are written in degrees."""
    f = repr
    out = ["atom type"]
    for t in range(len(sp.names)):
        out.append(f"{t + 1}\t{_type_code(sp, t)}\t{f(float(sp.mass[t]))}\t{f(float(sp.eps[t]))}\t"
                   f"{f(float(sp.sigma[t]))}")
    if len(sp.bond_coeff):
        out += ["", "bond type"]
        for b, (K, r0) in enumerate(np.asarray(sp.bond_coeff, float)):
            out.append(f"{b + 1}\tb{b + 1}\t{f(float(K))}\t{f(float(r0))}")
    if len(sp.angle_coeff):
        out += ["", "angle type"]
        for a, (K, th) in enumerate(np.asarray(sp.angle_coeff, float)):
            out.append(f"{a + 1}\ta{a + 1}\t{f(float(K))}\t{f(float(th) * 180.0 / math.pi)}")
    if len(sp.dih_multi):
        out += ["", "dihedral type"]
        for d, (m, row) in enumerate(zip(np.asarray(sp.dih_multi), np.asarray(sp.dih_coeff, float))):
            terms = "\t".join(f"{f(float(row[5 * k]))}\t{f(float(row[5 * k + 1]))}\t{f(float(row[5 * k + 2]))}"
                              for k in range(3))
            out.append(f"{d + 1}\td{d + 1}\t{int(m)}\t{terms}")
    top = sp.top
    out += ["", "atoms"]
    x = np.asarray(top.x, float).reshape(-1, 3)
    for i in range(top.n):
        out.append(f"{i + 1}\t{int(top.type[i]) + 1}\t{f(float(top.charge[i]))}\t"
                   f"{f(float(x[i, 0]))}\t{f(float(x[i, 1]))}\t{f(float(x[i, 2]))}")
    bonds = [list(b) for b in np.asarray(top.bonds, int).reshape(-1, 3)]
    bonds += [list(b) for b in np.asarray(top.rigid, int).reshape(-1, 3)]
    if bonds:
        out += ["", "bonds"]
        out += [f"{i + 1}\t{j + 1}\t{t + 1}" for i, j, t in bonds]
    ang = np.asarray(top.angles, int).reshape(-1, 4)
    if len(ang):
        out += ["", "angles"]
        out += [f"{i + 1}\t{j + 1}\t{k + 1}\t{t + 1}" for i, j, k, t in ang]
    dih = np.asarray(top.dihedrals, int).reshape(-1, 5)
    if len(dih):
        out += ["", "dihedrals"]
        out += [f"{i + 1}\t{j + 1}\t{k + 1}\t{l + 1}\t{t + 1}" for i, j, k, l, t in dih]
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def write_reference_inputs(directory: str, ion: Species, vapor: Species, *, gas: str, n_gas: int, n_vapor: int,
                           T: float = 300.0, p: float = 1e5, dt: float = 1.0, total_steps: int = 1000,
                           relax_steps: int = 0, observe: int = 100, interactions: int = 0,
                           shake_h: bool = False, nvt: str = "OFF", output: str = "dump",
                           efield=None) -> str:
    """Writes ion.txt, vapor.txt and cond.txt under `directory` in the
    reference's formats (MD::readCondFile, src/initialization/setCondition.cpp:4-254)
    and returns the condition file's path.  `interactions` takes MDN_I_* bits
    (gi, gv, vi, vv, gg, AMBER or BMH for the ion); nvt is "OFF", "scale" or a
    temperature."""
    os.makedirs(directory, exist_ok=True)
    ion_path = os.path.join(directory, "ion.txt")
    vap_path = os.path.join(directory, "vapor.txt")
    write_molecule_file(ion_path, ion)
    write_molecule_file(vap_path, vapor)
    I = interactions
    lines = [f"Input {ion_path}", f"Vapor {vap_path} {n_vapor}", f"Gas {gas} {n_gas}",
             f"Temperature {T!r}", f"Pressure {p!r}", f"dt {dt!r}", f"TotalSteps {total_steps}",
             f"RelaxSteps {relax_steps}", f"Output {os.path.join(directory, output)} {observe}",
             f"NVTion {nvt}"]
    if shake_h:
        lines.append("SHAKE H")
    lines.append("Interactions")
    if I & abi.I_AMBER:
        lines.append(" ion AMBER")
    if I & abi.I_BMH:
        lines.append(" ion Born-Mayer-Huggins-NaCl")
    lines.append(f" gg {'LJ' if I & abi.I_GG else 'OFF'}")
    lines.append(f" gi {'LJ' if I & abi.I_GI else 'OFF'}")
    lines.append(f" vi {'LJcoul' if I & abi.I_VI else 'OFF'}")
    lines.append(f" vv {'LJcoul' if I & abi.I_VV else 'OFF'}")
    lines.append(f" gv {'LJ' if I & abi.I_GV else 'OFF'}")
    if efield is not None:
        lines.append(" Efield " + " ".join(repr(float(e)) for e in efield))
    cond = os.path.join(directory, "cond.txt")
    with open(cond, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return cond
