"""Pins the FP64 CPU restatement (oracle/mdn_oracle.cpp) to the reference.

The reference ships no tests or golden vectors, so the pins are:
  * Philox4x32-10 against the published known-answer vectors;
  * the reference program's own routines, compiled from its sources and driven
    on identical injected states through oracle/ref_harness.cpp: forces,
    energies, kicks, drift, centres, taper weights, thermostats and the
    deterministic part of the effective-domain rebuild bit-for-bit; SHAKE to
    the constraint tolerance (the two iterations differ, see mdn_oracle.cpp);
  * the committed golden fixtures (tests/golden/), which carry the same
    comparisons to machines without the reference sources.
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from tests import systems

# Random123's published known-answer vectors for philox4x32-10:
# (counter, key) -> output
PHILOX_KAT = [
    ((0, 0, 0, 0), 0x0000000000000000, (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, 0xFFFFFFFFFFFFFFFF, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), 0x299F31D0A4093822,
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def test_philox_known_answers(oracle_libs):
    for ctr, key, want in PHILOX_KAT:
        assert tuple(oracle_libs.orc_philox(key, ctr)) == want


def _pair(ref_bind, name, **over):
    spec = systems.make(name, **over)
    r = ref_bind.RefReplica(spec)
    o = ref_bind.OracleReplica(spec)
    o.set_state(r.get_state())  # identical in-domain state and lists
    return spec, r, o


def _same_state(a, b, spec, exact=True, tol=0.0):
    gm = a.region[1:1 + spec.n_gas].astype(bool)
    vm = a.region[1 + spec.n_gas:].astype(bool)
    pairs = [(a.ion_x, b.ion_x), (a.ion_v, b.ion_v), (a.ion_f, b.ion_f),
             (a.gas_ax[gm], b.gas_ax[gm]), (a.gas_av[gm], b.gas_av[gm]), (a.gas_af[gm], b.gas_af[gm]),
             (a.vap_ax[vm], b.vap_ax[vm]), (a.vap_av[vm], b.vap_av[vm]), (a.vap_af[vm], b.vap_af[vm]),
             (a.vap_w[vm], b.vap_w[vm]), (a.mol_x[:1], b.mol_x[:1]), (a.mol_v[:1], b.mol_v[:1])]
    for k, (x, y) in enumerate(pairs):
        if exact:
            assert np.array_equal(x, y), f"array {k} differs: max {np.abs(x - y).max()}"
        else:
            assert np.allclose(x, y, rtol=tol, atol=tol), f"array {k}: max {np.abs(x - y).max()}"


@pytest.mark.parametrize("name", list(systems.ALL))
def test_forces_bit_exact(ref_bind, name):
    spec, r, o = _pair(ref_bind, name)
    info = r.info()
    assert info["n_gas_in"] > 50 and info["n_vapor_in"] >= 2
    Ur = r.compute_forces()
    Uo = o.compute_forces()
    assert np.array_equal(Ur, Uo)
    _same_state(r.get_state(), o.get_state(), spec)


@pytest.mark.parametrize("name", list(systems.ALL))
@pytest.mark.parametrize("term", [abi.I_GI, abi.I_VI, abi.I_VV, abi.I_GV, abi.I_AMBER, abi.I_BMH,
                                  abi.I_GAS_INTRA, abi.I_VAPOR_INTRA])
def test_each_term_bit_exact(ref_bind, name, term):
    spec, r, o = _pair(ref_bind, name)
    if not spec.interactions & term:
        pytest.skip("term not enabled in this system")
    Ur = r.compute_forces(term)
    Uo = o.compute_forces(term)
    assert np.array_equal(Ur, Uo)
    _same_state(r.get_state(), o.get_state(), spec)


def test_efield_bit_exact(ref_bind):
    spec = systems.make("nacl_n2_meoh")
    spec.interactions |= abi.I_EFIELD
    spec.efield = (0.3, -1.2, 2.0)
    r = ref_bind.RefReplica(spec)
    o = ref_bind.OracleReplica(spec)
    o.set_state(r.get_state())
    r.compute_forces(abi.I_EFIELD)
    o.compute_forces(abi.I_EFIELD)
    assert np.array_equal(r.get_state().ion_f, o.get_state().ion_f)


@pytest.mark.parametrize("name", systems.NO_SHAKE)
def test_verlet_bit_exact_between_rebuilds(ref_bind, name):
    """MD::verlet without a rebuild: kick, drift, centre, weights, forces, kick."""
    spec, r, o = _pair(ref_bind, name)
    st = r.get_state()
    st.loop_pair, st.loop_update = 0, 10 ** 6
    r.set_state(st)
    o.set_state(st)
    Ur = r.verlet(25, energy_mode=1)
    o.step(25, energy_mode=1)
    assert np.array_equal(Ur, o.energies())
    _same_state(r.get_state(), o.get_state(), spec)


@pytest.mark.parametrize("mode", [abi.NVT_SCALE, abi.NVT_NH])
def test_thermostats_bit_exact(ref_bind, mode):
    spec = systems.make("nacl_n2_meoh")
    spec.nvt_mode = mode
    spec.nvt_temperature = 450.0
    r = ref_bind.RefReplica(spec)
    o = ref_bind.OracleReplica(spec)
    st = r.get_state()
    st.loop_pair, st.loop_update = 0, 10 ** 6
    r.set_state(st)
    o.set_state(st)
    r.verlet(10)
    o.step(10)
    a, b = r.get_state(), o.get_state()
    assert a.zeta == b.zeta
    _same_state(a, b, spec)


@pytest.mark.parametrize("name", list(systems.ALL))
def test_make_pair_deterministic_part(ref_bind, name):
    """MD::make_pair after some free flight: free flight, centres, in/out
    classification, periodic wrap and the pair lists (as sets) are
    deterministic and must agree exactly; the draws (resampled velocities,
    insertion rotations) follow different generators and are compared
    statistically elsewhere."""
    spec, r, o = _pair(ref_bind, name)
    st = r.get_state()
    # 2000 steps of free flight inside make_pair move the molecules ~10 A,
    # so some enter and some leave the domain
    st.loop_pair = 2000
    st.loop_update = 1999
    r.set_state(st)
    o.set_state(st)
    r.call("make_pair")
    o.make_pair()
    a, b = r.get_state(), o.get_state()
    assert np.array_equal(a.region, b.region)
    gm = a.region[1:1 + spec.n_gas].astype(bool)
    # centres: in molecules (recomputed from atoms) and out molecules (free flight + wrap)
    assert np.array_equal(a.mol_x, b.mol_x)
    inside = a.region == 1  # velocities of molecules inside are deterministic
    assert np.array_equal(a.mol_v[inside], b.mol_v[inside])
    # atoms of molecules that stayed inside are untouched by the rebuild
    stayed = (st.region[1:1 + spec.n_gas] == 1) & gm
    assert np.array_equal(a.gas_ax[stayed], b.gas_ax[stayed])
    for kind in (0, 1):
        la = {tuple(p) for p in r.pair_list(kind)}
        lb = {tuple(p) for p in o.pair_list(kind)}
        assert la == lb
    ia, ib = r.info(), o.info()
    assert ia["n_gas_in"] == ib.n_gas_in and ia["n_vapor_in"] == ib.n_vapor_in
    assert gm.sum() == ia["n_gas_in"]


def test_rotation_bit_exact(ref_bind):
    rng = np.random.default_rng(3)
    for _ in range(200):
        A, B, C = rng.uniform(0, 2 * np.pi, 3)
        x, y, z = rng.normal(size=3)
        assert np.array_equal(ref_bind.ref_rotation(A, B, C, x, y, z),
                              ref_bind.orc_rotate(A, B, C, x, y, z, 0))


def test_shake_converges_to_reference(ref_bind):
    """MD::shake (src/shake.cpp:44-92) and the restated iteration reach the
    same constrained positions to the constraint tolerance
    (|s^2 - d^2| <= 1e-10 A^2)."""
    spec = systems.make("chain_ar_meoh_shake")
    r = ref_bind.RefReplica(spec)
    st = r.get_state()
    rng = np.random.default_rng(5)
    old = st.ion_x.copy()
    new = old + rng.normal(scale=0.02, size=old.shape)
    st.ion_x = new.copy()
    r.set_state(st)
    r.shake(0, old)
    ref_x = r.get_state().ion_x
    # the restatement: no force term, x = old and v = (new - old) / dt, so its
    # drift lands on `new` and its SHAKE uses `old` as the reference vectors
    spec_q = systems.make("chain_ar_meoh_shake")
    spec_q.interactions = abi.I_SHAKE
    o = ref_bind.OracleReplica(spec_q)
    st2 = st.copy()
    st2.ion_x = old.copy()
    st2.ion_v = (new - old) / spec.dt
    st2.ion_f[:] = 0
    st2.loop_pair, st2.loop_update = 0, 10 ** 6
    o.set_state(st2)
    o.step(1)
    x = o.get_state().ion_x
    rig = spec.ion.rigid
    d0 = spec.bond_coeff[rig[:, 2], 1]
    assert len(rig) > 10
    for X in (ref_x, x):
        d = np.linalg.norm(X[rig[:, 0]] - X[rig[:, 1]], axis=1)
        assert np.all(np.abs(d * d - d0 * d0) <= 1.0001e-10)
    assert np.abs(ref_x - x).max() < 1e-8


def test_kinetic_matches_reference(ref_bind):
    spec = systems.make("nacl_n2_meoh")
    r = ref_bind.RefReplica(spec)
    o = ref_bind.OracleReplica(spec)
    st = r.get_state()
    o.set_state(st)
    kr = r.kinetic()
    ko = o.kinetic()
    assert np.array_equal(kr[[1, 2, 3]], ko[[1, 2, 3]])
    assert abs(kr[0] - ko[0]) <= 1e-12 * abs(kr[0])
