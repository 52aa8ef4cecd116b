"""gg LJ on the GPU (the corrected form of PotentialGasGas,
src/potential/GasGas.cpp:4-62) against the FP64 oracle, through the C ABI.

Bars as in test_gpu_parity.py: pair lists equal as sets; forces within 1e-5
relative RMS of FP64 (FP32 pair arithmetic, int64 fixed-point sums),
energies within 1e-4 of the largest bucket; the FP64 pair mode within 1e-9;
30 steps across a rebuild within 1e-6 A / 1e-7 A/fs.
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from tests import systems
from tests.gpu_helpers import FORCE_ATOL, compare_states, force_ok, forces_of, need_gpu, rel_rms

pytestmark = pytest.mark.gpu

CHECKED = abi.Q_ALL & ~abi.Q_BLIND_INSERT
# a two-atom gas (N2) and a one-atom gas (He), gg on beside the other terms
NAMES = ["nacl_n2_meoh", "chain_he_water"]


def gg_system(name):
    """gas centres at least 4 A apart: the placement (like the reference's,
    src/initialization/initializationGas.cpp:36-56) keeps molecules only
    clear of the ion, which gas that does not interact with itself allows"""
    return systems.with_terms(systems.make(name, gas_min_dist=4.0), extra=abi.I_GG)


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


@pytest.mark.parametrize("name", NAMES)
def test_gg_pair_list_matches_oracle(eng, oracle_libs, name):
    spec = gg_system(name)
    e = eng.Engine([spec])
    o = oracle_libs.OracleReplica(spec)
    got = {tuple(p) for p in e.pair_list(0, 2)}
    want = {tuple(p) for p in o.pair_list(2)}
    assert len(want) > 100 and got == want
    assert e.info(0).gg_pairs == len(want)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("term", [abi.I_GG, 0])
def test_gg_forces_match_fp64_oracle(eng, oracle_libs, name, term):
    spec = gg_system(name)
    o = oracle_libs.OracleReplica(spec)
    o.step(3)  # weights of the gas atoms set by the drift, no rebuild on the last step
    assert o.info().loop_pair > 0
    st = o.get_state()
    e = eng.Engine([spec])
    e.upload(0, st)
    e.compute_forces(term)
    Uo = o.compute_forces(term)
    Ue = e.energies()[0]
    fe, fo = forces_of(e.state(0), spec), forces_of(o.get_state(), spec)
    ok, err, rms = force_ok(fe, fo)
    assert ok, f"relative RMS force error {err:.2e} (RMS {rms:.2e} kcal/mol/A)"
    assert Uo[abi.U_GG] != 0.0
    scale = max(np.abs(Uo).max(), 1e-3)
    assert np.all(np.abs(Ue - Uo) <= 1e-4 * scale + 1e-6), f"energies {Ue} vs {Uo}"


@pytest.mark.parametrize("name", NAMES)
def test_gg_fp64_pair_mode_forces(eng, oracle_libs, name):
    spec = gg_system(name)
    o = oracle_libs.OracleReplica(spec)
    o.step(3)
    st = o.get_state()
    e = eng.Engine([spec], force_mode=1)
    e.upload(0, st)
    e.compute_forces(abi.I_GG)
    o.compute_forces(abi.I_GG)
    fe, fo = forces_of(e.state(0), spec), forces_of(o.get_state(), spec)
    err = rel_rms(fe, fo)
    # helium's gas-gas forces are small: a few 2^-40 kcal/mol/A fixed-point
    # quanta per atom then exceed 1e-9 of them
    rms = np.sqrt(np.mean((fe - fo) ** 2))
    assert err <= 1e-9 or rms <= FORCE_ATOL, f"relative RMS force error {err:.2e} (RMS {rms:.2e})"


@pytest.mark.parametrize("name", NAMES)
def test_gg_trajectory_across_rebuild(eng, oracle_libs, name):
    """30 steps with a rebuild at the first step, checked insertion (which
    with the gas-gas term also keeps entering gas 2 A from the gas in the
    domain; the reference's blind insertion can drop one gas molecule onto
    another): molecules entering carry taper weight 0 for that step in both."""
    quirks = CHECKED
    spec = gg_system(name)
    o = oracle_libs.OracleReplica(spec, quirks=quirks)
    o.step(2)
    st = o.get_state()
    st.loop_pair, st.loop_update = 5, 5
    e = eng.Engine([spec], quirks=quirks)
    e.upload(0, st)
    o.set_state(st)
    e.step(30, energy_mode=1)
    o.step(30, energy_mode=1)
    a, b = e.state(0), o.get_state()
    assert e.info(0).n_rebuilds >= 2 and e.status()[0] == 0
    compare_states(a, b, spec, xtol=1e-6, vtol=1e-7, what=name)
    assert rel_rms(forces_of(a, spec), forces_of(b, spec)) <= 1e-4
    Ue, Uo = e.energies()[0], o.energies()
    assert np.all(np.abs(Ue - Uo) <= 1e-4 * max(np.abs(Uo).max(), 1e-3) + 1e-6)


def test_gg_launch_shape_invariance(eng):
    """Each molecule sums its own gas-gas force over its full partner list:
    bit-identical across cluster sizes."""
    specs = [gg_system(n) for n in NAMES]
    e0 = eng.Engine(specs, cluster_size=1)
    e1 = eng.Engine(specs, cluster_size=4, threads=256)
    e0.step(25, energy_mode=1)
    e1.step(25, energy_mode=1)
    for r, s in enumerate(specs):
        compare_states(e0.state(r), e1.state(r), s, 0.0, 0.0, what=f"replica {r}")
    assert np.array_equal(e0.energies(), e1.energies())
