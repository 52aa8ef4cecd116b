"""GPU parity of the thermostats, the observer and the electric field
against the FP64 oracle (itself pinned bit for bit to the reference's
MD::velocity_scaling / nosehoover_* (src/nvt.cpp:5-42),
Observer::computeProps (src/output/observer.cpp:5-36) and
PotentialEfield::compute (src/potential/electricField.cpp:54-64) in
tests/test_oracle_pins.py).

Bars: 50 thermostatted steps within 1e-6 A / 1e-7 A/fs and zeta within
1e-6 relative; kinetic energies within 1e-12 relative (parallel sums of the
same FP64 terms); field forces within 2^-39 kcal/mol/A (two fixed-point
quanta).
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from tests import systems
from tests.gpu_helpers import compare_states, need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


@pytest.mark.parametrize("mode", [pytest.param(abi.NVT_SCALE, id="scale"), pytest.param(abi.NVT_NH, id="nose-hoover")])
@pytest.mark.parametrize("name", ["chain_he_water", "nacl_n2_meoh"])
def test_thermostat_matches_oracle(eng, oracle_libs, name, mode):
    spec = systems.make(name)
    spec.nvt_mode = mode
    spec.nvt_temperature = 450.0
    o = oracle_libs.OracleReplica(spec)
    st = o.get_state()
    st.loop_pair, st.loop_update = 0, 10 ** 6
    o.set_state(st)
    e = eng.Engine([spec])
    e.upload(0, st)
    e.step(50)
    o.step(50)
    a, b = e.state(0), o.get_state()
    compare_states(a, b, spec, xtol=1e-6, vtol=1e-7, what=f"{name} nvt {mode}")
    # zeta integrates the ion temperature, which the FP32 pair forces move
    # at ~1e-7 relative over the window
    assert abs(a.zeta - b.zeta) <= 1e-6 * abs(b.zeta) + 1e-12
    if mode == abi.NVT_NH:
        assert b.zeta != 0.0
    Te, To = e.kinetic()[0, 3], o.kinetic()[3]
    assert abs(Te - To) <= 1e-6 * To


def test_thermostat_switch_per_replica(eng, oracle_libs):
    """mdn_set_nvt on one replica of a batch: it follows the oracle with the
    thermostat, its neighbour the oracle without."""
    a_spec, b_spec = systems.make("chain_he_water"), systems.make("nacl_n2_meoh")
    e = eng.Engine([a_spec, b_spec])
    e.set_nvt(abi.NVT_NH, 420.0, replica=0)
    oa, ob = oracle_libs.OracleReplica(a_spec), oracle_libs.OracleReplica(b_spec)
    oa.set_nvt(abi.NVT_NH, 420.0)
    e.step(30)
    oa.step(30)
    ob.step(30)
    compare_states(e.state(0), oa.get_state(), a_spec, 1e-6, 1e-7, what="thermostatted")
    compare_states(e.state(1), ob.get_state(), b_spec, 1e-6, 1e-7, what="NVE neighbour")


@pytest.mark.parametrize("name", list(systems.ALL))
def test_kinetic_matches_oracle_and_reference(eng, oracle_libs, name):
    spec = systems.make(name)
    o = oracle_libs.OracleReplica(spec)
    o.step(7)
    st = o.get_state()
    e = eng.Engine([spec])
    e.upload(0, st)
    ke, ko = e.kinetic()[0], o.kinetic()
    assert np.all(np.abs(ke - ko) <= 1e-12 * np.abs(ko) + 1e-300), f"{ke} vs {ko}"
    if oracle_libs.have_reference():
        r = oracle_libs.RefReplica(spec)
        r.set_state(st)
        kr = r.kinetic()  # Kion, K_g, K_v, Tion, T_g, T_v
        assert np.all(np.abs(ke - kr[:4]) <= 1e-12 * np.abs(kr[:4]) + 1e-300), f"{ke} vs {kr[:4]}"


def test_efield_matches_oracle(eng, oracle_libs):
    spec = systems.make("chain_he_water")
    spec.interactions |= abi.I_EFIELD
    spec.efield = (0.3, -1.2, 2.0)
    o = oracle_libs.OracleReplica(spec)
    o.step(3)
    st = o.get_state()
    e = eng.Engine([spec])
    e.upload(0, st)
    e.compute_forces(abi.I_EFIELD)
    o.compute_forces(abi.I_EFIELD)
    fe, fo = e.state(0).ion_f, o.get_state().ion_f
    assert np.abs(fo).max() > 1e-6
    assert np.abs(fe - fo).max() <= 2.0 ** -39
    # and over 30 steps with every term on
    o2 = oracle_libs.OracleReplica(spec)
    e2 = eng.Engine([spec])
    e2.step(30, energy_mode=1)
    o2.step(30, energy_mode=1)
    compare_states(e2.state(0), o2.get_state(), spec, 1e-6, 1e-7, what="efield")
