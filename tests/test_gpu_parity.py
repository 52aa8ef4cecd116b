"""Parity of the CUDA engine (through the C ABI) with the FP64 oracle.

Bars (the tolerance of each comparison is stated where it is made):
  * the effective-domain rebuild uses the same Philox draws as the oracle, so
    the whole state after MD::MD's initial make_pair agrees to FP64 rounding
    of the transcendental functions (sin/cos/log of CUDA vs glibc);
  * pair lists are equal as sets;
  * forces: relative RMS error <= 1e-5 against FP64 (FP32 pair arithmetic,
    int64 fixed-point sums); energies per bucket likewise;
  * short trajectories, across a rebuild, stay within 1e-6 A / 1e-7 A/fs;
  * results are bit-identical across launch shapes and batch compositions
    (every multi-writer sum is an integer sum).
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from tests import systems
from tests.gpu_helpers import compare_states, force_ok, forces_of, need_gpu, rel_rms

pytestmark = pytest.mark.gpu

NAMES = list(systems.ALL)
# the reference's insertion (one random rotation, no overlap test) and the
# checked insertion (rotation re-drawn until nothing lies within 2 A)
CHECKED = abi.Q_ALL & ~abi.Q_BLIND_INSERT
INSERTION = [pytest.param(abi.Q_ALL, id="blind"), pytest.param(CHECKED, id="checked")]


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


@pytest.mark.parametrize("quirks", INSERTION)
@pytest.mark.parametrize("name", NAMES)
def test_initial_make_pair_matches_oracle(eng, oracle_libs, name, quirks):
    spec = systems.make(name)
    e = eng.Engine([spec], quirks=quirks)
    o = oracle_libs.OracleReplica(spec, quirks=quirks)
    a, b = e.state(0), o.get_state()
    i = e.info(0)
    assert i.status == 0
    assert i.n_gas_in == o.info().n_gas_in and i.n_vapor_in == o.info().n_vapor_in
    compare_states(a, b, spec, xtol=1e-11, vtol=1e-13, what=name)
    assert abs(a.loop_update - b.loop_update) <= 1
    for kind in (0, 1):
        assert {tuple(p) for p in e.pair_list(0, kind)} == {tuple(p) for p in o.pair_list(kind)}


def test_pair_lists_after_steps_match_oracle(eng, oracle_libs):
    """The cell-binned list build against the oracle's all-pairs rule on two
    replicas of the batched workload (a 69- and a 221-atom ion, dozens to a
    hundred in-domain vapor molecules) after 300 steps: the state is loaded
    into a fresh engine, whose upload rebuilds the lists, and into the oracle,
    whose set_state does; the lists are equal as sets."""
    from md_nucleation_b200 import generate
    specs = [generate.config2_replica(r) for r in (24, 42)]
    e = eng.Engine(specs, quirks=CHECKED)
    e.step(300)
    assert (e.status() & abi.ST_FATAL).sum() == 0
    for r, spec in enumerate(specs):
        S = e.state(r)
        o = oracle_libs.OracleReplica(spec, quirks=CHECKED)
        o.set_state(S)
        f = eng.Engine([spec], quirks=CHECKED)
        f.upload(0, S)
        for kind in (0, 1):
            got = {tuple(p) for p in f.pair_list(0, kind)}
            want = {tuple(p) for p in o.pair_list(kind)}
            assert got == want and len(want) > 0, (r, kind)
        f.close()
        o.close()
    e.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("term", [0, abi.I_GI, abi.I_VI, abi.I_VV, abi.I_GV, abi.I_AMBER, abi.I_BMH,
                                  abi.I_GAS_INTRA, abi.I_VAPOR_INTRA])
def test_forces_match_fp64_oracle(eng, oracle_libs, name, term):
    spec = systems.make(name)
    if term and not spec.interactions & term:
        pytest.skip("term not enabled")
    o = oracle_libs.OracleReplica(spec)
    o.step(3)  # weights and forces populated
    st = o.get_state()
    e = eng.Engine([spec])
    e.upload(0, st)
    o.set_state(st)
    e.compute_forces(term)
    Uo = o.compute_forces(term)
    Ue = e.energies()[0]
    fe, fo = forces_of(e.state(0), spec), forces_of(o.get_state(), spec)
    if np.abs(fo).max() == 0:
        assert np.abs(fe).max() == 0
        return
    ok, err, rms = force_ok(fe, fo)
    assert ok, f"relative RMS force error {err:.2e} (RMS {rms:.2e} kcal/mol/A)"
    # energies are sums of FP32 pair terms of both signs: the bound is the FP32
    # rounding of the terms, 1e-4 of the largest bucket (reported per config)
    scale = max(np.abs(Uo).max(), 1e-3)
    assert np.all(np.abs(Ue - Uo) <= 1e-4 * scale + 1e-6), f"energies {Ue} vs {Uo}"


@pytest.mark.parametrize("name", NAMES)
def test_fp64_pair_mode_forces(eng, oracle_libs, name):
    """force_mode 1: the pair terms in FP64 (64-bit fixed-point sums of
    2^-40 kcal/mol/A quanta) agree with the FP64 oracle within 1e-9."""
    spec = systems.make(name)
    o = oracle_libs.OracleReplica(spec)
    o.step(3)
    st = o.get_state()
    e = eng.Engine([spec], force_mode=1)
    e.upload(0, st)
    o.set_state(st)
    e.compute_forces(0)
    o.compute_forces(0)
    err = rel_rms(forces_of(e.state(0), spec), forces_of(o.get_state(), spec))
    assert err <= 1e-9, f"relative RMS force error {err:.2e}"


@pytest.mark.parametrize("quirks", INSERTION)
@pytest.mark.parametrize("name", NAMES)
def test_trajectory_across_rebuild(eng, oracle_libs, name, quirks):
    """30 steps with a rebuild at the first step (loop_pair = loop_update)."""
    spec = systems.make(name)
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
    err = rel_rms(forces_of(a, spec), forces_of(b, spec))
    assert err <= 1e-4
    Ue, Uo = e.energies()[0], o.energies()
    assert np.all(np.abs(Ue - Uo) <= 1e-4 * max(np.abs(Uo).max(), 1e-3) + 1e-6)


def test_dense_batched_replica_tracks_oracle(eng, oracle_libs):
    """A replica of the 256-replica batch workload at full density (about
    14,000 gas molecules in the domain) with the checked insertion: four
    blocks of 100 steps, each started from the oracle's state (a free-running
    comparison separates chaotically, FP32 pair sums against FP64), blocks 1
    and 3 with a rebuild at their first step; the rebuild count and the in-domain sets agree and positions
    stay within 1e-5 A, velocities within 1e-6 A/fs (in this 5.5e6 Pa helium
    the FP32 rounding of the pair forces grows to ~1.5e-6 A within one block)."""
    from md_nucleation_b200 import generate
    spec = generate.config2_replica(2)
    e = eng.Engine([spec], quirks=CHECKED)
    o = oracle_libs.OracleReplica(spec, quirks=CHECKED)
    rebuilds = 0
    for block in range(4):
        assert e.info(0).n_rebuilds == o.info().n_rebuilds
        st = o.get_state()
        if block % 2:  # a rebuild at the block's first step
            st.loop_pair, st.loop_update = 5, 5
            o.set_state(st)
        e.upload(0, st)
        r0 = o.info().n_rebuilds
        e.step(100)
        o.step(100)
        assert e.status()[0] == 0
        assert e.info(0).n_rebuilds == o.info().n_rebuilds
        rebuilds += o.info().n_rebuilds - r0
        compare_states(e.state(0), o.get_state(), spec, xtol=1e-5, vtol=1e-6, what=f"config2[2] block {block}")
    assert rebuilds >= 2


def test_shake_constraints_hold(eng):
    spec = systems.make("chain_ar_meoh_shake")
    e = eng.Engine([spec])
    e.step(200)
    st = e.state(0)
    rig = spec.ion.rigid
    d0 = spec.bond_coeff[rig[:, 2], 1]
    d = np.linalg.norm(st.ion_x[rig[:, 0]] - st.ion_x[rig[:, 1]], axis=1)
    assert np.all(np.abs(d * d - d0 * d0) <= 1.0001e-10)
    assert e.status()[0] == 0


def test_batch_equals_single_replicas(eng):
    """Replicas are independent: stepping them together is bit-identical to
    stepping each alone."""
    specs = [systems.make(n) for n in ("nacl_n2_meoh", "chain_he_water", "nacl_n2mono_meoh")]
    eb = eng.Engine(specs)
    eb.step(40)
    for r, s in enumerate(specs):
        es = eng.Engine([s])
        es.step(40)
        compare_states(eb.state(r), es.state(0), s, 0.0, 0.0, what=f"replica {r}")


@pytest.mark.parametrize("threads,cluster", [(256, 1), (512, 2), (256, 4)])
def test_launch_shape_invariance(eng, threads, cluster):
    specs = [systems.make("chain_ar_meoh_shake"), systems.make("nacl_n2_meoh")]
    e0 = eng.Engine(specs)
    e1 = eng.Engine(specs, threads=threads, cluster_size=cluster)
    e0.step(25, energy_mode=1)
    e1.step(25, energy_mode=1)
    for r, s in enumerate(specs):
        compare_states(e0.state(r), e1.state(r), s, 0.0, 0.0, what=f"replica {r}")
    assert np.array_equal(e0.energies(), e1.energies())


def test_tuned_launch_keeps_the_trajectory(eng):
    """mdn_tune_launch runs ordinary steps at four cluster sizes, with the
    cycle accounting on, in the measured job order and in split launches:
    the state equals that of the same number of steps at one fixed shape,
    bit for bit."""
    specs = [systems.make(n) for n in ("nacl_n2_meoh", "chain_he_water")]
    a = eng.Engine(specs, cluster_size=1)
    b = eng.Engine(specs)
    best = b.tune_launch(20)
    assert best in (1, 2, 4, 8) and b.get_launch()[0] == best
    steps = b.info(0).step
    assert steps >= 4 * 20 and steps % 20 == 0
    a.step(steps)
    for r in range(2):
        sa, sb = a.state(r), b.state(r)
        for name in ("ion_x", "ion_v", "mol_x", "mol_v", "gas_ax", "gas_av", "vap_ax", "vap_av"):
            assert np.array_equal(getattr(sa, name), getattr(sb, name)), name


def test_split_launch_keeps_the_trajectory(eng):
    """The two largest replicas in a concurrent second launch on clusters of 4
    (mdn_set_split), the rest at 2: the states equal those of one launch."""
    specs = [systems.make(n) for n in systems.ALL]
    a = eng.Engine(specs, cluster_size=2)
    b = eng.Engine(specs, cluster_size=2)
    b.set_split(2, 4)
    assert b.get_split() == (2, 4)
    a.step(40)
    b.step(40)
    _, launches = b.last_timing()
    assert launches == 2
    for r, spec in enumerate(specs):
        compare_states(a.state(r), b.state(r), spec, 0.0, 0.0)
    b.set_split(0)
    assert b.get_split() == (0, 0)


def test_steps_per_launch_invariance(eng):
    spec = systems.make("nacl_n2rigid_water")
    e0 = eng.Engine([spec])
    e1 = eng.Engine([spec], steps_per_launch=1)
    e0.step(20)
    e1.step(20)
    compare_states(e0.state(0), e1.state(0), spec, 0.0, 0.0)


def test_upload_capacity_is_an_error(eng):
    spec = systems.make("nacl_n2_meoh")
    e = eng.Engine([spec])
    st = e.state(0)
    st.region[1:1 + spec.n_gas] = 1  # every gas molecule claimed in-domain
    with pytest.raises(eng.MdnError) as ex:
        e.upload(0, st)
    assert ex.value.code == abi.ERR_CAPACITY
