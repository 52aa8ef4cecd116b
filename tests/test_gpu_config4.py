"""The large low-vapor-pressure configuration at full size: 1,000,000 N2,
1,000 rigid 3-site water, a +2 chain of 500 atoms (SHAKE on X-H bonds).

One replica against the FP64 oracle from the same state (three oracle steps
after the initial rebuild, so forces and weights are populated): the force
error of the FP32 pair terms (force_mode 0) and of FP64 pair terms (force_mode
1), both with 64-bit fixed-point sums, and a short trajectory.
"""
import numpy as np
import pytest

from tests.gpu_helpers import FORCE_RTOL, compare_states, forces_of, need_gpu, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(oracle_libs):
    eng = need_gpu()
    from md_nucleation_b200 import generate
    spec = generate.config4_replica(0)
    o = oracle_libs.OracleReplica(spec)
    o.step(3)
    return eng, spec, o


def test_config4_forces_fp32_and_fp64(case):
    eng, spec, o = case
    st = o.get_state()
    o.set_state(st)
    o.compute_forces(0)
    fo = forces_of(o.get_state(), spec)
    errs = {}
    for mode in (0, 1):
        e = eng.Engine([spec], force_mode=mode)
        e.upload(0, st)
        e.compute_forces(0)
        errs[mode] = rel_rms(forces_of(e.state(0), spec), fo)
        e.close()
    print(f"config 4 force error vs FP64: FP32 pair terms {errs[0]:.2e}, FP64 pair terms {errs[1]:.2e}")
    assert errs[0] <= FORCE_RTOL
    assert errs[1] <= 1e-9


def test_config4_trajectory(case):
    eng, spec, o = case
    st = o.get_state()
    e = eng.Engine([spec])
    e.upload(0, st)
    o.set_state(st)
    e.step(20)
    o.step(20)
    assert e.status()[0] == 0
    compare_states(e.state(0), o.get_state(), spec, xtol=1e-6, vtol=1e-7, what="config 4")


def test_config4_pair_lists_match_oracle(case):
    """The cell-binned list build on the largest core (the 500-atom chain and
    the in-domain water) against the oracle's all-pairs rule for the same
    state (GasIon.cpp:41-60, VaporGas.cpp:5-64): equal as sets."""
    eng, spec, o = case
    st = o.get_state()
    o.set_state(st)
    e = eng.Engine([spec])
    e.upload(0, st)
    n = 0
    for kind in (0, 1):
        got = {tuple(p) for p in e.pair_list(0, kind)}
        want = {tuple(p) for p in o.pair_list(kind)}
        assert got == want, kind
        n += len(want)
    assert n > 0
    e.close()
