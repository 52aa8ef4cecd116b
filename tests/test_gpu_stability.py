"""Long runs of the batched-replica workload on the GPU.

The bench advances 256 replicas for hundreds of 100-step blocks; a replica
that reaches a singular configuration (an atom on top of another, a torsion
through a collinear bond) raises MDN_ST_NONFINITE and is frozen.  These tests
run a sample of the batch for 3,000 steps with the checked insertion and
require every replica to stay clean, and follow replica 96 -- whose chain,
as first generated, carried a hydrogen at 176 degrees from a backbone bond and
blew up after 2,463 steps in the engine and in the FP64 oracle alike -- with
the oracle restarted from the engine's state on one 100-step block.
"""
import multiprocessing as mp

import numpy as np
import pytest

from md_nucleation_b200 import abi
from tests.gpu_helpers import compare_states, need_gpu

pytestmark = pytest.mark.gpu

CHECKED = abi.Q_ALL & ~abi.Q_BLIND_INSERT
SAMPLE = [96] + list(range(0, 256, 16))


def _make(r):
    from md_nucleation_b200 import generate
    return generate.config2_replica(r)


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


@pytest.fixture(scope="module")
def sample_specs():
    with mp.get_context("spawn").Pool(8) as pool:
        return pool.map(_make, SAMPLE, chunksize=1)


def test_batch_sample_stays_clean_for_3000_steps(eng, sample_specs):
    e = eng.Engine(sample_specs, quirks=CHECKED, use_graph=1)
    for block in range(30):
        e.step(100)
        st = e.status()
        bad = {SAMPLE[r]: hex(int(st[r])) for r in np.nonzero(st)[0]}
        assert not bad, f"after {100 * (block + 1)} steps: replica status {bad}"
    assert all(e.info(r).n_rebuilds >= 2 for r in range(e.n))


def test_replica_96_tracks_the_oracle_late_in_the_run(eng, oracle_libs, sample_specs):
    """2,400 steps free-running, then one block with the oracle restarted from
    the engine's state: in-domain sets equal, positions within 1e-5 A,
    velocities within 1e-6 A/fs (the bars of the dense parity test)."""
    spec = sample_specs[0]
    e = eng.Engine([spec], quirks=CHECKED, use_graph=1)
    o = oracle_libs.OracleReplica(spec, quirks=CHECKED)
    for _ in range(24):
        o.set_state(e.state(0))  # the oracle follows, so its rebuild count stays equal
        e.step(100)
        o.step(100)
    assert e.status()[0] == 0
    o.set_state(e.state(0))
    e.step(100)
    o.step(100)
    assert e.status()[0] == 0 and o.status() == 0
    compare_states(e.state(0), o.get_state(), spec, xtol=1e-5, vtol=1e-6, what="config2[96] block 24")
