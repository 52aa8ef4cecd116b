"""Per-replica status words under host-side fault injection.

The reference has no failure detection: a non-finite state propagates, its
SHAKE loops until converged with no cap (src/shake.cpp:51), and a list or
slab cannot overflow because it grows on the heap.  The engine bounds every
such loop and reports a status bit per replica instead (include/mdn.h,
MDN_ST_*).  Every fault here is made on the host -- a NaN or an overlap in
an uploaded state, an impossible constraint in the descriptor, molecules
packed into the domain -- so no kernel faults, traps or hangs.  Each test
checks the bit, whether mdn_step reports the replica (fatal bits), and that
the replica steps cleanly again after mdn_clear_status and a clean upload.
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from tests import systems
from tests.gpu_helpers import need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


def relaunch_clean(e, clean):
    e.clear_status()
    assert e.status()[0] == 0
    e.upload(0, clean)
    e.step(5)
    assert e.status()[0] == 0


def test_nonfinite_state_is_fatal_and_recoverable(eng):
    e = eng.Engine([systems.make("nacl_n2_meoh")])
    clean = e.state(0)
    bad = clean.copy()
    bad.ion_x[0, 0] = np.nan
    e.upload(0, bad)
    with pytest.raises(eng.MdnError) as ex:
        e.step(1)
    assert ex.value.code == abi.ERR_REPLICA
    assert e.status()[0] & abi.ST_NONFINITE
    step = e.info(0).step
    with pytest.raises(eng.MdnError):
        e.step(3)                   # a fatal replica is frozen, not stepped
    assert e.info(0).step == step
    relaunch_clean(e, clean)


def test_overlapping_atoms_saturate_as_a_warning(eng):
    """A gas atom 0.05 A from an ion atom: its pair force saturates at
    2^21 kcal/mol/A per term -- MDN_ST_FIXED_OVERFLOW, not fatal."""
    spec = systems.make("nacl_n2_meoh")
    e = eng.Engine([spec])
    clean = e.state(0)
    bad = clean.copy()
    gin = np.nonzero(bad.region[1:1 + spec.n_gas])[0]
    L = e.pair_list(0, 0)
    m = int(L[0, 0]) if len(L) else int(gin[0])
    j = int(L[0, 1]) if len(L) else 0
    shift = bad.ion_x[j] + np.array([0.05, 0.0, 0.0]) - bad.gas_ax[m, 0]
    bad.gas_ax[m] += shift
    bad.mol_x[1 + m] += shift
    e.upload(0, bad)
    e.compute_forces(abi.I_GI)
    assert e.status()[0] & abi.ST_FIXED_OVERFLOW
    assert not e.status()[0] & abi.ST_FATAL
    relaunch_clean(e, clean)


def test_impossible_constraint_hits_the_sweep_cap(eng):
    """Rigid water whose H-H constraint (3 A) exceeds the two O-H
    constraints (0.96 A each): no position satisfies all three, so SHAKE
    stops at MDN_SHAKE_MAX_SWEEPS and raises MDN_ST_SHAKE_NOCONV, where the
    reference's loop would never end."""
    spec = systems.make("nacl_n2rigid_water")
    hh = int(spec.vapor.rigid[2, 2])
    spec.bond_coeff[hh, 1] = 3.0
    e = eng.Engine([spec])
    if e.info(0).n_vapor_in == 0:
        pytest.fail("the system has no water in the domain")
    try:
        e.step(2)
    except eng.MdnError as ex:
        assert ex.code == abi.ERR_REPLICA
    assert e.status()[0] & abi.ST_SHAKE_NOCONV


def _pack_gas_near_ion(spec, st, n, spacing=4.0, r_min=4.0):
    """moves n gas molecules that are outside the domain onto lattice points
    around the ion centre (no point within r_min of an ion atom); they enter
    at the next rebuild"""
    out = np.nonzero(st.region[1:1 + spec.n_gas] == 0)[0][:n]
    c = st.ion_x.mean(axis=0)
    k = int(np.ceil(n ** (1 / 3))) + 4
    g = (np.arange(k) - k / 2) * spacing
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + c
    d = np.linalg.norm(pts[:, None] - st.ion_x[None], axis=2).min(axis=1)
    pts = pts[d > r_min]
    pts = pts[np.argsort(np.linalg.norm(pts - c, axis=1))][:len(out)]
    assert len(pts) == len(out)
    st.mol_x[1 + out] = pts
    st.loop_pair, st.loop_update = 5, 5   # rebuild on the next step
    return len(out)


def test_list_overflow_is_fatal_and_recoverable(eng):
    """500 gas molecules packed within 22 A of the ion: far more
    gas-ion list entries than the list was sized for (MDN_ST_LIST_OVERFLOW)."""
    spec = systems.make("nacl_n2_meoh")
    e = eng.Engine([spec], quirks=abi.Q_ALL)
    clean = e.state(0)
    bad = clean.copy()
    _pack_gas_near_ion(spec, bad, 500)
    e.upload(0, bad)
    with pytest.raises(eng.MdnError) as ex:
        e.step(1)
    assert ex.value.code == abi.ERR_REPLICA
    assert e.status()[0] & abi.ST_LIST_OVERFLOW
    relaunch_clean(e, clean)


def test_slab_overflow_is_fatal_and_recoverable(eng):
    """More gas molecules entering than the slab holds (the slab is sized
    for the expected in-domain count, binomial mean + 6 sigma + 64)."""
    spec = systems.make("chain_he_water")
    e = eng.Engine([spec], quirks=abi.Q_ALL, capacity_factor=1.0)
    clean = e.state(0)
    bad = clean.copy()
    gin = int(bad.region[1:1 + spec.n_gas].sum())
    free = int((bad.region[1:1 + spec.n_gas] == 0).sum())
    _pack_gas_near_ion(spec, bad, min(free, 2 * gin + 500), spacing=3.5)
    e.upload(0, bad)
    with pytest.raises(eng.MdnError) as ex:
        e.step(1)
    assert ex.value.code == abi.ERR_REPLICA
    assert e.status()[0] & abi.ST_SLAB_OVERFLOW
    relaunch_clean(e, clean)
