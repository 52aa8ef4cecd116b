"""The oracle's gas-gas term (the corrected PotentialGasGas) on the CPU:
its list is every pair of in-domain gas molecules whose centres lie within
CutOff + Margin (src/potential/GasGas.cpp:41-62 applied to gas_in), and a
molecule entering the domain carries taper weight 0 on the step of its entry
(MD::update_position ran before the rebuild, src/verlet.cpp:109-134)."""
import numpy as np

from md_nucleation_b200 import abi
from tests import systems


def test_gg_list_is_every_close_in_domain_pair(oracle_libs):
    spec = systems.with_terms(systems.make("nacl_n2_meoh"), extra=abi.I_GG)
    o = oracle_libs.OracleReplica(spec)
    o.step(4)
    st = o.get_state()
    gin = np.nonzero(st.region[1:1 + spec.n_gas])[0]
    c = st.mol_x[1 + gin]
    d2 = ((c[:, None, :] - c[None, :, :]) ** 2).sum(axis=2)
    ml2 = (spec.cutoff + spec.margin) ** 2
    i, j = np.nonzero(np.triu(d2 < ml2, 1))
    want = {(int(gin[a]), int(gin[b])) for a, b in zip(i, j)}
    got = {tuple(p) for p in o.pair_list(2)}
    assert len(want) > 100 and got == want


def test_gg_forces_are_a_pair_sum(oracle_libs):
    """The gas-gas forces sum to zero (Newton's third law within each pair)
    and the term books its energy in Ugg only."""
    spec = systems.with_terms(systems.make("chain_he_water"), extra=abi.I_GG)
    o = oracle_libs.OracleReplica(spec)
    o.step(3)
    U = o.compute_forces(abi.I_GG)
    st = o.get_state()
    g = st.region[1:1 + spec.n_gas].astype(bool)
    F = st.gas_af[g].reshape(-1, 3)
    assert np.abs(F).max() > 0
    assert np.abs(F.sum(axis=0)).max() <= 1e-9 * np.abs(F).sum()
    assert U[abi.U_GG] != 0 and np.all(np.delete(U, abi.U_GG) == 0)
