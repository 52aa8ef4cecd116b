"""Statistical checks of the random parts of the effective-domain rebuild.

The reference draws them from unseeded std::random_device streams
(src/pairList/updateGasIn.cpp:16-17, updateVaporIn.cpp), so its runs can
only be compared by distribution.  The restatement (and the engine, which
reproduces it draw for draw, tests/test_gpu_parity.py) draws from
Philox4x32-10; these tests check the distributions that come out:

  * every molecule found outside the domain at a rebuild gets a fresh
    Maxwell-Boltzmann centre velocity, N(0, sqrt(kT/m)) * 1e-5 A/fs per
    component (updateGasIn.cpp:43-45, updateVaporIn.cpp): starting from zero
    velocities, the out-of-domain molecules pass a Kolmogorov-Smirnov test
    against that normal and the in-domain ones keep their velocity;
  * the components are uncorrelated.
"""
import numpy as np
from scipy import stats

from md_nucleation_b200 import generate as g
from md_nucleation_b200.system import mb_sigma


def resampled(oracle_libs, seed):
    spec = g.small_system(seed=seed, gas="He", vapor="water", n_gas=6000, n_vap=300, box=700.0)
    spec.gas_v[:] = 0.0
    spec.vapor_v[:] = 0.0
    o = oracle_libs.OracleReplica(spec)  # its creation runs the first MD::make_pair
    st = o.get_state()
    out = st.region[1:] == 0
    V = st.mol_v[1:]
    ng = spec.n_gas
    sg = mb_sigma(spec.temperature, spec.gas_mb_mass)
    sv = mb_sigma(spec.temperature, spec.vapor_mb_mass)
    return spec, out[:ng], out[ng:], V[:ng], V[ng:], sg, sv


def test_out_of_domain_velocities_are_maxwell_boltzmann(oracle_libs):
    spec, gout, vout, Vg, Vv, sg, sv = resampled(oracle_libs, 21)
    assert gout.sum() > 4000 and vout.sum() > 200
    for V, out, s in ((Vg, gout, sg), (Vv, vout, sv)):
        z = V[out] / s
        for c in range(3):
            assert stats.kstest(z[:, c], "norm").pvalue > 1e-3, c
        assert abs(np.corrcoef(z.T)[0, 1]) < 0.1
        assert abs(np.corrcoef(z.T)[1, 2]) < 0.1
    # molecules inside the domain are not resampled
    assert np.all(Vg[~gout] == 0.0) and np.all(Vv[~vout] == 0.0)


def test_streams_differ_between_seeds(oracle_libs):
    _, g1, _, V1, _, _, _ = resampled(oracle_libs, 21)
    _, g2, _, V2, _, _, _ = resampled(oracle_libs, 22)
    assert not np.array_equal(V1[g1][:50], V2[g2][:50])
