"""mdn_place (GPU initial placement) against the oracle's sequential loop
(orc_place): the same counter-based stream, so the centres are identical bit
for bit and the Box-Muller velocities agree to rounding (CUDA's and the C
library's log / cos / sin differ in the last bits)."""
import math

import numpy as np
import pytest

from md_nucleation_b200 import generate as g
from tests.gpu_helpers import need_gpu
from tests.test_placement import KB, exemption_seed, min_image_dist

pytestmark = pytest.mark.gpu

VEL_RTOL = 1e-13


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


def same(eng, oracle_libs, box, ion, ng, nv, sg, sv, seed):
    got = eng.place(box, ion, ng, nv, sg, sv, seed)
    want = oracle_libs.orc_place(box, ion, ng, nv, sg, sv, seed)
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[2], want[2])
    for a, b in ((got[1], want[1]), (got[3], want[3])):
        assert np.allclose(a, b, rtol=VEL_RTOL, atol=0)
    return got


def test_nacl_box(eng, oracle_libs):
    same(eng, oracle_libs, 436.0, g.nacl_cluster().top.x, 20000, 300, 421.0, 263.0, 0x4D444E55)


def test_long_chain_large_box(eng, oracle_libs):
    rng = np.random.default_rng(9)
    ion = g.chain(500, 1.0, rng).top.x
    gx, _, vx, _ = same(eng, oracle_libs, 1606.0, ion, 100000, 1000, 298.0, 263.0, 17)
    assert min_image_dist(gx[:5000], ion, 1606.0).min() > 10.0


def test_ion_larger_than_one_tile(eng, oracle_libs):
    """2,500 ion atoms: the test kernel stages them in three shared tiles."""
    rng = np.random.default_rng(4)
    ion = rng.uniform(-60, 60, (2500, 3))
    same(eng, oracle_libs, 300.0, ion, 3000, 50, 300.0, 300.0, 23)


def test_low_acceptance_spans_many_rounds(eng, oracle_libs):
    """An ion lattice that leaves ~8 % of the box free: the kept molecules
    come from several candidate rounds."""
    s = np.arange(-30.0, 30.0, 15.0)
    ion = np.array([[x, y, z] for x in s for y in s for z in s])
    same(eng, oracle_libs, 60.0, ion, 6000, 400, 300.0, 300.0, 31)


def test_first_gas_molecule_exemption(eng, oracle_libs):
    box, ion = 30.0, np.array([[12.0, 12.0, 12.0]])
    seed = exemption_seed(oracle_libs, box, ion)
    gx, _, _, _ = same(eng, oracle_libs, box, ion, 40, 10, 300.0, 300.0, seed)
    assert np.sqrt((gx[0] ** 2).sum()) <= 10.0


def test_no_gas_then_vapor_takes_the_exemption(eng, oracle_libs):
    same(eng, oracle_libs, 50.0, np.array([[20.0, 0.0, 0.0]]), 0, 200, 300.0, 300.0, 8)


def test_no_room_is_an_error(eng):
    with pytest.raises(eng.MdnError, match="did not converge"):
        eng.place(10.0, np.zeros((1, 3)), 1, 0, 300.0, 300.0, 1)


def test_host_places_on_the_gpu(eng, oracle_libs, tmp_path):
    """mdnh_load_ex with a device: the host's descriptor carries the stream's
    centres for its seed (0x4D444E55 + calculation number)."""
    from md_nucleation_b200 import host as H
    from tests.test_host import write_case
    s = H.HostSystem(write_case(tmp_path, "nacl"), calc_number=3, place_device=0)
    d = s.desc
    ion = s.topology("ion")["x"]
    sg = math.sqrt(KB * d.temperature / d.gas_mb_mass)
    sv = math.sqrt(KB * d.temperature / d.vapor_mb_mass)
    want = oracle_libs.orc_place(d.box, ion, d.n_gas, d.n_vapor, sg, sv, 0x4D444E55 + 3)
    gx = np.ctypeslib.as_array(d.gas_x, shape=(3 * d.n_gas,)).reshape(-1, 3)
    vx = np.ctypeslib.as_array(d.vapor_x, shape=(3 * d.n_vapor,)).reshape(-1, 3)
    gv = np.ctypeslib.as_array(d.gas_v, shape=(3 * d.n_gas,)).reshape(-1, 3)
    assert np.array_equal(gx, want[0])
    assert np.array_equal(vx, want[2])
    assert np.allclose(gv, want[1], rtol=VEL_RTOL, atol=0)
