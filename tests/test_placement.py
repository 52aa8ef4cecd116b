"""Initial placement (MD::initialization_gas / initialization_vapor,
src/initialization/initializationGas.cpp:24-100,
src/initialization/initializationVapor.cpp:14-76): the oracle's restatement
(orc_place) and the C++ host's CPU placement, on the CPU.

The reference keeps a uniformly drawn centre when every row of its atom table
is farther than 10 A (minimum image).  The rows are the ion's atoms and, per
molecule already placed, its atoms parked at the origin.  So the first gas
molecule is tested against the ion alone, and every later one against the
ion and the origin.

  * the oracle equals a plain Python loop over the same counter-based stream
    (the first n kept candidates, in stream order), bit for bit;
  * every kept centre obeys the reference's rule; the first gas molecule
    alone may sit within 10 A of the origin, and a seed where it does is
    kept there;
  * velocities are Maxwell-Boltzmann with the stated sigma;
  * a box with no room fails instead of looping for ever.
"""
import math

import numpy as np
import pytest

from md_nucleation_b200 import generate as g

KB = 1.38e-23
TAG = 0x706C6163


def u01(w):
    return (float(w) + 0.5) * (1.0 / 4294967296.0)


def python_place(bind, box, ion, n, seed, species=0, origin_from_start=False, dis=10.0):
    """The reference's loop over candidate k = 0, 1, ... of the stream."""
    L, LH = box, 0.5 * box
    out, k = [], 0
    while len(out) < n:
        w = bind.orc_philox(seed, (k & 0xFFFFFFFF, k >> 32, species, TAG))
        k += 1
        X = [(u01(w[c]) - 0.5) * L for c in range(3)]
        rows = [tuple(a) for a in ion] + ([(0.0, 0.0, 0.0)] if (out or origin_from_start) else [])
        min_dis = 10000.0
        for a in rows:
            d = []
            for c in range(3):
                v = a[c] - X[c]
                if v < -LH:
                    v += L
                if v > LH:
                    v -= L
                d.append(v)
            dd = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
            min_dis = min(min_dis, dd)
        if min_dis > dis:
            out.append(X)
    return np.array(out).reshape(-1, 3)


def min_image_dist(X, P, L):
    d = X[:, None, :] - P[None, :, :]
    d -= L * np.round(d / L)
    return np.sqrt((d ** 2).sum(-1)).min(axis=1)


def nacl():
    return g.nacl_cluster().top.x


def test_oracle_is_the_sequential_loop(oracle_libs):
    ion = nacl()
    gx, gv, vx, vv = oracle_libs.orc_place(60.0, ion, 80, 20, 300.0, 200.0, 77)
    assert np.array_equal(gx, python_place(oracle_libs, 60.0, ion, 80, 77, 0))
    assert np.array_equal(vx, python_place(oracle_libs, 60.0, ion, 20, 77, 1, origin_from_start=True))


@pytest.mark.parametrize("case", ["nacl", "chain", "offset"])
def test_oracle_follows_the_reference_rule(oracle_libs, case):
    rng = np.random.default_rng(3)
    if case == "nacl":
        box, ion, ng, nv = 436.0, nacl(), 20000, 300
    elif case == "chain":
        box, ion, ng, nv = 400.0, g.chain(300, 1.0, rng).top.x, 20000, 500
    else:  # an ion away from the origin in a small box: the origin rule bites
        box, ion, ng, nv = 80.0, nacl() + np.array([25.0, 0.0, 0.0]), 300, 30
    gx, gv, vx, vv = oracle_libs.orc_place(box, ion, ng, nv, 300.0, 150.0, 11)
    for X in (gx, vx):
        assert np.all(np.abs(X) < box / 2)
        assert min_image_dist(X, ion, box).min() > 10.0
    r0 = np.sqrt((gx ** 2).sum(1))
    assert np.all(r0[1:] > 10.0)
    assert np.all(np.sqrt((vx ** 2).sum(1)) > 10.0)


def exemption_seed(bind, box, ion):
    """A seed whose first kept gas centre lies within 10 A of the origin."""
    for seed in range(1, 20000):
        X = python_place(bind, box, ion, 1, seed)[0]
        if np.sqrt((X ** 2).sum()) <= 10.0:
            return seed
    raise AssertionError("no seed found")


def test_first_gas_molecule_skips_the_origin(oracle_libs):
    box, ion = 30.0, np.array([[12.0, 12.0, 12.0]])
    seed = exemption_seed(oracle_libs, box, ion)
    gx, _, _, _ = oracle_libs.orc_place(box, ion, 40, 0, 300.0, 300.0, seed)
    assert np.sqrt((gx[0] ** 2).sum()) <= 10.0
    assert np.all(np.sqrt((gx[1:] ** 2).sum(1)) > 10.0)


def test_velocities_are_maxwell_boltzmann(oracle_libs):
    sg, sv = 421.0, 263.0
    gx, gv, vx, vv = oracle_libs.orc_place(2000.0, nacl(), 200000, 20000, sg, sv, 5)
    for V, s in ((gv, sg), (vv, sv)):
        z = V / (s * 1e-5)
        assert abs(z.mean()) < 0.02
        assert abs(z.std() - 1.0) < 0.02
        assert abs(np.mean(z ** 4) / np.mean(z ** 2) ** 2 - 3.0) < 0.1


def test_no_room_fails(oracle_libs):
    with pytest.raises(RuntimeError, match="converge"):
        oracle_libs.orc_place(10.0, np.zeros((1, 3)), 1, 0, 300.0, 300.0, 1)


def test_host_cpu_placement_rule(tmp_path):
    """The host's CPU placement (its own generator) obeys the same rule."""
    from md_nucleation_b200 import build
    build.build()
    from md_nucleation_b200 import host as H
    from tests.test_host import write_case
    s = H.HostSystem(write_case(tmp_path, "chain"), calc_number=2)
    d = s.desc
    ion = s.topology("ion")["x"]
    gx = np.ctypeslib.as_array(d.gas_x, shape=(3 * d.n_gas,)).reshape(-1, 3)
    vx = np.ctypeslib.as_array(d.vapor_x, shape=(3 * d.n_vapor,)).reshape(-1, 3)
    for X in (gx, vx):
        assert min_image_dist(X, ion, d.box).min() > 10.0
    assert np.all(np.sqrt((gx[1:] ** 2).sum(1)) > 10.0)
    assert np.all(np.sqrt((vx ** 2).sum(1)) > 10.0)


def test_gpu_placement_fails_loudly_without_a_gpu(tmp_path):
    """mdn_place and the host's GPU placement report the missing device."""
    from md_nucleation_b200 import build, engine
    build.build()
    if engine.device_count() > 0:
        pytest.skip("a GPU is present (tests/test_gpu_placement.py runs the placement)")
    with pytest.raises(engine.MdnError, match="no CUDA device"):
        engine.place(100.0, np.zeros((1, 3)), 10, 0, 300.0, 300.0, 1)
    from md_nucleation_b200 import host as H
    from tests.test_host import write_case
    with pytest.raises(H.HostError, match="no CUDA device"):
        H.HostSystem(write_case(tmp_path, "nacl"), calc_number=1, place_device=0)
