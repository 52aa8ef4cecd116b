"""The FP64 CPU adjoint of the gradient harness (oracle/adjoint_ad.h:
reverse-mode differentiation of the window's steps on a tape) on the CPU.

It is the reference point of the engine's hand-written adjoint
(tests/test_gpu_adjoint.py), so it is checked here on its own: its forward
window equals orc_window's exactly (same expressions, same order), and its
gradient agrees with FP64 central differences of orc_window within 1e-4
relative (h = 1e-4 relative; 1e-3 with SHAKE, whose 1e-20 A^4 convergence
tolerance blurs smaller steps), per parameter, below 1e-3 of the largest
derivative (1e-2 with SHAKE) within 1e-4 of that floor.
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from md_nucleation_b200 import generate as g
from md_nucleation_b200.gradients import apply

KW = dict(R0=40.0, W=5.0, w_energy=1.0, w_count=1.0)


def params(spec):
    """theta0 and rows in mdn_adjoint_params order (gas-ion then vapor-ion
    type pairs, ascending types, then the ion charge scale)"""
    gt, it, vt = (sorted(set(t.type.tolist())) for t in (spec.gas, spec.ion, spec.vapor))
    rows = []
    if spec.interactions & abi.I_GI:
        rows += [(0, a, b) for a in gt for b in it]
    if spec.interactions & abi.I_VI:
        rows += [(1, a, b) for a in vt for b in it]
    rows.append((2, 0, 0))
    eps, sig = spec.pair_parameters()
    th = [x for (_, a, b) in rows[:-1] for x in (eps[a, b], sig[a, b])] + [1.0]
    return np.array(th), np.array(rows, np.int32)


def system(shake):
    spec = g.small_system(seed=31, gas="N2", vapor="methanol", ion="nacl", n_gas=1500, n_vap=40, box=220.0,
                          shake_h=shake, rigid_gas=shake)
    spec.margin = 80.0
    return spec


@pytest.mark.parametrize("shake", [False, True])
def test_cpu_adjoint_matches_differences(oracle_libs, shake):
    spec = system(shake)
    th, rows = params(spec)
    n = 60
    J, grad = oracle_libs.OracleReplica(spec).adjoint(n, th, rows, **KW)
    Jw = oracle_libs.OracleReplica(spec).window(n, KW["R0"], KW["W"], KW["w_energy"], KW["w_count"])
    assert J == Jw
    rel = 1e-3 if shake else 1e-4
    fd = np.zeros(len(th))
    for k in range(len(th)):
        h = rel * abs(th[k])
        Js = []
        for sgn in (1, -1):
            t = th.copy()
            t[k] += sgn * h
            Js.append(oracle_libs.OracleReplica(apply(spec, t, rows)).window(n, KW["R0"], KW["W"], KW["w_energy"],
                                                                             KW["w_count"]))
        fd[k] = (Js[0] - Js[1]) / (2 * h)
    floor = (1e-2 if shake else 1e-3) * np.abs(fd).max()
    for k in range(len(th)):
        assert abs(grad[k] - fd[k]) <= 1e-4 * max(abs(fd[k]), floor), f"parameter {k}: {grad[k]} vs {fd[k]}"


def test_cpu_adjoint_from_a_stepped_state(oracle_libs):
    """After some steps the start forces F(x_0; theta) carry parameter
    dependence: the derivative through them is included."""
    spec = system(False)
    th, rows = params(spec)
    o = oracle_libs.OracleReplica(spec)
    o.step(15)
    st = o.get_state()
    J, grad = o.adjoint(40, th, rows, **KW)
    fd = np.zeros(len(th))
    for k in range(len(th)):
        h = 1e-4 * abs(th[k])
        Js = []
        for sgn in (1, -1):
            t = th.copy()
            t[k] += sgn * h
            q = oracle_libs.OracleReplica(apply(spec, t, rows))
            q.step(15)
            q.set_state(st)
            q.compute_forces(0)
            Js.append(q.window(40, KW["R0"], KW["W"], KW["w_energy"], KW["w_count"]))
        fd[k] = (Js[0] - Js[1]) / (2 * h)
    floor = 1e-3 * np.abs(fd).max()
    for k in range(len(th)):
        assert abs(grad[k] - fd[k]) <= 1e-4 * max(abs(fd[k]), floor), f"parameter {k}: {grad[k]} vs {fd[k]}"


def test_cpu_adjoint_refuses_a_window_across_a_rebuild(oracle_libs):
    spec = system(False)
    spec.margin = 10.0
    th, rows = params(spec)
    with pytest.raises(RuntimeError):
        oracle_libs.OracleReplica(spec).adjoint(100000, th, rows, **KW)
