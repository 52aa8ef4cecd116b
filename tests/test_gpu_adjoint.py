"""mdn_adjoint (the gradient harness) against FP64 central differences.

The objective is the window average of U_vi + the smooth vapor count
(mdn.h); the parameters are (eps, sigma) of every gas-ion and vapor-ion type
pair and the ion charge scale.  The differences come from the FP64
restatement (oracle/mdn_oracle.cpp: orc_window, whose forces are pinned bit
for bit to the reference's routines) run from the same initial state with
the parameters moved by +-h, h = 1e-4 relative: at 1e-6 a move changes J by
~1e-14 for the weakest (gas-ion) parameters, which the window's FP64
rounding already blurs; at 1e-4 the truncation error is ~1e-8 relative.

Bars: with the engine's FP64 pair arithmetic (force_mode 1) the forward
trajectory is the oracle's, and every derivative agrees within 1e-4
relative (per parameter; below 1e-3 of the largest derivative, 1e-2 with
SHAKE, within 1e-4 of that floor); with the default FP32 pair terms within
1e-2.
"""
import numpy as np
import pytest

from md_nucleation_b200 import abi
from md_nucleation_b200 import generate as g
from tests.gpu_helpers import need_gpu

pytestmark = pytest.mark.gpu

WINDOW = dict(n_steps=150, checkpoint_every=50, count_radius=40.0, count_width=5.0, w_energy=1.0, w_count=1.0)


@pytest.fixture(scope="module")
def eng():
    return need_gpu()


def system(shake):
    spec = g.small_system(seed=31, gas="N2", vapor="methanol", ion="nacl", n_gas=1500, n_vap=40, box=220.0,
                          shake_h=shake, rigid_gas=shake)
    spec.margin = 80.0  # no effective-domain rebuild inside the window
    return spec


def finite_differences(oracle_libs, spec, theta0, rows, rel=1e-4, start=None):
    """Central differences of the oracle's window objective; `start` (a
    state) replaces the initial make_pair's state, with its forces evaluated
    at the moved parameters."""
    from md_nucleation_b200.gradients import apply
    n = len(theta0)
    out = np.zeros(n)
    kw = dict(R0=WINDOW["count_radius"], W=WINDOW["count_width"], w_energy=WINDOW["w_energy"],
              w_count=WINDOW["w_count"])
    for k in range(n):
        h = rel * abs(theta0[k])
        J = []
        for sgn in (1, -1):
            th = theta0.copy()
            th[k] += sgn * h
            o = oracle_libs.OracleReplica(apply(spec, th, rows))
            if start is not None:
                o.set_state(start)
                o.compute_forces(0)
            J.append(o.window(WINDOW["n_steps"], **kw))
        out[k] = (J[0] - J[1]) / (2 * h)
    return out


def check(grad, fd, tol, floor=1e-3):
    scale = np.abs(fd).max()
    assert scale > 0
    for k in range(len(fd)):
        den = max(abs(fd[k]), floor * scale)
        assert abs(grad[k] - fd[k]) <= tol * den, f"parameter {k}: adjoint {grad[k]:.8e} fd {fd[k]:.8e}"


@pytest.mark.parametrize("shake", [False, True])
def test_adjoint_matches_fp64_differences(eng, oracle_libs, shake):
    from md_nucleation_b200.gradients import parameters
    spec = system(shake)
    theta0, rows = parameters(spec)
    theta0 = theta0.numpy()
    e = eng.Engine([spec], force_mode=1)
    assert e.info(0).n_vapor_in >= 3
    J, grad, ms = e.adjoint(**WINDOW)
    o = oracle_libs.OracleReplica(spec)
    Jo = o.window(WINDOW["n_steps"], WINDOW["count_radius"], WINDOW["count_width"], WINDOW["w_energy"],
                  WINDOW["w_count"])
    assert abs(J - Jo) <= 1e-8 * max(abs(Jo), 1.0)
    # SHAKE stops at (s^2 - d^2)^2 <= 1e-20 A^4: positions carry ~1e-10 A of
    # convergence noise that is not smooth in theta (~1e-13 in J), so the
    # differences take a 1e-3 step there (truncation ~1e-6 relative) and the
    # weakest derivatives are held to 1e-2 of the largest one
    fd = finite_differences(oracle_libs, spec, theta0, rows, rel=1e-3 if shake else 1e-4)
    check(grad, fd, 1e-4, floor=1e-2 if shake else 1e-3)


def test_adjoint_from_a_stepped_state(eng, oracle_libs):
    """After 20 steps the start forces are F(x_0; theta) and enter the gradient."""
    from md_nucleation_b200.gradients import parameters
    spec = system(False)
    theta0, rows = parameters(spec)
    e = eng.Engine([spec], force_mode=1)
    e.step(20)
    st0 = e.state(0)
    J, grad, ms = e.adjoint(**WINDOW)
    fd = finite_differences(oracle_libs, spec, theta0.numpy(), rows, start=st0)
    check(grad, fd, 1e-4)


def test_adjoint_on_the_fp32_forward(eng, oracle_libs):
    from md_nucleation_b200.gradients import parameters
    spec = system(False)
    theta0, rows = parameters(spec)
    e = eng.Engine([spec])
    J, grad, ms = e.adjoint(**WINDOW)
    fd = finite_differences(oracle_libs, spec, theta0.numpy(), rows)
    check(grad, fd, 1e-2)


def test_window_across_a_rebuild_is_refused(eng):
    spec = system(False)
    spec.margin = 10.0
    e = eng.Engine([spec])
    with pytest.raises(eng.MdnError, match="crosses the rebuild"):
        e.adjoint(n_steps=100000, checkpoint_every=100)


def test_torch_harness_returns_the_adjoint(eng):
    import torch
    from md_nucleation_b200.gradients import parameters, window_objective
    spec = system(False)
    theta0, rows = parameters(spec)
    theta = theta0.clone().requires_grad_()
    J = window_objective(theta, spec, rows, engine_options={"force_mode": 1}, **WINDOW)
    J.backward()
    e = eng.Engine([spec], force_mode=1)
    J2, grad, _ = e.adjoint(**WINDOW)
    assert abs(J.item() - J2) <= 1e-12 * max(abs(J2), 1.0)
    # the reverse sweep sums x-bar and the parameter rows with FP64 atomics
    # from several CTAs, whose order varies from run to run: two runs agree
    # to FP64 rounding of those sums, not bit for bit
    g = torch.tensor(grad)
    assert torch.allclose(theta.grad, g, rtol=1e-9, atol=1e-9 * float(g.abs().max()))


CONFIG3_WINDOW = dict(n_steps=300, checkpoint_every=100, count_radius=10.0, count_width=1.0, w_energy=1.0,
                      w_count=1.0)


def test_adjoint_on_the_config3_window(eng, oracle_libs):
    """The bench's adjoint system (configuration 1 with 8 methanol started
    8-28 A from the chain): J is not zero, and with the FP64 forward every
    derivative agrees with FP64 central differences within 1e-4 (1e-3 steps
    and a 1e-2 floor: the system carries SHAKE, see above)."""
    from md_nucleation_b200.gradients import apply, parameters
    spec = g.config3(0)
    theta0, rows = parameters(spec)
    theta0 = theta0.numpy()
    e = eng.Engine([spec], force_mode=1)
    assert e.info(0).n_vapor_in >= 8
    J, grad, ms = e.adjoint(**CONFIG3_WINDOW)
    assert J < -0.1 and np.abs(grad).max() > 0
    w = CONFIG3_WINDOW
    fd = np.zeros(len(theta0))
    for k in range(len(theta0)):
        h = 1e-3 * abs(theta0[k])
        Jk = []
        for sgn in (1, -1):
            th = theta0.copy()
            th[k] += sgn * h
            o = oracle_libs.OracleReplica(apply(spec, th, rows))
            Jk.append(o.window(w["n_steps"], w["count_radius"], w["count_width"], w["w_energy"], w["w_count"]))
        fd[k] = (Jk[0] - Jk[1]) / (2 * h)
    check(grad, fd, 1e-4, floor=1e-2)


@pytest.mark.parametrize("shake", [False, True])
def test_adjoint_matches_the_cpu_adjoint(eng, oracle_libs, shake):
    """The engine's adjoint (hand-written transposes, the adjoint of the
    converged SHAKE projection) against the FP64 CPU adjoint (reverse-mode
    differentiation of the oracle's step, oracle/adjoint_ad.h) on the same
    window with the FP64 forward: J within 1e-9 and every derivative within
    1e-6 relative (1e-5 with SHAKE, differentiated through its iterations on
    the CPU), below 1e-4 of the largest within 1e-6 of that floor."""
    from md_nucleation_b200.gradients import parameters
    spec = system(shake)
    theta0, rows = parameters(spec)
    e = eng.Engine([spec], force_mode=1)
    J, grad, _ = e.adjoint(**WINDOW)
    kw = dict(R0=WINDOW["count_radius"], W=WINDOW["count_width"], w_energy=WINDOW["w_energy"],
              w_count=WINDOW["w_count"])
    Jc, gc = oracle_libs.OracleReplica(spec).adjoint(WINDOW["n_steps"], theta0.numpy(), rows, **kw)
    assert abs(J - Jc) <= 1e-9 * max(abs(Jc), 1.0)
    tol = 1e-5 if shake else 1e-6
    floor = 1e-4 * np.abs(gc).max()
    for k in range(len(gc)):
        assert abs(grad[k] - gc[k]) <= tol * max(abs(gc[k]), floor), f"parameter {k}: {grad[k]} vs {gc[k]}"
