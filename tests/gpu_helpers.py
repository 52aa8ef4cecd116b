"""Helpers of the GPU parity tests: comparisons against the FP64 oracle."""
import numpy as np
import pytest

from md_nucleation_b200 import build

FORCE_RTOL = 1e-5   # relative RMS force error bound of the FP32 pair path vs FP64
FORCE_ATOL = 1e-9   # RMS floor (kcal/mol/A) for terms whose forces vanish: a few
                    # 2^-40 fixed-point quanta per atom


def need_gpu():
    build.build()
    from md_nucleation_b200 import engine
    if engine.device_count() == 0:
        pytest.skip("no CUDA device")
    return engine


def in_masks(st, spec):
    g = st.region[1:1 + spec.n_gas].astype(bool)
    v = st.region[1 + spec.n_gas:].astype(bool)
    return g, v


def forces_of(st, spec):
    g, v = in_masks(st, spec)
    return np.concatenate([st.ion_f.reshape(-1, 3), st.gas_af[g].reshape(-1, 3), st.vap_af[v].reshape(-1, 3)])


def rel_rms(a, b):
    den = np.sqrt(np.sum(b * b))
    return np.sqrt(np.sum((a - b) ** 2)) / max(den, 1e-300)


def force_ok(a, b):
    """relative RMS <= FORCE_RTOL, or RMS error <= FORCE_ATOL when the forces
    themselves are at the fixed-point resolution"""
    err = rel_rms(a, b)
    rms = np.sqrt(np.mean((a - b) ** 2)) if a.size else 0.0
    return err <= FORCE_RTOL or rms <= FORCE_ATOL, err, rms


def compare_states(a, b, spec, xtol, vtol, what=""):
    """Positions and velocities of every in-domain atom and molecule centre."""
    if not np.array_equal(a.region, b.region):
        bad = np.nonzero(a.region != b.region)[0]
        c = b.mol_x[0]
        desc = [f"mol {m}: engine {a.region[m]} oracle {b.region[m]} "
                f"r/R_I {np.linalg.norm(b.mol_x[m] - c) / spec.r_inter:.9f}" for m in bad[:6]]
        raise AssertionError(f"{what}: region flags differ for {len(bad)} molecules: " + "; ".join(desc))
    g, v = in_masks(a, spec)
    checks = [("ion_x", a.ion_x, b.ion_x, xtol), ("ion_v", a.ion_v, b.ion_v, vtol),
              ("gas_x", a.gas_ax[g], b.gas_ax[g], xtol), ("gas_v", a.gas_av[g], b.gas_av[g], vtol),
              ("vap_x", a.vap_ax[v], b.vap_ax[v], xtol), ("vap_v", a.vap_av[v], b.vap_av[v], vtol),
              ("mol_x", a.mol_x, b.mol_x, xtol), ("mol_v", a.mol_v, b.mol_v, vtol)]
    for name, x, y, tol in checks:
        err = np.abs(x - y).max() if x.size else 0.0
        assert err <= tol, f"{what}: {name} differs by {err:.3e} (tol {tol:.1e})"
