"""The committed golden vectors (tests/golden/*.npz, written by
tests/golden/make_golden.py from the reference program's own routines)
against the FP64 restatement on the CPU and the CUDA engine on the GPU.

The restatement reproduces them bit for bit: forces and energies of each
Potential, and 20 MD::verlet steps.  The engine reproduces the forces within
the FP32 pair-term tolerance of the parity tests (1e-5 relative RMS) and the
20-step trajectory within 1e-6 A.
"""
import os

import numpy as np
import pytest

from md_nucleation_b200.system import StateArrays
from tests import systems
from tests.golden.make_golden import NAMES, TERMS, VERLET_STEPS, spec_digest
from tests.gpu_helpers import FORCE_ATOL, FORCE_RTOL, rel_rms

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    g = np.load(os.path.join(HERE, f"{name}.npz"))
    spec = systems.make(name)
    assert str(g["digest"]) == spec_digest(spec), "the system generator no longer makes the golden system"
    return g, spec


def unpack(g, spec, prefix) -> StateArrays:
    st = StateArrays.for_spec(spec)
    st.region[:] = g[prefix + "region"]
    st.mol_x[:] = g[prefix + "mol_x"]
    st.mol_v[:] = g[prefix + "mol_v"]
    for k in ("ion_x", "ion_v", "ion_f"):
        getattr(st, k)[:] = g[prefix + k]
    gm = st.region[1:1 + spec.n_gas].astype(bool)
    vm = st.region[1 + spec.n_gas:].astype(bool)
    for k in ("gas_ax", "gas_av", "gas_af"):
        getattr(st, k)[gm] = g[prefix + k]
    for k in ("vap_ax", "vap_av", "vap_af", "vap_w"):
        getattr(st, k)[vm] = g[prefix + k]
    st.loop_pair, st.loop_update = (int(v) for v in g[prefix + "loop"])
    st.zeta, st.margin_length = (float(v) for v in g[prefix + "scalars"])
    return st


def forces(st, spec):
    gm = st.region[1:1 + spec.n_gas].astype(bool)
    vm = st.region[1 + spec.n_gas:].astype(bool)
    return st.ion_f.copy(), st.gas_af[gm].copy(), st.vap_af[vm].copy()


def golden_forces(g, term):
    return g[f"f_{term}_ion"], g[f"f_{term}_gas"], g[f"f_{term}_vap"]


def terms_of(g):
    return [t for t in TERMS if f"u_{t}" in g.files]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden_forces(oracle_libs, name):
    g, spec = load(name)
    st0 = unpack(g, spec, "state_")
    o = oracle_libs.OracleReplica(spec)
    for term in terms_of(g):
        o.set_state(st0)
        U = o.compute_forces(TERMS[term])
        assert np.array_equal(U, g[f"u_{term}"]), term
        for a, b in zip(forces(o.get_state(), spec), golden_forces(g, term)):
            assert np.array_equal(a, b), term


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden_verlet(oracle_libs, name):
    g, spec = load(name)
    st = unpack(g, spec, "state_")
    st.loop_pair, st.loop_update = 0, 10 ** 6
    o = oracle_libs.OracleReplica(spec)
    o.set_state(st)
    o.step(VERLET_STEPS, energy_mode=1)
    want = unpack(g, spec, "verlet_")
    got = o.get_state()
    for k in ("ion_x", "ion_v", "mol_x", "mol_v"):
        assert np.array_equal(getattr(got, k)[:1] if k.startswith("mol") else getattr(got, k),
                              getattr(want, k)[:1] if k.startswith("mol") else getattr(want, k)), k
    gm = want.region[1:1 + spec.n_gas].astype(bool)
    vm = want.region[1 + spec.n_gas:].astype(bool)
    assert np.array_equal(got.gas_ax[gm], want.gas_ax[gm])
    assert np.array_equal(got.vap_ax[vm], want.vap_ax[vm])
    assert np.array_equal(o.energies(), g["verlet_u"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_engine_matches_golden(name):
    from tests.gpu_helpers import need_gpu
    eng = need_gpu()
    g, spec = load(name)
    st0 = unpack(g, spec, "state_")
    e = eng.Engine([spec])
    for term in terms_of(g):
        e.upload(0, st0)
        e.compute_forces(TERMS[term])
        fe = np.concatenate([a.reshape(-1, 3) for a in forces(e.state(0), spec)])
        fg = np.concatenate([a.reshape(-1, 3) for a in golden_forces(g, term)])
        if np.abs(fg).max() == 0:
            assert np.abs(fe).max() == 0
            continue
        err = rel_rms(fe, fg)
        rms = np.sqrt(np.mean((fe - fg) ** 2))
        assert err <= FORCE_RTOL or rms <= FORCE_ATOL, f"{term}: relative RMS {err:.2e}"
        Ug = g[f"u_{term}"]
        assert np.all(np.abs(e.energies()[0] - Ug) <= 1e-4 * max(np.abs(Ug).max(), 1e-3) + 1e-6), term
    st = st0.copy()
    st.loop_pair, st.loop_update = 0, 10 ** 6
    e.upload(0, st)
    e.step(VERLET_STEPS, energy_mode=1)
    want = unpack(g, spec, "verlet_")
    got = e.state(0)
    gm = want.region[1:1 + spec.n_gas].astype(bool)
    vm = want.region[1 + spec.n_gas:].astype(bool)
    assert np.abs(got.ion_x - want.ion_x).max() <= 1e-6
    assert np.abs(got.gas_ax[gm] - want.gas_ax[gm]).max() <= 1e-6
    assert np.abs(got.vap_ax[vm] - want.vap_ax[vm]).max() <= 1e-6
