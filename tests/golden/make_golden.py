"""Writes tests/golden/<system>.npz from the reference program's own routines.

The reference is compiled from its sources into oracle/_ref/libref_harness.so
by oracle/Makefile (oracle/ref_harness.cpp drives single routines of a real
MD object).  For each small seeded system of tests/systems.py this records:

  * the state MD::make_pair leaves (src/pairList/pairlist.cpp:16-49): molecule
    centres and flags of every molecule, atoms of the in-domain ones;
  * the forces and energies of each Potential alone and of all together
    (Potential::compute, src/verlet.cpp:31-32);
  * the state and energies after 20 MD::verlet steps (src/verlet.cpp:20-39)
    started from it with the rebuild pushed past the window.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from md_nucleation_b200 import abi  # noqa: E402
from oracle import bind  # noqa: E402
from tests import systems  # noqa: E402

TERMS = {"all": 0, "gi": abi.I_GI, "vi": abi.I_VI, "vv": abi.I_VV, "gv": abi.I_GV, "amber": abi.I_AMBER,
         "bmh": abi.I_BMH, "gas_intra": abi.I_GAS_INTRA, "vapor_intra": abi.I_VAPOR_INTRA}
NAMES = ["nacl_n2_meoh", "chain_he_water", "nacl_n2mono_meoh"]
VERLET_STEPS = 20


def spec_digest(spec) -> str:
    """A fingerprint of the generated system, to detect generator drift."""
    h = hashlib.sha256()
    for a in (spec.gas_x, spec.gas_v, spec.vapor_x, spec.vapor_v, spec.ion.x, spec.ion_v):
        h.update(np.ascontiguousarray(a, np.float64).tobytes())
    return h.hexdigest()


def pack(st, spec):
    """The in-domain part of a state (the rows the dynamics reads)."""
    g = st.region[1:1 + spec.n_gas].astype(bool)
    v = st.region[1 + spec.n_gas:].astype(bool)
    return {"region": st.region.copy(), "mol_x": st.mol_x.copy(), "mol_v": st.mol_v.copy(),
            "ion_x": st.ion_x.copy(), "ion_v": st.ion_v.copy(), "ion_f": st.ion_f.copy(),
            "gas_ax": st.gas_ax[g].copy(), "gas_av": st.gas_av[g].copy(), "gas_af": st.gas_af[g].copy(),
            "vap_ax": st.vap_ax[v].copy(), "vap_av": st.vap_av[v].copy(), "vap_af": st.vap_af[v].copy(),
            "vap_w": st.vap_w[v].copy(),
            "loop": np.array([st.loop_pair, st.loop_update], np.int64),
            "scalars": np.array([st.zeta, st.margin_length])}


def main():
    if not bind.have_reference():
        raise SystemExit("oracle/_ref/libref_harness.so is not built (make -C oracle reference)")
    for name in NAMES:
        spec = systems.make(name)
        r = bind.RefReplica(spec)
        st0 = r.get_state()
        out = {"digest": np.array(spec_digest(spec))}
        for k, v in pack(st0, spec).items():
            out["state_" + k] = v
        for term, mask in TERMS.items():
            if mask and not spec.interactions & mask:
                continue
            r.set_state(st0)
            U = r.compute_forces(mask)
            st = r.get_state()
            p = pack(st, spec)
            out[f"f_{term}_ion"] = p["ion_f"]
            out[f"f_{term}_gas"] = p["gas_af"]
            out[f"f_{term}_vap"] = p["vap_af"]
            out[f"u_{term}"] = U
        st = st0.copy()
        st.loop_pair, st.loop_update = 0, 10 ** 6
        r.set_state(st)
        U = r.verlet(VERLET_STEPS, energy_mode=1)
        for k, v in pack(r.get_state(), spec).items():
            out["verlet_" + k] = v
        out["verlet_u"] = U
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KB")


if __name__ == "__main__":
    main()
