"""The C++ host (lib/libmdn_host.so) against the reference's own routines.

  * condition, ion and vapor files: what the host reads equals what
    MD::readCondFile, Variables::readIonFile and Variables::readVaporFile
    store (oracle/ref_harness.cpp: ref_read_inputs), field by field, exactly;
  * initial placement: every centre farther than 10 A (minimum image) from
    the ion atoms and the origin (src/initialization/initializationGas.cpp:44-54),
    velocities Maxwell-Boltzmann;
  * dump frames: the host's writer reproduces MD::export_dump_close
    (src/output/output.cpp:133-170) byte for byte on the same state.
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from md_nucleation_b200 import abi, build
from md_nucleation_b200 import generate as g

KB = 1.38e-23
NW = 6.02e23


@pytest.fixture(scope="module")
def host():
    build.build()
    from md_nucleation_b200 import host as H
    return H


def write_case(tmp, name):
    """Two systems in the reference's formats: NaCl / methanol / He with BMH,
    and a chain / water / N2 with AMBER and SHAKE H."""
    d = os.path.join(str(tmp), name)
    if name == "nacl":
        I = abi.I_GI | abi.I_GV | abi.I_VI | abi.I_VV | abi.I_BMH
        return g.write_reference_inputs(d, g.nacl_cluster(), g.methanol(), gas="He", n_gas=2000, n_vapor=20,
                                        T=300.0, p=1e5, dt=1.0, total_steps=400, relax_steps=100, observe=50,
                                        interactions=I, shake_h=False, nvt="scale")
    rng = np.random.default_rng(5)
    I = abi.I_GI | abi.I_GV | abi.I_VI | abi.I_VV | abi.I_AMBER
    return g.write_reference_inputs(d, g.chain(30, 1.0, rng), g.water(), gas="N2", n_gas=3000, n_vapor=30,
                                    T=310.0, p=2e5, dt=0.5, total_steps=1000, relax_steps=0, observe=100,
                                    interactions=I, shake_h=True, nvt="320", efield=(0.0, 0.0, 0.01))


def ref_inputs(ref_bind, cond, calc):
    L = ref_bind.ref_lib()
    f = L.ref_read_inputs
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int]
    buf = C.create_string_buffer(1 << 22)
    n = f(cond.encode(), calc, buf, len(buf))
    assert n > 0
    return json.loads(buf.value.decode())


@pytest.mark.parametrize("case", ["nacl", "chain"])
def test_inputs_match_reference_readers(host, ref_bind, tmp_path, case, capfd):
    cond = write_case(tmp_path, case)
    ref = ref_inputs(ref_bind, cond, 3)
    capfd.readouterr()  # the reference's readers print their settings
    s = host.HostSystem(cond, calc_number=3)
    st, d = s.settings, s.desc
    # run parameters (src/initialization/setCondition.cpp:119-157, 247)
    assert d.temperature == ref["T"] and st.pressure == ref["p"] and d.dt == ref["dt"]
    assert d.cutoff == ref["cutoff"] and d.margin == ref["margin"] and d.box == ref["box"]
    assert st.total_steps == ref["total"] and st.relax_steps == ref["relax"] and st.observe == ref["observe"]
    assert d.gas_kind == ref["gastype"] and d.n_gas == ref["n_gas"] and d.n_vapor == ref["n_vapor"]
    assert s.dump_path == ref["dump_path"]
    fl = ref["flags"]
    I = d.interactions
    for bit, name in [(abi.I_GI, "force_lj"), (abi.I_VI, "inter_vi"), (abi.I_VV, "inter_vv"),
                      (abi.I_GV, "inter_vg"), (abi.I_GG, "inter_gg"), (abi.I_AMBER, "intra_AMBER"),
                      (abi.I_BMH, "force_born"), (abi.I_EFIELD, "efield"), (abi.I_GAS_INTRA, "gas_intra"),
                      (abi.I_VAPOR_INTRA, "vapor_intra"), (abi.I_SHAKE, "shakeH")]:
        assert bool(I & bit) == bool(fl[name]), name
    mode = abi.NVT_NH if fl["nose_hoover_ion"] else abi.NVT_SCALE if fl["velocity_scaling"] else abi.NVT_OFF
    assert d.nvt_mode == mode
    if mode == abi.NVT_NH:
        assert d.nvt_temperature == ref["Tnh_ion"]
    assert list(d.efield) == ref["Ecoeff"]
    # type tables, in the reference's order (gas, ion, vapor)
    nt = d.n_atom_types
    assert nt == len(ref["atypes"])
    for t, (name, m, e, sg) in enumerate(ref["atypes"]):
        assert s.type_name(t) == name
        assert (d.atom_mass[t], d.atom_eps[t], d.atom_sigma[t]) == (m, e, sg)
    assert [[d.bond_coeff[2 * b], d.bond_coeff[2 * b + 1]] for b in range(d.n_bond_types)] == ref["btypes"]
    assert [[d.angle_coeff[2 * a], d.angle_coeff[2 * a + 1]] for a in range(d.n_angle_types)] == ref["ctypes"]
    dt = [[float(d.dihedral_multi[k])] + [d.dihedral_coeff[15 * k + j] for j in range(15)]
          for k in range(d.n_dihedral_types)]
    assert dt == ref["dtypes"]
    # molecules: the host turns the ion about the origin (Variables::ionInitial),
    # so the ion is compared by its internal distances
    for which, key in (("ion", "ion"), ("vapor", "vapor"), ("gas", "gas")):
        top, r = s.topology(which), ref[key]
        assert top["type"].tolist() == r["type"], which
        assert top["charge"].tolist() == r["charge"], which
        rx = np.array(r["x"], float).reshape(-1, 3)
        if which == "ion":
            dh = np.linalg.norm(top["x"][:, None] - top["x"][None], axis=2)
            dr = np.linalg.norm(rx[:, None] - rx[None], axis=2)
            assert np.allclose(dh, dr, rtol=0, atol=1e-11)
        else:
            assert np.array_equal(top["x"], rx), which
        for part in ("bonds", "rigid", "angles", "dihedrals"):
            if part not in r:
                continue
            assert top[part].tolist() == [[int(v) for v in row] for row in r[part]], f"{which} {part}"


def test_placement_follows_the_reference_rule(host, tmp_path):
    cond = write_case(tmp_path, "nacl")
    s = host.HostSystem(cond, calc_number=1)
    d = s.desc
    L = d.box
    ion = s.topology("ion")["x"]
    for n, px, pv, mass in ((d.n_gas, d.gas_x, d.gas_v, d.gas_mb_mass),
                            (d.n_vapor, d.vapor_x, d.vapor_v, d.vapor_mb_mass)):
        X = np.ctypeslib.as_array(px, shape=(3 * n,)).reshape(-1, 3)
        V = np.ctypeslib.as_array(pv, shape=(3 * n,)).reshape(-1, 3)
        assert np.all(np.abs(X) <= L / 2)
        for c in np.vstack([ion, np.zeros((1, 3))]):
            dd = X - c
            dd -= L * np.round(dd / L)
            assert np.linalg.norm(dd, axis=1).min() > 10.0
        sigma = math.sqrt(KB * d.temperature / mass) * 1e-5
        assert abs(V.std() / sigma - 1) < 0.1
    # the same calculation number gives the same system; another one does not
    s2 = host.HostSystem(cond, calc_number=1)
    s3 = host.HostSystem(cond, calc_number=2)
    x1 = np.ctypeslib.as_array(d.gas_x, shape=(3 * d.n_gas,))
    assert np.array_equal(x1, np.ctypeslib.as_array(s2.desc.gas_x, shape=(3 * d.n_gas,)))
    assert not np.array_equal(x1, np.ctypeslib.as_array(s3.desc.gas_x, shape=(3 * d.n_gas,)))


def test_dump_frame_matches_export_dump_close(host, ref_bind, tmp_path, capfd):
    """One frame of the reference's dump and of the host's writer, from the
    same state: the reference replica built from the host's descriptor."""
    cond = write_case(tmp_path, "nacl")
    s = host.HostSystem(cond, calc_number=4)
    L = ref_bind.ref_lib()
    L.ref_create.argtypes = [C.POINTER(abi.ReplicaDesc), C.c_int]
    h = L.ref_create(s.desc_ptr(), 1)
    capfd.readouterr()
    ref_path = os.path.join(str(tmp_path), "ref.dump")
    L.ref_export_dump(h, ref_path.encode(), 1234.9)
    # the frame's rows: in-domain atoms, molecule order (ion, gas, vapor)
    from md_nucleation_b200.system import StateArrays
    d = s.desc
    state = StateArrays(d.ion.n_atoms, d.gas.n_atoms, d.vapor.n_atoms, d.n_gas, d.n_vapor)
    cs = state.to_c()
    L.ref_get_state(h, C.byref(cs))
    state.pull_scalars(cs)
    rows_t, rows_x, rows_v = [], [], []
    ion_t = s.topology("ion")["type"]
    rows_t += ion_t.tolist()
    rows_x.append(state.ion_x.reshape(-1, 3))
    rows_v.append(state.ion_v.reshape(-1, 3))
    gt, vt = s.topology("gas")["type"], s.topology("vapor")["type"]
    for q in range(d.n_gas):
        if state.region[1 + q]:
            rows_t += gt.tolist()
            rows_x.append(state.gas_ax[q].reshape(-1, 3))
            rows_v.append(state.gas_av[q].reshape(-1, 3))
    for q in range(d.n_vapor):
        if state.region[1 + d.n_gas + q]:
            rows_t += vt.tolist()
            rows_x.append(state.vap_ax[q].reshape(-1, 3))
            rows_v.append(state.vap_av[q].reshape(-1, 3))
    mine = os.path.join(str(tmp_path), "host.dump")
    s.write_dump_frame(mine, 1234, np.array(rows_t), np.vstack(rows_x), np.vstack(rows_v),
                       shift=state.mol_x[0])
    L.ref_destroy(h)
    ref_lines = open(ref_path).read().splitlines()
    my_lines = open(mine).read().splitlines()
    assert len(ref_lines) == len(my_lines) and len(my_lines) > 9 + d.ion.n_atoms
    # the harness names type t "T<t>"; the host prints the file's names
    for a, b in zip(ref_lines, my_lines):
        fa, fb = a.split(" "), b.split(" ")
        if len(fa) == 8 and fa[1].startswith("T"):
            fa[1] = s.type_name(int(fa[1][1:]))
        assert fa == fb


def test_errors_are_reported(host, tmp_path):
    cond = write_case(tmp_path, "nacl")
    text = open(cond).read()
    bad = os.path.join(str(tmp_path), "bad.txt")
    with open(bad, "w") as f:
        f.write(text.replace("Gas He 2000", "Gas Xe 2000"))
    with pytest.raises(host.HostError, match="unknown gas Xe"):
        host.HostSystem(bad)
    with open(bad, "w") as f:
        f.write(text.replace(" ion Born-Mayer-Huggins-NaCl", " ion Tersoff"))
    with pytest.raises(host.HostError, match="unsupported ion potential"):
        host.HostSystem(bad)
    with pytest.raises(host.HostError, match="cannot open"):
        host.HostSystem(os.path.join(str(tmp_path), "missing.txt"))


def test_mdn_run_fails_loudly_without_a_gpu(host, tmp_path):
    from md_nucleation_b200 import engine
    if engine.device_count() > 0:
        pytest.skip("a GPU is present (the GPU tests run the command line)")
    import subprocess
    cond = write_case(tmp_path, "nacl")
    r = subprocess.run([host.MDN_RUN, cond, "1", "1"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "no CUDA device" in r.stderr
