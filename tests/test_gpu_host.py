"""bin/mdn_run -- the reference's command line on the engine -- end to end.

The run writes the reference's files at the reference's cadence; the frames
of its main run agree with the FP64 oracle started from the same descriptor
(the host's GPU placement for the same calculation number, as mdn_run does) through the same
re-initialisation (re-centre, rebuild, NVE): to the dump's 6 decimals on the
first frame and within 2e-5 A after 30 steps.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from md_nucleation_b200 import abi
from md_nucleation_b200 import generate as g
from tests.gpu_helpers import need_gpu

pytestmark = pytest.mark.gpu

TERMS = abi.I_GI | abi.I_GV | abi.I_VI | abi.I_VV | abi.I_BMH


@pytest.fixture(scope="module")
def host():
    need_gpu()
    from md_nucleation_b200 import host as H
    return H


def read_dump(path):
    """frames of an OVITO dump: (timestep, [(name, x, y, z, vx, vy, vz)])"""
    frames = []
    lines = open(path).read().splitlines()
    i = 0
    while i < len(lines):
        assert lines[i] == "ITEM: TIMESTEP"
        ts = int(lines[i + 1])
        n = int(lines[i + 3])
        assert lines[i + 8] == "ITEM: ATOMS id type x y z vx vy vz"
        rows = []
        for k in range(n):
            f = lines[i + 9 + k].split(" ")
            assert int(f[0]) == k
            rows.append((f[1],) + tuple(float(v) for v in f[2:]))
        frames.append((ts, rows))
        i += 9 + n
    return frames


def run_cli(host, cond, calc, replicas, cwd):
    r = subprocess.run([host.MDN_RUN, cond, str(calc), str(replicas)], cwd=cwd, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def test_mdn_run_writes_the_reference_files(host, tmp_path):
    d = str(tmp_path)
    cond = g.write_reference_inputs(os.path.join(d, "in"), g.nacl_cluster(), g.methanol(), gas="He", n_gas=2000,
                                    n_vapor=20, total_steps=100, relax_steps=60, observe=30, interactions=TERMS,
                                    nvt="scale")
    run_cli(host, cond, 5, 2, d)
    for c in (5, 6):
        frames = read_dump(os.path.join(d, "in", f"dump_{c}.dump"))
        # relaxation frames at steps 0, 30; main-run frames at 0, 30, 60, 90
        assert len(frames) == math.ceil(60 / 30) + math.ceil(100 / 30)
        for ts, rows in frames:
            assert {r[0] for r in rows[:7]} == {"Na", "Cl"}
            assert {r[0] for r in rows[7:]} <= {"He(g)", "C(v)", "O(v)", "H(v)"}
        K = np.loadtxt(os.path.join(d, f"K_{c}.dat"))
        U = np.loadtxt(os.path.join(d, f"U_{c}.dat"))
        assert K.shape == (6, 5) and U.shape == (6, 9)
        assert np.allclose(K[:, 4], K[:, 1:4].sum(axis=1))
        ion = np.loadtxt(os.path.join(d, f"ion_300_{c}.dat"), ndmin=2)
        assert ion.shape == (1, 7)
        for name in (f"vapor_in_{c}.dat", f"vapor_out_{c}.dat", f"vapor_collision_{c}.dat"):
            assert os.path.exists(os.path.join(d, name))
    # main-run energies on the OBSERVE boundaries are computed (eflag), the
    # relaxation's are not (the reference never sets eflag while relaxing)
    U = np.loadtxt(os.path.join(d, "U_5.dat"))
    assert np.all(U[:2, 1:] == 0) and np.any(U[3:, 1:] != 0)


@pytest.mark.parametrize("terms", [pytest.param(TERMS, id="base"), pytest.param(TERMS | abi.I_GG, id="gg-LJ")])
def test_mdn_run_main_run_matches_oracle(host, oracle_libs, tmp_path, terms):
    """With `gg LJ` in the condition file too: the host takes the keyword
    (src/initialization/setCondition.cpp:187-189) and the engine runs it."""
    d = str(tmp_path)
    cond = g.write_reference_inputs(os.path.join(d, "in"), g.nacl_cluster(), g.methanol(), gas="He", n_gas=2000,
                                    n_vapor=20, total_steps=60, relax_steps=0, observe=30, interactions=terms)
    run_cli(host, cond, 9, 1, d)
    frames = read_dump(os.path.join(d, "in", "dump_9.dump"))
    assert len(frames) == 2
    # MD::run advances vars->time by 10000 dt before the first frame (src/run.cpp:60-63)
    assert frames[0][0] == 10000 and frames[1][0] == 10000
    s = host.HostSystem(cond, calc_number=9, place_device=0)   # the same placement as mdn_run
    o = oracle_libs.OracleReplica.from_desc(s.desc_ptr())
    o.recenter(1)      # src/run.cpp:42-53
    o.make_pair()      # src/run.cpp:54
    o.set_nvt(abi.NVT_OFF)
    dd = s.desc
    ion_t, gas_t, vap_t = (s.topology(w)["type"] for w in ("ion", "gas", "vapor"))
    mass = np.array([dd.atom_mass[t] for t in range(dd.n_atom_types)])

    def rows(st):
        t, x, v = [ion_t], [st.ion_x], [st.ion_v]
        for q in range(dd.n_gas):
            if st.region[1 + q]:
                t.append(gas_t), x.append(st.gas_ax[q]), v.append(st.gas_av[q])
        for q in range(dd.n_vapor):
            if st.region[1 + dd.n_gas + q]:
                t.append(vap_t), x.append(st.vap_ax[q]), v.append(st.vap_av[q])
        t, x, v = np.concatenate(t), np.vstack(x), np.vstack(v)
        m = mass[ion_t]
        c = (st.ion_x * m[:, None]).sum(0) / m.sum()
        return t, x - c, v

    for k, (tol_x, tol_v) in enumerate([(1e-6, 1e-6), (2e-5, 2e-6)]):
        if k:
            o.step(30)
        t, x, v = rows(o.get_state())
        got = frames[k][1]
        assert [r[0] for r in got] == [s.type_name(int(q)) for q in t]
        gx = np.array([r[1:4] for r in got])
        gv = np.array([r[4:7] for r in got])
        assert np.abs(gx - x).max() <= tol_x + 5e-7, f"frame {k}"
        assert np.abs(gv - v).max() <= tol_v + 5e-7, f"frame {k}"


@pytest.mark.parametrize("nvt", ["scale", "330"])
def test_mdn_run_relaxation_matches_oracle(host, oracle_libs, tmp_path, nvt):
    """RelaxSteps > 0 with NVTion scale or Nose-Hoover (src/run.cpp:22-30),
    then the re-centring and rebuild (src/run.cpp:42-54, the reference's
    shift quirk) and the NVE main run: every frame against the oracle driven
    through the same sequence."""
    d = str(tmp_path)
    cond = g.write_reference_inputs(os.path.join(d, "in"), g.nacl_cluster(), g.methanol(), gas="He", n_gas=2000,
                                    n_vapor=20, total_steps=60, relax_steps=60, observe=30, interactions=TERMS,
                                    nvt=nvt)
    run_cli(host, cond, 4, 1, d)
    frames = read_dump(os.path.join(d, "in", "dump_4.dump"))
    assert len(frames) == 4
    s = host.HostSystem(cond, calc_number=4, place_device=0)
    o = oracle_libs.OracleReplica.from_desc(s.desc_ptr())
    dd = s.desc
    assert dd.nvt_mode == (abi.NVT_SCALE if nvt == "scale" else abi.NVT_NH)
    ion_t, gas_t, vap_t = (s.topology(w)["type"] for w in ("ion", "gas", "vapor"))
    mass = np.array([dd.atom_mass[t] for t in range(dd.n_atom_types)])

    def rows(st):
        t, x, v = [ion_t], [st.ion_x], [st.ion_v]
        for q in range(dd.n_gas):
            if st.region[1 + q]:
                t.append(gas_t), x.append(st.gas_ax[q]), v.append(st.gas_av[q])
        for q in range(dd.n_vapor):
            if st.region[1 + dd.n_gas + q]:
                t.append(vap_t), x.append(st.vap_ax[q]), v.append(st.vap_av[q])
        t, x, v = np.concatenate(t), np.vstack(x), np.vstack(v)
        m = mass[ion_t]
        c = (st.ion_x * m[:, None]).sum(0) / m.sum()
        return t, x - c, v

    def check(k, tol):
        t, x, v = rows(o.get_state())
        got = frames[k][1]
        assert [r[0] for r in got] == [s.type_name(int(q)) for q in t], f"frame {k}: rows differ"
        gx = np.array([r[1:4] for r in got])
        gv = np.array([r[4:7] for r in got])
        assert np.abs(gx - x).max() <= tol + 5e-7, f"frame {k}"
        assert np.abs(gv - v).max() <= 0.1 * tol + 5e-7, f"frame {k}"

    check(0, 1e-6)           # relaxation, step 0
    o.step(30)
    check(1, 2e-5)           # relaxation, step 30
    o.step(30)
    o.recenter(1)            # src/run.cpp:42-53
    o.make_pair()            # src/run.cpp:54
    o.set_nvt(abi.NVT_OFF)   # src/run.cpp:56
    check(2, 5e-5)           # main run, step 0
    o.step(30)
    check(3, 1e-4)           # main run, step 30
