"""Throughput of the batched replica workload: 256 independent nucleation
replicas (gas He/Ar/N2/N2-monoatomic, 5,000-100,000 molecules; methanol or
3-site water vapor, 10-300 molecules; NaCl cluster or a 50-300 atom +1 chain;
500-20,000 atoms inside each 10 nm effective domain; SHAKE on X-H bonds;
300 K, dt = 1 fs), advanced 100 MD steps per bench step by the persistent
step kernel.

metric: in-domain atom-steps per second, summed over replicas (the atoms the
reference's pair forces and dump loop visit, src/output/output.cpp:136-143).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--replicas R]
  python bench.py --impl reference ...   the reference's own CPU routines
                                         (oracle/_ref) on the host cores

Under torchrun every rank runs its own R replicas (seeds offset by rank):
weak scaling, no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "replica atom-steps/s on 1 B200, batched vs plain at force err≤1e-5; adjoint/fwd"
UNIT = "atom-steps/s"
MD_STEPS = 100          # MD steps per bench step (one bench step = one 100-step block)
WORKLOAD = "batched replicas: 256 independent systems, 100 MD steps per step"

# FP32 flops of one pair evaluation (distance, r^-2, r^-6, the LJ force
# factor; + r^-1 and the Coulomb factor; BMH: + sqrt, exp and its r^-8 and
# r^-10 terms): the algorithmic count takes each pair once.
FLOPS_LJ = 20
FLOPS_LJ_COUL = 29
FLOPS_BMH = 35


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def _make_replica(r):
    from md_nucleation_b200 import generate
    return generate.config2_replica(r)


def make_specs(first: int, n: int, workers: int, indices=None):
    """Generates the replicas first..first+n-1 (or the listed indices) in a
    spawn pool (the chain growth and the placement of up to 100,000
    molecules take seconds per replica)."""
    t0 = time.time()
    idx = list(indices) if indices is not None else list(range(first, first + n))
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(1, min(workers, len(idx)))) as pool:
        specs = pool.map(_make_replica, idx, chunksize=1)
    log(f"generated {len(idx)} replicas in {time.time() - t0:.1f} s on {workers} workers")
    return specs


def sample_indices(n_replicas: int, threads: int):
    """The replicas the CPU samples run: 2 per host thread, spread evenly
    over the batch."""
    stride = max(1, n_replicas // (2 * threads))
    return list(range(0, n_replicas, stride))[:2 * threads], stride


def in_domain_atoms(infos, specs):
    return np.array([i.n_ion + i.n_gas_in * s.gas.n + i.n_vapor_in * s.vapor.n for i, s in zip(infos, specs)],
                    np.int64)


# Algorithmic HBM bytes (the byte model of a streaming implementation):
# per in-domain atom-step 164 B of integration (read x, v FP64, fixed-point F,
# 1/m; write x, v, the float4 copy, a zeroed F) + 40 B of forces (float4 read,
# F write), 4 B per pair-list entry and step, and per rebuild 72 B per
# molecule (centre read, free flight and resampling write).
BYTES_PER_ATOM_STEP = 164 + 40
BYTES_PER_LIST_ENTRY = 4
BYTES_PER_MOLECULE_REBUILD = 72


def algorithmic_bytes(infos0, infos1, specs, md_steps):
    """Bytes of the byte model over md_steps steps of every replica."""
    b = 0.0
    for i0, i1, s in zip(infos0, infos1, specs):
        atoms = 0.5 * ((i0.n_ion + i0.n_gas_in * s.gas.n + i0.n_vapor_in * s.vapor.n) +
                       (i1.n_ion + i1.n_gas_in * s.gas.n + i1.n_vapor_in * s.vapor.n))
        lists = 0.5 * ((i0.gi_pairs + i0.gv_pairs) + (i1.gi_pairs + i1.gv_pairs))
        b += md_steps * (atoms * BYTES_PER_ATOM_STEP + lists * BYTES_PER_LIST_ENTRY)
        b += (i1.n_rebuilds - i0.n_rebuilds) * (1 + s.n_gas + s.n_vapor) * BYTES_PER_MOLECULE_REBUILD
    return b


def traffic_per_atom_step():
    """DRAM bytes (read + write) per in-domain atom-step of mdn_advance: the
    `dram_bytes_per_atom_step:` line of the ncu summary in
    profiles/mdn_advance_batched.md, or None."""
    import re
    try:
        with open(os.path.join(HERE, "profiles", "mdn_advance_batched.md")) as f:
            m = re.search(r"dram_bytes_per_atom_step:\s*([0-9.eE+-]+)", f.read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def measured_hbm_peak():
    """(GB/s, source): the copy bandwidth measured on these GPUs, else the
    earlier measurement on the same pool."""
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured copy bandwidth (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def algorithmic_flops(infos, specs):
    """FP32 flops of one MD step's pair terms, each pair once:
    gas-ion (gas atom x ion atom of listed molecule pairs, LJ), gas-vapor
    (atoms of listed molecule pairs, LJ), vapor-ion and vapor-vapor (all
    in-domain atoms, LJ + Coulomb), the ion's own non-bonded pairs (LJ +
    Coulomb for a chain, BMH for a salt cluster)."""
    from md_nucleation_b200 import abi
    tot = 0.0
    for i, s in zip(infos, specs):
        ag, av, ni = s.gas.n, s.vapor.n, i.n_ion
        vin = i.n_vapor_in * av
        f = i.gi_pairs * ag * FLOPS_LJ + i.gv_pairs * ag * av * FLOPS_LJ
        f += vin * ni * FLOPS_LJ_COUL
        f += i.n_vapor_in * (i.n_vapor_in - 1) / 2 * av * av * FLOPS_LJ_COUL
        ion_pairs = ni * (ni - 1) / 2
        f += ion_pairs * (FLOPS_BMH if s.interactions & abi.I_BMH else FLOPS_LJ_COUL)
        tot += f
    return tot


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.p is not None:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, local, backend):
    if ws == 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist


def max_over_ranks(dist, value: float, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value: float, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own routines, one replica per OpenMP thread
# ---------------------------------------------------------------------------
class stdout_to_stderr:
    """Sends file descriptor 1 to stderr: the reference's constructor prints
    its interaction table on stdout, which carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def _cpu_sample_child(specs, threads, budget_s, n_samples, q):
    import tempfile
    from oracle import bind
    # the reference's make_pair appends vapor in/out logs to the working
    # directory (src/output/output.cpp:44-65): keep them out of the tree
    os.chdir(tempfile.mkdtemp(prefix="mdn_ref_sample_"))
    with stdout_to_stderr():
        reps = [bind.RefReplica(sp) for sp in specs]
    t0 = time.perf_counter()
    bind.ref_verlet_many(reps, 5, threads)
    cal = (time.perf_counter() - t0) / 5
    n = max(5, int(budget_s / max(cal, 1e-6)))
    out = []
    for _ in range(n_samples):
        atoms0 = sum(r.in_domain_atoms() for r in reps)
        t0 = time.perf_counter()
        bind.ref_verlet_many(reps, n, threads)
        dt = time.perf_counter() - t0
        atoms1 = sum(r.in_domain_atoms() for r in reps)
        out.append((0.5 * (atoms0 + atoms1) * n / dt, n, atoms0, dt))
    q.put(out)


def cpu_samples(specs, n_total: int, stride: int, threads: int, budget_s: float, n_samples: int = 1):
    """Times the reference's MD::verlet on the sampled replicas `specs`, one
    replica per OpenMP thread at a time (src/main.cpp:22-29), in
    `n_samples` consecutive samples of about `budget_s` each (the step
    count is sized from a 5-step calibration); the replicas are built once
    in a child process, which is ended after n_samples * 3 * budget_s + 120 s.
    Returns ([atom-steps/s per sample], what was sampled) or (None, reason)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_cpu_sample_child, args=(specs, threads, budget_s, n_samples, q))
    p.start()
    limit = n_samples * 3 * budget_s + 120
    try:
        out = q.get(timeout=limit)
        n, atoms, dt = out[-1][1], out[-1][2], out[-1][3]
        values = [o[0] for o in out]
        sample = (f"{len(specs)} of the {n_total} replicas (every {stride}th), {n} MD steps each per sample "
                  f"(MD::verlet as shipped: X-H bonds unconstrained, no SHAKE), {atoms} in-domain "
                  f"atoms, {dt:.1f} s wall on {threads} threads")
    except Exception:
        values, sample = None, f"the reference sample did not finish within {limit:.0f} s"
    p.join(timeout=10)
    if p.is_alive():
        p.kill()
        p.join()
    return values, sample


def plain_sample(engine, specs, quirks, n_pick: int):
    """The plain GPU path: each sampled replica alone in its own engine, one
    kernel launch per MD step (the cluster size is then automatic: 8 CTAs on
    the one replica).  The replicas run one after another, so the aggregate
    is their atom-steps over the summed device time."""
    stride = max(1, len(specs) // n_pick)
    picks = list(range(0, len(specs), stride))[:n_pick]
    atom_steps, seconds = 0.0, 0.0
    for r in picks:
        e = engine.Engine([specs[r]], quirks=quirks, steps_per_launch=1)
        e.step(10)
        a0 = in_domain_atoms([e.info(0)], [specs[r]])[0]
        e.step(MD_STEPS)
        ms, _ = e.last_timing()
        a1 = in_domain_atoms([e.info(0)], [specs[r]])[0]
        atom_steps += 0.5 * (a0 + a1) * MD_STEPS
        seconds += ms * 1e-3
        e.close()
    sample = (f"{len(picks)} of the {len(specs)} replicas (every {stride}th), each alone, "
              f"{MD_STEPS} MD steps at one launch per step, {seconds:.2f} s of device time")
    return atom_steps / seconds, sample


PLACE_GAS, PLACE_VAPOR, PLACE_REF_GAS, PLACE_REF_VAPOR = 1_000_000, 1000, 20_000, 100


def placement_measurement(engine):
    """Initial placement of the configuration-4 system (1,000,000 N2 and
    1,000 water around the 500-atom chain, 300 K, 1e5 Pa) through mdn_place,
    host buffers in and out, against the reference's own
    MD::initialization_gas / initialization_vapor timed on a bounded sample
    (their loop scans every row placed so far for every candidate, so the
    cost grows with the square of the molecule count)."""
    import ctypes as C
    import math
    from md_nucleation_b200 import generate
    from md_nucleation_b200.system import GAS_TABLE, mb_mass_kg
    T = 300.0
    box = generate.box_from_pressure(PLACE_GAS, T, 1e5)
    spec = generate.config4_replica(0, n_gas=2000, n_vap=10)  # the configuration-4 ion, placed in its box
    spec.box = box
    ion = spec.ion.x
    sg = math.sqrt(1.38e-23 * T / mb_mass_kg(GAS_TABLE["N2"]["mol_mass"]))
    sv = math.sqrt(1.38e-23 * T / spec.vapor_mb_mass)
    engine.place(box, ion, 1000, 10, sg, sv, 1)  # loads the kernels
    times = []
    for rep in range(3):
        t0 = time.perf_counter()
        engine.place(box, ion, PLACE_GAS, PLACE_VAPOR, sg, sv, 0x4D444E55 + 4000 + rep)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    n = PLACE_GAS + PLACE_VAPOR
    out = {"workload": f"configuration 4: {PLACE_GAS:,} N2 + {PLACE_VAPOR:,} water around a {len(ion)}-atom "
                       f"chain, box {box:.0f} A",
           "value": n / t, "unit": "molecules/s", "seconds": t,
           "measured": "mdn_place wall time, host buffers in and out (device buffers allocated in the call)"}
    from oracle import bind
    if bind.have_reference():
        L = bind.ref_lib()
        L.ref_time_placement.restype = C.c_double
        L.ref_time_placement.argtypes = [C.c_void_p, C.c_int, C.c_int]
        d, keep = spec.to_desc()
        with stdout_to_stderr():
            s = L.ref_time_placement(C.addressof(d), PLACE_REF_GAS, PLACE_REF_VAPOR)
        m = PLACE_REF_GAS + PLACE_REF_VAPOR
        out["reference"] = {
            "seconds": s, "molecules": m, "value": m / s, "unit": "molecules/s", "cores": 1,
            "sample": f"{PLACE_REF_GAS:,} N2 + {PLACE_REF_VAPOR} water in the same box around the same chain, "
                      "MD::initialization_gas / initialization_vapor as shipped",
            "full_size_estimate_s": s * (n / m) ** 2,
        }
    return out


def _in_domain_energy(e, r, mass):
    """K + U of replica r's in-domain atoms after a step with energies:
    K = sum 1/2 m v^2 (kcal/mol, the reference's real_to_kcalmol), U the sum
    of the eight energy buckets."""
    from md_nucleation_b200.system import REAL_TO_KCALMOL
    t, _, v = e.in_domain(r)
    K = 0.5 * float((mass[t] * (v * v).sum(axis=1)).sum()) * REAL_TO_KCALMOL
    return K + float(e.energies()[r].sum()), len(t)


def nve_drift(engine, spec, force_mode, steps, every=100):
    """Total energy of the in-domain atoms over `steps` NVE steps with the
    membership fixed (no rebuild in the window: loop_update set beyond it,
    so the molecules in the domain at the start are the system, and nothing
    enters or is resampled); the drift is the slope of a straight-line fit,
    per ns.  The taper weights act on vapor forces but not on the energy (the
    reference's PotentialVaporIon / PotentialVaporVapor), so a molecule in the
    100-110 A shell moves the energy too; that is part of what is measured."""
    from md_nucleation_b200 import abi
    checked = abi.Q_ALL & ~abi.Q_BLIND_INSERT
    mass = np.asarray(spec.atom_mass)
    with engine.Engine([spec], quirks=checked, force_mode=force_mode) as e:
        st = e.state(0)
        st.loop_pair, st.loop_update = 0, 10 ** 8
        e.upload(0, st)
        t, E = [], []
        n_atoms = 0
        for k in range(steps // every):
            e.step(every, energy_mode=1)
            en, n_atoms = _in_domain_energy(e, 0, mass)
            t.append((k + 1) * every * spec.dt)
            E.append(en)
        ok = e.status()[0] == 0
    E = np.array(E)
    slope = np.polyfit(np.array(t), E, 1)[0] * 1e6  # kcal/mol per ns
    return {"drift_kcal_mol_per_ns": slope, "drift_per_atom_kcal_mol_per_ns": slope / max(n_atoms, 1),
            "E_mean_kcal_mol": float(E.mean()), "E_rms_fluctuation_kcal_mol": float(E.std()),
            "in_domain_atoms": n_atoms, "window_ps": steps * spec.dt / 1000, "status_clean": bool(ok)}


def force_energy_error(engine, specs, steps=20):
    """FP32 pair terms (force_mode 0) against FP64 pair terms (force_mode 1,
    which the parity tests hold within 1e-9 of the FP64 oracle) on the same
    states: relative RMS of the in-domain forces, and the largest energy
    bucket difference relative to the largest bucket, per replica."""
    from md_nucleation_b200 import abi
    checked = abi.Q_ALL & ~abi.Q_BLIND_INSERT
    out = []
    with engine.Engine(specs, quirks=checked, force_mode=1) as e64, \
            engine.Engine(specs, quirks=checked, force_mode=0) as e32:
        e64.step(steps)
        for r, sp in enumerate(specs):
            st = e64.state(r)
            e32.upload(r, st)
            e64.upload(r, st)
        e64.compute_forces(0)
        e32.compute_forces(0)
        U64, U32 = e64.energies(), e32.energies()
        for r, sp in enumerate(specs):
            a, b = e32.state(r), e64.state(r)
            g = b.region[1:1 + sp.n_gas].astype(bool)
            v = b.region[1 + sp.n_gas:].astype(bool)
            fa = np.concatenate([a.ion_f.reshape(-1, 3), a.gas_af[g].reshape(-1, 3), a.vap_af[v].reshape(-1, 3)])
            fb = np.concatenate([b.ion_f.reshape(-1, 3), b.gas_af[g].reshape(-1, 3), b.vap_af[v].reshape(-1, 3)])
            ferr = float(np.sqrt(((fa - fb) ** 2).sum() / max((fb ** 2).sum(), 1e-300)))
            scale = max(float(np.abs(U64[r]).max()), 1e-12)
            out.append({"force_rel_rms": ferr,
                        "energy_rel": float(np.abs(U32[r] - U64[r]).max()) / scale,
                        "U_total_fp64": float(U64[r].sum()), "U_total_fp32": float(U32[r].sum())})
    return out


C4_GAS, C4_VAPOR = 1_000_000, 1000


def _config4_unplaced(r):
    """A configuration-4 replica without its molecules (the bench places
    them with mdn_place on the GPU; nothing to pickle back from the pool)"""
    from md_nucleation_b200 import generate

    def later(box, ion_x, n_gas, n_vap, gs, vs, seed):
        e = np.zeros((0, 3))
        return e, e, e, e
    return generate.config4_replica(r, n_gas=C4_GAS, n_vap=C4_VAPOR, placer=later)


def config4_specs(engine, n, workers):
    """n configuration-4 replicas (1,000,000 N2, 1,000 rigid water at 10 Pa,
    the 500-atom +2 chain): chains grown in a spawn pool, molecules placed
    by mdn_place (the reference's placement rule, on the GPU)."""
    from md_nucleation_b200.system import mb_sigma
    with mp.get_context("spawn").Pool(max(1, min(workers, n))) as pool:
        specs = pool.map(_config4_unplaced, range(n), chunksize=1)
    for sp in specs:
        gx, gv, vx, vv = engine.place(sp.box, sp.ion.x, C4_GAS, C4_VAPOR,
                                      mb_sigma(sp.temperature, sp.gas_mb_mass),
                                      mb_sigma(sp.temperature, sp.vapor_mb_mass), sp.seed)
        sp.gas_x, sp.gas_v, sp.vapor_x, sp.vapor_v = gx, gv, vx, vv
    return specs


def accuracy_report(engine, specs2, c4specs, drift_steps):
    """The numbers the FP32 pair arithmetic is judged by, per configuration:
    FP32-vs-FP64 force and energy error, and the NVE energy drift per ns of
    both pair modes in a fixed-membership window."""
    from md_nucleation_b200 import generate
    out = {}
    cfg = {"config0": generate.config0(0), "config1": generate.config1(0)}
    for name, sp in cfg.items():
        out[name] = {"fp32_vs_fp64": force_energy_error(engine, [sp])[0],
                     "nve_fp32": nve_drift(engine, sp, 0, drift_steps),
                     "nve_fp64": nve_drift(engine, sp, 1, drift_steps)}
    pick = [0, len(specs2) // 3, 2 * len(specs2) // 3, len(specs2) - 1]
    sample = [specs2[i] for i in pick]
    errs = force_energy_error(engine, sample)
    out["config2"] = {"replicas": pick, "fp32_vs_fp64": errs,
                      "nve_fp32": [nve_drift(engine, sample[k], 0, drift_steps // 2) for k in (0, 3)],
                      "nve_fp64": [nve_drift(engine, sample[k], 1, drift_steps // 2) for k in (0, 3)]}
    if c4specs:
        out["config4"] = {"fp32_vs_fp64": force_energy_error(engine, c4specs[:2])}
    return out


def config4_measurement(engine, specs, blocks):
    """Configuration 4 batched: 16 replicas of 1,000,000 N2, 1,000 water and
    the 500-atom chain, advanced in 100-step launches with the checked
    insertion; device time from CUDA events."""
    from md_nucleation_b200 import abi
    checked = abi.Q_ALL & ~abi.Q_BLIND_INSERT
    with engine.Engine(specs, quirks=checked, use_graph=1) as e:
        e.step(100)
        i0 = [e.info(r) for r in range(e.n)]
        ms = 0.0
        for _ in range(blocks):
            e.step(100)
            ms += e.last_timing()[0]
        i1 = [e.info(r) for r in range(e.n)]
        st = e.status()
    a0 = in_domain_atoms(i0, specs)
    a1 = in_domain_atoms(i1, specs)
    atom_steps = 0.5 * float(a0.sum() + a1.sum()) * 100 * blocks
    return {"replicas": len(specs), "molecules_per_replica": specs[0].n_mol, "md_steps": 100 * blocks,
            "value": atom_steps / (ms * 1e-3), "unit": UNIT, "ms_per_100_steps": ms / blocks,
            "in_domain_atoms": int(a1.sum()), "rebuilds": int(sum(i.n_rebuilds for i in i1)),
            "replicas_failed": int(np.sum((st & abi.ST_FATAL) != 0)),
            "ns_per_day_per_replica": 100 * blocks * specs[0].dt * 1e-6 / (ms * 1e-3) * 86400}


def adjoint_measurement(engine):
    """The gradient harness on the adjoint configuration: a 2,000-step window
    of the production system (150-atom +1 chain, 100 methanol, 100,000 rigid
    N2, SHAKE on X-H bonds, 300 K, 1e5 Pa) with 8 of the methanol started
    8-28 A from the chain (generate.config3; otherwise the domain holds no
    vapor and the objective is identically zero), checkpoints every 100
    steps, FP32 forward on the engine, FP64 adjoint.  The margin is raised to
    40 A so that the window holds no effective-domain rebuild (mdn_adjoint
    needs a fixed molecule set)."""
    from md_nucleation_b200 import generate
    spec = generate.config3(0)
    with engine.Engine([spec]) as e:
        e.step(10)
        info = e.info(0)
        window = 2000
        if info.loop_update - info.loop_pair < window:
            return {"unavailable": f"the next rebuild is {info.loop_update - info.loop_pair} steps away"}
        J, grad, (fwd_ms, adj_ms) = e.adjoint(n_steps=window, checkpoint_every=100, count_radius=10.0,
                                              count_width=1.0)
        rows, _ = e.adjoint_params()
        return {"cost_ratio": adj_ms / fwd_ms, "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "n_params": len(grad),
                "window_steps": window, "checkpoint_every": 100, "J": J,
                "max_abs_dJ_dtheta": float(np.abs(grad).max()), "charge_scale_dJ": float(grad[-1]),
                "in_domain_atoms": int(info.n_ion + info.n_gas_in * spec.gas.n + info.n_vapor_in * spec.vapor.n),
                "vapor_in_domain": int(info.n_vapor_in),
                "system": "150-atom +1 chain, 100 methanol (8 started 8-28 A from the chain), 100,000 rigid N2 "
                          "(margin 40 A)"}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from oracle import bind
    if not bind.have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_harness.so was not built"}))
        return 0
    threads = host_threads()
    pick, stride = sample_indices(args.replicas, threads)
    specs = make_specs(0, 0, threads, indices=pick)
    values, sample = cpu_samples(specs, args.replicas, stride, threads, args.ref_budget,
                                 args.warmup + args.steps)
    if values is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return 0
    for k, v in enumerate(values):
        log(f"reference step {k}: {v:.4g} atom-steps/s")
    values = values[args.warmup:]
    value = float(np.mean(values))
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "replicas": args.replicas, "md_steps_per_step": MD_STEPS,
                   "path": "reference routines (MD::verlet as shipped, which never calls SHAKE) compiled from the "
                           "reference sources, one replica per OpenMP thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
# the CUDA engine
# ---------------------------------------------------------------------------
def run_engine(args):
    ws, rank, local = dist_env()
    threads = host_threads()
    # replicas are generated in a spawn pool before any CUDA call
    specs = make_specs(rank * args.replicas, args.replicas, max(1, threads // max(ws, 1)))
    dist = dist_init(ws, local, "nccl")
    import torch
    from md_nucleation_b200 import abi, engine
    if engine.device_count() == 0:
        raise SystemExit("bench.py: no CUDA device")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    free0, total = torch.cuda.mem_get_info(device)
    checked = abi.Q_ALL & ~abi.Q_BLIND_INSERT
    t0 = time.time()
    eng = engine.Engine(specs, quirks=checked, device=local, use_graph=1,
                        **({"threads": args.threads} if args.threads else {}))
    free1, _ = torch.cuda.mem_get_info(device)
    resident = free0 - free1
    log(f"rank {rank}: engine created in {time.time() - t0:.1f} s, {resident / 2**30:.2f} GiB resident")

    def barrier():
        torch.cuda.synchronize(device)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    # warm-up: the launch-shape tuner (a block of MD_STEPS per cluster size,
    # then up to 3 blocks of split launches; results do not depend on the
    # shape), then the warm-up steps
    def step_block(n, energy_mode=0):
        """n MD steps; a replica that raises a fatal status is frozen by the
        engine (mdn_step returns MDN_ERR_REPLICA) and counted below instead
        of ending the run"""
        try:
            eng.step(n, energy_mode)
        except engine.MdnError as ex:
            if ex.code != abi.ERR_REPLICA:
                raise

    if args.cluster:
        eng.set_launch(args.cluster)
        eng.set_split(args.split, 2 * args.cluster if args.split else 0)
        chosen_by = "--cluster / --split"
    else:
        try:
            tuned = eng.tune_launch(MD_STEPS)
        except engine.MdnError as ex:
            if ex.code != abi.ERR_REPLICA:
                raise
            tuned = eng.get_launch()[0]
        chosen_by = "mdn_tune_launch during warm-up"
        log(f"rank {rank}: tuned cluster size {tuned}")
    for _ in range(args.warmup):
        step_block(MD_STEPS)
    barrier()
    live0 = (eng.status() & abi.ST_FATAL) == 0
    infos0 = [eng.info(r) for r in range(eng.n)]
    # timed region: K bench steps, device time from CUDA events on the
    # launching stream (mdn_last_timing)
    ms_total, launches = 0.0, 0
    barrier()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            step_block(MD_STEPS)
            ms, nl = eng.last_timing()
            ms_total += ms
            launches += nl
        barrier()
    infos1 = [eng.info(r) for r in range(eng.n)]
    status = eng.status()
    fatal = int(np.sum((status & abi.ST_FATAL) != 0))
    warned = int(np.sum((status != 0) & ((status & abi.ST_FATAL) == 0)))
    # only replicas that advanced through the whole timed region count
    live = live0 & ((status & abi.ST_FATAL) == 0)
    keep = [r for r in range(eng.n) if live[r]]
    infos0 = [infos0[r] for r in keep]
    infos1 = [infos1[r] for r in keep]
    kspecs = [specs[r] for r in keep]
    atoms0 = in_domain_atoms(infos0, kspecs)
    atoms1 = in_domain_atoms(infos1, kspecs)
    flops0 = algorithmic_flops(infos0, kspecs)
    flops1 = algorithmic_flops(infos1, kspecs)
    atom_steps = 0.5 * float(atoms0.sum() + atoms1.sum()) * MD_STEPS * args.steps
    ms_max = max_over_ranks(dist, ms_total, device)
    atom_steps_all = sum_over_ranks(dist, atom_steps, device)
    value = atom_steps_all / (ms_max * 1e-3)
    flops_per_md_step = 0.5 * (flops0 + flops1)
    achieved_tflops = flops_per_md_step * MD_STEPS * args.steps / (ms_total * 1e-3) / 1e12
    bytes_timed = algorithmic_bytes(infos0, infos1, kspecs, MD_STEPS * args.steps)
    achieved_gbs = bytes_timed / (ms_total * 1e-3) / 1e9
    clocks = clk.summary()

    # end to end through the C ABI: per bench step the thermostat controls go
    # host -> device from page-locked memory and every replica's in-domain
    # atoms come back into page-locked host buffers (the dump path)
    modes = engine.PinnedArray((eng.n,), np.int32)
    temps = engine.PinnedArray((eng.n,), np.float64)
    modes.array[:] = [s.nvt_mode for s in specs]
    temps.array[:] = [s.nvt_temperature for s in specs]
    cap = int(in_domain_atoms([eng.info(r) for r in range(eng.n)], specs).max() * 1.5 * eng.n) + 1024
    snap = engine.SnapshotBuffer(eng.n, cap, pinned=True)
    e2e_steps = max(1, min(args.steps, 3))
    # one untimed pass loads the snapshot kernels and touches the host pages
    eng.set_nvt_batch(modes.array, temps.array)
    step_block(MD_STEPS, energy_mode=1)
    eng.snapshot(snap, energies=True)
    barrier()
    t0 = time.perf_counter()
    d2h = 0
    e2e_atom_steps = 0.0
    for _ in range(e2e_steps):
        eng.set_nvt_batch(modes.array, temps.array)
        step_block(MD_STEPS, energy_mode=1)
        eng.snapshot(snap, energies=True)
        d2h += snap.nbytes_used + (eng.n + 1) * 8 + eng.n * 64
        e2e_atom_steps += float(snap.offset[-1]) * MD_STEPS
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(dist, e2e_s, device)
    e2e_all = sum_over_ranks(dist, e2e_atom_steps, device)
    e2e_value = e2e_all / e2e_s
    h2d_per_step = eng.n * (4 + 8)
    launch_shape = eng.get_launch()
    split = eng.get_split()

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 forces / f64 integration",
            "data": "synthetic (seeded generator of the batched-replica configuration)",
            "config": {
                "workload": WORKLOAD, "replicas_per_gpu": eng.n, "md_steps_per_step": MD_STEPS,
                "in_domain_atoms_per_gpu": int(atoms1.sum()),
                "in_domain_atoms_range": [int(atoms1.min()), int(atoms1.max())] if len(atoms1) else None,
                "insertion": "checked (rotation re-drawn until no atom within 2 A)",
                "l2": f"inputs larger than L2: {resident / 2**30:.2f} GiB resident per GPU",
                "replicas_with_warnings": warned, "replicas_failed": fatal,
                "parallelism": f"replicas sharded over {ws} GPU(s), no collective in the step",
                "launch": {"cluster_ctas_per_replica": launch_shape[0], "threads_per_cta": launch_shape[1],
                           "md_steps_per_launch": MD_STEPS if launch_shape[2] <= 0 else launch_shape[2],
                           "split": {"largest_replicas": split[0], "cluster_ctas": split[1]},
                           "chosen_by": chosen_by},
            },
            "roofline": {
                "bound": "fp32", "achieved": achieved_tflops, "peak": None, "unit": "TFLOP/s", "frac": None,
                "traffic": None, "kernel": "mdn_advance", "launch": f"{MD_STEPS} MD steps of every replica",
                "algorithmic_flops_per_launch": flops_per_md_step * MD_STEPS,
                "hbm": {"achieved": achieved_gbs, "unit": "GB/s",
                        "algorithmic_bytes_per_launch": bytes_timed / args.steps,
                        "model": "streaming byte model: 204 B per in-domain atom-step, 4 B per list entry and "
                                 "step, 72 B per molecule and rebuild"},
            },
            "gpu_launches": launches,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_per_step,
                    "d2h_bytes_per_step": int(d2h / e2e_steps)},
        }
        # the kernel's bound is FP32 issue and latency, not DRAM (each
        # replica's core sits in shared memory, its gas slab in L2): the
        # headline fraction is the algorithmic pair flops against the FP32
        # pipes, 148 SMs x 128 lanes x 2 flops (FMA) at the SM clock sampled
        # during the timed region (no FP32 figure is measured separately on
        # these GPUs); the byte model against the measured copy bandwidth is
        # kept beside it
        props = torch.cuda.get_device_properties(device)
        mhz = clocks["sm_mhz"] or 1965.0
        peak = props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
        out["roofline"].update({"peak": peak, "frac": achieved_tflops / peak,
                                "peak_source": f"{props.multi_processor_count} SMs x 128 FP32 lanes x 2 at the "
                                               f"sampled median {mhz:.0f} MHz"})
        hbm, hbm_src = measured_hbm_peak()
        out["roofline"]["hbm"].update({"peak": hbm, "frac": achieved_gbs / hbm, "peak_source": hbm_src})
        # DRAM bytes of one launch from ncu (a 32-replica capture scaled by
        # atom-steps; profiles/mdn_advance_batched.md)
        traffic = traffic_per_atom_step()
        if traffic is not None:
            out["roofline"]["traffic"] = traffic * atom_steps / args.steps
    # the plain one-system-per-launch path on the same GPU (rank 0, N = 1)
    if rank == 0 and ws == 1 and not args.no_plain:
        pv, psample = plain_sample(engine, specs, checked, args.plain_replicas)
        out["plain"] = {"value": pv, "unit": UNIT, "sample": psample, "batched_over_plain": value / pv}
    # the gradient harness's cost against its own forward window (rank 0, N = 1)
    if rank == 0 and ws == 1 and not args.no_adjoint:
        out["adjoint"] = adjoint_measurement(engine)
    # initial placement of the configuration-4 system (rank 0, N = 1)
    if rank == 0 and ws == 1 and not args.no_placement:
        out["placement"] = placement_measurement(engine)
    # ns/day of the batched run: every replica advances MD_STEPS * dt per step
    if rank == 0:
        per = MD_STEPS * specs[0].dt * 1e-6 / (ms_max / args.steps * 1e-3) * 86400
        out["ns_per_day"] = {"per_replica": per, "aggregate": per * eng.n * ws}
    # configuration 4 batched and the accuracy report (rank 0, N = 1)
    if rank == 0 and ws == 1 and not args.no_accuracy:
        t0 = time.time()
        c4 = config4_specs(engine, args.config4_replicas, threads) if args.config4_replicas else []
        if c4:
            out["config4"] = config4_measurement(engine, c4, args.config4_blocks)
        out["accuracy"] = accuracy_report(engine, specs, c4, args.drift_steps)
        log(f"config 4 and accuracy report in {time.time() - t0:.0f} s")
    # CPU baseline on rank 0 at N = 1 only
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import bind
        if bind.have_reference():
            pick, stride = sample_indices(len(specs), threads)
            v, sample = cpu_samples([specs[i] for i in pick], len(specs), stride, threads, args.cpu_budget)
            out["cpu_baseline"] = {"value": v[0] if v else None, "unit": UNIT, "cores": threads,
                                   "kind": "reference", "sample": sample}
        else:
            out["cpu_baseline"] = None
    if rank == 0:
        print(json.dumps(out))
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of the CPU-baseline sample")
    ap.add_argument("--ref-budget", type=float, default=3.0, help="seconds per reference-arm step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the one-system-per-launch measurement")
    ap.add_argument("--plain-replicas", type=int, default=16)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the gradient-harness measurement")
    ap.add_argument("--no-placement", action="store_true", help="skip the initial-placement measurement")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip configuration 4 and the FP32/FP64 accuracy and NVE drift report")
    ap.add_argument("--config4-replicas", type=int, default=16)
    ap.add_argument("--config4-blocks", type=int, default=10, help="100-step launches of configuration 4")
    ap.add_argument("--drift-steps", type=int, default=10000, help="NVE window of the drift measurement")
    ap.add_argument("--cluster", type=int, default=0, help="CTAs per replica (1..8); 0 = tuned in the warm-up")
    ap.add_argument("--threads", type=int, default=0, help="threads per CTA (multiple of 32, <= 512); 0 = 512")
    ap.add_argument("--split", type=int, default=0,
                    help="with --cluster: the N largest replicas on clusters twice as large, in a concurrent launch")
    ap.add_argument("--only-placement", action="store_true",
                    help="print only the initial-placement measurement (mdn_place on configuration 4)")
    ap.add_argument("--only-adjoint", action="store_true",
                    help="print only the gradient-harness measurement (mdn_adjoint on configuration 1)")
    args = ap.parse_args()
    if args.warmup < 3 and not os.environ.get("MDN_BENCH_ALLOW_SHORT"):
        raise SystemExit("bench.py: --warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.only_placement:
        from md_nucleation_b200 import engine
        print(json.dumps(placement_measurement(engine)))
        return 0
    if args.only_adjoint:
        from md_nucleation_b200 import engine
        print(json.dumps(adjoint_measurement(engine)))
        return 0
    return run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
