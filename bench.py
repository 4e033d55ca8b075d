"""Benchmark: rigid TIP4P/2005 water timesteps/s and ns/day on B200.

Workload (default): 4,096 molecules (16,384 sites incl. M), cubic lattice at
0.997 g/cm^3 with seeded random orientations, LJ + Coulomb 9 A cutoff, skin
1 A, Ewald real space + P3M 64^3 order 5, SETTLE, dt 2 fs, Nose-Hoover NVT at
298 K, FP32 with FP64 reductions and FP64 SETTLE, neighbour check every 10
steps.  The seeded start is relaxed into the liquid (4,000 untimed steps
with a tight thermostat) before the warm-up.  A "step" is one MD timestep of
that system.

  python bench.py [--gpus N] [--steps K] [--warmup W]
                  [--workload water|water_e3b|lj|batched|surrogate]
  python bench.py --impl reference ...   # the reference's CPU arm (the oracle)

Under torchrun every rank steps its own independent replica (the path does
not shard: replicas only); value = sum over ranks of steps / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "water timesteps/s & ns/day on 1 B200, plain vs surrogate/batched at force RMSE"
L2_FLUSH_BYTES = 256 << 20
EQ_STEPS = 4000  # untimed relaxation of the seeded start


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="water", choices=["water", "water_e3b", "lj", "batched", "surrogate"])
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--frames", type=int, default=40, help="surrogate: frames per training temperature")
    ap.add_argument("--train-iters", type=int, default=4000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-nve", action="store_true", help="skip the NVE energy-drift measurement")
    ap.add_argument("--batch-eq-steps", type=int, default=BATCH_EQ_STEPS,
                    help="batched: untimed relaxation of the replicas' seeded starts (0: the lattice starts)")
    ap.add_argument("--eq-steps", type=int, default=EQ_STEPS,
                    help="untimed relaxation steps of the seeded start before the warm-up")
    return ap.parse_args()


# nominal FP32 rate of a B200 at its maximum SM clock (no measured figure)
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_pg(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def reduce_max(dist, value, device=None):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device=None):
    if dist is None:
        return
    import torch
    t = torch.zeros(1, device=device)
    dist.all_reduce(t)


def workload_cfg(name, sysd):
    """the config object of a single-system workload (both arms print it)"""
    if name == "lj":
        return {"workload": "LJ fluid 32,000 atoms FCC rho*=0.8442 T*=1.2, rc 2.5 skin 0.3, dt 0.005, NH",
                "atoms": len(sysd.pos)}
    e3b = name == "water_e3b"
    return {"workload": ("TIP4P/2005" + ("+E3B3" if e3b else "") +
                         " 4,096 molecules (16,384 sites), LJ+Coulomb 9 A, skin 1 A, P3M 64^3 order 5, "
                         "SETTLE, dt 2 fs, Nose-Hoover 298 K"),
            "molecules": int(len(sysd.molecules)), "sites": int(len(sysd.pos))}


def _water_state(sysd, e3b, tau):
    from md_engine_b200 import systems
    return systems.build_water_state(sysd, rcut=9.0, skin=1.0, dt=2.0, interval=10, grid=64, e3b=e3b,
                                     T=298.0, tau=tau)


def _lj_state(sysd, tau):
    from md_engine_b200 import systems
    return systems.build_lj_state(sysd, rcut=2.5, skin=0.3, dt=0.005, interval=10, T=1.2, tau=tau)


def equilibrate(name, sysd, steps=EQ_STEPS):
    """The seeded lattice start relaxed into the workload's liquid before
    anything is timed: `steps` MD steps of the same system and step with a
    tight Nose-Hoover coupling (tau 25 fs for water, 0.1 for the LJ fluid) at
    the workload's temperature; returns the system with the final positions
    and velocities.  The reference benchmarks equilibrated liquid water at
    298 K; the lattice start alone turns its potential energy into heat and
    the timed steps would run a hot, near-lattice system instead."""
    import dataclasses
    from md_engine_b200 import IntegratorVerlet
    st, _ = _lj_state(sysd, 0.1) if name == "lj" else _water_state(sysd, name == "water_e3b", 25.0)
    IntegratorVerlet(st).run(steps)
    x, v, _ = st.getAtoms()
    return dataclasses.replace(sysd, pos=np.asarray(x, np.float64), vel=np.asarray(v, np.float64))


def workload(name, seed=20261203, eq_steps=EQ_STEPS):
    from md_engine_b200 import systems
    if name == "lj":
        sysd = equilibrate(name, systems.lj_fcc(ncell=20, seed=seed), eq_steps)
        st, fx = _lj_state(sysd, 0.5)
        return sysd, st, fx, workload_cfg(name, sysd), 0.005
    sysd = equilibrate(name, systems.water_tip4p2005(nside=16, seed=seed), eq_steps)
    st, fx = _water_state(sysd, name == "water_e3b", 100.0)
    return sysd, st, fx, workload_cfg(name, sysd), 2.0


def timed_temperature(name, sysd, st):
    """instantaneous temperature from the FP64 kinetic sum (rigid water:
    6 degrees of freedom per molecule, 3 of them removed for the momentum)"""
    from md_engine_b200 import systems
    mv2, _ = st.kinetic()
    if name == "lj":
        return {"value": mv2 / (3 * len(sysd.pos) - 3), "unit": "epsilon/k_B"}
    ndf = 6 * len(sysd.molecules) - 3
    return {"value": mv2 * systems.MVV_TO_ENG_REAL / (ndf * systems.BOLTZ_REAL), "unit": "K"}


def nve_drift(name, x, v, seed):
    """Total-energy drift of an NVE continuation of the timed run: the same
    system, cutoffs, mesh and step with the thermostat off, started from the
    timed run's final positions and velocities.  After 200 steps, the total
    energy (FP64 kinetic sum + the potential energy of every fix) is sampled
    every 500 steps over 5,000 steps; the drift is the least-squares slope,
    per molecule in kcal/mol per ns (water) or per atom in epsilon per tau
    (LJ).  Not timed."""
    import dataclasses
    from md_engine_b200 import IntegratorVerlet, systems
    if name == "lj":
        sysd = systems.lj_fcc(ncell=20, seed=seed)
        sysd = dataclasses.replace(sysd, pos=np.asarray(x), vel=np.asarray(v))
        st, _ = systems.build_lj_state(sysd, rcut=2.5, skin=0.3, dt=0.005, interval=10)
        nunit, mvv, t_step, unit = len(sysd.pos), 1.0, 0.005, "epsilon per atom per tau"
    else:
        sysd = systems.water_tip4p2005(nside=16, seed=seed)
        sysd = dataclasses.replace(sysd, pos=np.asarray(x), vel=np.asarray(v))
        st, _ = systems.build_water_state(sysd, rcut=9.0, skin=1.0, dt=2.0, interval=10, grid=64,
                                          e3b=name == "water_e3b", thermostat=False)
        nunit, mvv, t_step, unit = len(sysd.molecules), systems.MVV_TO_ENG_REAL, 2.0e-6, "kcal/mol per molecule per ns"
    it = IntegratorVerlet(st)
    it.run(200)
    ts, es = [], []
    for k in range(11):
        if k:
            it.run(500)
        mv2, _ = st.kinetic()
        es.append((0.5 * mv2 * mvv + float(np.sum(st.potentialEnergy()))) / nunit)
        ts.append(k * 500 * t_step)
    slope = float(np.polyfit(ts, es, 1)[0])
    return {"value": slope, "unit": unit, "steps": 5000, "samples": len(es),
            "energy_per_unit_first_last": [es[0], es[-1]],
            "integrator": "velocity Verlet, FP32 forces, FP64 SETTLE, same dt, thermostat off"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return None
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 5 + k and s[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(key):
    """dram bytes per launch of the dominant kernel from the committed ncu summary"""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            e = json.load(f).get(key)
        return None if e is None else float(e["traffic_bytes"])
    return None


def fp64_errors(name, sysd, st, fx):
    """Error of every reported quantity of the timed state against the FP64
    oracle on the same positions: per-site forces (the largest error vector
    and the RMS error, both over the RMS force), potential energy per term
    and in total, and the total virial (largest component error over the
    largest component).  The kinetic energy is an FP64 device sum of the FP32
    velocities (no separate error).  Part of the CPU-baseline leg."""
    from oracle import cpu_step
    st.computeForces(virialMode=1)
    x, _, fg = st.getAtoms()
    _, vir = st.virials()
    eg = np.asarray(st.potentialEnergy(), np.float64)
    if name == "lj":
        ref = cpu_step.lj_reference(sysd, x, rcut=2.5, skin=0.3)
        e_terms = {"pair": (eg[0], ref["energy"]["pair"])}
    else:
        ref = cpu_step.water_reference(sysd, x, rcut=9.0, skin=1.0, grid=64, alpha=fx["ewald"].alpha,
                                       e3b=name == "water_e3b")
        e_terms = {"pair": (eg[0], ref["energy"]["pair"]), "p3m": (eg[1], ref["energy"]["p3m"])}
        if name == "water_e3b":
            e_terms["e3b_two_body"] = (eg[2], ref["energy"]["e3b2"])
            e_terms["e3b_three_body"] = (eg[3], ref["energy"]["e3b3"])
    fr = ref["f"]
    rms = float(np.sqrt(np.mean(np.sum(fr ** 2, 1))))
    d = np.linalg.norm(fg - fr, axis=1)
    etot_g = sum(a for a, _ in e_terms.values())
    etot_r = sum(b for _, b in e_terms.values())
    vr = ref["virial"]
    return {"oracle": "FP64 CPU restatement (oracle/), same positions, list, alpha and mesh",
            "force_max_err_over_rms": float(d.max() / rms), "force_rms_err_over_rms": float(np.sqrt(np.mean(d ** 2)) / rms),
            "force_rms": rms,
            "energy_rel": {k: float(abs(a - b) / max(abs(b), 1e-300)) for k, (a, b) in e_terms.items()},
            "energy_total_rel": float(abs(etot_g - etot_r) / abs(etot_r)),
            "virial_max_err_over_max": float(np.abs(np.asarray(vir) - vr).max() / np.abs(vr).max())}


def run_reference_arm(args, rank, world):
    """--impl reference: the oracle's CPU step (OpenMP, all host threads),
    rank 0 only; other ranks exit without work."""
    if rank != 0:
        return
    from md_engine_b200 import systems
    from oracle import cpu_step
    if args.workload == "lj":
        sysd = systems.lj_fcc(ncell=20)
        dt = 0.005
    else:
        sysd = systems.water_tip4p2005(nside=16)
        dt = 2.0
    # a bounded sample: up to 5 warm-up and 50 timed whole steps (a few
    # seconds to a minute on the host cores)
    steps = max(1, min(args.steps, 50))
    warm = min(args.warmup, 5)
    res = cpu_step.time_steps(sysd, args.workload, nsample=steps, warmup=warm)
    v = res["steps_per_s"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "timesteps/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": dict(workload_cfg(args.workload, sysd), reference_sample=res["workload"],
                           start="the seeded start as generated (the FP64 CPU step's cost does not depend "
                                 "on the relaxation; relaxing it here would take the GPU)"),
            "ns_per_day": v * dt * 86400 / 1e6 if args.workload != "lj" else None,
            "cpu_baseline": {"value": v, "unit": "timesteps/s", "cores": res["cores"], "kind": "port",
                             "sample": res["sample"]},
            "e2e": {"value": v, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


BATCH_EQ_STEPS = 2000  # untimed relaxation of the replicas' seeded starts


def _replica_state(sysd, T, e3b, tau):
    from md_engine_b200 import systems
    st, _ = systems.build_water_state(sysd, rcut=9.0, skin=0.8, dt=2.0, interval=10,
                                      grid=systems.p3m_mesh_for(sysd.L[0]), e3b=e3b, T=float(T), tau=tau)
    st.nThreadPerAtom = 8
    return st


def batched_systems(nrep, seed, e3b=True, subset=None, eq_steps=BATCH_EQ_STEPS):
    """the batched-replica workload: nrep TIP4P/2005(+E3B3) boxes, molecule
    counts log-uniform in [256, 2048], T uniform in [260, 360] K, rc 9 A,
    skin 0.8 A, P3M mesh 32^3 or 64^3 by box size; subset: only these replica
    indices (each replica is seeded by its index, whoever builds it).  As the
    single-system workloads, every seeded lattice start is relaxed first
    (eq_steps batched steps with a tight Nose-Hoover coupling, tau 25 fs, at
    the replica's temperature), so that the timed steps run liquid water at
    the replicas' temperatures rather than a lattice melting.  Returns
    [(system, T, molecules)]."""
    import dataclasses
    from md_engine_b200 import BatchReplicas, systems
    sizes, temps = systems.water_replica_sizes(nrep, seed=seed)
    raw = [(systems.water_tip4p2005(nmol=int(m), T=float(T), seed=seed + 1000 + r), float(T), int(m))
           for r, (m, T) in enumerate(zip(sizes, temps)) if subset is None or r in subset]
    if eq_steps <= 0:
        return raw
    states = [_replica_state(sysd, T, e3b, 25.0) for sysd, T, _ in raw]
    b = BatchReplicas(states)
    b.prepare()
    b.run(eq_steps)
    out = []
    for (sysd, T, m), st in zip(raw, states):
        x, v, _ = st.getAtoms()
        out.append((dataclasses.replace(sysd, pos=np.asarray(x, np.float64), vel=np.asarray(v, np.float64)), T, m))
    del b
    return out


def batched_states(systems_, e3b=True):
    """the timed replicas: states (tau 100 fs) from batched_systems' output"""
    return [(_replica_state(sysd, T, e3b, 100.0), m) for sysd, T, m in systems_]


def side_line(args, world, value, unit, K, ms_max, cfg, extra, clk, launches):
    line = {"metric": METRIC, "value": value, "unit": unit, "n_gpus": world, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 reductions, f64 SETTLE)",
            "data": "synthetic (seeded lattice + random orientations + Maxwell-Boltzmann)", "config": cfg,
            "gpu_launches": launches, "clocks": clk.summary()}
    line.update(extra)
    print(json.dumps(line))


def run_batched(args, rank, world, local):
    """replica timesteps/s of the batched form against the same replicas run
    one after another through IntegratorVerlet (the plain per-replica path)"""
    import torch
    from md_engine_b200 import BatchReplicas, IntegratorVerlet, kernel_launches
    from md_engine_b200 import systems
    from md_engine_b200.replicas import gather_replica_scalars, shard_by_sites
    dist = init_pg(world, "nccl")
    dev = torch.device("cuda", local)
    # one ensemble of replicas x world boxes (per-GPU work fixed: weak
    # scaling), dealt to the ranks by balanced site count; no exchange while
    # stepping, one gather of per-replica scalars at the end
    seed = 20261203
    total = args.replicas * world
    sizes, _ = systems.water_replica_sizes(total, seed=seed)
    mine = shard_by_sites([4 * int(m) for m in sizes], world)[rank]
    eq = batched_systems(total, seed, subset=set(mine), eq_steps=args.batch_eq_steps)
    reps = batched_states(eq)
    states = [s for s, _ in reps]
    mols = sum(m for _, m in reps)
    b = BatchReplicas(states)
    team, tune_ms = b.autotune(steps=20, teams=(4, 8, 16, 32))
    b.run(max(args.warmup, 3))
    K = args.steps
    barrier(dist, dev)
    torch.cuda.synchronize()
    k0 = kernel_launches()
    with ClockSampler(local) as clk:
        ms = b.runTimed(K, 10, L2_FLUSH_BYTES)
    k1 = kernel_launches()
    barrier(dist, dev)
    ms_max = reduce_max(dist, ms, dev)
    R = len(states)
    value = total * K / (ms_max * 1e-3)
    # the end-of-run collective: every replica's temperature, in replica order
    temps = []
    for st in states:
        mv2, ndf = st.kinetic()
        temps.append(mv2 * systems.MVV_TO_ENG_REAL / (max(ndf, 1.0) * systems.BOLTZ_REAL))
    all_t = gather_replica_scalars(dist, mine, temps, total, device=dev)
    # the plain path: every replica alone (fresh copies), same step count
    seq_ms = 0.0
    Ks = min(K, 50)
    for st, _ in batched_states(eq):
        it = IntegratorVerlet(st)
        it.run(3)
        seq_ms += it.runTimed(Ks, 10, 0)
    seq = R * Ks / (seq_ms * 1e-3)
    if rank == 0:
        cfg = {"workload": f"{total} TIP4P/2005+E3B3 replicas ({args.replicas} per GPU), sizes log-uniform "
                           "256-2048 molecules, T 260-360 K, rc 9 A, skin 0.8 A, P3M 32^3/64^3",
               "start": (f"equilibrated: {args.batch_eq_steps} batched steps, tight Nose-Hoover, before warm-up"
                         if args.batch_eq_steps > 0 else "seeded lattice starts"),
               "replicas": total, "replicas_rank0": R, "molecules_rank0": mols, "autotuned_team": team,
               "l2": "flushed between timed 10-step chunks (256 MiB write)",
               "parallelism": f"replicas dealt to {world} GPUs by site count" if world > 1 else "one batch"}
        side_line(args, world, value, "replica timesteps/s", K, ms_max, cfg,
                  {"sequential_plain": {"value": seq, "unit": "replica timesteps/s", "steps_per_replica": Ks},
                   "batched_over_sequential": (R * K / (ms * 1e-3)) / seq,
                   "replica_temperature_K": {"mean": float(np.mean(all_t)), "min": float(np.min(all_t)),
                                             "max": float(np.max(all_t))}}, clk, int(k1 - k0))
    if dist is not None:
        barrier(dist, dev)
        dist.destroy_process_group()


def run_surrogate(args, rank, world, local):
    """TIP4P/2005+E3B3, 4,096 molecules: the exact E3B step against the step
    with the learned three-body surrogate, trained here on frames the exact
    kernel labels (NVT runs at 260, 310 and 360 K), scored on a frame of an
    unseen 330 K run"""
    import torch
    from md_engine_b200 import IntegratorVerlet, kernel_launches, systems
    dist = init_pg(world, "nccl")
    dev = torch.device("cuda", local)
    seed = 20261203 + 7919 * rank

    def state(T, sd):
        sysd = systems.water_tip4p2005(nside=16, seed=sd, T=T)
        return systems.build_water_state(sysd, rcut=9.0, skin=1.0, dt=2.0, interval=10, grid=64, e3b=True,
                                         T=T, tau=100.0)

    st, fx = state(298.0, seed)
    it = IntegratorVerlet(st)
    it.run(max(args.warmup, 3))
    K = args.steps
    ms_exact = it.runTimed(K, 10, L2_FLUSH_BYTES)
    e3 = fx["e3b"]
    t0 = time.perf_counter()
    nframes = 0
    for T, sd in ((260.0, seed + 1), (310.0, seed + 2), (360.0, seed + 3)):
        st_t, _ = state(T, sd)
        it_t = IntegratorVerlet(st_t)
        it_t.run(200)
        for _ in range(args.frames):
            it_t.run(10)
            x, v, _ = st_t.getAtoms()
            st.putAtoms(x, v)
            st.buildNeighborlists(force=True)
            e3.surrogateCollect()
            nframes += 1
    t_collect = time.perf_counter() - t0
    t0 = time.perf_counter()
    l0, l1 = e3.surrogateTrain(args.train_iters, batch=4096, lr=2e-3, seed=seed)
    t_train = time.perf_counter() - t0
    st_h, _ = state(330.0, seed + 4)
    IntegratorVerlet(st_h).run(300)
    x, v, _ = st_h.getAtoms()
    st.putAtoms(x, v)
    st.buildNeighborlists(force=True)
    rmse, rms = e3.surrogateEval()
    e3.surrogateEnable(True)
    it.run(max(args.warmup, 3))
    barrier(dist, dev)
    k0 = kernel_launches()
    with ClockSampler(local) as clk:
        ms_sur = it.runTimed(K, 10, L2_FLUSH_BYTES)
    k1 = kernel_launches()
    ms_max = reduce_max(dist, ms_sur, dev)
    value = world * K / (ms_max * 1e-3)
    if rank == 0:
        cfg = {"workload": "TIP4P/2005+E3B3 4,096 molecules, LJ+Coulomb 9 A, skin 1 A, P3M 64^3, SETTLE, "
                           "dt 2 fs, Nose-Hoover 298 K; E3B three-body from the BF16 MLP surrogate",
               "molecules": 4096, "training_frames": nframes, "train_iters": args.train_iters,
               "l2": "flushed between timed 10-step chunks (256 MiB write)", "parallelism": "single system"}
        side_line(args, world, value, "timesteps/s", K, ms_max, cfg,
                  {"exact_e3b": {"value": K / (ms_exact * 1e-3), "unit": "timesteps/s"},
                   "surrogate_over_exact": (K / (ms_max * 1e-3)) / (K / (ms_exact * 1e-3)),
                   "threebody_force_rmse_over_rms": rmse / rms, "threebody_force_rms": rms,
                   "train_loss_first_last": [l0, l1], "collect_s": t_collect, "train_s": t_train},
                  clk, int(k1 - k0))
    if dist is not None:
        barrier(dist, dev)
        dist.destroy_process_group()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.workload in ("batched", "surrogate"):
        import torch
        from md_engine_b200._lib import lib
        torch.cuda.set_device(local)
        lib().mdx_set_device(local)
        (run_batched if args.workload == "batched" else run_surrogate)(args, rank, world, local)
        return
    import torch
    from md_engine_b200 import IntegratorVerlet, kernel_launches
    from md_engine_b200._lib import lib
    torch.cuda.set_device(local)
    lib().mdx_set_device(local)
    dist = init_pg(world, "nccl")
    dev = torch.device("cuda", local)
    sysd, st, fx, cfg, dt = workload(args.workload, seed=20261203 + rank, eq_steps=args.eq_steps)
    it = IntegratorVerlet(st)
    # warm-up: prepare, capture graphs, settle clocks (untimed)
    it.run(max(args.warmup, 3))
    # the run-start tuning of the molecule form's pair grid (Integrator::tune's
    # role); a no-op for the per-site form.  Untimed, state untouched.
    tuned_cap, tuned_ms = it.autotune()
    it.run(3)
    K = args.steps
    P = 10
    barrier(dist, dev)
    torch.cuda.synchronize()
    k0 = kernel_launches()
    with ClockSampler(local) as clk:
        ms = it.runTimed(K, P, L2_FLUSH_BYTES)
    k1 = kernel_launches()
    torch.cuda.synchronize()
    barrier(dist, dev)
    ms_max = reduce_max(dist, ms, dev)
    value = world * K / (ms_max * 1e-3)
    t_end = timed_temperature(args.workload, sysd, st)
    # end to end through the C ABI with host buffers: H2D positions+velocities,
    # P steps, D2H positions+velocities+forces, per call
    x, v, _ = st.getAtoms()
    n = len(x)
    e2e_calls = max(1, K // P)
    # one untimed call first (pinned staging allocation, graph shapes)
    out = it.runHost(P, positions=x, velocities=v)
    x, v = out["pos"], out["vel"]
    barrier(dist, dev)
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        out = it.runHost(P, positions=x, velocities=v)
        x, v = out["pos"], out["vel"]
    t_e2e = time.perf_counter() - t0
    t_e2e = reduce_max(dist, t_e2e, dev)
    e2e = world * e2e_calls * P / t_e2e
    # roofline of the dominant kernel (pair forces): algorithmic bytes per
    # launch = 16N (x) + 4N (q) + 16N (f) + 4 N nbar (directed list entries)
    counts, nbr, _ = st.getNeighborList()
    nbar = float(np.mean(counts))
    # FP32 view of the same kernel: 75 flops per directed pair within the
    # pair cutoff (every listed pair with r < rc, zero pairs included, the
    # counting convention of the water pair figure of 0.50 GFLOP per launch)
    xa, _, _ = st.getAtoms()
    rc = 2.5 if args.workload == "lj" else 9.0
    Lb = np.asarray(sysd.L, np.float64)
    ii = np.repeat(np.arange(len(counts)), counts)
    jj = nbr[np.arange(nbr.shape[1])[None, :] < counts[:, None]]
    dd = xa[jj] - xa[ii]
    dd -= Lb * np.rint(dd / Lb)
    pairs_rc = int(np.count_nonzero(np.einsum("ij,ij->i", dd, dd) < rc * rc))
    charged = args.workload != "lj"
    mol_form = int(st.pairForm) == 2
    if mol_form:
        # the molecule form's kernel (k_pair_mol): 16 B positions read + 16 B
        # forces written per site, 4 B per molecule-pair list entry (the site
        # charges and types are per-molecule constants, not streamed)
        nmol = n // 4
        nbar_mol = float(st.molListEntries) / nmol
        alg_bytes = n * (16 + 16) + 4.0 * nmol * nbar_mol
    else:
        nbar_mol = None
        alg_bytes = n * (16 + (4 if charged else 0) + 16) + 4.0 * n * nbar
    # the kernel as the step launches it (molecule form: its grid capped so
    # the P3M chain runs beside it)
    pair_ms = st.timeStage("pair", iters=20, flushBytes=L2_FLUSH_BYTES)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (pair_ms * 1e-3) / 1e9
    stages = {}
    for sname in ("pair", "p3m", "e3b", "nlist"):
        try:
            stages[sname] = round(st.timeStage(sname, iters=10, flushBytes=L2_FLUSH_BYTES) * 1000.0, 2)
        except Exception:
            pass
    line = None
    if rank == 0:
        ns_day = value / world * dt * 86400 / 1e6 if args.workload != "lj" else None
        line = {
            "metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 reductions, f64 SETTLE)",
            "data": "synthetic (seeded lattice + random orientations + Maxwell-Boltzmann, "
                    f"relaxed {args.eq_steps} untimed steps at the target temperature)",
            "config": dict(cfg, l2="flushed between timed 10-step chunks (256 MiB write)",
                           start=f"equilibrated: {args.eq_steps} steps, tight Nose-Hoover, before warm-up",
                           parallelism="replicas only" if world > 1 else "single system",
                           pair_grid_autotuned={"blocks_per_sm": tuned_cap, "ms_per_force_phase": tuned_ms}
                           if tuned_cap else "per-site form: no grid shape tuned"),
            "ns_per_day": ns_day,
            "temperature_end_of_timed_region": t_end,
            "e2e": {"value": e2e, "unit": "timesteps/s",
                    "h2d_bytes_per_step": int(2 * 24 * n / P), "d2h_bytes_per_step": int(3 * 24 * n / P)},
            "gpu_launches": int(k1 - k0),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": profile_traffic(args.workload + ("_pair_mol" if mol_form else "_pair")),
                         "kernel": ("k_pair_mol (molecule form: LJ + Ewald real space by molecule pair)" if mol_form
                                    else "k_pair (LJ + Ewald real space)"),
                         "kernel_ms": pair_ms, "alg_bytes_per_launch": alg_bytes, "nbar": nbar,
                         "nbar_molecule_pairs": nbar_mol, "peak_source": peak_kind,
                         "fp32": None if not charged else {"achieved": 75.0 * pairs_rc / (pair_ms * 1e-3) / 1e12,
                                  "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s",
                                  "frac": 75.0 * pairs_rc / (pair_ms * 1e-3) / 1e12 / FP32_PEAK_TFLOPS,
                                  "pairs_within_rc": pairs_rc, "flops_per_pair": 75,
                                  "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 x 1.965 GHz"}},
            "stage_us": stages,
            "clocks": clk.summary(),
        }
        if not args.no_nve:
            try:
                xf, vf, _ = st.getAtoms()
                line["nve_drift"] = nve_drift(args.workload, xf, vf, 20261203 + rank)
            except Exception as ex:  # reported, never required
                line["nve_drift"] = {"value": None, "error": str(ex)}
        if world == 1 and not args.no_cpu_baseline:
            # the CPU baseline leg: the oracle's FP64 step timed on the host
            # cores, and the same FP64 evaluation as the reference values of
            # the timed state's forces, energies and virial (outside the
            # timed region)
            try:
                from oracle import cpu_step
                res = cpu_step.time_steps(sysd, args.workload, nsample=10, warmup=2, repeats=3)
                line["cpu_baseline"] = {"value": res["steps_per_s"], "unit": "timesteps/s", "cores": res["cores"],
                                        "kind": "port", "sample": res["sample"]}
            except Exception as ex:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "unit": "timesteps/s", "cores": os.cpu_count(),
                                        "kind": "port", "sample": f"failed: {ex}"}
            try:
                line["fp64_oracle_error"] = fp64_errors(args.workload, sysd, st, fx)
            except Exception as ex:
                line["fp64_oracle_error"] = {"error": str(ex)}
        print(json.dumps(line))
    if dist is not None:
        barrier(dist, dev)
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
