"""Throughput of the MD hot path on B200: MATS (million atom-timesteps per
second) and TPS for the Kob-Andersen NVT system with cell lists.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n PARTICLES] [--impl reference]

Workload (one rank): Kob-Andersen 80:20 LJ mixture, shifted force at 2.5
sigma_ab, density 1.2, Nose-Hoover NVT T = 0.45 (tau 0.2), dt 0.005, float32,
cell-list neighbour list with skin 0.3, N = 1,048,576 by default (the largest
N of the reference's KA sweep), seeded synthetic input.  A step is one MD time
step (forces, integration, runtime actions, neighbour-list check/rebuild);
TPS counts steps over the timeblock's device time as gamdpy does
(benchmarks/benchmark_LJ.py:90).  The working set per step (neighbour list,
~0.45 GB) is larger than the 126 MB L2, so no flush is needed between steps.

--gpus N (one process per GPU under torchrun): N independent replicas with
different seeds ("replicas only": one MD system does not shard); value = total
atom-steps / max over ranks of the device time.

--impl reference: the reference's algorithm on the host cores (the CPU
oracle, all threads), same workload, a bounded sample of steps.
"""
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

METRIC = "MATS (million atom-timesteps/s), KA-LJ NVT cell lists, 1 B200"
UNIT = "Matom-steps/s"
MOMENTUM_RESET_EVERY = 100  # the only runtime action, as benchmarks/benchmark_LJ.py:28-47
# Untimed steps that take the seeded lattice through its first melting (the
# neighbour list is rebuilt far more often while the lattice breaks up)
# before the warm-up, in both arms: the workload is the liquid at the state
# point.  The reference's benchmark likewise runs an untimed timeblock before
# timing (benchmarks/benchmark_LJ.py:71-80).
EQUILIBRATION_STEPS = 200
PATH_NAMES = {0: "graph", 1: "persistent", 2: "cluster", 3: "cluster-global", 4: "persistent-staged-halos"}


def ka_workload(n, langevin=False):
    """The workload string both arms print in ``config`` (the same system,
    integrator, list and runtime actions)."""
    thermo = "NVT_Langevin alpha=0.2" if langevin else "NVT Nose-Hoover tau=0.2"
    return (f"KA-LJ 80:20 SF rc=2.5 sigma_ab, rho=1.2, {thermo} T=0.45, dt=0.005, cells skin=0.3, "
            f"MomentumReset({MOMENTUM_RESET_EVERY}), N={n}, timed after {EQUILIBRATION_STEPS} untimed steps "
            "from the seeded lattice")


def ka_config(n, langevin=False):
    return {"workload": ka_workload(n, langevin), "n": n,
            "l2": "per-step working set (neighbour list, ~0.45 GB at N=1M) > 126 MB L2, no flush"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=200)
    p.add_argument("--n", "--particles", dest="n", type=int, default=1_048_576)
    p.add_argument("--impl", default="b200", choices=["b200", "reference", "numba"],
                   help="reference: the CPU port of the reference on the host cores; numba: gamdpy's own "
                        "numba.cuda path from baseline/_ref on the same GPU, beside this library")
    p.add_argument("--block", type=int, default=500, help="steps per timeblock")
    p.add_argument("--profile", action="store_true",
                   help="only warm-up and timed steps (for ncu): no e2e, CPU baseline or clock sampling")
    p.add_argument("--tp", type=int, default=0, help="lanes per particle (0 = library default)")
    p.add_argument("--trace", action="store_true", help="with --profile: phase trace of the persistent kernel")
    p.add_argument("--workload", default="ka", choices=["ka", "lj2048", "lj8m", "batch", "adjoint"],
                   help="ka: one KA system of --n particles; batch: --replicas KA replicas of uneven N, "
                        "density and temperature advanced together, against the same replicas run one by one")
    p.add_argument("--replicas", type=int, default=128)
    p.add_argument("--langevin", action="store_true",
                   help="ka: NVT_Langevin (T 0.45, alpha 0.2, seed 1) in place of the Nose-Hoover thermostat")
    p.add_argument("--sweep", action="store_true",
                   help="ka: MATS/TPS vs N over 512 ... 1 048 576, one JSON line per N with the oracle beside it")
    p.add_argument("--lj-cells", type=int, default=128,
                   help="lj8m: FCC unit cells per side (128: 8 388 608 particles; smaller for profiling)")
    p.add_argument("--autotune", action="store_true",
                   help="batch: pick the batch shape (particles per CTA, lanes) by timing")
    p.add_argument("--no-extras", action="store_true",
                   help="default line without the small-N and batch sub-measurements")
    return p.parse_args()


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def allreduce_max(pg, x, local):
    if pg is None:
        return x
    import torch
    dev = torch.device("cuda", local) if pg.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # sampling is running before the timed region starts
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # the first sample was taken before the timed region started
        lines = self.lines[1:] if len(self.lines) > 1 else self.lines
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic_per_atom_step():
    """DRAM bytes per atom-step of k_run (rebuilds included) from the committed
    ncu summary (profiles/run_kernel_ka.txt, line 'traffic_bytes_per_atom_step')."""
    path = os.path.join(ROOT, "profiles", "run_kernel_ka.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_atom_step"):
                    return float(line.split("=")[1].split()[0])
    except (OSError, ValueError, IndexError):
        pass
    return None


def trace_summary(tags, ns):
    """Per-phase times from the persistent kernel's barrier trace (tags:
    1 step, 2 evaluation, 3 rebuild phase, 4 rebuild done, 5 start, 6 end of
    block 0's step phase; 7 and 8 the last block's arrival and release)."""
    tags, ns = np.asarray(tags), np.asarray(ns)
    order = np.argsort(ns, kind="stable")
    tags, ns = tags[order], ns[order]
    # the step barrier split: block 0's phase end -> last arrival -> release
    # -> block 0 past the barrier (tags 7 and 8 come from the last block)
    arrive_us, book_us, release_us = [], [], []
    for k in range(len(tags) - 3):
        if tags[k] == 6 and tags[k + 1] == 7 and tags[k + 2] == 8 and tags[k + 3] == 1:
            arrive_us.append((ns[k + 1] - ns[k]) / 1e3)
            book_us.append((ns[k + 2] - ns[k + 1]) / 1e3)
            release_us.append((ns[k + 3] - ns[k + 2]) / 1e3)
    keep = (tags != 7) & (tags != 8)
    tags, ns = tags[keep], ns[keep]
    step_us, rebuild_us, phase_us, sphase_us, bar_us = [], [], [], [], []
    start = None
    for k in range(1, len(tags)):
        dt = (ns[k] - ns[k - 1]) / 1e3
        if tags[k] == 6 and k >= 1 and tags[k - 1] in (1, 4, 5):
            sphase_us.append(dt)
        if tags[k] == 1 and tags[k - 1] == 6:
            bar_us.append(dt)
            if k >= 2 and tags[k - 2] in (1, 4):
                step_us.append((ns[k] - ns[k - 2]) / 1e3)
        if tags[k] == 3 and tags[k - 1] in (1, 5) and start is None:
            start = ns[k - 1]
        if tags[k] in (3, 4):
            phase_us.append(dt)
        if tags[k] == 4:
            if start is None:  # builds without intermediate marks
                start = ns[k - 1]
            rebuild_us.append((ns[k] - start) / 1e3)
            start = None
    med = lambda x: float(np.median(x)) if x else None
    return {"entries": int(len(tags)), "steps": len(step_us), "step_us_median": med(step_us),
            "step_phase_us_median": med(sphase_us), "step_barrier_us_median": med(bar_us),
            "step_us_mean": float(np.mean(step_us)) if step_us else None, "rebuilds": len(rebuild_us),
            "rebuild_us_median": med(rebuild_us),
            "rebuild_phase_us": [round(x, 1) for x in phase_us[:5]],
            "barrier_split_us_median": {"to_last_arrival": med(arrive_us), "bookkeeping": med(book_us),
                                        "release_to_block0": med(release_us)}}


def cpu_reference(args, n, steps, seed=0):
    """The oracle on the host cores: ka workload, `steps` steps after one
    build.  Returns (MATS, threads, seconds)."""
    from gamdpy_b200 import workloads
    from oracle import oracle as O
    conf = workloads.ka_configuration(n, seed=seed)
    tab = O.param_table([workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT])
    # the reference's default list kind by size (get_default_compute_plan.py:83-86)
    nblist = "linked lists" if n > 6000 else "N squared"
    run = O.Run(conf["r"], conf["v"], conf["m"], conf.ptype, conf.simbox.lengths, tab, nblist=nblist,
                skin=0.3, max_nbs=300, integrator="NVT", dt=0.005, temperature=0.45, tau=0.2,
                reset_every=MOMENTUM_RESET_EVERY)
    run.run_timeblock(EQUILIBRATION_STEPS)  # the workload's untimed equilibration
    r0 = run.rebuilds
    t0 = time.perf_counter()
    run.run_timeblock(steps)
    dt = time.perf_counter() - t0
    return n * steps / dt / 1e6, O.num_threads(), dt, run.rebuilds - r0


SWEEP_N = (512, 2048, 8192, 65536, 262144, 1048576)


def run_sweep(args):
    """MATS and TPS vs N for the KA workload (rho 1.2, NVT T 0.45, cells skin
    0.3), N = 512 ... 1 048 576 as the reference's benchmark sweep
    (benchmarks/benchmark_LJ.py:100-146): per N about 2e8 atom-steps on the
    device (at most 10^5 steps, timeblocks of 500 or fewer), the path the
    library chose, the HBM roofline fraction of the timed launches, and the
    oracle on the host cores over a bounded sample of the same system."""
    import gamdpy_b200 as gp
    from gamdpy_b200 import workloads
    rank, world, local, pg = dist_setup(args)
    peak, peak_kind = measured_peak_hbm()
    for n in SWEEP_N:
        conf = workloads.ka_configuration(n, seed=1234 + rank)
        pp = workloads.ka_pair_potential(max_num_nbs=300)
        integ = gp.integrators.NVT(temperature=0.45, tau=0.2, dt=0.005)
        block = 500
        nblocks = max(2, min(200, int(2e8 / n / block)))
        plan = {"pb": 64, "tp": 1, "lanes": args.tp, "skin": 0.3, "UtilizeNIII": False, "gridsync": False,
                "nblist": "linked lists"}
        sim = gp.Simulation(conf, pp, integ, [gp.MomentumReset(MOMENTUM_RESET_EVERY)], num_timeblocks=8,
                            steps_per_timeblock=block, compute_plan=plan, storage="memory", device=local)
        dev = sim._sim
        dev.run(0.0, EQUILIBRATION_STEPS)
        dev.run(0.0, max(3, args.warmup))
        dev.clear_status()
        barrier(pg)
        ms = sum(dev.run(float(b * block * 0.005), block) for b in range(nblocks))
        t_max = allreduce_max(pg, ms / 1e3, local)
        steps = nblocks * block
        mean_nbs, _ = dev.nblist_stats()
        bpa = 4.0 * mean_nbs + 64.0
        achieved = bpa * n * steps / t_max / 1e9
        line = {"sweep": True, "n": n, "mats": n * steps * world / t_max / 1e6, "tps": steps / t_max,
                "steps": steps, "ms_per_step": t_max * 1e3 / steps, "path": PATH_NAMES.get(dev.last_path(), dev.last_path()),
                "hbm_frac": achieved / peak, "hbm_peak": peak, "peak_source": peak_kind,
                "algorithmic_bytes_per_atom_step": bpa, "n_gpus": world}
        if rank == 0 and world == 1:
            cps = max(2, min(400, int(3e6 / n)))
            cmats, threads, secs, _ = cpu_reference(args, n, cps)
            line["cpu_baseline"] = {"value": cmats, "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": f"{cps} steps ({secs:.1f} s)"}
        if rank == 0:
            print(json.dumps(line), flush=True)
        del sim, dev
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()


def run_reference_arm(args):
    rank, world, local, pg = dist_setup(args)
    if rank != 0:
        barrier(pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    # bounded sample of the same workload: up to 50 steps of the full-size
    # system after the first list build (~10 s on 16 host threads at N = 1M),
    # so the sample holds neighbour-list rebuilds as the GPU arm's steps do
    steps = max(1, min(args.steps, 50))
    mats, threads, secs, rebuilds = cpu_reference(args, args.n, steps)
    sample = (f"{steps} steps of the N={args.n} system after its {EQUILIBRATION_STEPS} untimed steps "
              f"({rebuilds} list rebuilds inside)")
    line = {
        "impl": "reference", "metric": METRIC, "value": mats, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": 1, "ms_per_step": secs / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded KA lattice)",
        "config": ka_config(args.n),
        "cpu_baseline": {"value": mats, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": mats, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()


# ---------------------------------------------------------------------------
# comparator: gamdpy's own numba.cuda path on the same GPU
# ---------------------------------------------------------------------------
GAMDPY_REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def _import_gamdpy_stock():
    """gamdpy, unmodified, from baseline/_ref.  h5py and matplotlib are not
    in this image: gamdpy imports them at module level
    (simulation/Simulation.py:20, interactions/pair_potential.py:5) and, with
    storage='memory', writes its output into an h5py.File; a dict with
    ``attrs`` stands in for that file and an empty module for matplotlib."""
    import types
    h5 = types.ModuleType("h5py")

    class File(dict):
        def __init__(self, *a, **k):
            super().__init__()
            self.attrs = {}

        def create_dataset(self, name, data=None, shape=None, dtype=None, **k):
            self[name] = np.zeros(shape, dtype=dtype) if data is None else np.array(data, dtype=dtype)
            return self[name]

        def create_group(self, name):
            self[name] = File()
            return self[name]

        def close(self):
            pass

    h5.File = File
    sys.modules.setdefault("h5py", h5)
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.path.insert(0, GAMDPY_REF_DIR)
    import warnings
    warnings.filterwarnings("ignore")
    from numba import config
    config.CUDA_LOW_OCCUPANCY_WARNINGS = False
    import gamdpy
    return gamdpy


def gamdpy_numba_tps(rp, case, n, steps):
    """TPS of gamdpy's Simulation on one of this bench's systems (the same
    seeded input), its default compute plan with the workload's list kind
    and skin, timed as benchmarks/benchmark_LJ.py:66-91: a first run of the
    timeblock (JIT and warm-up), then a second whose CUDA-event block time
    gives TPS."""
    from gamdpy_b200 import workloads
    if case == "lj2048":
        src = workloads.lj_configuration([8, 8, 8], 0.973, 0.7, seed=0)
        params = [1.0, 1.0, 2.5]
        integ = rp.integrators.NVE(dt=0.005)
        skin, nblist = 0.5, "N squared"
    else:
        src = workloads.ka_configuration(n, seed=1234)
        params = [workloads.KA_SIGMA, workloads.KA_EPSILON, workloads.KA_CUT]
        integ = rp.integrators.NVT(temperature=0.45, tau=0.2, dt=0.005)
        skin, nblist = 0.3, "linked lists"
    conf = rp.Configuration(D=3)
    conf["r"] = src["r"].copy()
    conf.simbox = rp.Orthorhombic(3, np.asarray(src.simbox.lengths, np.float32))
    conf.ptype[:] = src.ptype
    conf["m"] = 1.0
    conf["v"] = src["v"].copy()
    pp = rp.PairPotential(rp.apply_shifted_force_cutoff(rp.LJ_12_6_sigma_epsilon), params=params, max_num_nbs=300)
    plan = rp.get_default_compute_plan(conf)
    plan["skin"] = np.float32(skin)
    plan["nblist"] = nblist
    sim = rp.Simulation(conf, pp, integ, [rp.MomentumReset(MOMENTUM_RESET_EVERY)], num_timeblocks=1,
                        steps_per_timeblock=steps, compute_plan=plan, storage="memory", verbose=False)
    for _ in sim.run_timeblocks():
        pass
    for _ in sim.run_timeblocks():
        pass
    tps = sim.last_num_blocks * sim.steps_per_block / np.sum(sim.timing_numba_blocks) * 1000
    return {"case": case, "n": int(conf.N), "steps": steps, "tps": float(tps), "mats": float(tps * conf.N / 1e6),
            "compute_plan": {k: (v.item() if hasattr(v, "item") else v) for k, v in sim.compute_plan.items()}}


def run_numba_comparator(args):
    """gamdpy's own numba.cuda path on this GPU, beside this library, on the
    KA workload at N = 2048, 65 536 and --n, and on the LJ 2048 case."""
    rank, world, local, pg = dist_setup(args)
    if rank != 0:
        barrier(pg)
        return
    if not os.path.isdir(os.path.join(GAMDPY_REF_DIR, "gamdpy")):
        print(json.dumps({"impl": "gamdpy-numba-cuda", "unavailable": "gamdpy is not installed in baseline/_ref"}))
        return
    rp = _import_gamdpy_stock()
    cases = [("lj2048", 2048, 10_000), ("ka", 2048, 10_000), ("ka", 65536, 2000), ("ka", args.n, 500)]
    out = []
    for case, n, steps in cases:
        try:
            g = gamdpy_numba_tps(rp, case, n, steps)
        except Exception as e:  # record and go on with the other sizes
            g = {"case": case, "n": n, "error": f"{type(e).__name__}: {e}"[:300]}
        if "error" not in g:
            b = measure_lj2048(local, steps, min(steps, 1000), 200) if case == "lj2048" else \
                measure_ka(local, n, steps, min(steps, 500), 200)
            g["b200_tps"] = b["tps"]
            g["ratio_tps"] = b["tps"] / g["tps"]
        out.append(g)
        print(json.dumps({"impl": "gamdpy-numba-cuda", **g}), flush=True)
    barrier(pg)


def measure_batch(local, replicas, steps, block, warmup, autotune=False, seed=2024, e2e_blocks=0):
    """Batched replicas: ``replicas`` KA systems (N log-uniform 256-32768,
    rho in [1.1, 1.3], T in [0.4, 1.0], NVT dt 0.005, cells skin 0.3) advanced
    together by SimulationBatch, against the same systems advanced one after
    another through Simulation (each its own launches).  Device times in ms;
    with e2e_blocks > 0 also the wall time of that many timeblocks through
    SimulationBatch.run_timeblocks (upload once, per timeblock every
    replica's state back to the host)."""
    import gamdpy_b200 as gp
    from gamdpy_b200 import workloads

    points = workloads.ka_replica_sweep(replicas, seed=seed)
    block = min(block, max(1, steps))
    nblocks = max(1, steps // block)
    steps = nblocks * block
    plan = {"pb": 64, "tp": 1, "lanes": 0, "skin": 0.3, "UtilizeNIII": False, "gridsync": False,
            "nblist": "linked lists"}
    sims = []
    for k, (n, rho, temp) in enumerate(points):
        conf = workloads.ka_configuration(n, rho=rho, temperature=temp, seed=k)
        integ = gp.integrators.NVT(temperature=temp, tau=0.2, dt=0.005)
        sims.append(gp.Simulation(conf, workloads.ka_pair_potential(max_num_nbs=300), integ,
                                  [gp.MomentumReset(MOMENTUM_RESET_EVERY)], num_timeblocks=max(nblocks, e2e_blocks),
                                  steps_per_timeblock=block, compute_plan=plan, storage="memory", device=local))
    total_n = sum(p[0] for p in points)
    batch = gp.SimulationBatch(sims)
    tuned = batch.autotune(steps=min(block, 200)) if autotune else batch.shape
    w = max(3, min(warmup, block))
    for s_ in sims:  # warm-up of both paths
        s_.configuration.copy_to_device()
        s_._sim.run(0.0, w)
    batch.integrate_self(0.0, w)
    # sequential: every replica's timeblocks, one replica after another
    for s_ in sims:
        s_.configuration.copy_to_device()
    ms_seq = 0.0
    for s_ in sims:
        for b in range(nblocks):
            ms_seq += s_._sim.run(float(b * block * 0.005), block)
    # batched: one call per timeblock for all replicas
    for s_ in sims:
        s_.configuration.copy_to_device()
    clocks = ClockSampler(local)
    clocks.start()
    ms_bat = 0.0
    for b in range(nblocks):
        ms_bat += batch.integrate_self(float(b * block * 0.005), block)
    clock_info = clocks.stop()
    paths = batch.paths()
    out = {"workload": f"{replicas} KA-LJ NVT replicas (N 256-32768 log-uniform, rho 1.1-1.3, T 0.4-1.0), "
                       f"cells skin=0.3, MomentumReset({MOMENTUM_RESET_EVERY}), total N={total_n}",
           "replicas": replicas, "total_n": total_n, "steps": steps, "timeblock_steps": block,
           "ms_batched": ms_bat, "ms_sequential": ms_seq,
           "mats_batched": total_n * steps / ms_bat / 1e3, "mats_sequential": total_n * steps / ms_seq / 1e3,
           "speedup_vs_sequential": ms_seq / ms_bat, "shape": {"particles_per_cta": tuned[0],
                                                               "clg_particles_per_cta": tuned[1],
                                                               "clg_tp": tuned[2], "autotuned": bool(autotune)},
           "cluster_systems": int(sum(1 for p in paths if p == 2)),
           "grid_systems": int(sum(1 for p in paths if p != 2)), "clocks": clock_info}
    if e2e_blocks > 0:
        t0 = time.perf_counter()
        for _ in batch.run_timeblocks(e2e_blocks):
            pass
        out["e2e_s"] = time.perf_counter() - t0
        out["e2e_blocks"] = e2e_blocks
    del batch, sims
    return out


def run_batch(args):
    rank, world, local, pg = dist_setup(args)
    r = measure_batch(local, args.replicas, args.steps, args.block, args.warmup, autotune=args.autotune,
                      seed=2024 + rank, e2e_blocks=2)
    steps, block, total_n = r["steps"], r["timeblock_steps"], r["total_n"]
    t_bat = allreduce_max(pg, r["ms_batched"] / 1e3, local)
    t_seq = allreduce_max(pg, r["ms_sequential"] / 1e3, local)
    e2e_s = allreduce_max(pg, r["e2e_s"], local)
    e2e_steps = r["e2e_blocks"] * block
    h2d = total_n * (12 + 12 + 4 + 4 + 12)
    d2h = total_n * (12 + 12 + 12 + 12 + 4 * 5)
    line = {
        "metric": "MATS batched KA replicas (N 256-32768, rho 1.1-1.3, T 0.4-1.0), 1 B200",
        "value": total_n * steps * world / t_bat / 1e6, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": max(3, min(args.warmup, block)), "ms_per_step": t_bat * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded KA lattices)",
        "config": {"workload": r["workload"], "replicas": args.replicas, "total_n": total_n,
                   "timeblock_steps": block, "shape": r["shape"],
                   "cluster_systems": r["cluster_systems"], "grid_systems": r["grid_systems"],
                   "l2": "working set of all replicas > 126 MB L2, no flush"},
        "sequential": {"value": total_n * steps * world / t_seq / 1e6, "unit": UNIT,
                       "ms_per_step": t_seq * 1e3 / steps,
                       "note": "the same replicas, one Simulation after another (device time summed)"},
        "speedup_vs_sequential": t_seq / t_bat,
        "e2e": {"value": total_n * e2e_steps * world / e2e_s / 1e6, "unit": UNIT,
                "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
                "timeblock_steps": block},
        "clocks": r["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()


def measure_lj2048(local, steps, block, warmup, seed=0, e2e_blocks=0):
    """The reference's small plain case: single-component LJ (shifted force,
    rc = 2.5), FCC 8x8x8 = 2048 particles at rho = 0.973, Maxwell-Boltzmann
    velocities at T = 0.7 (seeded), NVE dt = 0.005, N^2 list with skin 0.5,
    MomentumReset(100) as the reference's benchmark.  TPS and MATS over the
    timeblocks' device time."""
    import gamdpy_b200 as gp
    from gamdpy_b200 import workloads
    conf = workloads.lj_configuration([8, 8, 8], 0.973, 0.7, seed=seed)
    n = conf.N
    pp = workloads.lj_pair_potential(cut=2.5, shifted_force=True, max_num_nbs=300)
    block = min(block, max(1, steps))
    nblocks = max(1, steps // block)
    steps = nblocks * block
    plan = {"pb": 8, "tp": 16, "lanes": 0, "skin": 0.5, "UtilizeNIII": False, "gridsync": True,
            "nblist": "N squared"}
    sim = gp.Simulation(conf, pp, gp.integrators.NVE(dt=0.005), [gp.MomentumReset(MOMENTUM_RESET_EVERY)],
                        num_timeblocks=nblocks, steps_per_timeblock=block, compute_plan=plan, storage="memory",
                        device=local)
    dev = sim._sim
    dev.run(0.0, max(3, warmup))
    clocks = ClockSampler(local)
    clocks.start()
    ms = sum(dev.run(float(b * block * 0.005), block) for b in range(nblocks))
    clock_info = clocks.stop()
    out = {"workload": "LJ SF rc=2.5, FCC 8x8x8 N=2048 rho=0.973 T=0.7, NVE dt=0.005, N^2 list skin 0.5, "
                       f"MomentumReset({MOMENTUM_RESET_EVERY})",
           "n": n, "steps": steps, "timeblock_steps": block, "ms": ms, "tps": steps / ms * 1e3,
           "mats": n * steps / ms / 1e3, "ms_per_step": ms / steps, "path": dev.last_path(), "clocks": clock_info}
    if e2e_blocks > 0:
        t0 = time.perf_counter()
        conf.copy_to_device()
        for b in range(e2e_blocks):
            dev.run(float(b * block * 0.005), block)
            conf.copy_to_host()
        out["e2e_s"] = time.perf_counter() - t0
        out["e2e_blocks"] = e2e_blocks
    return out


def measure_ka(local, n, steps, block, warmup, seed=1234, tp=0):
    """KA workload at N particles (the default line's system at another
    size): TPS and MATS over the timeblocks' device time, with the path the
    library chose."""
    import gamdpy_b200 as gp
    from gamdpy_b200 import workloads
    conf = workloads.ka_configuration(n, seed=seed)
    pp = workloads.ka_pair_potential(max_num_nbs=300)
    integ = gp.integrators.NVT(temperature=0.45, tau=0.2, dt=0.005)
    block = min(block, max(1, steps))
    nblocks = max(1, steps // block)
    steps = nblocks * block
    plan = {"pb": 64, "tp": 1, "lanes": tp, "skin": 0.3, "UtilizeNIII": False, "gridsync": False,
            "nblist": "linked lists"}
    sim = gp.Simulation(conf, pp, integ, [gp.MomentumReset(MOMENTUM_RESET_EVERY)], num_timeblocks=nblocks,
                        steps_per_timeblock=block, compute_plan=plan, storage="memory", device=local)
    dev = sim._sim
    dev.run(0.0, EQUILIBRATION_STEPS)
    dev.run(0.0, max(3, warmup))
    clocks = ClockSampler(local)
    clocks.start()
    ms = sum(dev.run(float(b * block * 0.005), block) for b in range(nblocks))
    clock_info = clocks.stop()
    path = dev.last_path()
    return {"workload": ka_workload(n), "n": n, "steps": steps, "timeblock_steps": block, "ms": ms,
            "tps": steps / ms * 1e3, "mats": n * steps / ms / 1e3, "ms_per_step": ms / steps,
            "path": PATH_NAMES.get(path, path), "clocks": clock_info}


def run_lj_small(args):
    rank, world, local, pg = dist_setup(args)
    r = measure_lj2048(local, args.steps, args.block, args.warmup, seed=rank, e2e_blocks=4)
    n, steps, block = r["n"], r["steps"], r["timeblock_steps"]
    t_max = allreduce_max(pg, r["ms"] / 1e3, local)
    e2e_s = allreduce_max(pg, r["e2e_s"], local)
    tps = steps / t_max
    e2e_blocks = r["e2e_blocks"]
    line = {
        "metric": "TPS (time steps/s), LJ N=2048 NVE N^2 list, 1 B200", "value": tps * world, "unit": "steps/s",
        "n_gpus": world, "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": t_max * 1e3 / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded FCC lattice)",
        "config": {"workload": r["workload"], "n": n, "mats": n * tps * world / 1e6, "timeblock_steps": block,
                   "path": r["path"], "l2": "working set < L2; the metric is step latency, so no flush"},
        "e2e": {"value": e2e_blocks * block * world / e2e_s, "unit": "steps/s",
                "h2d_bytes_per_step": n * 44 / (e2e_blocks * block), "d2h_bytes_per_step": n * 68 / block},
        "clocks": r["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()


def measure_lj_large(local, cells, steps, warmup, seed=0, tp=0):
    """Large-N LJ with on-the-fly structure: FCC cells^3 (128^3 = 8 388 608
    particles) at rho = 0.84, T = 1.0 (seeded), shifted-force rc = 2.5, NVE
    dt = 0.004, cell lists skin 0.5; every 100 steps the RDF over [0, 5) with
    1000 bins (integer counts) and S(q) on the q-vectors of the first 200
    |n|^2 shells (the reference's non-negative generator), both from the
    device-resident state.  Device times (CUDA events on the library's
    stream) of MD, RDF and S(q), seconds; wall times of the update() calls."""
    import gamdpy_b200 as gp
    from gamdpy_b200 import workloads
    c = cells
    conf = workloads.lj_configuration([c, c, c], 0.84, 1.0, seed=seed)
    n = conf.N
    pp = workloads.lj_pair_potential(cut=2.5, shifted_force=True, max_num_nbs=200)
    every = 100
    nblocks = max(1, steps // every)
    steps = nblocks * every
    plan = {"pb": 256, "tp": 1, "lanes": tp, "skin": 0.5, "UtilizeNIII": False, "gridsync": False,
            "nblist": "linked lists"}
    sim = gp.Simulation(conf, pp, gp.integrators.NVE(dt=0.004), [], num_timeblocks=nblocks, steps_per_timeblock=every,
                        compute_plan=plan, storage="memory", device=local)
    dev = sim._sim
    rdf = gp.CalculatorRadialDistribution(conf, bins=1000, r_max=5.0)
    sq = gp.CalculatorStructureFactor(conf)
    L = float(conf.simbox.lengths[0])
    sq.generate_q_vectors(2 * np.pi * np.sqrt(237.5) / L)
    nq = len(sq.q_vectors)
    dev.run(0.0, max(3, warmup))
    rdf.update()
    sq.update()
    clocks = ClockSampler(local)
    clocks.start()
    t_md = t_rdf = t_sq = 0.0
    w_rdf = w_sq = 0.0
    each_rdf, each_sq = [], []
    t0 = time.perf_counter()
    for b in range(nblocks):
        t_md += dev.run(float(b * every * 0.004), every) / 1e3
        t1 = time.perf_counter()
        rdf.update()
        each_rdf.append(dev.last_analysis_ms())
        t_rdf += each_rdf[-1] / 1e3
        t2 = time.perf_counter()
        sq.update()
        each_sq.append(dev.last_analysis_ms())
        t_sq += each_sq[-1] / 1e3
        t3 = time.perf_counter()
        w_rdf += t2 - t1
        w_sq += t3 - t2
    wall = time.perf_counter() - t0
    clock_info = clocks.stop()
    pairs = float(rdf.rdf_list[-1].sum())  # ordered pairs counted in one update
    out = {"workload": f"LJ SF rc=2.5, FCC {c}^3 rho=0.84 T=1.0, NVE dt=0.004, cells skin 0.5; RDF r<5 "
                       "1000 bins and S(q) on the first 200 |n|^2 shells every 100 steps",
           "n": n, "nq": nq, "steps": steps, "t_md": t_md, "t_rdf": t_rdf, "t_sq": t_sq,
           "mats": n * steps / (t_md + t_rdf + t_sq) / 1e6, "md_ms_per_step": t_md * 1e3 / steps,
           "rdf_ms_per_update": t_rdf * 1e3 / nblocks, "rdf_pairs_per_update": pairs,
           "rdf_pairs_per_s": pairs * nblocks / t_rdf if t_rdf > 0 else None,
           "sq_ms_per_update": t_sq * 1e3 / nblocks, "sq_terms_per_s": n * nq * nblocks / t_sq if t_sq > 0 else None,
           "rdf_ms_min_max": [min(each_rdf), max(each_rdf)], "sq_ms_min_max": [min(each_sq), max(each_sq)],
           "rdf_wall_ms_per_update": w_rdf * 1e3 / nblocks, "sq_wall_ms_per_update": w_sq * 1e3 / nblocks,
           "wall_s": wall, "timing": "device (CUDA events) for MD, RDF and S(q); wall times beside them",
           "clocks": clock_info}
    del sim, dev, rdf, sq
    return out


def run_lj_large(args):
    """The large-N LJ workload with on-the-fly structure (measure_lj_large);
    MATS counts the analysis device time too.  --lj-cells sets a smaller
    lattice for profiling."""
    rank, world, local, pg = dist_setup(args)
    barrier(pg)
    r = measure_lj_large(local, args.lj_cells, args.steps, args.warmup, seed=rank, tp=args.tp)
    t_all = allreduce_max(pg, r["t_md"] + r["t_rdf"] + r["t_sq"], local)
    n, steps = r["n"], r["steps"]
    cfg = {k: v for k, v in r.items() if k not in ("t_md", "t_rdf", "t_sq", "mats", "steps", "clocks")}
    cfg["l2"] = "working set of several GB > 126 MB L2, no flush"
    line = {
        "metric": f"MATS (million atom-timesteps/s), LJ N={n} NVE cells with RDF and S(q) every 100 steps, 1 B200",
        "value": n * steps * world / t_all / 1e6, "unit": "Matom-steps/s", "n_gpus": world, "steps": steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_all * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 sums)", "data": "synthetic (seeded FCC lattice)",
        "config": cfg, "clocks": r["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()


def measure_adjoint(local, steps, warmup, seed=77, growth=True):
    """Adjoint workload: KA N=4096, rho 1.2, T 0.6, an NVE trajectory of
    `steps` steps with checkpoints every 50; loss = squared deviations of
    <U>/N and P plus the L2 distance of the soft A-A g(r) from targets made at
    eps_AB = 1.45, sigma_AB = 0.82; gradients with respect to the 6 pair
    parameters (wall times of whole gradients through AdjointNVE)."""
    import torch

    from gamdpy_b200 import adjoint, workloads
    n = 4096
    conf = workloads.ka_configuration(n, rho=1.2, temperature=0.6, seed=seed)
    rdf = {"bins": 40, "r_lo": 0.7, "r_hi": 2.7, "width": 0.05, "every": 10}
    cut = workloads.KA_CUT.astype(np.float64)
    eng = adjoint.AdjointNVE(conf, cut, dt=0.005, steps=steps, checkpoint_every=50, rdf=rdf, device=local)

    def theta(eps_ab, sig_ab):
        sig = workloads.KA_SIGMA.astype(np.float64).copy()
        eps = workloads.KA_EPSILON.astype(np.float64).copy()
        sig[0, 1] = sig[1, 0] = sig_ab
        eps[0, 1] = eps[1, 0] = eps_ab
        return adjoint.theta_from_tables(sig, eps)

    target = torch.tensor(eng.forward(theta(1.45, 0.82)))
    vol = float(np.prod(conf.simbox.lengths))
    dr = (rdf["r_hi"] - rdf["r_lo"]) / rdf["bins"]

    def gradient():
        th = torch.tensor(theta(1.5, 0.8), requires_grad=True)
        loss = adjoint.matching_loss(eng.observables(th), target, n, vol, dr)
        loss.backward()
        return float(loss), th.grad.detach().numpy().copy()

    for _ in range(max(1, min(warmup, 3))):
        gradient()
    reps = max(1, min(steps // 1000, 3)) if steps >= 1000 else 3
    tf = 0.0
    for _ in range(reps):
        t1 = time.perf_counter()
        eng.forward(theta(1.5, 0.8))
        tf += time.perf_counter() - t1
    t_fwd = tf / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        loss, g = gradient()
    t_grad = (time.perf_counter() - t0) / reps
    # truncated adjoint (window of 100 steps) on the same trajectory
    eng.set_window(100)
    loss_w, g_w = gradient()
    eng.set_window(0)
    out = {"workload": f"KA-LJ NVE N={n} rho=1.2 T=0.6, {steps} steps, checkpoints every 50, "
                       "loss = (<U>/N, P, soft g_AA(r)) vs targets at eps_AB=1.45 sigma_AB=0.82",
           "n": n, "steps": steps, "rdf": rdf, "gradients_per_s": 1.0 / t_grad, "forward_ms": t_fwd * 1e3,
           "gradient_ms": t_grad * 1e3, "backward_over_forward": (t_grad - t_fwd) / t_fwd, "loss": loss,
           "gradient": [float(x) for x in g], "gradient_window100": [float(x) for x in g_w],
           "gradient_order": "eps_AA, eps_AB, eps_BB, sigma_AA, sigma_AB, sigma_BB"}
    if growth:
        # the growth of the exact gradient with the horizon (chaos: ~exp(lambda t))
        gr = {}
        for t in (50, 100, 200, 400, 800):
            e2 = adjoint.AdjointNVE(conf, cut, dt=0.005, steps=t, checkpoint_every=50, rdf=rdf, device=local)
            tgt = torch.tensor(e2.forward(theta(1.45, 0.82)))
            th = torch.tensor(theta(1.5, 0.8), requires_grad=True)
            adjoint.matching_loss(e2.observables(th), tgt, n, vol, dr).backward()
            gr[str(t)] = float(np.linalg.norm(th.grad.detach().numpy()))
        out["exact_gradient_norm_vs_steps"] = gr
        # the plain path on the same system and trajectory length (forward only)
        import gamdpy_b200 as gp
        c2 = workloads.ka_configuration(n, rho=1.2, temperature=0.6, seed=seed)
        sim = gp.Simulation(c2, workloads.ka_pair_potential(), gp.integrators.NVE(dt=0.005), [], num_timeblocks=1,
                            steps_per_timeblock=steps, storage="memory", steps_in_kernel_test=0, device=local,
                            compute_plan={"pb": 64, "tp": 1, "lanes": 0, "skin": 0.3, "UtilizeNIII": False,
                                          "gridsync": False, "nblist": "linked lists"})
        sim._sim.run(0.0, steps)
        out["plain_forward_ms"] = sim._sim.run(0.0, steps)
    del eng
    return out


def run_adjoint(args):
    """The adjoint workload (measure_adjoint): one gradient per timed
    iteration, with the horizon study and the plain path beside it."""
    rank, world, local, pg = dist_setup(args)
    steps = args.steps
    r = measure_adjoint(local, steps, args.warmup, seed=77 + rank, growth=True)
    n, rdf = r["n"], r["rdf"]
    t_grad = r["gradient_ms"] / 1e3
    line = {
        "metric": "adjoint gradients/s, KA N=4096 NVE trajectory, 6 pair parameters, 1 B200",
        "value": 1.0 / t_grad, "unit": "gradients/s", "n_gpus": world, "steps": steps, "warmup": 1,
        "ms_per_step": t_grad * 1e3 / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 forward, f64 adjoint", "data": "synthetic (seeded KA lattice)",
        "config": {"workload": r["workload"], "rdf": rdf},
        **{k: r[k] for k in ("forward_ms", "gradient_ms", "backward_over_forward", "plain_forward_ms", "loss",
                             "gradient", "gradient_window100", "exact_gradient_norm_vs_steps", "gradient_order")},
        "e2e": {"value": 1.0 / t_grad, "unit": "gradients/s", "h2d_bytes_per_step": n * 24 / steps,
                "d2h_bytes_per_step": 8 * (3 + rdf["bins"]) / steps,
                "note": "host initial state in, observables and gradient out, through AdjointNVE"},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(pg)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.impl == "numba":
        run_numba_comparator(args)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.workload == "lj2048":
        run_lj_small(args)
        return
    if args.workload == "lj8m":
        run_lj_large(args)
        return
    if args.sweep:
        run_sweep(args)
        return
    rank, world, local, pg = dist_setup(args)
    import gamdpy_b200 as gp
    from gamdpy_b200 import _lib, workloads

    n = args.n
    conf = workloads.ka_configuration(n, seed=1234 + rank)
    pp = workloads.ka_pair_potential(max_num_nbs=300)
    if args.langevin:
        integ = gp.integrators.NVT_Langevin(temperature=0.45, alpha=0.2, dt=0.005, seed=1 + rank)
    else:
        integ = gp.integrators.NVT(temperature=0.45, tau=0.2, dt=0.005)
    block = min(args.block, max(1, args.steps))
    plan = {"pb": 64, "tp": 1, "lanes": args.tp, "skin": 0.3, "UtilizeNIII": False, "gridsync": False,
            "nblist": "linked lists"}
    nblocks = max(1, args.steps // block)
    steps = nblocks * block
    e2e_blocks = max(1, min(nblocks, 4))
    sim = gp.Simulation(conf, pp, integ, [gp.MomentumReset(MOMENTUM_RESET_EVERY)],
                        num_timeblocks=max(nblocks, e2e_blocks), steps_per_timeblock=block, compute_plan=plan,
                        storage="memory", device=local)
    dev = sim._sim
    # the workload's untimed equilibration, then the warm-up (device resident)
    dev.run(0.0, EQUILIBRATION_STEPS)
    dev.run(0.0, max(3, args.warmup))
    dev.clear_status()

    # ---- timed: K steps, device-resident inputs ---------------------------
    if args.profile:
        if args.trace:
            dev.set_trace(1 << 20)
        ms = sum(dev.run(float(b * block * 0.005), block) for b in range(nblocks))
        mean_nbs, max_nbs = dev.nblist_stats()
        out = {"profile": True, "n": n, "steps": steps, "ms_per_step": ms / steps, "mats": n * steps / ms / 1e3,
               "mean_neighbours": mean_nbs, "tp": args.tp}
        if args.trace:
            out["trace"] = trace_summary(*dev.trace(1 << 20))
            dev.set_trace(0)
        out["step_kernel_ms"] = dev.time_step_kernel(20)
        print(json.dumps(out), flush=True)
        return
    clocks = ClockSampler(local)
    barrier(pg)
    clocks.start()
    ms_total = 0.0
    for b in range(nblocks):
        ms_total += dev.run(float(b * block * 0.005), block)
    clock_info = clocks.stop()
    barrier(pg)
    t_max = allreduce_max(pg, ms_total / 1e3, local)
    mats = n * steps * world / t_max / 1e6
    tps = steps / t_max
    mean_nbs, max_nbs = dev.nblist_stats()

    # ---- end to end through the public API (host buffers) ------------------
    # gamdpy's pattern (Simulation.run_timeblocks): upload once, then every
    # timeblock run on the device and copy r, v, f, images and the per-particle
    # scalars back into the Configuration's arrays
    barrier(pg)
    t0 = time.perf_counter()
    for _ in sim.run_timeblocks(e2e_blocks):
        pass
    e2e_s = allreduce_max(pg, time.perf_counter() - t0, local)
    e2e_steps = e2e_blocks * block
    h2d = n * (12 + 12 + 4 + 4 + 12)  # r, v, m, type, images
    d2h = n * (12 + 12 + 12 + 12 + 4 * 5)  # r, v, f, images, 5 scalar planes
    e2e = {"value": n * e2e_steps * world / e2e_s / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
           "timeblock_steps": block, "note": "Simulation.run_timeblocks: upload once + per-timeblock "
                                             "device->host copy of the state into the Configuration"}

    # ---- roofline of the dominant kernel: k_run, one launch per timeblock --
    # (block steps + the final evaluation, rebuilds included).  Algorithmic
    # bytes per atom-step B = 4 n + 64 (one index per stored neighbour, float4
    # r and v read and written); per launch B * N * block.  The launch time is
    # the timeblock's CUDA-event time on the library's stream (the events
    # bracket k_block_begin + k_run, nothing else runs on that stream).
    bytes_per_atom = 4.0 * mean_nbs + 64.0
    ms_launch = t_max * 1e3 / nblocks
    achieved = bytes_per_atom * n * block / (ms_launch * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = ncu_traffic_per_atom_step()
    # the fused step alone (standalone k_step, no rebuild), for comparison
    ms_step_only = dev.time_step_kernel(50)

    # launches inside the timed region: per timeblock k_block_begin and the
    # persistent k_run
    launches_per_block = 2
    line = {
        "metric": METRIC, "value": mats, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_max * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded KA lattice)",
        "config": ka_config(n, args.langevin),
        "measured": {"tps": tps, "timeblock_steps": block, "parallelism": f"replicas x{world}",
                     "mean_neighbours": mean_nbs, "max_neighbours": max_nbs,
                     "path": PATH_NAMES.get(dev.last_path(), dev.last_path())},
        "e2e": e2e,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": (traffic * n * block if traffic else None),
                     "algorithmic_bytes_per_atom_step": bytes_per_atom,
                     "kernel": "k_run (persistent: steps, rebuilds, thermostat of one timeblock)",
                     "ms_per_launch": ms_launch, "atom_steps_per_launch": n * block,
                     "k_step_alone_ms": ms_step_only,
                     "k_step_alone_gbs": bytes_per_atom * n / (ms_step_only * 1e-3) / 1e9},
        "clocks": clock_info,
        "gpu_launches": launches_per_block * nblocks,
    }
    del sim, dev
    if not args.no_extras:
        # the reference's small plain case and the KA system at N = 2048 (TPS,
        # 10^4 steps each), and batched replicas against sequential runs; each
        # with its own clock record, measured after the main timed region
        line["small_n"] = {
            "lj2048": measure_lj2048(local, 10_000, 1000, 200, seed=rank),
            "ka2048": measure_ka(local, 2048, 10_000, 1000, 200, seed=1234 + rank),
        }
        # the batch shape is the project's autotuner's choice (untimed)
        line["batch"] = measure_batch(local, 128, 1000, 500, 10, autotune=True, seed=2024 + rank)
        # the large-N structure workload (200 steps: two RDF and S(q) updates)
        # and one adjoint gradient of the 2000-step KA trajectory
        for key, fn in (("lj8m", lambda: measure_lj_large(local, 128, 200, 10, seed=rank)),
                        ("adjoint", lambda: measure_adjoint(local, 2000, 1, seed=77 + rank, growth=False))):
            try:
                line[key] = fn()
            except Exception as e:  # a sub-measurement never costs the main line
                line[key] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0 and world == 1:
        cps = max(1, min(50, args.steps))  # about 10 s of host work at N = 1M
        cmats, threads, secs, rebuilds = cpu_reference(args, n, cps)
        line["cpu_baseline"] = {"value": cmats, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{cps} steps of the same N={n} system ({secs:.1f} s, "
                                          f"{rebuilds} list rebuilds)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
