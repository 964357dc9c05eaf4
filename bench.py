"""Benchmark of the DEM step: particle-updates/s on one or more B200s.

A "step" is one MoveParticles (src/MDEM.f90:285-369) of a whole system: two
force passes (cell rebuild, contact search + history, forces/torques) plus
the AB predictor and AM corrector.  particle-updates/s = particles x steps / s.

Default workload: 1,000,000 polydisperse spheres (radii U[0.4,0.6]) in a
fully periodic cube at volume fraction 0.55, kn = 1e5, e = 0.8, mu = 0.5,
dt = 1e-4, no gravity.  With --gpus N every rank advances its own
independent system (ensemble members, seed + rank): weak scaling, no
collective on the data path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # CPU implementation (oracle port)
    python bench.py --workload ensemble4096 # 4,096 settling systems, one context

The ensemble workload advances 4,096 independent gravity-settling systems
(log-uniform sizes in [200, 20000], ~17.4M spheres, per-system friction and
restitution) in one context, mixed precision, and compares it with the plain
FP64 step launched system by system (timed on a sample of systems,
extrapolated by particle count).

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-updates/s @1M spheres: FP32-mixed vs FP64 plain, force err <=1e-5 rel"
UNIT = "particle-updates/s"
WORKLOADS = {
    "dense1m": dict(n=1_000_000, phi=0.55, seed=1001, tile=8000),
    "dense16m": dict(n=16_000_000, phi=0.60, seed=1002, tile=16000),
    "dense64k": dict(n=64_000, phi=0.55, seed=1001, tile=8000),
    "ensemble4096": dict(kind="ensemble", n_systems=4096, seed=1003, skip=3000),
    "bidisperse4m": dict(kind="bidisperse", n=4_000_000, seed=1004),
    "ensemble64": dict(kind="ensemble", n_systems=64, seed=1003),
    # small systems (200-2,000 spheres), where a step is a few microseconds of
    # work per kernel: the case for one persistent launch per 4-step chunk
    "ensemble16small": dict(kind="ensemble", n_systems=16, seed=1003, nmin=200, nmax=2000),
    # above jamming (about six contacts per sphere): the contact-dense case
    "jammed1m": dict(n=1_000_000, phi=0.65, seed=1012, tile=8000, relax=4000),
    "jammed16m": dict(n=16_000_000, phi=0.65, seed=1012, tile=16000, relax=4000),
    "jammed216k": dict(n=216_000, phi=0.65, seed=1012, tile=8000, relax=4000),
}


# --------------------------------------------------------------------------
# helpers

def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def test_bytes_per_particle(z_pp, m_cand):
    """Algorithmic DRAM bytes of one test-kernel launch per particle: position
    + R 32, row length 4, candidate row 4*m_cand (the "i" partners only) read;
    the particle's place in the contact list 8 and one list entry (8 B) per
    contact it evaluates (0.5*z_pp) written.  Partner positions are other
    particles' own data (L1/L2) and add nothing."""
    return 32 + 4 + 4 * m_cand + 8 + 0.5 * z_pp * 8


def pair_bytes_per_particle(mixed, update, z_pp):
    """Algorithmic DRAM bytes of one pair-kernel launch per particle (0.5*z_pp
    contacts): per contact its list entry 8 and i's place 4 read, the pair's
    history record (key 4 + 36 B FP32 / 48 B FP64) read, the "i" half
    (48 / 80 B) and the "j" half (48 / 80 B + its count 4) written, and in
    the history-updating pass the new record written.  The two particles'
    positions and velocities are their own data (L1/L2)."""
    rec = 4 + (36 if mixed else 48)
    half = 48 if mixed else 80
    per = 8 + 4 + rec + half + half + 4 + (rec if update else 0)
    return 0.5 * z_pp * per


def fold_bytes_per_particle(mixed, epi, z_pp, z_pw=0.0, nw=0, nprev=3):
    """Algorithmic DRAM bytes of one fold-kernel launch per particle:
      reads: cell 4, rank 4, "j" count 4 (reset), matched bits 4, place in
        the contact list 8, position + R 32 (and the FP64 velocity copies 48
        in FP64 mode, the FP32 ones 24 with walls), the "i" halves and the
        "j" halves of its contacts (0.5*z_pp each, 48 / 80 B), wall flags and
        records;
      epi "predict" (pass 1, src/MDEM.f90:296-331, history-updating): the
        record count 4 read and written, new wall records; ring nprev*72
        read, Particle v,w 48 read (mixed), ring slot 72 + the corrector's
        ring sums 72 + next-pass copies (32 + velocities) + cell 4 written,
        and of Particle a,alpha and Predicted x,v,w only what no other array
        holds: a,alpha 48 only without a ring (nprev = 0), Predicted v,w 48
        only in mixed mode (its velocity copies are FP32);
      epi "correct" (pass 2, :340-367): the ring sums 72, Predicted v 24
        (mixed) read, Particle x,v,w 72 read and written, Predicted a,alpha
        48 + next-pass copies + cell 4 written."""
    vel = 24 if mixed else 48
    half = 48 if mixed else 80
    wrec = 4 + (36 if mixed else 48)
    base = (4 + 4 + 4 + 4 + 8 + 32 + (0 if mixed else 48) + (24 if mixed and nw else 0)
            + z_pp * half + nw * 4 + z_pw * (wrec - 4))
    sums = 72 if nprev else 0
    if epi == "predict":
        base += 8 + nw * 4 + z_pw * (wrec - 4)
        epil = (nprev * 72 + (48 if mixed else 0) + (0 if nprev else 48) + (48 if mixed else 0)
                + (72 if nprev else 0) + sums + 32 + vel + 4)
    else:
        epil = sums + (24 if mixed else 0) + 72 + 72 + 48 + 32 + vel + 4
    return base + epil


def step_bytes_per_particle(mixed, z_pp, m_cand, z_pw=0.0, nw=0, nprev=3):
    """Bytes of one particle-update (MoveParticles: two passes of a test, a
    pair and a fold kernel) under the kernels' own model; the relink and
    candidate-row kernels touch only the few particles near cells that
    changed and are not counted."""
    return (2 * test_bytes_per_particle(z_pp, m_cand) +
            pair_bytes_per_particle(mixed, True, z_pp) +
            pair_bytes_per_particle(mixed, False, z_pp) +
            fold_bytes_per_particle(mixed, "predict", z_pp, z_pw, nw, nprev) +
            fold_bytes_per_particle(mixed, "correct", z_pp, z_pw, nw, nprev))


def survey_bytes_per_particle(mixed, z_pp, z_pw=0.0):
    """Compulsory bytes of one particle-update of a fused gather design
    (the hot-path scope table's model): FP64 656 + 84*Z_pp + 168*Z_pw,
    mixed 608 + 48*Z_pp + 96*Z_pw, with Z_pp the pair contacts and Z_pw the
    wall contacts per particle."""
    if mixed:
        return 608.0 + 48.0 * z_pp + 96.0 * z_pw
    return 656.0 + 84.0 * z_pp + 168.0 * z_pw


def reduce_max(x, world, device="cuda"):
    """Max over ranks (the timed region is the slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(n_per_rank, world, steps, max_ms):
    """Whole-job particle-updates/s: every rank advances its own system."""
    return n_per_rank * world * steps / (max_ms / 1000.0)


def rank_seed(base, rank):
    return base + rank


# --------------------------------------------------------------------------
# workload

def make_workload(name, precision, rank, factory=None):
    from dem3d_b200 import configs
    from dem3d_b200 import params as P
    spec = WORKLOADS[name]
    prec = P.PREC_MIXED if precision == "mixed" else P.PREC_FP64
    if spec.get("kind") == "bidisperse":
        return configs.bidisperse_settling(n=spec["n"], seed=rank_seed(spec["seed"], rank),
                                           precision=prec)
    return configs.dense_packing(n=spec["n"], phi=spec["phi"], seed=rank_seed(spec["seed"], rank),
                                 tile=spec["tile"], precision=prec, system_factory=factory,
                                 relax_steps=spec.get("relax", 2000))


def config_block(name, w, world, precision):
    spec = WORKLOADS[name]
    if spec.get("kind") == "bidisperse":
        return {
            "workload": (f"{w.n:,} bidisperse spheres (d 1 and 3, {w.info['n_large']:,} large), "
                         "settling under gravity in a 200x200 box with floor and four side walls, "
                         "mu=0.5, e=0.7, dt=5e-5, ABM4"),
            "particles_per_gpu": w.n, "global_particles": w.n * world, "precision": precision,
            "l2": "inputs larger than L2", "parallelism": f"{world} independent systems"}
    return {
        "workload": (f"{spec['n']:,} polydisperse spheres R~U[0.4,0.6], periodic cube "
                     f"phi={spec['phi']}, kn=1e5, e=0.8, mu=0.5, dt=1e-4, ABM4"),
        "particles_per_gpu": spec["n"], "global_particles": spec["n"] * world,
        "box": round(w.info["L"], 4), "precision": precision,
        "input": (f"{spec['tile']}-sphere tile relaxed {spec.get('relax', 2000)} steps "
                  f"(e=0.1, no friction) x {w.info['copies']} copies, seeded"),
        "l2": "inputs larger than L2 (state + history >> 126 MB)",
        "parallelism": f"{world} independent systems (ensemble, seed+rank)",
    }


# --------------------------------------------------------------------------
# CPU timing (oracle port: the reference is Fortran and cannot be built here)

def _oracle_variant():
    """-O3 -march=native build of the oracle on this host, else the portable one."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_build",
                                                  os.path.join(ROOT, "oracle", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    try:
        libs = mod.build(native_dir=tempfile.mkdtemp())
        return libs["libdem_oracle_native.so"], "-O3 -march=native -ffp-contract=off"
    except Exception:
        libs = mod.build()
        return libs["libdem_oracle_fast.so"], "-O3 -ffp-contract=off"


def cpu_model():
    """The host CPU's model name (first "model name" line of /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def cpu_time_steps(w, max_steps=3, budget_s=25.0, lib_path=None, warmup=1, core=None):
    """Time oracle MoveParticles steps on w (single thread), after `warmup`
    untimed steps (the first steps also allocate the contact lists).  With
    `core`, the calling thread is pinned to that core (the k-th core it may
    run on) while it times, and its affinity is restored afterwards."""
    import ctypes as C

    from dem3d_b200 import _abi
    from dem3d_b200.system import DEMSystem
    lib = C.CDLL(lib_path)
    _abi.bind(lib, "orc_", _abi.SIGNATURES)
    s = DEMSystem(w.params, lib=lib, prefix="orc_")
    old = None
    if core is not None and hasattr(os, "sched_setaffinity"):
        old = os.sched_getaffinity(0)
        allowed = sorted(old)
        os.sched_setaffinity(0, {allowed[core % len(allowed)]})
    try:
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
        for k in range(warmup):
            s.move_particles(4 + k)
        steps = 0
        t0 = time.perf_counter()
        while steps < max_steps:
            s.move_particles(4 + warmup + steps)
            steps += 1
            if time.perf_counter() - t0 > budget_s:
                break
        dt = time.perf_counter() - t0
    finally:
        s.close()
        if old is not None:
            os.sched_setaffinity(0, old)
    return w.n * steps / dt, steps, dt


def _ref_worker(args):
    name, rank, tile_pos, tile_rad, L_t, lib_path, steps_cap, warmup, budget = args
    from dem3d_b200 import configs
    spec = WORKLOADS[name]
    k = configs.tile_count(spec["n"], spec["tile"])
    pos, radius, L = configs.replicate(tile_pos, tile_rad, L_t, k)
    rng = np.random.default_rng(spec["seed"] + rank + 7919)
    n = spec["n"]
    vel = rng.normal(0.0, 0.1, size=(n, 3))
    prm = configs.dense_packing_params(0.6, L)
    w = configs.Workload("dense_packing", prm, pos, vel, np.zeros((n, 3)), radius=radius,
                         info={"L": L, "copies": k ** 3})
    return cpu_time_steps(w, steps_cap, budget, lib_path, warmup, core=rank)


def run_reference(args):
    """--impl reference: the CPU implementation of the path on all host cores
    (one independent system per process; the reference program is serial)."""
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    if rank != 0:
        return 0
    import multiprocessing as mp

    import psutil
    from dem3d_b200 import configs
    lib_path, flags = _oracle_variant()
    spec = WORKLOADS[args.workload]
    # the same relaxed tile as the GPU arm, relaxed here by the oracle
    import ctypes as C

    from dem3d_b200 import _abi
    from dem3d_b200.system import DEMSystem

    def factory(p):
        lib = C.CDLL(lib_path)
        _abi.bind(lib, "orc_", _abi.SIGNATURES)
        return DEMSystem(p, lib=lib, prefix="orc_")
    t0 = time.perf_counter()
    tp, tr, L_t = configs.relaxed_tile(spec["tile"], spec["phi"], spec["seed"],
                                       relax_steps=spec.get("relax", 2000),
                                       system_factory=factory)
    t_relax = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    mem = psutil.virtual_memory().available
    per_proc = 1.6e9 * spec["n"] / 1e6
    procs = max(1, min(cores, int(mem * 0.6 // per_proc), 32))
    steps_cap = max(1, min(args.steps, 3))
    warmup = max(0, min(args.warmup, 3))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(args.workload, r, tp, tr, L_t, lib_path, steps_cap, warmup,
                                      60.0)
                                     for r in range(procs)])
    wall = time.perf_counter() - t0
    value = sum(r[0] for r in res)
    w_dummy = type("W", (), {"info": {"L": configs.replicate(tp, tr, L_t, 1)[2] *
                                       configs.tile_count(spec["n"], spec["tile"]),
                                       "copies": configs.tile_count(spec["n"],
                                                                    spec["tile"]) ** 3}})
    sample = (f"{procs} processes x {res[0][1]} MoveParticles steps (after {warmup} untimed) "
              f"of an independent "
              f"{spec['n']:,}-sphere system each, one process pinned per core of "
              f"{cpu_model()} (oracle C port {flags}; reference Fortran "
              f"not buildable here: no Fortran compiler); tile relaxed by the oracle in "
              f"{t_relax:.1f}s")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": res[0][1], "warmup": warmup, "ms_per_step": 1000.0 * max(r[2] / r[1] for r in res),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_block(args.workload, w_dummy, 1, "fp64"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 2),
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# GPU arm

def traffic_per_particle():
    """DRAM bytes per particle of the pass kernels from a committed ncu
    capture summary (profiles/pass_traffic.json), if present."""
    p = os.path.join(ROOT, "profiles", "pass_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


def kernel_bytes(name, n, mixed, z_pp, m_cand, z_pw, nw):
    """Algorithmic bytes of one launch of a force-pass kernel (mean of the
    two passes of a step)."""
    if name.startswith("test"):
        return n * test_bytes_per_particle(z_pp, m_cand)
    if name.startswith("pair"):
        return n * 0.5 * (pair_bytes_per_particle(mixed, True, z_pp) +
                          pair_bytes_per_particle(mixed, False, z_pp))
    if name.startswith("fold"):
        return n * 0.5 * (fold_bytes_per_particle(mixed, "predict", z_pp, z_pw, nw) +
                          fold_bytes_per_particle(mixed, "correct", z_pp, z_pw, nw))
    return None


def measure(s, w, args, world, local, torch, dist, first_step=1):
    """Warm-up (and the autotuner's trials, on the live run), then the timed
    region (graph replay of K steps)."""
    s.run(first_step, first_step + 2 + args.warmup)
    first = first_step + 3 + args.warmup
    tuning = None
    if not args.no_autotune:
        tuning = s.autotune(first, 40)
        first = tuning["last_step"] + 1
    last = first + args.steps - 1
    if world > 1:
        dist.barrier()
    l0 = s.launch_count()
    steps_done = args.steps
    retunes = []
    with ClockSampler(local) as clk:
        # NVTX range "dem_timed": lets a profiler select exactly these launches
        torch.cuda.nvtx.range_push("dem_timed")
        if args.retune_every > 0 and tuning is not None:
            # long runs whose dynamics change: the autotuner's trials (real
            # steps of the same run) again every `retune_every` steps
            s.timer_start()
            step, steps_done = first, 0
            while steps_done < args.steps:
                seg = min(args.retune_every, args.steps - steps_done)
                s.run(step, step + seg - 1)
                step += seg
                steps_done += seg
                if steps_done < args.steps:
                    t = s.autotune(step, 40)
                    retunes.append((step, t["skin_factor"], t["pass_variant"]))
                    steps_done += t["last_step"] - step + 1
                    step = t["last_step"] + 1
            ms = s.timer_stop()
            last = step - 1
        else:
            ms = s.run_timed(first, last)
        torch.cuda.nvtx.range_pop()
    launches = s.launch_count() - l0
    ms = reduce_max(ms, world)
    if retunes:
        tuning = dict(tuning, retunes=retunes, steps_timed=steps_done)
    return {"ms": ms, "launches": launches, "last": last, "clocks": clk.summary(),
            "value": aggregate_rate(w.n, world, steps_done, ms), "tuning": tuning,
            "steps": steps_done}


def window_observables(s, first, window, every):
    """Observables averaged over `window` further steps of a run, sampled
    after every `every` steps (the instantaneous wall force of a settling
    bed fluctuates; its time average is what compares between runs).
    Returns (averages, last step, samples)."""
    every = max(1, min(every, window))
    samples = []
    step = first
    while step - first < window:
        last = min(step + every - 1, first + window - 1)
        s.run(step, last)
        step = last + 1
        samples.append(s.observables())
    avg = {}
    for k, v in samples[0].items():
        if isinstance(v, (int, float)):
            avg[k] = float(np.mean([x[k] for x in samples]))
        elif isinstance(v, (list, tuple, np.ndarray)):
            avg[k] = [float(y) for y in np.mean([np.asarray(x[k], dtype=float)
                                                 for x in samples], axis=0)]
    return avg, step - 1, len(samples)


def snapshot(src):
    """State, contact history and integration ring of a context, on the host."""
    return {"state": src.get_state(), "contacts": src.get_contacts(),
            "integration": src.get_integration()}


def force_error(w_fp64, w_mixed, snap):
    """Per-step force error of the mixed path: one force pass from the same
    state and contact history (``snapshot`` of a context) in both precisions;
    the error is normed by the largest |a| (net forces cancel in packings)."""
    from dem3d_b200.system import DEMSystem
    st = snap["state"]
    c = snap["contacts"]
    prev, ipc = snap["integration"]
    acc = {}
    for name, w in (("fp64", w_fp64), ("mixed", w_mixed)):
        t = DEMSystem(w.params)
        t.set_state(st["pos"], st["vel"], st["omega"], comp=w.comp, radius=w.radius,
                    acc=st["acc"], alpha=st["alpha"])
        t.set_integration(prev, ipc)
        t.set_contacts(c["imin"], c["imax"], c["ft"], c["vt"], c["ip"], c["iw"], c["ftw"],
                       c["vtw"])
        t.initialize_cell_distribution()
        t.compute_accelerations(update=True)
        acc[name] = t.get_state()
        t.close()
    out = {}
    for k in ("acc", "alpha"):
        ref = acc["fp64"][k]
        out[k] = float(np.abs(acc["mixed"][k] - ref).max() / max(np.abs(ref).max(), 1e-300))
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    from dem3d_b200 import _abi
    from dem3d_b200.system import DEMSystem

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    lib = _abi.load_library()
    st = lib.dem_select_device(local)
    if st != 0:
        raise RuntimeError(f"dem_select_device({local}) failed: {st}")

    def barrier_max(x):
        return reduce_max(x, world)

    # the metric compares the mixed path with the plain FP64 path: by default
    # both are timed on the same workload, the headline value is the mixed one
    precisions = [args.precision] if args.precision != "auto" else ["fp64", "mixed"]
    headline = precisions[-1]

    t0 = time.perf_counter()
    base = make_workload(args.workload, "fp64", rank)
    t_gen = time.perf_counter() - t0
    n = base.n
    works = {}
    from dem3d_b200 import params as P
    import copy
    for prec in precisions:
        w = copy.copy(base)
        w.params = copy.deepcopy(base.params)
        w.params.precision = P.PREC_MIXED if prec == "mixed" else P.PREC_FP64
        works[prec] = w
    res = {}
    systems = {}
    for prec in precisions:
        w = works[prec]
        s = DEMSystem(w.params)
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
        if args.reorder_every > 0:
            s.set_reorder(args.reorder_every)
        if args.no_early_launch:
            s.set_early_launch(False)
        res[prec] = measure(s, w, args, world, local, torch, dist)
        systems[prec] = s
    s = systems[headline]
    w = works[headline]
    ms = res[headline]["ms"]
    value = res[headline]["value"]
    launches = res[headline]["launches"]
    last = res[headline]["last"]
    clocks = res[headline]["clocks"]

    ferr = None
    obs_cmp = None
    if "fp64" in systems and "mixed" in systems:
        # both runs advanced the same steps from the same state: ensemble
        # observables of the mixed run against the FP64 run (with
        # --obs-window, time averages over that many further steps)
        window = None
        if args.obs_window > 0:
            avg = {p: window_observables(systems[p], res[p]["last"] + 1, args.obs_window,
                                         args.obs_every) for p in ("fp64", "mixed")}
            ob = {p: avg[p][0] for p in avg}
            window = {"from_step": res["fp64"]["last"] + 1, "to_step": avg["fp64"][1],
                      "samples": avg["fp64"][2]}
        else:
            ob = {p: systems[p].observables() for p in ("fp64", "mixed")}
        # the FP64 context closes before the two force-pass contexts open
        # (three contexts of the 16M-sphere workload do not fit one GPU)
        snap = snapshot(systems["fp64"])
        systems.pop("fp64").close()
        ferr = force_error(works["fp64"], works["mixed"], snap)
        del snap
        keys = ("kinetic_energy", "mean_coordination", "packing_fraction", "bed_height")
        pick = {p: {k: ob[p][k] for k in keys} for p in ob}
        for p in ob:
            pick[p]["floor_force"] = ob[p]["wall_normal_force"][0]
            pick[p]["floor_pressure"] = ob[p]["wall_pressure"][0]
        rel = {k: (abs(pick["mixed"][k] - pick["fp64"][k]) / abs(pick["fp64"][k])
                   if pick["fp64"][k] else None) for k in pick["fp64"]}
        obs_cmp = {"after_step": res["fp64"]["last"], **pick, "rel_diff": rel,
                   "time_average": window}
    cell_occ = None
    if WORKLOADS[args.workload].get("kind") == "bidisperse":
        # cell-cost imbalance: cells are sized by the large spheres, so a cell
        # of small ones holds many; spheres per occupied cell at the end
        _, _, cs = systems[headline].get_cells()
        cnt = np.diff(cs)
        occ = cnt[cnt > 0]
        cell_occ = {"cells": int(cnt.size), "occupied": int(occ.size),
                    "mean_per_occupied_cell": float(occ.mean()) if occ.size else 0.0,
                    "p99": float(np.percentile(occ, 99)) if occ.size else 0.0,
                    "max": int(occ.max()) if occ.size else 0}
    for prec, sy in systems.items():
        if prec != headline:
            sy.close()

    # contacts and candidates per particle for the byte model
    ps = s.pass_stats()
    obs = s.observables()
    z_pp = 2.0 * obs["n_pair_contacts"] / n
    z_pw = obs["n_wall_contacts"] / n
    nw = int(w.params.n_walls)
    rs = s.row_stats()
    m_cand = rs["candidates"] / n
    mixed = headline == "mixed"
    # per-kernel timing (instrumented steps, not graph-replayed)
    s.reset_kernel_stats()
    s.set_profiling(True)
    nprof = 6
    for k in range(nprof):
        s.move_particles(last + 1 + k)
    stats = s.kernel_stats()
    s.set_profiling(False)
    last += nprof
    total_prof = sum(v[1] for v in stats.values())
    dom = max(stats, key=lambda k: stats[k][1])
    b_launch = kernel_bytes(dom, n, mixed, z_pp, m_cand, z_pw, nw)
    avg_ms = stats[dom][1] / stats[dom][0]
    achieved = b_launch / (avg_ms / 1000.0) / 1e9 if b_launch else None
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak = peaks.get("hbm_gbs", 6650.0)
    tr = traffic_per_particle()
    traffic, traffic_src = None, None
    if tr and dom in tr.get("bytes_per_particle", {}):
        # ncu DRAM bytes per particle of one launch, captured on a smaller
        # case of the same workload, scaled to this launch by the particles
        traffic = tr["bytes_per_particle"][dom] * n
        traffic_src = tr.get("state", "profiles/pass_traffic.json")
    # every force-pass kernel against its own byte model
    per_kernel = {}
    for k, v in stats.items():
        kb = kernel_bytes(k, n, mixed, z_pp, m_cand, z_pw, nw)
        if kb and v[0]:
            kms = v[1] / v[0]
            per_kernel[k] = {"bytes_per_launch": kb, "avg_launch_ms": kms,
                             "achieved_gbs": kb / (kms / 1000.0) / 1e9,
                             "frac": kb / (kms / 1000.0) / 1e9 / peak}
    step_b = step_bytes_per_particle(mixed, z_pp, m_cand, z_pw, nw)
    step_ms = ms / res[headline]["steps"]
    step_gbs = step_b * n / (step_ms / 1000.0) / 1e9
    # the hot-path table's compulsory bytes per particle-update over the
    # whole step (every kernel of it) and over the force-pass kernels alone
    surv_b = survey_bytes_per_particle(mixed, z_pp, z_pw)
    pass_ms = sum(v[1] for k, v in stats.items()
                  if k.startswith(("test", "pair", "fold"))) / nprof
    surv_step = surv_b * n / (step_ms / 1000.0) / 1e9
    surv_pass = surv_b * n / (pass_ms / 1000.0) / 1e9 if pass_ms > 0 else None

    # e2e: a driver that keeps Particle(1:n) on the host: each step uploads
    # positions, velocities and angular velocities from pinned host memory,
    # advances one MoveParticles through the C-ABI and downloads them again
    # (accelerations are recomputed by the step's first pass and are not an
    # input of MoveParticles).
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        ke = max(3, min(args.steps, 20))
        fields = ("pos", "vel", "omega")
        host = {k: torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
                for k in fields}
        stt = s.get_state()
        for k in host:
            host[k][...] = stt[k]
        ptr = {k: host[k].ctypes.data_as(C.POINTER(C.c_double)) for k in fields}
        if world > 1:
            dist.barrier()
        s.timer_start()
        for k in range(ke):
            s._call("update_state", ptr["pos"], ptr["vel"], ptr["omega"], None, None)
            s.move_particles(last + 1 + k)
            s._call("get_state", ptr["pos"], ptr["vel"], ptr["omega"], None, None)
        e2e_ms = barrier_max(s.timer_stop())
        last += ke
        e2e = {"value": n * world * ke / (e2e_ms / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": 3 * 24 * n, "d2h_bytes_per_step": 3 * 24 * n,
               "steps": ke, "path": "dem_update_state + dem_move_particles + dem_get_state "
                                    "(positions, velocities, angular velocities)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        lib_path, flags = _oracle_variant()
        v, k, dt = cpu_time_steps(base, max_steps=30, budget_s=10.0, lib_path=lib_path, core=0)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{k} MoveParticles steps (after 1 untimed; the GPU arm times "
                         f"{res[headline]['steps']}) of the same {n:,}-sphere "
                         f"system, oracle "
                         f"C port ({flags}), 1 thread pinned to one core of {cpu_model()}, "
                         f"{dt:.1f}s"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": res[headline]["steps"], "warmup": args.warmup,
            "ms_per_step": ms / res[headline]["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if headline == "fp64" else "f32+f64", "data": "synthetic",
            "config": dict(config_block(args.workload, w, world, headline),
                           storage_reorder_every=args.reorder_every,
                           early_launch=not args.no_early_launch),
            "gpu_launches": int(launches),
            "launches_per_step": launches / res[headline]["steps"],
            "precisions": {p: {"value": r["value"], "ms_per_step": r["ms"] / r["steps"],
                               "launches_per_step": r["launches"] / r["steps"],
                               "tuning": r["tuning"]}
                           for p, r in res.items()},
            "mixed_over_fp64": (res["mixed"]["value"] / res["fp64"]["value"]
                                if "mixed" in res and "fp64" in res else None),
            "force_err_vs_fp64": ferr,
            "observables_mixed_vs_fp64": obs_cmp,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes_per_launch": b_launch,
                         "avg_launch_ms": avg_ms, "peak_source": "MEASURED_PEAKS.json hbm_gbs"
                         if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                         "traffic_source": traffic_src,
                         "step_bytes_per_particle_update": step_b,
                         "step_achieved_gbs": step_gbs, "step_frac": step_gbs / peak,
                         "kernels": per_kernel,
                         "survey_bytes_per_particle_update": surv_b,
                         "frac_survey": surv_step / peak,
                         "frac_survey_force_passes": surv_pass / peak if surv_pass else None,
                         "kernel_share": {k: round(v[1] / total_prof, 4)
                                          for k, v in sorted(stats.items(),
                                                             key=lambda kv: -kv[1][1])}},
            "contacts_per_particle": z_pp, "candidates_per_particle": m_cand,
            "movers_last_pass": ps["movers"],
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
            "gen_s": round(t_gen, 2),
        }
        if cell_occ is not None:
            line["cell_occupancy"] = cell_occ
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ensemble(args):
    """The batched workload: all systems in one context (one launch per
    stage), mixed precision, against the plain FP64 step run system by
    system in its own context (a sample of systems, extrapolated)."""
    import torch
    import torch.distributed as dist

    from dem3d_b200 import _abi
    from dem3d_b200 import configs
    from dem3d_b200 import params as P
    from dem3d_b200.system import DEMSystem

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    lib = _abi.load_library()
    if lib.dem_select_device(local) != 0:
        raise RuntimeError("dem_select_device failed")
    spec = WORKLOADS[args.workload]
    prec = "fp64" if args.precision == "fp64" else "mixed"
    t0 = time.perf_counter()
    # one ensemble for the whole job; rank r advances every world-th system
    # (no exchange between ranks: the systems are independent)
    e_all = configs.settling_ensemble(n_systems=spec["n_systems"], seed=spec["seed"],
                                      nmin=spec.get("nmin", 200), nmax=spec.get("nmax", 20000),
                                      precision=P.PREC_MIXED if prec == "mixed" else P.PREC_FP64)
    e = e_all.shard(rank, world)
    t_gen = time.perf_counter() - t0
    n = e.n
    s = DEMSystem.ensemble(e.params, e.counts)
    s.set_state(e.pos, e.vel, e.omega, radius=e.radius)
    s.initialize_cell_distribution()
    if args.no_early_launch:
        s.set_early_launch(False)
    skip = args.skip_steps if args.skip_steps >= 0 else spec.get("skip", 0)
    if skip > 0:
        # the beds start to form: untimed steps before the warm-up
        s.run(1, skip)
    w = type("W", (), {"n": n})
    res = measure(s, w, args, world, local, torch, dist, first_step=skip + 1)
    # whole-job rate: every particle of the ensemble over the slowest rank's time
    res["value"] = e_all.n * res["steps"] / (res["ms"] / 1000.0)
    obs = s.observables()
    z_pp = 2.0 * obs["n_pair_contacts"] / n
    z_pw = obs["n_wall_contacts"] / n
    # job-wide observables: sums over the ranks' systems
    tot = np.array([obs["kinetic_energy"], obs["n_pair_contacts"], obs["n_wall_contacts"], n],
                   dtype=np.float64)
    if world > 1:
        t = torch.tensor(tot, device="cuda")
        dist.all_reduce(t)
        tot = t.cpu().numpy()
    job_obs = {"kinetic_energy": float(tot[0]), "pair_contacts": int(tot[1]),
               "wall_contacts": int(tot[2]), "particles": int(tot[3])}
    m_cand = s.row_stats()["candidates"] / n
    # per-kernel timing of a few instrumented steps
    s.reset_kernel_stats()
    s.set_profiling(True)
    for k in range(4):
        s.move_particles(res["last"] + 1 + k)
    stats = s.kernel_stats()
    s.set_profiling(False)
    total_prof = sum(v[1] for v in stats.values())
    dom = max(stats, key=lambda k: stats[k][1])
    b_launch = kernel_bytes(dom, n, prec == "mixed", z_pp, m_cand, z_pw, 1)
    avg_ms = stats[dom][1] / stats[dom][0]
    achieved = b_launch / (avg_ms / 1000.0) / 1e9 if b_launch else None
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    s.close()

    # the reference's way: one system per context, plain FP64, one after the
    # other (a seeded sample of systems, extrapolated by particle count)
    seq = None
    if rank == 0:
        rng = np.random.default_rng(5)
        sample = rng.choice(len(e.counts), size=min(16, len(e.counts)), replace=False)
        ks = max(8, min(args.steps, 40))
        ms_tot, n_tot = 0.0, 0
        for k in sample:
            prm, pos, vel, om, rad = e.system(int(k))
            prm.precision = P.PREC_FP64
            q = DEMSystem(prm)
            q.set_state(pos, vel, om, radius=rad)
            q.initialize_cell_distribution()
            q.run(1, 3 + args.warmup)
            ms_tot += q.run_timed(4 + args.warmup, 3 + args.warmup + ks)
            n_tot += pos.shape[0]
            q.close()
        rate = n_tot * ks / (ms_tot / 1000.0)
        seq = {"value": rate, "unit": UNIT, "systems_sampled": int(len(sample)),
               "particles_sampled": int(n_tot), "steps": ks,
               "sample": "plain FP64 step, one context per system, systems run one after the "
                         "other (dem_run, graph replay); rate extrapolates to all systems"}
    if rank == 0:
        value = res["value"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": res["steps"],
            "warmup": args.warmup, "ms_per_step": res["ms"] / res["steps"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": (f"{len(e.counts)} gravity-settling systems, sizes log-uniform "
                                    f"in [{spec.get('nmin', 200)}, {spec.get('nmax', 20000)}] "
                                    f"({n:,} spheres), R~U[0.45,0.55], per-system "
                                    "mu~U[0.2,0.8], e~U[0.5,0.95], 10x10 x-y periodic box with "
                                    "floor, dt=1e-4, ABM4, one context"),
                       "particles_per_gpu": n, "global_particles": e_all.n,
                       "precision": prec, "timed_from_step": res["last"] - res["steps"] + 1,
                       "l2": "inputs larger than L2",
                       "parallelism": f"systems sharded over {world} ranks (every "
                                      f"{world}-th system per rank), no exchange"},
            "job_observables": job_obs,
            "gpu_launches": int(res["launches"]),
            "launches_per_step": res["launches"] / res["steps"],
            "tuning": res["tuning"],
            "sequential_fp64_systems": seq,
            "ensemble_over_sequential_fp64": value / seq["value"] if seq else None,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak if achieved else None,
                         "traffic": None, "algorithmic_bytes_per_launch": b_launch,
                         "avg_launch_ms": avg_ms,
                         "kernel_share": {k: round(v[1] / total_prof, 4) for k, v in
                                          sorted(stats.items(), key=lambda kv: -kv[1][1])}},
            "contacts_per_particle": z_pp, "wall_contacts_per_particle": z_pw,
            "candidates_per_particle": m_cand, "e2e": None, "cpu_baseline": None,
            "clocks": res["clocks"], "gen_s": round(t_gen, 2),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_slabs(args):
    """One system cut into --slabs z-slabs, all on this GPU (every slab its
    own context, the exchanges as device copies between them): the cost of
    the decomposition's exchanges against the undivided context, and the
    composed state checked against it bit for bit.  Not a multi-GPU number."""
    import torch

    from dem3d_b200 import _abi
    from dem3d_b200 import slab as S
    from dem3d_b200.system import DEMSystem
    lib = _abi.load_library()
    lib.dem_select_device(0)
    prec = "mixed" if args.precision == "mixed" else "fp64"
    w = make_workload(args.workload, prec, 0)
    w.params.hist_capacity = max(w.params.hist_capacity, 16)
    g = DEMSystem(w.params)
    g.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    g.initialize_cell_distribution()
    first = 4 + args.warmup
    g.run(1, first - 1)

    def copy_of(src):
        d = DEMSystem(w.params)
        st = src.get_state()
        d.set_state(st["pos"], st["vel"], st["omega"], comp=w.comp, radius=w.radius,
                    acc=st["acc"], alpha=st["alpha"])
        prev, ipc = src.get_integration()
        d.set_integration(prev, ipc)
        c = src.get_contacts()
        d.set_contacts(c["imin"], c["imax"], c["ft"], c["vt"], c["ip"], c["iw"], c["ftw"],
                       c["vtw"])
        d.set_ncol(src.ncol())
        d.initialize_cell_distribution()
        return d

    ref = copy_of(g)
    nz = g.grid()[2]
    slabs = []
    for z0, z1 in S.slab_ranges(nz, args.slabs):
        sl = copy_of(g)
        sl.slab_set_range(z0, z1)
        slabs.append(sl)
    periodic = bool(w.params.pbc[2])
    tr = S.LocalTransport(slabs, periodic=periodic, cap_bytes=256 << 20)
    last = first + args.steps - 1
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for step in range(first, last + 1):
        S.move_particles(tr, step)
    torch.cuda.synchronize()
    ms_slab = (time.perf_counter() - t0) * 1000.0
    ms_whole = ref.run_timed(first, last)
    want = ref.get_state()
    got = S.compose_state(slabs)
    exact = all(np.array_equal(got[k], want[k]) for k in want)
    line = {"metric": f"particle-updates/s, one system in {args.slabs} z-slabs on one GPU "
                      "(decomposition emulated: slab contexts, exchanges as device copies)",
            "value": w.n * args.steps / (ms_slab / 1000.0), "unit": "particle-updates/s",
            "n_gpus": 1, "steps": args.steps, "ms_per_step": ms_slab / args.steps,
            "undivided_ms_per_step": ms_whole / args.steps,
            "exchange_bytes_per_step": tr.bytes_moved / args.steps,
            "bit_exact_vs_undivided": bool(exact), "slabs": args.slabs, "grid_layers": nz,
            "timing": "host clock around device-synchronised steps (the exchanges are host "
                      "driven)", "dtype": "f64" if prec == "fp64" else "f32+f64",
            "data": "synthetic", "config": {"workload": args.workload, "particles": w.n}}
    print(json.dumps(line), flush=True)
    return 0 if exact else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dense1m", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--retune-every", type=int, default=0,
                    help="run the autotuner's trials again every N timed steps (0: never)")
    ap.add_argument("--obs-window", type=int, default=0,
                    help="after the timed steps, compare the two precisions' observables "
                         "averaged over this many further steps (0: the values at the end)")
    ap.add_argument("--obs-every", type=int, default=500,
                    help="steps between the samples of --obs-window")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the autotuner's trials (default settings)")
    ap.add_argument("--no-early-launch", action="store_true",
                    help="launch the pass kernels in plain stream order (dem_set_early_launch 0)")
    ap.add_argument("--reorder-every", type=int, default=0,
                    help="keep the particle storage in cell order, permuting it every N steps "
                         "of the run (0: never)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="cut the system into this many z-slabs on one GPU (the spatial "
                         "decomposition, emulated) and report its cost and bit-exactness")
    ap.add_argument("--skip-steps", type=int, default=-1,
                    help="untimed steps before the warm-up (ensembles: the beds start to "
                         "form; default: the workload's own)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = env_int("WORLD_SIZE", 1)
    if args.gpus != world:
        # one process per GPU: N > 1 must come from a launcher (torchrun)
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch --gpus N with "
              "python -m torch.distributed.run --nproc-per-node N", file=sys.stderr)
        return 2
    if args.impl == "reference":
        return run_reference(args)
    if args.slabs > 1:
        return run_slabs(args)
    if WORKLOADS[args.workload].get("kind") == "ensemble":
        return run_ensemble(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
