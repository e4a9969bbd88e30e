#!/usr/bin/env python
"""Benchmark: ns/day of the nonbonded hot path on the 96,000-atom solvated PME box.

One step = one NVE MD step as SPONGE's driver runs it (SPONGE/main.cu:162-210, :283-329, :376)
with the nonbonded path on the GPU: the neighbor-list update by its policy (rebuild every 20
steps), fixed-point coordinates, LJ + PME direct, the long-range correction, the exclusion
correction, PME reciprocal space, then the leap-frog and SETTLE of the rigid waters, for 96,000
atoms (31,000 rigid waters + 3,000 solute atoms, 98.6 A box, rc 10 A, skin 2 A, PME 96^3) on
moving coordinates (Maxwell-Boltzmann velocities at 300 K after a steepest-descent relaxation
of the free solute atoms, then 300 equilibration steps with velocity rescaling).
ns/day = steps/s * 2 fs * 86400 / 1e6.

  value   device time per MD step (CUDA events on the launching stream), state resident in HBM,
          L2 flushed (256 MiB write) before every timed step
  e2e     the same MD steps with the state owned by the host: every step the coordinates are
          copied in from pinned host memory and the new coordinates copied back
  force_only  the list update + force graph on frozen coordinates (no integrator)
  --impl reference  the CPU baseline: the FP64 multithreaded restatement of the same path
          (SPONGE has no CPU implementation) on the host cores, one full evaluation per step
  fep48   beside the headline: the 48 batched FEP/TI lambda windows (618,180 atoms, soft core,
          dU/dlambda every step) as --workload fep48 times them, 40 steps (--no-fep skips it)
  --workload water1m  the 1,000,512-atom water box with PME 216^3, both forms
  --workload fep48    the 48 windows with their baselines (per-window graph branches, windows
          one after another in both forms)

Multi-GPU: independent replicas (one system per rank, no collective in the data path).
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DT_FS = 2.0
FLOP_PER_PAIR = 50.0       # in-cutoff pair: dr 3, r^2 5, rsqrt 1, powers 4, LJ 3, Ewald 26, scale 3, accumulate 6
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal at max SM clock
# DRAM bytes read + written by one launch of the pair kernel walking the pruned list on this
# workload, from an ncu capture of that kernel: the list plus the packed coordinates
PAIR_DRAM_BYTES = 25.01e6
# pair-kernel shape (sb_lj_set_kernel_variant) -> kernel name
PAIR_KERNEL = {2: "k_pair_x2", 8: "k_pair_fixed<8>", 4: "k_pair_fixed<4>", 1: "k_pair_compact"}


def ns_per_day(sec_per_step):
    return DT_FS * 86400.0 / 1e6 / sec_per_step


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise max of per-rank timings (every rank gets the result); identity without a
    process group. Replicas report the slowest rank, as the driver's clock would see it."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

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
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def pair_counts(system, uc):
    """List pairs (rc+skin) and in-cutoff pairs from the FP64 oracle (algorithmic work)."""
    import oracle
    keys = oracle.pairs(uc, system, "cells")
    _, _, d = oracle.direct(uc, system, keys, oracle.get_beta(system["cutoff"]))
    return int(keys.size), int(d["n_in_cutoff"])


def run_reference(args, rank, world):
    """CPU baseline: FP64 multithreaded restatement of the path, one evaluation per step."""
    if rank != 0:
        return
    import oracle
    from sponge_b200 import systems
    s = systems.config1()
    uc = oracle.crd_to_uint(oracle.periodic_map(s["crd"], s["box"]), s["box"])
    beta = oracle.get_beta(s["cutoff"])
    nthreads = oracle.threads()
    for _ in range(max(0, min(args.warmup, 1))):
        oracle.nonbonded(uc, s, beta)
    times = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t = time.perf_counter()
        oracle.nonbonded(uc, s, beta)
        times.append(time.perf_counter() - t)
    total = time.perf_counter() - t0
    sec = total / max(1, args.steps)
    v = ns_per_day(sec)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ns/day",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": v, "unit": "ns/day", "cores": nthreads, "kind": "port",
                         "sample": "one full FP64 evaluation of the 96,000-atom path per step "
                                   "(cell list + LJ/Ewald direct + exclusions + SPME 96^3)"},
        "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    rc = reference_cuda(s, uc, args.steps)
    if rc is not None:
        line["reference_cuda"] = rc
    print(json.dumps(line), flush=True)


def reference_cuda(s, uc, steps):
    """The reference's own CUDA modules (NEIGHBOR_LIST, LENNARD_JONES_INFORMATION,
    Particle_Mesh_Ewald as shipped, built for sm_100a from the reference's sources into
    oracle/_ref by oracle/ref_harness) on the same system and GPU: CUDA-event time of a force step
    (list update every 20 steps + LJ/PME direct + long-range correction + exclusion correction +
    PME reciprocal) on frozen coordinates, as oracle/ref_harness/harness.cu times it. None where
    the harness binary or a GPU is absent."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except ImportError:
        return None
    import oracle
    from oracle.ref_harness import run as refrun
    if not refrun.available():
        return None
    keys = oracle.pairs(uc, s, "cells")
    r = refrun.run(s, uc, keys, timing_steps=max(20, steps))
    ms_step = float(r["summary"]["ms_step"])
    ms_force = float(r["summary"]["ms_force_only"])
    return {"kind": "the reference's CUDA modules, built for sm_100a from its sources",
            "ms_per_step": ms_step, "ns_per_day": ns_per_day(ms_step * 1e-3),
            "ms_per_force_evaluation": ms_force,
            "what": "list update every 20 steps + LJ/PME direct + long-range correction + "
                    "exclusion correction + PME reciprocal on frozen coordinates (compare with "
                    "the force_only field of the chosen form's line)",
            "timing_steps": max(20, steps)}


METRIC = "ns/day, 96k-atom PME water, 1 B200 (nonbonded path, fixed-point form)"


def workload_config():
    return {"workload": "solvated96k_pme96: 31,000 rigid waters + 3,000 solute atoms (20 LJ "
                        "types), 98.6 A cube, rc 10 A, skin 2 A, PME 96^3, list rebuilt every "
                        "20 steps, dt 2 fs, NVE leap-frog + SETTLE at 300 K on moving coordinates; pair "
                        "kernel on the list pruned to rc + 1 A (renewed after each rebuild and on "
                        "any 0.5 A move)",
            "atoms": 96000, "l2": "flushed (256 MiB write) before every timed step",
            "parallelism": "replicas"}


WATER1M_METRIC = "ns/day, 1,000,512-atom PME water (216^3), 1 B200: chosen vs plain form"


def water1m_config():
    return {"workload": "water1m_pme216: 333,504 rigid waters (70^3 lattice minus 9,496 sites), "
                        "215.3 A cube, rc 10 A, skin 2 A, PME 216^3, list rebuilt every 20 "
                        "steps, dt 2 fs, NVE leap-frog + SETTLE at 300 K; pair kernel on the list "
                        "pruned to rc + 1 A",
            "atoms": 1000512, "l2": "flushed (256 MiB write) before every timed step",
            "parallelism": "replicas"}


FEP_METRIC = "aggregate ns/day, %d FEP/TI lambda windows (soft-core), 1 B200"


def run_fep(args, rank, world, local, dist=None, emit=True):
    """48 uneven water boxes with a vanishing 20-atom solute, one lambda each, batched on each
    GPU: one launch per stage over all boxes (sb_fep_batch_step) under one captured CUDA graph
    (boxes sharded over ranks, the per-window dU/dlambda gathered at the end). Baselines on the
    same GPU: the per-box steps as concurrent graph branches on tuned streams (same steps, same
    list rebuilds), and, as force steps without list rebuilds, the 48 boxes one after another
    through the fixed-form fused step without the graph and through the plain-form modules
    (float atomics, per-atom lists, cuFFT)."""
    import torch
    from sponge_b200 import FORM_PLAIN, systems
    from sponge_b200.fep import FepBatch, FepEngine, box_cost, shard_boxes
    torch.cuda.set_device(local)
    own = False  # the process group is this function's (standalone run) or the caller's
    if world > 1 and dist is None:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        own = True
    nbox = args.fep_boxes  # 48 for the workload; fewer (its first windows) for profiling
    boxes = [systems.config4(k) for k in range(nbox)]
    mine = shard_boxes([box_cost(b) for b in boxes], world)[rank]
    batch = FepBatch([boxes[k] for k in mine], mode=args.fep_mode)
    batch.rebuild()
    ns, tune_ms = batch.tune()
    stream = torch.cuda.current_stream()
    # launches per list rebuild of one box: k_prepare, k_colscan, k_colsort, k_scatter,
    # k_excl_range, k_search, k_crd_to_uint
    rebuild_launches = 7 * len(mine)

    def timed(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    # the NVTX range marks the timed steps for a profiler's launch list (no cost without one)
    with torch.cuda.nvtx.range("fep_steps"):
        ms = timed(batch.step, args.steps)
    ms = max_over_ranks([ms], dist, "cuda")[0]
    # per-window dU/dlambda of all 48 boxes on rank 0 (the only collective)
    dudl = torch.zeros(nbox, dtype=torch.float64, device="cuda")
    dudl[torch.tensor(mine, device="cuda")] = batch.dudl
    if dist is not None:
        dist.all_reduce(dudl)
    # the two parts of a step: the captured force step of all boxes, and the list rebuild of
    # all boxes (every refresh_interval steps)
    replay_ms = timed(batch.graph.replay, 20)
    rebuild_ms = timed(batch.rebuild, 3)
    launches = None
    if batch.launches is not None:
        rebuilds = sum(1 for c in range(batch.count - args.steps, batch.count)
                       if c % batch.refresh_interval == 0)
        launches = args.steps * batch.launches + rebuilds * rebuild_launches
    base_plain = base_seq = base_streams = None
    if rank == 0 and not args.no_plain:
        if args.fep_mode == "kernels":
            other = FepBatch([boxes[k] for k in mine], mode="streams")
            other.rebuild()
            other.tune()
            # the same steps and rebuild phase as the timed batch
            base_streams = timed(other.step, args.steps) * len(boxes) / len(mine)
            del other

        def fixed_sequential():
            for e in batch.engines:
                e.frc.zero_()
                e.step()
        base_seq = timed(fixed_sequential, max(5, args.steps // 10)) * len(boxes) / len(mine)
        plain = [FepEngine(boxes[k], form=FORM_PLAIN) for k in mine]
        for e in plain:
            e.update_list(forced=1)
            e.to_uint()

        def plain_sequential():
            for e in plain:
                e.frc.zero_()
                e.forces_modules()
                e.sc.Get_Partial_H_Partial_Lambda(e.uint_crd, e.charge, e.nl, e.pme.beta)
        base_plain = timed(plain_sequential, max(5, args.steps // 10)) * len(boxes) / len(mine)
    if dist is not None:
        dist.barrier()
    if rank != 0:
        if own:
            dist.destroy_process_group()
        return None
    atoms = sum(len(b["charge"]) for b in boxes)
    value = nbox * ns_per_day(ms * 1e-3)
    line = {
        "metric": FEP_METRIC % nbox, "value": value, "unit": "ns/day", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 pair math, int64 fixed-point accumulation, f64 dU/dlambda",
        "data": "synthetic (seeded generator, sponge_b200.systems.config4)",
        "config": {"workload": ("fep48: 48 water boxes" if nbox == 48 else
                                "the first %d windows of fep48: water boxes" % nbox) +
                               " (500-8,000 waters, 0.997 g/cm^3) with a "
                               "20-atom solute vanishing in lambda, soft core alpha 0.5, p 1, "
                               "sigma 3 A, lambda = k/47, rc 9 A, skin 2 A, PME ~1 A grids, "
                               "list rebuilt every 20 steps",
                   "atoms": atoms, "boxes_per_rank": len(mine), "mode": args.fep_mode,
                   "graph_branches": ns, "parallelism": "boxes sharded over ranks"},
        "gpu_launches": launches,
        "gpu_launches_per_step": batch.launches,
        "force_step_ms": replay_ms, "rebuild_ms": rebuild_ms,
        "rebuild_interval": batch.refresh_interval,
        "dudl_per_window": [float(x) for x in dudl.cpu().numpy()],
        "baselines_ns_per_day": {
            "per_box_graph_branches":
                nbox * ns_per_day(base_streams * 1e-3) if base_streams else None,
            "plain_form_sequential": nbox * ns_per_day(base_plain * 1e-3) if base_plain else None,
            "fixed_form_sequential_no_graph":
                nbox * ns_per_day(base_seq * 1e-3) if base_seq else None},
    }
    if emit:
        print(json.dumps(line), flush=True)
    if own:
        dist.destroy_process_group()
    return line


def hbm_view(traffic_bytes, ms):
    """The pair kernel's DRAM traffic rate against the measured HBM copy rate of this GPU type
    (MEASURED_PEAKS.json beside this file), or the pool's earlier measurement where that file is
    absent."""
    peak, src = 6650.0, "fallback"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, src = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        pass
    achieved = traffic_bytes / (ms * 1e-3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": src}


MODULES_METRIC = "us per call, SPONGE's covid-tip4p modules beside the nonbonded path, 1 B200"


def run_modules(args, rank, world, local):
    """Device time per call of the modules beside the nonbonded path on the reference's own real
    system (covid-tip4p, 98,282 atoms; tests/golden fixture): the 1-4 pairs (force, atom energy
    and virial), the virtual atoms (coordinate refresh, force redistribution), and the NVE
    leap-frog with SETTLE as separate module calls (the system keeps constraint pairs that SETTLE
    leaves to another scheme, so the fused launch does not apply). CUDA events, L2 flushed before
    every call. Rank 0 only."""
    import importlib.util
    import torch
    from sponge_b200 import (NonBond14, NonbondedEngine, Settle, VirtualAtoms,
                             constrain_pairs_from_bonds, md_leap_frog, nb14_pair_tables)
    if rank != 0:
        return
    torch.cuda.set_device(local)
    spec = importlib.util.spec_from_file_location(
        "make_covid", os.path.join(ROOT, "tests", "golden", "make_covid.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    s = mod.load_system()
    n = len(s["charge"])
    eng = NonbondedEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    dev = lambda x: torch.tensor(np.ascontiguousarray(x), device="cuda")  # noqa: E731
    A, B = nb14_pair_tables(s["nb14_a"], s["nb14_b"], s["nb14_lj_scale"],
                            np.float32(12.0) * s["lj_A"], np.float32(6.0) * s["lj_B"],
                            s["lj_type"])
    nb14 = NonBond14(n, s["nb14_a"], s["nb14_b"], A, B, s["nb14_cf"])
    vs = VirtualAtoms(n, s["vs_type"], s["vs_atoms"], s["vs_param"])
    pi, pj, pr = constrain_pairs_from_bonds(s["bond_a"], s["bond_b"], s["bond_r"], s["mass"])
    dt = float(s["md_dt"])
    st = Settle(n, pi, pj, pr, s["mass"], dt)
    m64 = s["mass"].astype(np.float64)
    inv = dev(np.divide(1.0, m64, out=np.zeros_like(m64), where=m64 != 0).astype(np.float32))
    mass = dev(s["mass"])
    frc = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    av = torch.zeros(n, dtype=torch.float32, device="cuda")
    vel = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    crd = eng.crd.clone()
    acc = torch.zeros_like(vel)
    press = torch.zeros(1, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    calls = {
        "nb14_force_energy_virial": lambda: nb14.Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial(
            eng.uint_crd, eng.charge, eng.scaler, frc, ae, av),
        "vsite_coordinate_refresh": lambda: vs.Coordinate_Refresh(eng.uint_crd, eng.scaler, crd),
        "vsite_force_redistribute": lambda: vs.Force_Redistribute(eng.uint_crd, eng.scaler, frc),
        "settle_remember": lambda: st.Remember_Last_Coordinates(eng.uint_crd, eng.scaler),
        "leap_frog": lambda: md_leap_frog(n, inv, frc, vel, crd, 0.0, acc=acc),
        "settle_apply": lambda: st.Do_SETTLE(mass, crd, eng.box, vel, 1, press),
    }
    out = {}
    for name, fn in calls.items():
        for _ in range(max(3, args.warmup)):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            fn()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        out[name] = 1e3 * float(np.mean([a.elapsed_time(b) for a, b in ev]))
    line = {
        "metric": MODULES_METRIC, "value": sum(out.values()), "unit": "us",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
        "scaling": "none", "vs_baseline": None,
        "dtype": "f32 arithmetic, int64 fixed-point accumulation (1-4 pairs)",
        "data": "SPONGE covid-tip4p inputs (tests/golden/covid_tip4p_inputs.npz)",
        "config": {"workload": "covid-tip4p: %d atoms, %d 1-4 pairs, %d virtual atoms, %d rigid "
                               "waters and %d rigid pairs (SETTLE), %d constraint pairs left"
                               % (n, len(s["nb14_a"]), len(s["vs_type"]), st.triangle_numbers,
                                  st.pair_numbers, st.remaining_pairs),
                   "l2": "flushed (256 MiB write) before every timed call",
                   "leap_frog": "dt 0 so the coordinates stay as read (same arithmetic)"},
        "us_per_call": out,
    }
    print(json.dumps(line), flush=True)


def md_degrees_of_freedom(n_atoms, n_constraints):
    """3 per atom, less one per distance constraint (a rigid water holds three) and the three of
    the removed centre-of-mass momentum."""
    return 3 * int(n_atoms) - int(n_constraints) - 3


def setup_md(eng, s, seed, relax_iters=300, temperature=300.0, equil_steps=300):
    """Untimed MD set-up on the device. The seeded generators place the free (unconstrained)
    solute atoms by random sequential addition at >= 2.2 A, which leaves LJ overlaps of several
    thousand kcal/mol/A: those atoms are first relaxed by steepest descent (every free atom moves
    along its force by at most 0.02 A per iteration, the waters stay as built), then velocities
    are drawn from the Maxwell-Boltzmann distribution at ``temperature`` (seeded), with the
    centre-of-mass momentum removed, and the system is equilibrated by `equil_steps` MD steps with
    velocity rescaling. Returns the buffers of the NVE leap-frog + SETTLE step."""
    import torch
    from sponge_b200 import TIME_CONVERSION, Settle, constrain_pairs_from_bonds, sponge_io
    ba, bb, br, mass = sponge_io.bonds_and_masses(s)
    pi, pj, pr = constrain_pairs_from_bonds(ba, bb, br, mass)
    n = eng.n
    constrained = np.zeros(n, bool)
    constrained[np.asarray(pi, np.int64)] = True
    constrained[np.asarray(pj, np.int64)] = True
    free = torch.tensor(np.nonzero(~constrained)[0], device="cuda")
    if free.numel():
        for it in range(relax_iters):
            eng.update_list(forced=1 if it % 20 == 0 else 0)
            eng.to_uint()
            eng.frc.zero_()
            eng.force()
            f = eng.frc[free]
            fn = f.norm(dim=1, keepdim=True)
            step = 0.02 * f / torch.clamp(fn, min=50.0)
            eng.crd[free] += step
    dt = float(np.float32(np.float32(DT_FS * 1e-3) * np.float32(TIME_CONVERSION)))
    settle = Settle(n, pi, pj, pr, mass, dt)
    m64 = mass.astype(np.float64)
    inv = np.divide(1.0, m64, out=np.zeros_like(m64), where=m64 != 0)
    vel = sponge_io.maxwell_boltzmann(m64, temperature, seed)
    inv_t = torch.tensor(inv.astype(np.float32), device="cuda")
    mass_t = torch.tensor(mass.astype(np.float32), device="cuda")
    vel_t = torch.tensor(vel.astype(np.float32), device="cuda")
    acc_t = torch.zeros_like(vel_t)
    eng.update_list(forced=1)
    # equilibration: the generated waters start with random orientations, so their first steps
    # carry the excess energy of close contacts; `equil_steps` NVE steps with the velocities
    # rescaled to `temperature` every 10 steps (a Berendsen thermostat with tau = dt) bring the
    # system to the motion of an equilibrated run before anything is timed
    ke_target = 0.5 * md_degrees_of_freedom(n, len(pi)) * 0.0019872041 * temperature
    for k in range(equil_steps):
        eng.update_list()
        eng.md_step(settle, inv_t, mass_t, vel_t, acc_t)
        if k % 10 == 9:
            ke = 0.5 * float((mass_t[:, None] * vel_t * vel_t).double().sum())
            if ke > 0:
                vel_t.mul_(float(np.sqrt(ke_target / ke)))
    eng.update_list(forced=1)
    return settle, inv_t, mass_t, vel_t, acc_t


def timed_steps(fn, steps, flush, stream, dist=None):
    """Per-step device time (CUDA events on the launching stream), L2 flushed (256 MiB write)
    before every step outside the events; a barrier and a synchronize on both sides."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        fn()
        ev[k][1].record(stream)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def kernel_times(eng, flush, stream, reps=10):
    """Device time of the parts of one force step, each called alone through its module entry
    point (CUDA events, L2 flushed before each call): the pair kernel with its pack and finalize
    (LJ + Ewald direct), the reciprocal chain (spread, FFTs with the convolution, gather) and a
    list rebuild (the whole sequence: fixed point, column sort, search)."""
    import torch
    out = {}
    parts = {"pair": lambda: eng.forces(parts=("direct",)),
             "reciprocal": lambda: eng.forces(parts=("reciprocal",)),
             "rebuild": lambda: eng.update_list(forced=1)}
    for name, fn in parts.items():
        fn()
        torch.cuda.synchronize()
        out[name] = float(np.mean(timed_steps(fn, reps, flush, stream)))
    eng.frc.zero_()
    return out


def pme_bytes(n_atoms, fft):
    """Algorithmic HBM bytes of one reciprocal evaluation: per atom 16 B read (coordinates,
    charge), 12 B force written, 16 B read again by the gather; per grid point 4 B x (zero,
    spread write, gather read) and 4 B x (2 real-to-complex, 2 complex-to-real, 2 Green's-function
    multiply) for the FFTs and the convolution."""
    G = int(np.prod(fft))
    return n_atoms * 44 + G * 4 * 9


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fixed", choices=["fixed", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-fep", action="store_true",
                    help="headline run: skip the batched FEP windows reported beside it")
    ap.add_argument("--fep-boxes", type=int, default=48,
                    help="fep48: number of windows (the first ones; 48 is the workload)")
    ap.add_argument("--fep-mode", default="kernels", choices=["kernels", "streams"],
                    help="fep48: one launch per stage over all boxes, or per-box graph branches")
    ap.add_argument("--pair-shape", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="pair-kernel shape (sb_lj_set_kernel_variant); 0 = pick by timing")
    ap.add_argument("--workload", default="solvated96k",
                    choices=["solvated96k", "water1m", "fep48", "modules"],
                    help="water1m: the 1,000,512-atom water box with PME 216^3 (both forms, "
                         "per-kernel roofline; reported separately from the headline line); "
                         "fep48: the 48 batched FEP/TI lambda windows; modules: the 1-4 pair, "
                         "virtual atom and integrator/SETTLE calls on covid-tip4p")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "fep48":
        run_fep(args, rank, world, local)
        return
    if args.workload == "modules":
        run_modules(args, rank, world, local)
        return
    run_md(args, rank, world, local)


def run_md(args, rank, world, local):
    """The headline (and the water1m line): NVE MD steps of the chosen form on moving
    coordinates, each the list update by its policy (rebuild every 20 steps; the pruned pair list
    renewed on 0.5 A moves) followed by one captured CUDA graph of fixed
    point, force step and the fused leap-frog + SETTLE launch."""
    import torch
    import sponge_b200  # noqa: F401  (fails loudly without the library)
    from sponge_b200 import FORM_FIXED, FORM_PLAIN, NonbondedEngine, systems

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    big = args.workload == "water1m"
    s = systems.config2() if big else systems.config1()
    cfg = water1m_config() if big else workload_config()
    metric = WATER1M_METRIC if big else METRIC
    form = FORM_FIXED if args.form == "fixed" else FORM_PLAIN
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def make(form_):
        eng = NonbondedEngine(s, form=form_, refresh_interval=20)
        eng.update_list(forced=1)
        eng.to_uint()
        shape = None
        if form_ == FORM_FIXED:
            # autotuner: time each pair-kernel shape on this list and keep the fastest (or the
            # shape given on the command line, e.g. for a profiler run)
            if args.pair_shape:
                eng.lj.set_kernel_variant(args.pair_shape)
                shape = args.pair_shape
            else:
                shape = eng.lj.tune(eng.nl, eng.uint_crd, eng.charge, eng.pme.beta)
        md = setup_md(eng, s, seed=2000 + rank)
        eng.md_step(*md)
        eng.capture_md_graph(*md)
        return eng, md, shape

    eng, md, pair_shape = make(form)
    for _ in range(max(3, args.warmup)):
        eng.md_step_graph()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    t_wall = time.perf_counter()
    # the NVTX range marks the timed MD steps for a profiler's launch list (no cost without one)
    with torch.cuda.nvtx.range("md_steps"):
        dev = timed_steps(eng.md_step_graph, args.steps, flush, stream, dist)
    t_wall = time.perf_counter() - t_wall

    # e2e through the public API with host buffers: every step the caller's coordinates are
    # copied in from pinned host memory, the MD step runs, and the new coordinates are copied
    # back (the host owns the state: step k + 1 starts from what step k returned)
    crd_host = torch.empty((eng.n, 3), dtype=torch.float32).pin_memory()
    crd_host.copy_(eng.crd)

    def e2e_step():
        eng.crd.copy_(crd_host, non_blocking=True)
        eng.md_step_graph()
        crd_host.copy_(eng.crd, non_blocking=True)
    e2e = timed_steps(e2e_step, args.steps, flush, stream, dist)
    clk = clocks.stop()

    # force-only step on frozen coordinates (the previous headline): list update + force graph
    eng.capture_force_graph()
    for _ in range(3):
        eng.step_graph()
    fo = timed_steps(eng.step_graph, args.steps, flush, stream, dist)
    kt = kernel_times(eng, flush, stream)
    crd_scratch = eng.crd.clone()
    md_ms = float(np.mean(timed_steps(
        lambda: md[0].nve_step(eng.uint_crd, eng.scaler, md[1], md[2], eng.frc, md[3],
                               crd_scratch, eng.box, acc=md[4]), 10, flush, stream)))

    ms, e2e_ms, fo_ms = max_over_ranks([float(np.mean(dev)), float(np.mean(e2e)),
                                        float(np.mean(fo))], dist, "cuda")
    # the chosen form's forces at the current coordinates (list rebuilt), for the force error
    eng.update_list(forced=1)
    eng.to_uint()
    eng.frc.zero_()
    eng.force()
    crd_snapshot = eng.crd.clone()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    f_fixed = eng.frc.cpu().numpy()
    # the batched FEP/TI windows (config 4) on the same GPU, reported beside the headline
    fep = None
    if not big and not args.no_fep:
        fa = argparse.Namespace(**vars(args))
        fa.fep_boxes, fa.fep_mode, fa.steps, fa.warmup, fa.no_plain = 48, "kernels", 40, 5, True
        fep = run_fep(fa, rank, world, local, dist=dist, emit=False)
    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    n_list, n_cut = pair_counts(s, uc)
    flops = FLOP_PER_PAIR * n_cut
    pair_ms = kt["pair"]
    achieved = flops / (pair_ms * 1e-3) / 1e12
    rb = pme_bytes(eng.n, (eng.pme.fftx, eng.pme.ffty, eng.pme.fftz))
    hbm_peak = hbm_view(0, 1.0)["peak"]
    # launches per MD step: fixed point, the 8 of the force step, the integrator; a rebuild (6)
    # every 20 steps
    launches = 10 if form == FORM_FIXED else None
    line = {
        "metric": metric,
        "value": world * ns_per_day(ms * 1e-3),
        "unit": "ns/day",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 pair math, int64 fixed-point accumulation, f64 energies" if form == FORM_FIXED
                 else "f32 float atomics",
        "data": "synthetic (seeded generator, sponge_b200.systems.%s; free solute atoms relaxed "
                "by steepest descent, Maxwell-Boltzmann velocities at 300 K, 300 equilibration "
                "steps with velocity rescaling)"
                % ("config2" if big else "config1"),
        "config": dict(cfg, form=args.form, pair_kernel_shape=pair_shape),
        "e2e": {"value": world * ns_per_day(e2e_ms * 1e-3), "unit": "ns/day",
                "h2d_bytes_per_step": int(eng.n * 12), "d2h_bytes_per_step": int(eng.n * 12)},
        "gpu_launches": None if launches is None else
            int(round(args.steps * (launches + 6 / 20.0))),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": FP32_PEAK_TFLOPS,
                     "unit": "TFLOP/s", "frac": achieved / FP32_PEAK_TFLOPS,
                     "traffic": PAIR_DRAM_BYTES if not big else None,
                     "kernel": "%s (LJ + Ewald direct; timed with its pack and finalize)"
                               % PAIR_KERNEL.get(pair_shape, "k_pair_fixed"),
                     "kernel_ms": pair_ms, "pairs_in_cutoff": n_cut, "pairs_in_list": n_list,
                     "peak_note": "nominal FP32 peak 148 SM x 128 lanes x 2 x 1.965 GHz (the "
                                  "measured peaks cover HBM copy and bf16 tensor throughput "
                                  "only); the kernel is bound by instruction issue"},
        "kernels": {
            "pair_ms": pair_ms,
            "reciprocal": {"ms": kt["reciprocal"], "algorithmic_bytes": rb,
                           "achieved_gbs": rb / (kt["reciprocal"] * 1e-3) / 1e9,
                           "peak_gbs": hbm_peak,
                           "frac": rb / (kt["reciprocal"] * 1e-3) / 1e9 / hbm_peak},
            "rebuild_ms": kt["rebuild"],
            "integrator_ms": md_ms,
        },
        "force_only": {"value": world * ns_per_day(fo_ms * 1e-3), "unit": "ns/day",
                       "ms_per_step": fo_ms,
                       "what": "list update by its policy + force graph on frozen coordinates"},
        "clocks": clk,
        "wall_s": t_wall,
    }
    if not big:
        line["roofline"]["hbm"] = hbm_view(PAIR_DRAM_BYTES, pair_ms)
    import oracle
    beta = oracle.get_beta(s["cutoff"])
    ref_f = None
    if not args.no_cpu_baseline:
        t = time.perf_counter()
        ref_f, _, _ = oracle.nonbonded(uc, s, beta)
        sec = time.perf_counter() - t
        line["cpu_baseline"] = {"value": ns_per_day(sec), "unit": "ns/day",
                                "cores": oracle.threads(), "kind": "port",
                                "sample": "one full FP64 evaluation of the same %d-atom path "
                                          "(%.2f s)" % (eng.n, sec)}
        line["force_error_vs_fp64"] = {args.form: rel_rms(f_fixed, ref_f)}
    if not args.no_plain and form == FORM_FIXED:
        del eng, md
        torch.cuda.synchronize()
        pe, pmd, _ = make(FORM_PLAIN)
        for _ in range(max(3, args.warmup)):
            pe.md_step_graph()
        pdev = timed_steps(pe.md_step_graph, min(args.steps, 100), flush, stream)
        pms = float(np.mean(pdev))
        plain = {"value": ns_per_day(pms * 1e-3), "unit": "ns/day", "ms_per_step": pms,
                 "speedup_fixed_over_plain": pms / ms}
        if ref_f is not None:
            # the plain form's forces at the same coordinates
            pe.crd.copy_(crd_snapshot)
            pe.update_list(forced=1)
            pe.to_uint()
            assert np.array_equal(pe.uint_crd.cpu().numpy().view(np.uint32), uc)
            pe.frc.zero_()
            pe.force()
            line["force_error_vs_fp64"]["plain"] = rel_rms(pe.frc.cpu().numpy(), ref_f)
        line["plain_form"] = plain
    if fep is not None:
        line["fep48"] = {k: fep[k] for k in ("metric", "value", "unit", "ms_per_step", "steps",
                                            "force_step_ms", "rebuild_ms", "rebuild_interval",
                                            "gpu_launches_per_step", "config")}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


if __name__ == "__main__":
    main()
