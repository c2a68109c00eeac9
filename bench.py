#!/usr/bin/env python
"""Benchmark of the B200 force path on the 1,000,000-atom primitive-model electrolyte.

Workload (one GPU): 1,000,000 atoms (10 % +/-1 ions, neutral LJ solvent, rho = 0.8 sigma^-3,
L = 107.72 sigma), LJ cutoff 2.5, real-space alpha with erfc(sqrt(alpha) rc) <= 1e-5, FP32 forces
with compensated accumulation, FP64 velocity-Verlet + Berendsen.  A "step" is one full MD step
(kick, drift, cell sort, neighbour list, RBE sampling and structure factors, near + k-space
force, kick, temperature, thermostat).

Metric: atom-steps/s at equal k-space force RMSE, learned vs plain RBE.  The plain arm samples
P = 500 k-vectors per step with the reference's Metropolis-Hastings chain over RBE's Gaussian.
The learned arm trains the k-proposal network on the workload (200 snapshots 10 MD steps apart),
measures both proposals' force RMSE at P = 500 (the estimator is unbiased, so its RMS deviation
over independent k-sets at fixed positions is its error against the exact Ewald k-space force),
sets P_learned = ceil(500 * MSE_learned / MSE_plain) and times that.  `value` is the learned arm;
the plain arm's numbers are in `comparison`.  With --gpus N (torchrun, one process per GPU) every
rank advances its own independent replica ("replicas only", weak scaling; no data-path
collective); value = total atom-steps / max-over-ranks device time.

--impl reference times the reference path's CPU implementation (the oracle restatement of the
reference's FP32 force path; the reference itself cannot be built here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s at equal force RMSE vs FP64 Ewald: learned vs plain RBE"
N_ATOMS = 1_000_000
P_PLAIN = 500


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--atoms", type=int, default=N_ATOMS)
    ap.add_argument("--P", type=int, default=P_PLAIN)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=20,
                    help="host-buffer force calls of the end-to-end leg, cycling through as many position "
                         "frames recorded along the trajectory (list rebuilds at their natural rate)")
    ap.add_argument("--snapshots", type=int, default=200, help="training snapshots of the learned proposal")
    ap.add_argument("--train-iters", type=int, default=1500, help="Adam steps of the proposal network")
    ap.add_argument("--no-graph", action="store_true", help="launch every kernel of a step directly "
                    "instead of replaying the captured step graph")
    ap.add_argument("--noise-steps", type=int, default=16,
                    help="k-sets per proposal for the force-RMSE measurement")
    ap.add_argument("--ion-frac", type=float, default=0.1,
                    help="fraction of charged atoms of the electrolyte (0.1 is the headline workload)")
    ap.add_argument("--workload", default="electrolyte",
                    choices=["electrolyte", "electrolyte_plain", "lj", "water", "eam", "batched", "molecular",
                             "molecular_verlet"],
                    help="electrolyte: the headline metric (default); the others time the remaining "
                         "configurations (plain MD steps, atom-steps/s) beside the CPU reference path; "
                         "electrolyte_plain: the headline system (--atoms) with the plain Gaussian RBE sampler")
    ap.add_argument("--tuning", default=None,
                    help="JSON object of kernel variants (the configuration's \"tuning\" keys, e.g. "
                         "'{\"list_block\": 256, \"force_block\": 64}') instead of the autotuner")
    ap.add_argument("--skin", type=float, default=0.3,
                    help="Verlet skin; the list is rebuilt when an atom moved more than skin/2 "
                         "(forces are those of a per-step rebuild); 0 rebuilds every step")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# Algorithmic bytes / sincos per unit of each phase: the bytes a launch must move per unit it
# processes (each listed in the entry below).  "units" is the number of atoms (or charged atoms)
# one launch processes.  `pair` is the force pass: "near" (LJ / LJ + erfc over a Verlet or RBL
# list), "near_typed" (the same reading the (type, molecule) record of every atom once more),
# "eam" (two passes over the list).
def algorithmic(n, nq, n_nbr_mean, P, pair="near"):
    force = {
        # list entries (4 B/nbr), own pos4 (16 B), count + slot id (8 B), force (24 B); each
        # neighbour position is some atom's own pos4, counted once
        "near": 4 * n_nbr_mean + 16 + 8 + 24,
        "near_typed": 4 * n_nbr_mean + 16 + 8 + 8 + 24,
        # pass 1: entries + own pos4 + count + F'(rho) out; pass 2: entries + own pos4 + count +
        # F'(rho) + force out (tables and neighbour F' are L2-resident)
        "eam": (4 * n_nbr_mean + 16 + 4 + 4) + (4 * n_nbr_mean + 16 + 4 + 4 + 24),
    }[pair]
    return {
        # list build: own pos4 (16 B) + cell ranges (8 B) + list entries written (4 B each) + count
        "neighbor_list": {"units": n, "bytes": 16 + 8 + 4 * n_nbr_mean + 4},
        "force": {"units": n, "bytes": force},
        # structure factors over charged atoms: position (24 B) -> frac (16 B) written and read
        "kspace": {"units": nq, "bytes": 24 + 16 + 16, "sincos": P},
        # RBE force over charged atoms: frac (16 B) + far force (24 B)
        "rbe_force": {"units": nq, "bytes": 16 + 24, "sincos": P},
        "cell_sort": {"units": n, "bytes": 4 + 4 + 4 + 4 + 4 + 24 + 8 + 16 + 8},
        "integrate": {"units": n, "bytes": 24 * 4 + 8 + 4 + 4 + 24 * 2},
    }


# Per-atom DRAM traffic and warp instructions of the dominant pair kernel of each workload,
# measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum, smsp__inst_executed.sum) on the
# case named beside each entry; a full-size launch has the same per-atom work (same density and
# neighbour count), so the figures scale by atoms.  Summaries under profiles/.
PAIR_PROFILE = {
    # profiles/k_near_lean_electrolyte_200k.md, profiles/pair_kernels_all_workloads.md
    "electrolyte": {"kernel": "k_near_lean", "atoms": 200_000, "dram_bytes": 68.64e6, "warp_inst": 45.68e6},
    "batched": {"kernel": "k_near_lean", "atoms": 2_164_302, "dram_bytes": 775.98e6, "warp_inst": 556.30e6},
    "eam": {"kernel": "k_eam_fp + k_eam_force", "atoms": 256_000, "dram_bytes": 124.95e6, "warp_inst": 91.38e6},
    "water": {"kernel": "k_near_force_group (16 lanes)", "atoms": 30_000, "dram_bytes": 70.59e6,
              "warp_inst": 89.23e6},
    "lj": {"kernel": "k_near_force_group (32 lanes, FP64)", "atoms": 4_000, "dram_bytes": 1.42e6,
           "warp_inst": 2.09e6},
    "molecular": {"kernel": "k_rbl_force (8 lanes)", "atoms": 97_600, "dram_bytes": 44.68e6, "warp_inst": 81.31e6},
    "molecular_verlet": {"kernel": "k_near_force_group (16 lanes)", "atoms": 97_600, "dram_bytes": 175.68e6,
                         "warp_inst": 233.34e6},
}


def max_over_ranks(value, dist, device):
    """Maximum of a per-rank scalar over all ranks (the slowest rank's time); identity on one rank."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    m = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(m.item())


def aggregate_rate(world, atoms_per_rank, steps, max_ms):
    """Whole-job atom-steps/s: every rank advanced its own replica for `steps` steps."""
    return world * atoms_per_rank * steps / (max_ms / 1e3)


def partition_replicas(sizes, world):
    """Independent replicas of uneven atom counts split over `world` ranks by atom count (longest
    first, each to the rank holding the fewest atoms; ties to the lowest rank): per rank the
    ascending list of its replica indices.  The batch has no exchange between replicas, so each
    rank advances its share alone and the job needs no data-path collective."""
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(p) for p in parts]


def replica_subset(r, boxes, keep):
    """The batch r (systems.replicas) restricted to the replicas in `keep`: system, boxes, offsets."""
    off = r["offsets"]
    idx = np.concatenate([np.arange(off[k], off[k + 1]) for k in keep])
    sub = {key: r[key][idx] for key in ("pos", "vel", "mass", "charge", "type")}
    sub.update(molecule=None, eps=r["eps"], sigma=r["sigma"], lo=r["lo"][keep], hi=r["hi"][keep])
    sizes = np.diff(off)[keep]
    sub["offsets"] = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    return sub, [boxes[k] for k in keep], sub["offsets"]


def make_handle(s, dev, P, proposal, seed, skin, dt=None, ensemble="NVT", params=None, graph=True):
    """ForceField over a copy of system s on `dev` (1 replica)."""
    import torch
    from copy_gpu_b200 import Box, ForceField, systems
    kw = {} if dt is None else {"dt": dt}
    cfg = systems.electrolyte_config(P=P, precision="fp32", seed=seed, ensemble=ensemble, **kw)
    cfg["hyper_parameters"]["neighbor"]["skin"] = skin
    cfg["hyper_parameters"]["coulomb"]["proposal"] = proposal
    cfg["execution"]["cuda_graph"] = graph
    n = s["pos"].shape[0]
    t = {k: torch.tensor(s[k], device=dev, dtype=torch.float64).contiguous() for k in ("pos", "vel", "mass", "charge")}
    t["type"] = torch.tensor(s["type"], device=dev, dtype=torch.int32)
    t["force"] = torch.zeros((n, 3), device=dev, dtype=torch.float64)
    t["image"] = torch.zeros((n, 3), device=dev, dtype=torch.int32)
    ff = ForceField(cfg, Box(tuple(s["lo"]), tuple(s["hi"])))
    ff.set_pair_coeffs(s["eps"], s["sigma"])
    ff.Init(t["pos"], t["force"], vel=t["vel"], mass=t["mass"], charge=t["charge"], type=t["type"],
            image=t["image"])
    if params is not None:
        ff.proposal_params(params)
    return ff, t, cfg


def kspace_noise(ff, steps, warm=3):
    """Per-atom mean squared deviation of the RBE force estimator at fixed positions (a dt = 0
    handle): half the mean squared difference of the k-space forces of consecutive steps, whose
    k-sets are independent.  The estimator is unbiased (importance weights), so this is its
    mean squared error against the exact Ewald k-space force."""
    import torch
    ff.step(warm)
    prev, acc, cnt, sq = None, 0.0, 0, 0.0
    for _ in range(steps):
        ff.step(1)
        torch.cuda.synchronize()
        f = ff.far_force()
        sq += float((f ** 2).sum())
        if prev is not None:
            acc += float(((f - prev) ** 2).sum()) / 2.0
            cnt += 1
        prev = f
    kspace_noise.mean_sq = sq / steps   # E |F_estimate|^2 summed over atoms = |F_exact|^2 + noise
    return acc / cnt


STEP_LAUNCH_GRAPH = ("cuda graph replay: the first step launched directly, then graphs of 8 captured steps "
                     "and single-step graphs for the rest; phase_ms_per_step from a second pass of the "
                     "same length with phase events, kernels launched one by one")
STEP_LAUNCH_NOGRAPH = "kernels launched one by one (--no-graph); phase_ms_per_step from a second pass"


def timed_run(ff, t, dev, steps, warmup, world, dist, e2e_steps, autotune=True):
    """Warm-up, then `steps` timed MD steps (CUDA events, max over ranks), phases, clocks and the
    end-to-end host-buffer force call."""
    import torch
    local = dev.index or 0
    stream = torch.cuda.current_stream(dev)
    blocks = ff.autotune() if autotune else ("fixed", "fixed")
    ff.Execute()
    ff.step(warmup)
    torch.cuda.synchronize(dev)
    k_per_step = ff.launches_per_step()
    clocks = Clocks(local)
    builds0 = ff.list_builds()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ff.step(steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    builds = ff.list_builds() - builds0
    # per-phase breakdown: a second pass of the same length with the phase events on; the step
    # graph is not used while they are recorded, so the kernels launch one by one there
    pb0 = ff.list_builds()
    ff.profile(True)
    ff.step(steps)
    torch.cuda.synchronize(dev)
    phases = ff.phase_ms()
    ff.profile(False)
    prof_builds = ff.list_builds() - pb0
    flags = ff.status()
    if world > 1:
        ms = max_over_ranks(ms, dist, dev)
    n = ff.n
    ff.Execute()
    cnt, _ = ff.neighbors(0)
    n_nbr = float(cnt.mean())
    # end-to-end through the host-buffer C-ABI call: pinned positions in, pinned forces out, in the
    # reference's own Vec3f (float32) layout (rbmd_force_compute_host_f32) and in float64.  The
    # positions cycle through e2e_steps frames recorded one MD step apart along the trajectory, so
    # the Verlet-skin check rebuilds the list at its natural rate inside the timed calls.
    nf = max(1, e2e_steps)
    frames = []
    for _ in range(nf):
        ff.step(1)
        torch.cuda.synchronize(dev)
        frames.append(t["pos"].cpu())
    e2e, e2e_builds = {}, {}
    for dt in (torch.float32, torch.float64):
        pins = []
        for fr in frames:
            ph = torch.empty((n, 3), dtype=dt, pin_memory=True)
            ph.copy_(fr)
            pins.append(ph.numpy())
        frc_h = torch.empty((n, 3), dtype=dt, pin_memory=True)
        fh = frc_h.numpy()
        ff.compute_host(pins[-1], fh, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        b0 = ff.list_builds()
        w0 = time.perf_counter()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for k in range(nf):
            ff.compute_host(pins[k], fh, stream=stream.cuda_stream)
        a1.record(stream)
        torch.cuda.synchronize(dev)
        ms_e = max(a0.elapsed_time(a1), (time.perf_counter() - w0) * 1e3) / nf
        if world > 1:
            ms_e = max_over_ranks(ms_e, dist, dev)
        e2e[dt] = ms_e
        e2e_builds[dt] = (ff.list_builds() - b0) / nf
    return dict(ms=ms, builds=builds, prof_builds=prof_builds, phases=phases, flags=flags, clk=clk, n_nbr=n_nbr, e2e_ms=e2e[torch.float32],
                e2e64_ms=e2e[torch.float64], e2e_builds=e2e_builds[torch.float32], e2e_frames=nf,
                k_per_step=k_per_step, blocks=blocks)


def roofline(run, n, nq, P, steps, dev, pair="near", profile=None, kernel=None, nrep=1):
    """Per-phase achieved GB/s and sin/cos rates from the CUDA-event phase times, and the roofline
    object of the dominant kernel.  The k-space phases run on a second stream concurrently with
    the list build and near pass, so their event intervals include time shared with those
    kernels; the dominant kernel is taken among the caller-stream force kernels.  With a profile
    (PAIR_PROFILE) the pair kernel's DRAM traffic and its fraction of the instruction-issue
    ceiling (warp instructions / (SMs x 4 schedulers x SM clock x time)) are added."""
    import torch
    peaks, src = measured_peaks()
    alg = algorithmic(n, nq, run["n_nbr"], P, pair)
    phases = run["phases"]
    launches = {k: phases[k][1] for k in phases}
    sm_mhz = run["clk"]["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    mufu_peak = 16 * n_sm * sm_mhz * 1e6 / 2.0 / 1e9        # G sincos/s (2 MUFU ops each)
    rl = {}
    for k, a in alg.items():
        if k not in phases or launches[k] == 0:
            continue
        tot_ms = phases[k][0]
        per_launch_s = tot_ms / 1e3 / launches[k]
        if k == "integrate":
            per_launch_s = tot_ms / 1e3 / steps
        if k == "neighbor_list" and run["prof_builds"] > 0:
            # with a Verlet skin: time per full build (replica builds / replicas) of the profiled
            # pass; the launches of list-reuse steps exit early (a few us each)
            per_launch_s = tot_ms / 1e3 / max(run["prof_builds"] / nrep, 1e-9)
        ent = {"ms_per_step": tot_ms / steps, "launches": launches[k], "ms_per_launch": per_launch_s * 1e3}
        ent["hbm_gbs"] = a["bytes"] * a["units"] / per_launch_s / 1e9
        ent["hbm_frac"] = ent["hbm_gbs"] / peaks["hbm_gbs"]
        if "sincos" in a:
            ent["gsincos_s"] = a["sincos"] * a["units"] / per_launch_s / 1e9
            ent["mufu_frac"] = ent["gsincos_s"] / mufu_peak
            ent["stream"] = "k-space (overlaps the caller stream)"
        rl[k] = ent
    single = [k for k in ("force", "neighbor_list") if k in rl]
    dom = max(single, key=lambda k: rl[k]["ms_per_step"])
    d = rl[dom]
    roof = {"bound": "hbm", "achieved": d["hbm_gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": d["hbm_frac"], "kernel": (kernel or "near/EAM pass") if dom == "force" else
            f"neighbour-list build ({'per build' if run['builds'] > 0 else 'every step'})",
            "peak_source": f"{src} hbm_gbs (MEASURED_PEAKS.json)", "traffic": None,
            "algorithmic_bytes_per_launch": alg[dom]["bytes"] * alg[dom]["units"],
            "ms_per_launch": d["ms_per_launch"]}
    if dom == "force" and profile is not None:
        scale = n / profile["atoms"]
        roof["kernel"] = profile["kernel"]
        roof["traffic"] = profile["dram_bytes"] * scale
        roof["traffic_source"] = (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of the {profile['atoms']}-atom "
                                  "launch (summary under profiles/) scaled by atoms")
        inst = profile["warp_inst"] * scale
        ceiling_s = inst / (n_sm * 4 * sm_mhz * 1e6)
        roof["issue"] = {"warp_instructions_per_launch": inst, "issue_ceiling_ms": ceiling_s * 1e3,
                         "issue_frac": ceiling_s / (d["ms_per_launch"] / 1e3),
                         "what": "the pair kernel is bound by instruction issue and dependent latency, not "
                                 "HBM: its fraction of the issue ceiling (SMs x 4 schedulers x clock) beside "
                                 "the HBM fraction"}
    return roof, rl, mufu_peak


def run_ours(args):
    import torch
    import torch.distributed as dist
    from copy_gpu_b200 import systems

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    s = systems.electrolyte(args.atoms, ion_frac=args.ion_frac, seed=3 + rank)
    n = s["pos"].shape[0]
    nq = int((s["charge"] != 0).sum())
    P0 = args.P

    # ---- plain arm: the reference's Metropolis-Hastings Gaussian sampler, P = 500 ----
    ff, t, cfg = make_handle(s, dev, P0, "gauss", 7 + rank, args.skin, graph=not args.no_graph)
    plain = timed_run(ff, t, dev, args.steps, args.warmup, world, dist, args.e2e_steps)
    ff.close()
    del t

    # ---- learned arm: train on the workload (200 snapshots 10 MD steps apart) ----
    ff, t, _ = make_handle(s, dev, P0, "learned", 11 + rank, args.skin)
    ff.Execute()
    report = ff.train_proposal(n_snapshots=args.snapshots, steps_between=10, k_per_snapshot=16384,
                               iterations=args.train_iters, learning_rate=3e-3, seed=5 + rank)
    params = ff.proposal_params()
    ff.close()
    del t

    # ---- force RMSE of both proposals at P = 500 (fixed positions, independent k-sets) ----
    ffn, tn, _ = make_handle(s, dev, P0, "gauss", 13 + rank, 0.0, dt=0.0, ensemble="NVE")
    ffn.Execute()
    mse_plain = kspace_noise(ffn, args.noise_steps) / nq
    # RMS of the exact k-space force per charged atom: E|F_est|^2 = |F_exact|^2 + MSE (unbiased
    # estimator), so the scale against which the RMSE reads as a relative error
    exact_rms = float(np.sqrt(max(kspace_noise.mean_sq / nq - mse_plain, 0.0)))
    ffn.close()
    ffn, tn, _ = make_handle(s, dev, P0, "learned", 17 + rank, 0.0, dt=0.0, ensemble="NVE", params=params)
    ffn.Execute()
    mse_learned = kspace_noise(ffn, args.noise_steps) / nq
    ffn.close()
    del tn
    ratio = mse_learned / mse_plain
    P_eq = int(np.ceil(P0 * ratio))                 # MSE ~ 1/P: the learned P of equal RMSE

    # ---- timed learned arm at P_eq ----
    ff, t, cfg_l = make_handle(s, dev, P_eq, "learned", 19 + rank, args.skin, params=params,
                               graph=not args.no_graph)
    ffn, tn, _ = make_handle(s, dev, P_eq, "learned", 23 + rank, 0.0, dt=0.0, ensemble="NVE", params=params)
    ffn.Execute()
    mse_learned_eq = kspace_noise(ffn, args.noise_steps) / nq
    ffn.close()
    del tn
    learned = timed_run(ff, t, dev, args.steps, args.warmup, world, dist, args.e2e_steps)
    ff.close()

    v_plain = aggregate_rate(world, n, args.steps, plain["ms"])
    v_learned = aggregate_rate(world, n, args.steps, learned["ms"])
    out = None
    if rank == 0:
        roof, rl, _ = roofline(learned, n, nq, P_eq, args.steps, dev, profile=PAIR_PROFILE["electrolyte"])
        out = {
            "metric": METRIC,
            "value": v_learned,
            "unit": "atom-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": learned["ms"] / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"electrolyte {n} atoms"
                                   + ("" if args.ion_frac == 0.1 else f" ({args.ion_frac:g} charged)")
                                   + f", full MD step, learned k-proposal at P={P_eq} "
                                   f"(equal k-space force RMSE to plain Gaussian RBE at P={P0})",
                       "atoms_per_gpu": n, "P": P_eq, "P_plain": P0, "proposal": "learned", "rc": 2.5,
                       "skin": args.skin, "list_builds_per_step": learned["builds"] / args.steps,
                       "threads_per_block": {"list": learned["blocks"][0], "force": learned["blocks"][1]},
                       "alpha": cfg["hyper_parameters"]["coulomb"]["alpha"], "box": float(s["hi"][0]),
                       "parallelism": "replicas" if world > 1 else "single",
                       "step_launch": STEP_LAUNCH_NOGRAPH if args.no_graph else STEP_LAUNCH_GRAPH,
                       "l2": "inputs larger than L2 (neighbour list %.0f MB + state %.0f MB)"
                             % (4 * learned["n_nbr"] * n / 1e6, 72 * n / 1e6)},
            "comparison": {
                "plain": {"value": v_plain, "ms_per_step": plain["ms"] / args.steps, "P": P0,
                          "sampler": "Metropolis-Hastings over RBE's Gaussian (the reference's)",
                          "kspace_force_rmse": float(np.sqrt(mse_plain)),
                          "e2e": world * n / (plain["e2e_ms"] / 1e3)},
                "learned": {"value": v_learned, "ms_per_step": learned["ms"] / args.steps, "P": P_eq,
                            "kspace_force_rmse": float(np.sqrt(mse_learned_eq)),
                            "kspace_force_rmse_at_P_plain": float(np.sqrt(mse_learned)),
                            "variance_ratio_at_P_plain": ratio,
                            "training": report},
                "speedup_at_equal_rmse": v_learned / v_plain,
                "rmse_how": "per-atom RMS of the RBE estimator's deviation from its mean (unbiased, so from "
                            "the exact Ewald k-space force): half the mean squared difference of two "
                            f"independent k-sets at fixed positions, {args.noise_steps - 1} pairs",
            },
            # the north-star comparison, flat: learned vs plain RBE at equal k-space force RMSE
            "speedup_at_equal_rmse": v_learned / v_plain,
            "plain_value": v_plain,
            "variance_ratio_at_P_plain": ratio,
            "kspace_force_rmse": float(np.sqrt(mse_plain)),
            "kspace_force_rms_exact": exact_rms,
            "kspace_force_rel_rmse": float(np.sqrt(mse_plain)) / exact_rms if exact_rms > 0 else None,
            "roofline": roof,
            "phases": rl,
            "phase_ms_per_step": {k: {"learned": learned["phases"][k][0] / args.steps,
                                      "plain": plain["phases"][k][0] / args.steps}
                                  for k in learned["phases"] if k in plain["phases"]},
            "e2e": {"value": world * n / (learned["e2e_ms"] / 1e3), "unit": "atom-steps/s",
                    "h2d_bytes_per_step": 12 * n, "d2h_bytes_per_step": 12 * n,
                    "what": "rbmd_force_compute_host_f32: pinned host positions in, forces out, in the reference's "
                            f"Vec3f (float32) layout, one force evaluation per step, positions cycling through "
                            f"{learned['e2e_frames']} frames recorded one MD step apart (list rebuilds at their "
                            f"natural rate: {learned['e2e_builds']:.2f} per call)",
                    "list_builds_per_call": learned["e2e_builds"],
                    "fp64_host_buffers": {"value": world * n / (learned["e2e64_ms"] / 1e3),
                                          "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n,
                                          "what": "rbmd_force_compute_host (float64 host arrays)"}},
            "gpu_launches": learned["k_per_step"] * args.steps,
            "kernels_per_step": learned["k_per_step"],
            "status_flags": learned["flags"] | plain["flags"],
            "clocks": learned["clk"],
            "clocks_plain_arm": plain["clk"],
            "mean_neighbors": learned["n_nbr"],
        }
        if not args.no_cpu and world == 1:
            out["cpu_baseline"] = cpu_baseline(P0)
    if world > 1:
        dist.destroy_process_group()
    return out


def _electrolyte_sample(n_atoms, seed=3):
    from copy_gpu_b200 import systems
    return systems.electrolyte(n_atoms, seed=seed)


def cpu_force_eval(n_atoms, P, seed=3, sysd=None, use_ref=None):
    """One force evaluation of the reference path on the host cores: neighbour list, LJ + erfc
    near force, RBE k-sampling, structure factors and force.  With the reference's own code
    compiled here (oracle/_ref, use_ref) its worklets run (ComputeNeighboursWorklet,
    ComputeNearForceVerletWorklet, RBEPSAMPLE::Fetch_P_Sample, ComputePnumberChargeStructureFactor-
    Worklet over all N x P terms, ComputeNewRBEForceWorklet); otherwise the oracle restatement in
    FP32.  Returns seconds."""
    import oracle
    from oracle import ref
    from copy_gpu_b200 import systems
    s = sysd if sysd is not None else _electrolyte_sample(n_atoms, seed)
    cfg = systems.electrolyte_config(P=P)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    pos32 = s["pos"].astype(np.float32)
    use_ref = ref.available() if use_ref is None else use_ref
    t0 = time.perf_counter()
    if use_ref:
        nl = ref.neighbors(pos32, s["lo"], s["hi"], 2.5, cap=128)
        ref.near_force(pos32, s["lo"], s["hi"], 2.5, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                       sigma=s["sigma"], alpha=alpha, with_coul=True)
        m, _ = ref.rbe_sample(alpha, L, P, np.random.default_rng(seed).random(64 * P))
        rho = ref.rhok(pos32, s["charge"], L, m)
        ref.rbe_force(pos32, s["charge"], s["lo"], s["hi"], alpha, m, rho)
    else:
        m = oracle.rbe_sample(alpha, L, 7, 0, 0, P)
        nl = oracle.neighbors(pos32, s["lo"], s["hi"], 2.5, "fp32")
        oracle.near_force(pos32, s["lo"], s["hi"], 2.5, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                          sigma=s["sigma"], with_coul=True, alpha=alpha, sum_mode=0, prec="fp32")
        rho = oracle.rhok(pos32, s["charge"], L, m, prec="fp32")
        oracle.rbe_force(pos32, s["charge"], L, alpha, 1.0, m, rho, prec="fp32")
    return time.perf_counter() - t0


def _cpu_kind():
    from oracle import ref
    return ("reference", "the reference's own force-path worklets compiled from its source (oracle/_ref)") \
        if ref.available() else ("port", "the oracle's FP32 restatement of the reference path")


def _sample_size(P, evals, budget_s, cap_atoms=N_ATOMS):
    """Atoms per evaluation so that `evals` evaluations take about budget_s seconds (the reference
    materialises N x P structure-factor terms, 8 bytes each: at most 2 GB of them)."""
    t = cpu_force_eval(100_000, P, sysd=_electrolyte_sample(100_000))
    n = int(100_000 * budget_s / max(evals, 1) / max(t, 1e-3))
    n = min(n, cap_atoms, int(2e9 / (8 * P)))
    return max(20_000, (n // 10_000) * 10_000)


def cpu_baseline(P, n_atoms=N_ATOMS, min_seconds=10.0, max_evals=10):
    """The reference path on the host cores (its own code where it compiled here): force
    evaluations of a sample of the workload repeated until about min_seconds of CPU work."""
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    kind, what = _cpu_kind()
    n = _sample_size(P, 5, min_seconds, n_atoms)
    sysd = _electrolyte_sample(n)
    tot, evals = 0.0, 0
    while evals < max_evals and (evals == 0 or tot < min_seconds):
        tot += cpu_force_eval(n, P, sysd=sysd)
        evals += 1
    return {"value": n * evals / tot, "unit": "atom-steps/s", "cores": cores, "kind": kind,
            "sample": f"{evals} force evaluations (neighbour list, LJ/erfc near force, RBE sampling, structure "
                      f"factors and force, P={P}) of a {n}-atom sample of the {n_atoms}-atom electrolyte (same "
                      f"composition and density): {what}, {cores} OpenMP threads, {tot:.1f} s"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    kind, what = _cpu_kind()
    n = _sample_size(args.P, args.steps + 1, 45.0, args.atoms)
    sysd = _electrolyte_sample(n)
    cpu_force_eval(n, args.P, sysd=sysd)
    times = [cpu_force_eval(n, args.P, sysd=sysd, seed=3 + k) for k in range(args.steps)]
    tot = sum(times)
    value = n * args.steps / tot
    sample = (f"per step one force evaluation (neighbour list, LJ/erfc near force, RBE k-sampling, structure "
              f"factors and force, P={args.P}) of a {n}-atom sample of the {args.atoms}-atom electrolyte (same "
              f"composition and density), no integration: {what}, {cores} OpenMP threads")
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "atom-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"electrolyte force evaluation (neighbour list + LJ/erfc near + RBE P={args.P}) "
                               f"on a {n}-atom sample of the {args.atoms}-atom workload, plain Gaussian RBE",
                   "sample_atoms": n, "P": args.P},
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---- the other configurations: plain MD steps, GPU vs the CPU oracle -------------------------
def config_system(name, tmpdir, atoms=N_ATOMS):
    """(system, config, boxes, offsets, description) of a secondary configuration."""
    from copy_gpu_b200 import Box, systems
    if name == "electrolyte_plain":
        s = systems.electrolyte(atoms, seed=3)
        cfg = systems.electrolyte_config(P=P_PLAIN, precision="fp32", seed=7, ensemble="NVT")
        cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
        return s, cfg, None, None, (f"electrolyte {atoms} atoms, plain Gaussian RBE P={P_PLAIN} (the reference's "
                                    "sampler), rc 2.5 + skin 0.3, FP32 forces, full MD step")
    if name == "lj":
        s = systems.lj_fcc(ncell=10, seed=1)
        cfg = systems.lj_config(cutoff=2.5, skin=0.3, precision="fp64", ensemble="NVE")
        cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
        return s, cfg, None, None, "LJ FCC 4000 atoms, rho 0.8442, T 0.72, rc 2.5 + skin 0.3, FP64, NVE"
    if name == "water":
        s = systems.water(n_mol=10000, seed=9)
        cfg = systems.water_config(P=200, precision="fp32")
        cfg["hyper_parameters"]["neighbor"]["skin"] = 1.0
        return s, cfg, None, None, ("SPC/E water 10000 molecules (30000 atoms), rc 10 A + skin 1.0, RBE P=200, "
                                    "alpha 0.09, SHAKE, REAL units, FP32 forces")
    if name == "eam":
        pot = systems.write_johnson_funcfl(os.path.join(tmpdir, "johnson.eam"))
        s = systems.eam_fcc(ncell=40, seed=13)
        cfg = systems.eam_config(pot, precision="fp32")
        cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
        return s, cfg, None, None, ("Johnson EAM Cu FCC 256000 atoms (5000-point funcfl), rc 5.0 A + skin 0.3, "
                                    "300 K displacements, FP32, NVE")
    if name == "molecular_verlet":
        # the same system with the Verlet list (rc 12 A + skin 1 A, list reuse) instead of RBL
        s, cfg, _, _, _ = config_system("molecular", tmpdir)
        cfg["hyper_parameters"]["neighbor"] = {"type": "VERLETLIST", "cut_off": 12.0, "skin": 1.0}
        return s, cfg, None, None, (f"flexible chains + ions, {len(s['pos'])} atoms, CVFF topology, special bonds "
                                    "0/0/0, VERLETLIST rc 12 A + skin 1.0 A, RBE P=100, REAL units, FP32 forces")
    if name == "molecular":
        # the shape of the reference's polymer-electrolyte input (rbmd/res/json_files/PEO): CVFF
        # with bonds, angles, dihedrals and special bonds 0/0/0, RBL rc 12 A / r_core 6 A / 100
        # samples, RBE P=100 at alpha 0.074, REAL units, 0.5 fs, Berendsen
        s = systems.molecular(n_chain=8000, chain_len=12, n_ion_pairs=800, step=1.5, cell=6.0, seed=31)
        cfg = systems.molecular_config(P=100, cutoff=12.0, alpha=0.074, neighbor="RBL", special=(0.0, 0.0, 0.0),
                                       dt=0.5, precision="fp32", r_core=6.0, sample_num=100)
        cfg["execution"].update({"ensemble": "NVT", "temp_ctrl_type": "BERENDSEN",
                                 "temperature": [298.0, 298.0, 100.0]})
        return s, cfg, None, None, (f"flexible chains + ions, {len(s['pos'])} atoms (8000 chains of 12, 800 ion "
                                    "pairs, 0.041 atoms/A^3), bonds/angles/dihedrals, special bonds 0/0/0, RBL "
                                    "rc 12 A r_core 6 A 100 samples, RBE P=100, REAL units, FP32 forces")
    r = systems.replicas(n_rep=512, seed=11)
    cfg = systems.electrolyte_config(P=100, precision="fp32", ensemble="NVE")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    boxes = [Box(tuple(r["lo"][k]), tuple(r["hi"][k])) for k in range(512)]
    return r, cfg, boxes, r["offsets"], (f"512 electrolyte replicas of 500-8000 atoms ({int(r['offsets'][-1])} atoms), "
                                         "RBE P=100 each, rc 2.5 + skin 0.3, FP32, one step for all replicas")


def cpu_config_eval(name, s, cfg, offsets, tmpdir):
    """Seconds and atoms of one CPU force evaluation of the configuration (oracle restatement of
    the reference path; the batched case is sampled on its first 16 replicas)."""
    import oracle
    hp = cfg["hyper_parameters"]
    rc = hp["neighbor"]["cut_off"]
    prec = cfg.get("precision", "fp32")
    if name == "batched":
        total, atoms = 0.0, 0
        for k in range(16):
            a, b = int(offsets[k]), int(offsets[k + 1])
            sub = {key: s[key][a:b] for key in ("pos", "charge", "type")}
            sub.update(lo=s["lo"][k], hi=s["hi"][k], eps=s["eps"], sigma=s["sigma"])
            sec, n = cpu_config_eval("electrolyte_sub", sub, cfg, None, tmpdir)
            total += sec
            atoms += n
        return total, atoms
    pos = s["pos"].astype(np.float32 if prec == "fp32" else np.float64)
    L = s["hi"] - s["lo"]
    if name == "molecular_verlet":
        co = hp["coulomb"]
        t0 = time.perf_counter()
        sp = oracle.special_lists(len(pos), s["bonds"], hp["extend"]["special_bonds"])
        nl = oracle.neighbors(pos, s["lo"], s["hi"], rc, prec)
        oracle.near_force(pos, s["lo"], s["hi"], rc, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                          sigma=s["sigma"], with_coul=True, alpha=co["alpha"], coul_scale=332.06371, prec=prec,
                          special=sp)
        m = oracle.rbe_sample(co["alpha"], L, 7, 0, 0, co["coulomb_sample_num"])
        rho = oracle.rhok(pos, s["charge"], L, m, prec=prec)
        oracle.rbe_force(pos, s["charge"], L, co["alpha"], 332.06371, m, rho, prec=prec)
        oracle.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], s["bonds"], s["bond_type"],
                          s["bond_coeffs"], s["angles"], s["angle_type"], s["angle_coeffs"], s["dihedrals"],
                          s["dihedral_type"], s["dihedral_coeffs"], special=sp)
        return time.perf_counter() - t0, len(pos)
    if name == "molecular":
        nb, co = hp["neighbor"], hp["coulomb"]
        t0 = time.perf_counter()
        _, _, pice = oracle.rbl_sizes(len(pos), s["lo"], s["hi"], nb["r_core"], rc, nb["neighbor_sample_num"],
                                      prec=prec)
        sp = oracle.special_lists(len(pos), s["bonds"], hp["extend"]["special_bonds"])
        rl = oracle.rbl_list(pos, s["lo"], s["hi"], rc, nb["r_core"], pice, 128, 160, prec=prec)
        oracle.rbl_near(pos, s["lo"], s["hi"], rc, nb["r_core"], pice, rl, 128, type=s["type"], charge=s["charge"],
                        eps=s["eps"], sigma=s["sigma"], with_coul=True, alpha=co["alpha"], qqr2e=332.06371,
                        prec=prec, special=sp)
        m = oracle.rbe_sample(co["alpha"], L, 7, 0, 0, co["coulomb_sample_num"])
        rho = oracle.rhok(pos, s["charge"], L, m, prec=prec)
        oracle.rbe_force(pos, s["charge"], L, co["alpha"], 332.06371, m, rho, prec=prec)
        oracle.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], s["bonds"], s["bond_type"],
                          s["bond_coeffs"], s["angles"], s["angle_type"], s["angle_coeffs"], s["dihedrals"],
                          s["dihedral_type"], s["dihedral_coeffs"], special=sp)
        return time.perf_counter() - t0, len(pos)
    from oracle import ref
    if ref.available() and name in ("lj", "eam", "water", "electrolyte_plain", "electrolyte_sub"):
        # the reference's own worklets (FP32 -- its Real), compiled from its source
        p32 = s["pos"].astype(np.float32)
        t0 = time.perf_counter()
        nl = ref.neighbors(p32, s["lo"], s["hi"], rc)
        if name == "eam":
            ref.eam(oracle.eam_tables(hp["force_field"]["potential_file"]), p32, s["lo"], s["hi"], rc, nl)
            return time.perf_counter() - t0, len(pos)
        coul = "coulomb" in hp and name != "lj"
        alpha = hp["coulomb"]["alpha"] if coul else 0.0
        ref.near_force(p32, s["lo"], s["hi"], rc, nl, type=s["type"], mol=s.get("molecule"),
                       charge=s["charge"] if coul else None, eps=s["eps"], sigma=s["sigma"], alpha=alpha,
                       with_coul=coul)
        if coul:
            P = hp["coulomb"]["coulomb_sample_num"]
            m, _ = ref.rbe_sample(alpha, L, P, np.random.default_rng(7).random(64 * P))
            rho = ref.rhok(p32, s["charge"], L, m)
            ref.rbe_force(p32, s["charge"], s["lo"], s["hi"], alpha, m, rho)
        if "hoh" in s:
            oracle.water_extras(s["hoh"], s["pos"], s["charge"], s["lo"], s["hi"], *s["bond"], *s["angle"])
        return time.perf_counter() - t0, len(pos)
    t0 = time.perf_counter()
    nl = oracle.neighbors(pos, s["lo"], s["hi"], rc, prec)
    if name == "eam":
        oracle.eam_force(hp["force_field"]["potential_file"], pos, s["lo"], s["hi"], rc, nl, prec=prec)
        return time.perf_counter() - t0, len(pos)
    coul = "coulomb" in hp and name != "lj"
    alpha = hp["coulomb"]["alpha"] if coul else 0.0
    oracle.near_force(pos, s["lo"], s["hi"], rc, nl, type=s["type"], mol=s.get("molecule"),
                      charge=s["charge"] if coul else None, eps=s["eps"], sigma=s["sigma"], with_coul=coul,
                      alpha=alpha, sum_mode=0, prec=prec)
    if coul:
        P = hp["coulomb"]["coulomb_sample_num"]
        m = oracle.rbe_sample(alpha, L, 7, 0, 0, P)
        rho = oracle.rhok(pos, s["charge"], L, m, prec=prec)
        oracle.rbe_force(pos, s["charge"], L, alpha, 1.0, m, rho, prec=prec)
    if "hoh" in s:
        oracle.water_extras(s["hoh"], s["pos"], s["charge"], s["lo"], s["hi"], *s["bond"], *s["angle"])
    return time.perf_counter() - t0, len(pos)


def run_config(args):
    """One of the secondary configurations: `steps` MD steps timed with CUDA events (graph replay,
    inputs resident), the host-buffer force call end to end, and the CPU oracle single-threaded
    and on all cores."""
    import tempfile
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    with tempfile.TemporaryDirectory() as tmpdir:
        s, cfg, boxes, offs, desc = config_system(args.workload, tmpdir, args.atoms)
        parallel = "single"
        if world > 1 and args.workload == "batched":
            # the 512 replicas split over the ranks by atom count; no exchange between them
            parts = partition_replicas(np.diff(offs), world)
            s, boxes, offs = replica_subset(s, boxes, parts[rank])
            parallel = f"replicas partitioned over {world} ranks by atom count"
        elif world > 1:
            parallel = f"one independent copy per rank ({world} ranks)"
        if args.tuning:
            cfg["tuning"] = json.loads(args.tuning)
        if args.no_graph:
            cfg.setdefault("execution", {})["cuda_graph"] = False
        from copy_gpu_b200 import Box, ForceField
        n_all = s["pos"].shape[0]
        t = {k: torch.tensor(s[k], device=dev, dtype=torch.float64).contiguous()
             for k in ("pos", "vel", "mass", "charge")}
        t["type"] = torch.tensor(s["type"], device=dev, dtype=torch.int32)
        t["force"] = torch.zeros((n_all, 3), device=dev, dtype=torch.float64)
        t["image"] = torch.zeros((n_all, 3), device=dev, dtype=torch.int32)
        if s.get("molecule") is not None:
            t["molecule"] = torch.tensor(s["molecule"], device=dev, dtype=torch.int32)
        ff = ForceField(cfg, boxes or Box(tuple(s["lo"]), tuple(s["hi"])))
        ff.set_pair_coeffs(s["eps"], s["sigma"])
        if "hoh" in s:
            ff.set_water(s["hoh"], s["bond"][0], s["bond"][1], s["angle"][0], s["angle"][1])
        if "bonds" in s:
            ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"],
                            s["angle_type"], s["angle_coeffs"], s["dihedrals"], s["dihedral_type"],
                            s["dihedral_coeffs"])
        ff.Init(t["pos"], t["force"], vel=t["vel"], mass=t["mass"], charge=t["charge"], type=t["type"],
                molecule=t.get("molecule"), image=t["image"], replica_offsets=offs)
        run = timed_run(ff, t, dev, args.steps, args.warmup, world, dist if world > 1 else None, args.e2e_steps,
                        autotune=not args.tuning)
        n = ff.n
        n_job = n
        if world > 1:
            cnt = torch.tensor([float(n)], device=dev, dtype=torch.float64)
            dist.all_reduce(cnt)
            n_job = int(cnt.item())
        value = n_job * args.steps / (run["ms"] / 1e3)
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if cfg.get("precision") == "fp64" else "f32",
            "data": "synthetic",
            "config": {"workload": desc, "atoms": n_job, "atoms_rank0": n, "parallelism": parallel,
                       "list_builds_per_step": run["builds"] / args.steps / (len(boxes) if boxes else 1),
                       "threads_per_block": {"list": run["blocks"][0], "force": run["blocks"][1]},
                       "step_launch": STEP_LAUNCH_NOGRAPH if args.no_graph else STEP_LAUNCH_GRAPH},
            "e2e": {"value": n_job / (run["e2e_ms"] / 1e3), "unit": "atom-steps/s", "h2d_bytes_per_step": 12 * n,
                    "d2h_bytes_per_step": 12 * n,
                    "what": "rbmd_force_compute_host_f32: pinned host positions in, forces out (the reference's "
                            f"Vec3f layout), one force evaluation per call, positions cycling through "
                            f"{run['e2e_frames']} frames recorded one MD step apart",
                    "list_builds_per_call": run["e2e_builds"],
                    "fp64_host_buffers": {"value": n_job / (run["e2e64_ms"] / 1e3), "h2d_bytes_per_step": 24 * n,
                                          "d2h_bytes_per_step": 24 * n}},
            "phase_ms_per_step": {k: v[0] / args.steps for k, v in run["phases"].items() if v[1]},
            "gpu_launches": run["k_per_step"] * args.steps, "kernels_per_step": run["k_per_step"],
            "status_flags": run["flags"], "clocks": run["clk"], "mean_neighbors": run["n_nbr"],
        }
        hp = cfg["hyper_parameters"]
        pair = {"eam": "eam", "water": "near_typed", "molecular": "near_typed",
                "molecular_verlet": "near_typed"}.get(args.workload, "near")
        prof = PAIR_PROFILE.get("electrolyte" if args.workload == "electrolyte_plain" else args.workload)
        nq = int((np.asarray(s["charge"]) != 0).sum())
        P = int(hp.get("coulomb", {}).get("coulomb_sample_num", 0)) if "coulomb" in hp else 0
        roof, rl, _ = roofline(run, n, nq, max(P, 1), args.steps, dev, pair=pair, profile=prof,
                               nrep=len(boxes) if boxes else 1)
        line["roofline"] = roof
        line["phases"] = rl
        del ff
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.destroy_process_group()
            if rank != 0:
                return None
        if not args.no_cpu and world == 1:
            import oracle
            oracle.build()
            cores = os.cpu_count() or 1
            res = {}
            for th in (1, cores):
                oracle.set_threads(th)
                sec, atoms = cpu_config_eval(args.workload, s, cfg, offs, tmpdir)
                res[th] = atoms / sec
            from oracle import ref
            on_ref = ref.available() and args.workload in ("lj", "eam", "water", "electrolyte_plain", "batched")
            line["cpu_baseline"] = {"value": res[cores], "unit": "atom-steps/s", "cores": cores,
                                    "kind": "reference" if on_ref else "port",
                                    "single_thread": res[1],
                                    "sample": "one force evaluation (list + pair terms (+ RBE, water extras, "
                                              "CVFF terms)) of the same system by "
                                              + ("the reference's own worklets compiled from its source (FP32; "
                                                 "the water's intramolecular terms by the oracle)" if on_ref else
                                                 "the FP32/FP64 oracle restatement")
                                              + (", first 16 replicas" if args.workload == "batched" else "")}
    return line


def main():
    args = parse()
    if args.impl != "reference" and args.workload != "electrolyte":
        line = run_config(args)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
