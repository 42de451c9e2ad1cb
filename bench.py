#!/usr/bin/env python
"""bench.py — SNAP atom-steps/s (E+F) on B200: adjoint vs plain dB/dr path; LJ pairs/s.

Workload (default `snap_j8`): SNAP twojmax=8, two species (weights 1.0/0.5, radii
0.5/0.45, rcutfac 5.0, switching on), BCC a=3.2 A 30^3 cells = 54,000 atoms, periodic,
species 70/30 and jitter N(0, 0.12 A) from seed 4, per-species beta ~ N(0, 1e-2).
A step is one energy + forces evaluation of all atoms, neighbor build included.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is the adjoint path's atom-steps/s with inputs resident in HBM, timed with CUDA
events on the launching stream, L2 flushed (256 MiB write) before every step, max over
ranks.  `e2e` is the same metric through the host-pointer C-ABI call
(ipg_snap_energy_forces) with pinned host buffers: the H2D copy of positions/species/
beta and the D2H copy of E, W and F are inside the timed region.  The plain dB/dr path
and the pair workloads (LJ 1000 atoms, the 5-term linear combination over 32,000 atoms)
are measured in the same run and reported as extra keys.  With --gpus N > 1 (torchrun)
every rank evaluates its own copy of the workload (weak scaling, no collective in the
data path).  `--impl reference` times the reference algorithm's CPU restatement
(oracle/, OpenMP over all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "interatomicpotentials.jl_b200"))

import numpy as np  # noqa: E402

METRIC = "SNAP atom-steps/s (E+F, 1 B200): adjoint vs plain dB/dr path; LJ pairs/s"
UNIT = "atom-steps/s"
WORKLOAD = ("snap_j8: SNAP twojmax=8 (55 components), 2 species (weights 1.0/0.5, radii 0.5/0.45, "
            "rcutfac 5.0, switching on), BCC a=3.2 A 30^3 = 54,000 atoms, periodic, jitter N(0,0.12 A), "
            "adjoint-Y energy+forces (neighbor build included)")


# timing name -> kernel
PAIR_KERNEL = "tangent" if os.environ.get("IPG_PAIR_TANGENT", "0") == "1" else "lie"
KERNEL_NAMES = {"snap_atom": "k_snap_yrows", "snap_utot": "k_snap_utot_all<8>",
                "snap_pair": "k_snap_pair_adj_all<8>" if PAIR_KERNEL == "tangent" else "k_snap_pair_lie<8>"}
# DRAM bytes (read + write) per atom of one launch, from the ncu --set full captures on the
# 16,000-atom case summarised in profiles/k_snap_{yrows,pair_lie,pair_adj_all,utot_all}_snap_j8.md;
# scaled by atoms (pairs per atom are the same).
NCU_DRAM_BYTES_PER_ATOM = {"snap_atom": (51.886336e6 + 2.899200e6) / 16000,
                           "snap_pair": ((52.742144e6 + 0.953088e6) if PAIR_KERNEL == "tangent"
                                         else (50.157056e6 + 0.847360e6)) / 16000,
                           "snap_utot": (11.558912e6 + 16.316928e6) / 16000}


def _hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0  # earlier measurement on this pool


HBM_PEAK = _hbm_peak()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()  # nvidia-smi takes a while to start: let it sample before the region
            while not self.lines and time.time() - t0 < 5.0:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def oracle_sample_rate(system, prm, beta, target_s):
    """The oracle (reference algorithm, C++/OpenMP) on the first M centre atoms of the
    workload, M sized for about `target_s` seconds.  Returns (atom-steps/s, M, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    orc = oracle.Snap(prm["twojmax"], prm["radii"], prm["weight"], prm["rcutfac"], prm["rmin0"], prm["rfac0"],
                      switch=prm.get("switch_flag", False))
    sp = np.array([prm["species"].index(s) for s in system.symbols], np.int32)
    args = (system.positions, sp, system.L, beta, 0.0)
    # the neighbor build of the whole system is a fixed cost; calibrate the per-atom cost
    # from two sample sizes, then time one sample of about target_s seconds
    def run(m):
        t0 = time.perf_counter()
        orc.energy_forces(*args, mode="plain", i0=0, i1=m)
        return time.perf_counter() - t0

    t_a, t_b = run(64), run(256)
    per_atom = max((t_b - t_a) / 192.0, 1e-7)
    m = int(min(len(system), max(256, target_s / per_atom)))
    dt = run(m)
    reps = 1
    while m == len(system) and dt < target_s and reps < 30:  # the whole system is shorter: repeat it
        dt += run(m)
        reps += 1
    return m * reps / dt, m * reps, dt


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from ipg import workloads as W
    system, prm, beta = W.snap_j8()
    cores = cpu_count()
    for _ in range(args.warmup):
        oracle_sample_rate(system, prm, beta, 0.5)
    rates, ms, secs = [], 0, 0.0
    for _ in range(args.steps):
        r, m, dt = oracle_sample_rate(system, prm, beta, 3.0)
        rates.append(r)
        ms, secs = m, secs + dt
    value = float(np.median(rates))
    sample = (f"{ms} centre-atom evaluations of the 54,000-atom workload per step (the first atoms, or repeated "
              f"passes over all of them; plain dB/dr path as in compute_all_descriptors, contracted with beta), "
              f"{cores} OpenMP threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * len(system) / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": WORKLOAD, "n_atoms": len(system)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="size of the CPU-baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-path and pair-workload lines")
    ap.add_argument("--extras", default="skin,batch,plain,vjp,desc,pair,j6",
                    help="comma list of the extra measurements to run (skin, batch, plain, vjp, desc, pair)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-tune", action="store_true", help="skip the (untimed) autotuner and use the default kernel "
                    "configuration, e.g. so that a profiler's launch list holds only the measured steps")
    ap.add_argument("--cells", type=int, default=30, help="BCC cells per axis (30 -> 54,000 atoms); smaller "
                    "values give the small cases used for profiling")
    ap.add_argument("--pair-cells", type=int, default=101, help="FCC cells per axis of the scaled linear "
                    "combination (101 -> 4.12 M atoms); smaller values give the pair kernel's profiling case")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import ipg
    from ipg import flops as FL
    from ipg import workloads as W
    from ipg._lib import SNAP_ADJOINT, SNAP_PLAIN, lib

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    system, prm, beta = W.snap_j8(cells=args.cells)
    n = len(system)
    snap = ipg.SNAP(n, prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], prm["radii"],
                    prm["weight"], switch_flag=True, ctx=ipg.Context(local))
    ctx = snap.ctx
    ctx.set_stream(stream.cuda_stream)
    K = len(snap)
    nsp = len(prm["species"])
    sp_host = snap.species_ids(system)
    beta_b = snap.beta_blocks(beta)
    npairs = len(ipg.neighborlist_snap(system, snap, ctx=ctx)._j)
    # untimed: picks the kernel configuration for this workload
    tuned = {"y_entries": 0, "pair_split": 0, "utot_split": 0, "utot_warps": 4, "walk_warps": 4} if args.no_tune \
        else snap.autotune(system, beta_b)

    pos_d = torch.tensor(system.positions, device=dev)
    sp_d = torch.tensor(sp_host, device=dev)
    E_d = torch.zeros(1, dtype=torch.float64, device=dev)
    F_d = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    W_d = torch.zeros(6, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    L = system.L
    vp = C.c_void_p

    def step(mode):
        ctx.check(lib().ipg_snap_energy_forces_dev(snap.handle, n, vp(pos_d.data_ptr()), vp(sp_d.data_ptr()),
                                                   L.ctypes.data_as(vp), beta_b.ctypes.data_as(vp), 0.0, mode,
                                                   vp(E_d.data_ptr()), vp(F_d.data_ptr()), vp(W_d.data_ptr())))

    # per-kernel device timing (ipg_timing_read names); snap_zrows .. snap_gbeta are the plain,
    # descriptor and pullback kernels of the register-chain path
    TIMED_KERNELS = ("snap_atom", "snap_utot", "snap_pair", "snap_gather", "snap_contract", "neighbor", "pair_eval",
                     "snap_zrows", "snap_bdesc", "snap_dbfused", "snap_vsum", "snap_gbeta", "snap_hvp", "snap_hvp_y")

    def timed(fn, steps, kernel_timing=False):
        for _ in range(args.warmup):
            fn()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        if kernel_timing:
            ctx.timing(True)
            for k in TIMED_KERNELS:
                ctx.timing_read(k)
        l0 = ctx.launch_count()
        evs = []
        gc.collect()  # no collector pause inside the timed loop (the batch extra leaves garbage)
        gc.disable()
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        gc.enable()
        if dist:
            dist.barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        launches = ctx.launch_count() - l0
        kt = {}
        if kernel_timing:
            for k in TIMED_KERNELS:
                kt[k] = ctx.timing_read(k)
            ctx.timing(False)
        if dist:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = t.item()
        return ms, launches, kt

    with ClockSampler(local) as clk:
        ms_adj, launches, kt = timed(lambda: step(SNAP_ADJOINT), args.steps, kernel_timing=True)
    clocks = clk.summary()
    value = world * n * args.steps / (ms_adj * 1e-3)

    # e2e through the host-pointer C-ABI call, pinned host buffers
    pos_h = torch.from_numpy(system.positions.copy()).pin_memory()
    sp_h = torch.from_numpy(sp_host.copy()).pin_memory()
    F_h = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    E_h = np.zeros(1)
    W_h = np.zeros(6)

    def step_e2e():
        ctx.check(lib().ipg_snap_energy_forces(snap.handle, n, vp(pos_h.data_ptr()), vp(sp_h.data_ptr()),
                                               L.ctypes.data_as(vp), beta_b.ctypes.data_as(vp), 0.0, SNAP_ADJOINT,
                                               E_h.ctypes.data_as(vp), vp(F_h.data_ptr()), W_h.ctypes.data_as(vp)))

    ms_e2e, _, _ = timed(step_e2e, args.steps)
    e2e = {"value": world * n * args.steps / (ms_e2e * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": int(24 * n + 4 * n + 8 * nsp * K), "d2h_bytes_per_step": int(24 * n + 8 * 8)}

    # roofline: every timed SNAP kernel against the measured FP64 peak; the dominant one (largest
    # share of the step) is the headline.  Flops are algorithmic (ipg/flops.py), per launch.
    probe = C.CDLL(os.path.join(ROOT, "interatomicpotentials.jl_b200", "ipg", "libipg_probe.so"))
    probe.ipg_probe_fp64_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    tf = C.c_double()
    probe.ipg_probe_fp64_peak(local, 5, C.byref(tf), None)
    fp64_peak = tf.value
    kflops = FL.adjoint_kernels(prm["twojmax"], n, npairs, PAIR_KERNEL)
    per_kernel = {}
    for k, fl in kflops.items():
        k_ms, k_n = kt.get(k, (0.0, 0))
        if not k_n:
            continue
        avg = k_ms / k_n
        ach = fl / (avg * 1e-3) / 1e12
        per_kernel[k] = {"kernel": KERNEL_NAMES[k], "flops_per_launch": fl, "avg_launch_ms": avg,
                         "achieved_tflops": ach, "frac": ach / fp64_peak, "share_of_step": k_ms / ms_adj}
    dom = max(per_kernel, key=lambda k: per_kernel[k]["share_of_step"]) if per_kernel else None
    traffic = None
    if dom in NCU_DRAM_BYTES_PER_ATOM:
        traffic = NCU_DRAM_BYTES_PER_ATOM[dom] * n
    roofline = {"bound": "fp64", "achieved": per_kernel[dom]["achieved_tflops"] if dom else None,
                "peak": fp64_peak, "unit": "TFLOP/s", "frac": per_kernel[dom]["frac"] if dom else None,
                "traffic": traffic, "kernel": KERNEL_NAMES.get(dom), "flops_per_launch": kflops.get(dom),
                "avg_launch_ms": per_kernel[dom]["avg_launch_ms"] if dom else None,
                "peak_source": "measured DFMA probe (libipg_probe.so) in this run; the HBM peak of "
                               "MEASURED_PEAKS.json does not bound these FP64-pipe kernels",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on the "
                                  "16,000-atom case, scaled by atoms (profiles/)" if traffic else None,
                "kernels": per_kernel}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_adj / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "n_atoms": n, "n_pairs": npairs, "twojmax": prm["twojmax"],
                       "path": "adjoint", "l2": "flushed before every step (256 MiB write)",
                       "autotuned": {k: tuned[k] for k in ("y_entries", "pair_split", "utot_split", "utot_warps", "walk_warps")},
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": roofline, "clocks": clocks, "e2e": e2e, "gpu_launches": int(launches),
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kt.items() if v[1]}}

    extras = set() if args.no_extras else set(x.strip() for x in args.extras.split(",") if x.strip())
    sp_np = np.ascontiguousarray(sp_host)
    pos_np = np.ascontiguousarray(system.positions)
    if "skin" in extras:
        # MD loops: the neighbor list reused under a 0.3 A Verlet skin (positions unchanged here,
        # so every timed step takes the reuse path: re-measure + filter instead of the cell walk)
        snap.set_skin(0.3)
        ms_skin, _, kts = timed(lambda: step(SNAP_ADJOINT), args.steps, kernel_timing=True)
        snap.set_skin(0.0)
        line["adjoint_value_skin_reuse"] = world * n * args.steps / (ms_skin * 1e-3)
        line["skin_kernel_ms_per_step"] = {k: v[0] / args.steps for k, v in kts.items() if v[1]}
    if "batch" in extras:
        # Batched: 512 configurations (32..2000 atoms, crystals and liquids, ~0.54 M atoms) in one
        # evaluation, eager and as a CUDA-graph replay (ipg_snap_batch_energy_forces_dev), and one
        # force-matching training step (loss and dL/dbeta, host buffers)
        systems_b = W.batch512()
        nb_atoms = sum(len(x) for x in systems_b)
        db = ipg.DeviceBatch(snap, systems_b)
        ms_be, _, _ = timed(lambda: db.evaluate(beta_b, 0.0, graph=False), max(2, args.steps // 5))
        db.evaluate(beta_b, 0.0, graph=True)  # capture (untimed)
        ms_bg, _, _ = timed(lambda: db.evaluate(beta_b, 0.0, graph=True), max(2, args.steps // 5))
        # the plain dB/dr path on the same batch (eager: its fused dB/dr kernel sizes its chunks
        # from the exact pair count, which graph capture does not read back)
        ms_bp, _, _ = timed(lambda: db.evaluate(beta_b, 0.0, mode="plain", graph=False), max(2, args.steps // 5))
        Fref_b = np.asarray(db.F.cpu().numpy()) * 1.01
        ms_bl, _, _ = timed(lambda: snap.batch_loss_grad(systems_b, beta_b, Fref_b), 2)
        ctx.set_stream(stream.cuda_stream)
        # one force-matching training step on device buffers (E, F, loss, dL/dbeta), eager and
        # as one CUDA-graph launch (ipg_snap_batch_loss_grad_dev)
        Fref_d = torch.tensor(Fref_b, device=dev)
        nts = max(2, args.steps // 5)
        ms_te, _, _ = timed(lambda: db.train_step(beta_b, Fref_d, 0.0, graph=False), nts)
        db.train_step(beta_b, Fref_d, 0.0, graph=True)  # capture (untimed)
        l0 = ctx.launch_count()
        ms_tg, _, _ = timed(lambda: db.train_step(beta_b, Fref_d, 0.0, graph=True), nts)
        ctx.set_stream(stream.cuda_stream)
        line["batch512"] = {"n_configs": len(systems_b), "n_atoms": nb_atoms,
                            "eager_atom_steps_per_s": world * nb_atoms * max(2, args.steps // 5) / (ms_be * 1e-3),
                            "graph_atom_steps_per_s": world * nb_atoms * max(2, args.steps // 5) / (ms_bg * 1e-3),
                            "plain_eager_atom_steps_per_s": world * nb_atoms * max(2, args.steps // 5) / (ms_bp * 1e-3),
                            "adjoint_over_plain_eager": ms_bp / ms_be, "adjoint_graph_over_plain_eager": ms_bp / ms_bg,
                            "ef_graph_ms": ms_bg / max(2, args.steps // 5),
                            "loss_grad_ms": ms_bl / 2,
                            "train_step_eager_ms": ms_te / nts, "train_step_graph_ms": ms_tg / nts,
                            "train_step_graph_library_launches": (ctx.launch_count() - l0) / (nts + args.warmup)}
        del db
    if "plain" in extras:
        ms_plain, _, ktp = timed(lambda: step(SNAP_PLAIN), max(2, args.steps // 2), kernel_timing=True)
        plain_value = world * n * max(2, args.steps // 2) / (ms_plain * 1e-3)
        line["plain_value"] = plain_value
        line["adjoint_over_plain"] = value / plain_value
        line["plain_kernel_ms_per_step"] = {k: v[0] / max(2, args.steps // 2) for k, v in ktp.items() if v[1]}
    if "vjp" in extras:
        # beta pullback (force-matching gradient, ipg_snap_vjp_beta through host buffers) and the
        # local descriptors (ipg_snap_descriptors) of the same 54,000 atoms
        # through the host-pointer C-ABI calls with the caller's (pageable) numpy buffers, species
        # ids prepared once (the Python wrapper's symbol lookup is not part of the entry point)
        gF = np.random.default_rng(5).normal(size=(n, 3))
        gb_h, gb0_h = np.zeros((nsp, K)), np.zeros(1)

        def vjp_call():
            ctx.check(lib().ipg_snap_vjp_beta(snap.handle, n, pos_np.ctypes.data_as(vp), sp_np.ctypes.data_as(vp),
                                              L.ctypes.data_as(vp), 0.5, gF.ctypes.data_as(vp),
                                              gb_h.ctypes.data_as(vp), gb0_h.ctypes.data_as(vp)))
        ms_v, _, ktv = timed(vjp_call, max(2, args.steps // 5), kernel_timing=True)
        ctx.set_stream(stream.cuda_stream)
        line["vjp_beta"] = {"ms_per_call": ms_v / max(2, args.steps // 5),
                            "kernel_ms_per_call": {k: v[0] / max(2, args.steps // 5) for k, v in ktv.items() if v[1]}}
        # the full pullback with the exact position term (-gE F - H gF, ipg_snap_vjp)
        ms_p, _, ktp2 = timed(lambda: snap.vjp(system, beta_b, 0.5, gF), 2, kernel_timing=True)
        ctx.set_stream(stream.cuda_stream)
        line["vjp_positions"] = {"ms_per_call": ms_p / 2,
                                 "kernel_ms_per_call": {k: v[0] / 2 for k, v in ktp2.items() if v[1]}}
    if "desc" in extras:
        B_h = np.zeros((n, K))

        def desc_call():
            ctx.check(lib().ipg_snap_descriptors(snap.handle, n, pos_np.ctypes.data_as(vp), sp_np.ctypes.data_as(vp),
                                                 L.ctypes.data_as(vp), B_h.ctypes.data_as(vp), None, None, 1))
        ms_d, _, ktd = timed(desc_call, max(2, args.steps // 5), kernel_timing=True)
        ctx.set_stream(stream.cuda_stream)
        line["descriptors"] = {"ms_per_call": ms_d / max(2, args.steps // 5),
                               "kernel_ms_per_call": {k: v[0] / max(2, args.steps // 5) for k, v in ktd.items()
                                                      if v[1]}}
        # compute_all_descriptors (B, dB and W: the fitting inputs; dB is 142 MB at 54,000 atoms)
        dB_h = np.zeros((n, K * nsp, 3))
        Wd_h = np.zeros((K * nsp, 6))

        def desc_all_call():
            ctx.check(lib().ipg_snap_descriptors(snap.handle, n, pos_np.ctypes.data_as(vp), sp_np.ctypes.data_as(vp),
                                                 L.ctypes.data_as(vp), B_h.ctypes.data_as(vp),
                                                 dB_h.ctypes.data_as(vp), Wd_h.ctypes.data_as(vp), 7))
        nda = 2
        ms_da, _, ktda = timed(desc_all_call, nda, kernel_timing=True)
        ctx.set_stream(stream.cuda_stream)
        line["all_descriptors"] = {"ms_per_call": ms_da / nda, "dB_bytes": dB_h.nbytes,
                                   "kernel_ms_per_call": {k: v[0] / nda for k, v in ktda.items() if v[1]}}
    if "j6" in extras:
        # SNAP single species, twojmax 6, 8,192 atoms (BCC 16^3, rcut 4.7 A): plain dB/dr path (the
        # reference's route) and the adjoint path, device buffers, neighbor build included
        s6, p6, b6 = W.snap_j6()
        snap6 = ipg.SNAP(len(s6), p6["twojmax"], p6["species"], p6["rcutfac"], p6["rmin0"], p6["rfac0"], p6["radii"],
                         p6["weight"], switch_flag=True, ctx=ctx)
        n6 = len(s6)
        b6b = snap6.beta_blocks(b6)
        p6_d = torch.tensor(s6.positions, device=dev)
        sp6_d = torch.tensor(snap6.species_ids(s6), device=dev)
        F6_d = torch.zeros((n6, 3), dtype=torch.float64, device=dev)
        L6 = s6.L

        def step6(mode):
            ctx.check(lib().ipg_snap_energy_forces_dev(snap6.handle, n6, vp(p6_d.data_ptr()), vp(sp6_d.data_ptr()),
                                                       L6.ctypes.data_as(vp), b6b.ctypes.data_as(vp), 0.0, mode,
                                                       vp(E_d.data_ptr()), vp(F6_d.data_ptr()), vp(W_d.data_ptr())))
        k6 = max(2, args.steps // 2)
        ms6p, _, _ = timed(lambda: step6(SNAP_PLAIN), k6)
        ms6a, _, _ = timed(lambda: step6(SNAP_ADJOINT), k6)
        line["snap_j6"] = {"n_atoms": n6, "twojmax": 6, "plain_atom_steps_per_s": world * n6 * k6 / (ms6p * 1e-3),
                           "adjoint_atom_steps_per_s": world * n6 * k6 / (ms6a * 1e-3),
                           "plain_ms_per_step": ms6p / k6, "adjoint_ms_per_step": ms6a / k6}
        del snap6
    if "pair" in extras:
        pair = {}
        for name, (s2, p2) in (("lj1000", W.lj1000()), ("lc32000", W.lc32000()), ("lc_scaled", W.lc32000(cells=args.pair_cells))):
            pairs = ipg.api.neighbor_count(s2, p2.get_rcutoff(), ctx=ctx)
            terms = ipg.empirical.empirical_terms(p2)
            idx = {s: k for k, s in enumerate(s2.unique_symbols())}
            arr = (ipg._lib.PairTerm * len(terms))()
            for q, (c, pp) in enumerate(terms):
                arr[q] = pp.term(idx, c)
            p_d = torch.tensor(s2.positions, device=dev)
            s_d = torch.tensor(np.array([idx[s] for s in s2.symbols], np.int32), device=dev)
            f_d = torch.zeros((len(s2), 3), dtype=torch.float64, device=dev)
            L2 = s2.L

            def pstep():
                ctx.check(lib().ipg_pair_eval_dev(ctx.handle, len(s2), vp(p_d.data_ptr()), vp(s_d.data_ptr()),
                                                  L2.ctypes.data_as(vp), C.cast(arr, vp), len(terms),
                                                  vp(E_d.data_ptr()), vp(f_d.data_ptr()), vp(W_d.data_ptr()), 7))
            psteps = args.steps if len(s2) < 1_000_000 else max(2, min(args.steps, 5))
            ms_p, _, kp = timed(pstep, psteps, kernel_timing=True)
            # pairs/s counts every term's half pairs, as the reference evaluates them
            term_pairs = pairs * len(terms)
            pair[name] = {"pairs_per_s": world * term_pairs * psteps / (ms_p * 1e-3), "ms_per_step":
                          ms_p / psteps, "n_atoms": len(s2), "half_pairs": pairs, "terms": len(terms)}
            if len(s2) < 1_000_000:
                # the same step as one CUDA-graph replay (IPG_PAIR_GRAPH: an MD loop with fixed
                # buffers); the first call captures, outside the timed steps
                def pstep_graph():
                    ctx.check(lib().ipg_pair_eval_dev(ctx.handle, len(s2), vp(p_d.data_ptr()), vp(s_d.data_ptr()),
                                                      L2.ctypes.data_as(vp), C.cast(arr, vp), len(terms),
                                                      vp(E_d.data_ptr()), vp(f_d.data_ptr()), vp(W_d.data_ptr()),
                                                      7 | 8))
                pstep_graph()
                ms_g, _, _ = timed(pstep_graph, psteps)
                pair[name]["graph_pairs_per_s"] = world * term_pairs * psteps / (ms_g * 1e-3)
                pair[name]["graph_ms_per_step"] = ms_g / psteps
            if name == "lc_scaled":
                # HBM roofline of the pair path: algorithmic bytes per step = positions (24 B),
                # species (4 B) and forces (24 B) per atom; no pair list is materialised.  The
                # kernel is bound by candidate filtering and FP64 term evaluation, not by HBM.
                k_ms = kp.get("pair_eval", (0.0, 0))[0] / psteps
                nbytes = 52.0 * len(s2)
                gbps = nbytes / (k_ms * 1e-3) / 1e9 if k_ms else None
                pair[name]["hbm"] = {"algorithmic_bytes": nbytes, "kernel_ms": k_ms, "achieved_GBps": gbps,
                                     "peak_GBps": HBM_PEAK, "frac": gbps / HBM_PEAK if gbps else None,
                                     "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
                # what bounds it instead: the ncu counters of k_pair_half<3> on the 1 M-atom
                # case of the same lattice (profiles/k_pair_half_lc_1m.md)
                pair[name]["ncu_pipes"] = {"kernel": "k_pair_half<3>", "fp64_pipe_pct": 19.7, "issue_active_pct": 40.2,
                                           "dram_pct_of_peak": 1.05, "bound": "FP64 latency (wait stalls)",
                                           "source": "profiles/k_pair_half_lc_1m.md"}
        line["lj_pairs_per_s"] = pair

    if rank == 0 and world == 1 and not args.no_cpu:
        rate, m, dt = oracle_sample_rate(system, prm, beta_b, args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cpu_count(), "kind": "port",
                                "sample": f"{m} centre-atom evaluations of the {n}-atom workload (repeated "
                                          f"passes when it is shorter), plain dB/dr path, {dt:.1f} s, "
                                          f"{cpu_count()} OpenMP threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.set_stream(None)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
