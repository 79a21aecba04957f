"""Benchmark: force evaluations per second of the B200 engine at 100k atoms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 100 A periodic box of about 32,000 flexible 3-site waters plus a
400-residue synthetic chain (99,844 atoms, seeded synthetic data), cutoff
10 A, skin 2 A, LJ switch 9-10 A, Ewald tolerance 1e-5, PME grid 100^3 order
4, PHYSICAL semantics, MIXED precision (FP32 pair/spread/FFT/gather, int64
fixed-point forces, FP64 bonded/corrections/energy sums).  A step is one full
energy + force evaluation on a pairlist built before the timed region (the
build is timed separately and reported).

value      device time of K steps with inputs resident in HBM (CUDA events on
           the engine's stream around each step; L2 flushed between steps by a
           256 MiB memset outside the events)
e2e        the same evaluation through the C ABI from pinned host memory:
           mdf_submit (3N doubles in, 3N doubles out) + mdf_collect (energy
           record), two evaluations in flight so one's copies overlap the
           other's computation; wall clock of the whole loop (serial_value:
           mdf_set_positions + mdf_compute one step at a time)
roofline   the pair kernel (the dominant kernel), FP32-pipe bound: 60 FP32
           flops per atom pair inside the cutoff over its mean CUDA-event
           duration, against the measured FMA peak of the same GPU
cpu_baseline / --impl reference
           the unmodified reference (oracle/_ref/o1_harness, single-threaded
           C++) on the same system: PME chain + list energies +
           calculate_forces per step

Launch shapes come from mdf_autotune before anything is timed.  The line also
carries: fp64 (the same system in FP64, the mixed/FP64 ratio and the per-term
errors), adjoint (c2: backward / forward cost), batched (c3: 256 systems per
graph launch, device and end-to-end frames/s), dynamics (c4: L-BFGS
minimisation, NVE steps/s and energy drift, mixed and FP64, with clocks and
the host time split; PME spread/gather alone against HBM), clocks (NVML
during the timed region) and gpu_launches.

Multi-GPU (torchrun): each rank evaluates its own replica of the system (no
data-path collective: a single 100k-atom system is not sharded), timings are
max-reduced over ranks and value is the whole-job rate (weak scaling).  The
c3 batch is sharded over the ranks by estimated cost, and c4_split times one
c4 evaluation split over all ranks (x-slab PME with NCCL reduce-scatter,
all-to-all and all-gather through mdf_set_collectives; energies by
all-reduce) against one GPU.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "force evals/s at 100k atoms: mixed vs FP64 GPU at ≤1e-5 rms rel force error"
CONFIG = "c1"
GRID = (100, 100, 100)
FLOPS_PER_PAIR = 60.0


# DRAM bytes (read + write) of one k_pairs_f32 launch at c1, from one ncu
# capture of `bench.py --profile c1` (dram__bytes.sum.per_second x duration)
PAIR_TRAFFIC_BYTES = 20.0e6
# algorithmic bytes of one k_pairs_f32 launch at c1: pruned list 13.6 MB + packed
# positions/charges 1.6 + types 0.4 + fixed-point force read-modify-write 2.4
PAIR_ALGO_BYTES = 18.0e6
HBM_FALLBACK_GBS = 6650.0   # earlier copy-bandwidth measurement on B200, when no measured peak is at hand


def hbm_peak_gbs():
    """(peak GB/s, source): the measured copy bandwidth next to this script, else the fallback."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured copy bandwidth (MEASURED_PEAKS.json)"
    except (OSError, ValueError, KeyError):
        return HBM_FALLBACK_GBS, "fallback 6.65 TB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-md", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the c4 evaluation split over the ranks (N > 1)")
    ap.add_argument("--profile", metavar="CONFIG", default=None,
                    help="profiling run: build CONFIG (tiny, small, c0, c1, c4, or c3: the batch), run --warmup + --steps "
                         "evaluations, print the per-phase times and exit (for ncu)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--pair-layout", type=int, default=0, choices=[0, 1],
                    help="profiling run: pair-kernel layout (0 whole 8x8 entries, 1 half entries)")
    ap.add_argument("--pair-schedule", type=int, default=0, choices=[0, 1],
                    help="profiling run: pair-kernel schedule (0 one warp per item, 1 persistent warps)")
    return ap.parse_args()


def run_profile(args):
    """Plain evaluation loop for profilers: no timing bookkeeping of our own.
    c3 runs the 256-system batch (one graph launch per evaluation)."""
    import torch
    from md_b200 import abi, engine, synth, topology
    if args.profile == "c3":
        members = make_batch_workload(range(256))
        ss = [m[0] for m in members]
        b = engine.Batch([m[1] for m in members], [x.box for x in ss], [x.meta["grid"] for x in ss],
                         precision=abi.MDF_PREC_MIXED, cutoff=9.0, skin=2.0, switch_radius=8.0, ewald_tol=1e-5,
                         pair_layout=args.pair_layout, pair_schedule=args.pair_schedule)
        b.set_positions([x.coords for x in ss])
        for _ in range(args.warmup + args.steps):
            b.compute(energy=True, forces=True)
        print(json.dumps({"profile": "c3", "systems": len(ss), "info": b.info()}))
        b.close()
        return
    s = synth.make_config(args.profile)
    flat = topology.flatten(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    prec = abi.MDF_PREC_MIXED if args.precision == "mixed" else abi.MDF_PREC_FP64
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=prec, ewald_tol=1e-5,
                        grid=synth.GRIDS[args.profile], pair_layout=args.pair_layout,
                        pair_schedule=args.pair_schedule)
    eng.set_positions(s.coords)
    eng.build_pairlist()
    for _ in range(args.warmup + args.steps):
        eng.compute_async(energy=True)
        eng.fetch(forces=False)
    eng.enable_timing(True)
    eng.compute()
    print(json.dumps({"profile": args.profile, "natoms": s.natoms, "precision": args.precision,
                      "pair_layout": args.pair_layout, "pair_schedule": args.pair_schedule,
                      "pairlist": eng.pairlist_info(), "phase_ms": dict(eng.kernel_times())}))
    eng.close()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """SM clock, power and clock-event reasons sampled during the timed region:
    NVML every 2 ms in a thread (read-only queries; the c1 region lasts
    ~10 ms), else nvidia-smi every 200 ms."""

    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []
        self.stop = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()

            def run():
                while not self.stop.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        pass
                    self.stop.wait(0.002)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.stop = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.stop is not None:
            self.stop.set()
            self.t.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.samples:
            sm = [c for c, _ in self.samples]
            reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS.items() if r & bit})
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "NVML, 2 ms"}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_workload():
    from md_b200 import abi, engine, synth, topology
    s = synth.make_config(CONFIG)
    flat = topology.flatten(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    return s, flat


def o1_files(s):
    from md_b200 import synth
    d = tempfile.mkdtemp(prefix="mdf_bench_")
    return synth.write_files(s, d, stem=CONFIG)


def reference_time(s, steps, warmup=1):
    from oracle import oracle as O
    prm, rst = o1_files(s)
    r = O.bench_o1(prm, rst, GRID, steps, warmup=warmup, tol=1e-5)
    return r


def run_reference_arm(args, rank):
    """The unmodified reference on the same c1 system: only the seeded
    generator and its prmtop/rst7 writer run in this process (no libmdf), the
    timed work is oracle/_ref/o1_harness in a subprocess, exactly --steps
    evaluations after --warmup untimed ones (about 4.5 s each on one core)."""
    if rank != 0:
        return
    import platform
    from md_b200 import synth
    s = synth.make_config(CONFIG)
    k = max(1, args.steps)
    w = max(0, args.warmup)
    r = reference_time(s, k, warmup=w)
    v = 1.0 / r["s_per_step"]
    sample = ("%d full reference evaluations of the %d-atom system (PME chain at 100^3 + list energies + "
              "calculate_forces; pairlist built once; O(N^2) calculate_EE_energy left out)" % (k, s.natoms))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": args.gpus,
            "steps": k, "warmup": w, "ms_per_step": r["s_per_step"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "c1: 100 A box, %d atoms, PME 100^3" % s.natoms, "semantics": "reference as-is",
                       "cpu": platform.processor() or platform.machine()},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_breakdown_s": {k2: r[k2] for k2 in ("s_pme_chain", "s_list_energies", "s_calculate_forces",
                                                          "s_pairlist")}}
    print(json.dumps(line), flush=True)


def adjoint_cost(dev, reps=10):
    """c2 workload: the c0 system (28,227 atoms, PME 72^3), loss = mean |F - F_t|^2
    + 1e-3 E_total.  Wall time of one forward evaluation (mdf_compute, energies
    and forces to host) against one mdf_backward (dL/dq, dL/dA, dL/dB to host),
    both synchronous calls through the C ABI, FP64 and mixed."""
    from md_b200 import abi, engine, synth, topology
    s = synth.make_config("c0")
    flat = topology.flatten(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    out = {"workload": "c2: c0 system, %d atoms, %d charges + 2 x %d LJ coefficients" % (
        s.natoms, s.natoms, len(flat.lj_a))}
    for name, prec in (("fp64", abi.MDF_PREC_FP64), ("mixed", abi.MDF_PREC_MIXED)):
        eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=prec, ewald_tol=1e-5,
                            grid=synth.GRIDS["c0"], device=dev)
        eng.set_positions(s.coords)
        eng.build_pairlist()
        E, F = eng.compute()
        Ft = F + np.random.default_rng(5).normal(0.0, 0.5, F.shape)
        gF, gE = 2.0 * (F - Ft) / F.shape[0], 1e-3
        for _ in range(3):
            eng.compute()
            eng.backward(gF, gE)
        tf = tb = 0.0
        for _ in range(reps):
            a = time.perf_counter()
            eng.compute()
            tf += time.perf_counter() - a
            a = time.perf_counter()
            eng.backward(gF, gE)
            tb += time.perf_counter() - a
        eng.close()
        out[name] = {"forward_ms": tf / reps * 1e3, "backward_ms": tb / reps * 1e3, "backward_over_forward": tb / tf}
    return out


def cufft_check(eng, dev, s, ours_ms, reps=20):
    """cuFFT (torch.fft on the GPU), timed beside the hand-written chain as a
    check: N * irfftn(c(m) * rfftn(Q)) on the engine's own FP32 charge grid of
    the last evaluation, against the potential grid the engine gathered from.
    Time: rfftn + influence multiply + irfftn per evaluation (CUDA events,
    L2-resident grid), against the engine's measured z/y/x+convolution/y/z
    phase."""
    import math
    import torch
    Q, P = eng.pme_grids()
    K = Q.shape
    box = s.box
    V = box[0] * box[1] * box[2]
    alpha = math.sqrt(-math.log(2e-5)) / 10.0

    def bmod(n):
        def card(o, x):
            if x <= 0 or x >= o:
                return 0.0
            if o == 2:
                return 1.0 - abs(x - 1.0)
            return (x * card(o - 1, x) + (o - x) * card(o - 1, x - 1.0)) / (o - 1)
        b = np.zeros(n)
        for m in range(n):
            sr = sum(card(4, k + 1.0) * math.cos(2 * math.pi * m * k / n) for k in range(3))
            si = sum(card(4, k + 1.0) * math.sin(2 * math.pi * m * k / n) for k in range(3))
            b[m] = sr * sr + si * si
        for m in range(n):
            if b[m] < 1e-7:
                b[m] = 0.5 * (b[(m - 1) % n] + b[(m + 1) % n])
        return 1.0 / b
    mx = np.fft.fftfreq(K[0], 1.0 / K[0]) / box[0]
    my = np.fft.fftfreq(K[1], 1.0 / K[1]) / box[1]
    mz = np.arange(K[2] // 2 + 1) / box[2]
    MX, MY, MZ = np.meshgrid(mx, my, mz, indexing="ij")
    m2 = MX ** 2 + MY ** 2 + MZ ** 2
    m2[0, 0, 0] = 1.0
    from md_b200 import synth
    c = (float(synth.KC) / (math.pi * V)) * np.exp(-math.pi ** 2 * m2 / alpha ** 2) / m2
    c = c * bmod(K[0])[:, None, None] * bmod(K[1])[None, :, None] * bmod(K[2])[None, None, :K[2] // 2 + 1]
    c[0, 0, 0] = 0.0
    q = torch.tensor(Q, dtype=torch.float32, device=dev)
    ct = torch.tensor(c, dtype=torch.float32, device=dev)
    run = lambda: torch.fft.irfftn(torch.fft.rfftn(q) * ct, s=K)
    for _ in range(3):
        run()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        out = run()
    b.record()
    torch.cuda.synchronize(dev)
    ref = out.cpu().numpy().astype(np.float64) * (K[0] * K[1] * K[2])
    return {"grid": list(K), "ours_ms": ours_ms, "cufft_ms": a.elapsed_time(b) / reps,
            "rel_l2_diff": float(np.linalg.norm(P - ref) / np.linalg.norm(ref))}


def split_bench(dev, ws, rank, cfg="c4", steps=20, warmup=3):
    """c4 (960k atoms, PME 216^3; `cfg` another named workload) evaluated by all ranks together: each rank
    takes the pair and PME spread/gather work of its band of space (and its
    share of the bonded lists), the reciprocal space is distributed as x-slabs
    of the grid whose charge and potential planes cross between neighbouring
    bands as halos, and the forces come back by reduce-scatter + all-gather
    (mdf_params.rank / nranks, mdf_set_allreduce + mdf_set_collectives +
    mdf_set_halo_exchange, NCCL).  Time: CUDA events on each rank's stream
    around `steps` evaluations, max over ranks.  Rank 0 also times one context
    doing the whole evaluation, for the speed-up."""
    import torch
    import torch.distributed as dist
    from md_b200 import abi, distributed, engine, synth, topology
    s = synth.make_config(cfg)
    flat = topology.flatten(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    kw = dict(semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED, ewald_tol=1e-5,
              grid=synth.GRIDS[cfg], device=dev)
    stream = torch.cuda.Stream(device=dev)

    def timed(eng, collective):
        eng.set_stream(stream.cuda_stream)
        eng.set_positions(s.coords)
        eng.build_pairlist()
        for _ in range(warmup):
            eng.compute_async(energy=True)
            eng.fetch(forces=False)
        if collective:
            dist.barrier()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            eng.compute_async(energy=True)
            eng.fetch(forces=False)
        b.record(stream)
        torch.cuda.synchronize(dev)
        t = a.elapsed_time(b) / 1e3
        if collective:
            tt = torch.tensor([t], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    eng = engine.Engine(flat, s.box, rank=rank, nranks=ws, **kw)
    eng.set_allreduce(distributed.torch_allreduce())
    eng.set_collectives(*distributed.torch_collectives())
    eng.set_halo_exchange(distributed.torch_alltoallv())
    t_split = timed(eng, True)
    eng.close()
    out = {"workload": "%s: %d atoms, PME %s, cutoff 10 A, mixed precision; one evaluation split over %d ranks "
                       "(bands of space; x-slab PME: halo planes of the charge grid to their owners, all-to-all "
                       "transposes around the x pass, halo planes of the potential back; forces by reduce-scatter "
                       "+ all-gather; energies all-reduced)"
                       % (cfg, s.natoms, "x".join(map(str, synth.GRIDS[cfg])), ws),
           "n_ranks": ws, "evals_per_s": steps / t_split, "ms_per_eval": t_split / steps * 1e3}
    if rank == 0:
        one = engine.Engine(flat, s.box, **kw)
        t_one = timed(one, False)
        one.close()
        out["one_gpu_evals_per_s"] = steps / t_one
        out["speedup"] = t_one / t_split
    dist.barrier()
    return out


def md_bench(dev, steps=1000, equil=200):
    """c4: 215 A box of 320,000 flexible waters (960,000 atoms), PME 216^3,
    cutoff 10 A + 2 A skin, velocity-Verlet NVE at 0.5 fs from 300 K Maxwell
    velocities (seeded), pairlist rebuilt every 10 steps.  The lattice start is
    first relaxed by the L-BFGS minimiser (the same positions feed both
    precisions), then `equil` steps are run before the measured `steps`.  The
    PME spread and gather of this workload are timed alone (phase events) and
    set against HBM with their algorithmic bytes: spread 16 B/atom + 8 B K^3
    grid write + 8 B K^3 clear, gather 16 B/atom + 4 B K^3 potential read +
    24 B/atom force read-modify-write.
    Steps/s is the host wall time of mdf_md_run (graph chunks of 10 steps,
    list rebuilds and the per-chunk energy read-back included); the energy
    drift is last minus first sample of the total energy over the measured
    steps, mixed against FP64 from the same start.  The pair lists prune
    themselves on the device (prune_every < 0, 0.2 A margin: the prune kernel
    runs when an atom moved more than 0.1 A since the last prune)."""
    from md_b200 import abi, engine, synth, topology
    s = synth.make_config("c4")
    flat = topology.flatten(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    kw = dict(semantics=abi.MDF_SEM_PHYSICAL, ewald_tol=1e-5, grid=synth.GRIDS["c4"], device=dev,
              prune_every=-1, prune_margin=0.2)
    eng = engine.Engine(flat, s.box, precision=abi.MDF_PREC_MIXED, **kw)
    eng.set_positions(s.coords)
    eng.build_pairlist()
    t0 = time.perf_counter()
    mrep = eng.minimize(max_iter=300, fmax_tol=10.0, method="lbfgs")
    mrep["method"] = "L-BFGS, 8 pairs"
    mrep["wall_s"] = time.perf_counter() - t0
    x0, _ = eng.md_state(velocities=False)
    # spread / gather alone at c4 (timing mode: one stream, phase events)
    eng.enable_timing(True)
    ph = {}
    for _ in range(6):
        eng.compute()
        for name, ms in eng.kernel_times():
            ph.setdefault(name, []).append(ms)
    eng.enable_timing(False)
    K3 = float(np.prod(synth.GRIDS["c4"]))
    sp_ms, ga_ms = float(np.median(ph["pme_spread"][1:])), float(np.median(ph["pme_gather"][1:]))
    sp_b, ga_b = 16.0 * s.natoms + 16.0 * K3, 40.0 * s.natoms + 4.0 * K3
    hbm, hbm_src = hbm_peak_gbs()
    pme = {"spread_ms": sp_ms, "gather_ms": ga_ms,
           "spread_gbs": sp_b / (sp_ms * 1e-3) / 1e9, "gather_gbs": ga_b / (ga_ms * 1e-3) / 1e9,
           "hbm_peak_gbs": hbm, "peak_source": hbm_src}
    pme["spread_hbm_frac"] = pme["spread_gbs"] / hbm
    pme["gather_hbm_frac"] = pme["gather_gbs"] / hbm
    # the grid stays in L2: the spread's roofline is the L2 int64 reduction
    # rate, measured on this GPU on a buffer of the same size (the larger of
    # the spread's own 32-byte-row pattern and 256-byte warp runs)
    nq = int(np.count_nonzero(flat.charge))
    red_rows = engine.probe_l2_reductions(dev, int(K3), 0)
    red_runs = engine.probe_l2_reductions(dev, int(K3), 1)
    l2_peak = max(red_rows, red_runs)
    pme["spread_reductions_per_s"] = 64.0 * nq / (sp_ms * 1e-3)
    pme["l2_reduction_peak_per_s"] = l2_peak
    pme["l2_reduction_probe"] = {"rows_32B": red_rows, "warp_runs_256B": red_runs,
                                 "buffer_words": int(K3), "source": "mdf_probe_l2_reductions"}
    pme["spread_l2_frac"] = pme["spread_reductions_per_s"] / l2_peak
    pme["note"] = ("the 80 MB int64 grid stays in L2: the spread (16 lanes per atom, 64 int64 reductions per "
                   "charged atom) is bound by L2 reduction throughput, spread_l2_frac is against the measured "
                   "L2 reduction peak; the gather by L1/L2 latency of its 64 loads per atom")
    out = {"workload": "c4: %d atoms (320,000 flexible waters), 215 A box, PME 216^3, cutoff 10 A, skin 2 A, "
                       "dt 0.5 fs, NVE, list rebuilt every 10 steps and pruned on the device when an atom moved "
                       "0.1 A, %d measured steps after %d equilibration steps" % (s.natoms, steps, equil),
           "minimiser": mrep, "pme_spread_gather": pme}
    for name, prec in (("mixed", abi.MDF_PREC_MIXED), ("fp64", abi.MDF_PREC_FP64)):
        if prec != abi.MDF_PREC_MIXED:
            eng.close()
            eng = engine.Engine(flat, s.box, precision=prec, **kw)
            eng.set_positions(x0)
            eng.build_pairlist()
        tune = eng.autotune(reps=3)   # launch shapes for this system (outside the timed region)
        eng.md_init(s.mass, temperature=300.0, seed=1234)
        eng.md_run(equil, 0.0005, chunk=10, rebuild_every=10)
        with ClockSampler(dev) as clk:
            rep, samp = eng.md_run(steps, 0.0005, chunk=10, rebuild_every=10)
        tot = samp[:, 1] + samp[:, 2]
        ke = float(samp[:, 2].mean())
        out[name] = {"steps_per_s": rep["steps"] / rep["wall_s"], "ms_per_step": rep["wall_s"] / rep["steps"] * 1e3,
                     "rebuilds": rep["rebuilds"], "e_total_first": float(tot[0]), "e_total_last": float(tot[-1]),
                     "drift": float(tot[-1] - tot[0]), "drift_over_ke": float((tot[-1] - tot[0]) / ke),
                     "e_total_std": float(tot.std()), "mean_ke": ke,
                     "temperature_k": 2.0 * ke / (3.0 * s.natoms * 0.0019872041), "clocks": clk.summary(),
                     "host_s": {"rebuild": rep["rebuild_s"], "graph_record": rep["record_s"],
                                "graph_wait": rep["wait_s"], "total": rep["wall_s"]},
                     "launch_shapes": tune}
    eng.close()
    out["mixed_over_fp64_speed"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    return out


def _batch_member(k):
    from md_b200 import abi, engine, synth, topology
    sysm = synth.make_batch_member(k)
    flat = topology.flatten(sysm, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    return sysm, flat


def batch_share(rank, ws, n=256):
    """This rank's systems of the c3 batch: a cost-balanced greedy partition
    (md_b200.shard), the same on every rank."""
    from md_b200 import shard, synth
    costs = []
    for L, nres in synth._batch_dims(n, 1003):
        nat = 3 * max(10, int(0.1 * L ** 3 / 3.0) - nres * 10 // 3) + 10 * nres
        g = synth.smooth_grid_size(L, 1.0)
        costs.append(shard.system_cost(nat, (g, g, g)))
    return shard.partition(costs, ws)[rank]


def make_batch_workload(indices):
    """The given systems of c3's 256, generated in spawned worker processes."""
    import concurrent.futures as cf
    import multiprocessing as mp
    with cf.ProcessPoolExecutor(max_workers=min(8, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_batch_member, list(indices)))


def batch_bench(dev, members, stream, steps=20):
    """c3: 256 uneven systems (25-40 A boxes, 1.5k-6k atoms, PME 24^3-40^3,
    cutoff 9 A), mixed precision, one CUDA graph launch per batch evaluation,
    launch shapes autotuned.  Device time per graph launch (CUDA events on the
    stream the graph is ordered on; the graph includes the host<->device copies
    of all positions and forces through pinned buffers) and the wall time of
    set_positions + compute through the C ABI, the positions sitting in the
    batch's pinned host buffer and the forces read from its pinned force
    buffer (mdf_batch_host_buffers: no extra host copy)."""
    import torch
    from md_b200 import abi, engine
    ss = [m[0] for m in members]
    flats = [m[1] for m in members]
    b = engine.Batch(flats, [x.box for x in ss], [x.meta["grid"] for x in ss], precision=abi.MDF_PREC_MIXED,
                     cutoff=9.0, skin=2.0, switch_radius=8.0, ewald_tol=1e-5, device=dev)
    b.set_positions([x.coords for x in ss])
    t0 = time.perf_counter()
    b.build_pairlists()
    t_build = time.perf_counter() - t0
    tune = b.autotune(reps=3)
    for _ in range(3):
        b.launch(stream_ptr=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        ev[k][0].record(stream)
        b.launch(stream_ptr=stream.cuda_stream)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    ms = float(np.mean([a.elapsed_time(c) for a, c in ev]))
    pos_h, _ = b.host_buffers()
    pos_h[:] = np.concatenate([x.coords for x in ss])
    e2e_t = 0.0
    for _ in range(max(5, steps // 2)):
        a = time.perf_counter()
        b.set_positions(pos_h)
        b.compute(energy=True, forces=True, copy_forces=False)
        e2e_t += time.perf_counter() - a
    serial_ms = e2e_t / max(5, steps // 2) * 1e3
    # pipelined (mdf_batch_submit / mdf_batch_collect): two batches in flight,
    # positions in and forces out through pinned buffers on their own copy
    # streams while the GPU computes; wall clock of the whole loop
    xin = [torch.from_numpy(pos_h.copy()).pin_memory() for _ in range(2)]
    fout = [torch.empty(pos_h.size, dtype=torch.float64).pin_memory() for _ in range(2)]
    for k in range(4):
        b.submit(xin[k % 2].data_ptr(), fout[k % 2].data_ptr())
        if k >= 1:
            b.collect()
    b.collect()
    n_pipe = max(20, steps)
    a = time.perf_counter()
    for k in range(n_pipe):
        b.submit(xin[k % 2].data_ptr(), fout[k % 2].data_ptr())
        if k >= 1:
            b.collect()
    b.collect()
    e2e_ms = (time.perf_counter() - a) / n_pipe * 1e3
    info = b.info()
    natoms = [x.natoms for x in ss]
    b.close()
    return {"workload": "c3: %d systems, %d-%d atoms (%d total), boxes 25-40 A, PME 24^3-40^3, cutoff 9 A, "
                        "mixed precision, one CUDA graph launch per evaluation" % (len(ss), min(natoms),
                                                                                   max(natoms), sum(natoms)),
            "frames_per_s": len(ss) / (ms * 1e-3), "ms_per_batch": ms,
            "e2e_frames_per_s": len(ss) / (e2e_ms * 1e-3), "e2e_ms_per_batch": e2e_ms,
            "e2e_api": "mdf_batch_submit / mdf_batch_collect, two batches in flight, pinned host buffers",
            "e2e_serial_frames_per_s": len(ss) / (serial_ms * 1e-3), "e2e_serial_ms_per_batch": serial_ms,
            "atoms_per_s": sum(natoms) / (ms * 1e-3), "graph_kernels": info["graph_kernels"],
            "pairlist_build_s": t_build, "autotune": tune}


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    if args.profile:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    batch_members = None
    if not args.no_batch:
        batch_members = make_batch_workload(batch_share(rank, ws))
    import torch
    import torch.distributed as dist
    from md_b200 import abi, engine
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = local
    torch.cuda.set_device(dev)

    s, flat = build_workload()
    stream = torch.cuda.Stream(device=dev)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED, ewald_tol=1e-5,
                        grid=GRID, device=dev)
    eng.set_stream(stream.cuda_stream)
    eng.set_positions(s.coords)
    t0 = time.perf_counter()
    eng.build_pairlist()
    torch.cuda.synchronize(dev)
    t_build = time.perf_counter() - t0
    # list rebuilds at the same positions (buffers already sized): host wall
    # time of mdf_build_pairlist, which returns after the build's one
    # synchronisation
    t_rebuild = []
    for _ in range(10):
        a = time.perf_counter()
        eng.build_pairlist()
        t_rebuild.append(time.perf_counter() - a)
    t_rebuild = float(np.median(t_rebuild))
    tune = eng.autotune(reps=5)   # launch shapes for this workload (outside every timed region)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # per-kernel times: a separate pass with the engine's phase events on (that
    # mode runs every kernel on one stream so the phases can be told apart)
    eng.enable_timing(True)
    ktimes = {}
    for k in range(max(3, args.warmup) + 20):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.compute_async(energy=True)
        eng.fetch(forces=False)
        if k >= max(3, args.warmup):
            for name, ms in eng.kernel_times():
                ktimes.setdefault(name, []).append(ms)
    eng.enable_timing(False)

    # warm-up
    for _ in range(max(3, args.warmup)):
        eng.compute_async(energy=True)
        eng.fetch(forces=False)

    # timed region: per-step CUDA events on the engine stream, L2 flushed in between
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = eng.launches()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev[k][0].record(stream)
            eng.compute_async(energy=True)
            ev[k][1].record(stream)
            eng.fetch(forces=False)
        torch.cuda.synchronize(dev)
    launches = eng.launches() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_total = sum(step_ms) / 1e3
    if ws > 1:
        tt = torch.tensor([t_total], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total = float(tt.item())
    value = ws * args.steps / t_total
    info = eng.pairlist_info()
    pair_ms = float(np.mean(ktimes.get("pairs", [float("nan")])))

    # e2e through the C ABI from pinned host buffers: every step copies its
    # positions in and its forces out.  Pipelined (mdf_submit / mdf_collect,
    # two evaluations in flight: the copies of one overlap the computation of
    # the other); the 256 MiB L2 flush runs on the evaluation stream before
    # each evaluation, inside the timed loop.
    pos_h = [torch.from_numpy(np.ascontiguousarray(s.coords.reshape(-1))).pin_memory() for _ in range(2)]
    f_hs = [torch.empty(3 * s.natoms, dtype=torch.float64).pin_memory() for _ in range(2)]
    f_h = f_hs[0]
    for _ in range(3):
        eng.set_positions_ptr(pos_h[0].data_ptr())
        eng.compute_into(f_h.data_ptr())
    e2e_steps = max(50, args.steps)
    # warm-up of the pipelined path: its first submit creates the copy streams,
    # the stage buffers and events
    for k in range(max(3, args.warmup)):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.submit(pos_h[k % 2].data_ptr(), f_hs[k % 2].data_ptr())
        if k >= 1:
            eng.collect()
    eng.collect()
    torch.cuda.synchronize(dev)
    # three timed loops, the median kept (host wall clock on a shared machine)
    e2e_loops = []
    for _ in range(3):
        a = time.perf_counter()
        for k in range(e2e_steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            eng.submit(pos_h[k % 2].data_ptr(), f_hs[k % 2].data_ptr())
            if k >= 1:
                eng.collect()
        eng.collect()
        e2e_loops.append(time.perf_counter() - a)
    e2e_t = float(np.median(e2e_loops))
    # the same calls without overlap: copy in, evaluate, copy out, one step at a time
    e2e_serial_t = 0.0
    for _ in range(e2e_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        stream.synchronize()
        a = time.perf_counter()
        eng.set_positions_ptr(pos_h[0].data_ptr())
        eng.compute_into(f_h.data_ptr())
        e2e_serial_t += time.perf_counter() - a
    if ws > 1:
        tt = torch.tensor([e2e_t, e2e_serial_t], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_t, e2e_serial_t = float(tt[0].item()), float(tt[1].item())
    e2e = ws * e2e_steps / e2e_t
    e2e_serial = ws * e2e_steps / e2e_serial_t
    F_mixed = f_h.numpy().reshape(-1, 3).copy()

    # FP64 path on the same system (the metric's comparison), and its force error
    fp64 = None
    if not args.no_fp64:
        eng64 = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_FP64,
                              ewald_tol=1e-5, grid=GRID, device=dev)
        eng64.set_stream(stream.cuda_stream)
        eng64.set_positions(s.coords)
        eng64.build_pairlist()
        tune64 = eng64.autotune(reps=3)
        for _ in range(3):
            eng64.compute_async(energy=True)
            eng64.fetch(forces=False)
        n64 = max(10, args.steps // 4)
        ev64 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n64)]
        for k in range(n64):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev64[k][0].record(stream)
            eng64.compute_async(energy=True)
            ev64[k][1].record(stream)
            eng64.fetch(forces=False)
        torch.cuda.synchronize(dev)
        t64 = sum(a.elapsed_time(b) for a, b in ev64) / 1e3 / n64
        E64, F64 = eng64.compute()
        Emx, _ = eng.compute()
        err = float(np.linalg.norm(F_mixed - F64) / np.linalg.norm(F64))
        terms = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "vdw14", "ee_direct", "ee14",
                 "ee_excl", "ee_self", "ee_recip", "total"]
        term_err = {k: (abs(Emx[k] - E64[k]) / abs(E64[k]) if E64[k] != 0 else abs(Emx[k])) for k in terms}
        fp64 = {"ms_per_step": t64 * 1e3, "value": 1.0 / t64, "mixed_over_fp64": (t_total / args.steps) ** -1 * t64,
                "rms_rel_force_err_mixed_vs_fp64": err, "energy_rel_err_mixed_vs_fp64": term_err,
                "launch_shapes": tune64}
        eng64.close()

    peak = engine.probe_fma_tflops(dev, abi.MDF_PREC_MIXED)
    achieved = FLOPS_PER_PAIR * info["pairs_in_cutoff"] / (pair_ms * 1e-3) / 1e12
    hbm_gbs, hbm_src = hbm_peak_gbs()
    kernel_ms = {k: float(np.mean(v)) for k, v in ktimes.items()}
    fft_check = cufft_check(eng, dev, s, kernel_ms.get("pme_fft_conv"))

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            r = reference_time(s, 1, warmup=0)
            cpu = {"value": 1.0 / r["s_per_step"], "unit": "evals/s", "cores": 1, "kind": "reference",
                   "sample": "one full evaluation of the same %d-atom system by the unmodified reference "
                             "(PME chain + list energies + calculate_forces, single-threaded; pairlist "
                             "built once, O(N^2) calculate_EE_energy left out)" % s.natoms,
                   "breakdown_s": {k2: r[k2] for k2 in ("s_pme_chain", "s_list_energies", "s_calculate_forces",
                                                        "s_pairlist")}}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "evals/s", "cores": 1, "kind": "reference", "sample": "failed: %s" % e}

    adj = None
    if rank == 0 and ws == 1 and not args.no_adjoint:
        adj = adjoint_cost(dev)
    batched = None
    if batch_members is not None:
        batched = batch_bench(dev, batch_members, stream)
        if ws > 1:
            # systems are independent: each rank ran its share; the batch time is the slowest rank's
            from md_b200 import shard
            ms = shard.max_over_ranks(batched["ms_per_batch"], device=dev)
            e2e_ms = shard.max_over_ranks(batched["e2e_ms_per_batch"], device=dev)
            batched.update({"workload": "c3: 256 systems sharded over %d GPUs by estimated cost (this line: "
                                        "all ranks, slowest rank's time)" % ws,
                            "ms_per_batch": ms, "frames_per_s": 256 / (ms * 1e-3),
                            "e2e_ms_per_batch": e2e_ms, "e2e_frames_per_s": 256 / (e2e_ms * 1e-3)})
    dynamics = None
    if rank == 0 and ws == 1 and not args.no_md:
        dynamics = md_bench(dev)
    split = None
    if ws > 1 and not args.no_split:
        split = split_bench(dev, ws, rank)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": ws, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": t_total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c1: 100 A cubic box, %d atoms (31,948 flexible waters + 400-residue chain), "
                                   "cutoff 10 A, skin 2 A, LJ switch 9 A, Ewald tol 1e-5, PME 100^3 order 4, "
                                   "PHYSICAL semantics, mixed precision" % s.natoms,
                       "parallelism": "replicas x%d" % ws if ws > 1 else "single GPU",
                       "l2": "flushed between steps (256 MiB memset outside the per-step events)",
                       "pairlist_build_ms": t_rebuild * 1e3, "pairlist_first_build_ms": t_build * 1e3,
                       "clusters": info["clusters"],
                       "cluster_pairs": info["cluster_pairs"],
                       "cluster_pairs_pruned": info["cluster_pairs_pruned"],
                       "prune": ("every evaluation, exact (margin 0)" if tune["prune_every"] == 1
                                 else "off (the pair kernel walks the rc + skin list)"),
                       "launch_shapes": tune,
                       "pairs_in_cutoff": info["pairs_in_cutoff"]},
            "roofline": {"kernel": "k_pairs (LJ + erfc Ewald pair kernel)", "bound": "fp32", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": PAIR_TRAFFIC_BYTES,
                         "traffic_source": "dram__bytes read+write per launch, one ncu capture of the same "
                                           "workload (bench.py --profile c1); algorithmic ~18 MB",
                         "peak_source": "measured FP32 FMA throughput of this GPU (mdf_probe_fma_tflops)",
                         "work": "%g FP32 flops x %d pairs in cutoff per launch" % (FLOPS_PER_PAIR,
                                                                                  info["pairs_in_cutoff"]),
                         "hbm_view": {"achieved": PAIR_ALGO_BYTES / (pair_ms * 1e-3) / 1e9, "peak": hbm_gbs,
                                      "unit": "GB/s", "frac": PAIR_ALGO_BYTES / (pair_ms * 1e-3) / 1e9 / hbm_gbs,
                                      "peak_source": hbm_src,
                                      "note": "the pair kernel is FP32-issue bound, not HBM bound"}},
            "evals_per_s_amortised_10": 1.0 / (t_total / args.steps + t_rebuild / 10.0),
            "kernel_ms": kernel_ms,
            "fft_vs_cufft": fft_check,
            "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": 3 * s.natoms * 8,
                    "d2h_bytes_per_step": 3 * s.natoms * 8 + 26 * 8,
                    "api": "mdf_submit / mdf_collect, two evaluations in flight, positions and forces through "
                           "pinned host buffers, L2 flushed before each evaluation inside the timed loop; median "
                           "of three loops of %d steps" % e2e_steps,
                    "loops_evals_per_s": [ws * e2e_steps / t for t in e2e_loops],
                    "serial_value": e2e_serial,
                    "serial_api": "mdf_set_positions + mdf_compute per step (no overlap), flush outside the timing"},
            "fp64": fp64,
            "adjoint": adj,
            "batched": batched,
            "dynamics": dynamics,
            "c4_split": split,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
