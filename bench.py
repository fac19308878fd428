#!/usr/bin/env python
"""Benchmark: zone-updates/s per RK2 step of the B200 Godunov MHD update.

Workload: 3-D ideal MHD on a uniform 128^3 grid of 512 blocks of 16^3 cells
(2 ghost zones), gamma = 5/3, seeded Fourier-mode initial data (32 modes,
|k|_inf <= 4; rho amplitude 0.1, v amplitude 0.1, A amplitude 0.05), MC + HLLD
+ CT, RK2, FP64 -- synthetic data generated on the host by
fornaxamr_b200.problems.

One step = one pass of the driver loop: calc_dt, dt limiting, both RK2
stages with ghost fills, dt_src clamp.  `value` is device time (CUDA events on
the library's stream, state resident in HBM) for the batched form (every
phase swept over all blocks, whole step replayed as one CUDA graph).  The
working set (~2.7 GB) is far larger than L2, so no explicit flush is needed.
`e2e` is the same metric through the C ABI with host buffers: each step
uploads the state (W and Bf, stage slot 0) from pinned host memory, steps,
and downloads it again.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--shard]
For N > 1 (torchrun) every rank runs an independent replica by default
(`value` is the sum); with --shard the ranks share one mesh of N x 512 blocks
(a 128^3 cube per GPU), exchanging ghost zones and dt minima over NCCL inside
each step's CUDA graph (weak scaling with the exchanges).
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "zone-updates/s per RK2 step"
UNIT = "zone-updates/s"
ROOT = 8                          # 8^3 blocks of 16^3 = 128^3
ZONES = ROOT ** 3 * 16 ** 3
BYTES_PER_ZONE_STEP = 360.0       # compulsory state traffic per zone per RK2 step (9 vars x 8 B x 5)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fx", choices=["fx", "reference"])
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--amr-interval", type=int, default=10,
                    help="steps between adapts of the dynamic-AMR key")
    ap.add_argument("--amr-dynamic-adapts", type=int, default=2,
                    help="adapts in the dynamic-AMR key (0: skip it)")
    ap.add_argument("--no-variants", dest="variants", action="store_false",
                    help="skip the WENO-Z3 / eSSPRK10_4 variant measurements")
    ap.add_argument("--ref-adapt", action="store_true",
                    help="also time the reference's adapt on the dynamic-AMR mesh (about a minute of CPU)")
    ap.add_argument("--amr-steps", type=int, default=50,
                    help="batched steps of the static-AMR measurements (0: skip them)")
    ap.add_argument("--no-collapse", dest="collapse", action="store_false",
                    help="skip the 4-level gravity collapse (about 4600 blocks; a minute of set-up)")
    ap.add_argument("--weno7-child", action="store_true",
                    help="internal: the WENO-Z7 measurement, run in a child process with FX_NGHOST=4")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: one mesh of N x 512 blocks sharded over the ranks (NCCL exchanges of ghost "
                         "zones and dt minima) instead of N independent replicas")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref: the reference's own C core), one process per core
# ---------------------------------------------------------------------------

def _avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return "avx512f" in f.read()
    except OSError:
        return False


def _timing_variant() -> str:
    """The reference build the CPU baseline times: the AVX-512 build
    (x86-64-v4, same doubles as the parity build) where the host has it."""
    from oracle import ref as R
    return "v4" if _avx512() and R.available(True, "v4") else ""


# CPU-baseline samples: (reference preset, its arguments).  The reference has
# no threads and this host has no MPI, so the baseline runs one independent
# instance per core; each instance is a scaled-down case of the measured
# workload (same recipe, same levels), small enough to time in seconds.
CPU_SAMPLES = {
    "fourier": ("params_fourier", dict(root=4)),
    "blast": ("params_amr_blast", dict(root=4, max_level=2, radii=(0.4, 0.2))),
    "collapse": ("params_collapse", dict(root=5)),
}


def _cpu_worker(args):
    kind, nsteps, warm, variant = args
    from oracle import ref as R
    r = R.Reference(True, variant)
    fn, kw = CPU_SAMPLES[kind]
    p = getattr(R, fn)(**kw)
    r.setup(p)
    ints, _, _ = r.mesh_arrays()
    active = int((ints[:, 2] == 1).sum())
    dt = r.calc_dt()
    if warm:
        r.time_steps(warm, dt)
    secs = r.time_steps(nsteps, dt)
    return nsteps * active * 4096, secs, active


def _cpu_variant_worker(variant):
    from oracle import ref as R
    r = R.Reference(True, variant)
    p = R.params_fourier(root=2)
    r.setup(p)
    dt = r.calc_dt()
    r.time_steps(1, dt)
    n = 2
    secs = r.time_steps(n, dt)
    return variant, n * 8 * 4096 / secs


def cpu_variants():
    """One core of the reference C core per build variant, on a 2^3-block
    (32^3-zone) instance of the workload recipe, two timed steps each."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(3) as pool:
        res = pool.map(_cpu_variant_worker, ["weno3", "ess", "ess_weno3"])
    return {v: {"value": x, "unit": UNIT, "cores": 1} for v, x in res}


def _ref_adapt_worker(_):
    from oracle import ref as R
    r = R.Reference(True)
    r.setup(R.params_amr_blast(root=8, max_level=2, radii=(0.4, 0.2)))
    r.amr_configure(R.amr_params(3, [dict(estimator=R.EST_LOEHNER, refine=0.3, derefine=0.1,
                                          lohner_var=R.LOHNER_PRESSURE)]))
    nb = r.nblocks()
    t0 = time.perf_counter()
    changed = r.amr_adapt()
    return time.perf_counter() - t0, nb, r.nblocks(), changed


def ref_adapt_sample():
    """The reference's prj_amr_adapt plus the driver's refill (one core, the
    serial reference C core) on the 2352-block blast mesh of the dynamic-AMR
    key, from its initial state."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        secs, nb0, nb1, changed = pool.map(_ref_adapt_worker, [0])[0]
    return {"seconds": secs, "blocks_before": nb0, "blocks_after": nb1, "changed": bool(changed), "cores": 1,
            "sample": "prj_amr_adapt + eos/ghost refill of src/main.c:571-606, blast 8^3 roots, 3 levels, "
                      "Loehner pressure 0.3 / 0.1 up to level 3, initial state"}


def cpu_reference(steps: int, warmup: int, seconds: float, kind: str = "fourier"):
    """Reference CPU path on all host cores: one independent instance of a
    scaled-down case of the workload per core (CPU_SAMPLES), timed over a
    bounded number of RK2 steps, then zone-updates/s summed over the cores
    (zones of every instance / the slowest instance's time).  The step count
    is bounded so the timed part takes about `seconds`."""
    cores = min(len(os.sched_getaffinity(0)), 128)
    variant = _timing_variant()
    ctx = mp.get_context("spawn")
    # seconds per RK2 step of one instance on one core (AVX-512 build)
    per_step = {"fourier": 0.9, "blast": 6.0, "collapse": 8.0}[kind]
    steps = max(1, min(steps, int(seconds / per_step)))
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(kind, steps, warmup, variant)] * cores)
    zones = sum(z for z, _, _ in res)
    wall = max(t for _, t, _ in res)
    fn, kw = CPU_SAMPLES[kind]
    build = "-O3 -march=x86-64-v4 -ffp-contract=off (AVX-512)" if variant == "v4" else "-O3 -march=x86-64-v3 -ffp-contract=off"
    return {"value": zones / wall, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{cores} independent instances of {fn}({', '.join(f'{k}={v}' for k, v in kw.items())}) "
                      f"({res[0][2]} active blocks of 16^3 each), {steps} RK2 step(s) each after {warmup} untimed, "
                      f"serial reference C core ({build}), one process per core; no MPI on this host"}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    """SM clock and clock-event reasons of the benchmark's GPU while the timed
    region runs.  NVML (read-only queries) is polled every 2 ms on a thread,
    so even a 50 ms timed region gets a few dozen samples; `mark()` brackets
    the timed region and only samples inside it count.  Without NVML the
    recipe's nvidia-smi line (-lms 200) is used instead."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.nvml = None
        self.samples = []          # (time, sm MHz, reason bits)
        self.window = None
        self.smax = None
        self.lines = []

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self):
        nv, h = self.nvml
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), float(sm), int(bits)))
            except Exception:
                return
            time.sleep(0.002)

    def __enter__(self):
        try:
            self.nvml = self._handle()
            nv, h = self.nvml
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = False
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def mark(self, t0, t1):
        """host times bracketing the timed region"""
        self.window = (t0, t1)

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.stop = True
            self.thread.join(timeout=1.0)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
            return
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        if self.nvml is not None:
            sel = [x for x in self.samples if self.window is None or self.window[0] <= x[0] <= self.window[1]]
            if not sel:
                return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": [], "samples": 0, "source": "nvml"}
            reasons = sorted({n for _, _, b in sel for bit, n in self.REASONS.items() if b & bit})
            return {"sm_mhz": statistics.median(x[1] for x in sel), "sm_max_mhz": self.smax,
                    "sm_min_mhz": min(x[1] for x in sel), "reasons": reasons, "samples": len(sel),
                    "source": "nvml, 2 ms polling inside the timed region"}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0, "source": "nvidia-smi"}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi -lms 200"}


# ---------------------------------------------------------------------------

def measured_peak_hbm():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def flux_profile_figures():
    """Figures of one face-flux launch of the 512-block step from the committed
    ncu summary: DRAM bytes (read + write) per launch and the FP64-pipe
    fraction; None where absent."""
    path = os.path.join(HERE, "profiles", "k_flux_traffic_fourier128.txt")
    out = {"dram_bytes_per_launch": None, "fp64_pipe_frac": None}
    try:
        with open(path) as f:
            for line in f:
                key, _, val = line.partition(":")
                if key.strip() in out:
                    out[key.strip()] = float(val)
    except (OSError, ValueError):
        pass
    return out


def run_amr(args, dev, kind):
    """Batched vs plain on a static AMR hierarchy built on the host by the
    product's mesh builder (the reference's refinement rule, 2:1 balance and
    slot order): kind "blast" = magnetised blast, 8^3 roots on [-0.7, 0.7]^3,
    levels refined inside r < 0.4 / 0.2 about (0.1, 0.05, 0) (3 levels);
    kind "collapse" = gravity collapse, 12^3 roots on [-1, 1]^3, spheres
    0.4 / 0.2 / 0.1 about the origin (4 levels).  Same metric as the headline
    (active zones x steps / device time)."""
    import numpy as np
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    t0 = time.time()
    if kind == "blast":
        hw, root, max_level, center, radii, gamma, gravity = 0.7, 8, 2, (0.1, 0.05, 0.0), (0.4, 0.2), 5.0 / 3.0, False
    else:
        hw, root, max_level, center, radii, gamma, gravity = 1.0, 12, 3, (0.0, 0.0, 0.0), (0.4, 0.2, 0.1), 4.0 / 3.0, True
    coord = (-hw, hw, -hw, hw, -hw, hw)
    blocks = mesh.static_amr_mesh((root,) * 3, coord, max_level, mesh.ball_refiner(center, radii))
    desc = mesh.to_desc(blocks)
    cfg = fx.make_config(True, gamma, coord)
    recs = fx.plan_export(cfg, desc, 3)
    t_mesh = time.time() - t0
    if kind == "blast":
        W0, Bf0 = problems.amr_blast(blocks, recs)
        grav = None
    else:
        W0, Bf0, grav = problems.collapse(blocks, recs, half_width=hw)
    t_init = time.time() - t0 - t_mesh
    ctx = fx.Context(True, gamma, coord, gravity=gravity, device=dev)
    t1 = time.time()
    ctx.set_mesh(desc)
    t_plan = time.time() - t1
    ctx.upload_all(np.ascontiguousarray(W0), np.ascontiguousarray(Bf0))
    if grav is not None:
        for b in range(len(blocks)):
            if blocks[b].active == 1:
                ctx.upload_block(b, W0[b].ravel(), [Bf0[b, d].ravel() for d in range(3)],
                                 [grav[b, d] for d in range(3)])
    del W0, Bf0, grav
    ctx.boundary_fill(1, 0)
    ctx.sync()
    ctx.autotune()
    active = [b for b in blocks if b.active == 1]
    zones = len(active) * 16 ** 3
    levels = [0] * (max_level + 1)
    for b in active:
        levels[b.level] += 1
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    state = ctx.run(fx.FORM_BATCHED, max(args.warmup, 3), 0.4, 1.2, 1.0e30, (0.0, 0.0, 0))
    ctx.sync()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    state = ctx.run(fx.FORM_BATCHED, args.amr_steps, 0.4, 1.2, 1.0e30, state)
    e1.record(stream)
    e1.synchronize()
    ms_batched = e0.elapsed_time(e1) / args.amr_steps
    dt = state[1]
    ctx.step(fx.FORM_PLAIN, dt, want_dt_src=False)
    ctx.sync()
    nplain = max(1, args.plain_steps)
    e0.record(stream)
    for _ in range(nplain):
        ctx.step(fx.FORM_PLAIN, dt, want_dt_src=False)
    e1.record(stream)
    e1.synchronize()
    ms_plain = e0.elapsed_time(e1) / nplain
    phases = {name: ctx.time_phase(ph, 3, dt) for name, ph in
              (("flux_launch", 0), ("emf", 1), ("ct", 2), ("cells", 3), ("ghost", 4))}
    out = {
        "workload": ("magnetised blast, static AMR 3 levels" if kind == "blast" else
                     "gravity collapse, static AMR 4 levels") + f", {len(active)} active blocks of 16^3",
        "blocks_per_level": levels, "zones": zones,
        "batched": {"ms_per_step": ms_batched, "value": zones / (ms_batched * 1e-3),
                    "hbm_gbs_step": zones * BYTES_PER_ZONE_STEP / (ms_batched * 1e-3) / 1e9},
        "plain": {"ms_per_step": ms_plain, "value": zones / (ms_plain * 1e-3)},
        "batched_over_plain": ms_plain / ms_batched,
        "phases_ms": phases,
        "ghost_waves": ctx.info(4), "launches_per_batched_step": ctx.info(0) + 4,
        "setup_s": {"mesh": round(t_mesh, 1), "initial_state": round(t_init, 1), "ghost_compiler": round(t_plan, 1)},
        "steps": args.amr_steps,
    }
    ctx.close()
    return out


def run_amr_dynamic(args, dev):
    """Dynamic AMR: the 3-level magnetised blast of run_amr (8^3 roots, 2352
    blocks) stepped with prj_amr_adapt every `interval` steps (Loehner
    pressure criterion, refine 0.3 / derefine 0.1, up to level 3), the driver
    loop of src/main.c.  Wall time per step includes the adapts (device tag,
    host remesh and ghost-fill compile, device prolongation / restriction,
    refill); the adapt phases are reported separately."""
    import numpy as np
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    hw, root = 0.7, 8
    coord = (-hw, hw, -hw, hw, -hw, hw)
    blocks = mesh.static_amr_mesh((root,) * 3, coord, 2, mesh.ball_refiner((0.1, 0.05, 0.0), (0.4, 0.2)))
    desc = mesh.to_desc(blocks)
    recs = fx.plan_export(fx.make_config(True, 5.0 / 3.0, coord), desc, 3)
    W0, Bf0 = problems.amr_blast(blocks, recs)
    ctx = fx.Context(True, 5.0 / 3.0, coord, device=dev)
    ctx.set_mesh(desc)
    ctx.upload_all(np.ascontiguousarray(W0), np.ascontiguousarray(Bf0))
    del W0, Bf0
    ctx.boundary_fill(1, 0)
    ctx.amr_configure(fx.amr_config((root,) * 3, 3, [
        dict(estimator=fx.AMR_LOEHNER, refine=0.3, derefine=0.1, var=fx.AMR_VAR_PRESSURE)]))
    interval = args.amr_interval
    state = ctx.run(fx.FORM_BATCHED, max(args.warmup, 3), 0.4, 1.2, 1.0e30, (0.0, 0.0, 0))
    ctx.sync()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    adapts, step_ms, zone_steps = [], [], 0
    t0 = time.perf_counter()
    for _ in range(args.amr_dynamic_adapts):
        nact = sum(1 for b in ctx.get_mesh() if b.id >= 0 and b.active == 1)
        e0.record(stream)
        state = ctx.run(fx.FORM_BATCHED, interval, 0.4, 1.2, 1.0e30, state)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1) / interval)
        zone_steps += nact * 4096 * interval
        changed = ctx.amr_adapt()
        t = ctx.amr_timings()
        t["changed"] = bool(changed)
        t["blocks_after"] = ctx.nblocks
        adapts.append(t)
    wall = time.perf_counter() - t0
    msh = ctx.get_mesh()
    levels = {}
    for b in msh:
        if b.id >= 0 and b.active == 1:
            levels[b.level] = levels.get(b.level, 0) + 1
    ctx.close()
    nsteps = interval * args.amr_dynamic_adapts
    return {"workload": "magnetised blast, 8^3 roots, 3 static levels then adapts every "
                        f"{interval} steps up to level 3 (Loehner pressure 0.3 / 0.1)",
            "steps": nsteps, "interval": interval,
            "wall_ms_per_step": 1e3 * wall / nsteps,
            "value_wall": zone_steps / wall,
            "device_ms_per_step": step_ms,
            "adapt_ms": [{k: (round(v, 2) if isinstance(v, float) else v) for k, v in a.items()} for a in adapts],
            "active_blocks_per_level_end": [levels.get(l, 0) for l in range(4)]}


def run_variants(args, dev, cpu):
    """The headline workload (128^3 Fourier MHD, 512 blocks) in the
    reference's other build variants: WENO-Z3 reconstruction, the
    eSSPRK10_4 integrator (ten substeps of dt / 6 per step, three stored
    states) and both.  Batched form, device time per driver step (each step
    advances by its own dt: eSSPRK's dt is 6x RK2's CFL step)."""
    import numpy as np
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    coord = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    blocks = mesh.uniform_mesh((ROOT, ROOT, ROOT), coord)
    W0, Bf0 = problems.fourier_mhd(blocks)
    out = {}
    variants = (("weno3", fx.RECON_WENO3, fx.INT_RK2), ("ess", fx.RECON_MC, fx.INT_ESSPRK10_4),
                ("ess_weno3", fx.RECON_WENO3, fx.INT_ESSPRK10_4))
    if fx.NG == 4:
        variants = (("mc_4ghost", fx.RECON_MC, fx.INT_RK2), ("weno7", fx.RECON_WENO7, fx.INT_RK2))
    for name, recon, integ in variants:
        ctx = fx.Context(True, 5.0 / 3.0, coord, device=dev, recon=recon, integrator=integ)
        ctx.set_mesh(mesh.to_desc(blocks))
        ns = ctx.ns
        W = np.zeros((len(blocks), 9, ns, fx.NCELLS))
        Bf = np.zeros((len(blocks), 3, ns, fx.NFACES))
        W[:, :, 0] = W0[:, :, 0]
        Bf[:, :, 0] = Bf0[:, :, 0]
        ctx.upload_state(W, Bf)
        ctx.boundary_fill(1, 0)
        ctx.autotune()
        stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
        state = ctx.run(fx.FORM_BATCHED, max(args.warmup, 3), 0.4, 1.2, 1.0e30, (0.0, 0.0, 0))
        ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        n = 4
        e0.record(stream)
        state = ctx.run(fx.FORM_BATCHED, n, 0.4, 1.2, 1.0e30, state)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / n
        out[name] = {"ms_per_step": ms, "value": ZONES / (ms * 1e-3), "unit": UNIT,
                     "dt": state[1], "launches_per_step": ctx.info(0),
                     "flux_launch_ms": ctx.time_phase(fx.PHASE_FLUX, 5, state[1])}
        if cpu and name in cpu:
            out[name]["cpu_reference_1core"] = cpu[name]
        ctx.close()
    return out


def run_weno7(args):
    """WENO-Z7 needs the four-ghost-layer build, which a process selects at
    start (FX_NGHOST=4): a child process measures it (and MC on the same
    24^3 layout) on the headline workload, plus one core of the reference
    built with WENO-Z7 on a 2^3-block instance."""
    env = dict(os.environ, FX_NGHOST="4")
    cmd = [sys.executable, os.path.abspath(__file__), "--weno7-child", "--warmup", str(args.warmup)]
    if args.no_cpu_baseline:
        cmd.append("--no-cpu-baseline")
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=1200)
    if r.returncode != 0:
        return {"unavailable": (r.stderr or r.stdout).strip().splitlines()[-1:]}
    return json.loads(r.stdout.strip().splitlines()[-1])


def weno7_child(args):
    cpu = None
    if not args.no_cpu_baseline:
        ctx = mp.get_context("spawn")
        with ctx.Pool(1) as pool:
            res = pool.map(_cpu_variant_worker, ["weno7"])
        cpu = {v: {"value": x, "unit": UNIT, "cores": 1} for v, x in res}
    return run_variants(args, 0, cpu)


def run_adjoint(args, dev):
    """Cost of the discrete adjoint on the 64^3 workload (4^3 blocks of 16^3,
    seeded Fourier-mode MHD with amplitude 0.01, |k|_inf <= 3): device time
    of the reverse sweep over 10 RK2 steps per step, against one batched
    forward step."""
    import numpy as np
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    coord = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    blocks = mesh.uniform_mesh((4, 4, 4), coord)
    W0, Bf0 = problems.fourier_mhd(blocks, nmodes=32, kmax=3, amp_rho=0.01, amp_v=0.01, amp_A=0.005)
    ctx = fx.Context(True, 5.0 / 3.0, coord, device=dev)
    ctx.set_mesh(mesh.to_desc(blocks))
    ctx.upload_all(np.ascontiguousarray(W0), np.ascontiguousarray(Bf0))
    ctx.boundary_fill(1, 0)
    dt = ctx.calc_dt(0.4)
    nsteps = 10
    ctx.adjoint_forward(nsteps, dt)
    seed = np.full(W0.size, 1.0e-3)
    ms = []
    for _ in range(3):
        ctx.adjoint_backward(seed)
        ms.append(ctx.adjoint_ms() / nsteps)
    ms_adj = min(ms)
    ms_fwd = ctx.time_phase(fx.PHASE_STEP, 20, dt)
    ctx.close()
    return {"workload": "64^3 MHD (4^3 blocks), 10 RK2 steps, fixed dt", "ms_per_step_adjoint": ms_adj,
            "ms_per_step_forward": ms_fwd, "adjoint_over_forward": ms_adj / ms_fwd}


def run_shard(args, rank, world, local_rank):
    """Weak scaling with exchanges: one uniform mesh of (8 N) x 8 x 8 blocks
    (N 128^3 cubes along x, outflow boundaries), the active blocks cut into
    N contiguous runs of the mesh order, one rank per GPU over NCCL.  Every
    stage exchanges the ghost zones at the rank boundaries and every step
    takes the dt minima over the ranks, inside the step's CUDA graph."""
    import numpy as np
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    dev = local_rank
    torch.cuda.set_device(dev)
    coord = (0.0, float(world), 0.0, 1.0, 0.0, 1.0)
    blocks = mesh.uniform_mesh((ROOT * world, ROOT, ROOT), coord)
    desc = mesh.to_desc(blocks)
    owner = fx.morton_owner(desc, world)
    mine = [int(b) for b in np.nonzero(owner == rank)[0]]
    W0, Bf0 = problems.fourier_mhd([blocks[b] for b in mine])
    ctx = fx.Context(True, 5.0 / 3.0, coord, device=dev)
    ctx.shard_set_mesh(desc, owner, world, rank)
    uid = torch.zeros(128, dtype=torch.uint8, device=f"cuda:{dev}")
    if world > 1:
        if rank == 0:
            uid.copy_(torch.frombuffer(bytearray(fx.nccl_unique_id()), dtype=torch.uint8))
        torch.distributed.broadcast(uid, 0)
    else:
        uid.copy_(torch.frombuffer(bytearray(fx.nccl_unique_id()), dtype=torch.uint8))
    ctx.attach_nccl(bytes(uid.cpu().numpy().tobytes()))
    for n, b in enumerate(mine):
        ctx.upload_block(b, W0[n].ravel(), [Bf0[n, d].ravel() for d in range(3)])
    ctx.boundary_fill(1, 0)
    ctx.sync()
    cfl, dt_factor, t_end = 0.4, 1.2, 1.0e30
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    state = ctx.run(fx.FORM_BATCHED, args.warmup, cfl, dt_factor, t_end, (0.0, 0.0, 0))
    ctx.sync()
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        torch.cuda.synchronize(dev)
        h0 = time.perf_counter()
        e0.record(stream)
        state = ctx.run(fx.FORM_BATCHED, args.steps, cfl, dt_factor, t_end, state)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize(dev)
        clk.mark(h0, time.perf_counter())
    if world > 1:
        torch.distributed.barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    nown, nlocal, doubles = ctx.shard_info()
    zones = world * ZONES
    line = {
        "metric": METRIC, "value": zones * args.steps / (ms_total / 1000.0), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Fourier-mode MHD, host-generated per rank)",
        "config": {"workload": f"3D ideal MHD, one mesh of {ROOT * world}x{ROOT}x{ROOT} blocks of 16^3 "
                               "(128^3 zones per GPU), MC+HLLD+CT RK2, batched form",
                   "blocks": len(desc), "zones": zones, "parallelism": f"shard x{world} (NCCL)",
                   "l2": "working set > 2.7 GB per GPU >> 126 MB L2 (no flush)"},
        "shard": {"owned_blocks": nown, "halo_blocks": nlocal - nown,
                  "bytes_sent_per_step_rank0": 8 * doubles},
        "clocks": clk.summary(),
    }
    ctx.close()
    return line


def run_fx(args, rank, world, local_rank):
    import numpy as np
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    dev = local_rank
    torch.cuda.set_device(dev)
    coord = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    blocks = mesh.uniform_mesh((ROOT, ROOT, ROOT), coord)
    W0, Bf0 = problems.fourier_mhd(blocks)
    nb = len(blocks)
    ctx = fx.Context(True, 5.0 / 3.0, coord, device=dev)
    ctx.set_mesh(mesh.to_desc(blocks))
    W0 = np.ascontiguousarray(W0)
    Bf0 = np.ascontiguousarray(Bf0)
    ctx.upload_all(W0, Bf0)
    ctx.boundary_fill(1, 0)       # the driver's initial ghost fill (src/main.c:446)
    ctx.sync()
    tuned, tune_ms = ctx.autotune()
    cfl, dt_factor, t_end = 0.4, 1.2, 1.0e30
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    state = (0.0, 0.0, 0)
    state = ctx.run(fx.FORM_BATCHED, args.warmup, cfl, dt_factor, t_end, state)
    ctx.sync()
    torch.cuda.synchronize(dev)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        torch.cuda.synchronize(dev)
        h0 = time.perf_counter()
        e0.record(stream)
        state = ctx.run(fx.FORM_BATCHED, args.steps, cfl, dt_factor, t_end, state)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize(dev)
        clk.mark(h0, time.perf_counter())
    barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    ms_step = ms_total / args.steps
    value = world * ZONES * args.steps / (ms_total / 1000.0)
    dt_fixed = state[1]

    # plain (per-block launch) form, same state, same metric
    ms_plain = None
    if args.plain_steps > 0:
        ctx.step(fx.FORM_PLAIN, dt_fixed, want_dt_src=False)
        ctx.sync()
        e0.record(stream)
        for _ in range(args.plain_steps):
            ctx.step(fx.FORM_PLAIN, dt_fixed, want_dt_src=False)
        e1.record(stream)
        e1.synchronize()
        ms_plain = max_over_ranks(e0.elapsed_time(e1)) / args.plain_steps

    # per-phase timings (batched sweeps; the face-flux launch dominates)
    phases = {}
    for name, ph in (("flux_launch", 0), ("emf", 1), ("ct", 2), ("cells", 3), ("ghost", 4)):
        phases[name] = ctx.time_phase(ph, 5, dt_fixed)
    ms_flux = phases["flux_launch"]

    # end to end through the C ABI with host buffers (page-locked): every
    # step uploads the state, steps, and downloads it.  Headline: the active
    # region (slot 0 of the active cells and faces, read and written by the
    # device straight from the host arrays, ghost zones refilled on the
    # device); beside it the full-array copies (every cell and face of slot 0)
    Wh = torch.empty(W0.size, dtype=torch.float64, pin_memory=True).numpy()
    Bh = torch.empty(Bf0.size, dtype=torch.float64, pin_memory=True).numpy()
    ctx.download_all(Wh, Bh)
    L = ctx.L
    dp = fx._dp
    h2d_full = nb * (9 * fx.NCELLS + 3 * fx.NFACES) * 8
    # active transfers: per block the rows of the active (i, j) range, ghost
    # columns along k included, of the three face directions and of the 6
    # non-field variables up (the cell field is recomputed from the faces),
    # all 9 variables down
    P = 16 + 2 * fx.NG
    faces_span = 17 * 16 * P + 16 * 17 * P + 16 * 16 * (P + 1)
    h2d_active = nb * (6 * 16 * 16 * P + faces_span) * 8
    d2h_active = nb * (9 * 16 * 16 * P + faces_span) * 8
    e2e_ms = e2e_full_ms = None
    if args.e2e_steps > 0:
        for kind in ("active", "full"):
            for rep in range(2):          # the first pass warms the copy paths
                torch.cuda.synchronize(dev)
                e0.record(stream)
                for _ in range(args.e2e_steps):
                    if kind == "active":
                        ctx._check(L.fx_upload_state_active(ctx._h, Wh.ctypes.data, Bh.ctypes.data))
                        ctx.step(fx.FORM_BATCHED, dt_fixed, want_dt_src=False)
                        ctx._check(L.fx_download_state_active(ctx._h, Wh.ctypes.data, Bh.ctypes.data))
                    else:
                        ctx._check(L.fx_upload_state(ctx._h, dp(Wh), dp(Bh)))
                        ctx.step(fx.FORM_BATCHED, dt_fixed, want_dt_src=False)
                        ctx._check(L.fx_download_state(ctx._h, dp(Wh), dp(Bh)))
                e1.record(stream)
                e1.synchronize()
                ctx.sync()
            ms = max_over_ranks(e0.elapsed_time(e1)) / args.e2e_steps
            if kind == "active":
                e2e_ms = ms
            else:
                e2e_full_ms = ms

    peak, peak_kind = measured_peak_hbm()
    # roofline of the face-flux launch (one RK stage's face sweep over all
    # blocks, three directions): algorithmic bytes = half of the step's
    # compulsory state traffic, 180 B per zone (9 FP64 variables x 8 B x 5
    # passes per RK2 step / 2 stages)
    alg_bytes = ZONES * BYTES_PER_ZONE_STEP / 2.0
    achieved = alg_bytes / (ms_flux * 1e-3) / 1e9
    # the kernel's own input and output bytes: per direction and block the 8
    # primitive inputs of the 20 x 18 x 18 stencil cells, and per face the
    # face field (8 B) plus the outputs later phases read (6 hydro fluxes, the
    # normal velocity, Bv1, Bv2: 9 doubles)
    faces = nb * 3 * 17 * 18 * 18
    kernel_bytes = nb * 3 * 20 * 18 * 18 * 8 * 8 + faces * 8 + faces * 9 * 8
    prof = flux_profile_figures()
    traffic = prof["dram_bytes_per_launch"]
    launches_per_step = ctx.info(0) + 4
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Fourier-mode MHD, host-generated)",
        "config": {
            "workload": "3D ideal MHD 128^3, 512 blocks of 16^3 + 2 ghosts, gamma 5/3, 32 seeded modes k<=4, "
                        "MC+HLLD+CT RK2, batched form (one CUDA graph per step)",
            "blocks": nb, "zones": ZONES, "form": "batched", "l2": "working set 2.7 GB >> 126 MB L2 (no flush)",
            "parallelism": f"replicas x{world}",
        },
        "hbm_gbs_step": ZONES * BYTES_PER_ZONE_STEP / (ms_step * 1e-3) / 1e9,
        "hbm_frac_step": ZONES * BYTES_PER_ZONE_STEP / (ms_step * 1e-3) / 1e9 / peak,
        "plain": None if ms_plain is None else {
            "ms_per_step": ms_plain, "value": world * ZONES / (ms_plain * 1e-3),
            "batched_over_plain": ms_plain / ms_step},
        "phases_ms": phases,
        "autotune": {"flux_shape": tuned, "flux_ms_per_shape": [round(x, 4) for x in tune_ms[:6]]},
        "roofline": {
            "kernel": "k_flux (face fluxes, three directions, all blocks; one launch per RK stage)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": alg_bytes,
            "traffic_over_algorithmic": None if traffic is None else traffic / alg_bytes,
            "kernel_bytes_per_launch": kernel_bytes,
            "kernel_bytes_gbs": kernel_bytes / (ms_flux * 1e-3) / 1e9,
            "ms_per_launch": ms_flux,
            "fp64": {"pipe_frac": prof["fp64_pipe_frac"],
                     "note": "the FP64 issue rate of the HLLD solver bounds this kernel before HBM; "
                             "pipe fraction from an ncu capture of one launch"},
        },
        "e2e": None if e2e_ms is None else {
            "value": world * ZONES / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms,
            "h2d_bytes_per_step": h2d_active, "d2h_bytes_per_step": d2h_active,
            "copies": "fx_upload_state_active / fx_download_state_active: copy-engine row copies of slot 0's "
                      "active region (cell field recomputed from the faces and ghost zones refilled on the "
                      "device after the upload)"},
        "e2e_full": None if e2e_full_ms is None else {
            "value": world * ZONES / (e2e_full_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_full_ms,
            "h2d_bytes_per_step": h2d_full, "d2h_bytes_per_step": h2d_full,
            "copies": "fx_upload_state / fx_download_state: every cell and face of slot 0 (copy engines)"},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
    }
    ctx.close()
    return line


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.weno7_child:
        print(json.dumps(weno7_child(args)))
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        t0 = time.time()
        cb = cpu_reference(args.steps, args.warmup, args.cpu_seconds)
        v = cb["value"]
        line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * ZONES / v, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Fourier-mode MHD)",
                "config": {"workload": "3D ideal MHD 128^3 recipe, reference CPU path (oracle/_ref)",
                           "zones": ZONES},
                "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "wall_s": time.time() - t0}
        print(json.dumps(line))
        return 0

    # CPU baseline first (spawned processes, before any GPU call)
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_reference(20, 1, args.cpu_seconds)
        except Exception as exc:  # oracle missing on this machine
            cb = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                  "sample": f"unavailable: {exc}"}
    cv = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.variants:
        try:
            cv = cpu_variants()
        except Exception as exc:
            cv = {"unavailable": str(exc)}
    cb_amr = {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.amr_steps > 0:
        for kind in ("blast",) + (("collapse",) if args.collapse else ()):
            try:
                cb_amr[kind] = cpu_reference(1, 0, 1.0, kind)
            except Exception as exc:
                cb_amr[kind] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                "sample": f"unavailable: {exc}"}
    ra = None
    if rank == 0 and world == 1 and args.ref_adapt:
        try:
            ra = ref_adapt_sample()
        except Exception as exc:
            ra = {"seconds": None, "sample": f"unavailable: {exc}"}
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.shard:
        line = run_shard(args, rank, world, local_rank)
        line["cpu_baseline"] = cb
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        if rank == 0:
            print(json.dumps(line))
        return 0
    line = run_fx(args, rank, world, local_rank)
    line["cpu_baseline"] = cb
    if world == 1:
        line["adjoint"] = run_adjoint(args, local_rank)
    if world == 1 and args.variants:
        line["variants"] = run_variants(args, local_rank, cv)
        line["variants"].update(run_weno7(args))
    if world == 1 and args.amr_steps > 0:
        line["amr_blast"] = run_amr(args, local_rank, "blast")
        line["amr_blast"]["cpu_reference"] = cb_amr.get("blast")
        if args.collapse:
            line["amr_collapse"] = run_amr(args, local_rank, "collapse")
            line["amr_collapse"]["cpu_reference"] = cb_amr.get("collapse")
    if world == 1 and args.amr_dynamic_adapts > 0:
        line["amr_dynamic"] = run_amr_dynamic(args, local_rank)
        if ra is not None:
            line["amr_dynamic"]["reference_adapt"] = ra
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
