"""Benchmark of the time-step hot path on B200.

Workload (the moist warm-rain benchmark grid and step structure): 1024 x 1024 x 64
cells, dx = dy = 3 km, 16 km model top, moist sounding (theta 300 K, +4 K/km
above 1 km, 90 % RH below 2 km decaying with a 1.5 km scale height to 1e-5,
0.5 K rms seeded theta noise below 1 km), one step = dry SSPRK3 with 6 acoustic
substeps + three-tracer SSPRK3 transport + warm rain with metric fallout
(terminal velocity 12 m/s).  The step is run at dt = 1 s: the reference's
discretisation is unstable at the configuration's 12 s on this grid.

One JSON line is printed by rank 0.  ``value`` is whole-job cell updates per
second (cells x steps / device time, max over ranks), with the state resident
in HBM; ``e2e`` is the same metric through the public C-ABI with the state in
pinned host memory, copied in and out every step.  ``--impl reference`` times
the CPU restatement of the reference algorithm on the host cores instead.
Under torchrun every rank advances an independent replica (the path is
single-device; replicas scale weakly with no collective).
"""
import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 1024, 1024, 64
DX = 3000.0
ZTOP = 16000.0
DT = 1.0
NS = 6
VT = 12.0
# the moist sounding of the workload (both arms build it: the library, or the oracle)
SOUNDING = dict(theta_ref=300.0, theta_lapse_k_per_m=0.004, relative_humidity=0.9, rh_top_m=2000.0,
                qv_scale_height_m=1500.0, qv_floor=1e-5, noise_rms_k=0.5, noise_depth_m=1000.0)


def grid_spec(gwm, nx=NX, ny=NY, nz=NZ):
    return gwm.GridSpec(nx, ny, nz, dx=DX, dy=DX, z_top=ZTOP)


def case_params(gwm, seed=1):
    return gwm.CaseParams(seed=seed, **SOUNDING)


def member_spec(gwm):
    return gwm.MemberSpec(step=gwm.StepConfig(dt=DT, fast_substeps=NS),
                          rain=gwm.WarmRainConfig(dt=DT, rain_terminal_velocity=VT), moist=True)


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    Reads NVML in a polling thread (10 ms period; read-only queries) on the NVML device
    whose PCI bus id matches the CUDA device, so that a sub-second timed region still
    gets tens of samples; falls back to an `nvidia-smi -lms 100` pipe when NVML is
    unavailable."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index=0, period_s=0.01):
        self.index = index
        self.period_s = period_s
        self.samples = []          # (sm_mhz, sm_max_mhz, {reason names})
        self._stop = threading.Event()
        self._proc = None
        self._thread = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            smmax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            self._start_smi()
            return
        self.source = "nvml"

        def poll():
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except Exception:
                    break
                self.samples.append((float(sm), float(smmax), {n for n, b in self.REASONS if bits & b}))
                self._stop.wait(self.period_s)

        self._thread = threading.Thread(target=poll, daemon=True)
        self._thread.start()

    def _start_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return
        self.source = "nvidia-smi"

        def read():
            for line in self._proc.stdout:
                s = [x.strip() for x in line.split(",")]
                if len(s) >= 6 and s[0].replace(".", "").isdigit() and s[1].replace(".", "").isdigit():
                    self.samples.append((float(s[0]), float(s[1]),
                                         {n for (n, _), v in zip(self.REASONS, s[2:6]) if v == "Active"}))

        self._thread = threading.Thread(target=read, daemon=True)
        self._thread.start()

    def wait_first(self, timeout):
        t = time.time()
        while self.source and not self.samples and time.time() - t < timeout:
            time.sleep(0.01)

    def mark(self):
        """Only samples taken after this point describe the timed region."""
        self._start = len(self.samples)

    def stop(self):
        self._stop.set()
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._thread:
            self._thread.join(timeout=5)

    def summary(self):
        s = self.samples[getattr(self, "_start", 0):]
        if not s:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median([x[0] for x in s])), "sm_max_mhz": max(x[1] for x in s),
                "reasons": sorted(set().union(*(x[2] for x in s))), "samples": len(s),
                "source": self.source}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes of one acoustic substep per cell (the dominant kernel): the
# hot-path byte model counts 12 FP32 field accesses per cell per substep
# (rho, theta, three momenta and three base momenta read; rho and three momenta
# written).
SUBSTEP_ALGO_BYTES_PER_CELL = 12 * 4


# CPU sample per step: the per-cell cost of the CPU restatement does not depend on the
# horizontal size (0.84e6, 0.86e6 and 0.80e6 cell-updates/s at 64^2, 128^2 and 256^2 x 64 on
# 8 threads), so a 256 x 256 x 64 periodic subdomain of the workload stands for it
CPU_SAMPLE = 256


def workload_config(nx=NX, ny=NY, world=1):
    """The workload both arms report (what is timed per step is stated beside it)."""
    return {"workload": "moist warm-rain step, 1024x1024x64 C3 grid",
            "nx": nx, "ny": ny, "nz": NZ, "dx_m": DX, "z_top_m": ZTOP,
            "dt_s": DT, "fast_substeps": NS, "rain_terminal_velocity": VT,
            "phases": "dry SSPRK3 + 3-tracer SSPRK3 + warm rain/fallout",
            "l2": "inputs larger than L2 (each field 282 MB)",
            "parallelism": f"replicas{world}"}


def oracle_sample(n, seed=1):
    """The CPU restatement and a periodic n x n x 64 subdomain of the workload, built by
    the oracle itself (no product code is loaded)."""
    import oracle
    oracle.build()
    threads = oracle.max_threads()
    oracle.set_threads(threads)
    og = oracle.GridSpec(n, n, NZ, dx=DX, dy=DX, z_top=ZTOP)
    st = oracle.moist_sounding(og, seed=seed, **SOUNDING)
    kw = dict(phases=oracle.PHASE_DRY | oracle.PHASE_TRACERS | oracle.PHASE_RAIN,
              rain=oracle.RainSpec(dt=DT, terminal_velocity=VT), precision=32)
    return oracle, og, st, oracle.StepSpec(dt=DT, fast_substeps=NS), kw, threads


def cpu_baseline(steps_sample=2, n=128):
    oracle, og, st, step, kw, threads = oracle_sample(n)
    t0 = time.perf_counter()
    oracle.run(og, step, st, steps_sample, **kw)
    dt = time.perf_counter() - t0
    cells = n * n * NZ * steps_sample
    return {"value": cells / dt, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{n}x{n}x{NZ} periodic subdomain of the workload, {steps_sample} full moist steps, "
                      f"FP32 oracle restatement, OpenMP {threads} threads, {dt:.2f} s"}


def run_reference(args, rank, world):
    """The reference's algorithm on the host cores.  The reference has no CPU step (its
    kernels are CUDA and its host code moves halos), so this times its CPU restatement,
    the oracle, with every host thread; each step advances a 256 x 256 x 64 periodic
    subdomain of the workload (initial state from the oracle's own builder)."""
    if rank != 0:
        return
    n = CPU_SAMPLE
    oracle, og, st, step, kw, threads = oracle_sample(n)
    for _ in range(args.warmup):
        st = oracle.run(og, step, st, 1, **kw)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = oracle.run(og, step, st, 1, **kw)
    el = time.perf_counter() - t0
    cells = n * n * NZ
    val = cells * args.steps / el
    sample = (f"{n}x{n}x{NZ} periodic subdomain of the 1024x1024x64 workload per step (the per-cell "
              f"cost does not depend on the horizontal size), FP32 oracle restatement, OpenMP {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": "cell-updates/s", "value": val, "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(world=world),
        "sampled_grid": {"nx": n, "ny": n, "nz": NZ},
        "cpu_baseline": {"value": val, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": val, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="launch kernels directly (profiling)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default tiles (no autotune)")
    ap.add_argument("--fast-tile", type=int, default=None,
                    help="acoustic-substep kernel (0 owned tile, 3 TMA-fed, 8/16 overlapped); implies --no-tune")
    ap.add_argument("--slow-tile", type=int, default=None,
                    help="slow-stage kernel (3 TMA-fed owned tile, 8/16 overlapped); implies --no-tune")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-member ensemble line")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned-microphysics line")
    ap.add_argument("--no-c2", action="store_true", help="skip the mountain-wave (512x512x80 terrain) line")
    ap.add_argument("--only-c2", type=int, default=None, metavar="N",
                    help="run only the mountain-wave object on an N x N x 80 grid (profiling); prints it alone; "
                         "--fast-tile/--slow-tile/--tracer-tile fix its tiles instead of tuning them")
    ap.add_argument("--only-ensemble", action="store_true",
                    help="run only the 64-member ensemble object (profiling); prints it alone")
    ap.add_argument("--no-persistent", action="store_true",
                    help="skip timing the acoustic substeps of a stage as one persistent launch")
    ap.add_argument("--tracer-tile", type=int, default=None,
                    help="tracer-stage kernel (3 TMA-fed owned tile, 8/16 overlapped); implies --no-tune")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    gwm = importlib.import_module("gpu-wm-next_b200")
    if args.only_c2:
        stream = torch.cuda.Stream()
        fixed = {k: r for k, r in (("fast_substep", args.fast_tile), ("slow_stage", args.slow_tile),
                                   ("tracer_stage", args.tracer_tile)) if r is not None}
        c2 = c2_line(gwm, torch, stream, dist, world, steps=args.steps, warmup=args.warmup, n=args.only_c2,
                     tiles=fixed or None)
        if rank == 0:
            print(json.dumps({"c2": c2}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.only_ensemble:
        stream = torch.cuda.Stream()
        ensemble = ensemble_line(gwm, torch, stream, dist, world)
        if rank == 0:
            print(json.dumps({"ensemble": ensemble}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    g = grid_spec(gwm, args.nx, args.ny, NZ)
    state = gwm.build_case("moist_sounding", g, case_params(gwm, seed=1 + rank), moist=True)
    model = gwm.Model(g, member_spec(gwm))
    stream = torch.cuda.Stream()
    model.set_stream(stream.cuda_stream)
    model.upload(state)
    tiles = None
    tile_ms = None
    if args.fast_tile is not None:
        args.no_tune = True
        model.set_tile("fast_substep", args.fast_tile)
    if args.slow_tile is not None:
        args.no_tune = True
        model.set_tile("slow_stage", args.slow_tile)
    if args.tracer_tile is not None:
        args.no_tune = True
        model.set_tile("tracer_stage", args.tracer_tile)
    if not args.no_tune:
        # pick each stencil kernel's tile by timing it, then restart from the initial state
        with torch.cuda.stream(stream):
            tiles = model.autotune(1)
        tile_ms = {k: {str(r): round(t, 4) for r, t in v.items()} for k, v in model.tile_times.items()}
        model.upload(state)
    else:
        tiles = {k: model.get_tile(k) for k in ("slow_stage", "fast_substep", "tracer_stage")}
    # the substeps of each RK stage as one persistent launch against one launch per
    # substep, on the same state; the faster form (equal results) is the one timed below
    persistent = None
    if tiles["fast_substep"] == 3 and not args.no_persistent and not args.no_graph:
        persistent = persistent_choice(model, state, stream, torch)
        tiles["fast_substep"] = persistent["chosen_tile"]
    model.use_graph(not args.no_graph)
    cells = args.nx * args.ny * NZ

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    # warm-up (also captures the step graph)
    with torch.cuda.stream(stream):
        model.step(max(args.warmup, 1))
    barrier()
    clocks.wait_first(10.0)
    clocks.mark()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    t0.record(stream)
    model.step(args.steps)
    t1.record(stream)
    barrier()
    clocks.stop()
    ms = t0.elapsed_time(t1)
    launches = model.launch_count
    ms_max = max_over_ranks(ms, torch, dist, "cuda")
    value = job_throughput(cells, args.steps, world, ms_max)
    budget = model.budgets()
    finite = all(np.isfinite(v) for v in budget.values())

    # dominant-kernel timing: one acoustic substep per launch; measured through a
    # fast-mode-only step sequence on the same state (device events, same stream)
    roof = substep_roofline(model, g, stream, torch)

    # end-to-end through the C-ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(gwm, model, g, stream, torch, max(2, min(args.steps, 5)), world, dist)
    # learned warm-rain microphysics against the plain scheme on the same state
    surrogate = None
    if not args.no_surrogate:
        surrogate = surrogate_line(gwm, model, stream, torch)
    model.close()
    ensemble = None
    if not args.no_ensemble:
        ensemble = ensemble_line(gwm, torch, stream, dist, world)
    c2 = None
    if not args.no_c2:
        c2 = c2_line(gwm, torch, stream, dist, world)

    if rank == 0:
        peak, which = load_peaks()
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "sim_s_per_wall_s": DT * args.steps / (ms_max * 1e-3),
            "config": dict(workload_config(args.nx, args.ny, world), graph=not args.no_graph,
                           tile_rows=tiles, tile_autotune_ms=tile_ms),
            "gpu_launches": launches,
            "state_finite": finite,
            "roofline": roof,
            "clocks": clocks.summary(),
        }
        line["roofline"]["peak"] = peak
        line["roofline"]["peak_source"] = which
        line["roofline"]["frac"] = roof["achieved"] / peak
        if e2e:
            line["e2e"] = e2e
        if surrogate:
            line["surrogate"] = surrogate
        if ensemble:
            line["ensemble"] = ensemble
        if c2:
            line["c2"] = c2
        if persistent:
            line["persistent_substeps"] = persistent
        if not args.no_cpu_baseline and world == 1:  # the host cores' baseline: rank 0 at N=1 only
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def persistent_choice(model, state, stream, torch, steps=5):
    """Step time (graph replay, CUDA events on the model's stream) with one launch per
    acoustic substep (tiles 3) and with each RK stage's substeps in one persistent
    cooperative launch (tiles 4), from the same state; the end states must agree bit for
    bit.  Leaves the faster tile set and the initial state uploaded."""
    ms, outs = {}, {}
    for rows in (3, 4):
        model.set_tile("fast_substep", rows)
        model.use_graph(True)
        model.upload(state)
        with torch.cuda.stream(stream):
            model.step(3)  # warm-up, graph capture
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        model.step(steps)
        t1.record(stream)
        torch.cuda.synchronize()
        ms[rows] = t0.elapsed_time(t1) / steps
        outs[rows] = model.download()
    identical = all(np.array_equal(outs[3][k], outs[4][k]) for k in outs[3])
    chosen = 4 if identical and ms[4] < ms[3] else 3
    model.set_tile("fast_substep", chosen)
    model.upload(state)
    return {"per_substep_launch_ms_per_step": ms[3], "persistent_stage_ms_per_step": ms[4],
            "saving_ms_per_step": ms[3] - ms[4], "bit_identical": identical, "chosen_tile": chosen,
            "steps": steps, "note": "acoustic substeps of an RK stage as one cooperative launch with a bounded "
                                    "grid barrier between substeps (the step's last substep keeps its own launch) "
                                    "against one launch per substep; both inside the replayed step graph"}


def substep_roofline(model, g, stream, torch, steps=2):
    """Per-kernel device time from CUDA events recorded around each launch on the
    launching stream (direct launches), for steps full steps after the timed region.
    The persistent form times a whole stage per launch, so the per-substep launches
    (the same tiles and arithmetic) are timed here."""
    tile = model.get_tile("fast_substep")
    if tile == 4:
        model.set_tile("fast_substep", 3)
    with torch.cuda.stream(stream):
        model.profile(True)
        model.step(steps)
        rep = model.profile_report()
        model.profile(False)
    if tile == 4:
        model.set_tile("fast_substep", 4)
    cells = g.nx * g.ny * g.nz
    fast = rep["k_fast_substep"]
    achieved = SUBSTEP_ALGO_BYTES_PER_CELL * cells / (fast["avg_ms"] * 1e-3) / 1e9
    total = sum(v["total_ms"] for v in rep.values())
    shares = {k: round(v["total_ms"] / total, 4) for k, v in rep.items()}
    fast_tile = 3 if tile == 4 else tile  # the kernel whose launches were timed
    kname = {0: "k_fast_flat", 3: "k_fast_tma"}.get(fast_tile, f"k_fast_substep<{fast_tile}>")
    return {"bound": "hbm", "achieved": achieved, "unit": "GB/s", "traffic": read_traffic(g, fast_tile),
            "kernel": f"{kname} (one acoustic substep)",
            "algorithmic_bytes_per_launch": SUBSTEP_ALGO_BYTES_PER_CELL * cells,
            "avg_launch_ms": fast["avg_ms"], "kernel_shares": shares,
            "kernel_avg_ms": {k: round(v["avg_ms"], 4) for k, v in rep.items()}}


# committed ncu summaries of the acoustic-substep kernels (DRAM bytes per cell of one launch)
TRAFFIC_PROFILES = {3: "k_fast_tma_768x768x64.txt"}


def read_traffic(g, fast_tile):
    """DRAM bytes per substep launch from the committed ncu summary of the substep kernel
    in use, captured on a 768 x 768 x 64 case and scaled by cells (traffic per cell does
    not depend on the horizontal size: inputs exceed L2 in both)."""
    name = TRAFFIC_PROFILES.get(fast_tile)
    if name is None:
        return None
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    vals = {}
    for line in open(p):
        if ":" in line:
            k, v = line.split(":", 1)
            vals[k.strip()] = v.strip()
    try:
        per_cell = float(vals["dram_bytes_per_cell"])
    except (KeyError, ValueError):
        return None
    return per_cell * g.nx * g.ny * g.nz


SURROGATE_WEIGHTS = os.path.join(ROOT, "gpu-wm-next_b200", "surrogate_c3.npz")


def rain_call_closure(model):
    """Total-water closure of one warm-rain call (microphysics and fallout): the column
    water paths sum(rho (qv + qc + qr) dz) plus the accumulated surface precipitation,
    reduced in FP64 on the device before and after the call; |after - before| / before.
    The fields are stored in FP32, so the residual is the rounding of the stored updates."""
    def total(b):
        return (b["vapor_water_path_sum_kg_m2"] + b["cloud_water_path_sum_kg_m2"] + b["rain_water_path_sum_kg_m2"]
                + b["accumulated_surface_precipitation_sum_mm"])
    w0 = total(model.budgets())
    model.apply_warm_rain_microphysics("metric")
    return abs(total(model.budgets()) - w0) / w0


def surrogate_line(gwm, model, stream, torch, steps=10):
    """Warm-rain kernel time with the plain scheme and with the trained network (device
    events around each launch, profiling mode), both continuing from the same state;
    precipitation and fallbacks of the network run."""
    if not os.path.exists(SURROGATE_WEIGHTS):
        return {"unavailable": "no trained weights (gpu-wm-next_b200/train_surrogate.py writes them)"}
    w = np.load(SURROGATE_WEIGHTS)
    snap = model.download()
    out = {}
    for mode in ("plain", "surrogate"):
        model.upload(snap)
        if mode == "surrogate":
            model.set_rain_surrogate(w["params"], w["norm"], w["range"])
            model.surrogate_stats(reset=True)
        with torch.cuda.stream(stream):
            model.profile(True)
            model.step(steps)
            rep = model.profile_report()
            model.profile(False)
        b = model.budgets()
        out[mode] = {"rain_kernel_ms": rep["k_warm_rain"]["avg_ms"],
                     "precip_sum_mm": b["accumulated_surface_precipitation_sum_mm"],
                     "water_closure_per_call": rain_call_closure(model)}
        if mode == "surrogate":
            st = model.surrogate_stats()
            out[mode]["stats"] = st
            cells = model.grids[0].nx * model.grids[0].ny * model.grids[0].nz * steps
            out[mode]["network_fraction"] = st["network_cells"] / cells
            out[mode]["fallback_fraction"] = st["fallbacks"] / max(st["network_cells"], 1)
            model.set_rain_surrogate(None)
    p0, p1 = out["plain"]["precip_sum_mm"], out["surrogate"]["precip_sum_mm"]
    return {"plain_rain_ms": out["plain"]["rain_kernel_ms"], "surrogate_rain_ms": out["surrogate"]["rain_kernel_ms"],
            "speedup": out["plain"]["rain_kernel_ms"] / out["surrogate"]["rain_kernel_ms"],
            "network_fraction": out["surrogate"]["network_fraction"],
            "fallback_fraction_of_network_cells": out["surrogate"]["fallback_fraction"],
            "precip_rel_diff": abs(p1 - p0) / max(abs(p0), 1e-30), "steps": steps,
            "water_closure_per_call": {"plain": out["plain"]["water_closure_per_call"],
                                       "surrogate": out["surrogate"]["water_closure_per_call"]},
            "training": json.loads(str(w["summary"])),
            "stats": out["surrogate"]["stats"],
            "note": "two kernels: gating warps pack the active cells (quiet cells gated) into 128-row "
                    "tiles, tcgen05 BF16 inference of process fractions with TMEM accumulators, per-cell "
                    "plain fallback; then the plain fallout sweep"}


# The mountain-wave configuration at full size: 512 x 512 x 80, dx = dy = 1 km, levels
# stretched to 20 km, Agnesi hill, constant N = 0.01 1/s from 288 K, 10 m/s, Rayleigh layer
# above 14 km, 6 acoustic substeps.  dt = 0.5 s: the configured 6 s exceeds the acoustic
# CFL bound of the reference's slow step on these levels (c dt / dz = 0.95 at 0.5 s on the
# 183 m bottom level).  Byte model: 322 FP32 accesses per cell and step (1288 B: the slow
# stages 40 + 9 metric, 18 substeps of 15, 3 stage exits).
C2_BYTES_PER_CELL = 1288


def c2_grid_and_state(gwm, nx=512, ny=512, nz=80, stretch=0.6):
    """Agnesi hill (400 m, 10 km half width), levels eta_k = (exp(a k / nz) - 1) / (exp(a) - 1)
    to 20 km (183 m at the ground, 331 m at the top for a = 0.6 and 80 levels), constant-N
    atmosphere from 288 K with a 10 m/s wind."""
    eta = (np.exp(stretch * np.arange(nz + 1) / nz) - 1.0) / (np.exp(stretch) - 1.0)
    terrain = gwm.build_terrain("agnesi", nx, ny, 1000.0, 1000.0, height=400.0, half_width_x=10000.0,
                                half_width_y=10000.0)
    g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=20000.0, terrain=terrain, eta_interfaces=eta)
    p = gwm.CaseParams(theta_ref=288.0, p_surface=100000.0, u_background=10.0, brunt_vaisala=0.01)
    s = gwm.build_case("stratified_mountain_wave", g, p)
    s["u"][:, :, -1] = s["u"][:, :, 0]
    return g, s


def c2_line(gwm, torch, stream, dist, world, steps=10, warmup=3, n=512, tiles=None):
    """The mountain-wave configuration: device-timed throughput and its roofline on the
    1288 B/cell model (tiles chosen by timing, the acoustic substep's candidates charged
    their column reference, see Model.autotune; or fixed by ``tiles``, kernel -> rows)."""
    g, s = c2_grid_and_state(gwm, n, n)
    uref = s["u"].astype(np.float64).mean(axis=(1, 2))
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=0.5, fast_substeps=6))
    cells = g.nx * g.ny * g.nz
    with gwm.Model(g, spec) as m:
        m.set_stream(stream.cuda_stream)
        m.upload(s)
        m.set_damping(14000.0, 0.05, u_ref=uref)
        if tiles:
            for kernel, rows in tiles.items():
                m.set_tile(kernel, rows)
            m.tile_times = {}
            tiles = {k: m.get_tile(k) for k in ("slow_stage", "fast_substep", "tracer_stage")}
        else:
            with torch.cuda.stream(stream):
                tiles = m.autotune(1)
        m.upload(s)
        m.use_graph(True)
        with torch.cuda.stream(stream):
            m.step(warmup)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        m.step(steps)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(t0.elapsed_time(t1), torch, dist, "cuda")
        finite = all(np.isfinite(v) for v in m.budgets().values())
        with torch.cuda.stream(stream):
            m.profile(True)
            m.step(1)
            rep = m.profile_report()
            m.profile(False)
    peak, which = load_peaks()
    achieved = C2_BYTES_PER_CELL * cells * steps / (ms * 1e-3) / 1e9
    return {"workload": f"dry mountain wave, {n}x{n}x80 Agnesi hill, stretched levels to 20 km, N = 0.01, "
                        "Rayleigh layer above 14 km", "dt_s": 0.5, "fast_substeps": 6, "steps": steps,
            "ms_per_step": ms / steps, "value": job_throughput(cells, steps, world, ms), "unit": "cell-updates/s",
            "tile_rows": tiles, "tile_autotune_ms": {k: {str(r): round(t, 4) for r, t in v.items()}
                                                     for k, v in m.tile_times.items()},
            "state_finite": finite,
            "kernel_avg_ms": {k: round(v["avg_ms"], 4) for k, v in rep.items()},
            "kernel_launches_per_step": {k: v["launches"] for k, v in rep.items()},
            "roofline": {"bound": "hbm", "bytes_per_cell_step": C2_BYTES_PER_CELL, "achieved": achieved,
                         "unit": "GB/s", "peak": peak, "peak_source": which, "frac": achieved / peak}}


def ensemble_line(gwm, torch, stream, dist, world, n=64, steps=20, warmup=3):
    """C5: 64 uneven members (nx, ny in [64, 512], nz in {40, 64, 80}; warm bubble, cold
    block, Agnesi mountain wave, moist warm rain) advanced by one captured graph with a
    branch per member; tiles autotuned on the ensemble itself, then `steps` steps from the
    initial states; device-timed throughput in cell updates per second."""
    ens = importlib.import_module("gpu-wm-next_b200.ensemble")
    grids, specs, states, damping, kinds = ens.c5_members(n, seed=5)
    cells = sum(g.nx * g.ny * g.nz for g in grids)
    with ens.build_model(grids, specs, states, damping, concurrent=True) as m:
        m.set_stream(stream.cuda_stream)
        # "some with warm rain and the surrogate": every other moist member takes the
        # learned warm rain (the shipped weights, trained at this dt)
        w = np.load(SURROGATE_WEIGHTS)
        moist = [i for i, k in enumerate(kinds) if k == "moist"]
        for i in moist[::2]:
            m.set_rain_surrogate(w["params"], w["norm"], w["range"], member=i)
        with torch.cuda.stream(stream):
            tiles = m.autotune(2, whole_step=True)  # the members share the GPU: time whole steps
        for i, st in enumerate(states):  # restart from the initial states
            m.upload(st, member=i)
        m.use_graph(True)
        with torch.cuda.stream(stream):
            m.step(warmup)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        m.step(steps)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(t0.elapsed_time(t1), torch, dist, "cuda")
        unstable = {}
        for i in range(n):  # a member whose state went non-finite or non-positive
            try:
                ok = all(np.isfinite(v) for v in m.budgets(member=i).values())
            except RuntimeError:
                ok = False
            if not ok:
                unstable[kinds[i]] = unstable.get(kinds[i], 0) + 1
        finite = not unstable
    return {"members": n, "cells": cells, "steps": steps, "ms_per_step": ms / steps,
            "unstable_members": unstable, "surrogate_members": len(moist[::2]),
            "value": job_throughput(cells, steps, world, ms), "unit": "cell-updates/s",
            "tile_rows": tiles, "tile_autotune_ms_per_step": {k: {str(r): round(t, 2) for r, t in v.items()}
                                                              for k, v in m.tile_times.items()},
            "cases": {k: kinds.count(k) for k in set(kinds)}, "state_finite": finite,
            "note": "one CUDA graph per step with a branch per member; dt 1 s, 4 substeps (4 s is beyond "
                    "the acoustic limit of the reference discretisation on these 250 m levels)"}


def max_over_ranks(x, torch, dist, device):
    """The slowest rank's time: every rank contributes its own device-timed value."""
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(cells_per_rank, steps, world, ms_max):
    """Whole-job cell updates per second: every rank advances its own replica of
    cells_per_rank cells, and the job takes as long as its slowest rank."""
    return cells_per_rank * steps * world / (ms_max * 1e-3)


def end_to_end(gwm, model, g, stream, torch, steps, world, dist):
    sh = g.shapes()
    keys = ("rho", "rho_theta", "u", "v", "w", "qv", "qc", "qr")
    host = {k: torch.empty(sh[k], dtype=torch.float32, pin_memory=True).numpy() for k in keys}
    host["precip"] = torch.empty(sh["precip"], dtype=torch.float64, pin_memory=True).numpy()
    model.download(out=host)
    h2d = sum(host[k].nbytes for k in host)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # device-timed on the model's stream: the span from before the first step's upload to
    # after the last step's download; every step is one host-to-host call (the full state
    # in from pinned host memory, one step, the full state out), whose copies overlap the
    # step's phases on copy streams
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        model.step_host(host, out=host)
    t1.record(stream)
    torch.cuda.synchronize()
    el_ms = max_over_ranks(t0.elapsed_time(t1), torch, dist, "cuda")
    return {"value": job_throughput(g.nx * g.ny * g.nz, steps, world, el_ms), "unit": "cell-updates/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
            "note": "full prognostic state copied host->device and back every step through the C-ABI "
                    "(gwm_b200_step_host: the moisture fields go up during the dry step, rho and the "
                    "momenta come down during the tracers and warm rain)"}


if __name__ == "__main__":
    main()
