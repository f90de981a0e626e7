"""Benchmark: LICOM3 baroclinic tracer step on B200.

Metric: tracer cell-steps/s (nx*ny*km physical cells, land included, halo
excluded, both T and S advanced per step) on the 0.1-degree grid
3600 x 2302 x 55, seeded synthetic inputs of that shape (no NetCDF here).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed|both]
                    [--impl ours|reference] [--grid NX NY KM]

One JSON line on rank 0.  Under torchrun each rank advances an independent
replica of the domain on its own GPU (the path has no cross-domain exchange on
one device: replicas only, weak scaling); the timed region is bracketed by a
barrier and a device synchronize and the max over ranks is reported.

Beside the headline (the mixed step, device-resident inputs) the default run
reports the FP64 drop-in, both forms' states compared after 100 steps, the
global tracer content drift over 100 zero-flux steps in both forms, the FP64
step with its diagnostics written, a reduced ensemble and serving run, the
kernels of the next rows, and the CPU baseline.

``--impl reference`` times the reference algorithm on the host cores: the
FP64 CPU restatement (bit-exact with the reference's own tracer.cpp), fed by
the host build of the input generator, never the CUDA library.  Each timed
step is one step of a full-width, full-depth band of the 0.1-degree grid (its
northern rows, with the fold); the whole grid is stepped twice beside it, and
a one-thread rate is measured on a narrower band.
"""
import argparse
import ctypes as C
from math import exp as math_exp, log as math_log
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(REPO, "licom3-hip_b200")
PEAKS = os.path.join(REPO, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# algorithmic bytes per cell-step (compulsory traffic of the whole step, both
# tracers; 2-D/1-D coefficients not counted) and of the fused column kernel:
# at, atb read and written (64), w (8 | 4), face transports uw, vs (16) or the
# U-point means wkd, wkb (8), akt (16 | 8)
STEP_BYTES = {"fp64": 136.0, "mixed": 100.0}
TRACER_KERNEL_BYTES = {"fp64": 104.0, "mixed": 84.0}
# DRAM bytes per cell (read + write) of the column kernel, from one ncu
# --set full capture of a 720x460x55 launch (profiles/); traffic grows with
# the cells, so it scales to the bench's launch
TRACER_KERNEL_TRAFFIC = {"fp64": (1.106355e9 + 0.653346e9) / (720 * 460 * 55),
                         "mixed": (0.963681e9 + 0.646199e9) / (720 * 460 * 55)}


def ICESNOW_BYTES_PER_POINT(km):
    """Sea-ice adjustment, per point of the domain (halo included): T read at
    every level, KMT read, QICE written; S and T are written only where water
    froze."""
    return 8.0 * km + 4.0 + 8.0


def load_package():
    if "licom3_hip_b200" in sys.modules:
        return sys.modules["licom3_hip_b200"]
    spec = importlib.util.spec_from_file_location("licom3_hip_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["licom3_hip_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-turb", action="store_true",
                    help="skip the timing of the turbulence closure and the momentum friction")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                    help="both: the mixed step as the headline, with the FP64 drop-in measured beside it")
    ap.add_argument("--grid", type=int, nargs=3, default=[3600, 2302, 55])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0, help="end-to-end steps (default: --steps)")
    ap.add_argument("--workload", default="tracer", choices=["tracer", "ensemble", "serving"],
                    help="tracer: the 0.1-degree step (default); ensemble: 64 perturbed members of the 1-degree "
                         "grid in one batch; serving: Poisson-arriving regional requests")
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=20.0, help="serving: mean arrivals per second")
    ap.add_argument("--accuracy-steps", type=int, default=100,
                    help="steps after which the mixed state is compared with the FP64 state")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the conservation, diagnostics, ensemble and serving figures of the default run")
    ap.add_argument("--hypsometry", type=int, default=0, choices=[0, 1],
                    help="ocean depths of the generator: 0 = linear in the land field (mostly shallow), "
                         "1 = the global ocean's area-depth curve (mean depth about 3.7 km)")
    ap.add_argument("--band-rows", type=int, default=0,
                    help="CPU baseline: physical rows of the band a timed host step advances (default ny/16)")
    return ap.parse_args()


def workload(args):
    nx, ny, km = args.grid
    deep = km >= 50
    return dict(nx=nx, ny=ny, km=km, umax=0.3 if deep else 0.1, dz_top=5.0 if deep else 10.0,
                dz_bot=300.0 if deep else 250.0, cap_north=0, forced=1, hypsometry=args.hypsometry)


HYPSOMETRY = {0: "KMT linear in the land field above its 30 % threshold (3..km levels, mostly shallow)",
              1: "the global ocean's area-depth curve (mean ocean depth about 3.7 km)"}


def bathymetry(syn, km):
    """Wet share of the grid's cell-levels and of the ocean columns' levels."""
    import numpy as np
    kmt = syn.field("KMT")[2:-2, 2:-2]
    ocean = kmt[kmt > 0]
    return {"wet_cell_levels_frac": round(float(kmt.mean()) / km, 4),
            "ocean_mean_kmt": round(float(ocean.mean()), 2) if ocean.size else 0.0,
            "land_columns_frac": round(float((kmt == 0).mean()), 4)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return None


def host_synth(args):
    """The bench configuration's inputs from the host build of the generator
    (oracle/liblicom_synth_host.so): the CPU baseline never loads the CUDA
    library."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle
    nx, ny, km = args.grid
    w = workload(args)
    return pyoracle, pyoracle.HostSynth(nx, ny, km, **{k: v for k, v in w.items() if k not in ("nx", "ny", "km")})


def band_rate(pyoracle, hs, rows, threads, steps, warmup):
    """The FP64 CPU restatement (OpenMP over `threads` host cores, diagnostics
    off as in the GPU headline) on the northern band of `rows` physical rows
    of the configuration (full width and depth, tripole fold included).
    Returns (cell-steps/s, seconds per step); the time is that of the
    tracer_ calls alone."""
    o = pyoracle.Oracle(hs.nx, rows, hs.km, hs.params, threads=threads, diagnostics=0)
    hs.fill(o, rows=rows + 4)
    for _ in range(warmup):
        o.step_timed(1)
    t = sum(o.step_timed(1) for _ in range(steps))
    del o
    cells = hs.nx * rows * hs.km
    return cells * steps / t, t / steps


def cpu_baseline(args, steps, warmup, full_grid=False):
    """CPU baseline on the host cores (the oracle port; see run_reference)."""
    pyoracle, hs = host_synth(args)
    cores = cpu_cores()
    nx, ny, km = args.grid
    rows = args.band_rows or max(8, ny // 16)
    rate, sec = band_rate(pyoracle, hs, rows, cores, steps, warmup)
    rate1, _ = band_rate(pyoracle, hs, 8, 1, 1, 1)
    pyoracle.Oracle(8, 8, 3, hs.params, threads=cores)   # restore the thread count
    cb = {"value": rate, "unit": "cell-steps/s", "cores": cores, "kind": "port", "cpu_model": cpu_model(),
          "sample": "northern band %dx%dx%d of the %dx%dx%d grid (full width and depth, fold included), "
                    "%d step(s) after %d warm-up, diagnostics off, time inside tracer_ only"
                    % (nx, rows, km, nx, ny, km, steps, warmup),
          "ms_per_sample_step": sec * 1e3,
          "one_thread": {"value": rate1, "sample": "northern band %dx8x%d, 1 step after 1 warm-up" % (nx, km)}}
    if full_grid:
        need = 36 * (nx + 4) * (ny + 4) * km * 8
        avail = host_mem_available()
        if avail is not None and avail < need:
            cb["full_grid"] = {"skipped": "host memory %.0f GB available, %.0f GB needed" % (avail / 1e9, need / 1e9)}
        else:
            o = pyoracle.Oracle(nx, ny, km, hs.params, threads=cores, diagnostics=0)
            t0 = time.perf_counter()
            hs.fill(o)
            t_fill = time.perf_counter() - t0
            t = o.step_timed(2)
            del o
            cb["full_grid"] = {"value": nx * ny * km * 2 / t, "steps": 2, "ms_per_step": t / 2 * 1e3,
                               "input_generation_s": t_fill, "cores": cores}
    return cb


def reference_own_code_rate():
    """The reference's own tracer.cpp compiled for the CPU through the HIP
    stand-in (oracle/_ref), one 36x40x55 block on one core, when it was built:
    the stand-in runs every GPU thread of a launch in turn, so this is a
    measure of that emulation, reported beside the port."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle
    if not pyoracle.reference_available():
        return None
    hs = pyoracle.HostSynth(36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0)
    o = pyoracle.Oracle(36, 40, 55, hs.params, threads=1)
    hs.fill(o)
    ref = pyoracle.Reference(hs.params)
    ref.load({n: o.get(n) for n in pyoracle.INPUTS})
    ref.tracer_call(0)
    n = 5
    t0 = time.perf_counter()
    for s in range(n):
        ref.tracer_call(s + 1)
    t = (time.perf_counter() - t0) / n
    t_port = o.step_timed(n) / n
    return {"value": 36 * 40 * 55 / t, "unit": "cell-steps/s", "cores": 1,
            "sample": "one 36x40x55 block (the reference's compiled size), %d steps" % n,
            "port_same_block_one_thread": 36 * 40 * 55 / t_port}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value, local):
    """Max of a per-rank value over all ranks (NCCL on the GPUs; gloo on CPU)."""
    if pg is None:
        return value
    import torch
    dev = "cpu" if pg.get_backend() == "gloo" else "cuda:%d" % local
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        pg.barrier()
        if pg.get_backend() != "gloo":
            import torch
            torch.cuda.synchronize(local)


def whole_job_rate(cells_per_rank, steps, world, max_ms):
    """cell-steps/s of the whole job: every rank advanced its own replica of
    cells_per_rank cells for `steps` steps, and the job lasted as long as the
    slowest rank's device time max_ms."""
    return cells_per_rank * steps * world / (max_ms * 1e-3)


def run_reference(args):
    """The reference arm: the reference algorithm on the host cores, on the
    same configuration, metric and unit as this build's arm.  The reference
    has no CPU implementation of this path of its own (its Fortran driver is
    compiled out and missing); the FP64 restatement is bit-exact with its
    tracer.cpp compiled for the CPU, whose HIP stand-in runs far slower than
    real CPU code (reported as reference_own_code), so the restatement is the
    timed baseline.  Rank 0 alone runs; other ranks exit without work."""
    world, rank, local, pg = dist_setup(args)
    if rank == 0:
        nx, ny, km = args.grid
        cb = cpu_baseline(args, args.steps, args.warmup, full_grid=True)
        rate = cb["value"]
        line = {"impl": "reference", "metric": "tracer cell-steps/s (0.1deg 3600x2302x55)", "value": rate,
                "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": cb["ms_per_sample_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generators with the configuration's shapes and distributions)",
                "config": config_of(args, world),
                "cpu_baseline": cb,
                "reference_own_code": reference_own_code_rate(),
                "e2e": {"value": rate, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def config_of(args, world):
    """The workload, identical in both arms (the arithmetic is in dtype)."""
    nx, ny, km = args.grid
    cells = nx * ny * km
    return {"workload": "0.1deg tracer step %dx%dx%d" % (nx, ny, km), "nx": nx, "ny": ny, "km": km,
            "hypsometry": args.hypsometry, "depths": HYPSOMETRY[args.hypsometry],
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs (~%.0f GB) far larger than L2; no flush" % (cells * 8 * 16 / 1e9)}


def measure(lt, args, pg, world, local, precision, keep_state):
    """One precision on the bench grid: device-resident throughput, the
    column kernel's roofline, end-to-end rate through the C ABI, and the
    final state (host copy) when asked.  The domain is freed on return."""
    nx, ny, km = args.grid
    w = workload(args)
    prec = lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64
    syn = lt.Synth(nx, ny, km, **{k: v for k, v in w.items() if k not in ("nx", "ny", "km")})
    bathy = bathymetry(syn, km)
    dom = syn.domain(precision=prec)
    cells = nx * ny * km

    # ---- device-resident throughput (value)
    dom.step(args.warmup)
    dom.sync()
    barrier(pg, local)
    dom.profile(True)
    n0 = lt.launch_count()
    with ClockSampler(local) as clk:
        dom.step(args.steps)
        dom.sync()
    launches = lt.launch_count() - n0
    barrier(pg, local)
    ms = reduce_max(pg, dom.last_step_ms(), local)
    nprof, phases = dom.phase_ms()
    dom.profile(False)
    value = whole_job_rate(cells, args.steps, world, ms)

    # ---- roofline of the dominant kernel (the fused tracer column kernel)
    hbm, hbm_kind = peaks()
    t_tracer = phases["tracer"] / max(nprof, 1)            # ms per launch
    kbytes = TRACER_KERNEL_BYTES[precision] * cells        # algorithmic bytes per launch
    achieved = kbytes / (t_tracer * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "tracer column kernel", "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm, "peak_kind": hbm_kind,
                "algorithmic_bytes_per_launch": kbytes,
                "traffic": TRACER_KERNEL_TRAFFIC[precision] * cells,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 720x460x55 launch, "
                                  "scaled by cells",
                "step_frac": STEP_BYTES[precision] * cells / (ms / args.steps * 1e-3) / 1e9 / hbm,
                "phase_ms_per_step": {k: v / max(nprof, 1) for k, v in phases.items()}}

    # ---- end to end through the C ABI with host buffers: every step copies
    # that step's surface forcing (6 fields) from pinned host memory and
    # reads the step's fw_norm2 back into pinned host memory.  The
    # asynchronous entry point double-buffers the forcing on the device, so
    # a step's copies overlap the previous step's kernels.
    import torch
    A = (nx + 4) * (ny + 4)
    pinned = torch.empty(6 * A, dtype=torch.float64, pin_memory=True)
    names = ("SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE")
    for m, nm in enumerate(names):
        pinned[m * A:(m + 1) * A] = torch.from_numpy(dom.get(nm).ravel())
    base = pinned.data_ptr()
    ptrs = [base + m * A * 8 for m in range(6)]
    e2e_steps = args.e2e_steps or args.steps
    fw_out = torch.zeros(e2e_steps + 1, dtype=torch.float64, pin_memory=True)
    fw_addr = fw_out.data_ptr()
    dom.step_host_async_ptrs(ptrs, fw_addr)
    dom.sync()
    barrier(pg, local)
    dom.mark(0)
    for i in range(e2e_steps):
        dom.step_host_async_ptrs(ptrs, fw_addr + 8 * (i + 1))
    dom.mark(1)
    dom.sync()
    barrier(pg, local)
    ms_e2e = reduce_max(pg, dom.last_step_ms(), local)
    fw = C.c_double(float(fw_out[e2e_steps]))
    e2e = {"value": whole_job_rate(cells, e2e_steps, world, ms_e2e), "unit": "cell-steps/s",
           "h2d_bytes_per_step": 6 * A * 8, "d2h_bytes_per_step": 8,
           "api": "lt_step_host_async (C ABI), pinned host forcing and fw_norm2, forcing double-buffered on the device"}
    steps_total = args.warmup + args.steps + 1 + e2e_steps
    state = kmt = None
    if keep_state:
        # both forms advance the same steps from the same inputs, then their
        # states are compared
        if steps_total < args.accuracy_steps:
            dom.step(args.accuracy_steps - steps_total)
            steps_total = args.accuracy_steps
        state = dom.get("AT")
        kmt = syn.field("KMT")

    # ---- the sea-ice adjustment that follows each tracer step in the model
    # (icesnow.cpp): its own HBM-bound kernel, timed over repeated launches
    ice = lt.IcesnowParams()
    for _ in range(3):
        dom.icesnow(ice)
    n_ice = 20
    dom.mark(0)
    for _ in range(n_ice):
        dom.icesnow(ice)
    dom.mark(1)
    dom.sync()
    ms_ice = dom.last_step_ms() / n_ice
    ice_bytes = ICESNOW_BYTES_PER_POINT(km) * (nx + 4) * (ny + 4)
    icesnow = {"ms_per_launch": ms_ice, "algorithmic_bytes_per_launch": ice_bytes,
               "achieved_gbs": ice_bytes / (ms_ice * 1e-3) / 1e9,
               "frac": ice_bytes / (ms_ice * 1e-3) / 1e9 / hbm, "peak_kind": hbm_kind,
               "share_of_step": ms_ice / (ms / args.steps)}
    dom.close()
    return {"value": value, "ms_per_step": ms / args.steps, "roofline": roofline, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk.summary(), "fw_norm2": fw.value, "state": state, "kmt": kmt,
            "steps_total": steps_total, "icesnow": icesnow, "bathymetry": bathy}


def deep_ocean_figures(lt, args, steps=5, warmup=3, accuracy_steps=100):
    """The bench grid with the global ocean's area-depth curve instead of
    the linear depth map (--hypsometry 1): most columns are abyssal, so the
    column march runs through most levels of most tiles.  Device-resident
    step rate of both forms (inputs far larger than L2), the same timing as
    the headline, and the mixed form's largest difference from the FP64 form
    after accuracy_steps steps."""
    nx, ny, km = args.grid
    w = dict(workload(args), hypsometry=1)
    cells = nx * ny * km
    hbm, hbm_kind = peaks()
    out = {"hypsometry": 1, "depths": HYPSOMETRY[1], "steps": steps, "warmup": warmup}
    states = {}
    for precision in ("fp64", "mixed"):
        syn = lt.Synth(nx, ny, km, **{k: v for k, v in w.items() if k not in ("nx", "ny", "km")})
        out["bathymetry"] = bathymetry(syn, km)
        kmt = syn.field("KMT")
        dom = syn.domain(precision=lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64)
        dom.step(warmup)
        dom.sync()
        dom.profile(True)
        with ClockSampler(0) as clk:
            dom.step(steps)
            dom.sync()
        ms = dom.last_step_ms() / steps
        nprof, ph = dom.phase_ms()
        dom.profile(False)
        # both forms advance to the same step count, then their states are compared
        dom.step(accuracy_steps - warmup - steps)
        states[precision] = dom.get("AT")
        dom.close()
        t_col = ph["tracer"] / max(nprof, 1)
        out[precision] = {"value": cells / (ms * 1e-3), "ms_per_step": ms,
                          "step_frac": STEP_BYTES[precision] * cells / (ms * 1e-3) / 1e9 / hbm,
                          "column_kernel_frac": TRACER_KERNEL_BYTES[precision] * cells / (t_col * 1e-3) / 1e9 / hbm,
                          "peak_kind": hbm_kind,
                          "phase_ms_per_step": {k: v / max(nprof, 1) for k, v in ph.items()},
                          "clocks": clk.summary()}
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    import numpy as np
    wet = (np.arange(km)[:, None, None] < kmt[None])[:, 2:-2, 2:-2]
    a, g = states["fp64"][:, :, 2:-2, 2:-2], states["mixed"][:, :, 2:-2, 2:-2]
    out["accuracy"] = {"max_abs_dT_K": float(np.abs(a[0] - g[0])[wet].max()),
                       "max_abs_dS_psu": float(np.abs(a[1] - g[1])[wet].max()) * 1e3,
                       "steps": accuracy_steps, "bound": {"T_K": 1e-4, "S_psu": 1e-5},
                       "against": "the FP64 drop-in on the same inputs (bit-exact with the oracle)"}
    return out


def measure_readyc(lt, args, precision):
    """The kernels of the next rows on a 720x460x55 patch of the bench
    configuration (their inputs are built on the host; 1/25 of the 0.1-degree
    columns): the Canuto closure (lt_turb) that produces the step's mixing,
    with the stand-in closure tables, and the momentum biharmonic friction
    (lt_hdiffu_del4).  Device time per launch over 10 launches after 3
    untimed ones."""
    sys.path.insert(0, os.path.join(REPO, "tests"))   # the stand-in closure and friction inputs
    import turb_synth
    nx, ny, km = 720, 460, 55
    w = workload(args)
    syn = lt.Synth(nx, ny, km, **{k: v for k, v in w.items() if k not in ("nx", "ny", "km")})
    f = {n: syn.field(n) for n in ("AT", "KMT", "DZP")}
    inp = turb_synth.inputs(f["AT"], f["KMT"], f["DZP"], seed=3)
    tab = lt.TurbTab(turb_synth.tables())
    dom = syn.domain(precision=lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64)
    for n, a in inp.items():
        dom.set(n, a)
    for _ in range(3):
        dom.turb(tab, ncc=4, dfricmx=0.1)
    dom.sync()
    reps = 10
    dom.mark(0)
    for _ in range(reps):
        dom.turb(tab, ncc=4, dfricmx=0.1)
    dom.mark(1)
    dom.sync()
    ms = dom.last_step_ms() / reps
    # the momentum biharmonic friction on the same patch (readyc.cpp:1754-1775)
    import del4u_synth
    fm = {n: syn.field(n) for n in ("HUN", "HUE", "HTW", "HTS", "DXU", "DYU", "TAREA_R", "KMU")}
    mom = del4u_synth.coefficients(fm)
    mom.update(del4u_synth.velocities(fm["KMU"], km, seed=3))
    for n, a in mom.items():
        dom.set(n, a)
    am = 4.0 * syn.params.ah
    for _ in range(3):
        dom.hdiffu_del4(am, 2.6e-3)
    dom.sync()
    dom.mark(0)
    for _ in range(reps):
        dom.hdiffu_del4(am, 2.6e-3)
    dom.mark(1)
    dom.sync()
    ms_d = dom.last_step_ms() / reps
    dom.close()
    tab.close()
    cells = nx * ny * km
    full = args.grid[0] * args.grid[1] * args.grid[2]
    hbm, hbm_kind = peaks()
    # per cell: up, vp read (16), dlu, dlv read and written (32), the drag
    # speed written (8); the 2-D coefficients are shared by the levels
    d_bytes = 56.0 * cells
    turb = {"grid": "%dx%dx%d patch of the bench grid" % (nx, ny, km), "ms_per_launch": ms,
            "cells_per_s": cells / (ms * 1e-3), "ms_scaled_to_bench_grid": ms * full / cells,
            "bound": "fp64 arithmetic (table-index logarithms, atan, sin, cos, acosh, divisions)",
            "tables": "stand-ins on the reference's table grids"}
    del4u = {"grid": turb["grid"], "ms_per_launch": ms_d, "cells_per_s": cells / (ms_d * 1e-3),
             "ms_scaled_to_bench_grid": ms_d * full / cells, "algorithmic_bytes_per_launch": d_bytes,
             "achieved_gbs": d_bytes / (ms_d * 1e-3) / 1e9, "frac": d_bytes / (ms_d * 1e-3) / 1e9 / hbm,
             "peak_kind": hbm_kind}
    return turb, del4u


def measure_conservation(lt, args, precision, steps, diagnostics=False):
    """Global tracer content (f64, fixed-order tree) before and after `steps`
    steps with zero surface flux and land rows capping the north and south
    edges (the fold averages the top row with its mirror, which moves content
    by design), on the bench grid; with diagnostics on, the step also writes
    the reference's diagnostic fields.  Returns the relative drift of T and S
    and the device time per step."""
    import numpy as np
    nx, ny, km = args.grid
    w = dict(workload(args), forced=0, cap_north=3, cap_south=3)
    syn = lt.Synth(nx, ny, km, **{k: v for k, v in w.items() if k not in ("nx", "ny", "km")})
    dom = syn.domain(precision=lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64, diagnostics=diagnostics)
    c0 = np.array(dom.tracer_content())
    dom.mark(0)
    dom.step(steps)
    dom.mark(1)
    dom.sync()
    ms = dom.last_step_ms() / steps
    c1 = np.array(dom.tracer_content())
    dom.close()
    rel = np.abs(c1 - c0) / np.abs(c0)
    return {"T": float(rel[0]), "S": float(rel[1])}, ms


def ensemble_figures(lt, nmem, steps, warmup, check):
    """Configuration 3: nmem members of the 1-degree 360x218x30 grid (T
    perturbed by seeded N(0, 0.01 K) per member) advanced as ONE batch (one
    continuity and one persistent column launch per step, CUDA-graph replay,
    autotuned launch shape), mixed precision.  The first `check` members are
    compared with their FP64 runs (the FP64 drop-in is bit-exact with the
    oracle on this grid)."""
    import numpy as np
    nx, ny, km = 360, 218, 30
    syns = [lt.Synth(nx, ny, km, member=m + 1, tpert=0.01, forced=1, cap_north=0) for m in range(nmem)]
    doms = [s.domain(precision=lt.PREC_MIXED) for s in syns]
    batch = lt.Batch(doms)
    cfg = batch.autotune(trial_steps=2)
    batch.step(warmup)
    batch.sync()
    n0 = lt.launch_count()
    with ClockSampler(0) as clk:
        batch.step(steps)
        batch.sync()
    launches = lt.launch_count() - n0
    ms = batch.last_ms()
    value = whole_job_rate(nx * ny * km * nmem, steps, 1, ms)
    worst_t = worst_s = 0.0
    for s, d in list(zip(syns, doms))[:check]:
        ref = s.domain(precision=lt.PREC_FP64)
        ref.step(warmup + steps)
        ref.sync()
        kmt = s.field("KMT")
        wet = (np.arange(km)[:, None, None] < kmt[None])[:, 2:-2, 2:-2]
        a, g = ref.get("AT")[:, :, 2:-2, 2:-2], d.get("AT")[:, :, 2:-2, 2:-2]
        worst_t = max(worst_t, float(np.abs(a[0] - g[0])[wet].max()))
        worst_s = max(worst_s, float(np.abs(a[1] - g[1])[wet].max()) * 1e3)
        ref.close()
    batch.close()
    for d in doms:
        d.close()
    return {"members": nmem, "grid": "%dx%dx%d" % (nx, ny, km), "value": value, "unit": "cell-steps/s",
            "ms_per_step": ms / steps, "steps": steps, "warmup": warmup, "launch_shape": cfg,
            "gpu_launches": launches, "clocks": clk.summary(),
            "accuracy": {"max_abs_dT_K": worst_t, "max_abs_dS_psu": worst_s, "steps": warmup + steps,
                         "members_checked": check, "against": "each checked member's FP64 run"}}


def serving_figures(lt, requests, rate):
    """Configuration 4: Poisson-arriving requests (mean `rate` per second) for
    closed regional domains, horizontal area log-uniform from 128x128 to
    1200x900 (4:3, km 30 below the geometric middle of the range, 55 above),
    10..200 steps each, mixed precision, through the request server
    (admission by free HBM, resident state, continuous batching)."""
    import random
    rng = random.Random(2024)
    srv = lt.Server(precision=lt.PREC_MIXED, chunk_steps=10)
    a_lo, a_hi = 128 * 128, 1200 * 900
    t, t0 = 0.0, srv.clock()
    for r in range(requests):
        t += rng.expovariate(rate)
        area = math_exp(rng.uniform(math_log(a_lo), math_log(a_hi)))
        nx = max(64, int(round((area * 4.0 / 3.0) ** 0.5)))
        ny = max(48, int(round(area / nx)))
        km = 30 if area < (a_lo * a_hi) ** 0.5 else 55
        srv.submit(nx, ny, km, rng.randint(10, 200), arrival=t0 + t, seed=1000 + r,
                   ew_cyclic=0, tripole=0, forced=1)
    n0 = lt.launch_count()
    with ClockSampler(0) as clk:
        srv.drain()
    st = srv.stats()
    srv.close()
    return {"requests": requests, "rate_per_s": rate, "value": st["cell_steps"] / st["wall_s"],
            "unit": "cell-steps/s", "latency_s": {"p50": st["latency_p50"], "p99": st["latency_p99"],
                                                  "max": st["latency_max"]},
            "device_busy_cell_steps_per_s": st["cell_steps"] / st["busy_s"] if st["busy_s"] else None,
            "server": st, "gpu_launches": lt.launch_count() - n0, "clocks": clk.summary()}


def run_ours(args):
    world, rank, local, pg = dist_setup(args)
    lt = load_package()
    lt.set_device(local)
    nx, ny, km = args.grid
    cells = nx * ny * km
    both = args.precision == "both"
    precs = ["fp64", "mixed"] if both else [args.precision]
    res = {p: measure(lt, args, pg, world, local, p, keep_state=both and rank == 0) for p in precs}
    main = "mixed" if both else args.precision
    r = res[main]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, 2, 1)

    if rank == 0:
        line = {"metric": "tracer cell-steps/s (0.1deg 3600x2302x55)",
                "value": r["value"], "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if main == "fp64" else "f32 arithmetic, f64 state",
                "data": "synthetic (seeded generators with the configuration's shapes and distributions)",
                "config": config_of(args, world),
                "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "gpu_launches": r["gpu_launches"],
                "clocks": r["clocks"], "fw_norm2": r["fw_norm2"], "icesnow": r["icesnow"],
                "bathymetry": r["bathymetry"]}
        if not args.no_turb and world == 1:
            line["turb"], line["hdiffu_del4"] = measure_readyc(lt, args, main)
        if both:
            import numpy as np
            f = res["fp64"]
            wet = (np.arange(km)[:, None, None] < f["kmt"][None])[:, 2:-2, 2:-2]
            a, g = f["state"][:, :, 2:-2, 2:-2], r["state"][:, :, 2:-2, 2:-2]
            line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "e2e": f["e2e"]["value"],
                            "roofline_frac": f["roofline"]["frac"], "step_frac": f["roofline"]["step_frac"],
                            "phase_ms_per_step": f["roofline"]["phase_ms_per_step"], "clocks": f["clocks"]}
            line["mixed_over_fp64"] = r["value"] / f["value"]
            line["accuracy"] = {"max_abs_dT_K": float(np.abs(a[0] - g[0])[wet].max()),
                                "max_abs_dS_psu": float(np.abs(a[1] - g[1])[wet].max()) * 1e3,
                                "steps": r["steps_total"], "bound": {"T_K": 1e-4, "S_psu": 1e-5},
                                "against": "the FP64 drop-in on the same inputs (bit-exact with the oracle)"}
        if both and world == 1 and not args.no_extras:
            hbm, hbm_kind = peaks()
            steps_c = args.accuracy_steps
            drift_m, _ = measure_conservation(lt, args, "mixed", steps_c)
            drift_f, ms_diag = measure_conservation(lt, args, "fp64", steps_c, diagnostics=True)
            line["conservation"] = {"steps": steps_c, "bound": 1e-13, "mixed": drift_m, "fp64": drift_f,
                                    "workload": "the bench grid with zero surface flux and land rows capping "
                                                "the north and south edges"}
            diag_bytes = STEP_BYTES["fp64"] + 104.0
            line["fp64_diagnostics_on"] = {
                "value": cells / (ms_diag * 1e-3), "ms_per_step": ms_diag, "steps": steps_c,
                "bytes_per_cell_step": diag_bytes,
                "step_frac": diag_bytes * cells / (ms_diag * 1e-3) / 1e9 / hbm, "peak_kind": hbm_kind,
                "writes": "ax, ay, az, dz, tend, dt_diff (both tracers) and penetrate, as tracer.cpp always does",
                "workload": "the conservation run above (zero surface flux, capped edges)"}
            if args.hypsometry == 0:
                line["deep_ocean"] = deep_ocean_figures(lt, args)
            line["ensemble"] = ensemble_figures(lt, args.members, 100, 3, check=4)
            line["ensemble"]["reduced"] = "4 of %d members checked against their FP64 runs" % args.members
            line["serving"] = serving_figures(lt, 60, args.rate)
            line["serving"]["reduced"] = "60 requests (the full workload is 200: bench.py --workload serving)"
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def run_ensemble(args):
    """Configuration 3 on its own line (bench.py --workload ensemble)."""
    lt = load_package()
    lt.set_device(0)
    e = ensemble_figures(lt, args.members, args.steps, args.warmup, check=args.members)
    hbm, hbm_kind = peaks()
    cells = 360 * 218 * 30
    line = {"metric": "ensemble tracer cell-steps/s (%d x 1deg 360x218x30, MIXED, one batch)" % args.members,
            "value": e["value"], "unit": "cell-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": e["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 arithmetic, f64 state", "data": "synthetic (seeded generators, perturbed members)",
            "config": {"workload": "ensemble %d x 360x218x30" % args.members, "members": args.members,
                       "launch_shape": e["launch_shape"], "l2": "%.1f GB resident, far larger than L2" % (
                           args.members * 66.8e9 / 4.56e8 * cells / 1e9)},
            "roofline": {"bound": "hbm", "achieved": e["value"] * STEP_BYTES["mixed"] / 1e9, "peak": hbm,
                         "unit": "GB/s", "frac": e["value"] * STEP_BYTES["mixed"] / 1e9 / hbm, "peak_kind": hbm_kind,
                         "basis": "whole step, 100 B per cell-step"},
            "accuracy": e["accuracy"], "gpu_launches": e["gpu_launches"], "clocks": e["clocks"],
            "cpu_baseline": None, "e2e": None}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """Configuration 4 on its own line (bench.py --workload serving)."""
    lt = load_package()
    lt.set_device(0)
    sv = serving_figures(lt, args.requests, args.rate)
    line = {"metric": "serving tracer cell-steps/s and latency (Poisson %.0f/s, regional 128x128..1200x900)" % args.rate,
            "value": sv["value"], "unit": "cell-steps/s", "n_gpus": 1, "steps": None, "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 arithmetic, f64 state", "data": "synthetic (seeded generators, seeded arrivals)",
            "config": {"workload": "serving %d requests" % args.requests, "rate_per_s": args.rate,
                       "chunk_steps": 10},
            "latency_s": sv["latency_s"], "device_busy_cell_steps_per_s": sv["device_busy_cell_steps_per_s"],
            "server": sv["server"], "gpu_launches": sv["gpu_launches"], "clocks": sv["clocks"],
            "cpu_baseline": None, "e2e": None}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
