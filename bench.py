"""Benchmark: six-face cubed-sphere MHD step on B200 (plain FP64 path).

Workload (the production-size configuration): each cube face 96 x 96
angular x 192 radial active cells (10,616,832 cells), 4 ghost layers,
log-stretched r in [2.5, 30] R_E, uniform solar wind n = 5 cm^-3,
V = -400 km/s, T = 1e5 K, IMF Bz = -5 nT, aligned 3.1e-5 T Earth dipole
background, seeded +-1 % density noise, CFL 0.3 with the reference Earth
driver's dt rule; outflow radial ghosts.  Synthetic state built on the
device; state arrays are several GB, far larger than L2.

Every 10 steps (--mi-every) the timed run also makes one magnetosphere-
ionosphere coupling update on the device: the field-aligned current on the
FAC shell (Stokes curl of the residual B), its samples on two 192 x 22
polar grids and both hemisphere potential solves.

Metric: cell-updates/s (active cells x steps / device time), whole job
over all ranks.  --gpus N runs N independent replicas (one per GPU, weak
scaling: the step has no inter-GPU exchange).  The line also carries the
standalone ionosphere solve ("mi": 181 x 361 polar cap per hemisphere,
constant Pedersen, rel. residual 1e-8): ms per call on the device, end to
end through the drop-in, and the reference's single-thread CPU solve.

--impl reference times the reference's own CPU step (oracle/_ref, the
unmodified reference library built from its sources, OpenMP on every
physical host core) on the same workload: the same 6 x 96x96x192 case built
through the reference's own set-up API, 1 warm-up step and a bounded number
of timed steps (--ref-steps).  That process loads no library of this
repository.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

NR, N = 192, 96                 # active radial, angular cells per face
KIND_WIND = 2
METRIC = "MHD cell-updates/s on 1 B200 (FP64 plain path)"
# Algorithmic bytes per cell-update of the whole step (state 192 B +
# compacted metric 664 B + background 192 B).
STEP_BYTES_PER_CELL = 1048
# Per-launch algorithmic bytes per face of the flux sweep: cells U~ (5),
# B~ (3), volume (1) counted once per face along the sweep, face Phi~ (1),
# area (1), frame (9), central8 volume (1), B0 face (3) + B0 normal (1),
# written fluid (5) + Maxwell (3) flux: 33 doubles.
FLUX_BYTES_PER_FACE = 33 * 8
# Edge EMF per edge: face velocities (3) and areas (1) of one face family,
# Phi~ (2) and areas (1) of the other, edge frame (6), 2x2 system (5),
# central8 area sums (2), length (1), B0 projections (2), edge density
# cells (1), written EMF (1): 25 doubles (each counted once per edge).
EMF_BYTES_PER_EDGE = 25 * 8
# Measured DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per
# face of a flux launch and per edge of an edge-EMF launch: the mean of the
# three launches of each sweep in an ncu capture of the 6 x 32x32x48 case
# (state arrays larger than L2), divided by the faces or edges one launch
# processes there.  The sweeps stream their arrays, so the traffic of a
# launch of the bench's workload is these figures times its faces or edges.
FLUX_TRAFFIC_BYTES_PER_FACE = 310.6
EMF_TRAFFIC_BYTES_PER_EDGE = 277.7


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()

    def summary(self):
        rows = []
        try:
            with open(self.file.name) as fh:
                for line in fh:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 7:
                        rows.append(parts)
        finally:
            os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[0]) for r in rows if r[0].replace(".", "").isdigit())
        mx = max(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4)
                          if r[3 + q].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(rows)}


def physical_cores():
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return int(n)
    except Exception:
        pass
    return os.cpu_count() or 1


def spawn_ranks(n_gpus):
    """--gpus N without a torchrun environment: start N ranks (one per GPU)
    through torch.distributed.run on 127.0.0.1 and return its exit code."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(n_gpus), "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def dist_init(n_gpus):
    if n_gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist.get_rank(), dist.get_world_size(), dist


def max_over_ranks(value, dist, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist, device):
    if dist is not None:
        import torch
        if device.type == "cuda":
            dist.barrier(device_ids=[device.index])
            torch.cuda.synchronize(device)
        else:
            dist.barrier()


def run_gpu(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    rank, world, dist = dist_init(args.gpus)
    import gamera_cube_b200
    from gamera_cube_b200 import abi
    from gamera_cube_b200.host import HostStorage
    lib = gamera_cube_b200.lib
    nr, n = args.nr, args.n
    cells = 6 * nr * n * n

    t0 = time.time()
    ctx = lib.gcs_context_create_case(KIND_WIND, nr, n, 1000 + rank)
    if not ctx:
        raise RuntimeError(lib.gcs_last_error().decode())
    setup_s = time.time() - t0
    if args.flux_staging and lib.gcs_context_set_flux_staging(ctx, 1) != 0:
        raise RuntimeError("flux staging rejected")
    opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
    lib.gcs_case_options(KIND_WIND, C.byref(opts), C.byref(ts))
    stream = torch.cuda.ExternalStream(lib.gcs_context_stream(ctx), device=device)

    # ionosphere coupling of the step (the reference Earth driver's MI:
    # 192 x 22 per hemisphere, FAC shell 1, 5 S), updated every
    # args.mi_every steps inside the timed region
    mi = None
    if args.mi_every > 0:
        from gamera_cube_b200 import cases
        mi_cfg, mi_startup = cases.mi_dipole_config(), cases.earth_startup()
        mi = C.c_void_p()
        if lib.gcs_context_mi_dipole_create(ctx, C.byref(mi_startup), C.byref(mi_cfg),
                                            C.byref(mi)) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        # the coupling update runs inside the step graph on its device-side
        # cadence: before every mi_every-th step (and the first)
        if lib.gcs_context_set_mi_coupling(ctx, mi, args.mi_every) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())

    def run_steps(count):
        # K graph launches, one per step, no host synchronisation
        if lib.gcs_context_run(ctx, C.byref(opts), C.byref(ts), 0.5, count, 1):
            raise RuntimeError("step run failed")

    # warm-up (also captures the CUDA graph of one step)
    run_steps(args.warmup)
    if lib.gcs_context_sync(ctx) != 0:
        raise RuntimeError("warm-up step failed")

    # ---- timed region: K graph-replayed steps, device time on the stream
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(
        enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    with ClockSampler(local) as clocks:
        start.record(stream)
        run_steps(args.steps)
        stop.record(stream)
        torch.cuda.synchronize(device)
    barrier(dist, device)
    if lib.gcs_context_sync(ctx) != 0:
        raise RuntimeError("a timed step failed")
    ms_local = start.elapsed_time(stop)
    ms = max_over_ranks(ms_local, dist, device)
    total_cells = sum_over_ranks(float(cells), dist, device)
    value = total_cells * args.steps / (ms * 1e-3)

    # ---- per-stage device times (CUDA events around each stage, same
    # stream, no graph) for the roofline of the dominant kernel
    lib.gcs_context_set_profiling(ctx, 1)
    prof_steps = max(2, min(args.steps, 5))
    barrier(dist, device)
    if lib.gcs_context_run(ctx, C.byref(opts), C.byref(ts), 0.5, prof_steps, 0):
        raise RuntimeError("profiled run failed")
    stage_ms = (C.c_double * 16)()
    stage_calls = (C.c_longlong * 16)()
    nst = lib.gcs_context_stage_times(ctx, stage_ms, stage_calls, 16)
    lib.gcs_context_set_profiling(ctx, 0)
    stages = {lib.gcs_stage_name(q).decode(): stage_ms[q] / prof_steps
              for q in range(nst)}
    step_ms_prof = sum(stages.values())
    dom = max(stages, key=stages.get)
    faces_per_dir = 6 * (nr * n * n + n * n)          # ~ faces of one family
    edges_per_dir = 6 * (nr * (n + 1) * (n + 1))
    if dom == "flux":
        alg = 3 * faces_per_dir * FLUX_BYTES_PER_FACE
    elif dom == "edge_emf":
        alg = 3 * edges_per_dir * EMF_BYTES_PER_EDGE
    else:
        alg = cells * STEP_BYTES_PER_CELL
    traffic = None
    if dom == "flux":
        traffic = faces_per_dir * FLUX_TRAFFIC_BYTES_PER_FACE
    elif dom == "edge_emf":
        traffic = edges_per_dir * EMF_TRAFFIC_BYTES_PER_EDGE
    per_launch_ms = stages[dom] / 3.0 if dom in ("flux", "edge_emf") else stages[dom]
    hbm, peak_kind = peaks()
    achieved = (alg / 3.0 if dom in ("flux", "edge_emf") else alg) / (
        per_launch_ms * 1e-3) / 1e9

    # ---- end to end through the drop-in step with pinned host buffers
    act = (C.c_size_t * 3)()
    g = C.c_size_t()
    lib.gcs_context_dims(ctx, act, C.byref(g))
    hs = HostStorage(list(act), g.value, pinned=True, scratch=False)
    if lib.gcs_context_download_state(ctx, hs.storage, 0) != 0:
        raise RuntimeError("download failed")
    dtv, ratio = C.c_double(), C.c_double()
    lib.gcs_context_params(ctx, C.byref(dtv), C.byref(ratio), None, None)
    e2e_steps = max(1, min(args.steps, 3))
    barrier(dist, device)
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        if lib.gcs_context_advance_host(ctx, hs.storage, C.byref(opts), 0.5,
                                        dtv.value) != 0:
            raise RuntimeError("drop-in step failed")
    torch.cuda.synchronize(device)
    e2e_s = max_over_ranks(time.perf_counter() - t1, dist, device)
    barrier(dist, device)
    e2e_value = total_cells * e2e_steps / e2e_s

    # the same drop-in call in resident mode: the device copy of the state
    # stays authoritative between calls (uploaded by the first call), each
    # call uploads its step parameters and reads back the step status
    if lib.gcs_context_set_resident(ctx, 1) != 0:
        raise RuntimeError("resident mode rejected")
    if lib.gcs_context_advance_host(ctx, hs.storage, C.byref(opts), 0.5, dtv.value) != 0:
        raise RuntimeError("drop-in step failed")
    res_steps = max(1, min(args.steps, 10))
    barrier(dist, device)
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    for _ in range(res_steps):
        if lib.gcs_context_advance_host(ctx, hs.storage, C.byref(opts), 0.5,
                                        dtv.value) != 0:
            raise RuntimeError("resident drop-in step failed")
    torch.cuda.synchronize(device)
    res_s = max_over_ranks(time.perf_counter() - t1, dist, device)
    barrier(dist, device)
    lib.gcs_context_set_resident(ctx, 0)
    e2e_resident = total_cells * res_steps / res_s

    mi_solo = run_mi(lib, torch, device, args.mi_solves) if args.mi_solves > 0 else None
    bulk = run_bulk(lib, torch, device, args, dist) if args.bulk else None
    earth = run_earth(lib, torch, device, args, dist, ctx) if args.earth_steps > 0 else None
    # the ensemble needs most of the GPU's memory: free the production run first
    had_mi = mi is not None
    if mi is not None:
        lib.gcs_context_set_mi_coupling(ctx, None, 0)
        lib.gamera_cs_mi_dipole_destroy(mi)
        mi = None
    lib.gcs_context_destroy(ctx)
    ctx = None
    ens = run_ensemble(lib, torch, device, args, dist, rank) if args.ens_steps > 0 else None
    c3 = run_c3(lib, args) if args.c3_steps > 0 else None

    result = None
    if rank == 0:
        clk = clocks.summary()
        launches_per_step = 24 + (7 if had_mi else 0)
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "cell-updates/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded solar wind + dipole, built on the device)",
            "config": {"workload": workload_name(nr, n),
                       "faces": 6, "angular": n, "radial": nr,
                       "cells_per_gpu": cells, "ghost": 4,
                       "graph": "one CUDA graph per step, device-side dt and "
                                "coupling cadence",
                       "mi_coupling": ("none" if not had_mi else
                                       "inside the step graph every %d steps: shell "
                                       "FAC curl + polar sampling + 2 hemisphere PCG "
                                       "solves, 192 x 22 per hemisphere" % args.mi_every),
                       "l2": "state arrays larger than L2 (no flush needed)",
                       "parallelism": "replicas x%d" % world,
                       "setup_s": round(setup_s, 2)},
            "gpu_launches": launches_per_step * args.steps,
            "gpu_launches_note": "24 kernels per step graph + 7 of the ionosphere "
                                 "coupling in every step's graph (cadence, 4 FAC "
                                 "kernels, 1 two-hemisphere solve, check), which "
                                 "return at once on steps where the update is not "
                                 "due; the standalone solves under \"mi\" are "
                                 "timed separately",
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": hs.bytes_state,
                    "d2h_bytes_per_step": hs.bytes_state,
                    "call": "gcs_context_advance_host (drop-in step, pinned host "
                            "buffers, %d steps)" % e2e_steps,
                    "resident": {"value": e2e_resident, "unit": "cell-updates/s",
                                 "steps": res_steps,
                                 "h2d_bytes_per_step": 56, "d2h_bytes_per_step": 120,
                                 "call": "the same drop-in call in resident mode "
                                         "(gcs_context_set_resident): step parameters "
                                         "up, step status down, state kept on the "
                                         "device"}},
            "roofline": {"bound": "hbm", "kernel": dom,
                         "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6650 GB/s",
                         "traffic": traffic,
                         "traffic_source": None if traffic is None else
                         "ncu DRAM bytes per launch of a 6x32x32x48 capture, scaled "
                         "by faces/edges per launch",
                         "algorithmic_bytes_per_launch": alg / 3.0
                         if dom in ("flux", "edge_emf") else alg,
                         "step_share": stages[dom] / step_ms_prof,
                         "step_hbm_frac": cells * STEP_BYTES_PER_CELL /
                         (ms_local / args.steps * 1e-3) / 1e9 / hbm},
            "stage_ms": {k: round(v, 4) for k, v in stages.items()},
            "flux_sweep": "TMA-staged" if args.flux_staging else "per-face",
        }
        if mi_solo is not None:
            result["mi"] = mi_solo
        if bulk is not None:
            result["fp32_bulk"] = bulk
        if ens is not None:
            result["ensemble"] = ens
        if c3 is not None:
            result["fp32_bulk_c3"] = c3
        if earth is not None:
            result["earth_boundary"] = earth
        if args.cpu_baseline and world == 1:
            result["cpu_baseline"] = cpu_baseline(args)
            if mi_solo is not None:
                result["mi"]["cpu_baseline"] = mi_cpu_baseline()
    if dist is not None:
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result))


def run_bulk(lib, torch, device, args, dist):
    """FP32-bulk variant: the same workload and timing as the main line,
    and its error after 1000 steps against the FP64 path on the
    6 x 32x32x48 wind case (same time levels, gamera_cube_b200.precision)."""
    from gamera_cube_b200 import abi, precision
    nr, n = args.nr, args.n
    ctx = lib.gcs_context_create_case(KIND_WIND, nr, n, 1000)
    if not ctx or lib.gcs_context_set_precision(ctx, 1) != 0:
        raise RuntimeError(lib.gcs_last_error().decode())
    split = lib.gcs_context_bulk_split(ctx)
    opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
    lib.gcs_case_options(KIND_WIND, C.byref(opts), C.byref(ts))
    stream = torch.cuda.ExternalStream(lib.gcs_context_stream(ctx), device=device)
    if lib.gcs_context_run(ctx, C.byref(opts), C.byref(ts), 0.5, args.warmup, 1) != 0:
        raise RuntimeError("bulk warm-up failed")
    lib.gcs_context_sync(ctx)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    start.record(stream)
    if lib.gcs_context_run(ctx, C.byref(opts), C.byref(ts), 0.5, args.steps, 1) != 0:
        raise RuntimeError("bulk run failed")
    stop.record(stream)
    torch.cuda.synchronize(device)
    if lib.gcs_context_sync(ctx) != 0:
        raise RuntimeError("a bulk step failed")
    ms = max_over_ranks(start.elapsed_time(stop), dist, device)
    lib.gcs_context_destroy(ctx)
    cells = sum_over_ranks(float(6 * nr * n * n), dist, device)
    err = precision.compare_bulk(lib, KIND_WIND, 48, 32, 1000)
    worst = max(err[v]["linf"] for v in precision.VARIABLES)
    return {"value": cells * args.steps / (ms * 1e-3), "unit": "cell-updates/s",
            "ms_per_step": ms / args.steps, "fp64_radial_layers": split,
            "radial_layers": nr + 8,
            "error_after_1000_steps": {"workload": "6 x 32x32x48 wind + dipole",
                                       "max_rel_linf": worst,
                                       "per_variable": {v: err[v] for v in
                                                        precision.VARIABLES},
                                       "div_b_bulk": err["div_b_bulk"],
                                       "div_b_fp64": err["div_b_fp64"]},
            "note": "flux/face-velocity/EMF sweeps in FP32 outside the layers "
                    "where |B0| > 8 (those stay FP64); state, face B, CT, "
                    "predictor and recovery FP64"}


def run_c3(lib, args):
    """Precision configuration 6 x 192x192x384 (84.9 M cells): the wind with
    a seeded 20 % sinusoidal density pulse of wavelength 10 R_E
    (V = -450 km/s, n = 5 cm^-3, Bz = -5 nT), args.c3_steps steps of the
    FP32-bulk path against the FP64 path on the same time levels, one
    context on the GPU at a time; per-variable L2/Linf relative errors and
    max |div B| of both, and both wall times per step."""
    from gamera_cube_b200 import precision
    r = precision.compare_bulk_sequential(lib, 3, 384, 192, args.c3_steps, seed=1000)
    r["workload"] = ("6 x 192x192x384 wind + dipole with a 20% density pulse "
                     "(lambda 10 R_E, V = -450 km/s)")
    r["max_rel_linf"] = max(r[v]["linf"] for v in precision.VARIABLES)
    return r


def run_earth(lib, torch, device, args, dist, ctx):
    """The production case stepped with the device Earth radial boundary
    (no-MI wall): radial ghosts from a constant upstream monitor (the case's
    own wind), inner flux trap, wind-driven outer EMF, in the device driver
    loop (gcs_context_run_earth: dt and times on the device, one CUDA graph
    per step)."""
    from gamera_cube_b200 import abi
    opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
    lib.gcs_case_options(KIND_WIND, C.byref(opts), C.byref(ts))
    bnorm = 100000.0 * (4.0e-7 * 3.141592653589793 * 1.67262192369e-21) ** 0.5
    st = (abi.SolarWindState * 1)()
    st[0].density = 5.0
    st[0].pressure = 5.0e6 * 1.380649e-23 * 1.0e5 / (1.67262192369e-21 * 1.0e10)
    st[0].velocity[:] = [-4.0, 0.0, 0.0]
    st[0].magnetic[:] = [0.0, 0.0, -5.0e-9 / bnorm]
    t0 = (C.c_double * 1)(0.0)
    wind = abi.SolarWindSeries()
    wind.count, wind.time, wind.state = 1, t0, st
    wind.reference[:] = [30.0, 0.0, 0.0]
    wind.linear_interpolation = 1
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    b = abi.EarthBoundary()
    b.startup, b.wind = C.pointer(startup), C.pointer(wind)
    b.density_floor, b.pressure_floor, b.cfl = 1e-6, 1e-8, 0.3
    earth = C.c_void_p()
    if lib.gcs_earth_create_case(ctx, C.byref(b), C.byref(earth)) != 0:
        return {"error": lib.gcs_last_error().decode()}
    stream = torch.cuda.ExternalStream(lib.gcs_context_stream(ctx), device=device)
    # driver mode: dt, predictor ratio and the boundary's times on the device,
    # one CUDA graph per step
    ok = lib.gcs_context_run_earth(ctx, earth, C.byref(opts), C.byref(ts), 0.5, 3, 1) == 0
    ok = ok and lib.gcs_context_sync(ctx) == 0
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize()
    start.record(stream)
    ok = ok and lib.gcs_context_run_earth(ctx, earth, C.byref(opts), C.byref(ts), 0.5,
                                          args.earth_steps, 1) == 0
    stop.record(stream)
    stop.synchronize()
    ok = ok and lib.gcs_context_sync(ctx) == 0
    ms = max_over_ranks(start.elapsed_time(stop), dist, device)
    # the same loop with the Earth drivers' post-step pressure control
    # (gamma, 1e-6, 1e-8, c = 10, 1e-3, 1e-7: the production arguments)
    pc = abi.PressureControl(5.0 / 3.0, 1e-6, 1e-8, 10.0, 1e-3, 1e-7)
    ok = ok and lib.gcs_context_set_pressure_control(ctx, None, C.byref(pc)) == 0
    ok = ok and lib.gcs_context_run_earth(ctx, earth, C.byref(opts), C.byref(ts), 0.5, 3, 1) == 0
    ok = ok and lib.gcs_context_sync(ctx) == 0
    barrier(dist, device)
    torch.cuda.synchronize()
    start.record(stream)
    ok = ok and lib.gcs_context_run_earth(ctx, earth, C.byref(opts), C.byref(ts), 0.5,
                                          args.earth_steps, 1) == 0
    stop.record(stream)
    stop.synchronize()
    ok = ok and lib.gcs_context_sync(ctx) == 0
    ms_pc = max_over_ranks(start.elapsed_time(stop), dist, device)
    pc_low, pc_hot = C.c_size_t(), C.c_size_t()
    ok = ok and lib.gcs_context_pressure_control_stats(ctx, C.byref(pc_low), C.byref(pc_hot),
                                                       None, None, 1) == 0
    # thresholds that make both branches work: from the run's own state, the
    # low-density threshold at the 30th percentile of the densities, 1.5 c at
    # the 60th percentile of the sound speeds, the low-density sound speed
    # half the 10th percentile (the rule of the pressure-control tests)
    frame = torch.empty(lib.gcs_analysis_frame_floats(ctx), dtype=torch.float32, device=device)
    ok = ok and lib.gcs_context_analysis_frame(ctx, 5.0 / 3.0, C.c_void_p(frame.data_ptr()),
                                               None) == 0
    torch.cuda.synchronize()
    fv = frame.view(6, 8, -1)
    rho = fv[:, 0].reshape(-1)[::7].double()
    cs = torch.sqrt(5.0 / 3.0 * fv[:, 1].reshape(-1)[::7].double() / rho)

    def quantile(x, f):
        return float(torch.kthvalue(x.cpu(), max(1, int(f * x.numel()))).values)

    pca = abi.PressureControl(5.0 / 3.0, 1e-6, 1e-8, quantile(cs, 0.6) / 1.5,
                              quantile(rho, 0.3), 0.5 * quantile(cs, 0.1))
    del frame, fv, rho, cs
    ok = ok and lib.gcs_context_set_pressure_control(ctx, None, C.byref(pca)) == 0
    barrier(dist, device)
    torch.cuda.synchronize()
    start.record(stream)
    ok = ok and lib.gcs_context_run_earth(ctx, earth, C.byref(opts), C.byref(ts), 0.5,
                                          args.earth_steps, 1) == 0
    stop.record(stream)
    stop.synchronize()
    ok = ok and lib.gcs_context_sync(ctx) == 0
    ms_pca = max_over_ranks(start.elapsed_time(stop), dist, device)
    pca_low, pca_hot = C.c_size_t(), C.c_size_t()
    ok = ok and lib.gcs_context_pressure_control_stats(ctx, C.byref(pca_low),
                                                       C.byref(pca_hot), None, None, 1) == 0
    ok = ok and lib.gcs_context_set_pressure_control(ctx, None, None) == 0
    act = (C.c_size_t * 3)()
    g = C.c_size_t()
    lib.gcs_context_dims(ctx, act, C.byref(g))
    cells = 6 * act[0] * act[1] * act[2]
    total = sum_over_ranks(float(cells), dist, device)
    nbytes = lib.gcs_earth_device_bytes(earth)
    lib.gcs_earth_destroy(earth)
    return {"value": total * args.earth_steps / (ms * 1e-3), "unit": "cell-updates/s",
            "ms_per_step": ms / args.earth_steps, "steps": args.earth_steps, "ok": bool(ok),
            "workload": "6 x %dx%dx%d wind + dipole, device Earth radial boundary (no-MI wall), "
                        "constant upstream monitor" % (act[1], act[2], act[0]),
            "call": "gcs_context_run_earth (device driver loop, one CUDA graph per step)",
            "boundary_device_bytes": nbytes,
            "gpu_launches_per_step": 24 + 18,
            "with_pressure_control": {
                "ms_per_step": ms_pc / args.earth_steps,
                "arguments": "gamma 5/3, floors 1e-6/1e-8, c 10, low density 1e-3, "
                             "low-density sound speed 1e-7",
                "low_density_cells": pc_low.value, "high_sound_speed_cells": pc_hot.value,
                "gpu_launches_per_step": 24 + 18 + 1,
                "active": {
                    "ms_per_step": ms_pca / args.earth_steps,
                    "arguments": "gamma 5/3, floors 1e-6/1e-8, thresholds from the state: "
                                 "low density %.4g, c %.4g, low-density sound speed %.4g"
                                 % (pca.low_density_threshold, pca.light_speed,
                                    pca.low_density_sound_speed),
                    "low_density_cells": pca_low.value,
                    "high_sound_speed_cells": pca_hot.value,
                    "steps": args.earth_steps}}}


ENS_SEED = 2024
ENS_RUNS = 16
TILE_FAMILIES = ["predict", "flux", "face_velocity", "edge_emf", "ct", "update",
                 "recover_cfl"]


def run_ensemble(lib, torch, device, args, dist, rank):
    """Sixteen wind runs drawn from a seed (angular size in {48, 64, 96, 128},
    radial 2n; upstream n, Vx, T, Bz uniform), FP32-bulk, tiles autotuned per
    size, advanced together: one CUDA graph per ensemble step, each run with
    its own device dt.  Value = all runs' active cells x steps / device
    time of the timed steps (CUDA events on the ensemble stream)."""
    from gamera_cube_b200 import abi
    k = ENS_RUNS
    n = (C.c_size_t * k)()
    drv = (abi.WindDriver * k)()
    lib.gcs_ensemble_draw(ENS_SEED, k, n, drv)
    nr = (C.c_size_t * k)(*[2 * x for x in n])
    cfg = abi.EnsembleConfig(k, nr, n, drv, ENS_SEED + 100 * rank, 1, 3, 0.5)
    t0 = time.time()
    ens = lib.gcs_ensemble_create(C.byref(cfg))
    if not ens:
        return {"error": lib.gcs_last_error().decode()}
    setup_s = time.time() - t0
    opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
    lib.gcs_case_options(KIND_WIND, C.byref(opts), C.byref(ts))
    tuning = {}
    for i in range(k):
        if lib.gcs_ensemble_grid_owner(ens, i) != i:
            continue
        ctx = lib.gcs_ensemble_run_context(ens, i)
        best, dflt = (C.c_double * 7)(), (C.c_double * 7)()
        lib.gcs_context_autotune(ctx, C.byref(opts), C.byref(ts), 3, best, dflt)
        tiles = {}
        for f, name in enumerate(TILE_FAMILIES):
            bx, by = C.c_int(), C.c_int()
            lib.gcs_context_tile(ctx, f, C.byref(bx), C.byref(by))
            tiles[name] = [bx.value, by.value]
        tuning["%dx%dx%d" % (n[i], n[i], nr[i])] = {
            "tiles": tiles, "tuned_ms": round(sum(best), 4),
            "default_ms": round(sum(dflt), 4)}
    stream = torch.cuda.ExternalStream(lib.gcs_ensemble_stream(ens), device=device)
    failed = C.c_int()
    ok = lib.gcs_ensemble_advance(ens, args.ens_warmup) == 0 and \
        lib.gcs_ensemble_sync(ens, C.byref(failed)) == 0
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize()
    start.record(stream)
    ok = ok and lib.gcs_ensemble_advance(ens, args.ens_steps) == 0
    stop.record(stream)
    stop.synchronize()
    ok = ok and lib.gcs_ensemble_sync(ens, C.byref(failed)) == 0
    torch.cuda.synchronize()
    barrier(dist, device)
    ms = max_over_ranks(start.elapsed_time(stop), dist, device)
    cells_local = sum(6 * nr[i] * n[i] * n[i] for i in range(k))
    cells = sum_over_ranks(float(cells_local), dist, device)
    nodes, grids = C.c_int(), C.c_int()
    lib.gcs_ensemble_graph_info(ens, C.byref(nodes), C.byref(grids))
    dts = []
    for i in range(k):
        dt, st = C.c_double(), C.c_int()
        lib.gcs_context_params(lib.gcs_ensemble_run_context(ens, i), C.byref(dt), None,
                               None, C.byref(st))
        dts.append(dt.value)
    out = {"value": cells * args.ens_steps / (ms * 1e-3), "unit": "cell-updates/s",
           "ms_per_ensemble_step": ms / args.ens_steps,
           "steps": args.ens_steps, "warmup": args.ens_warmup,
           "all_runs_ok": bool(ok), "failed_run": failed.value,
           "projected_500_steps_s": ms / args.ens_steps * 500 * 1e-3,
           "workload": "16 wind runs, seed %d: angular sizes %s, radial 2n, FP32-bulk, "
                       "drivers n [1,20] cm^-3, Vx [-800,-300] km/s, T [5e4,2e5] K, "
                       "Bz [-10,5] nT" % (ENS_SEED, sorted(list(n))),
           "cells_per_gpu": cells_local, "grids": grids.value,
           "graph": "one CUDA graph per ensemble step, %d kernel nodes; one branch per "
                    "grid size, runs of a size in sequence" % nodes.value,
           "gpu_launches": nodes.value * args.ens_steps,
           "device_bytes": lib.gcs_ensemble_device_bytes(ens),
           "setup_s": round(setup_s, 2),
           "dt_range": [min(dts), max(dts)],
           "autotune": tuning}
    lib.gcs_ensemble_destroy(ens)
    return out


MI_GRID = (361, 181)            # longitudes, colatitudes per hemisphere
MI_SEED = 2024
# Algorithmic bytes of one PCG iteration if its vectors streamed from memory:
# about 20 FP64 vector touches per unknown.
MI_BYTES_PER_UNKNOWN_ITER = 160


def mi_cases():
    from gamera_cube_b200 import cases
    npl, nt = MI_GRID
    return [cases.mi_case(npl, nt, seed=MI_SEED, hemisphere=h)
            for h in (cases.NORTH, cases.SOUTH)]


def run_mi(lib, torch, device, solves):
    """Constant-Pedersen ionosphere solves on the 181 x 361 polar cap
    (colatitude 0-45 deg), rel. residual 1e-8, zero initial guess: one
    hemisphere per call, and both hemispheres in one launch.  Device time
    with CUDA events around each solve; L2 flushed between solves."""
    import numpy as np
    from gamera_cube_b200 import abi
    cs = mi_cases()
    npl, nt = MI_GRID
    nodes = npl * nt
    unknowns = 1 + npl * (nt - 2)
    fac = torch.from_numpy(np.concatenate([c.fac.ravel() for c in cs])).to(device)
    pot = torch.zeros(2 * nodes, dtype=torch.float64, device=device)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    out = {}
    for label, count in (("one", 1), ("pair", 2)):
        cfgs = (abi.MiSolverConfig * count)(*[c.config for c in cs[:count]])
        plan = C.c_void_p()
        if lib.gcs_mi_plan_create(cfgs, count, C.byref(plan)) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        stats = (abi.MiSolverStats * count)()
        status = (C.c_int * count)()
        times = []
        stream = torch.cuda.current_stream(device)
        for q in range(3 + solves):
            pot.zero_()
            flush.fill_(float(q))
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            if lib.gcs_mi_solve_constant_pedersen_async(
                    plan, C.c_void_p(fac.data_ptr()), C.c_void_p(pot.data_ptr()),
                    C.c_void_p(stream.cuda_stream)) != 0:
                raise RuntimeError(lib.gcs_last_error().decode())
            ev1.record(stream)
            if lib.gcs_mi_plan_results(plan, stats, status) != 0:
                raise RuntimeError(lib.gcs_last_error().decode())
            if any(status[h] != 0 for h in range(count)):
                raise RuntimeError("MI solve did not converge")
            if q >= 3:
                times.append(ev0.elapsed_time(ev1))
        csize = C.c_int()
        lib.gcs_mi_plan_info(plan, C.byref(csize), None, None)
        lib.gcs_mi_plan_destroy(plan)
        out[label] = (sorted(times)[len(times) // 2], [stats[h].iterations
                                                       for h in range(count)],
                      csize.value)
    # end to end through the drop-in (host arrays, copies inside)
    c0 = cs[0]
    e2e = []
    for q in range(3 + solves):
        guess = np.zeros((nt, npl))
        st = abi.MiSolverStats()
        torch.cuda.synchronize(device)
        t = time.perf_counter()
        rc = lib.gamera_mi_solve_constant_pedersen(
            C.byref(c0.config), c0.fac.ctypes.data_as(C.POINTER(C.c_double)),
            guess.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st))
        e2e_ms = (time.perf_counter() - t) * 1e3
        if rc != 0:
            raise RuntimeError("drop-in MI solve failed")
        if q >= 3:
            e2e.append(e2e_ms)
    # conductance tensor (Hall = 1.5 Pedersen): SSOR-BiCGStab, one hemisphere
    tcfg = abi.MiSolverConfig.from_buffer_copy(cs[0].config)
    tcfg.maximum_iterations = 20000
    P = C.POINTER(C.c_double)
    zero_guess = np.zeros((nt, npl))

    def tensor_times(colored):
        tplan = C.c_void_p()
        if lib.gcs_mi_tensor_plan_create(C.byref(tcfg), C.byref(tplan)) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        ttimes, tst, tstatus = [], abi.MiSolverStats(), C.c_int()
        try:
            if lib.gcs_mi_tensor_plan_set_ordering(tplan, colored) != 0:
                raise RuntimeError("MI tensor ordering rejected")
            for q in range(3 + solves):
                if lib.gcs_mi_tensor_plan_upload(tplan, cs[0].fac.ctypes.data_as(P),
                                                 cs[0].pedersen.ctypes.data_as(P),
                                                 cs[0].hall.ctypes.data_as(P),
                                                 zero_guess.ctypes.data_as(P)) != 0:
                    raise RuntimeError(lib.gcs_last_error().decode())
                flush.fill_(float(q))
                stream = torch.cuda.current_stream(device)
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                if lib.gcs_mi_tensor_solve_async(tplan, C.c_void_p(stream.cuda_stream)) != 0:
                    raise RuntimeError(lib.gcs_last_error().decode())
                ev1.record(stream)
                if lib.gcs_mi_tensor_results(tplan, C.byref(tst), C.byref(tstatus)) != 0 or \
                        tstatus.value != 0:
                    raise RuntimeError("MI tensor solve did not converge")
                if q >= 3:
                    ttimes.append(ev0.elapsed_time(ev1))
        finally:
            lib.gcs_mi_tensor_plan_destroy(tplan)
        return sorted(ttimes)[len(ttimes) // 2], tst.iterations

    tensor_ms, tensor_its = tensor_times(0)
    colored_ms, colored_its = tensor_times(1)
    pcg = pedersen_pcg_times(lib, torch, device, solves, flush)
    two_level, learned = mi_flexible(lib, cs[0], solves, pcg)
    ms_one, it_one, csize = out["one"]
    ms_pair, it_pair, _ = out["pair"]
    us_iter = ms_one * 1e3 / it_one[0]
    eff = MI_BYTES_PER_UNKNOWN_ITER * unknowns / (us_iter * 1e-6) / 1e9
    return {
        "workload": "ionosphere potential, %d colat x %d lon polar cap (0-45 deg), "
                    "constant Pedersen 5 S, R1/R2 FAC +-1 uA/m^2 + noise, "
                    "rel. residual 1e-8, zero initial guess" % (nt, npl),
        "unknowns_per_hemisphere": unknowns,
        "ms_per_call": ms_one,
        "ms_per_call_both_hemispheres_one_launch": ms_pair,
        "iterations": it_pair,
        "us_per_iteration": us_iter,
        "cluster_ctas": csize,
        "e2e_ms_per_call": sorted(e2e)[len(e2e) // 2],
        "e2e_call": "gamera_mi_solve_constant_pedersen (drop-in, host arrays, "
                    "H2D/D2H of %d B each way)" % (2 * nodes * 8),
        "effective_gbs": eff,
        "bound": "latency (2 cluster barriers per iteration; vectors on chip)",
        "solves_timed": solves,
        "tensor": {"operator": "Pedersen + Hall (1.5x) tensor, SSOR-BiCGStab",
                   "ms_per_call": tensor_ms,
                   "iterations": tensor_its,
                   "launch": "one thread-block cluster (16 CTAs); SSOR sweeps by one warp along anti-diagonals, diagonals moved by bulk async copies",
                   "colored_ordering": {"ms_per_call": colored_ms, "iterations": colored_its,
                                        "sweep": "four-colour SSOR, each colour by the whole cluster"}},
        "tensor_two_level": two_level,
        "tensor_learned": learned,
        "pedersen_pcg": pcg,
    }


def pedersen_case(hemisphere):
    """The C5 conductances with Hall = 0 and one conductance at the pole
    point (the pole row's mean): the operator on which plain PCG is defined
    (symmetric positive definite)."""
    from gamera_cube_b200 import cases
    npl, nt = MI_GRID
    c = cases.mi_case(npl, nt, seed=MI_SEED, hemisphere=hemisphere)
    ped = c.pedersen.copy()
    ped[0, :] = ped[0, :].mean()
    import numpy as np
    return cases.MiCase(c.config, c.fac, np.ascontiguousarray(ped), np.zeros_like(ped),
                        c.potential)


def pedersen_pcg_times(lib, torch, device, solves, flush):
    """Plain PCG (Jacobi) on the variable-Pedersen, Hall-free operator,
    181 x 361, rel. residual 1e-8, zero guess: one hemisphere per launch and
    both in one launch; device time with CUDA events, L2 flushed between
    solves."""
    import numpy as np
    from gamera_cube_b200 import abi, cases
    hs = [pedersen_case(h) for h in (cases.NORTH, cases.SOUTH)]
    npl, nt = MI_GRID
    out = {"operator": "variable Pedersen (C5 field, pole row its mean), Hall = 0: "
                       "symmetric positive definite; Jacobi-preconditioned CG, "
                       "one thread-block cluster per hemisphere"}
    for label, count in (("one", 1), ("pair", 2)):
        cfgs = (abi.MiSolverConfig * count)(*[c.config for c in hs[:count]])
        ped = np.ascontiguousarray(np.concatenate([c.pedersen.ravel() for c in hs[:count]]))
        plan = C.c_void_p()
        if lib.gcs_mi_plan_create_pedersen(cfgs, ped.ctypes.data_as(C.POINTER(C.c_double)),
                                           count, C.byref(plan)) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        fac = torch.from_numpy(np.concatenate([c.fac.ravel() for c in hs[:count]])).to(device)
        pot = torch.zeros_like(fac)
        stats, status = (abi.MiSolverStats * count)(), (C.c_int * count)()
        times = []
        stream = torch.cuda.current_stream(device)
        for q in range(3 + solves):
            pot.zero_()
            flush.fill_(float(q))
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            if lib.gcs_mi_solve_constant_pedersen_async(
                    plan, C.c_void_p(fac.data_ptr()), C.c_void_p(pot.data_ptr()),
                    C.c_void_p(stream.cuda_stream)) != 0:
                raise RuntimeError(lib.gcs_last_error().decode())
            ev1.record(stream)
            if lib.gcs_mi_plan_results(plan, stats, status) != 0 or \
                    any(status[h] != 0 for h in range(count)):
                raise RuntimeError("Pedersen PCG did not converge")
            if q >= 3:
                times.append(ev0.elapsed_time(ev1))
        lib.gcs_mi_plan_destroy(plan)
        key = "ms_per_call" if count == 1 else "ms_per_call_both_hemispheres_one_launch"
        out[key] = sorted(times)[len(times) // 2]
        out["iterations" if count == 1 else "iterations_both"] = \
            [stats[h].iterations for h in range(count)]
    return out


def mi_flexible(lib, case, solves, pcg=None, train_steps=600):
    """The conductance-tensor case by flexible GMRES: left two-level
    preconditioner (ring-mean coarse correction + damped Jacobi) alone, and
    with the learned network as the right preconditioner after a short
    training on the GPU (random potentials and solved R1/R2 cases on the
    seeded production conductances).  Host arrays, synchronous calls, wall
    clock (the solve reads one Hessenberg column per iteration)."""
    import numpy as np
    from gamera_cube_b200 import cases, learn
    tcase = cases.mi_case(case.config.longitude_count, case.config.colatitude_count, seed=7,
                          max_iterations=3000)
    runs = []
    for q in range(2 + solves):
        rc, _, st, fb, sec = learn.solve(lib, None, tcase, method=2)
        if rc != 0 or fb:
            raise RuntimeError("two-level MI solve failed")
        if q >= 2:
            runs.append(sec * 1e3)
    two_level = {"operator": "Pedersen + Hall (1.5x) tensor, flexible GMRES(40), left "
                             "two-level preconditioner (ring-mean coarse correction, 2 damped "
                             "Jacobi steps)",
                 "ms_per_call": sorted(runs)[len(runs) // 2], "iterations": st.iterations}
    t0 = time.perf_counter()
    net = learn.create_net(lib, tcase.config, batch=8, seed=3)
    try:
        pool = learn.Pool(lib, npl=tcase.config.longitude_count,
                          nt=tcase.config.colatitude_count, random_fields=128, solved=4,
                          conductances=8)
        losses = learn.train(lib, net, pool, steps=train_steps, batch=8, lr=1e-3)
        train_s = time.perf_counter() - t0
        rc, _, st, fb, sec = learn.solve(lib, net, tcase, method=0)
        rc, _, st, fb, sec = learn.solve(lib, net, tcase, method=0)
    finally:
        lib.gcs_mi_net_destroy(net)
    learned = {"operator": "as tensor_two_level with the BF16 conv net (194,769 parameters) as "
                           "the flexible right preconditioner",
               "training": {"steps": train_steps, "batch": 8, "triples": pool.triples,
                            "seconds": train_s, "loss_first": float(losses[0]),
                            "loss_last": float(np.mean(losses[-20:]))},
               "ms_per_call": sec * 1e3, "iterations": st.iterations,
               "fell_back_to_reference_algorithm": bool(fb), "converged": rc == 0}
    if pcg is not None:
        # the same learned method and the two-level method on the operator
        # where plain PCG is defined (Hall = 0), against plain PCG
        from gamera_cube_b200 import cases as _cases
        hcase = pedersen_case(_cases.NORTH)
        hcase.config.maximum_iterations = 3000
        net = learn.create_net(lib, hcase.config, batch=8, seed=3)
        try:
            pool = learn.Pool(lib, npl=hcase.config.longitude_count,
                              nt=hcase.config.colatitude_count, random_fields=128, solved=4,
                              conductances=8, hall_ratio=0.0)
            learn.train(lib, net, pool, steps=train_steps, batch=8, lr=1e-3)
            learn.solve(lib, net, hcase, method=0)
            rc0, _, st0, fb0, sec0 = learn.solve(lib, net, hcase, method=0)
        finally:
            lib.gcs_mi_net_destroy(net)
        rc2, _, st2, fb2, sec2 = learn.solve(lib, None, hcase, method=2)
        learned["on_pcg_operator"] = {
            "operator": pcg["operator"],
            "learned_ms_per_call": sec0 * 1e3, "learned_iterations": st0.iterations,
            "learned_fell_back": bool(fb0),
            "two_level_ms_per_call": sec2 * 1e3, "two_level_iterations": st2.iterations,
            "plain_pcg_ms_per_call": pcg["ms_per_call"],
            "plain_pcg_iterations": pcg["iterations"][0],
            "speedup_learned_over_plain_pcg": pcg["ms_per_call"] / (sec0 * 1e3)}
    return two_level, learned


def mi_cpu_baseline():
    """The reference's constant-Pedersen and tensor solves (oracle/_ref, one
    thread: the reference MI solver is serial) on the north hemisphere."""
    from oracle import refbind
    from gamera_cube_b200 import abi, cases
    if not refbind.ref_available():
        return None
    lib = refbind.ref()
    c = mi_cases()[0]
    P = C.POINTER(C.c_double)
    pot = c.potential.copy()
    st = abi.MiSolverStats()
    t = time.perf_counter()
    rc = lib.gamera_mi_solve_constant_pedersen(C.byref(c.config), c.fac.ctypes.data_as(P),
                                               pot.ctypes.data_as(P), C.byref(st))
    const_ms = (time.perf_counter() - t) * 1e3
    npl, nt = MI_GRID
    tcfg = cases.mi_config(npl, nt, max_iterations=20000)
    pot = c.potential.copy()
    st2 = abi.MiSolverStats()
    t = time.perf_counter()
    rc2 = lib.gamera_mi_solve_conductance_tensor(
        C.byref(tcfg), c.fac.ctypes.data_as(P), c.pedersen.ctypes.data_as(P),
        c.hall.ctypes.data_as(P), pot.ctypes.data_as(P), C.byref(st2))
    tensor_ms = (time.perf_counter() - t) * 1e3
    return {"ms_per_call": const_ms, "iterations": st.iterations, "converged": rc == 0,
            "tensor_ms_per_call": tensor_ms, "tensor_iterations": st2.iterations,
            "tensor_converged": rc2 == 0, "cores": 1, "kind": "reference",
            "sample": "one north-hemisphere call of each solver"}


def _ref_bench_path():
    return os.path.join(REPO, "oracle", "_ref", "ref_bench")


def ref_bench(nr, n, warmup, steps, seed=1000):
    """The unmodified reference step (oracle/_ref/ref_bench: the case built by
    the reference's set-up API, then the Earth driver's dt rule and one
    planned six-face step per iteration, only the step loop timed), OpenMP
    on every physical core.  Returns its JSON record."""
    cores = physical_cores()
    env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="close",
               OMP_PLACES="cores")
    out = subprocess.run([_ref_bench_path(), "2", str(nr), str(n), str(warmup),
                          str(steps), str(seed)],
                         capture_output=True, text=True, env=env, timeout=3000)
    if out.returncode != 0:
        raise RuntimeError("reference CPU run failed: " + out.stderr[-500:])
    rec = json.loads(out.stdout.strip().splitlines()[-1])
    rec["cores"] = cores
    return rec


def cpu_baseline(args):
    """The reference's own CPU step on a bounded sample of the workload (the
    same case at 48 radial x 32 x 32 angular cells per face: set-up about
    10 s and 3 timed steps), all physical cores; falls back to the CPU
    restatement (one thread) if the reference library was not built."""
    nr, n, steps = args.cpu_nr, args.cpu_n, args.cpu_steps
    if os.path.exists(_ref_bench_path()):
        rec = ref_bench(nr, n, 1, steps)
        return {"value": rec["cell_updates_per_s"], "unit": "cell-updates/s",
                "cores": rec["cores"], "threads": rec["threads"],
                "kind": "reference",
                "sample": "reference CPU step (OpenMP), 6 x %dx%dx%d wind+dipole "
                          "case, %d timed steps after 1 warm-up" % (n, n, nr, steps)}
    from oracle import oracle_cases
    case = oracle_cases.Case("wind", nr, n, 1000)
    dt = 0.5 * case.local_timestep()
    case.step(0.0, dt)
    t = time.perf_counter()
    for _ in range(steps):
        case.step(0.5, dt)
    sec = time.perf_counter() - t
    return {"value": 6 * nr * n * n * steps / sec, "unit": "cell-updates/s",
            "cores": 1, "threads": 1, "kind": "port",
            "sample": "CPU restatement, 6 x %dx%dx%d wind+dipole case, %d steps"
                      % (n, n, nr, steps)}


def workload_name(nr, n):
    return ("cubed-sphere 6 x %dx%dx%d FP64 MHD step, solar wind + aligned dipole"
            % (n, n, nr))


def run_reference(args):
    """The reference arm: rank 0 times the reference's own CPU step on this
    bench's workload (same sizes and case), the other ranks exit."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(_ref_bench_path()):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference library not built (make -C oracle ref)"}))
        return
    steps = max(1, min(args.steps, args.ref_steps))
    rec = ref_bench(args.nr, args.n, 1, steps)
    value = rec["cell_updates_per_s"]
    base = {"value": value, "unit": "cell-updates/s", "cores": rec["cores"],
            "threads": rec["threads"], "kind": "reference",
            "sample": "reference CPU step (OpenMP, %d threads on %d physical cores, "
                      "1 process), the full 6 x %dx%dx%d case, %d timed steps after "
                      "1 warm-up (set-up %.0f s not timed)"
                      % (rec["threads"], rec["cores"], args.n, args.n, args.nr, steps,
                         rec["setup_seconds"])}
    line = {"impl": "reference", "metric": METRIC, "value": value,
            "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": 1, "ms_per_step": rec["seconds"] / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded solar wind + dipole, built by "
                                    "the reference's set-up API)",
            "config": {"workload": workload_name(args.nr, args.n), "faces": 6,
                       "angular": args.n, "radial": args.nr,
                       "cells_per_gpu": 6 * args.nr * args.n * args.n, "ghost": 4,
                       "same_config": True},
            "cpu_baseline": base,
            "e2e": {"value": value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.mi_solves > 0:
        line["mi"] = mi_cpu_baseline()
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nr", type=int, default=NR)
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--cpu-nr", type=int, default=48)
    ap.add_argument("--cpu-n", type=int, default=32)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--ref-steps", type=int, default=2,
                    help="timed reference CPU steps of the full workload "
                         "(--impl reference)")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--mi-every", type=int, default=10,
                    help="steps between ionosphere coupling updates in the "
                         "timed MHD run (0: no coupling)")
    ap.add_argument("--mi-solves", type=int, default=10,
                    help="timed ionosphere solves (0 skips the MI measurement)")
    ap.add_argument("--no-bulk", dest="bulk", action="store_false",
                    help="skip the FP32-bulk variant measurement")
    ap.add_argument("--earth-steps", type=int, default=20,
                    help="timed steps with the device Earth boundary (0 skips them)")
    ap.add_argument("--ens-steps", type=int, default=20,
                    help="timed steps of the 16-run ensemble (0 skips it)")
    ap.add_argument("--ens-warmup", type=int, default=3)
    ap.add_argument("--flux-staging", action="store_true",
                    help="use the TMA-staged flux sweep (gcs_context_set_flux_staging) "
                         "instead of the default per-face sweep")
    ap.add_argument("--c3-steps", type=int, default=0,
                    help="steps of the 6 x 192x192x384 density-pulse precision run "
                         "(FP32-bulk against FP64 on the same time levels; about "
                         "5 minutes for 1000 steps, so off by default)")
    ap.add_argument("--only-mi", action="store_true",
                    help="run only the standalone ionosphere solve measurement "
                         "(prints its JSON object; for profiling)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.gpus > 1 and "RANK" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.impl == "reference":
        run_reference(args)
    elif args.only_mi:
        import torch
        import gamera_cube_b200
        torch.cuda.set_device(0)
        print(json.dumps(run_mi(gamera_cube_b200.lib, torch, torch.device("cuda", 0),
                                max(1, args.mi_solves))))
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
