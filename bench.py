"""Benchmark of the hydro advance on B200: zone-updates/s at FP64.

Workload (the headline single-GPU configuration): a 256^3 periodic cube,
rho = 1 + 0.1 sin(2 pi x) sin(2 pi y) sin(2 pi z), p = 1, zero velocity, with
16 seeded spherical overpressure blobs (p = 10, radius 0.03-0.08); unsplit
CTU Godunov with PPM characteristic tracing and the reference's two-shock
Riemann solver, CFL 0.7, gamma = 1.4.  A "step" is one coarse time step of
the whole domain (clean, ghost fill, hydro, update, next dt).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl camr|reference]

N > 1 (torchrun, one rank per GPU): every rank advances its own replica of
the domain (weak scaling, no data-path collective: the single-GPU path has no
exchange step); time is the max over ranks.

--impl reference times the reference's own CPU implementation (its hydro
sources compiled against the AMReX stand-in, oracle/_ref, with the restated
level driver) on the host cores, on a bounded 128^3 sample of the workload
per step.
"""
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

METRIC = "zone-updates/s (FP64, 1xB200)"
UNIT = "zone-updates/s"
N_DEFAULT = 256
CFL = 0.7

# Algorithmic bytes per cell of each stage: every array the stage must read
# or write, once (FP64).  Stage -> (bytes/cell, what).
STAGE_BYTES = {
    "clean_copy": (160, "read U, write U_old (10 comps)"),
    "expand": (160, "read U_old, write Sborder (10 comps)"),
    "ctoprim": (168, "read Sborder (10), write q (11)"),
    "flatten_divu": (48, "read q p,u,v,w; write flat, divu"),
    "trace": (528, "read q (11) + flat, write 6 edge states x 9"),
    "flux1": (688, "read 6 edge states x 9 + c,csml, write 3 flux records x 10"),
    "flux2": (1168, "read 6 x 9 states + 3 x 10 records, write 6 x 10 records"),
    "flux3": (1288, "read states, 6 x 10 records, divu, U; write 3 x 10 fluxes + 3 x 2"),
    # the second and final passes fused (k_flux23): the 6 x 10 second-pass
    # records stay in shared memory
    "flux23": (1496, "read 6 x 9 edge states, 3 x 10 first-pass records, divu, U; "
                     "write 3 x 10 fluxes + 3 x 2"),
    "update": (528, "read Sborder, U_old, 3 x 10 fluxes, 3 x 2; write U"),
}
# Whole-step algorithmic bytes per zone-update: CTU reads U^n and writes
# U^n+1 (160 B); SSP-RK2 reads U^n, writes U*, reads U* and U^n, writes
# U^n+1 (400 B).  FP64, NVAR = 10; ghosts and temporaries excluded.
STEP_BYTES_PER_ZONE = 160
MOL_BYTES_PER_ZONE = 400
# Algorithmic flops per zone-update (+, -, *, / and sqrt, one each), counted
# on the reference's own per-box hydro with a counting amrex::Real on one
# 64^3 box of the configuration's data (oracle/count_flops.py; recounted by
# tests/test_flops.py).  CTU-PPM: 3239 adds, 3362 muls, 345 divisions, 65
# square roots; SSP-RK2 MOL-PLM: two hydro evaluations per step.
FLOPS_PER_ZONE_UPDATE = {"ctu_ppm": 7011.0, "mol_plm": 2770.3}
# Divisions and square roots per zone-update among those flops: on the GPU
# each expands into a reciprocal or root estimate and Newton steps, and with
# -fmad=false (bit-exact parity with the reference's unfused CPU arithmetic)
# no add or multiply fuses into an FMA, so the FP64 pipe's ceiling for this
# code is half the DFMA peak in flop/s.
DIVSQRT_PER_ZONE_UPDATE = {"ctu_ppm": 410.3, "mol_plm": 296.8}
# DRAM bytes (read + write) per valid cell of one launch, from an ncu
# capture of the same kernel on the 128^3 case of this workload (inputs
# larger than L2; traffic grows with the cell count, so the per-cell figure
# scales to 256^3): k_flux2 3.344 GB read + 1.037 GB written per launch
# over 128^3 cells (profiles/ncu_k_flux2_128cube_ctu_ppm.txt).
STAGE_TRAFFIC_PER_CELL = {"flux2": (3.344e9 + 1.037e9) / 128 ** 3}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


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
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
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
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def profile_range(args, on):
    """With --profile-range, bracket a timed region with cudaProfilerStart /
    cudaProfilerStop so that `ncu --profile-from-start off` lists exactly the
    launches of that region."""
    if not getattr(args, "profile_range", False):
        return
    import torch
    torch.cuda.synchronize()
    if on:
        torch.cuda.profiler.start()
    else:
        torch.cuda.profiler.stop()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x, pg, device="cuda"):
    """The largest of every rank's x (every rank gets it); x itself on one
    process.  The timing of a multi-GPU run is the slowest rank's."""
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, zones_per_rank, steps, ms):
    """Zone-updates/s of the whole job: every rank advances its own replica
    of zones_per_rank cells `steps` times in `ms` (the slowest rank's)."""
    return world * zones_per_rank * steps / (ms * 1e-3)


def c1_config(n, world):
    """The `config` of the C1 line (both arms report the same one)."""
    state_gb = 10 * n[0] * n[1] * n[2] * 8 / 1e9
    return {"workload": f"c1: {n[0]}^3 periodic CTU-PPM, CFL 0.7, 16 blobs",
            "domain": list(n), "method": "CTU Godunov, PPM, two-shock Riemann",
            "cfl": CFL,
            "boxes": f"{(n[0] // 64) * (n[1] // 64) * (n[2] // 64)} x 64^3 "
                     "(advanced as one padded domain)",
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 (state {state_gb:.2g} GB, intermediates "
                  f"~{state_gb * 18.7:.2g} GB)"}


def c1_rooflines(zones, acc, dom, ms_step, hbm_peak, peak_kind, fp64_peak):
    """The roofline objects of the C1 line.  `roofline` is the dominant
    kernel against HBM on the workload's algorithmic bytes (160 B per
    zone-update: read U^n, write U^n+1) with the FP64 side beside it (the
    reference's counted flops per zone-update); the kernel's own
    intermediate-array bytes are kept apart under `kernel_intermediates`.
    `step_roofline` is the same for the whole step."""
    t_dom = acc[dom] * 1e-3
    achieved = STEP_BYTES_PER_ZONE * zones / t_dom / 1e9
    flops = FLOPS_PER_ZONE_UPDATE["ctu_ppm"]
    inter = STAGE_BYTES[dom][0] * zones / t_dom / 1e9
    roofline = {
        "kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
        "frac": achieved / hbm_peak, "peak_source": f"{peak_kind} hbm_gbs",
        "algorithmic_bytes_per_zone_update": STEP_BYTES_PER_ZONE,
        "units_per_launch": zones,
        "avg_launch_ms": acc[dom],
        "traffic": (STAGE_TRAFFIC_PER_CELL[dom] * zones if dom in STAGE_TRAFFIC_PER_CELL
                    else None),
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per cell of a "
                          "128^3 capture, times the cells of one launch",
        "kernel_intermediates": {
            "bytes_per_cell": STAGE_BYTES[dom][0], "what": STAGE_BYTES[dom][1],
            "achieved_gbs": inter, "frac": inter / hbm_peak},
        "fp64_whole_step": fp64_roofline("ctu_ppm", zones / (ms_step * 1e-3), fp64_peak),
    }
    step_achieved = STEP_BYTES_PER_ZONE * zones / (ms_step * 1e-3) / 1e9
    step_roofline = {"bytes_per_zone_update": STEP_BYTES_PER_ZONE, "achieved": step_achieved,
                     "peak": hbm_peak, "unit": "GB/s", "frac": step_achieved / hbm_peak,
                     "fp64": fp64_roofline("ctu_ppm", zones / (ms_step * 1e-3), fp64_peak)}
    return roofline, step_roofline


def level_hbm(method, zone_rate):
    """Achieved algorithmic HBM bandwidth of a level step: 400 B per
    zone-update for SSP-RK2 (MOL), 160 B for CTU."""
    peak, kind = measured_peaks()
    b = MOL_BYTES_PER_ZONE if method.startswith("mol") else STEP_BYTES_PER_ZONE
    gbs = b * zone_rate / 1e9
    return {"bytes_per_zone_update": b, "achieved_gbs": gbs, "peak_gbs": peak,
            "frac": gbs / peak, "peak_source": f"{kind} hbm_gbs"}


def fp64_roofline(method, zone_rate, fp64_peak):
    """Counted flops per zone-update x zone-updates/s against the measured
    DFMA peak (an FMA counts 2 flops there; this code issues no FMAs, so
    frac_of_unfused_peak, against half that peak, is its pipe's ceiling)."""
    f = FLOPS_PER_ZONE_UPDATE[method]
    tf = f * zone_rate / 1e12
    return {"flops_per_zone_update": f, "divisions_and_sqrts_per_zone_update":
            DIVSQRT_PER_ZONE_UPDATE[method], "achieved_tflops": tf,
            "peak_tflops": fp64_peak, "peak_source": "measured DFMA (camr_measure_fp64_peak)",
            "frac": tf / fp64_peak if fp64_peak else None,
            "frac_of_unfused_peak": 2 * tf / fp64_peak if fp64_peak else None,
            "flop_source": "reference hydro with a counting amrex::Real, one 64^3 box "
                           "(oracle/count_flops.py)"}


def c1_state(n):
    from camr_b200 import problems as P
    dx = tuple(1.0 / v for v in n)
    return P.blobs(n, dx, nblobs=16, seed=1)


def cpu_reference_rate(n, nsteps, warmup=0):
    """Zone-updates/s of the reference's CPU hydro (oracle/_ref) on the host cores."""
    import oracle
    kind = "ref" if os.path.exists(oracle.lib_path("ref")) else "restate"
    nth = os.cpu_count() or 1
    p = oracle.default_params(do_mol=0, ppm_type=1, cfl=CFL)
    # the reference's OpenMP hydro tile (Source/CAMR.cpp:29-30), 64^3 boxes
    lev = oracle.make_level(n, tile_size=(1024, 16, 16), max_grid_size=(64, 64, 64),
                            nthreads=nth)
    s = c1_state(n)
    oracle.init_finalize(kind, p, lev, s)
    dtp, _, _ = oracle.advance(kind, p, lev, s, 1 + warmup)
    t0 = time.perf_counter()
    oracle.advance(kind, p, lev, s, nsteps, first_step=False, dt_prev=dtp)
    dt = time.perf_counter() - t0
    return n[0] * n[1] * n[2] * nsteps / dt, dt, kind, nth


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle
    if not os.path.exists(oracle.lib_path("ref")) and not os.path.exists(oracle.lib_path("restate")):
        print(json.dumps({"impl": "reference", "unavailable": "oracle libraries not built"}))
        return
    n = (128, 128, 128)
    rate, secs, kind, nth = cpu_reference_rate(n, args.steps, warmup=args.warmup)
    sample = (f"{n[0]}^3 sample of the workload (the same blob field at half the "
              f"resolution), {args.steps} steps, tiles 1024x16x16, {nth} threads")
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic (seeded overpressure blobs, numpy PCG64 seed 1)",
        "config": dict(c1_config(n, world),
                       workload=f"c1 sample: {n[0]}^3 periodic CTU-PPM, CFL 0.7, 16 blobs "
                                f"(the {args.n}^3 workload's blob field at {n[0]}^3; "
                                "zone-updates/s does not depend on the domain size)"),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": nth,
                         "kind": "reference" if kind == "ref" else "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_camr(args, world, rank, local, pg):
    import ctypes as C

    import torch

    from camr_b200 import build, hydro, native

    if not os.path.exists(native.LIB_PATH):
        build.build()
    lib = native.lib()
    torch.cuda.set_device(local)
    n = (args.n, args.n, args.n)
    zones = n[0] * n[1] * n[2]
    s0 = c1_state(n)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=0, ppm_type=1, cfl=CFL)
    L = hydro.Level(geom, prm, max_grid_size=(64, 64, 64), use_graph=True)
    st = L.torch_stream()
    L.set_state(s0)
    L.init_finalize()
    L.advance(max(args.warmup, 3))
    torch.cuda.synchronize()
    # the state the timed steps start from: also the input of every
    # end-to-end step below
    s_start = L.get_state()

    def barrier():
        if pg is not None:
            pg.barrier()

    fp64_peak = C.c_double()
    lib.camr_measure_fp64_peak(C.byref(fp64_peak), C.c_void_p(L.stream_ptr))
    args.fp64_peak = fp64_peak.value

    sampler = ClockSampler(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = lib.camr_launch_count()
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    profile_range(args, True)
    e0.record(st)
    L.advance(args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    profile_range(args, False)
    clocks = sampler.stop()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = lib.camr_launch_count() - launches0
    err = L.error()
    # conservation over the timed steps, outside the timed region: the
    # integrated quantities of the state they started from and of the one
    # they left (a periodic domain: mass and total energy to round-off)
    try:
        from camr_b200 import metrics
        dxs = tuple(geom.dx[d] for d in range(3))
        conservation = dict(metrics.drift(metrics.integrated_quantities(s_start, dxs),
                                          metrics.integrated_quantities(L.get_state(), dxs)),
                            steps=args.steps)
    except Exception as exc:  # a diagnostic: it never costs the benchmark line
        conservation = {"error": f"{type(exc).__name__}: {exc}"}
    ms = max_over_ranks(ms, pg)
    ms_step = ms / args.steps
    value = whole_job_rate(world, zones, args.steps, ms)

    # Per-stage device times, live (uncaptured profiled steps).
    names = (C.c_char_p * 40)()
    times = (C.c_float * 40)()
    cnt = C.c_int()
    acc = {}
    nprof = 3
    for _ in range(nprof):
        native.check(lib.camr_level_profile_step(L._h, times, names, 40, C.byref(cnt)),
                     "profile_step")
        for i in range(cnt.value):
            k = names[i].decode()
            acc[k] = acc.get(k, 0.0) + times[i] / nprof
    hbm_peak, peak_kind = measured_peaks()
    dom = max((k for k in acc if k in STAGE_BYTES), key=lambda k: acc[k])
    roofline, step_roofline = c1_rooflines(zones, acc, dom, ms_step, hbm_peak, peak_kind,
                                           fp64_peak.value)

    # End to end through the C ABI with host buffers: every step uploads a
    # state from pinned host memory, advances it one step (a step after a
    # new state computes its dt afresh, as a first step does), and reads the
    # state back.  The uploads and downloads run on the level's copy
    # streams, so the upload of step k+1 and the download of step k overlap
    # the kernels of step k (and k+1); the region ends when the last
    # download has landed.  The uploaded state is the one the device-timed
    # steps start from (the blobs after the warm-up steps); the first steps
    # from the initial blobs, whose fronts are still sharp, cost ~10% more
    # in the kernels and are timed as well.
    host = torch.from_numpy(s_start).pin_memory()
    host0 = torch.from_numpy(s0).pin_memory()
    out = torch.empty_like(host).pin_memory()
    # as many steps as the device-timed loop, so that the pipeline's fill
    # (the first upload) and drain (the last download) weigh as they would
    # in a run of that length
    e2e_steps = max(2, args.steps)

    def e2e_run(overlap, src, up=True, step=True, down=True):
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(e2e_steps):
            if up:
                native.check(lib.camr_level_set_state(L._h, C.c_void_p(src.data_ptr()), 1),
                             "set")
            if step:
                L.advance(1)
            if down:
                get = lib.camr_level_get_state_async if overlap else lib.camr_level_get_state
                native.check(get(L._h, C.c_void_p(out.data_ptr()), 1), "get")
        native.check(lib.camr_level_sync(L._h), "sync")
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / e2e_steps

    e2e_serial_ms = e2e_run(False, host)
    e2e_initial_ms = e2e_run(True, host0)
    # the copy pipeline without the step (upload + unpack, pack + download,
    # both directions at once), and each direction alone: the PCIe floor the
    # end-to-end step sits on
    copies_ms = e2e_run(True, host, step=False)
    up_ms = e2e_run(True, host, step=False, down=False)
    down_ms = e2e_run(True, host, up=False, step=False)
    e2e_ms = e2e_run(True, host)
    e2e_ms = max_over_ranks(e2e_ms, pg)
    state_bytes = host.numel() * 8
    e2e = {"value": whole_job_rate(world, zones, 1, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
           "ms_per_step": e2e_ms, "steps": e2e_steps,
           "ms_per_step_without_overlap": e2e_serial_ms,
           "ms_per_step_from_initial_state": e2e_initial_ms,
           "ms_per_step_copies_only": copies_ms,
           "ms_per_step_upload_only": up_ms, "ms_per_step_download_only": down_ms,
           "pcie_gbs_upload_only": state_bytes / up_ms / 1e6,
           "pcie_gbs_download_only": state_bytes / down_ms / 1e6,
           "input": "the state after the warm-up steps, uploaded every step",
           "timing": "CUDA events on the level's stream around the loop; the level's copy "
                     "streams are synchronised before the closing event"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, secs, kind, nth = cpu_reference_rate(n, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": nth,
               "kind": "reference" if kind == "ref" else "port",
               "sample": f"one full {n[0]}^3 step of the workload ({secs:.1f} s), "
                         "reference hydro kernels, tiles 1024x16x16, all host threads"}

    batched = None
    amr = None
    adj = None
    ebc = None
    if rank == 0 and world == 1 and not args.no_batched:
        L.close()
        batched = batched_comparison(args)
        amr = amr_comparison(args)
        adj = adjoint_comparison(args, fd_cells=args.fd_cells)
        ebc = eb_comparison(args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded overpressure blobs, numpy PCG64 seed 1)",
            "config": c1_config(n, world),
            "roofline": roofline, "step_roofline": step_roofline, "cpu_baseline": cpu,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "conservation": conservation,
            "stages_ms": acc, "device_error": list(err),
            "batched_amr_patches": batched,
            "amr_two_level": amr,
            "adjoint_c3": adj,
            "eb_c4": ebc,
        }
        print(json.dumps(line))
    L.close()


def amr_box_inputs(boxes, fine_n, dev):
    """Per-box Sborder fabs (box grown by 4) of a smooth flow with overpressure
    blobs, evaluated at the fine cells' centres on the device (test data)."""
    import torch
    gamma = 1.4
    brng = np.random.default_rng(1)
    blobs = []
    for _ in range(16):
        c = brng.uniform(0.0, 1.0, size=3)
        r = brng.uniform(0.03, 0.08)
        blobs.append((c, r))
    out = []
    two_pi = 2 * np.pi
    for lo, hi in boxes:
        ax = [torch.arange(lo[d] - 4, hi[d] + 5, device=dev, dtype=torch.float64) for d in range(3)]
        x = ((ax[0] + 0.5) / fine_n)[None, None, :]
        y = ((ax[1] + 0.5) / fine_n)[None, :, None]
        z = ((ax[2] + 0.5) / fine_n)[:, None, None]
        rho = 1.0 + 0.1 * torch.sin(two_pi * x) * torch.sin(two_pi * y) * torch.sin(two_pi * z)
        p = torch.ones_like(rho)
        for c, r in blobs:
            d2 = 0.0
            for arr, cc in zip((x, y, z), c):
                dd = torch.abs(arr - cc)
                dd = torch.minimum(dd, 1.0 - dd)
                d2 = d2 + dd * dd
            p = torch.where(d2 < r * r, torch.full_like(p, 10.0), p)
        u = 0.2 * torch.sin(two_pi * y) * torch.ones_like(rho)
        v = 0.2 * torch.sin(two_pi * z) * torch.ones_like(rho)
        w = 0.2 * torch.sin(two_pi * x) * torch.ones_like(rho)
        U = torch.empty((10,) + rho.shape, dtype=torch.float64, device=dev)
        U[0] = rho
        U[1], U[2], U[3] = rho * u, rho * v, rho * w
        U[5] = p / (gamma - 1.0)
        U[4] = U[5] + 0.5 * rho * (u * u + v * v + w * w)
        U[6] = (gamma - 1.0) * (U[5] / rho) * 26.93 / 8.31446261815324e7
        U[7], U[8], U[9] = rho, 0.0 * rho, 0.0 * rho
        nb = [hi[d] - lo[d] + 1 for d in range(3)]
        dsdt = torch.zeros((10, nb[2], nb[1], nb[0]), dtype=torch.float64, device=dev)
        flx = []
        for d in range(3):
            sh = list(nb)
            sh[d] += 1
            flx.append(torch.zeros((10, sh[2], sh[1], sh[0]), dtype=torch.float64, device=dev))
        out.append((list(lo), list(hi), U.contiguous(), [lo[d] - 4 for d in range(3)], dsdt, flx))
    return out


def batched_comparison(args, steps=5, warmup=2):
    """Hydro of one level step over the uneven fine-level boxes: batched
    work-list launches vs per-box launches (same plan, same boxes)."""
    import torch

    from camr_b200 import hydro, native, problems
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    fine_n = 512
    boxes = problems.amr_box_list(nbox=args.nbox, fine_n=fine_n)
    cells = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in boxes)
    items = amr_box_inputs(boxes, fine_n, dev)
    geom = hydro.make_geom((fine_n,) * 3)
    prm = native.default_params(do_mol=0, ppm_type=1, cfl=CFL)
    dt = 0.25 / fine_n / 4.0
    b = hydro.Batch(items, geom, prm)
    torch.cuda.synchronize()
    b.autotune(dt)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    res = {}
    for name, mode in (("per_box", hydro.Batch.PER_BOX), ("batched", hydro.Batch.PERSISTENT)):
        for _ in range(warmup):
            b.run(dt, mode)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            b.run(dt, mode)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        res[name] = {"ms": ms, "zone_updates_per_s": cells / (ms * 1e-3)}
    out = {"boxes": len(boxes), "cells": cells, "per_box": res["per_box"],
           "batched": res["batched"],
           "speedup_batched_vs_per_box": res["per_box"]["ms"] / res["batched"]["ms"],
           "tuning_cells_per_block_and_grid": b.tuning()}
    b.close()
    del items
    torch.cuda.empty_cache()
    return out


def amr_comparison(args, steps=None, per_box_steps=2, warmup=3):
    """The two-level configuration end to end on the device: base 256^3 +
    the uneven fine boxes (ratio 2, two subcycled fine steps per coarse
    step, flux-register reflux, average down).  Zone-updates per coarse
    step = base cells + 2 x fine cells.  The fine hydro runs as the batched
    work-list launches inside one graph-captured step, and, for comparison,
    as plain per-box launch sequences (no graph)."""
    import torch

    from camr_b200 import hydro, native, problems
    if steps is None:
        steps = args.amr_steps
    n0 = (args.amr_n0,) * 3
    fine_n = 2 * args.amr_n0
    boxes = problems.amr_box_list(nbox=args.nbox, fine_n=fine_n)
    S0, S1 = problems.amr_initial(n0, boxes, vel=None)
    geom = hydro.make_geom(n0)
    out = {"base": list(n0), "boxes": len(boxes),
           "parity": "hydro: the reference's kernels bit for bit; the coarse-fine coupling "
                     "(FillPatch interpolation, flux register, average down) equals the "
                     "restated AMReX algorithms of the oracle bit for bit; AMReX itself is "
                     "absent, so that coupling is unpinned against AMReX"}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    methods = (("mol_plm", dict(do_mol=1, ppm_type=0, cfl=0.3), True),
               ("ctu_ppm", dict(do_mol=0, ppm_type=1, cfl=CFL), False))
    for name, kw, compare in methods:
        h = hydro.AmrHierarchy(geom, native.default_params(**kw), boxes,
                               max_grid_size=(64, 64, 64))
        st = h.torch_stream()
        zones = n0[0] * n0[1] * n0[2] + 2 * h.fine_cells
        h.set_state(S0, S1)
        h.init_finalize()
        h.advance(1)
        h.autotune()
        h.advance(warmup)
        torch.cuda.synchronize()
        res = {"fine_cells": h.fine_cells, "zone_updates_per_step": zones}
        modes = [("batched_graph", h.PERSISTENT, steps)]
        if compare:
            modes.append(("per_box", h.PER_BOX, per_box_steps))
        for mname, mode, k in modes:
            h.set_fine_mode(mode)
            h.advance(1)
            torch.cuda.synchronize()
            prof = name == "mol_plm" and mname == "batched_graph"
            if prof:
                profile_range(args, True)
            e0.record(st)
            h.advance(k)
            e1.record(st)
            torch.cuda.synchronize()
            if prof:
                profile_range(args, False)
            ms = e0.elapsed_time(e1) / k
            rate = zones / (ms * 1e-3)
            res[mname] = {"ms_per_step": ms, "zone_updates_per_s": rate,
                          "hbm": level_hbm(name, rate), "fp64": fp64_roofline(
                              "mol_plm" if name == "mol_plm" else "ctu_ppm", rate,
                              args.fp64_peak)}
        res["kernels_per_step_graph"] = h.kernels_per_step()
        res["device_error"] = list(h.error())
        if compare:
            res["speedup_batched_graph_vs_per_box"] = (res["per_box"]["ms_per_step"] /
                                                       res["batched_graph"]["ms_per_step"])
        out[name] = res
        h.close()
        torch.cuda.empty_cache()
    return out


def eb_comparison(args, n=(256, 128, 128), nsteps=None, warmup=3, cpu_n=(64, 32, 32)):
    """The embedded-boundary configuration: Sod (x < 0.5 left) with a rigid
    sphere r = 0.15 at (1, 0.5, 0.5) on [0,2]x[0,1]^2 (256x128x128), x
    outflow, y/z slip walls, MOL-PLM RK2 at CFL 0.3 with flux
    redistribution, 150 steps (dt on the device, graph-captured); also the
    Godunov-PLM (CTU) EB level on the same problem.  The
    domain is one EB box: regular, cut and covered cells share every launch.
    Also the same level without the sphere (the regular MOL level driver)
    for the EB overhead, and the reference's EB kernels on the host on a
    small sample of the same problem."""
    import torch

    from camr_b200 import eb_geometry, hydro, native, problems
    if nsteps is None:
        nsteps = args.eb_steps
    dx = 2.0 / n[0]
    t0 = time.time()
    geo = eb_geometry.sphere_geometry((-5, -5, -5), (n[0] + 4, n[1] + 4, n[2] + 4), dx,
                                      center=(1.0, 0.5, 0.5), radius=0.15)
    geo_s = time.time() - t0
    s0 = problems.sod_sphere(n, (dx,) * 3, geo)
    geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                           dx=(dx,) * 3)
    prm = native.default_params(do_mol=1, ppm_type=0, cfl=0.3)
    typ = geo["flag"][5:-5, 5:-5, 5:-5] & 3
    gtyp = geo["flag"] & 3
    boxes = {"regular": 0, "cut": 0, "covered": 0}
    for k in range(0, n[2], 32):
        for j in range(0, n[1], 32):
            for i in range(0, n[0], 32):
                b = typ[k:k + 32, j:j + 32, i:i + 32]
                g2 = gtyp[3 + k:7 + k + 32, 3 + j:7 + j + 32, 3 + i:7 + i + 32]
                boxes["covered" if np.all(b == 3) else
                      "regular" if np.all(g2 == 0) else "cut"] += 1
    zones = n[0] * n[1] * n[2]
    out = {"domain": list(n), "cells": zones, "cut_cells": int((typ == 1).sum()),
           "covered_cells": int((typ == 3).sum()), "boxes_32": boxes,
           "geometry_build_s": geo_s, "method": "MOL-PLM RK2, two-shock Riemann, FluxRedist",
           "cfl": 0.3, "steps": nsteps,
           "parity": "EB hydro: the reference's EB kernels bit for bit; flux and state "
                     "redistribution and the sphere geometry are restated (AMReX absent: "
                     "unpinned against AMReX)"}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # 32^3 boxes (the configuration): regular boxes through the batched
    # regular hydro, cut boxes through the EB hydro, covered boxes skipped;
    # then the whole domain as one EB box for comparison
    for key, mgs, k in (("eb_level", (32, 32, 32), nsteps),
                        ("eb_level_one_box", (0, 0, 0), max(1, nsteps // 5))):
        L = hydro.EBLevel(geom, prm, geo, redist=1, max_grid_size=mgs)
        st = L.torch_stream()
        L.set_state(s0)
        L.init_finalize()
        L.advance(1)
        L.autotune()
        L.advance(warmup)
        torch.cuda.synchronize()
        prof = key == "eb_level"
        if prof:
            profile_range(args, True)
        e0.record(st)
        L.advance(k)
        e1.record(st)
        torch.cuda.synchronize()
        if prof:
            profile_range(args, False)
        ms = e0.elapsed_time(e1) / k
        fin = L.get_state()
        out[key] = {"ms_per_step": ms, "zone_updates_per_s": zones / (ms * 1e-3),
                    "steps": k, "max_grid_size": list(mgs),
                    "kernels_per_step_graph": L.kernels_per_step(),
                    "boxes": L.boxes(),
                    "device_error": list(L.error()),
                    "t_final": float(L.dts().sum()),
                    "finite": bool(np.isfinite(fin).all())}
        if prof:
            ms_main = ms
        L.close()
        del L
        torch.cuda.empty_cache()
    ms = ms_main
    # the same domain and flow without the sphere, regular MOL level driver
    R = hydro.Level(geom, prm, use_graph=True)
    st = R.torch_stream()
    R.set_state(problems.sod(n, (dx,) * 3))
    R.init_finalize()
    R.advance(warmup)
    torch.cuda.synchronize()
    e0.record(st)
    R.advance(nsteps)
    e1.record(st)
    torch.cuda.synchronize()
    msr = e0.elapsed_time(e1) / nsteps
    out["regular_level_same_domain"] = {"ms_per_step": msr,
                                        "zone_updates_per_s": zones / (msr * 1e-3)}
    out["eb_over_regular_time"] = ms / msr
    # with the same geometry and 32^3 boxes: Godunov-PLM (CTU, 6 ghost
    # cells) and MOL with state redistribution (6 ghost cells)
    geo6 = eb_geometry.sphere_geometry((-6, -6, -6), (n[0] + 5, n[1] + 5, n[2] + 5), dx,
                                       center=(1.0, 0.5, 0.5), radius=0.15)
    for key, kw, redist in (("eb_level_godunov_plm", dict(do_mol=0, ppm_type=0), 1),
                            ("eb_level_state_redist", dict(do_mol=1, ppm_type=0), 2)):
        L = hydro.EBLevel(geom, native.default_params(cfl=0.3, **kw), geo6, redist=redist,
                          max_grid_size=(32, 32, 32))
        st = L.torch_stream()
        L.set_state(s0)
        L.init_finalize()
        L.advance(1)
        L.autotune()
        L.advance(warmup)
        torch.cuda.synchronize()
        e0.record(st)
        L.advance(nsteps)
        e1.record(st)
        torch.cuda.synchronize()
        msc = e0.elapsed_time(e1) / nsteps
        fin = L.get_state()
        out[key] = {"ms_per_step": msc, "zone_updates_per_s": zones / (msc * 1e-3),
                    "steps": nsteps, "max_grid_size": [32, 32, 32], "redist": redist,
                    "kernels_per_step_graph": L.kernels_per_step(),
                    "boxes": L.boxes(), "device_error": list(L.error()),
                    "t_final": float(L.dts().sum()),
                    "finite": bool(np.isfinite(fin).all())}
        L.close()
        del L
        torch.cuda.empty_cache()
    R.close()
    del R
    torch.cuda.empty_cache()
    if not args.no_cpu:
        import oracle
        if os.path.exists(oracle.lib_path_eb()):
            cdx = 2.0 / cpu_n[0]
            cgeo = eb_geometry.sphere_geometry((-5, -5, -5), tuple(v + 4 for v in cpu_n), cdx,
                                               center=(1.0, 0.5, 0.5), radius=0.15)
            cs = np.ascontiguousarray(problems.sod_sphere(cpu_n, (cdx,) * 3, cgeo))
            cp = oracle.default_params(do_mol=1, cfl=0.3)
            clev = oracle.make_level(cpu_n, periodic=(0, 0, 0), bc_lo=(2, 4, 4),
                                     bc_hi=(2, 4, 4), dx=(cdx,) * 3)
            oracle.eb_init_finalize(cp, clev, cs)
            csteps = 2
            t0 = time.time()
            oracle.eb_advance(cp, clev, cgeo, cs, csteps)
            secs = time.time() - t0
            out["cpu_baseline"] = {
                "value": cpu_n[0] * cpu_n[1] * cpu_n[2] * csteps / secs,
                "unit": "zone-updates/s", "cores": 1, "kind": "reference",
                "sample": f"{cpu_n[0]}x{cpu_n[1]}x{cpu_n[2]} Sod+sphere, {csteps} level steps, "
                          "the reference's EB hydro kernels (one thread)"}
    return out


def adjoint_comparison(args, n=128, nsteps=200, every=20, fd_cells=0):
    """The adjoint configuration: 128^3 periodic, MOL-PLM RK2 (CFL 0.3),
    200 steps with a checkpoint every 20, J = mass inside the sphere r < 0.2
    at the final time, dJ/d(initial rho) from the hand-written adjoint.
    Reports forward and backward device times and their ratio per step;
    with fd_cells > 0 also central differences (eps = 1e-6 rho) at that many
    seeded cells inside the sphere."""
    import torch

    from camr_b200 import adjoint, hydro, native, problems
    nn = (n, n, n)
    s, r = problems.grf_blast(nn)
    geom = hydro.make_geom(nn)
    prm = native.default_params(do_mol=1, ppm_type=0, cfl=0.3)
    A = adjoint.AdjointLevel(geom, prm, checkpoint_every=every)
    S0 = torch.from_numpy(s).cuda()
    dV = 1.0 / (n ** 3)
    mask = torch.from_numpy((r < 0.2).astype(np.float64)).cuda()
    lam = torch.zeros_like(S0)
    lam[0] = mask * dV
    A.forward(S0, 2)          # warm-up (module load, allocation)
    A.backward(lam)
    torch.cuda.synchronize()
    st = A._stream if A._stream is not None else torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(st)
    A.forward(S0, nsteps)
    ev[1].record(st)
    g = A.backward(lam)
    ev[2].record(st)
    torch.cuda.synchronize()
    fwd_ms = ev[0].elapsed_time(ev[1])
    bwd_ms = ev[1].elapsed_time(ev[2])
    dts = A.dts()
    grad = (g[0] + g[7]).cpu().numpy()  # d/d rho at fixed p, u = 0
    out = {"domain": list(nn), "steps": nsteps, "checkpoint_every": every,
           "forward_ms_per_step": fwd_ms / nsteps,
           "backward_ms_per_step": bwd_ms / nsteps,
           "adjoint_over_forward": bwd_ms / fwd_ms,
           "timing": "CUDA events on the adjoint's stream",
           "device_error": list(A.error())}
    if fd_cells:
        # Central differences (eps = 1e-6 rho at fixed p, u) of J at seeded
        # cells inside the sphere, with the forward dt sequence frozen.  The
        # one-sided differences D+ and D- are kept too: where the +-eps runs
        # straddle a limiter or Riemann branch (a kink of J), D+ and D- part
        # and the central difference is the mean of two one-sided slopes,
        # while the adjoint takes the slope of the branch the forward took.
        rng = np.random.default_rng(64)
        inside = np.argwhere(r < 0.2)
        cells = [tuple(int(v) for v in inside[t])
                 for t in rng.choice(len(inside), fd_cells, replace=False)]

        # The change of J, not J itself, is summed: J - J0 = dV sum(mask
        # (rho - rho0)) over the final densities.  J is ~0.03 and its change
        # ~1e-13, so differences of two separately rounded sums of J would
        # leave only ~1e4 ulps of J and a quantised difference quotient.
        rho0 = A.forward(torch.from_numpy(s).cuda(), nsteps, fixed_dts=dts)[0].clone()

        def dJ(state):
            o = A.forward(torch.from_numpy(state).cuda(), nsteps, fixed_dts=dts)
            return float(((o[0] - rho0) * mask).sum()) * dV

        samples = []
        for (k, j, i) in cells:
            eps = 1e-6 * s[0, k, j, i]
            res = []
            for sg in (1.0, -1.0):
                st = s.copy()
                st[0, k, j, i] += sg * eps
                st[7, k, j, i] += sg * eps
                res.append(dJ(st))
            fd = (res[0] - res[1]) / (2 * eps)
            dp = res[0] / eps
            dm = -res[1] / eps
            ad = float(grad[k, j, i])
            scale = max(abs(fd), abs(ad), 1e-300)
            kink = abs(dp - dm) / max(abs(dp), abs(dm), 1e-300)
            samples.append({"cell": [i, j, k], "adjoint": ad, "central": fd, "d_plus": dp,
                            "d_minus": dm, "rel_err": abs(fd - ad) / scale,
                            "one_sided_split": kink,
                            "rel_err_nearest_one_sided": min(abs(dp - ad), abs(dm - ad)) / scale})
        errs = np.array([x["rel_err"] for x in samples])
        # a sample straddles a kink when its one-sided slopes part by far
        # more than the O(eps) curvature of a smooth J allows
        kinked = [x for x in samples if x["one_sided_split"] > 1e-4]
        smooth = [x for x in samples if x["one_sided_split"] <= 1e-4]
        out["fd_check"] = {
            "cells": fd_cells, "seed": 64, "eps_rel": 1e-6, "steps": nsteps,
            "median_rel_err": float(np.median(errs)), "max_rel_err": float(errs.max()),
            "frac_within_1e-6": float(np.mean(errs <= 1e-6)),
            "kinked_samples": len(kinked), "kink_criterion": "|D+ - D-| / max|D+-| > 1e-4",
            "smooth_samples": len(smooth),
            "smooth_median_rel_err": (float(np.median([x["rel_err"] for x in smooth]))
                                      if smooth else None),
            "smooth_max_rel_err": (float(max(x["rel_err"] for x in smooth)) if smooth else None),
            "kinked_max_rel_err_vs_nearest_one_sided": (
                float(max(x["rel_err_nearest_one_sided"] for x in kinked)) if kinked else None),
            "samples": samples}
    A.close()
    torch.cuda.empty_cache()
    return out


def run_batched(args, rank):
    """Batched vs per-box launches over the uneven fine-level boxes of the
    two-level configuration (hydro of one level step, CTU-PPM)."""
    import torch

    from camr_b200 import build, hydro, native, problems
    if not os.path.exists(native.LIB_PATH):
        build.build()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    fine_n = 512
    boxes = problems.amr_box_list(nbox=args.nbox, fine_n=fine_n)
    cells = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in boxes)
    items = amr_box_inputs(boxes, fine_n, dev)
    geom = hydro.make_geom((fine_n,) * 3)
    prm = native.default_params(do_mol=0, ppm_type=1, cfl=CFL)
    dt = 0.25 / fine_n / 4.0
    b = hydro.Batch(items, geom, prm)
    torch.cuda.synchronize()
    b.autotune(dt)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    res = {}
    for name, mode in (("per_box", hydro.Batch.PER_BOX), ("batched", hydro.Batch.PERSISTENT)):
        for _ in range(args.warmup):
            b.run(dt, mode)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            b.run(dt, mode)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        res[name] = {"ms": ms, "zone_updates_per_s": cells / (ms * 1e-3)}
    tuning = b.tuning()
    b.close()
    if rank == 0:
        line = {
            "metric": "zone-updates/s (FP64, 1xB200), batched uneven AMR patches",
            "value": res["batched"]["zone_updates_per_s"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["batched"]["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (uneven fine boxes around seeded blobs, box seed 7)",
            "config": {"workload": "c2 fine level: hydro of one level step over uneven boxes",
                       "boxes": len(boxes), "cells": cells, "box_sizes": [16, 24, 32, 48, 64],
                       "method": "CTU-PPM"},
            "per_box": res["per_box"], "batched": res["batched"],
            "speedup_batched_vs_per_box": res["per_box"]["ms"] / res["batched"]["ms"],
            "tuning": tuning,
        }
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["camr", "reference"], default="camr")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", choices=["c1", "c2-batched", "c2-amr", "c3-adjoint", "c4-eb"],
                    default="c1")
    ap.add_argument("--adj-n", type=int, default=128, help="c3-adjoint domain size")
    ap.add_argument("--adj-steps", type=int, default=200, help="c3-adjoint steps")
    ap.add_argument("--fd-cells", type=int, default=64,
                    help="finite-difference cells of the c3-adjoint workload")
    ap.add_argument("--nbox", type=int, default=350)
    ap.add_argument("--amr-steps", type=int, default=4, help="timed coarse steps of c2-amr")
    ap.add_argument("--amr-n0", type=int, default=256,
                    help="base level size of c2-amr (fine index space twice that)")
    ap.add_argument("--eb-steps", type=int, default=150, help="timed steps of c4-eb")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the timed region (C1 steps; c2-amr MOL batched steps; "
                         "c4-eb EB level steps) with cudaProfilerStart/Stop")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-vs-per-box comparison in the default line")
    args = ap.parse_args()
    if args.workload == "c3-adjoint":
        import torch
        from camr_b200 import build, native
        if not os.path.exists(native.LIB_PATH):
            build.build()
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"workload": "c3-adjoint",
                              **adjoint_comparison(args, n=args.adj_n, nsteps=args.adj_steps,
                                                   fd_cells=args.fd_cells)}))
        return
    if args.workload == "c4-eb":
        import torch
        from camr_b200 import build, native
        if not os.path.exists(native.LIB_PATH):
            build.build()
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"workload": "c4-eb", **eb_comparison(args)}))
        return
    if args.workload == "c2-amr":
        import ctypes as C

        import torch
        from camr_b200 import build, native
        if not os.path.exists(native.LIB_PATH):
            build.build()
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        peak = C.c_double()
        native.lib().camr_measure_fp64_peak(C.byref(peak), None)
        args.fp64_peak = peak.value
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"workload": "c2-amr", **amr_comparison(args)}))
        return
    if args.workload == "c2-batched":
        run_batched(args, int(os.environ.get("RANK", "0")))
        return
    if args.impl == "reference":
        # CPU-only arm: rank 0 alone runs it; other ranks exit without work.
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        run_camr(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
