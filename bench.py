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
    "update": (528, "read Sborder, U_old, 3 x 10 fluxes, 3 x 2; write U"),
}
# Whole-step algorithmic bytes per zone-update (read U^n + write U^n+1).
STEP_BYTES_PER_ZONE = 160


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
    sample = (f"{n[0]}^3 sample of the workload (same blob statistics), {args.steps} steps, "
              f"tiles 1024x16x16, {nth} threads")
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic (seeded blobs)",
        "config": {"workload": "c1 CTU-PPM periodic blobs, CFL 0.7", "domain": list(n),
                   "method": "CTU-PPM", "cfl": CFL},
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

    def barrier():
        if pg is not None:
            pg.barrier()

    fp64_peak = C.c_double()
    lib.camr_measure_fp64_peak(C.byref(fp64_peak), C.c_void_p(L.stream_ptr))

    sampler = ClockSampler(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = lib.camr_launch_count()
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    e0.record(st)
    L.advance(args.steps)
    e1.record(st)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = lib.camr_launch_count() - launches0
    err = L.error()
    if pg is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * zones * args.steps / (ms * 1e-3)

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
    dom_bytes = STAGE_BYTES[dom][0] * zones
    achieved = dom_bytes / (acc[dom] * 1e-3) / 1e9
    roofline = {
        "kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
        "frac": achieved / hbm_peak, "peak_source": f"{peak_kind} hbm_gbs",
        "traffic": None, "algorithmic_bytes_per_cell": STAGE_BYTES[dom][0],
        "avg_launch_ms": acc[dom],
        "fp64_peak_tflops_measured": fp64_peak.value,
    }
    step_achieved = STEP_BYTES_PER_ZONE * zones / (ms_step * 1e-3) / 1e9
    step_roofline = {"bytes_per_zone_update": STEP_BYTES_PER_ZONE, "achieved": step_achieved,
                     "peak": hbm_peak, "unit": "GB/s", "frac": step_achieved / hbm_peak}

    # End to end through the C ABI with host buffers: every step uploads the
    # state from pinned host memory, advances, and reads the state back.
    host = torch.from_numpy(s0).pin_memory()
    out = torch.empty_like(host).pin_memory()
    e2e_steps = max(1, min(args.steps, 5))
    e0.record(st)
    for _ in range(e2e_steps):
        native.check(lib.camr_level_set_state(L._h, C.c_void_p(host.data_ptr()), 1), "set")
        L.advance(1)
        native.check(lib.camr_level_get_state(L._h, C.c_void_p(out.data_ptr()), 1), "get")
    e1.record(st)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    if pg is not None:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    state_bytes = host.numel() * 8
    e2e = {"value": world * zones / (e2e_ms * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
           "ms_per_step": e2e_ms}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, secs, kind, nth = cpu_reference_rate(n, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": nth,
               "kind": "reference" if kind == "ref" else "port",
               "sample": f"one full {n[0]}^3 step of the workload ({secs:.1f} s), "
                         "reference hydro kernels, tiles 1024x16x16, all host threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded overpressure blobs, numpy PCG64 seed 1)",
            "config": {"workload": "c1: 256^3 periodic CTU-PPM, CFL 0.7, 16 blobs",
                       "domain": list(n), "method": "CTU Godunov, PPM, two-shock Riemann",
                       "cfl": CFL, "boxes": "64 x 64^3 (advanced as one padded domain)",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (state 1.3 GB, intermediates ~25 GB)"},
            "roofline": roofline, "step_roofline": step_roofline, "cpu_baseline": cpu,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "stages_ms": acc, "device_error": list(err),
        }
        print(json.dumps(line))
    L.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["camr", "reference"], default="camr")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
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
