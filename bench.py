"""Benchmark of the B200 ALE-BGK step: cavity3d Nx=40 Nv=10, quadratic MLS.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is the full time step of the 64 000-particle x 1 000-velocity cloud
(transport, positivity + MOOD screen, mass rescale, diffuse wall, moments, BGK
collision, moments, moodCheck).  The metric is particle x velocity updates
per second.  Under torchrun (N > 1) every rank advances its own independent
cavity on its own GPU -- the cavities do not exchange data -- so per-GPU work
is fixed and scaling is weak; the step time is the max over ranks.

Rank 0 prints one JSON line.  ``--impl reference`` times the reference's own
CPU implementation (compiled unmodified into oracle/_ref) on this host's cores
instead.
"""
from __future__ import annotations

import argparse
import ctypes
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

WORKLOAD = dict(case="cavity3d", Nx=40, Nv=10, mls_order=2)
METRIC = "cavity3d Nx40 Nv10 updates/s"
BYTES_PER_UPDATE_FP32 = 8.0     # read f once + write f once, FP32
# The reference's Solver/CudaBackend.cu, compiled unmodified for sm_100a, on
# this workload (cavity3d Nx40 Nv10, quadratic MLS, FP64): recorded.
REFERENCE_GPU = {"ms_per_step": 99.50, "updates_per_s": 6.432e8, "kind": "recorded",
                 "sample": "10 timed cudaStep calls after 3, one B200, SM 1965 MHz"}
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--workload", default="cavity3d",
                    choices=["cavity3d", "batched-cavity2d", "warm-start", "free-body",
                             "fp32-error"],
                    help="cavity3d (the headline line), the batched cavity2d workload "
                         "(96 seeded cavities advanced by one graph launch per step), or the "
                         "learned warm start on 32 held-out cavity2d cases")
    ap.add_argument("--batch", type=int, default=96)
    ap.add_argument("--batch-form", default="auto",
                    choices=["auto", "stages", "branches", "persistent"],
                    help="batched-cavity2d graph form: autotuned, stage groups (4), one "
                         "persistent launch per step, or per-cavity branches")
    ap.add_argument("--screen-floor-run", action="store_true",
                    help="free-body: a fourth run, FP64 with the FP32 MOOD screen's rounding "
                         "floor, to separate the screen's decisions from FP32 arithmetic")
    ap.add_argument("--no-steady", action="store_true",
                    help="batched-cavity2d: skip the run to the steady residual")
    ap.add_argument("--ncu", action="store_true",
                    help="profiler mode: --warmup steps then --steps steps, no timing "
                         "and no JSON (for ncu launch lists and captures)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of every rank's x (a step time): the job is as fast as
    its slowest cavity.  Every rank must call it, in the same order."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(world: int, updates_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job updates/s: every rank advances its own cavity of the same
    size, so the job does world x updates x steps in the max-over-ranks time."""
    return world * updates_per_rank * steps / seconds


def e2e_bytes(N: int, V: int, gstride: int, precision: int):
    """(host-to-device, device-to-host, host input) bytes of one end-to-end
    step: alebgk_upload_state of the FP64 host rows (N x gstride) and macros
    (N x 7), then alebgk_download_moments.  An FP32 context whose FP32 rows
    (the device stride: V rounded up to a multiple of four) take at least
    32 MiB rounds them on the host and copies FP32 rows; smaller FP32 clouds
    and FP64 contexts copy the FP64 rows.  The macros cross as N x 6 doubles
    plus the N MOOD flags (4-byte ints), each way."""
    ldf = (V + 3) // 4 * 4
    ring = precision == 32 and N * ldf * 4 >= (32 << 20)
    h2d = (N * ldf * 4 if ring else N * gstride * 8) + N * (48 + 4)
    d2h = N * (48 + 4)
    host_in = N * gstride * 8 + N * 7 * 8
    return h2d, d2h, host_in


# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def recorded_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d[kernel]
        return float(e["bytes_per_launch"]), e.get("source", "")
    except (OSError, KeyError, ValueError):
        return None, ""


# ---------------------------------------------------------------------------
class _StdoutToStderr:
    """Sends file descriptor 1 to stderr while the reference's CPU code runs:
    it prints progress lines, and stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def cpu_baseline_reference(seconds_budget: float = 40.0):
    with _StdoutToStderr():
        return _cpu_baseline_reference(seconds_budget)


def _cpu_baseline_reference(seconds_budget: float):
    """One full reference CPU step of the same workload on all host cores."""
    from oracle.oracle import RefCase, ref_library
    if ref_library() is None:
        return None
    r = RefCase(WORKLOAD["case"], WORKLOAD["Nx"], WORKLOAD["Nv"], -1.0, WORKLOAD["mls_order"])
    cores = os.cpu_count() or 1
    r.set_threads(cores)
    r.step(1)                      # step 1 (first touch of every buffer) untimed
    t0 = time.perf_counter()
    r.step(1)
    t = time.perf_counter() - t0
    updates = r.N * r.Nv ** 3
    return {"value": updates / t, "unit": "updates/s", "cores": cores, "kind": "reference",
            "sample": f"step 2 of {WORKLOAD['case']} Nx40 Nv10 quadratic "
                      f"({r.N} x {r.Nv ** 3} updates, {t:.1f} s) after an untimed step 1, "
                      f"reference CPU build {os.path.basename(r.path)}, OpenMP {cores} threads"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    with _StdoutToStderr():
        line = _run_reference(args)
    print(json.dumps(line))


def _run_reference(args):
    from oracle.oracle import RefCase, ref_library
    if ref_library() is None:
        return {"impl": "reference",
                "unavailable": "oracle/_ref (the compiled reference) is not built"}
    cores = os.cpu_count() or 1
    r = RefCase(WORKLOAD["case"], WORKLOAD["Nx"], WORKLOAD["Nv"], -1.0, WORKLOAD["mls_order"])
    r.set_threads(cores)
    updates = r.N * r.Nv ** 3
    # A bounded sample: the first warm-up step is timed to project the run;
    # steps are capped so that the whole arm ends within a few minutes.  At
    # the reference's 7.9 s per step on the box's 16 cores, 240 s covers the
    # default 3 warm-up and 20 timed steps in full.
    budget = float(os.environ.get("ALEBGK_REF_BUDGET_S", "240"))
    t0 = time.perf_counter()
    r.step(1)
    t1 = time.perf_counter() - t0
    warm = max(0, min(args.warmup, int(budget * 0.25 / max(t1, 1e-9))) - 1)
    if warm:
        r.step(warm)
    k = max(1, min(args.steps, int(budget / max(t1, 1e-9))))
    t0 = time.perf_counter()
    r.step(k)
    t = time.perf_counter() - t0
    v = updates * k / t
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "updates/s",
        "n_gpus": 0, "steps": k, "warmup": warm + 1, "ms_per_step": 1e3 * t / k,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: the reference's own cavity3d case set-up (start from rest)",
        "config": {"workload": "cavity3d Nx=40 Nv=10 quadratic MLS, 64000 particles x "
                               "1000 velocities, dt=1e-11", "mls_order": 2},
        "cpu_baseline": {"value": v, "unit": "updates/s", "cores": cores, "kind": "reference",
                         "sample": f"{k} timed full steps after {warm + 1} warm-up, reference "
                                   f"CPU build {os.path.basename(r.path)}, {cores} OpenMP threads"},
        "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
def run_ours(args):
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    import alebgk4paper_b200 as ab
    from alebgk4paper_b200 import _abi

    case = ab.Case(WORKLOAD["case"], WORKLOAD["Nx"], WORKLOAD["Nv"], -1.0, WORKLOAD["mls_order"])
    N, V = case.N, case.Nv ** 3
    updates = N * V
    s = ab.Solver(case, precision=args.precision, device=local)
    lib = s.lib

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    ms = ctypes.c_float()
    with ClockSampler(local) as clk:
        # warm-up (also captures the two step graphs), held for at least half
        # a second so that the clock samples see the GPU under this load
        s.cudaStep(max(3, args.warmup))
        s.sync()
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 0.5:
            s.cudaStep(4)
            s.sync()
        barrier()
        rc = lib.alebgk_step_timed(s.ctx, args.steps, ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"alebgk_step_timed failed ({rc})")
        barrier()
    t_ms = max_over_ranks(ms.value, dist, "cuda")
    value = weak_value(world, updates, args.steps, t_ms / 1e3)

    # per-stage device times (kernel by kernel, events on the launching stream)
    prof = (ctypes.c_float * _abi.NSTAGES)()
    nprof = 3
    rc = lib.alebgk_profile_steps(s.ctx, nprof, prof)
    if rc != 0:
        raise RuntimeError("alebgk_profile_steps failed")
    stage_ms = {name: prof[i] / nprof for i, name in enumerate(_abi.STAGES)}
    peak, peak_src = measured_peak()
    es = 4 if args.precision == 32 else 8
    cnt0 = s.counters()
    kernels = {"transport": "k_march" if cnt0["transport_kernel"] == 2 else "k_transport",
               "particle": {1: "k_particle", 2: "k_particle_stream",
                            3: "k_particle_rows"}[cnt0["particle_kernel"]]}
    # Algorithmic bytes per update: the transport reads f once and writes it
    # once (FP32: 4 + 4 bytes); so does the particle stage.  The roofline is
    # the transport's, the step's single largest kernel.
    per_update = 2 * es
    kern_name = kernels["transport"]
    achieved = per_update * updates / (stage_ms["transport"] / 1e3) / 1e9
    traffic, traffic_src = recorded_traffic(kern_name)
    # The transport's own bound is the FP32 FMA pipe: one FMA per stencil
    # slot and velocity (slots = neighbours + self), against the nominal
    # 128 FP32 FMA per clock per SM at the sampled SM clock.
    fmas = float((case.nnb.astype(np.int64) + 1).sum()) * V
    props = torch.cuda.get_device_properties(local)
    clk_mhz = clk.summary().get("sm_mhz") or 1965.0
    fma_peak = props.multi_processor_count * 128 * clk_mhz * 1e6 / 1e12

    # end to end through the C-ABI with host buffers: every step uploads the
    # full FP64 state from pinned host memory (alebgk_upload_state, the
    # cudaUploadCloud of the reference's hybrid loop), runs one step and reads
    # the moment field back (alebgk_download_moments).
    g_host = torch.empty((N, case.gstride), dtype=torch.float64, pin_memory=True)
    mac_host = torch.empty((N, 7), dtype=torch.float64, pin_memory=True)
    gd, md = s.cudaDownloadFull()
    g_host.copy_(torch.from_numpy(gd))
    mac_host.copy_(torch.from_numpy(md))
    gp = ctypes.cast(g_host.data_ptr(), _abi.c_double_p)
    mp = ctypes.cast(mac_host.data_ptr(), _abi.c_double_p)

    def e2e_step():
        r1 = lib.alebgk_upload_state(s.ctx, gp, mp)
        r2 = lib.alebgk_step(s.ctx, 1)
        r3 = lib.alebgk_download_moments(s.ctx, mp)
        if r1 or r2 or r3:
            raise RuntimeError("e2e step failed")

    for _ in range(2):
        e2e_step()
    # Three windows of e2e_steps steps each; the median window is reported
    # (host-side timing varies from window to window on a shared host).
    windows = []
    for _ in range(3):
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        barrier()
        windows.append(max_over_ranks(time.perf_counter() - t0, dist, "cuda"))
    te = sorted(windows)[1]
    e2e_value = weak_value(world, updates, args.e2e_steps, te)
    h2d, d2h, host_in = e2e_bytes(N, V, case.gstride, args.precision)

    cnt = s.counters()
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_reference()
        except Exception as exc:  # reported, never gating
            cpu = {"value": None, "unit": "updates/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"not run: {exc}"}

    out = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup),
        "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
        "data": "synthetic: the reference's cavity3d case set-up, gas at rest at t=0",
        "config": {"workload": "cavity3d Nx=40 Nv=10 quadratic MLS, 64000 particles x 1000 "
                               "velocities, dt=1e-11, FP32 f storage + FP32 MLS "
                               "reconstruction, FP64 sums",
                   "particles": N, "velocities": V, "mls_order": 2,
                   "parallelism": f"{world} independent cavities, one per GPU",
                   "l2": "inputs larger than L2: two 256 MB distribution buffers "
                         "ping-pong, no flush needed"},
        # per step in the step graph: k_step_begin twice (the one-block
        # scalar reset, then the NAD ranges on the side stream beside the
        # transport), then transport, particle, redo, sigma, fixup, mass_sum,
        # scale_mood, recollide, mass_end
        "gpu_launches": 11 * args.steps,
        "kernels": kernels,
        "stage_ms": {k: round(v, 5) for k, v in stage_ms.items()},
        "roofline": {"bound": "hbm", "kernel": kern_name, "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "algorithmic_bytes_per_launch": per_update * updates},
        # the reference's own GPU path (Solver/CudaBackend.cu for sm_100a,
        # FP64, quadratic MLS) on the same workload, timed by
        # oracle/time_reference_gpu.py on a B200 of this pool
        "reference_gpu": REFERENCE_GPU,
        "vs_reference_gpu": value / REFERENCE_GPU["updates_per_s"],
        "transport_fma_roofline": {
            "bound": "fp32-fma", "kernel": kernels["transport"],
            "achieved": fmas / (stage_ms["transport"] / 1e3) / 1e12,
            "peak": fma_peak, "unit": "TFMA/s",
            "frac": fmas / (stage_ms["transport"] / 1e3) / 1e12 / fma_peak,
            "peak_source": "nominal: SMs x 128 FP32 FMA/clk at the sampled SM clock",
            "algorithmic_fma_per_launch": fmas},
        "particle_roofline": {
            "bound": "hbm", "kernel": kernels["particle"],
            "achieved": per_update * updates / (stage_ms["particle"] / 1e3) / 1e9,
            "peak": peak, "unit": "GB/s",
            "frac": per_update * updates / (stage_ms["particle"] / 1e3) / 1e9 / peak,
            "traffic": recorded_traffic(kernels["particle"])[0]},
        "step_roofline": {"achieved": BYTES_PER_UPDATE_FP32 * (es / 4) * updates /
                                      (t_ms / args.steps / 1e3) / 1e9,
                          "peak": peak, "unit": "GB/s",
                          "frac": BYTES_PER_UPDATE_FP32 * (es / 4) * updates /
                                  (t_ms / args.steps / 1e3) / 1e9 / peak,
                          "note": "whole step against 8 B/update (FP32) algorithmic bytes"},
        "e2e": {"value": e2e_value, "unit": "updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
                "windows_ms_per_step": [round(1e3 * w / args.e2e_steps, 3) for w in windows],
                "timing": "median of three windows of the steps",
                "host_input_bytes_per_step": host_in,
                "path": "alebgk_upload_state + alebgk_step + alebgk_download_moments, "
                        "pinned host buffers, wall clock" +
                        ("; FP32 rows rounded on the host cores into a pinned ring, "
                         "overlapped with the copies" if h2d < host_in else "")},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "counters": {"transport_flags": cnt["transport_flags"],
                     "mood_fail": cnt["mood_fail"]},
    }
    print(json.dumps(out))


def batched_roofline(updates, steps, seconds, precision):
    es = 4 if precision == 32 else 8
    achieved = 2 * es * updates * steps / seconds / 1e9
    peak, src = measured_peak()
    return {"bound": "hbm", "kernel": "whole batch step", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_source": src, "traffic": None,
            "bytes_per_update": 2 * es}


def run_batched(args):
    """Batched cavity2d on one GPU (ranks > 0 of a torchrun take their LPT
    share of the instances): step throughput of the whole batch, then the
    steps and wall time until every cavity is steady (residual < 1e-6)."""
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    from alebgk4paper_b200.batch import BatchSolver, batched_cavity2d, partition_lpt
    specs = batched_cavity2d(args.batch, seed=0)
    mine = partition_lpt([s["Nx"] ** 2 * s["Nv"] ** 2 for s in specs], world)[rank]
    b = BatchSolver([specs[i] for i in mine], precision=args.precision, device=local,
                    launch="stages" if args.batch_form == "auto" else args.batch_form)
    if args.batch_form == "auto":
        b.autotune(3)
    with ClockSampler(local) as clk:
        b.step(max(3, args.warmup))
        b.sync()
        t0 = time.perf_counter()
        b.step(args.steps)
        b.sync()
        t = time.perf_counter() - t0
    updates = b.updates_per_step
    form, launch = b.staged, b.launch
    b.close()
    # Steps and wall time to steady from the Maxwellian at rest: a fresh
    # batch, timed from before its autotuning (the host set-up excluded).
    done, t_steady = np.zeros(1, np.int64), None
    if not args.no_steady:
        b = BatchSolver([specs[i] for i in mine], precision=args.precision, device=local,
                        launch="stages" if args.batch_form == "auto" else args.batch_form)
        b.sync()
        t1 = time.perf_counter()
        if args.batch_form == "auto":
            b.autotune(3)
        done = b.run_to_steady(tol=1e-6, check_every=100, max_steps=50000)
        t_steady = time.perf_counter() - t1
        b.close()
    if rank != 0:
        return
    print(json.dumps({
        "metric": "batched cavity2d updates/s", "value": updates * args.steps / t,
        "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == 32 else "f64",
        "data": "synthetic: seeded batched cavity2d instances (Nx, Nv, lid, density)",
        "config": {"workload": f"batched cavity2d, {len(mine)} of {args.batch} instances on "
                               f"rank 0, one CUDA graph launch per step, launch form "
                               f"{args.batch_form}", "instances": len(mine),
                   "launch_form": ("one persistent launch per step" if launch == "persistent"
                                   and form else f"stage launches in {form} groups" if form
                                   else "per-cavity graph branches")},
        "timing": "wall clock around synchronised graph launches",
        # the whole step's algorithmic traffic: every update reads f and
        # writes it once in the transport+particle stage (4 + 4 bytes FP32)
        # and the macros' traffic is small beside it
        "roofline": batched_roofline(updates, args.steps, t, args.precision),
        "steady": None if args.no_steady else {
            "tol": 1e-6, "max_steps_to_steady": int(done.max()),
            "all_steady": bool((done > 0).all()), "seconds": t_steady,
            "seconds_cover": "autotuning and every step from the Maxwellian at rest"},
        "clocks": clk.summary(),
    }))


def run_warm_start(args):
    """Learned warm start on held-out cavities (Nx = 48, Nv = 20): wall time
    to the steady residual from the plain start over that from the seeded
    start, plus the network kernels' own throughput.  Steady: the mean change
    per step over a 200-step interval below 5e-7, momentum against the lid
    momentum; both steady states are compared with each other and with a
    40000-step cold run."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    from alebgk4paper_b200 import warm_train as wt
    from alebgk4paper_b200 import warmstart as ws
    net = ws.WarmStartNet.load(wt.DEFAULT_MODEL, device=local)
    with ClockSampler(local) as clk:
        r = wt.evaluate(net, wt.heldout_specs(32), reference_steps=40000)
    # network throughput: inference over the 32 cases' points, one training step
    rng = np.random.default_rng(0)
    pts = torch.as_tensor(rng.uniform(0, 1, (73728, 4)).astype(np.float32), device="cuda")
    tgt = torch.zeros((16384, 16), dtype=torch.float32, device="cuda")
    for _ in range(3):
        net.forward(pts)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(20):
        net.forward(pts)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / 20
    flop_fwd = 2 * (64 * 128 + 3 * 128 * 128 + 128 * 16)
    print(json.dumps({
        "metric": "warm-start wall-time speed-up to the steady residual",
        "value": r["wall_ratio"], "unit": "x", "n_gpus": 1, "steps": None, "warmup": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 network, f32 solver",
        "data": "synthetic: 32 held-out seeded cavity2d cases (seed 2000), model trained on "
                "2000 seeded steady states of the batched solver (seed 1000)",
        "config": {"workload": "learned warm start, cavity2d Nx=48 Nv=20, 32 held-out cases",
                   "steady": {"tol": r["tol"], "check_every": r["check_every"],
                              "residual": r["residual"]}},
        "steps_ratio": r["steps_ratio"], "cold_steps_mean": r["cold_steps_mean"],
        "warm_steps_mean": r["warm_steps_mean"], "cold_seconds": r["cold_seconds"],
        "warm_seconds": r["warm_seconds"], "all_steady": r["all_steady"],
        "field_rel_err_max": r["field_rel_err_max"],
        "vs_converged_max": r["vs_converged_max"],
        "network": {"forward_points": 73728, "forward_ms": fwd_ms,
                    "forward_tflops": flop_fwd * 73728 / (fwd_ms * 1e-3) / 1e12},
        "clocks": clk.summary(),
    }))
    net.close()


def run_ncu(args):
    import alebgk4paper_b200 as ab
    case = ab.Case(WORKLOAD["case"], WORKLOAD["Nx"], WORKLOAD["Nv"], -1.0, WORKLOAD["mls_order"])
    s = ab.Solver(case, precision=args.precision)
    s.cudaStep(args.warmup)
    s.cudaStep(args.steps)
    s.sync()
    s.close()


def run_fp32_error(args):
    """cavity3d Nx40 Nv10 from rest in FP32 (the bench's mode) and in FP64 on
    the device, side by side for --steps steps (the configuration's length
    is 2000): the relative L2 error of every macroscopic field and of f
    against the FP64 run, at checkpoints along the way."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    import alebgk4paper_b200 as ab
    steps = args.steps
    c = ab.Case(WORKLOAD["case"], WORKLOAD["Nx"], WORKLOAD["Nv"], -1.0, WORKLOAD["mls_order"])
    s32 = ab.Solver(c, precision=32, device=local)
    s64 = ab.Solver(c, precision=64, device=local)
    names = ("rho", "ux", "uy", "uz", "T", "p")
    marks = sorted({k for k in (1, 10, 100, 250, 500, 1000, 1500, 2000) if k <= steps} | {steps})
    rows, done = [], 0

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    with ClockSampler(local) as clk:
        for k in marks:
            s32.cudaStep(k - done)
            s64.cudaStep(k - done)
            done = k
            g32, m32 = s32.cudaDownloadFull()
            g64, m64 = s64.cudaDownloadFull()
            row = {"step": k, "f": rel(g32, g64)}
            for j, n in enumerate(names):
                if n in ("ux", "uy", "uz"):
                    # velocities against the thermal speed sqrt(R T) of the FP64 run
                    th = np.sqrt(208.0 * m64[:, 4])
                    row[n] = float(np.linalg.norm((m32[:, j] - m64[:, j]) / th) /
                                   np.sqrt(len(th)))
                else:
                    row[n] = rel(m32[:, j], m64[:, j])
            rows.append(row)
    s32.close()
    s64.close()
    print(json.dumps({
        "metric": "FP32 field error against the FP64 device run", "value": rows[-1]["rho"],
        "unit": "relative L2 (rho)", "n_gpus": 1, "steps": steps, "warmup": 0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 against f64", "data": "synthetic: the reference's cavity3d case from rest",
        "config": {"workload": "cavity3d Nx=40 Nv=10 quadratic MLS, 64000 x 1000",
                   "velocity_error": "RMS of (u32 - u64) / sqrt(R T64) over particles"},
        "errors": rows, "clocks": clk.summary(),
    }))


def run_free_body(args):
    """The free-body cube (cavity3d-cube Nx40 Nv10, density 4.4, parabolic lid
    10 m/s, dt 1.5e-11): --warmup untimed then --steps timed steps of fluid
    step, Heun body step and cloud management, in FP32, in FP64, and in FP64
    from the FP32-rounded initial state; per-step wall time, the cube's path
    (all steps) and accumulated rotation, and the deviations of the FP32 run
    and of the rounded-start FP64 run from the FP64 run."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    import alebgk4paper_b200 as ab
    runs = {}
    # FP32, FP64, and FP64 started from the FP32-rounded initial state: the
    # third run measures how far the body's path moves under a perturbation
    # of the size of FP32 rounding alone, against which the FP32 run's
    # deviation from FP64 is read.
    plan = [(32, 32, False), (64, 64, False), ("64r", 64, True)]
    if args.screen_floor_run:
        plan.append(("64f", 64, False))
    for tag, prec, rounded in plan:
        c = ab.Case("cavity3d-cube", 40, 10, -1.0, 2, fixed_body=False)
        if rounded:
            c.g[:] = c.g.astype(np.float32).astype(np.float64)
        s = ab.Solver(c, precision=prec, device=local)
        st = c.bodies.copy()
        path, t_step, t_body, t_refresh, changes = [st.copy()], 0.0, 0.0, 0.0, 0
        # the density range every 100 steps (the scheme's own instability
        # shows there first), and the first step with a non-finite body state
        rho_range, nonfinite = [], None
        with ClockSampler(local) as clk:
            for k in range(args.warmup + args.steps):
                if tag == "64f":
                    # the FP32 screen's floor (a rebuilt context starts without it)
                    s.set_nad_floor(64 * 2.0 ** -24)
                if k == args.warmup:
                    t_step = t_body = t_refresh = 0.0
                t0 = time.perf_counter()
                s.cudaStep(1)
                s.sync()
                t1 = time.perf_counter()
                st = s.body_step(st)
                c.bodies = st
                t2 = time.perf_counter()
                changes += sum(s.refresh_geometry())
                t3 = time.perf_counter()
                t_step += t1 - t0
                t_body += t2 - t1
                t_refresh += t3 - t2
                path.append(st.copy())
                if not np.isfinite(st).all():
                    nonfinite = k + 1
                    break
                if (k + 1) % 100 == 0:
                    m = s.cudaDownloadMoments()
                    rho_range.append([k + 1, float(np.nanmin(m[:, 0])), float(np.nanmax(m[:, 0]))])
        s.close()
        path = np.array(path)[:, 0]
        R = path[:, 22:31].reshape(-1, 3, 3)
        R0T = R[0].T
        ang = [float(np.degrees(np.arccos(np.clip((np.trace(Ri @ R0T) - 1) / 2, -1, 1))))
               for Ri in R]
        done = max(1, len(path) - 1 - args.warmup)
        runs[tag] = dict(path=path, angle=np.array(ang), rho_range=rho_range, nonfinite=nonfinite,
                          s_per_step=(t_step + t_body + t_refresh) / done,
                          fluid_ms=1e3 * t_step / done, body_ms=1e3 * t_body / done,
                          refresh_ms=1e3 * t_refresh / done, cloud_changes=changes,
                          clocks=clk.summary())
    a, b, br = runs[32], runs[64], runs["64r"]
    allr = list(runs.values())
    # compare over the steps every run finished with a finite body state
    n = min(len(x["path"]) for x in allr)
    while n > 1 and not all(np.isfinite(x["path"][n - 1]).all() for x in allr):
        n -= 1
    for x in allr:
        x["path"], x["angle"] = x["path"][:n], x["angle"][:n]
    disp64 = b["path"][-1, 0:3] - b["path"][0, 0:3]
    dev_centre = float(np.abs(a["path"][:, 0:3] - b["path"][:, 0:3]).max())
    dev_centre_r = float(np.abs(br["path"][:, 0:3] - b["path"][:, 0:3]).max())

    def rot_rel(x, y):
        return float(abs(x["angle"][-1] - y["angle"][-1]) / max(abs(y["angle"][-1]), 1e-300))
    print(json.dumps({
        "metric": "free-body cube steps/s", "value": 1.0 / a["s_per_step"], "unit": "steps/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 fluid, f64 body",
        "data": "synthetic: the reference's cavity3d-cube free-body case set-up",
        "config": {"workload": "cavity3d-cube free body Nx=40 Nv=10, rho 4.4, parabolic lid "
                               "10 m/s, dt 1.5e-11"},
        "f32": {k: a[k] for k in ("s_per_step", "fluid_ms", "body_ms", "refresh_ms",
                                  "cloud_changes", "nonfinite", "rho_range")},
        "f64": {k: b[k] for k in ("s_per_step", "fluid_ms", "body_ms", "refresh_ms",
                                  "cloud_changes", "nonfinite", "rho_range")},
        "compared_steps": n - 1,
        "rotation_deg": {"f32": float(a["angle"][-1]), "f64": float(b["angle"][-1]),
                         "f64_rounded_start": float(br["angle"][-1]),
                         "rel_diff": rot_rel(a, b),
                         "rel_diff_f64_rounded_start": rot_rel(br, b)},
        "rotation_rel_diff_by_step": {
            str(k): {"f32": rot_rel({"angle": a["angle"][:k + 1]}, {"angle": b["angle"][:k + 1]}),
                     "f64_rounded_start": rot_rel({"angle": br["angle"][:k + 1]},
                                                  {"angle": b["angle"][:k + 1]})}
            for k in sorted({min(len(b["angle"]) - 1, m) for m in (500, 1000, 2000, 3000,
                                                                   4000, 5000)})},
        # FP32 against FP64 run with the FP32 screen's floor: what FP32
        # arithmetic alone contributes
        "rotation_rel_diff_f32_vs_f64_fp32_floor": None if "64f" not in runs else {
            str(k): rot_rel({"angle": a["angle"][:k + 1]}, {"angle": runs["64f"]["angle"][:k + 1]})
            for k in sorted({min(len(b["angle"]) - 1, m) for m in (100, 250, 500, 1000, 2000,
                                                                   3000)})},
        "displacement_m": {"f64": disp64.tolist(),
                           "max_centre_diff_m": dev_centre,
                           "max_centre_diff_f64_rounded_start_m": dev_centre_r,
                           "rel_to_displacement": dev_centre / max(np.linalg.norm(disp64),
                                                                   1e-300)},
        "clocks": a["clocks"],
    }))


def run_ncu_warm(args):
    """Profiler mode of the warm-start workload: the network kernels alone,
    three inference passes and three training steps on seeded points."""
    import torch
    from alebgk4paper_b200 import warm_train as wt
    from alebgk4paper_b200 import warmstart as ws
    net = ws.WarmStartNet.load(wt.DEFAULT_MODEL)
    rng = np.random.default_rng(0)
    pts = rng.uniform(0, 1, (73728, 4)).astype(np.float32)
    tgt = rng.normal(size=(73728, 9)).astype(np.float32)
    for _ in range(3):
        net.forward(pts)
    net.fit(pts, tgt, steps=3, batch=16384, log_every=0)
    torch.cuda.synchronize()
    net.close()


def main():
    args = parse()
    if args.ncu and args.workload == "warm-start":
        run_ncu_warm(args)
    elif args.ncu:
        run_ncu(args)
    elif args.workload == "batched-cavity2d" and args.impl == "ours":
        run_batched(args)
    elif args.workload == "warm-start" and args.impl == "ours":
        run_warm_start(args)
    elif args.workload == "free-body" and args.impl == "ours":
        run_free_body(args)
    elif args.workload == "fp32-error" and args.impl == "ours":
        run_fp32_error(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
