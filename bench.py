"""Benchmark of the quantized MLS-MPM substep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one substep over all particles): the 3D mixed scene,
128^3 grid, 2,097,152 particles in 4 random boxes (2 fixed-corotated
elastic, 2 fluid), dt 2e-5, quantized records of 395 bits (7 words, 56 B):
x 3x21 fixed, v 3x12 digits + shared 6-bit exponent, C 9x16 fixed, F 9x16
fixed, 2-bit material id; dithering on.  Synthetic seeded input (numpy
default_rng), no dataset.  Particle records (117 MB) and grids (67 MB) exceed
the 126 MB L2, so no flush is needed between steps.

Reported: particle-substeps/s of the quantized state (`value`), the same
scene with FP32 particle state, the errors of both against an FP64 GPU run
(per field group x, v, C, F, accumulated in FP64 on the device, checked
against a stated bound: position RMS and the reference drivers' loss test),
the same scene on a scheme the analytical solver derives at compression
rate 0.5, the fused kernel's roofline (CUDA-event time per launch vs. the
measured HBM copy bandwidth), end-to-end numbers through the public API with
host buffers (frames of 100 substeps and of 1 substep), and the oracle CPU
port as baseline.

--impl reference times the CPU restatement of the reference's substep
(oracle/, C + OpenMP, all host cores) on a bounded sample of the same scene:
the reference's Taichi build cannot run here (it needs LLVM >= 10 and
Python < 3.10), so the oracle port stands in for it.

With torchrun (N>1) each rank runs an independent replica (the path does not
shard across GPUs without a halo exchange); value = all ranks' particle-
substeps / max over ranks of the timed region.
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

METRIC = "particle-substeps/s quantized vs FP32 on 1 B200 at stated error; HBM GB/s"
UNIT = "particle-substeps/s"
WORKLOAD = "mixed_boxes_3d: 3D MLS-MPM, 128^3 grid, 2,097,152 particles, 4 boxes (2 corotated elastic, 2 fluid), dt 2e-5"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_step
# launch of this workload, from an ncu capture made apart from the bench (a
# number printed under a profiler is never a bench value):
#   ncu --set full --clock-control none -k regex:k_step -s 20 -c 1 \
#       python -m autoquantizer_b200.run_scene --scene mixed_boxes_3d --substeps 40
# It is re-captured whenever k_step changes.
NCU_TRAFFIC_BYTES = 219590144.0
NCU_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, one k_step launch of this workload "
                      "(run_scene --scene mixed_boxes_3d, launch 21), captured separately")

# field groups of the 3D record: slots [lo, hi)
GROUPS_3D = (("x", 0, 3), ("v", 3, 6), ("C", 6, 15), ("F", 15, 24))


def field_errors(a, b):
    """Per field group, RMS and max of |a - b| over particles and components
    (a, b: CUDA float64 n x n_slots states in particle order), the squares
    and maxima accumulated in FP64 on the device (aq_state_error)."""
    import ctypes as C

    from autoquantizer_b200 import _lib

    n, ns = a.shape
    sq = (C.c_double * ns)()
    mx = (C.c_double * ns)()
    _lib.check(_lib.lib().aq_state_error(C.c_void_p(a.data_ptr()), 1, C.c_void_p(b.data_ptr()), 1, n, ns, sq, mx,
                                         _lib.stream_ptr()), "aq_state_error")
    out = {}
    for name, lo, hi in GROUPS_3D:
        out[name] = {"rms": (sum(sq[lo:hi]) / (n * (hi - lo))) ** 0.5, "max": max(mx[lo:hi])}
    return out


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def wait_live(self, limit_s=5.0):
        """Block until the sampler has printed its first line (bounded)."""
        t0 = time.monotonic()
        while self.proc and not self.lines and time.monotonic() - t0 < limit_s:
            time.sleep(0.01)

    def samples_since(self, t):
        return sum(1 for ts, _ in self.lines if ts >= t)

    def stop(self, since=0.0):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if ts < since:
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(backend="nccl"):
    """One process per GPU (torchrun env); each rank is an independent replica
    of the whole workload.  backend "gloo" runs the same host logic on CPU."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ms_per_rank, ws):
    """Whole-job throughput of ws replicas: every rank processes
    units_per_rank; the job takes as long as the slowest rank."""
    ms = max_over_ranks(ms_per_rank, ws)
    return ws * units_per_rank / (ms * 1e-3), ms


def cpu_oracle_rate(cfg, vals, seconds=15.0, stride=16, threads=None):
    """Oracle port (C + OpenMP) on every `stride`-th particle of the scene:
    substeps until `seconds` of wall time; particle-substeps/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from tests.helpers import oracle_layout_from, oracle_params_from
    from autoquantizer_b200.mpm_solver import MPMSolver

    sub = vals[::stride]
    s = MPMSolver(cfg)
    s.set_particles(sub)
    L = oracle_layout_from(s.record())
    P = oracle_params_from(s._params())
    th = threads or host_cores()
    o = O.Sim(P, L, threads=th)
    o.set_state(sub)
    o.substeps(1)  # warm-up
    t0 = time.perf_counter()
    k = 0
    while True:
        o.substeps(1)
        k += 1
        if time.perf_counter() - t0 > seconds or k >= 1000:
            break
    dt = time.perf_counter() - t0
    del s
    return sub.shape[0] * k / dt, th, "every %d-th particle of the scene (%d particles) x %d substeps, %.1f s" % (
        stride, sub.shape[0], k, dt)


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from autoquantizer_b200 import scenes

    cfg, vals = scenes.mixed_boxes_3d(seed=0)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from tests.helpers import oracle_layout_from, oracle_params_from
    from autoquantizer_b200 import quant as Q  # noqa: F401
    from autoquantizer_b200.mpm_solver import MPMSolver

    s = MPMSolver(cfg)  # layout only; no device state is created
    s.set_particles(vals)
    L = oracle_layout_from(s.record())
    th = host_cores()
    # the whole scene when its warm-up and timed substeps fit the budget,
    # else every stride-th particle: one substep of the whole scene first
    # measures what a substep costs here
    o = O.Sim(oracle_params_from(s._params()), L, threads=th)
    o.set_state(vals)
    t0 = time.perf_counter()
    o.substeps(1)
    t1 = time.perf_counter() - t0
    stride = max(1, int(np.ceil((args.steps + args.warmup) * t1 / args.reference_budget_s)))
    sub = vals[::stride]
    if stride > 1:
        s.set_particles(sub)
        o = O.Sim(oracle_params_from(s._params()), L, threads=th)
        o.set_state(sub)
        o.substeps(1)
    for _ in range(max(0, args.warmup - 1)):
        o.substeps(1)
    t0 = time.perf_counter()
    o.substeps(args.steps)
    dt = time.perf_counter() - t0
    v = sub.shape[0] * args.steps / dt
    sample = ("the whole scene (%d particles), one substep per step" % sub.shape[0] if stride == 1 else
              "every %d-th particle of the scene (%d particles), one substep per step" % (stride, sub.shape[0]))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": sample, "same_config": stride == 1,
                       "l2": "inputs larger than L2 not applicable (CPU)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": th, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import ctypes as C

    import torch

    from autoquantizer_b200 import _lib, scenes
    from autoquantizer_b200.mpm_solver import MPMSolver

    torch.cuda.set_device(local)
    cfg, vals = scenes.mixed_boxes_3d(seed=rank)
    n = vals.shape[0]
    K, W = args.steps, args.warmup
    L = _lib.lib()

    def timed(solver, k, prof=False):
        if prof:
            _lib.check(L.aq_sim_profile_enable(solver._sim, 1))
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = solver.launches()
        e0.record()
        solver.substeps(k)
        e1.record()
        torch.cuda.synchronize()
        barrier(ws)
        return e0.elapsed_time(e1), solver.launches() - l0

    # ---- quantized state (the headline)
    q = MPMSolver(cfg)
    q.set_particles(vals)
    q.substeps(W)
    clocks = Clocks(local)
    clocks.start()
    clocks.wait_live()
    t_load = time.monotonic()
    ms, launches = timed(q, K, prof=True)
    t_timed = time.monotonic() - t_load
    value, ms = job_rate(n * K, ms, ws)
    tot = C.c_double()
    cnt = C.c_int64()
    _lib.check(L.aq_sim_profile_get(q._sim, 0, C.byref(tot), C.byref(cnt)))
    step_ms = tot.value / max(1, cnt.value)
    _lib.check(L.aq_sim_profile_get(q._sim, 1, C.byref(tot), C.byref(cnt)))
    grid_ms = tot.value / max(1, cnt.value)
    _lib.check(L.aq_sim_profile_enable(q._sim, 0))
    # A timed region shorter than the sampler's period holds no sample: the
    # same substeps then go on, untimed, until three samples under this load
    # are in (bounded); the error check below runs the other solvers as far.
    extra = 0
    while clocks.samples_since(t_load) < 3 and extra < 20000:
        q.substeps(100)
        torch.cuda.synchronize()
        extra += 100
    ck = clocks.stop(since=t_load)
    ck["window"] = {"timed_s": round(t_timed, 4), "untimed_substeps_after": extra}
    S = q.bytes_per_particle()
    alg_bytes = 2.0 * S * n  # one read + one write of every record per fused launch
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (step_ms * 1e-3) / 1e9
    flags, fallbacks = q.status()

    # ---- FP32 particle state, same scene and code path
    cfg32, _ = scenes.mixed_boxes_3d(seed=rank, quantized=False)
    f = MPMSolver(cfg32)
    f.set_particles(vals)
    S32 = f.bytes_per_particle()
    f.substeps(W)
    ms32, _ = timed(f, K)
    value32, ms32 = job_rate(n * K, ms32, ws)

    # ---- FP64 oracle run on the GPU; per-field errors of both runs after
    # the same W+K(+extra) substeps, accumulated in FP64 on the device
    total = W + K + extra
    cfg64, _ = scenes.mixed_boxes_3d(seed=rank, quantized=False, precision="f64")
    d = MPMSolver(cfg64)
    d.set_particles(vals)
    d.substeps(total)
    f.substeps(extra)
    ref = d.state_tensor(True)
    loss64 = d.compute_loss()
    errs = {}
    for name, sol in (("quantized", q), ("fp32_state", f)):
        fe = field_errors(sol.state_tensor(True), ref)
        loss = sol.compute_loss()
        rel = abs(loss - loss64) / abs(loss64)
        errs[name] = {"fields": fe, "x_rms": fe["x"]["rms"], "x_max": fe["x"]["max"], "loss": loss,
                      "loss_rel_err": rel,
                      "within_bound": bool(fe["x"]["rms"] <= args.x_bound and rel <= 3 * args.loss_eps)}
    del f

    # ---- a scheme derived by the analytical solver at compression rate 0.5
    cr, cfg_cr = None, None
    if not args.no_cr:
        cr, cfg_cr = cr_half_run(args, rank, vals, ref, loss64, total, K, W, ws)
    del d, ref

    # ---- end to end through the public API with host buffers: per step the
    # packed records come from pinned host memory, a frame of substeps runs,
    # the records and the loss go back to the host.
    words = q.words()
    h_in = torch.from_numpy(words.view(np.int64)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    d_words = torch.empty_like(h_in, device="cuda")

    def e2e_step(frame):
        d_words.copy_(h_in, non_blocking=True)
        _lib.check(L.aq_sim_set_words(q._sim, C.c_void_p(d_words.data_ptr()), _lib.stream_ptr()))
        q.substeps(frame)
        _lib.check(L.aq_sim_get_words(q._sim, C.c_void_p(d_words.data_ptr()), _lib.stream_ptr()))
        h_out.copy_(d_words, non_blocking=True)
        return q.compute_loss()  # device->host read of the step's result

    def e2e(frame, steps):
        e2e_step(frame)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            e2e_step(frame)
        e1.record()
        torch.cuda.synchronize()
        v, ms_ = job_rate(n * frame * steps, e0.elapsed_time(e1), ws)
        return {"value": v, "unit": UNIT, "h2d_bytes_per_step": int(h_in.numel() * 8),
                "d2h_bytes_per_step": int(h_out.numel() * 8 + 8), "substeps_per_step": frame, "steps": steps,
                "ms_per_step": ms_ / steps}

    e2e_main = e2e(args.frame, max(1, args.e2e_steps))
    e2e_one = e2e(1, max(3, args.e2e_steps * 4))

    # ---- streamed (out-of-core) mode: the records in pinned host memory,
    # passed through the device in chunks every substep; the host link bounds
    # it, so the record's bytes set the speed
    streamed = None
    if args.stream_steps > 0:
        streamed = streamed_run(q, cfg32, vals, n, args.stream_steps, args.stream_parts, ws, cfg_cr)

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        v, th, sample = cpu_oracle_rate(cfg, vals, seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": th, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (numpy default_rng seeded scene)",
            "config": {"workload": WORKLOAD, "record_bits": q.layout().total_bits, "bytes_per_particle": S,
                       "fp32_bytes_per_particle": 4 * 24, "fp32_record_bytes": S32, "particles_per_gpu": n,
                       "grid": [128, 128, 128],
                       "l2": "inputs larger than L2 (117 MB records + 67 MB grids), no flush",
                       "parallelism": "replicas" if ws > 1 else "single"},
            "fp32_state": {"value": value32, "unit": UNIT, "ms_per_step": ms32 / K,
                           "quantized_speedup": value / value32, "record_bytes": S32,
                           "record": "24 f32 values + 2-bit material id, padded to 13 words"},
            "compression": 96.0 / S,
            "compression_detail": {"vs_fp32_values_96B": 96.0 / S, "vs_fp32_record_run_%dB" % S32: S32 / S,
                                   "bit_dense_vs_fp32_values": 768.0 / q.layout().total_bits},
            "error_vs_fp64": {"substeps": total, **errs,
                              "bound": {"x_rms": args.x_bound, "loss_rel_err": 3 * args.loss_eps,
                                        "stated": "requested: position RMS error <= %g (domain [0,1]^3, "
                                                  "dx = 1/128) and |loss - loss_f64| < 3 eps |loss_f64| with "
                                                  "eps = %g (the reference drivers' success test, "
                                                  "run_mpm_elastic_2d.py:205-207; loss = compute_ek)"
                                                  % (args.x_bound, args.loss_eps)},
                              "loss_f64": loss64,
                              "accumulation": "per slot sum of squares and max in FP64 on the device "
                                              "(aq_state_error); RMS over particles and components of a group"},
            "cr_half_scheme": cr,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": NCU_TRAFFIC_BYTES, "traffic_source": NCU_TRAFFIC_SOURCE,
                         "peak_kind": peak_kind, "kernel": "k_step (fused G2P+P2G)", "avg_launch_ms": step_ms,
                         "alg_bytes_per_launch": alg_bytes, "grid_clear_avg_ms": grid_ms},
            "cpu_baseline": cpu,
            "e2e": e2e_main,
            "e2e_frame1": e2e_one,
            "streamed": streamed,
            "gpu_launches": int(launches),
            "kernel_jit": q.kernel_is_jit(),
            "status": {"flags": flags, "tile_fallbacks": fallbacks},
            "clocks": ck,
        }
        print(json.dumps(line), flush=True)


def streamed_run(q, cfg32, vals, n, steps, parts, ws, cfg_cr=None):
    """Particle-substeps/s of the streamed mode (aq_sim_create_streamed:
    records in pinned host memory, `parts` chunks through the device per
    pass) for the quantized record (from the quantized run's current
    state), the FP32-state record and, when given, the compression-rate-0.5
    scheme's record (both from the scene's initial values), timed with CUDA
    events over `steps` substeps after two untimed ones."""
    import torch

    from autoquantizer_b200.mpm_solver import MPMSolver
    from autoquantizer_b200.streamed import StreamedSolver

    out = {"mode": "records in pinned host memory, %d chunks through the device per pass "
                   "(aq_sim_create_streamed); every pass uploads and downloads every record" % parts,
           "chunk": n // parts, "steps": steps}
    f = MPMSolver(cfg32)
    f.set_particles(vals)
    runs = [("quantized", q), ("fp32_state", f)]
    if cfg_cr is not None:
        c = MPMSolver(cfg_cr)
        c.set_particles(vals)
        runs.append(("cr_half_scheme", c))
    for name, sol in runs:
        st = StreamedSolver(sol, chunk=n // parts)
        st.substeps(2)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st.substeps(steps)
        e1.record()
        torch.cuda.synchronize()
        v, ms_ = job_rate(n * steps, e0.elapsed_time(e1), ws)
        rb = sol.bytes_per_particle()
        out[name] = {"value": v, "unit": UNIT, "ms_per_step": ms_ / steps, "record_bytes": rb,
                     "host_bytes_per_substep": 2 * rb * n,
                     "host_link_gbs": 2 * rb * n / (ms_ / steps * 1e-3) / 1e9,  # both directions together
                     "status_flags": st.status()[0]}
        st.close()
    del f
    out["quantized_speedup"] = out["quantized"]["value"] / out["fp32_state"]["value"]
    if cfg_cr is not None:
        out["cr_half_speedup"] = out["cr_half_scheme"]["value"] / out["fp32_state"]["value"]
    return out


def cr_half_run(args, rank, vals, ref, loss64, total, K, W, ws):
    """The same scene on a scheme the analytical solver derives at compression
    rate 0.5 (LagrangianCR, the drivers' solve() recipe: position ranges 1,
    other ranges doubled, one sign bit added), all fields fixed point, so
    that the record with its 2-bit material id fits 6 words (48 B): 2x
    compression against the 96 B of FP32 values.
    Sensitivities: the hand-written adjoint (64 substeps, checkpoints every
    16, loss compute_ek) on a single-material stand-in of the scene, since
    the adjoint runs the reference's material laws only: the same particles,
    all elastic with the reference's 3D law at the geometric-mean E and mean
    nu of the scene's two elastic boxes.  Ranges: the FP32-state run's range
    detection over the same substeps.  Returns its throughput, compression
    and errors against the FP64 run, with the scheme's config (None if no rate fits)."""
    import torch

    from autoquantizer_b200 import _lib, scenes
    from autoquantizer_b200.adjoint import Adjoint, ek_seed
    from autoquantizer_b200.mpm_solver import MPMSolver
    from autoquantizer_b200.solvers import scheme_from_sensitivities

    cfg, _ = scenes.mixed_boxes_3d(seed=rank, quantized=False)
    el = [m for m in cfg.materials if m[0] != _lib.AQ_MAT_FLUID]
    stand = scenes.mixed_boxes_3d(seed=rank, n=4, quantized=False)[0]
    stand.materials = None
    stand.use_fluid = False
    stand.E = float(np.exp(np.mean([np.log(m[1]) for m in el])))
    stand.nu = float(np.mean([m[2] for m in el]))
    stand.n_particles = vals.shape[0]
    s = MPMSolver(stand)
    s.set_particles(vals[:, :24])
    adj = Adjoint(s._params())
    s0 = torch.from_numpy(np.ascontiguousarray(vals[:, :24])).to("cuda", torch.float32)
    t0 = time.perf_counter()
    sT = adj.forward(s0, 64, 16)
    _, sens = adj.backward(ek_seed(sT, 3, s.p_mass, s.g))
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t0
    adj.close()
    del sT, s0
    # ranges: FP32 state with range detection over the same substeps
    r = MPMSolver(cfg)
    r.set_particles(vals)
    limits = r.run_forward_detect_ranges(total)
    del r
    budget = 6 * 64 - 2  # six words minus the material id
    sens = np.maximum(np.asarray(sens, dtype=np.float64), 1e-30 * float(np.max(sens)))
    raw, _ = scheme_from_sensitivities(sens, limits[:24], 3, mode="CR", eps=0.5)
    chosen = None
    for k in range(81):
        # widths outside what a fixed-point slot holds are clamped (a slot
        # needs its sign bit and one more; 32 bits is the codec's maximum),
        # the rate lowered until the clamped widths fit six words
        rate = 0.5 - 0.0025 * k
        bits, ranges = scheme_from_sensitivities(sens, limits[:24], 3, mode="CR", eps=rate)
        bits = np.clip(bits, 2, 32)
        if int(np.sum(bits)) <= budget:
            chosen = (rate, bits, ranges)
            break
    if chosen is None:
        return {"error": "no rate in [0.3, 0.5] fits six words", "bits_at_0.5": [int(b) for b in raw]}, None
    rate, bits, ranges = chosen
    cq, _ = scenes.mixed_boxes_3d(seed=rank)
    cq.quant_bits = np.asarray(bits)
    cq.quant_ranges = np.asarray(ranges)
    cq.v_exp_bits = 0
    sq = MPMSolver(cq)
    sq.set_particles(vals)
    S = sq.bytes_per_particle()
    sq.substeps(W)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sq.substeps(K)
    e1.record()
    torch.cuda.synchronize()
    value, ms = job_rate(vals.shape[0] * K, e0.elapsed_time(e1), ws)
    sq.substeps(total - W - K)
    fe = field_errors(sq.state_tensor(True), ref)
    loss = sq.compute_loss()
    rel = abs(loss - loss64) / abs(loss64)
    flags, _ = sq.status()
    return {"value": value, "unit": UNIT, "ms_per_step": ms / K, "rate": rate, "bits": [int(b) for b in bits],
            "solver_bits_at_0.5_unclamped": [int(b) for b in raw], "sensitivities_sum_sq": [float(x) for x in sens],
            "record_bits": sq.layout().total_bits, "bytes_per_particle": S, "compression": 96.0 / S,
            "fields": fe, "x_rms": fe["x"]["rms"], "loss_rel_err": rel,
            "within_bound": bool(fe["x"]["rms"] <= args.x_bound and rel <= 3 * args.loss_eps),
            "status_flags": flags, "adjoint_s": t_adj,
            "sensitivities": "adjoint on a single-material stand-in (reference 3D elastic law, E %.4g, nu %.3f)"
                             % (stand.E, stand.nu)}, cq


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frame", type=int, default=100)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-cr", action="store_true", help="skip the compression-rate-0.5 scheme run")
    ap.add_argument("--reference-budget-s", type=float, default=90.0,
                    help="--impl reference: the whole scene if warm-up + timed substeps fit this many seconds")
    ap.add_argument("--stream-steps", type=int, default=16,
                    help="substeps timed in the streamed (out-of-core) mode; 0 skips it")
    ap.add_argument("--stream-parts", type=int, default=4, help="chunks per pass in the streamed mode")
    ap.add_argument("--x-bound", type=float, default=1e-4, help="requested position RMS error bound")
    ap.add_argument("--loss-eps", type=float, default=1e-3, help="eps of the |loss - loss_f64| < 3 eps test")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
