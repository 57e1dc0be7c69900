#!/usr/bin/env python
"""Throughput of the WannierNLQG k-mesh response hot path on B200s, in k-points/s.

Workload (one GPU): the nw=32 synthetic orthogonal Wannier model (|R_i| <= 4, 729 R-vectors,
full off-diagonal position operator, seed 0) evaluated on its 256^3 Gamma-centred mesh:
Berry curvature Omega^z (occupied sum), quantum metric g^xx (band sum) and the shift current
sigma^xyy(omega) on 512 photon energies in [0, 4] eV with Lorentzian eta = 0.01 eV, mu = 0, T = 0.
A step is one contiguous block of `--batch` mesh points pushed through the whole path
(phases -> Fourier -> eigensolve -> integrands -> deterministic reduction).  With N ranks each rank
takes its own blocks (weak scaling, no data-path collective); the lane tensors are combined
once at the end with one NCCL all-reduce outside the timed region.

`--sampling random` replaces the mesh blocks by seeded uniformly random k-points (the nodes of an
adaptive integrator), evaluated through the weighted-points entry point: there the Fourier step
is the tcgen05 tensor-core GEMM instead of the staged mesh contraction.

`--impl reference` times the reference algorithm's CPU restatement (the FP64 oracle, all host
threads) on a bounded sample of the same mesh.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from wanniernlqg_b200 import _abi  # noqa: E402
from wanniernlqg_b200.model import reference_workload_model  # noqa: E402

METRIC = "k-points/s"
WORKLOAD = "nw32_R729_fullA_mesh256^3_sigma_xyy_512w_OmegaZ_gxx"
WORKLOAD_RANDOM = "nw32_R729_fullA_random_k_sigma_xyy_512w_OmegaZ_gxx"
MESH = (256, 256, 256)


def make_task(precision: int) -> _abi.TaskArrays:
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"]),
                            (_abi.QUANTUM_METRIC, ["xx"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.01,
                           photon_energies=np.linspace(0.0, 4.0, 512), fermi_energy=0.0, temperature=0.0,
                           precision=precision)


def mesh_kpoints(start: int, count: int) -> np.ndarray:
    idx = np.arange(start, start + count, dtype=np.int64)
    n1, n2, n3 = MESH
    return np.stack([(idx % n1) / n1, ((idx // n1) % n2) / n2, (idx // (n1 * n2)) / n3], axis=1)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

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
        if self.thread:
            self.thread.join(timeout=2)
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
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            p = json.load(fh)
        return p, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def cpu_baseline_run(model, task, target_seconds: float, threads: int):
    """Time the FP64 oracle on a bounded sample of the workload mesh (contiguous points from the
    start of a lane)."""
    from oracle import oracle
    oracle.build()
    probe = max(4, threads)
    start = 1_000_003
    t0 = time.perf_counter()
    oracle.integrate_mesh(model, task, MESH, start, start + probe, threads=threads)
    per_point = (time.perf_counter() - t0) / probe
    n = int(max(probe, min(200_000, target_seconds / max(per_point, 1e-9))))
    t0 = time.perf_counter()
    oracle.integrate_mesh(model, task, MESH, start, start + n, threads=threads)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    model = reference_workload_model("nw32")
    task = make_task(_abi.PRECISION_FP64)
    threads = os.cpu_count() or 1
    from oracle import oracle
    oracle.build()
    # Calibrate a step of about 4 s of CPU work.
    probe = max(4, threads)
    t0 = time.perf_counter()
    oracle.integrate_mesh(model, task, MESH, 0, probe, threads=threads)
    per_point = (time.perf_counter() - t0) / probe
    n = int(max(probe, min(200_000, 4.0 / max(per_point, 1e-9))))
    for w in range(args.warmup):
        oracle.integrate_mesh(model, task, MESH, w * n, (w + 1) * n, threads=threads)
    t0 = time.perf_counter()
    for s in range(args.steps):
        b = (args.warmup + s) * n
        oracle.integrate_mesh(model, task, MESH, b, b + n, threads=threads)
    dt = time.perf_counter() - t0
    value = n * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded model; no dataset)",
        "config": {"workload": WORKLOAD, "k_per_step_per_gpu": n, "mesh": list(MESH)},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{n} contiguous mesh points per step, oracle FP64 with {threads} OpenMP threads"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--batch", type=int, default=65536, help="mesh points per step and rank")
    ap.add_argument("--sampling", default="mesh", choices=["mesh", "random"],
                    help="mesh blocks (staged Fourier) or random k-points (tensor-core Fourier)")
    ap.add_argument("--max-batch", type=int, default=0,
                    help="plan batch capacity (0: one step, --batch points; a 65536-point nw=32 step holds ~11 GB)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched uneven-models measurement (one GPU only)")
    ap.add_argument("--no-time-to-tolerance", action="store_true",
                    help="skip the time-to-1e-4 convergence study of sigma^xyy (one GPU only)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in eigensolver team and contraction tile rules")
    ap.add_argument("--adaptive-study", action="store_true",
                    help="add the learned adaptive refinement study (one GPU; a few minutes)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from wanniernlqg_b200 import build
    from wanniernlqg_b200.engine import ResponseEngine
    build.build()
    precision = _abi.PRECISION_FP64 if args.precision == "fp64" else _abi.PRECISION_MIXED
    model = reference_workload_model("nw32")
    task = make_task(precision)
    nk = int(np.prod(MESH))
    batch = args.batch
    engine = ResponseEngine(model, task, device=local_rank, max_batch=args.max_batch or batch)
    vc = engine.value_count
    out = torch.zeros(2 * vc, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def block(step):
        b = ((step * world + rank) * batch) % nk
        return b, min(nk, b + batch)

    # The autotuner picks the eigensolver team and the contraction tile on the first step's block
    # (untimed; every rank tunes its own plan).
    tuning = None if args.no_autotune else engine.autotune(MESH, *block(0))

    random_mode = args.sampling == "random"
    if random_mode:
        gen = torch.Generator(device="cuda")
        gen.manual_seed(1234 + rank)
        kdev = torch.rand((args.warmup + args.steps) * batch, 3, dtype=torch.float64, device="cuda", generator=gen)
        wdev = torch.full((batch,), 1.0 / (world * batch), dtype=torch.float64, device="cuda")

    def run_step(step):
        if random_mode:
            engine.weighted_sum_device(kdev.data_ptr() + step * batch * 3 * 8, wdev.data_ptr(), batch,
                                       out.data_ptr(), stream.cuda_stream)
        else:
            kb, ke = block(step)
            engine.integrate_mesh_device(MESH, kb, ke, out.data_ptr(), stream.cuda_stream)

    for s in range(args.warmup):
        run_step(s)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.4)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    launches = 0
    for s in range(args.steps):
        run_step(args.warmup + s)
        launches += engine.last_launch_count()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    fourier_ms, eigen_ms, response_ms, total_ms = engine.last_timing()
    if dist:
        t = torch.tensor([elapsed_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
        dist.barrier()
    value = world * batch * args.steps / (elapsed_ms / 1e3)
    # The data path's one exchange, outside the timed region: the ranks' lane tensors (here each
    # rank's last block sum, value_count complex values) combined by one NCCL all-reduce, then read
    # back on rank 0; every rank's block is different, so the combined sum checks the exchange.
    combined = out.clone()
    if dist:
        dist.all_reduce(combined)
    lane_sum = combined.cpu().numpy().view(np.complex128)

    # End to end through the public host API: the step's mesh indices and weights in pinned
    # host memory (H2D), the weighted mesh sum, and the result read back (D2H); synchronous,
    # wall clock.
    e2e_steps = max(1, min(args.steps, 3))
    if random_mode:
        # Host k-points and weights (pinned), the weighted-points call, the result read back.
        idx = kdev[:batch].cpu().pin_memory().numpy()
        w = torch.full((batch,), 1.0 / batch, dtype=torch.float64).pin_memory().numpy()
        e2e_call = lambda: engine.weighted_sum(idx, w)  # noqa: E731
    else:
        kb, _ = block(args.warmup + args.steps)
        idx = torch.arange(kb, kb + batch, dtype=torch.int64).pin_memory().numpy()
        w = torch.full((batch,), 1.0 / nk, dtype=torch.float64).pin_memory().numpy()
        e2e_call = lambda: engine.mesh_weighted_sum(MESH, idx, w)  # noqa: E731
    e2e_call()
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        e2e_call()
    e2e_dt = (time.perf_counter() - t0) / e2e_steps
    e2e_value = world * batch / e2e_dt

    # Roofline of the dominant stage, from the last step's CUDA events on the plan stream.
    peaks, peak_src = load_peaks()
    stages = {"fourier": fourier_ms, "eigen": eigen_ms, "response": response_ms}
    # The roofline describes the dominant kernel: the Fourier and response stages are one kernel
    # each on the measured paths, the eigensolve stage two (an FP32 Jacobi and an FP64 refinement
    # kernel, about 40 / 60 % of the stage in the launch lists), so it is compared at its larger
    # kernel's share.
    kernel_ms = {"fourier": fourier_ms, "eigen": 0.6 * eigen_ms, "response": response_ms}
    dominant = max(kernel_ms, key=kernel_ms.get)
    nw, nr = model.num_orbitals, model.num_r_vectors
    C = fourier_channels(task)
    # Algorithmic work per k-point (counts of the algorithms executed):
    #   staged Fourier (mesh): 8*P1*C*nw^2 flop (P1 = 9 distinct r1 on the |R_i|<=4 cube) and
    #     C*nw^2*16 B written (the FP64 Wannier-gauge channels) plus the line stage's reads,
    #     P1*C*nw^2*16 B per line of n1 = 256 points (the channels' later read belongs to the
    #     response kernel);
    #   tensor-core Fourier (random): S(S+1)/2 int8 slice products of 2*Kpad*Npad ops each
    #     (Kpad = 2*NR rounded up to 64, Npad = 2*C*nw^2 rounded up to the tile width);
    #   eigensolve: 30*nw^3 flop (LAPACK-class modelling count for a Hermitian eigensolve);
    #   response: 18 complex nw^3 products (8*nw^3 flop each) + 4*nw^2*Nw flop contraction.
    p1 = 9
    flop = {"fourier": 8.0 * p1 * C * nw * nw, "eigen": 30.0 * nw ** 3,
            "response": 18 * 8.0 * nw ** 3 + 4.0 * nw * nw * 512}
    hbm = {"fourier": C * nw * nw * 16 * (1.0 + p1 / MESH[0]), "eigen": nw * nw * 16 * 2.0 + nw * 8,
           "response": (C - 1) * nw * nw * 16 + nw * nw * 16}
    # SM-bound stages: measured on this device after the timed region (FP64 DMMA, FP64 FMA, FP32 FMA
    # probes of wnlqg_b200_measure_peaks); the nominal figures only if the probe fails.
    try:
        from wanniernlqg_b200 import _lib
        sm_measured = _lib.measure_peaks(torch.cuda.current_device())
    except Exception:   # noqa: BLE001 - the roofline then names its nominal source
        sm_measured = None
    if sm_measured is not None and precision == _abi.PRECISION_FP64:
        sm_peak = max(sm_measured["fp64_dmma_tflops"], sm_measured["fp64_fma_tflops"])
        sm_src = ("measured in this run: FP64 DMMA %.1f, FP64 FMA %.1f TFLOP/s (the larger)"
                  % (sm_measured["fp64_dmma_tflops"], sm_measured["fp64_fma_tflops"]))
    elif sm_measured is not None:
        sm_peak = sm_measured["fp32_fma_tflops"]
        sm_src = "measured in this run: FP32 FMA %.1f TFLOP/s" % sm_measured["fp32_fma_tflops"]
    else:
        sm_peak = {"fp64": 37.0, "mixed": 74.0}["fp64" if precision == _abi.PRECISION_FP64 else "mixed"]
        sm_src = "nominal B200 CUDA-core peak (FP64 37 / FP32 74 TFLOP/s; the probe failed)"
    slices = 7 if precision == _abi.PRECISION_FP64 else 4
    tile_n = 64 if slices == 7 else 128
    kpad = -(-2 * nr // 64) * 64
    npad = -(-2 * C * nw * nw // tile_n) * tile_n
    tc_ops = slices * (slices + 1) / 2 * 2.0 * kpad * npad

    def stage_roofline(name):
        t_s = stages[name] / 1e3
        if name == "fourier" and random_mode:
            achieved = tc_ops * batch / t_s / 1e12
            return {"bound": "tensor", "kernel": "tcgen05 int8 slice GEMM (tc_fourier_kernel)",
                    "achieved": achieved, "unit": "TOP/s", "peak": 2.0 * peaks["bf16_tflops"],
                    "peak_source": f"2 x {peak_src} dense bf16 (the dense int8 rate is twice bf16)",
                    "fp64_equivalent_tflops": 8.0 * nr * C * nw * nw * batch / t_s / 1e12}
        if name == "fourier":
            return {"bound": "hbm", "kernel": "staged Fourier (staged_r1_kernel)",
                    "achieved": hbm[name] * batch / t_s / 1e9, "unit": "GB/s", "peak": peaks["hbm_gbs"],
                    "peak_source": f"{peak_src} HBM copy bandwidth"}
        return {"bound": "sm", "kernel": {"eigen": "Jacobi eigensolver", "response": "fused response kernel"}[name],
                "achieved": flop[name] * batch / t_s / 1e12, "unit": "TFLOP/s", "peak": sm_peak, "peak_source": sm_src,
                "hbm_gbs": hbm[name] * batch / t_s / 1e9}

    # DRAM bytes per k-point (read + write) of each stage's kernel, from ncu captures of
    # 8192-point launches of the same kernels, scaled to the step's batch: the kernels
    # stream their inputs point by point, so traffic grows in proportion to the points.
    # The eigensolve stage is two kernels (FP32 Jacobi, FP64 refinement): their bytes are summed.
    traffic_per_k = {
        ("fp64", "response"): (1.079503e9 + 4.992e6) / 8192,
        ("fp64", "eigen"): (0.135450e9 + 35.735e6 + 0.201901e9 + 97.160e6) / 8192,
        ("fp64", "fourier"): (37.772e6 + 1.014368e9) / 8192,
        ("mixed", "fourier"): (37.772e6 + 1.014368e9) / 8192,
        ("mixed", "response"): (1.082281e9 + 9.649408e6) / 8192,
        ("mixed", "eigen"): (0.134329e9 + 35.740160e6 + 0.201393e9 + 98.023680e6) / 8192,
        ("mixed", "fourier_random"): (436.281088e6 + 1.025739e9) / 8192,
    }
    prec_key = "fp64" if precision == _abi.PRECISION_FP64 else "mixed"
    per_stage = {}
    for name in stages:
        r = stage_roofline(name)
        r["frac"] = r["achieved"] / r["peak"] if r["peak"] else None
        r["ms_last_step"] = stages[name]
        key = (prec_key, "fourier_random" if (name == "fourier" and random_mode) else name)
        r["traffic"] = traffic_per_k[key] * batch if key in traffic_per_k else None
        per_stage[name] = r
    roofline = dict(per_stage[dominant])
    roofline.update({
        "stage_ms_last_step": {"fourier": fourier_ms, "eigen": eigen_ms, "response": response_ms, "total": total_ms},
        "stages": per_stage,
        "algorithmic_per_k": {"flop": flop, "hbm_bytes": hbm, "tensor_int8_ops": tc_ops if random_mode else None},
        "launches_per_step": launches // max(1, args.steps),
        "sm_peaks_measured_tflops": sm_measured,
    })
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if precision == _abi.PRECISION_FP64 else "f32+f64",
        "data": ("synthetic (seeded nw=32 model, seeded random k-points; no dataset)" if random_mode else
                 "synthetic (seeded nw=32 model, 256^3 mesh blocks; no dataset)"),
        "config": {"workload": WORKLOAD_RANDOM if random_mode else WORKLOAD, "k_per_step_per_gpu": batch,
                   "mesh": None if random_mode else list(MESH), "sampling": args.sampling,
                   "precision": args.precision, "l2": "inputs larger than L2 (per-step workspace >> 126 MB)",
                   "parallelism": f"k-blocks x{world}",
                   "autotune": tuning},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": int(idx.nbytes + w.nbytes),
                "d2h_bytes_per_step": int(16 * vc)},
        "clocks": clocks,
        "gpu_launches": launches,
        "lane_exchange": {"ranks": world, "collective": "all_reduce (NCCL)" if dist else "none (one rank)",
                          "values": int(vc), "max_abs": float(np.max(np.abs(lane_sum)))},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, n, dt = cpu_baseline_run(model, make_task(_abi.PRECISION_FP64), args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                                "sample": f"{n} contiguous mesh points, FP64 oracle, {threads} OpenMP threads, {dt:.1f} s"}
    engine.close()
    if rank == 0 and world == 1 and not args.no_time_to_tolerance:
        line["time_to_tolerance"] = time_to_tolerance(model, local_rank)
    if rank == 0 and world == 1 and args.adaptive_study:
        line["learned_adaptive"] = learned_time_to_tolerance(local_rank)
    if rank == 0 and world == 1 and not args.no_batched:
        line["batched_uneven"] = batched_uneven(local_rank)
        line["graph_small_calls"] = graph_small_calls(local_rank)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def time_to_tolerance(model, device: int, rtol: float = 1e-4, blocks: int = 4, block: int = 65536,
                      repeats: int = 3) -> dict:
    """Mixed path against the plain FP64 path on the workload mesh: the same `blocks` blocks of
    `block` consecutive 256^3 mesh points (spread over the mesh) through both, and the largest
    relative error of the mixed sigma^xyy(omega) block sums (max norm over the 512 energies)
    against the FP64 ones.  Each path first runs one full-size block untimed (so every lazily
    sized workspace exists), then the blocks `repeats` times; times are the plan's CUDA events
    (whole call and per stage), the median over the repeats.  The speed-up at the stated accuracy
    is the time ratio; the full-mesh times follow by scaling."""
    from wanniernlqg_b200.engine import ResponseEngine

    nk = int(np.prod(MESH))
    starts = [(i * nk) // blocks for i in range(blocks)]
    res = {}
    for name, prec in (("fp64", _abi.PRECISION_FP64), ("mixed", _abi.PRECISION_MIXED)):
        with ResponseEngine(model, make_task(prec), device=device, max_batch=block) as eng:
            eng.autotune(MESH, starts[0], starts[0] + block)
            eng.integrate_mesh(MESH, starts[-1], starts[-1] + block)
            totals, stage_sums = [], []
            vals = []
            for rep_i in range(repeats):
                tot, st = 0.0, np.zeros(3)
                for s0 in starts:
                    v = eng.integrate_mesh(MESH, s0, s0 + block)[:512]
                    if rep_i == 0:
                        vals.append(v)
                    f, e, r, t = eng.last_timing()
                    tot += t
                    st += (f, e, r)
                totals.append(tot)
                stage_sums.append(st)
            order = int(np.argsort(totals)[len(totals) // 2])
        res[name] = (vals, totals[order] / 1e3, stage_sums[order], totals)
    err = max(float(np.max(np.abs(m - f)) / np.max(np.abs(f))) for m, f in zip(res["mixed"][0], res["fp64"][0]))
    t64, tmx = res["fp64"][1], res["mixed"][1]
    scale = nk / (blocks * block)
    return {"quantity": "sigma^xyy(omega), 512 energies", "mesh": list(MESH),
            "sample": f"{blocks} blocks of {block} consecutive mesh points, median of {repeats} repeats (CUDA events)",
            "rtol": rtol, "mixed_vs_fp64_max_rel_error": err, "within_rtol": err <= rtol,
            "fp64_seconds_full_mesh": t64 * scale, "mixed_seconds_full_mesh": tmx * scale,
            "fp64_stage_ms_per_block": {k: float(v) / blocks for k, v in zip(("fourier", "eigen", "response"),
                                                                             res["fp64"][2])},
            "mixed_stage_ms_per_block": {k: float(v) / blocks for k, v in zip(("fourier", "eigen", "response"),
                                                                              res["mixed"][2])},
            "repeat_seconds": {"fp64": res["fp64"][3], "mixed": res["mixed"][3]},
            "speedup_mixed_vs_fp64": t64 / tmx}


def adaptive_study(model, make_task_fn, device: int, *, omegas, support, n0: int, rtol: float, max_level: int,
                   max_leaves: int = 1_500_000, max_evaluations: int = 30_000_000, seed: int = 3) -> dict:
    """Time to tolerance of one response with the cell-adaptive integrator: the plain FP64 path
    (every leaf checked, FP64 kernels) against the mixed + batched + learned path (mixed-precision
    kernels, each round's uneven cells in one batched device call, the GPU-trained MLP choosing
    which leaves to check, with the support guard).  Both run to `rtol` or to the leaf / evaluation
    budget; times are wall clock of the whole adaptive run (device calls, host bookkeeping, feature
    spectra and network training).  The plain run's value judges the learned run's."""
    from wanniernlqg_b200.adaptive import MlpProposer, integrate_cells
    from wanniernlqg_b200.engine import ResponseEngine

    warm = np.random.default_rng(0).random((4096, 3))
    kw = dict(n0=n0, rtol=rtol, max_level=max_level, max_leaves=max_leaves, max_evaluations=max_evaluations)
    with ResponseEngine(model, make_task_fn(_abi.PRECISION_FP64), device=device) as eng:
        eng.point_values(warm)
        plain = integrate_cells(eng.point_values, **kw)
    with ResponseEngine(model, make_task_fn(_abi.PRECISION_MIXED), device=device) as eng:
        eng.point_values(warm)
        eng.spectrum(warm, vectors=False)
        prop = MlpProposer(0.0, omegas, lambda k: eng.spectrum(k, vectors=False), device=device, seed=seed,
                           lattice=model.lattice, support=support)
        try:
            learned = integrate_cells(eng.point_values, proposer=prop, seed=seed, **kw)
            spectra = prop.spectrum_evaluations
        finally:
            prop.close()

    def summary(r):
        scale = float(np.max(np.abs(r.value)))
        return {"seconds": r.seconds, "evaluations": int(r.evaluations), "leaves": int(r.leaves),
                "checked_cells": int(r.checked_cells), "rounds": int(r.rounds), "converged": bool(r.converged),
                "error_estimate_rel": float(r.error_estimate / scale) if scale > 0 else None}

    out = {"n0": n0, "max_level": max_level, "rtol": rtol, "max_leaves": max_leaves,
           "plain_fp64": summary(plain), "mixed_batched_learned": summary(learned)}
    out["mixed_batched_learned"].update({"fallback_rounds": int(learned.fallbacks), "feature_spectra": int(spectra),
                                         "value_vs_plain_rel": float(np.max(np.abs(learned.value - plain.value)) /
                                                                     np.max(np.abs(plain.value)))})
    out["speedup"] = plain.seconds / learned.seconds
    return out


def learned_time_to_tolerance(device: int) -> dict:
    """The learned adaptive refinement workload at its stated parameters and the nw = 32 shift
    current on a low photon window (both opt-in: `--adaptive-study`).

    * Band-crossing model: nw = 16 (|R_i| <= 2) with its onsite energies shifted so that a Weyl
      crossing of bands 8/9 sits at mu = 0; injection current eta^xyz and eta^xyy at 20 photon
      energies in [0.005, 0.1] eV, width 0.005 eV with the reference's default (Gaussian)
      broadening, T = 0; cells from 48^3, up to 8 levels, rtol 1e-4.
    * nw = 32 workload model: sigma^xyy at 32 photon energies in [0.01, 0.25] eV, Gaussian 0.01 eV,
      mu = 0; cells from 24^3, up to 6 levels, rtol 1e-4."""
    from wanniernlqg_b200.model import crossing_model

    res = {}
    om4 = np.linspace(0.005, 0.1, 20)
    eta4 = 0.005
    crossing = crossing_model(16, 2, 0)
    for comp in ("xyz", "xyy"):
        res[f"injection_{comp}_nw16_crossing"] = adaptive_study(
            crossing, lambda prec, comp=comp: _abi.TaskArrays(
                [(_abi.INJECTION_CURRENT, [comp])], broadening_type=_abi.GAUSSIAN, broadening=eta4,
                photon_energies=om4, fermi_energy=0.0, precision=prec),
            device, omegas=om4, support=(om4.min() - np.sqrt(200.0) * eta4, om4.max() + np.sqrt(200.0) * eta4),
            n0=48, rtol=1e-4, max_level=8)
    res["crossing"] = {"bands": [int(b) + 1 for b in crossing.crossing["bands"]], "gap_ev": crossing.crossing["gap_ev"]}
    om2 = np.linspace(0.01, 0.25, 32)
    res["shift_xyy_nw32_low_window"] = adaptive_study(
        reference_workload_model("nw32"),
        lambda prec: _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"])], broadening_type=_abi.GAUSSIAN, broadening=0.01,
                                     photon_energies=om2, fermi_energy=0.0, precision=prec),
        device, omegas=om2, support=(om2.min() - np.sqrt(200.0) * 0.01, om2.max() + np.sqrt(200.0) * 0.01),
        n0=24, rtol=1e-4, max_level=6)
    return res


def cfg3_models(seed: int = 2024):
    """The batched uneven workload's 24 seeded models: orbital counts drawn from {6, 8, 12, 16,
    24, 32, 48, 64, 96}, R cubes |R_i| <= 2, 3 or 4, every second model Kramers-doubled (a model
    of half the drawn count, doubled as H (x) I_2 + i 1e-3 eV M (x) sigma_z), each with its own mesh
    from {64, 96, 128, 160, 192}^3."""
    from wanniernlqg_b200.model import kramers_doubled_model, synthetic_orthogonal_model
    rng = np.random.default_rng(seed)
    choices = [6, 8, 12, 16, 24, 32, 48, 64, 96]
    out = []
    for i in range(24):
        nw = int(rng.choice(choices))
        cube = int(rng.integers(2, 5))
        mesh = int(rng.choice([64, 96, 128, 160, 192]))
        doubled = i % 2 == 1
        base = synthetic_orthogonal_model(nw // 2 if doubled else nw, cube, seed=300 + i, full_position=True)
        model = kramers_doubled_model(base, 1e-3, seed=i) if doubled else base
        out.append((model, (mesh, mesh, mesh), doubled, cube))
    return out


def batched_uneven(device: int, points_per_model: int = 65536) -> dict:
    """The batched uneven workload: the 24 models of cfg3_models, the Berry-curvature channel of
    the linear transport conductivity sigma^xy (the reference's finite-temperature Hall response;
    its intrinsic AHC is zero-temperature only) and the Berry-curvature dipole D^xz (Omega^xy with
    the x velocity, component xyx) at mu in {-0.5, 0, 0.5} eV and T = 50 K.  The dipole threshold
    is 1e-12 eV, so that the Kramers splittings (1e-3 eV typically, 6e-10 eV at the closest sampled
    point) count as isolated (the reference's 2e-3 eV default refuses those models).  Every plan is autotuned on its own first block (choices cached
    per orbital count); each model then sums the first `points_per_model` points of its own mesh
    (a lane range).  Timed with CUDA events on the caller's stream: one concurrent
    wnlqg_b200_eval_mesh_many call, the models one call after another, and the concurrent call
    captured once as a CUDA graph and replayed."""
    import torch
    from wanniernlqg_b200.engine import CapturedGraph, ResponseEngine, integrate_meshes_many

    task = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy"]), (_abi.BERRY_DIPOLE, ["xyx"])],
                           fermi_energies=[-0.5, 0.0, 0.5], temperature=50.0, degeneracy_threshold=1e-12)
    spec = cfg3_models()
    engines = []
    try:
        tuning = {}
        for model, mesh, _, _ in spec:
            # Small models hold one whole sample per batch; large ones take the library's ~4 GiB
            # batch workspace (a 65536-point batch at 96 orbitals would need ~70 GB).
            eng = ResponseEngine(model, task, device=device,
                                 max_batch=points_per_model if model.num_orbitals <= 48 else 0)
            engines.append(eng)
            rep = eng.autotune(mesh, 0, min(points_per_model, 16384))
            tuning.setdefault(model.num_orbitals, {"eigh_team": rep["eigh_team"], "eigh_grid": rep["eigh_grid"],
                                                   "response_grid": rep["response_grid"],
                                                   "warm_start": rep["warm_start"]})
        outs = [torch.zeros(2 * e.value_count, dtype=torch.float64, device="cuda") for e in engines]
        meshes = [m for _, m, _, _ in spec]
        ranges = [(0, min(points_per_model, int(np.prod(m)))) for m in meshes]
        stream = torch.cuda.current_stream()
        ptrs = [o.data_ptr() for o in outs]

        def concurrent():
            integrate_meshes_many(engines, meshes, ranges, ptrs, stream.cuda_stream)

        def sequential():
            for e, m, r, o in zip(engines, meshes, ranges, outs):
                e.integrate_mesh_device(m, r[0], r[1], o.data_ptr(), stream.cuda_stream)
                torch.cuda.synchronize()

        def timed(fn):
            fn()
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            fn()
            ev1.record(stream)
            torch.cuda.synchronize()
            return ev0.elapsed_time(ev1)

        t_conc = timed(concurrent)
        for e in engines:
            e.status()
        t_seq = timed(sequential)
        graph = CapturedGraph.mesh_many(engines, meshes, ranges, ptrs)
        try:
            t_graph = timed(lambda: graph.launch(stream.cuda_stream))
            graph.status()
            graph_kernels = graph.kernel_count
        finally:
            graph.close()
    finally:
        for e in engines:
            e.close()
    total = sum(r[1] - r[0] for r in ranges)
    return {"models": len(spec), "orbitals": [m.num_orbitals for m, _, _, _ in spec],
            "kramers_doubled": [bool(d) for _, _, d, _ in spec], "r_cube": [c for _, _, _, c in spec],
            "meshes": [m[0] for m in meshes], "points_per_model": points_per_model,
            "responses": "linear transport Berry channel xy + Berry dipole xyx (D^xz) at 3 Fermi energies, T = 50 K",
            "autotune_per_orbitals": {str(k): v for k, v in sorted(tuning.items())},
            "concurrent_ms": t_conc, "sequential_ms": t_seq, "speedup": t_seq / t_conc,
            "graph_ms": t_graph, "graph_kernels": graph_kernels, "kpoints_per_s_graph": total / (t_graph / 1e3),
            "kpoints_per_s": total / (t_conc / 1e3)}


def graph_small_calls(device: int, n: int = 512, calls: int = 100) -> dict:
    """Launch-bound calls, as an adaptive controller makes them: weighted sums over n arbitrary
    k-points of the 4-orbital workload model (shift + injection current xyy at 128 energies), the
    points and weights already on the device, enqueued back to back on one stream and timed with
    CUDA events per call: the direct call against the same call captured once as a CUDA graph."""
    import torch
    from wanniernlqg_b200.engine import CapturedGraph, ResponseEngine

    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["xyy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02,
                           photon_energies=np.linspace(0, 3, 128))
    with ResponseEngine(reference_workload_model("nw4"), task, device=device, max_batch=n) as eng:
        gen = torch.Generator(device="cuda")
        gen.manual_seed(77)
        k = torch.rand((n, 3), dtype=torch.float64, device="cuda", generator=gen)
        w = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
        out = torch.zeros(2 * eng.value_count, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()

        def per_call(fn):
            for _ in range(5):
                fn()
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(calls):
                fn()
            ev1.record(stream)
            torch.cuda.synchronize()
            return ev0.elapsed_time(ev1) / calls

        t_direct = per_call(lambda: eng.weighted_sum_device(k.data_ptr(), w.data_ptr(), n, out.data_ptr(),
                                                            stream.cuda_stream))
        ref = out.clone()
        with CapturedGraph.points_weighted(eng, k.data_ptr(), w.data_ptr(), n, out.data_ptr()) as graph:
            t_graph = per_call(lambda: graph.launch(stream.cuda_stream))
            kernels = graph.kernel_count
        same = bool(torch.equal(ref, out))
    return {"orbitals": 4, "points_per_call": n, "calls": calls, "kernels_per_call": kernels,
            "direct_ms_per_call": t_direct, "graph_ms_per_call": t_graph, "speedup": t_direct / t_graph,
            "bitwise_equal": same}


def fourier_channels(task) -> int:
    # H, dH_x, dH_y, A_x, A_y, dA[y][x], ddH_xy, dA[x][y]  for sigma^xyy + Omega^xy + g^xx.
    return 8


if __name__ == "__main__":
    sys.exit(main())
