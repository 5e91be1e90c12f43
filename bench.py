#!/usr/bin/env python
"""Benchmark of the static-geometry uniform dipole FMM on B200.

Workload (one GPU): N = 1,048,576 dipoles uniform in the unit cube (seeded),
targets = sources with self exclusion, moments = random unit direction x
U[0.5, 1.5], expansion order p = 6, depth 5 (32,768 leaves, ~32 per leaf),
field + potential, K = 64 moment states per step evaluated in one batched
call.  Metric: target x state evaluations per second (N * K / step time).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) every rank evaluates its own K states on the same
geometry (replicas, no data-path collective; weak scaling); the step time is
the max over ranks of the CUDA-event time.

Reported beside `value` (device-resident inputs):
  e2e           the same metric through the C ABI with pinned host buffers,
                H2D of moments and D2H of results inside the timed region;
  plain         the plain per-state FP32 path (K = 1 calls, FP32 SIMT M2L);
  rel_l2_*      accuracy of state 0 vs the FP64 direct sum on 16,384 targets;
  roofline      dominant kernel: algorithmic work / CUDA-event duration;
  near_field    the step with the FP32 SIMT near field (co-resident with
                the M2L) and with the tensor-core near field;
  cpu_baseline  the reference CpuStatic (oracle/_ref, built from the upstream
                sources) on the host cores, on a bounded sample;
  backward      reverse mode on the same workload: device time of the field
                forward and of the backward (dL/dmoments + dL/dtarget-positions);
  multi_geometry  48 clustered problems of uneven size (N log-uniform in
                [8192, 524288], p = 6, one state each) evaluated by one CUDA
                graph launch: total targets / launch time.
--impl reference times the reference CpuStatic path (FP32, field+potential)
on the host cores on that same bounded sample and prints the same line.
"""

from __future__ import annotations

import argparse
import datetime
import json
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "dip-fmm_b200", "python")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "target·state field evals/s at rel-L2≤1e-5 vs FP64: batched B200 vs plain path"
UNIT = "target-state evals/s"
REF_SAMPLE = dict(n=131072, order=6, depth=4)  # ~32 dipoles per leaf, like the full workload
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=1048576)
    ap.add_argument("--order", type=int, default=6)
    ap.add_argument("--depth", type=int, default=5)
    ap.add_argument("--states", type=int, default=64)
    ap.add_argument("--m2l", choices=["auto", "fp32", "bf16x3"], default="auto")
    ap.add_argument("--near", choices=["auto", "fp32", "tf32x3"], default="auto",
                    help="near-field arithmetic of the K-state evaluation (auto: tensor cores)")
    ap.add_argument("--seed", type=int, default=314159)
    ap.add_argument("--plain-states", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-backward", action="store_true")
    ap.add_argument("--no-multi", action="store_true")
    ap.add_argument("--no-lattice", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--nvtx", action="store_true",
                    help="mark the timed steps with the NVTX range 'timed_steps' (for ncu --nvtx-include)")
    ap.add_argument("--corun-shape-sweep", action="store_true",
                    help="time every M2L pipeline shape under the co-resident schedule")
    ap.add_argument("--multi-problems", type=int, default=48)
    return ap.parse_args()


def unit_moments(rng, k, n):
    d = rng.normal(size=(k, n, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    return (d * rng.uniform(0.5, 1.5, size=(k, n, 1))).astype(np.float32)


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except OSError:
        return dict(FALLBACK_PEAKS), "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled DURING the timed
    region: NVML read every 20 ms from a background thread (the timed region
    of a short run lasts only a few hundred ms), or `nvidia-smi -lms 100`
    when NVML is not importable.  Reads only; changes no GPU setting."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))

    def __init__(self, gpu_index, pci_bus_id=None):
        self.gpu = gpu_index
        self.pci = pci_bus_id
        self.proc = None
        self.file = None
        self.thread = None
        self.samples = []
        self.kind = None

    def _nvml_loop(self, nvml, handle, stop):
        while not stop.is_set():
            try:
                sm = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                reasons = nvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                self.samples.append((float(sm), int(reasons)))
            except Exception:  # noqa: BLE001 - a failed read is a missing sample
                pass
            stop.wait(0.02)

    def start(self):
        try:
            import threading

            import pynvml as nvml

            nvml.nvmlInit()
            handle = None
            if self.pci:
                try:
                    handle = nvml.nvmlDeviceGetHandleByPciBusId(self.pci)
                except Exception:  # noqa: BLE001
                    handle = None
            if handle is None:
                handle = nvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.smax = float(nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM))
            self.stop_event = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nvml, handle, self.stop_event), daemon=True)
            self.kind = "nvml, 20 ms"
            self.thread.start()
            return
        except Exception:  # noqa: BLE001 - fall back to nvidia-smi
            self.thread = None
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
            self.kind = "nvidia-smi, 100 ms"
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_event.set()
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = {name for name, bit in self.REASON_BITS for _, r in self.samples if r & bit}
            return {"sm_mhz": statistics.median(s for s, _ in self.samples), "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(self.samples), "sampler": self.kind}
        if self.proc is None:
            return None
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "sampler": self.kind}


# --------------------------------------------------------------- reference
def write_ref_input(path, x, moments, order, depth, warmup, steps, output=3, backend=0):
    n = len(x)
    hdr = np.array([n, n, order, depth, 0, output, len(moments), warmup, steps, 1, 0, backend], dtype=np.int32)
    with open(path, "wb") as f:
        f.write(b"CDFMMIN1")
        f.write(hdr.tobytes())
        f.write(np.zeros(4).tobytes())
        f.write(np.ascontiguousarray(x, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(x, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(moments, dtype=np.float64).tobytes())
        f.write(np.arange(n, dtype=np.int32).tobytes())


def ref_sample_inputs(seed, states):
    """The bounded sample the reference is timed on: N = 131,072 uniform
    dipoles (seeded) and `states` unit-direction x U[0.5, 1.5] moment states."""
    s = REF_SAMPLE
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, size=(s["n"], 3))
    return x, unit_moments(rng, states, s["n"])


def run_reference_binary(x, m, warmup, steps, output, backend, threads):
    """Runs oracle/_ref/ref_bench (the reference built from its own sources)
    on inputs x, m (m: states x N x 3); a timed step evaluates every state
    once.  Returns its JSON summary."""
    s = REF_SAMPLE
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    with tempfile.TemporaryDirectory() as tmp:
        inp, out = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        write_ref_input(inp, x, m, s["order"], s["depth"], warmup, steps, output=output, backend=backend)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
        r = subprocess.run([exe, inp, out], capture_output=True, text=True, env=env, timeout=1800)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed: {r.stderr[-400:]}")
        return json.loads(r.stdout.strip().splitlines()[-1])


def run_reference_cpu(seed, warmup, steps, per_step=1):
    """Reference CpuStatic (FP32, field+potential) on the host cores: `warmup`
    untimed evaluations, then the median of `steps` samples of `per_step`
    evaluations each.  Returns (target-states/s, detail).  Falls back to the
    oracle port if the reference build is absent."""
    s = REF_SAMPLE
    x, m = ref_sample_inputs(seed, per_step)
    cores = os.cpu_count() or 1
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    sample = (f"N={s['n']} uniform dipoles, p={s['order']}, depth {s['depth']} (~32/leaf), one state per "
              f"evaluation, field+potential, FP32 CpuStatic; median of {steps} samples of {per_step} evaluations "
              f"after {warmup} warm-up evaluations")
    if os.path.exists(exe):
        info = run_reference_binary(x, m, warmup, steps, 3, 0, cores)
        per_eval = info["median_step_s"] / per_step
        return s["n"] / per_eval, {"kind": "reference", "cores": info["threads"], "sample": sample,
                                   "setup_s": info["setup_s"], "ms_per_state": per_eval * 1e3}
    import oracle

    t0 = time.perf_counter()
    oracle.fmm(x, x, m[0], s["order"], s["depth"], identities=np.arange(s["n"]))
    per_eval = time.perf_counter() - t0
    return s["n"] / per_eval, {"kind": "port", "cores": cores, "sample": sample.replace("FP32 CpuStatic",
                                                                                         "FP64 oracle port"),
                               "ms_per_state": per_eval * 1e3}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    value, info = run_reference_cpu(args.seed, max(1, args.warmup), max(1, args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["ms_per_state"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded uniform dipoles, unit-direction x U[0.5,1.5] moments",
            "config": {"workload": "reference CpuStatic on a bounded sample of the uniform p=6 workload",
                       "n_dipoles": REF_SAMPLE["n"], "order": REF_SAMPLE["order"], "depth": REF_SAMPLE["depth"],
                       "states_per_step": 1, "output": "field+potential"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- ranks (replicas)
def rank_moment_seed(seed, rank):
    """Replicas: every rank evaluates its own K states (seeded by rank) on the
    same geometry; no data-path collective."""
    return seed + 1000 * (rank + 1)


def reduce_max_over_ranks(v, dist, device):
    """Max of a per-rank time over all ranks (the job's step time)."""
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_step):
    """Aggregate throughput: the units all ranks processed / the max step time."""
    return units_per_rank * world / (ms_step * 1e-3)


# --------------------------------------------------------------------- B200
def b200_arm(args):
    import torch

    import cdfmm
    import cdfmm_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    if cdfmm_b200.device_count() == 0:
        raise RuntimeError("bench.py needs a CUDA device")

    N, K, p, d = args.n, args.states, args.order, args.depth
    mode = {"auto": cdfmm_b200.M2L_AUTO, "fp32": cdfmm_b200.M2L_FP32, "bf16x3": cdfmm_b200.M2L_BF16X3}[args.m2l]
    rng = np.random.default_rng(args.seed)
    x = rng.uniform(0.0, 1.0, size=(N, 3))
    opts = cdfmm.UniformTreeOptions()
    opts.max_level = d
    tree = cdfmm.UniformTree(x, x, opts)
    sorted_self = np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)]
    plan = cdfmm_b200.DevicePlan.from_tree(tree, p, max_states=K, m2l_mode=mode, device=local)
    plan.set_self_indices(sorted_self)
    near_mode = {"auto": cdfmm_b200.NEAR_AUTO, "fp32": cdfmm_b200.NEAR_FP32,
                 "tf32x3": cdfmm_b200.NEAR_TF32X3}[args.near]
    plan.set_near_mode(near_mode)
    moments = unit_moments(np.random.default_rng(rank_moment_seed(args.seed, rank)), K, N)
    # A dedicated stream: torch's events and our kernels are ordered on it.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dm = torch.from_numpy(moments).cuda()
    dH = torch.empty((K, N, 3), dtype=torch.float32, device="cuda")
    dphi = torch.empty((K, N), dtype=torch.float32, device="cuda")

    def step():
        plan.evaluate(dm, output="both", field=dH, potential=dphi, stream=stream.cuda_stream, synchronize=False)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        return reduce_max_over_ranks(v, dist, "cuda")

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(local)
    pci = None
    if all(hasattr(props, f) for f in ("pci_domain_id", "pci_bus_id", "pci_device_id")):
        pci = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
    clocks = ClockSampler(local, pci)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if args.nvtx:
        torch.cuda.nvtx.range_push("timed_steps")
    for _ in range(args.steps):
        step()
    if args.nvtx:
        torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    ms_step = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    value = whole_job_rate(N * K, world, ms_step)
    launches = plan.stats()["kernel_launches_last"] * args.steps

    # accuracy of state 0 (FP64 direct sum on a 16,384-target subsample)
    sub = np.random.default_rng(args.seed + 7).choice(N, size=min(N, 16384), replace=False)
    phi_ref, H_ref = cdfmm_b200.direct_fp64(x, moments[0].astype(np.float64), x[sub], sub, device=local)
    H0 = dH[0].cpu().numpy()[sub]
    phi0 = dphi[0].cpu().numpy()[sub]
    rel_h = float(np.sqrt(np.sum((H0 - H_ref) ** 2) / np.sum(H_ref ** 2)))
    rel_phi = float(np.sqrt(np.sum((phi0 - phi_ref) ** 2) / np.sum(phi_ref ** 2)))

    near_tc_used = bool(plan.stats()["near_tc_last"])
    # near/far schedules (with the FP32 near field, which has a co-resident
    # form): device time per step of each, and one concurrent trace each
    # (per-stream events: when the near field and the M2L ran)
    plan.set_near_mode(cdfmm_b200.NEAR_FP32)
    schedules = schedule_leg(plan, step, stream, args.steps, max_over_ranks, args.corun_shape_sweep)
    # the step with each near-field form (FP32 SIMT in its automatic
    # schedule, tensor cores beside the far field)
    near_field = {"used": "tf32x3" if near_tc_used else "fp32"}
    for name, nm in (("fp32", cdfmm_b200.NEAR_FP32), ("tf32x3", cdfmm_b200.NEAR_TF32X3)):
        try:
            plan.set_near_mode(nm)
        except cdfmm_b200.CdfmmError:
            continue
        near_field[name + "_ms_per_step"] = timed_steps(step, stream, args.steps, max_over_ranks)
    plan.set_near_mode(near_mode)
    step()
    torch.cuda.synchronize()

    # per-stage device times (separate, instrumented evaluations)
    plan.set_timing(True)
    stage_runs = []
    for _ in range(3):
        step()
        torch.cuda.synchronize()
        stage_runs.append(plan.stats())
    plan.set_timing(False)
    st = plan.stats()
    stages = {k[3:]: statistics.median(r[k] for r in stage_runs) for k in st if k.startswith("ms_")}

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        hm = torch.from_numpy(moments).pin_memory()
        hH = torch.empty((K, N, 3), dtype=torch.float32).pin_memory()
        hphi = torch.empty((K, N), dtype=torch.float32).pin_memory()

        def host_step():
            plan.evaluate(hm, output="both", field=hH, potential=hphi, stream=stream.cuda_stream,
                          synchronize=True, memory=cdfmm_b200.MOMENTS_ON_HOST | cdfmm_b200.RESULTS_ON_HOST)

        host_step()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            host_step()
        t_e2e = max_over_ranks((time.perf_counter() - t0) / args.steps)
        barrier()
        e2e = {"value": N * K * world / t_e2e, "unit": UNIT, "ms_per_step": t_e2e * 1e3,
               "h2d_bytes_per_step": int(hm.numel() * 4), "d2h_bytes_per_step": int((hH.numel() + hphi.numel()) * 4)}
        del hm, hH, hphi

    # the plain per-state FP32 path on the same GPU (K sequential single-state calls)
    plain_plan = cdfmm_b200.DevicePlan.from_tree(tree, p, max_states=1, m2l_mode=cdfmm_b200.M2L_FP32, device=local)
    plain_plan.set_self_indices(sorted_self)
    ks = max(1, min(args.plain_states, K))
    pH = torch.empty((1, N, 3), dtype=torch.float32, device="cuda")
    pphi = torch.empty((1, N), dtype=torch.float32, device="cuda")
    states = [dm[k:k + 1] for k in range(ks)]

    def plain_step():
        for s in states:
            plain_plan.evaluate(s, output="both", field=pH, potential=pphi, stream=stream.cuda_stream,
                                synchronize=False)

    plain_step()
    torch.cuda.synchronize()
    barrier()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    plain_step()
    p1.record(stream)
    torch.cuda.synchronize()
    ms_state_plain = max_over_ranks(p0.elapsed_time(p1) / ks)
    plain_value = N * world / (ms_state_plain * 1e-3)
    plain_plan.close()

    # Reverse mode on the same workload: the forward (field output) against
    # the backward of L = sum w . H giving dL/dmoments (transposed plan) and
    # dL/dtarget-positions, both device-timed on the bench stream.
    backward = None
    if not args.no_backward:
        dW = torch.from_numpy(np.random.default_rng(args.seed + 3).normal(size=(K, N, 3)).astype(np.float32)).cuda()
        gm = torch.empty_like(dm)
        gx = torch.empty((N, 3), dtype=torch.float32, device="cuda")

        def fwd():
            plan.evaluate(dm, output="field", field=dH, stream=stream.cuda_stream, synchronize=False)

        def bwd():
            plan.backward(dW, moments=dm, grad_moments=gm, grad_target_positions=gx, want_moments=True,
                          want_positions=True, stream=stream.cuda_stream, synchronize=False)

        def timed(fn, reps):
            fn()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(reps):
                fn()
            b.record(stream)
            torch.cuda.synchronize()
            return max_over_ranks(a.elapsed_time(b) / reps)

        def train_step():
            # forward then backward reusing its sorted moments and leaf locals
            fwd()
            evaluation = plan.stats()["evaluations"]
            plan.backward(dW, moments=dm, grad_moments=gm, grad_target_positions=gx, want_moments=True,
                          want_positions=True, stream=stream.cuda_stream, synchronize=False,
                          forward_evaluation=evaluation)

        reps = max(1, args.steps)
        ms_f = timed(fwd, reps)
        ms_b = timed(bwd, reps)
        ms_fb = timed(train_step, reps)
        backward = {"ms_forward_field": ms_f, "ms_backward": ms_b, "backward_over_forward": ms_b / ms_f,
                    "ms_forward_plus_backward": ms_fb,
                    "backward_after_forward_over_forward": (ms_fb - ms_f) / ms_f,
                    "outputs": "dL/dmoments (K x N x 3) + dL/dtarget_positions (N x 3), L = sum w.H",
                    "note": "ms_backward recomputes the forward far pass; after a forward the backward reuses it"}
        del dW, gm, gx

    multi = None
    if not args.no_multi and world == 1:
        multi = multi_geometry_leg(args, stream, local)
    lattice = None
    if not args.no_lattice and world == 1:
        lattice = lattice_leg(args, stream, local)
    differentiable = None
    if not args.no_backward and world == 1:
        differentiable = differentiable_leg(args, stream, local)

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    peaks, peak_kind = load_peaks()
    n = (p + 1) * (p + 2) * (p + 3) // 6
    # the tensor-core M2L applies the traceless-reduced operator: (p+1)^2 - 1
    # folded moments in, (p+1)^2 locals out (the other locals follow from the
    # trace relations); the full-basis count 2 n^2 is kept beside it
    m2l_full_flop = 2.0 * n * n * st["m2l_interactions"] * K
    m2l_flop = (2.0 * ((p + 1) ** 2 - 1) * (p + 1) ** 2 * st["m2l_interactions"] * K if st["m2l_mode_resolved"] == 2
                else m2l_full_flop)
    p2p_flop = (st["p2p_pairs"] - N) * (13.0 + 20.0 * K)
    near_key = "near_tc" if near_tc_used else "p2p"
    cand = {"m2l": (stages.get("m2l", 0.0), m2l_flop), near_key: (stages.get("p2p", 0.0), p2p_flop)}
    dom = max(cand, key=lambda k: cand[k][0])
    ms_dom, flop_dom = cand[dom]
    if dom == "m2l":
        peak = peaks.get("bf16_tflops_sustained", FALLBACK_PEAKS["bf16_tflops_sustained"])
        roofline = {"kernel": "m2l", "bound": "tensor", "unit": "TFLOP/s",
                    "algorithmic_flop": m2l_flop, "full_basis_flop": m2l_full_flop,
                    "peak_source": f"{peak_kind} bf16_tflops_sustained"}
    elif dom == "near_tc":
        # TF32 MMAs run at half the BF16 rate on this part (nominal 1.1 vs
        # 2.25 PFLOP/s dense)
        peak = 0.5 * peaks.get("bf16_tflops_sustained", FALLBACK_PEAKS["bf16_tflops_sustained"])
        # issued tensor work: 128 rows x 3 split products x the units' padded
        # reduction length x the states padded to 16
        issued = 2.0 * 128 * 3 * st["near_tc_k_cols"] * (16 * ((K + 15) // 16))
        roofline = {"kernel": "near_tc", "bound": "tensor", "unit": "TFLOP/s", "algorithmic_flop": p2p_flop,
                    "peak_source": f"{peak_kind} bf16_tflops_sustained / 2 (TF32 rate)",
                    "fp32_fma_frac": p2p_flop / (ms_dom * 1e-3) / 1e12 / FP32_NOMINAL_TFLOPS if ms_dom > 0 else None,
                    "issued_flop": issued,
                    "issued_frac": issued / (ms_dom * 1e-3) / 1e12 / peak if ms_dom > 0 else None}
    else:
        peak = FP32_NOMINAL_TFLOPS
        roofline = {"kernel": "p2p", "bound": "fp32", "unit": "TFLOP/s", "algorithmic_flop": p2p_flop,
                    "peak_source": "nominal FP32 FMA (148 SM x 128 lanes x 2 x 1.965 GHz)"}
    achieved = flop_dom / (ms_dom * 1e-3) / 1e12 if ms_dom > 0 else 0.0
    roofline.update({"achieved": achieved, "peak": peak, "frac": achieved / peak if peak else None,
                     "kernel_ms": ms_dom, "traffic": traffic_from_profiles(dom)})

    # HBM-bound stages: compulsory DRAM bytes per evaluation (FP32) / stage time
    # -- P2M and L2P 12N + 12NK + 4 n L_leaf K (+ 4NK potential for L2P), M2M
    # 4nK (nodes - 1) read + 4nK non-leaf written, L2L reads the locals of
    # levels 2..d-1 and reads + writes those of levels 3..d, gather 12NK read +
    # 16NK written.
    n_leaves = 8 ** d
    nodes = (8 ** (d + 1) - 1) // 7
    nonleaf = nodes - n_leaves
    hbm_peak = peaks.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"])
    hbm_bytes = {
        "gather": 12.0 * N * K + 16.0 * N * K,
        "p2m": 12.0 * N + 12.0 * N * K + 4.0 * n * n_leaves * K,
        "m2m": 4.0 * n * K * (nodes - 1) + 4.0 * n * K * nonleaf,
        "l2l": 4.0 * n * K * (nonleaf - 9) + 8.0 * n * K * (nodes - 73),  # parents at levels 2..d-1, children 3..d
        "l2p": 12.0 * N + 12.0 * N * K + 4.0 * N * K + 4.0 * n * n_leaves * K,
    }
    hbm = {}
    for k, b in hbm_bytes.items():
        ms_k = stages.get(k, 0.0)
        if ms_k > 0:
            gbs = b / (ms_k * 1e-3) / 1e9
            hbm[k] = {"bytes": b, "ms": ms_k, "GB/s": gbs, "frac": gbs / hbm_peak}
    hbm["_peak"] = {"GB/s": hbm_peak, "source": f"{peak_kind} hbm_gbs"}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        # the reference's own protocol: 2 warm-ups, median of 5 samples x 10 evaluations
        v, info = run_reference_cpu(args.seed, 2, 5, 10)
        cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"], "sample": info["sample"],
               "ms_per_state": info["ms_per_state"]}
    reference_gpu = None
    if world == 1 and not args.no_reference_gpu:
        reference_gpu = reference_gpu_leg(args, stream, local)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded uniform dipoles in the unit cube, unit-direction x U[0.5,1.5] moments",
        "config": {"workload": f"uniform N={N} dipoles, p={p}, depth {d}, K={K} states per step, field+potential",
                   "n_dipoles": N, "order": p, "depth": d, "states_per_step": K, "output": "field+potential",
                   "m2l": ["auto", "fp32", "bf16x3"][st["m2l_mode_resolved"]],
                   "m2l_shape": {"accumulators_per_cta": st["m2l_tc_m_tiles"], "stages": st["m2l_tc_stages"],
                                 "fused_hi_lo_mma": bool(st["m2l_tc_fused"]),
                                 "chosen_by": "autotuner"},
                   "l2": f"inputs larger than L2 ({dm.numel() * 4 / 2**20:.0f} MiB of moments per step)",
                   "parallelism": "replicas (independent states per GPU)" if world > 1 else "single GPU"},
        "rel_l2_H": rel_h, "rel_l2_phi": rel_phi,
        "e2e": e2e, "gpu_launches": int(launches), "clocks": clock_info, "roofline": roofline,
        "cpu_baseline": cpu, "reference_gpu": reference_gpu, "stages_ms": stages, "hbm_stages": hbm,
        "schedules": schedules, "near_field": near_field,
        "plain": {"value": plain_value, "unit": UNIT, "ms_per_state": ms_state_plain, "states_timed": ks,
                  "m2l": "fp32"},
        "batched_over_plain": value / plain_value,
        "backward": backward,
        "multi_geometry": multi,
        "lattice_p8": lattice,
        "differentiable_p8": differentiable,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def reference_gpu_leg(args, stream, local):
    """The reference's own GPU path (CudaFull: cuSPARSE near field, cuBLAS
    M2L; FP32, field only, one state per call, host arrays in and out) on
    this GPU, on the bounded sample N = 131,072, p = 6, depth 4 where its
    host plan fits, timed by the reference itself (median per evaluation of
    its device-kernel and whole-call seconds, 2 warm-ups then 5 x 10
    evaluations), beside this library on the same inputs: one state per
    call (the plain path, host arrays, as the reference's API) and K = 64
    states per call (device-resident and through host arrays)."""
    import cdfmm
    import cdfmm_b200
    import torch

    s = REF_SAMPLE
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_bench")):
        return {"unavailable": "reference build (oracle/_ref) absent"}
    x, m = ref_sample_inputs(args.seed + 5, 10)
    try:
        info = run_reference_binary(x, m, 2, 5, 2, 2, os.cpu_count() or 1)
    except (RuntimeError, subprocess.TimeoutExpired, ValueError) as e:
        return {"unavailable": f"reference CudaFull run failed: {str(e)[-300:]}"}
    per_call = info["median_step_s"] / len(m)
    ref = {"ms_kernel": info["median_kernel_s"] * 1e3, "ms_h2d": info["median_h2d_s"] * 1e3,
           "ms_d2h": info["median_d2h_s"] * 1e3, "ms_call": per_call * 1e3, "setup_s": info["setup_s"],
           "value_call": s["n"] / per_call, "value_kernel": s["n"] / info["median_kernel_s"]}

    o = cdfmm.UniformTreeOptions()
    o.max_level = s["depth"]
    tree = cdfmm.UniformTree(x, x, o)
    sorted_self = np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)]

    def timed_ms(fn, reps):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    plain = cdfmm_b200.DevicePlan.from_tree(tree, s["order"], max_states=1, m2l_mode=cdfmm_b200.M2L_FP32,
                                            device=local)
    plain.set_self_indices(sorted_self)
    hm1 = torch.from_numpy(m[:1]).pin_memory()
    hH1 = torch.empty((1, s["n"], 3), dtype=torch.float32).pin_memory()

    def plain_host():
        plain.evaluate(hm1, output="field", field=hH1, stream=stream.cuda_stream, synchronize=True,
                       memory=cdfmm_b200.MOMENTS_ON_HOST | cdfmm_b200.RESULTS_ON_HOST)

    dm1 = hm1.cuda()
    dH1 = torch.empty((1, s["n"], 3), dtype=torch.float32, device="cuda")

    def plain_dev():
        plain.evaluate(dm1, output="field", field=dH1, stream=stream.cuda_stream, synchronize=False)

    ms_plain_call = timed_ms(plain_host, 10)
    ms_plain_dev = timed_ms(plain_dev, 10)
    plain.close()
    K = 64
    batched = cdfmm_b200.DevicePlan.from_tree(tree, s["order"], max_states=K, device=local)
    batched.set_self_indices(sorted_self)
    mk = unit_moments(np.random.default_rng(args.seed + 6), K, s["n"])
    dmk = torch.from_numpy(mk).cuda()
    dHk = torch.empty((K, s["n"], 3), dtype=torch.float32, device="cuda")
    hmk = torch.from_numpy(mk).pin_memory()
    hHk = torch.empty((K, s["n"], 3), dtype=torch.float32).pin_memory()

    def batched_dev():
        batched.evaluate(dmk, output="field", field=dHk, stream=stream.cuda_stream, synchronize=False)

    def batched_host():
        batched.evaluate(hmk, output="field", field=hHk, stream=stream.cuda_stream, synchronize=True,
                         memory=cdfmm_b200.MOMENTS_ON_HOST | cdfmm_b200.RESULTS_ON_HOST)

    ms_k_dev = timed_ms(batched_dev, 5)
    ms_k_call = timed_ms(batched_host, 5)
    batched.close()
    n = s["n"]
    ours = {"plain_ms_call": ms_plain_call, "plain_ms_device": ms_plain_dev,
            "plain_value_call": n / (ms_plain_call * 1e-3),
            "batched_ms_device": ms_k_dev, "batched_ms_call": ms_k_call,
            "batched_value_device": n * K / (ms_k_dev * 1e-3), "batched_value_call": n * K / (ms_k_call * 1e-3)}
    return {"workload": f"uniform N={n}, p={s['order']}, depth {s['depth']}, field only, FP32",
            "reference_cudafull": ref, "b200": ours, "unit": UNIT,
            "plain_over_reference_call": ours["plain_value_call"] / ref["value_call"],
            "batched_over_reference_call": ours["batched_value_call"] / ref["value_call"],
            "batched_device_over_reference_kernel": ours["batched_value_device"] / ref["value_kernel"]}


SCHEDULE_NAMES = {1: "separate", 2: "corun"}


def timed_steps(step, stream, steps, max_over_ranks):
    """Device ms per step over `steps` steps after one untimed step."""
    import torch

    step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(max(1, steps)):
        step()
    b.record(stream)
    torch.cuda.synchronize()
    return max_over_ranks(a.elapsed_time(b) / max(1, steps))


def schedule_leg(plan, step, stream, steps, max_over_ranks, shape_sweep=False):
    """Each near/far schedule of the K-state evaluation: device time per step
    (CUDA events around `steps` steps after a warm-up) and a trace of one
    evaluation (device events on the near and far streams, ms from its
    start).  The plan returns to its automatic schedule afterwards."""
    import cdfmm_b200
    import torch

    out = {}
    for sched, name in SCHEDULE_NAMES.items():
        plan.set_schedule(sched)
        step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(max(1, steps)):
            step()
        b.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b) / max(1, steps))
        plan.set_timing(2)
        step()
        torch.cuda.synchronize()
        st = plan.stats()
        plan.set_timing(0)
        trace = {k[6:]: st[k] for k in st if k.startswith("trace_")}
        overlap = max(0.0, min(trace["p2p_end"], trace["far_end"]) - max(trace["p2p_begin"], trace["m2l_begin"]))
        out[name] = {"ms_per_step": ms, "trace_ms": trace, "p2p_m2l_overlap_ms": overlap}
    if shape_sweep:
        # every M2L pipeline shape pinned in turn under the co-resident schedule
        plan.set_schedule(cdfmm_b200.SCHEDULE_CORUN)
        sweep = []
        for mt, st, fused in plan.m2l_shapes():
            plan.set_m2l_shape(mt, st, fused)
            step()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(max(1, steps)):
                step()
            b.record(stream)
            torch.cuda.synchronize()
            plan.set_timing(2)
            step()
            torch.cuda.synchronize()
            tr = plan.stats()
            plan.set_timing(0)
            sweep.append({"shape": [mt, st, bool(fused)], "ms_per_step": a.elapsed_time(b) / max(1, steps),
                          "p2p_ms": tr["trace_p2p_end"] - tr["trace_p2p_begin"],
                          "m2l_ms": tr["trace_far_end"] - tr["trace_m2l_begin"]})
        plan.set_m2l_shape(0)
        out["corun_shape_sweep"] = sweep
    plan.set_schedule(cdfmm_b200.SCHEDULE_AUTO)
    step()
    torch.cuda.synchronize()
    out["auto"] = SCHEDULE_NAMES.get(plan.stats()["schedule_last"])
    return out


def clustered_points(rng, n, clusters=8, sigma=0.05):
    """n points from `clusters` isotropic Gaussians (sigma 0.05, centres
    U[0.1, 0.9]^3); points outside the unit cube are rejected and redrawn."""
    centres = rng.uniform(0.1, 0.9, (clusters, 3))
    out = np.empty((0, 3))
    while len(out) < n:
        c = centres[rng.integers(0, clusters, size=2 * n)]
        p = c + rng.normal(scale=sigma, size=c.shape)
        out = np.concatenate([out, p[np.all((p >= 0.0) & (p < 1.0), axis=1)]])
    return out[:n]


def multi_geometry_leg(args, stream, local):
    """Uneven multi-geometry batch: `--multi-problems` independent problems,
    N log-uniform in [8192, 524288], clustered positions, depth
    round(log8(N/32)), p = 6, unit random-direction moments, one state each,
    field output, all evaluated by ONE CUDA graph launch (cdfmm_b200_batch)."""
    import math

    import cdfmm
    import cdfmm_b200
    import torch

    rng = np.random.default_rng(args.seed + 77)
    count = args.multi_problems
    sizes = np.round(np.exp(rng.uniform(math.log(8192), math.log(524288), size=count))).astype(int)
    points = [clustered_points(rng, int(n)) for n in sizes]
    depths = [max(1, int(round(math.log(int(n) / 32.0, 8)))) for n in sizes]
    # plan set-up from the host tree (cdfmm.UniformTree + self map + plan)
    t0 = time.perf_counter()
    for x, depth in zip(points, depths):
        o = cdfmm.UniformTreeOptions()
        o.max_level = depth
        tree = cdfmm.UniformTree(x, x, o)
        plan = cdfmm_b200.DevicePlan.from_tree(tree, 6, max_states=1, device=local)
        plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
        plan.close()
    setup_host_s = time.perf_counter() - t0
    # plan set-up with the octree built on the device (the plans used below)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plans = [cdfmm_b200.DevicePlan.from_points(x, 6, depth, max_states=1, device=local)
             for x, depth in zip(points, depths)]
    setup_s = time.perf_counter() - t0
    phases = {}
    for plan in plans:
        for key, v in plan.stats().items():
            if key.startswith("setup_ms_"):
                phases[key[9:]] = phases.get(key[9:], 0.0) + v
    probs, items = [], []
    for x, plan in zip(points, plans):
        n = len(x)
        d = rng.normal(size=(1, n, 3))
        d /= np.linalg.norm(d, axis=2, keepdims=True)
        dm = torch.from_numpy(d.astype(np.float32)).cuda()
        dH = torch.empty((1, n, 3), dtype=torch.float32, device="cuda")
        probs.append((x, plan, d, dH))
        items.append((plan, dm, dH, None))
    batch = cdfmm_b200.Batch(items, output="field")
    for _ in range(3):
        batch.launch(stream=stream.cuda_stream, synchronize=False)
    torch.cuda.synchronize()
    reps = max(3, args.steps)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        batch.launch(stream=stream.cuda_stream, synchronize=False)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    # the same problems evaluated one call after another (no graph)
    def sequential():
        for plan, dm, dH, _ in items:
            plan.evaluate(dm, output="field", field=dH, stream=stream.cuda_stream, synchronize=False)

    sequential()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        sequential()
    b.record(stream)
    torch.cuda.synchronize()
    ms_seq = a.elapsed_time(b) / reps
    # accuracy vs the FP64 direct sum: 4,096 sampled targets of the largest,
    # the median-size and the smallest problem
    order = np.argsort(sizes)
    worst = 0.0
    for idx in (order[-1], order[len(order) // 2], order[0]):
        x, plan, d, dH = probs[int(idx)]
        sub = np.random.default_rng(args.seed + 9).choice(len(x), size=min(len(x), 4096), replace=False)
        _, H_ref = cdfmm_b200.direct_fp64(x, d[0], x[sub], sub, device=local)
        H = dH[0].cpu().numpy()[sub]
        worst = max(worst, float(np.sqrt(np.sum((H - H_ref) ** 2) / np.sum(H_ref ** 2))))
    batch.close()
    for _, plan, _, _ in probs:
        plan.close()
    total = int(sizes.sum())
    return {"problems": count, "total_targets": total, "n_min": int(sizes.min()), "n_max": int(sizes.max()),
            "order": 6, "states": 1, "output": "field", "graph_launches_per_step": 1, "ms_per_launch": ms,
            "ms_sequential_calls": ms_seq,
            "value": total / (ms * 1e-3), "unit": "target evals/s", "rel_l2_H_max_checked": worst,
            "plan_setup_s": setup_s, "plan_setup_host_tree_s": setup_host_s,
            "plan_setup_phases_ms": {k: round(v, 1) for k, v in phases.items()},
            "plan_setup_note": "device octree (cdfmm_b200_plan_create_from_points) vs host tree + from_tree + self "
                               "map; point generation excluded",
            "data": "synthetic: 8 Gaussian clusters (sigma 0.05, centres U[0.1,0.9]^3, out-of-cube points redrawn)"}


def lattice_leg(args, stream, local):
    """Batched moments + split-precision M2L: a 64^3 lattice (spacing 1/64,
    each coordinate jittered by U(-0.1, 0.1) spacings), N = 262,144, exactly
    8 per leaf at depth 5, K = 64 states of i.i.d. N(0, 1) moments, p = 8,
    field only, split-BF16 M2L on the tensor cores."""
    import cdfmm
    import cdfmm_b200
    import torch

    rng = np.random.default_rng(args.seed + 11)
    g = np.stack(np.meshgrid(np.arange(64), np.arange(64), np.arange(64), indexing="ij"), axis=-1).reshape(-1, 3)
    x = (g + rng.uniform(-0.1, 0.1, size=g.shape)) / 64.0
    N, K, p, d = len(x), 64, 8, 5
    o = cdfmm.UniformTreeOptions()
    o.max_level = d
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, p, max_states=K, device=local)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = rng.normal(size=(K, N, 3)).astype(np.float32)
    dm = torch.from_numpy(m).cuda()
    dH = torch.empty((K, N, 3), dtype=torch.float32, device="cuda")

    def run():
        plan.evaluate(dm, output="field", field=dH, stream=stream.cuda_stream, synchronize=False)

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    reps = max(3, args.steps)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        run()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    sub = np.random.default_rng(args.seed + 12).choice(N, size=16384, replace=False)
    _, H_ref = cdfmm_b200.direct_fp64(x, m[0].astype(np.float64), x[sub], sub, device=local)
    H = dH[0].cpu().numpy()[sub]
    rel = float(np.sqrt(np.sum((H - H_ref) ** 2) / np.sum(H_ref ** 2)))
    st = plan.stats()
    plan.close()
    return {"workload": "64^3 jittered lattice, N=262144, p=8, depth 5, K=64, field only", "ms_per_step": ms,
            "value": N * K / (ms * 1e-3), "unit": UNIT, "rel_l2_H": rel,
            "m2l": ["auto", "fp32", "bf16x3"][st["m2l_mode_resolved"]],
            "m2l_shape": {"accumulators_per_cta": st["m2l_tc_m_tiles"], "stages": st["m2l_tc_stages"],
                          "fused_hi_lo_mma": bool(st["m2l_tc_fused"])}}


def differentiable_leg(args, stream, local):
    """Differentiable FMM: N = 524,288 uniform, p = 8, depth 5, one state;
    L = sum_i w_i . H_i with w_i ~ N(0, 1)^3; device time of the field forward
    and of the backward (dL/dmoments + dL/dtarget-positions); the gradients
    checked against the FP64 direct sums on 4,096 sampled points."""
    import cdfmm
    import cdfmm_b200
    import torch

    rng = np.random.default_rng(args.seed + 21)
    N, p, d = 524288, 8, 5
    x = rng.uniform(0.0, 1.0, size=(N, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = d
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, p, max_states=1, device=local)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = unit_moments(rng, 1, N)
    w = rng.normal(size=(1, N, 3)).astype(np.float32)
    dm, dw = torch.from_numpy(m).cuda(), torch.from_numpy(w).cuda()
    dH = torch.empty((1, N, 3), dtype=torch.float32, device="cuda")
    gm = torch.empty_like(dm)
    gx = torch.empty((N, 3), dtype=torch.float32, device="cuda")

    def fwd():
        plan.evaluate(dm, output="field", field=dH, stream=stream.cuda_stream, synchronize=False)

    def bwd():
        plan.backward(dw, moments=dm, grad_moments=gm, grad_target_positions=gx, want_moments=True,
                      want_positions=True, stream=stream.cuda_stream, synchronize=False)

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    reps = max(3, args.steps)
    ms_f = timed(fwd, reps)
    ms_b = timed(bwd, reps)
    sub = np.random.default_rng(args.seed + 22).choice(N, size=4096, replace=False)
    # dL/dm_j = field of the weights (as dipoles at the targets) at source j
    _, gm_ref = cdfmm_b200.direct_fp64(x, w[0].astype(np.float64), x[sub], sub, device=local)
    gx_ref = cdfmm_b200.direct_grad_fp64(x, m[0].astype(np.float64), x[sub], w[0][sub].astype(np.float64), sub,
                                         device=local)
    gm_s = gm[0].cpu().numpy()[sub]
    gx_s = gx.cpu().numpy()[sub]
    plan.close()
    return {"workload": "uniform N=524288, p=8, depth 5, one state, L = sum w.H", "ms_forward_field": ms_f,
            "ms_backward": ms_b, "backward_over_forward": ms_b / ms_f,
            "rel_l2_grad_moments": float(np.sqrt(np.sum((gm_s - gm_ref) ** 2) / np.sum(gm_ref ** 2))),
            "rel_l2_grad_positions": float(np.sqrt(np.sum((gx_s - gx_ref) ** 2) / np.sum(gx_ref ** 2))),
            "checked": "4096 sampled points vs FP64 direct sums (transpose field; position gradient)"}


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel)
    except (OSError, ValueError):
        return None


def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
