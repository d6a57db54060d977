#!/usr/bin/env python
"""Benchmark of the motion-stereo depth-map pipeline on B200.

One step = one depth map per sequence: a reference frame plus S source frames (cost volume),
8-path SGM, winner-take-all / flatness / uniqueness / subpixel, and one Bayesian fusion step
against the previous keyframe's state.  Workload: 640x480, 128 inverse-depth planes uniform in
[0.1, 2.0] 1/m, 5 sources, f = 520, seeded synthetic scenes (six textured planes).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--form batched|plain|mixed] [--precision fp16|fp32] [--batch B] [--lanes L]

Default (the headline): the FP16 form, B sequences batched (one CUDA-graph launch per step for
all B), sources sampled by the texture unit from FP32 texels of FP16-rounded values (as the
reference's own textures: 8-bit bilinear weights), against the plain FP32 form (one
StereoMapper, one map after the other, exact bilinear weights) measured in the same run.  `value` is depth maps/s with inputs resident in HBM; `e2e` is the same through the
public C ABI with pinned host frames and outputs copied inside the timed region.  Under
torchrun every rank maps its own sequences (no collective on the data path) and the slowest
rank's time is used.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "depth maps/s @640x480x128 planes, FP16-batched vs plain FP32; % HBM roofline"
W, H, D, S, F_PX = 640, 480, 128, 5, 520.0
PATHS = 8
# tau_so = 3.5/255: on uint8 intensities scaled by 1/255 this is the reference's |dI| < 4
# (parameters.cpp:14) without a threshold that sits exactly on an intensity step, where FP32
# and FP64 rounding would disagree.
P1, P2, TAU, UNIQ = 0.003, 0.01, 3.5 / 255.0, 0.95
N_KEYFRAMES = 4
SAMPLERS = {"exact": 0, "texture": 1, "texture_f32": 2}   # PM_SAMPLER_* (FP32 form: exact or texture_f32)


def peaks():
    """HBM copy bandwidth (GB/s) and the SM clock the FP32 SIMT peak is derived from."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d.get("sm_max_mhz", 1965.0)), "measured"
    except Exception:
        return 6650.0, 1965.0, "fallback"


def fp32_peak_tflops(sm_mhz: float) -> float:
    """Non-tensor FP32 peak: 148 SMs x 128 FP32 lanes x 2 flop (FMA) per clock."""
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


def ncu_traffic(kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` at this workload, from the committed ncu
    summary profiles/traffic.json (written from a capture of this same bench command)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)["kernels"][kernel]["dram_bytes_per_launch"]
    except Exception:
        return None


class ClockSampler:
    """Polls SM clock and clock-event (throttle) reasons through NVML every 10 ms while the timed
    region runs (read-only queries; no GPU setting is changed)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.cuda_index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def __enter__(self):
        try:
            import pynvml
            h = self._handle()
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append((float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                                             int(get_reasons(h))))
                    except Exception:
                        pass
                    self._stop.wait(0.01)

            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        reasons = set()
        for _, r in self.samples:
            for bit, name in self.REASONS.items():
                if r & bit:
                    reasons.add(name)
        return {"sm_mhz": float(np.median([c for c, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def sampler_name(args, precision) -> str:
    """The source sampler of a form: --sampler for the FP16 form, --fp32-sampler for the FP32 one."""
    return args.sampler if precision in ("fp16", 1) else args.fp32_sampler


def make_mapper(precision: int, device: int, cost_mode: int = 0, sampler: int = 0):
    from probabilistic_mapping_b200 import scene
    from probabilistic_mapping_b200.mapper import StereoMapper
    rho0, drho = scene.plane_range(D)
    m = StereoMapper(W, H, D, rho0=rho0, intensity_scale=1 / 255, num_paths=PATHS, p1=P1, p2=P2, tau_so=TAU,
                     uniqueness_ratio=UNIQ, cost_mode=cost_mode, precision=precision, device=device,
                     sampler=sampler)
    return m, drho


def algorithmic_bytes(e: int):
    """Per depth map: B_alg = (S+1) N + 3 e V + 8 V + 60 N (path-grouped lower bound), and the
    bytes the SGM stage of this implementation must move."""
    N = W * H
    V = N * D
    b_alg = (S + 1) * N + 3 * e * V + 8 * V + 60 * N
    # every path reads C and the reference image; each opposite-path pair stores one volume (FP32,
    # or FP16 in the FP16 form, the element size of its cost volume) and adds into it once (a read
    # and a write); the combine reads the pair volumes and writes depth and index
    pairs = PATHS // 2
    sgm_pass = PATHS * (e * V + 4 * N) + pairs * (e * V + 2 * e * V) + pairs * e * V + 8 * N
    return b_alg, sgm_pass


# Cost construction: 9 projective warps + 9 bilinear samples + 9 absolute differences per voxel
# and source, 144 FP32 flop counting a division as one: per sample 8 for the warp (three
# multiply-adds and the division), 6 for the bilinear interpolation (three lerps), 2 for the
# absolute difference and its sum.  With a texture sampler the texture unit does the
# interpolations (54 of the 144), so the SIMT pipes are credited with the other 90 only.
FLOP_PER_VOXEL_SOURCE = 144
FLOP_BILINEAR_PER_VOXEL_SOURCE = 9 * 6


def cost_kernel_work(e: int, texels: bool = False):
    """Algorithmic flop and bytes of one cost-kernel launch (all S sources folded at once): the
    volume written once (e V), the reference image and the S source images read once (16-byte
    quads for the exact sampler, 4-byte texels for the texture sampler).  Returns (flop on the
    SIMT pipes, flop done by the texture unit, bytes)."""
    N = W * H
    V = N * D
    tex_flop = FLOP_BILINEAR_PER_VOXEL_SOURCE * V * S if texels else 0
    return FLOP_PER_VOXEL_SOURCE * V * S - tex_flop, tex_flop, e * V + 4 * N + (4 if texels else 16) * N * S


# The texture samplers' binding unit: ncu counts at most one texture output wavefront per SM and
# cycle, and eight per 32-lane bilinear fetch instruction, so an SM filters 4 fetches per clock.
TEX_FETCHES_PER_SM_CLK = 4


def cost_kernel_fetches(reference_mode: bool):
    """Filtered texture fetches of one cost-kernel launch with a texture sampler.  Algorithmic: one
    per warped position, plane and source (the row sample the 3x3 window shares) plus, in reference
    mode, the two corrupted-neighbour samples per voxel and source.  Issued: the tile design's
    fetch instructions x 32 lanes -- 30x8-pixel tiles of 16 planes, one plane pair per warp, each
    warp sampling 10 rows for its 8 output rows (+ 2 samples per output row in reference mode)."""
    V = W * H * D
    alg = V * S * (3 if reference_mode else 1)
    tiles = -(-W // 30) * -(-H // 8) * (D // 16)
    per_warp_source = 10 * 2 + (8 * 2 * 2 if reference_mode else 0)
    return alg, tiles * 8 * S * per_warp_source * 32


def cost_roofline(cost_ms, cost_stage_ms, e, texels, reference_mode, sm_mhz, peak_hbm, peak_kind, precision,
                  traffic):
    """The cost kernel against its binding roof.  It is not HBM-bound: with exact bilinear the FP32
    SIMT pipes bind (algorithmic flop on the SIMT pipes against the derived FP32 peak); with a
    texture sampler the texture unit's filtering rate binds (ncu: the texture pipe near its peak),
    so `achieved` is the algorithmic fetch count per launch over the kernel's time, against the
    derived 4 fetches per SM and clock, with the FP32 figures under `fp32_simt`.  cost_ms is the
    kernel alone (CUDA events on the mapper's stream, the FP16 form's rebase pass excluded)."""
    simt_flop, tex_flop, cost_bytes = cost_kernel_work(e, texels)
    peak_fp32 = fp32_peak_tflops(sm_mhz)
    sec = cost_ms / 1000.0 if cost_ms and cost_ms > 0 else None
    tflops = simt_flop / sec / 1e12 if sec else None
    gbs = cost_bytes / sec / 1e9 if sec else None
    fp32 = {"bound": "fp32", "kernel": "cost_kernel", "achieved": tflops, "peak": peak_fp32, "unit": "TFLOP/s",
            "frac": tflops / peak_fp32 if tflops else None,
            "algorithmic_flop_per_launch": simt_flop, "texture_unit_flop_per_launch": tex_flop,
            "frac_counting_texture_interpolation": (simt_flop + tex_flop) / sec / 1e12 / peak_fp32 if sec else None,
            "algorithmic_bytes_per_launch": cost_bytes, "hbm_achieved_gbs": gbs,
            "hbm_frac": gbs / peak_hbm if gbs else None,
            "peak_kind": f"derived FP32 peak: 148 SM x 128 lanes x 2 flop x {sm_mhz:.0f} MHz ({peak_kind} clock); "
                         "no measured FP32 SIMT peak exists"}
    common = {"traffic": traffic, "ms_per_launch": cost_ms, "stage_ms_with_rebase": cost_stage_ms,
              "precision": precision}
    if not texels:
        return {**fp32, **common}
    f_alg, f_issued = cost_kernel_fetches(reference_mode)
    peak_tex = 148 * TEX_FETCHES_PER_SM_CLK * sm_mhz * 1e6 / 1e9   # G fetches/s
    got = f_alg / sec / 1e9 if sec else None
    return {"bound": "texture", "kernel": "cost_kernel", "achieved": got, "peak": peak_tex, "unit": "G fetches/s",
            "frac": got / peak_tex if got else None, **common,
            "fetches_algorithmic_per_launch": f_alg, "fetches_issued_per_launch": f_issued,
            "frac_issued": f_issued / sec / 1e9 / peak_tex if sec else None,
            "peak_kind": f"derived: 148 SM x {TEX_FETCHES_PER_SM_CLK} filtered fetches per clock x {sm_mhz:.0f} MHz "
                         "(ncu: one texture output wavefront per SM and cycle at peak, eight per 32-lane fetch "
                         "instruction); no measured texture peak exists",
            "fp32_simt": fp32}


def sgm_alg_bytes(e: int):
    """The SGM + winner-take-all + fusion share of B_alg per map: two sweeps over the cost volume
    (2 e V), the forward sweep's path sum written and read back once (8 V), the reference image
    (4 N) and the fusion state and outputs (56 N)."""
    N = W * H
    V = N * D
    return 2 * e * V + 8 * V + 4 * N + 56 * N


def run_ours(args, rank, world, precision: str = "fp32", passes=("dev", "e2e", "stage")):
    """The plain form: one StereoMapper, one depth map after the other (device-resident frames for
    `dev` and the stage times, pinned host frames for `e2e`)."""
    import torch
    from probabilistic_mapping_b200 import scene
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    seq = scene.make_sequence(W, H, F_PX, S, N_KEYFRAMES, seed=1000 + rank)
    K = seq[0].K
    fx, fy, cx, cy = K[0, 0], K[1, 1], K[0, 2], K[1, 2]
    prec = 1 if precision == "fp16" else 0
    m, drho = make_mapper(prec, dev, 1 if args.cost_mode == "corrected" else 0, SAMPLERS[sampler_name(args, prec)])
    m.initIntrinsic(K, 0.0, drho)
    stream = torch.cuda.Stream(device=dev)
    m.set_stream(stream.cuda_stream)

    # device-resident inputs
    d_ref = [torch.from_numpy(fs.ref).cuda() for fs in seq]
    d_src = [[torch.from_numpy(np.ascontiguousarray(fs.srcs[s])).cuda() for s in range(S)] for fs in seq]
    d_depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
    d_var = torch.empty((H, W), dtype=torch.float32, device="cuda")
    # pinned host buffers for the end-to-end run
    h_ref = [torch.from_numpy(fs.ref).pin_memory() for fs in seq]
    h_src = [[torch.from_numpy(np.ascontiguousarray(fs.srcs[s])).pin_memory() for s in range(S)] for fs in seq]
    h_depth = torch.empty((H, W), dtype=torch.float32).pin_memory()
    h_var = torch.empty((H, W), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()

    def step(i, ref, src, dep, var):
        fs = seq[i % N_KEYFRAMES]
        k = i % N_KEYFRAMES
        m.initReference(ref[k])
        for s in range(S):
            m.update(src[k][s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        m.outputFusion(fs.R_ref, fs.T_ref, fx, fy, cx, cy, out=dep, variance=var)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(ref, src, dep, var, stage_timing=False):
        for i in range(args.warmup):
            step(i, ref, src, dep, var)
        m.enable_stage_timing(stage_timing)
        stage = np.zeros(5)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            step(args.warmup + i, ref, src, dep, var)
            if stage_timing:
                stage += m.stage_times()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        m.enable_stage_timing(False)
        return e0.elapsed_time(e1), stage / args.steps

    t_dev = t_e2e = 0.0
    stage_ms = np.zeros(5)
    clk = ClockSampler(dev)
    if "dev" in passes:
        with clk:
            t_dev, _ = timed(d_ref, d_src, d_depth, d_var)
    if "e2e" in passes:
        t_e2e, _ = timed(h_ref, h_src, h_depth, h_var)
    if "stage" in passes:
        # per-stage CUDA-event times (separate pass; the stage events synchronise every step)
        _, stage_ms = timed(d_ref, d_src, d_depth, d_var, stage_timing=True)
    t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], world)
    m.close()
    return t_dev, t_e2e, stage_ms, clk.summary() if "dev" in passes else None


def max_over_ranks(vals, world):
    """Element-wise maximum of the ranks' values (device tensors over nccl, host over gloo)."""
    if world <= 1:
        return vals
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def run_batched(args, rank, world, precision: str, B: int, host_io: bool, clocks: bool, persistent: bool = False):
    """B sequences of the bench workload in one pm_batch: each step is one CUDA-graph launch that
    maps every sequence.  The two frame sets of the batch hold keyframes 0 and 1 of each
    sequence (device memory, or pinned host memory copied inside the graph with host_io); the
    steps alternate between them with the matching poses."""
    import torch
    from probabilistic_mapping_b200 import _lib, scene
    from probabilistic_mapping_b200.batch import StereoBatch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    rho0, drho = scene.plane_range(D)
    prec = _lib.PM_PREC_FP16 if precision == "fp16" else _lib.PM_PREC_FP32
    cfg = dict(width=W, height=H, num_planes=D, rho0=rho0, intensity_scale=1 / 255, num_paths=PATHS, p1=P1, p2=P2,
               tau_so=TAU, uniqueness_ratio=UNIQ, cost_mode=1 if args.cost_mode == "corrected" else 0,
               precision=prec, device=dev, sampler=SAMPLERS[sampler_name(args, prec)])
    seqs = [scene.make_sequence(W, H, F_PX, S, 2, seed=2000 + 97 * rank + i) for i in range(B)]
    b = StereoBatch([cfg] * B, S, lanes=0, host_io=host_io, autotune=not persistent, priority=args.priority,
                    persistent=persistent)
    for i in range(B):
        b.init_intrinsic(i, seqs[i][0].K, drho)

    def feed(step):
        k = step % 2
        for i in range(B):
            fs = seqs[i][k]
            if step < 2:   # frames stay in the batch's buffer set k after the first two steps
                b.set_frame(i, 0, fs.ref)
                for s in range(S):
                    b.set_frame(i, 1 + s, fs.srcs[s])
            b.set_poses(i, fs.R_ref, fs.T_ref, list(fs.R_srcs), list(fs.T_srcs))

    for i in range(args.warmup):
        feed(i)
        b.run()
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(dev) if clocks else None
    if sampler:
        sampler.__enter__()
    e0.record(stream)
    for i in range(args.steps):
        feed(args.warmup + i)
        b.run()
    e1.record(stream)
    b.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    t = e0.elapsed_time(e1)
    tuning = None if persistent else b.tuning(0)
    b.close()
    t = max_over_ranks([t], world)[0]
    return t, (sampler.summary() if sampler else None), tuning


# The mixed batch: 48 sequences, 16 at each size, 4 sources (the batching form's workload).
MIXED = [(320, 240, 64, 260.0), (640, 480, 128, 520.0), (1280, 720, 192, 1040.0)]
MIXED_PER_SHAPE, MIXED_S = 16, 4


def run_mixed(args, rank, world, precision: str, host_io: bool, clocks: bool, persistent: bool = False):
    """This rank's shard (balanced by voxels x sources) of the 48-sequence mixed batch in one
    pm_batch; each step is one CUDA-graph launch that maps every sequence of the shard.  Two
    seeded scenes per size are shared by that size's sequences (the inputs only need the size)."""
    import torch
    from probabilistic_mapping_b200 import _lib, scene
    from probabilistic_mapping_b200.batch import StereoBatch
    from probabilistic_mapping_b200.shard import shard_sequences
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    prec = _lib.PM_PREC_FP16 if precision == "fp16" else _lib.PM_PREC_FP32
    cfgs, shapes = [], []
    for k, (w, h, d, f) in enumerate(MIXED):
        rho0, _ = scene.plane_range(d)
        for _ in range(MIXED_PER_SHAPE):
            cfgs.append(dict(width=w, height=h, num_planes=d, rho0=rho0, intensity_scale=1 / 255, num_paths=PATHS,
                             p1=P1, p2=P2, tau_so=TAU, uniqueness_ratio=UNIQ,
                             cost_mode=1 if args.cost_mode == "corrected" else 0, precision=prec, device=dev,
                             sampler=SAMPLERS[sampler_name(args, prec)]))
            shapes.append(k)
    mine = shard_sequences(cfgs, world, MIXED_S)[rank]
    scenes = {k: [scene.make_sequence(w, h, f, MIXED_S, 2, seed=3000 + 10 * k + j) for j in range(2)]
              for k, (w, h, d, f) in enumerate(MIXED) if any(shapes[i] == k for i in mine)}
    b = StereoBatch([cfgs[i] for i in mine], MIXED_S, lanes=0 if persistent else args.lanes, host_io=host_io,
                    autotune=not persistent, priority=args.priority, persistent=persistent)
    seqs = []
    for j, i in enumerate(mine):
        seqs.append(scenes[shapes[i]][i % 2])
        b.init_intrinsic(j, seqs[-1][0].K, scene.plane_range(MIXED[shapes[i]][2])[1])

    def feed(step):
        k = step % 2
        for j, sq in enumerate(seqs):
            fs = sq[k]
            if step < 2:
                b.set_frame(j, 0, fs.ref)
                for s in range(MIXED_S):
                    b.set_frame(j, 1 + s, fs.srcs[s])
            b.set_poses(j, fs.R_ref, fs.T_ref, list(fs.R_srcs), list(fs.T_srcs))

    for i in range(args.warmup):
        feed(i)
        b.run()
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(dev) if clocks else None
    if sampler:
        sampler.__enter__()
    e0.record(stream)
    for i in range(args.steps):
        feed(args.warmup + i)
        b.run()
    e1.record(stream)
    b.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    t = e0.elapsed_time(e1)
    b.close()
    t = max_over_ranks([t], world)[0]
    h2d = sum(cfgs[i]["width"] * cfgs[i]["height"] * (MIXED_S + 1) for i in mine)
    d2h = sum(cfgs[i]["width"] * cfgs[i]["height"] * 8 for i in mine)
    return t, (sampler.summary() if sampler else None), len(mine), h2d, d2h


def run_mixed_plain_fp32(args, rank, world):
    """The plain FP32 form run per sequence over this rank's shard of the mixed batch: one
    StereoMapper per size, each sequence's keyframe mapped after the other (initReference, the
    updates, outputFusion), device-resident frames; ms per step of all the shard's sequences."""
    import torch
    from probabilistic_mapping_b200 import scene
    from probabilistic_mapping_b200.mapper import StereoMapper
    from probabilistic_mapping_b200.shard import shard_sequences
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    cfgs, shapes = [], []
    for k, (w, h, d, f) in enumerate(MIXED):
        for _ in range(MIXED_PER_SHAPE):
            cfgs.append(dict(width=w, height=h, num_planes=d))
            shapes.append(k)
    mine = shard_sequences(cfgs, world, MIXED_S)[rank]
    stream = torch.cuda.Stream(device=dev)   # every mapper on it, so that its events bracket the work
    mappers, frames = {}, {}
    for k, (w, h, d, f) in enumerate(MIXED):
        if not any(shapes[i] == k for i in mine):
            continue
        rho0, drho = scene.plane_range(d)
        m = StereoMapper(w, h, d, rho0=rho0, intensity_scale=1 / 255, num_paths=PATHS, p1=P1, p2=P2, tau_so=TAU,
                         uniqueness_ratio=UNIQ, precision=0, device=dev)
        seq = [scene.make_sequence(w, h, f, MIXED_S, 2, seed=3000 + 10 * k + j) for j in range(2)]
        m.initIntrinsic(seq[0][0].K, 0.0, drho)
        m.set_stream(stream.cuda_stream)
        mappers[k] = m
        frames[k] = [[(torch.from_numpy(fs.ref).cuda(), [torch.from_numpy(np.ascontiguousarray(x)).cuda()
                                                         for x in fs.srcs], fs) for fs in sq] for sq in seq]
    outs = {k: torch.empty((MIXED[k][1], MIXED[k][0]), dtype=torch.float32, device="cuda") for k in mappers}

    def step(t):
        for i in mine:
            k = shapes[i]
            ref, srcs, fs = frames[k][i % 2][t % 2]
            m = mappers[k]
            m.initReference(ref)
            for s in range(MIXED_S):
                m.update(srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            K = fs.K
            m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2], out=outs[k], want_variance=False)

    for t in range(args.warmup):
        step(t)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for t in range(args.steps):
        step(args.warmup + t)
    e1.record(stream)
    torch.cuda.synchronize()
    for m in mappers.values():
        m.close()
    return max_over_ranks([e0.elapsed_time(e1)], world)[0]


def mixed_measure(args, rank, world):
    """The mixed batch in both batched modes (graph and persistent) and the plain FP32 form per
    sequence; returns (best mode name, per-mode results, plain FP32 ms, shard size, h2d, d2h)."""
    precision = args.precision or "fp16"
    total = len(MIXED) * MIXED_PER_SHAPE
    res = {}
    for mode in args.batch_modes:
        persistent = mode == "persistent"
        t, clocks, n_mine, _, _ = run_mixed(args, rank, world, precision, host_io=False, clocks=True,
                                            persistent=persistent)
        te, _, _, h2d, d2h = run_mixed(args, rank, world, precision, host_io=True, clocks=False,
                                       persistent=persistent)
        res[mode] = {"value": total * args.steps / (t / 1000.0), "e2e": total * args.steps / (te / 1000.0),
                     "ms_per_step": t / args.steps, "clocks": clocks}
    best = max(res, key=lambda k: res[k]["value"])
    t_plain = run_mixed_plain_fp32(args, rank, world)
    return best, res, t_plain, n_mine, h2d, d2h


def mixed_main(args, rank, world):
    precision = args.precision or "fp16"
    best, res, t_plain, n_mine, h2d, d2h = mixed_measure(args, rank, world)
    total = len(MIXED) * MIXED_PER_SHAPE
    if rank == 0:
        vox = sum(w * h * d for w, h, d, _ in MIXED) * MIXED_PER_SHAPE
        r = res[best]
        line = {"metric": "depth maps/s, 48-sequence mixed batch (16 each at 320x240x64, 640x480x128, "
                          "1280x720x192), 4 sources", "value": r["value"], "unit": "depth maps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f16" if precision == "fp16" else "f32", "data": "synthetic",
                "config": {"workload": f"48 sequences, {MIXED_S} sources, {PATHS}-path SGM, fusion step, "
                                       f"{precision} {sampler_name(args, precision)} sampler, {best} batch",
                           "global_batch": total, "seq_len": 0,
                           "parallelism": f"sequence shards x{world}, balanced by voxels x sources",
                           "l2": "per-map working sets exceed the 126 MB L2"},
                "voxels_per_s": vox * args.steps / (r["ms_per_step"] * args.steps / 1000.0),
                "batch_modes": {k: {kk: vv for kk, vv in v.items() if kk != "clocks"} for k, v in res.items()},
                "plain_fp32_per_sequence": {"value": total * args.steps / (t_plain / 1000.0),
                                            "unit": "depth maps/s", "ms_per_step": t_plain / args.steps},
                "speedup_vs_plain_fp32_per_sequence": r["value"] / (total * args.steps / (t_plain / 1000.0)),
                "sequences_on_rank0": n_mine,
                "e2e": {"value": r["e2e"], "unit": "depth maps/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "note": "rank 0's shard bytes"},
                "clocks": r["clocks"]}
        print(json.dumps(line))


# The configuration the reference's own CUDA is compiled for (parameters.h: 640x480, 64 planes;
# sgm2's 4 paths; parameters.cpp's penalties on 0..255 intensities; DEP_SAMPLE with plane 0 at
# infinity), 5 sources, cost + SGM + winner-take-all (stereo_mapper.cpp:63-109), no fusion.
REF_CFG = dict(W=640, H=480, D=64, S=5, f=520.0, seed=99)
REF_CFG_NAME = ("640x480, 64 planes, 5 sources, 4-path SGM, reference parameters (pi1 8, pi2 24, tau_so 4, "
                "q1 2, q2 3) on 0..255 intensities, plane 0 at inverse depth 0; initReference + 5 updates + "
                "output (cost, SGM, winner-take-all), device-resident inputs")


def ref_cfg_frames():
    from probabilistic_mapping_b200 import scene
    c = REF_CFG
    return scene.make_frameset(c["W"], c["H"], c["f"], c["S"], seed=c["seed"]), 2.0 / (c["D"] - 1)


def run_matched_reference_config(args, sampler: str):
    """This library's plain FP32 form at the reference CUDA's own configuration (REF_CFG): ms per
    depth map by CUDA events over args.steps maps after args.warmup, inputs resident on the device."""
    import torch
    from probabilistic_mapping_b200.mapper import StereoMapper
    c = REF_CFG
    fs, dep_sample = ref_cfg_frames()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    m = StereoMapper(c["W"], c["H"], c["D"], rho0=0.0, intensity_scale=1.0, num_paths=4, p1=8.0, p2=24.0,
                     tau_so=4.0, q1=2.0, q2=3.0, uniqueness_ratio=0.0, cost_mode=0, precision=0, device=dev,
                     sampler=SAMPLERS[sampler])
    m.initIntrinsic(fs.K, 0.0, dep_sample)
    stream = torch.cuda.Stream(device=dev)
    m.set_stream(stream.cuda_stream)
    d_ref = torch.from_numpy(fs.ref).cuda()
    d_src = [torch.from_numpy(np.ascontiguousarray(fs.srcs[s])).cuda() for s in range(c["S"])]
    out = torch.empty((c["H"], c["W"]), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    def one():
        m.initReference(d_ref)
        for s in range(c["S"]):
            m.update(d_src[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        m.output(out)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    m.close()
    return e0.elapsed_time(e1) / args.steps


def reference_cuda_sample(reps: int):
    """The reference's own CUDA (calc_cost.cu, sgm.cu, filter_cost.cu built unmodified for sm_100a
    through a texture-object shim into oracle/_ref/libref_640x480x64.so) on REF_CFG: ms per depth
    map (CUDA events inside the library), or None with the reason."""
    import ctypes
    try:
        import torch
        if not torch.cuda.is_available():
            return None, "no CUDA device"
    except Exception as ex:   # noqa: BLE001
        return None, f"torch unavailable: {ex}"
    path = os.path.join(ROOT, "oracle", "_ref", "libref_640x480x64.so")
    if not os.path.exists(path):
        return None, "oracle/_ref/libref_640x480x64.so was not built (the reference sources were absent at build time)"
    import oracle
    lib = ctypes.CDLL(path)
    lib.ref_set_params(ctypes.c_float(8.0), ctypes.c_float(24.0), ctypes.c_float(4.0), ctypes.c_float(2.0),
                       ctypes.c_float(3.0), ctypes.c_float(1.02))
    fs, dep_sample = ref_cfg_frames()
    ref = np.ascontiguousarray(fs.ref.astype(np.float32))
    srcs = np.ascontiguousarray(fs.srcs.astype(np.float32))
    homs = np.ascontiguousarray(np.stack([oracle.compose_homography(fs.K, fs.R_ref, fs.T_ref, fs.R_srcs[s],
                                                                     fs.T_srcs[s]) for s in range(REF_CFG["S"])]
                                         ).astype(np.float32))
    ms = np.zeros(1, np.float32)
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))   # noqa: E731
    st = lib.ref_bench(P(ref), P(srcs), REF_CFG["S"], P(homs), ctypes.c_float(dep_sample), int(reps), P(ms))
    if st != 0:
        return None, f"ref_bench returned CUDA error {st}"
    return float(ms[0]), None


def cpu_baseline_sample(threads: int | None = None, maps: int = 1):
    """FP64 oracle (all host threads) on full-size depth maps of the same workload."""
    import oracle
    from probabilistic_mapping_b200 import scene
    oracle.build()
    if threads:
        oracle.set_threads(threads)
    seq = scene.make_sequence(W, H, F_PX, S, 2, seed=99)
    rho0, drho = scene.plane_range(D)
    p = oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, cost_mode=0,
                      num_paths=PATHS, p1=P1, p2=P2, tau_so=TAU, uniqueness=UNIQ)
    K = seq[0].K
    o = oracle.Mapper(p, K)

    def one(i):
        fs = seq[i % 2]
        o.init_reference(fs.ref)
        for s in range(S):
            o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        o.output_fusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])

    one(0)   # first keyframe initialises the fusion state
    t0 = time.perf_counter()
    for i in range(maps):
        one(1 + i)
    dt = time.perf_counter() - t0
    return maps / dt, oracle.num_threads()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["batched", "plain", "mixed"], default="batched",
                    help="batched: B sequences of the headline workload; plain: one map after the other; "
                         "mixed: the 48-sequence three-size batch, sharded over ranks")
    ap.add_argument("--lanes", type=int, default=0, help="volume sets per size in the mixed batch (0: one each)")
    ap.add_argument("--sampler", choices=list(SAMPLERS), default="texture_f32",
                    help="FP16 form: source sampling (exact FP32 bilinear, or the texture unit from FP16 / FP32 texels)")
    ap.add_argument("--fp32-sampler", choices=["exact", "texture_f32"], default="exact",
                    help="FP32 form: exact FP32 bilinear (bit-exact against the FP32 oracle) or the texture "
                         "unit on FP32 texels (the reference's own sampler)")
    ap.add_argument("--batch-mode", choices=["graph", "persistent", "best"], default="best",
                    help="batched forms: per-sequence kernels in one CUDA graph, the persistent kernel "
                         "(PM_BATCH_PERSISTENT), or both with the faster as the headline")
    ap.add_argument("--no-mixed", action="store_true",
                    help="batched form: skip the 48-sequence mixed batch reported beside the headline")
    ap.add_argument("--priority", type=int, default=1, choices=[0, 1],
                    help="batched forms: SGM kernels at the greatest launch priority (1) or not (0)")
    ap.add_argument("--precision", choices=["fp32", "fp16"], default=None,
                    help="precision of the measured form (default: fp16 batched, fp32 plain)")
    # 32 sequences per step: the device rate is the same as at 16 (902 against 902 maps/s), but
    # the copies at either end of a step that cannot overlap compute are spread over twice the
    # maps (e2e 897 against 872 maps/s)
    ap.add_argument("--batch", type=int, default=32, help="sequences per batch (batched form)")
    ap.add_argument("--cost-mode", choices=["reference", "corrected"], default="reference")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-matched", action="store_true",
                    help="skip the plain FP32 form at the reference CUDA's own configuration")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    args.batch_modes = ["graph", "persistent"] if args.batch_mode == "best" else [args.batch_mode]

    if args.impl == "reference":
        # The reference implements this path only in CUDA (its host code adds the CPU fusion
        # variant alone), so its CPU arm is the FP64 port of that CUDA, on all host cores.
        if rank != 0:
            return
        warm = max(0, min(args.warmup, 1))
        if warm:
            cpu_baseline_sample(maps=1)
        rate, cores = cpu_baseline_sample(maps=args.steps)
        line = {"metric": METRIC, "value": rate, "unit": "depth maps/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 / rate, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": f"{W}x{H}, {D} planes, {S} sources, {PATHS}-path SGM, fusion step",
                           "global_batch": 1, "seq_len": 0, "parallelism": "cpu"},
                "cpu_baseline": {"value": rate, "unit": "depth maps/s", "cores": cores, "kind": "port",
                                 "sample": f"{args.steps} full {W}x{H}x{D} depth maps (FP64 oracle, OpenMP)"},
                "e2e": {"value": rate, "unit": "depth maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        # the reference's own CUDA on this GPU, at the configuration it is compiled for; this
        # library's plain FP32 form at the same configuration is in the other arm's line
        # ("matched_reference_config")
        ms, why = reference_cuda_sample(max(args.steps, 1))
        line["reference_cuda"] = ({"ms_per_map": ms, "maps_per_s": 1000.0 / ms, "config": REF_CFG_NAME,
                                   "source": "oracle/_ref/libref_640x480x64.so: the reference's calc_cost.cu, "
                                             "sgm.cu and filter_cost.cu compiled unmodified for sm_100a through "
                                             "a texture-object shim (texture references were removed in CUDA 12)"}
                                  if ms else {"unavailable": why})
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    if args.form == "mixed":
        mixed_main(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.precision is None:
        args.precision = "fp16" if args.form == "batched" else "fp32"
    # the plain FP32 form, always measured: the baseline of the batched form's speed-up and the
    # source of the per-kernel stage times
    t_plain, t_plain_e2e, stage_ms, clocks_plain = run_ours(args, rank, world, "fp32")
    plain_value = world * args.steps / (t_plain / 1000.0)
    plain_e2e = world * args.steps / (t_plain_e2e / 1000.0)
    batch_modes = None
    if args.form == "batched":
        B = args.batch
        batch_modes = {}
        for mode in args.batch_modes:
            persistent = mode == "persistent"
            t_b, clocks_b, tuning_b = run_batched(args, rank, world, args.precision, B, host_io=False, clocks=True,
                                                  persistent=persistent)
            t_be, _, _ = run_batched(args, rank, world, args.precision, B, host_io=True, clocks=False,
                                     persistent=persistent)
            batch_modes[mode] = {"value": world * B * args.steps / (t_b / 1000.0),
                                 "e2e": world * B * args.steps / (t_be / 1000.0), "ms_per_step": t_b / args.steps,
                                 "clocks": clocks_b, "tuning": tuning_b}
        best = max(batch_modes, key=lambda k: batch_modes[k]["value"])
        value, e2e = batch_modes[best]["value"], batch_modes[best]["e2e"]
        ms_per_step, clocks, tuning = (batch_modes[best]["ms_per_step"], batch_modes[best]["clocks"],
                                       batch_modes["graph"]["tuning"] if "graph" in batch_modes else None)
        if args.precision == "fp16":   # stage times of the FP16 form's kernels (plain mapper)
            _, _, stage_ms, _ = run_ours(args, rank, world, "fp16", passes=("stage",))
    else:
        B = 1
        tuning = None
        if args.precision == "fp32":
            t_dev, t_e2e, clocks = t_plain, t_plain_e2e, clocks_plain
        else:
            t_dev, t_e2e, stage_ms, clocks = run_ours(args, rank, world, args.precision)
        value = world * args.steps / (t_dev / 1000.0)
        e2e = world * args.steps / (t_e2e / 1000.0)
        ms_per_step = t_dev / args.steps
    e = 2 if args.precision == "fp16" else 4
    b_alg, sgm_bytes = algorithmic_bytes(e)
    b_sgm_alg = sgm_alg_bytes(e)
    peak_hbm, sm_mhz, peak_kind = peaks()
    peak_fp32 = fp32_peak_tflops(sm_mhz)
    cost_stage_ms, sgm_ms, fuse_ms = float(stage_ms[0]), float(stage_ms[1]), float(stage_ms[2])
    cost_ms = float(stage_ms[4]) if stage_ms[4] > 0 else cost_stage_ms   # the cost kernel alone
    texels = sampler_name(args, args.precision) != "exact"
    simt_flop, tex_flop, _ = cost_kernel_work(e, texels)
    sgm_gbs = sgm_bytes / (sgm_ms / 1000.0) / 1e9 if sgm_ms > 0 else None
    sgm_alg_gbs = b_sgm_alg / ((sgm_ms + fuse_ms) / 1000.0) / 1e9 if sgm_ms > 0 else None
    map_s = 1.0 / (value / world)   # seconds per map per GPU
    # to_float (reference) + one conversion per source, cost (+ the FP16 volume's rebase), one
    # kernel per opposite-path pair, combine + winner-take-all, fusion transform + update
    launches_per_map = 1 + S + 1 + (1 if e == 2 else 0) + PATHS // 2 + 1 + 2
    mixed = None
    if args.form == "batched" and not args.no_mixed:
        best_m, res_m, t_plain_m, _, _, _ = mixed_measure(args, rank, world)
        total_m = len(MIXED) * MIXED_PER_SHAPE
        plain_m = total_m * args.steps / (t_plain_m / 1000.0)
        mixed = {"workload": "48 sequences (16 each at 320x240x64, 640x480x128, 1280x720x192), 4 sources, "
                             f"{PATHS}-path SGM, fusion step, {args.precision} {sampler_name(args, args.precision)} "
                             "sampler", "unit": "depth maps/s", "best_mode": best_m,
                 "batch_modes": {k: {kk: vv for kk, vv in v.items() if kk != "clocks"} for k, v in res_m.items()},
                 "plain_fp32_per_sequence": plain_m,
                 "speedup_vs_plain_fp32_per_sequence": res_m[best_m]["value"] / plain_m}
    matched = None
    if rank == 0 and not args.no_matched:
        matched = {"config": REF_CFG_NAME,
                   "ms_per_map_fp32_exact": run_matched_reference_config(args, "exact"),
                   "ms_per_map_fp32_texture_f32": run_matched_reference_config(args, "texture_f32"),
                   "note": "the reference's own CUDA at this configuration is timed by the reference arm "
                           "(bench.py --impl reference, key reference_cuda)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "depth maps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if e == 4 else "f16", "data": "synthetic",
            "config": {"workload": f"{W}x{H}, {D} planes, {S} sources, {PATHS}-path SGM, uniqueness {UNIQ}, "
                                   f"fusion step; {args.precision} {args.form} form"
                                   + (f", {B} sequences per CUDA-graph launch ({best} batch)"
                                      if args.form == "batched" else "")
                                   + f", {sampler_name(args, args.precision)} sampler"
                                   + f", {args.cost_mode} cost samples",
                       "global_batch": world * B, "seq_len": 0, "parallelism": f"replicas x{world}",
                       "l2": "per-map working set (cost + path volumes, >1 GB) exceeds the 126 MB L2"},
            "plain_fp32": {"value": plain_value, "e2e": plain_e2e, "ms_per_map": t_plain / args.steps,
                           "unit": "depth maps/s"},
            "speedup_vs_plain_fp32": value / plain_value,
            # the dominant kernel (cost_kernel, more than half of a map), against the roof that binds it
            "roofline": cost_roofline(cost_ms, cost_stage_ms, e, texels, args.cost_mode != "corrected", sm_mhz,
                                      peak_hbm, peak_kind, args.precision,
                                      ncu_traffic("cost_kernel" if e == 4 and args.fp32_sampler == "exact"
                                                  else "cost_kernel_fp16" if e == 2 else None)),
            # the SGM stage against the bytes this implementation moves, and the SGM + winner-take-
            # all + fusion stages against their share of the path-grouped lower bound B_alg
            "roofline_sgm": {"bound": "hbm", "kernel": "sgm_pair_kernel x 4 + combine_kernel (winner-take-all)",
                             "achieved": sgm_gbs, "peak": peak_hbm, "unit": "GB/s",
                             "frac": (sgm_gbs / peak_hbm) if sgm_gbs else None,
                             "implementation_bytes_per_map": sgm_bytes, "ms": sgm_ms, "peak_kind": peak_kind,
                             "b_alg_share_bytes": b_sgm_alg, "b_alg_share_ms": sgm_ms + fuse_ms,
                             "b_alg_share_achieved_gbs": sgm_alg_gbs,
                             "b_alg_share_frac": (sgm_alg_gbs / peak_hbm) if sgm_alg_gbs else None,
                             "implementation_over_algorithmic_bytes": sgm_bytes / (b_sgm_alg - 60 * W * H)},
            "map_roofline": {"b_alg_bytes": b_alg, "f_alg_flop": simt_flop + tex_flop,
                             "ms_per_map_per_gpu": map_s * 1000,
                             "frac_of_hbm": b_alg / map_s / 1e9 / peak_hbm,
                             "frac_of_fp32": (simt_flop + tex_flop) / map_s / 1e12 / peak_fp32},
            "stage_ms": {"cost": cost_stage_ms, "cost_kernel": cost_ms, "sgm_wta": sgm_ms, "fusion": fuse_ms,
                         "copy_out": float(stage_ms[3]), "source": f"plain {args.precision} mapper, CUDA events"},
            "e2e": {"value": e2e, "unit": "depth maps/s", "h2d_bytes_per_step": B * (S + 1) * W * H,
                    "d2h_bytes_per_step": B * 2 * 4 * W * H},
            # the persistent batch: per sequence the conversions and the two fusion kernels, plus one
            # persistent kernel per step for all sequences
            "gpu_launches": ((1 + S + 2) * B + 1) * args.steps if batch_modes and best == "persistent"
            else launches_per_map * B * args.steps,
            "clocks": clocks,
        }
        if matched:
            line["matched_reference_config"] = matched
        if tuning:
            line["sgm_schedule"] = {"pair_warps": tuning[0], "serial_pairs": tuning[1], "tuned_ms": tuning[2]}
        if batch_modes:
            line["batch_modes"] = {k: {kk: vv for kk, vv in v.items() if kk not in ("clocks", "tuning")}
                                   for k, v in batch_modes.items()}
        if mixed:
            line["mixed_batch"] = mixed
        if not args.no_cpu_baseline:
            rate, cores = cpu_baseline_sample(maps=3)
            line["cpu_baseline"] = {"value": rate, "unit": "depth maps/s", "cores": cores, "kind": "port",
                                    "sample": f"3 full {W}x{H}x{D} depth maps, FP64 oracle with OpenMP"}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
