"""Template-matching benchmark: match-score Gtaps/s on one B200 (or N).

Workload (one step): the five ImageProximity measures (SqrDistance,
SqrDistance_Norm, AbsDistance, CrossCorr, CrossCorr_Norm) of a 4096x4096
single-channel F32 image against a 31x31 F32 template cut from it. The
image is a seeded sum of 200 isotropic Gaussian blobs (sigma uniform in
4-40 px, amplitude uniform in 0-1) plus uniform noise in [0, 0.05]; the
template is cut at a seeded offset. Taps are counted over the valid region
((W-tw+1) x (H-th+1) x tw x th per measure); each call computes the full
same-size map as the drop-in does.

Timing: inputs resident on the device, the L2 flushed (256 MiB write, not
timed) before every step, each step timed with CUDA events on the library's
stream, K steps after W warm-up steps, max over ranks. `e2e` times the same
step through the C ABI with host buffers in pinned memory: the source is
sent each step and the five score maps read back.

Ranks (torchrun, N>1): every rank runs its own copy of the workload on its
own GPU (independent images; no collective on the data path), so the job's
throughput is the sum of the ranks' taps over the slowest rank's time
("scaling": "weak").

--impl reference times the reference's own kernel source
(cl-files/ImageProximity.cl, compiled for the host, oracle/_ref) on the host
cores on a band of rows of the same workload.

Other workloads (--workload): batch (16 x 2048^2 U8 images x 64 uneven
templates in persistent launches), backward (gradients vs forward time on 32 x
1024^2 F32), integral (4096^2 F32 -> F64 Integral + SqrIntegral, GB/s against
the HBM peak) and sad (4096^2 U8 AbsDistance on packed-byte SAD).
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_IMG, H_IMG, T_SIDE = 4096, 4096, 31
MEASURES = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]
METRIC = "match-score Gtaps/s, tensor vs plain FP32 on one B200, <=1e-5 rel err vs FP64"


def blob_field(W, H, nblobs=200, seed=0):
    """Seeded sum of isotropic Gaussian blobs plus uniform noise (float32)."""
    rng = np.random.default_rng(seed)
    img = np.zeros((H, W), np.float64)
    xs = rng.uniform(0, W, nblobs)
    ys = rng.uniform(0, H, nblobs)
    sig = rng.uniform(4, 40, nblobs)
    amp = rng.uniform(0, 1, nblobs)
    for x, y, s, a in zip(xs, ys, sig, amp):
        r = int(np.ceil(5 * s))
        x0, x1 = max(0, int(x) - r), min(W, int(x) + r + 1)
        y0, y1 = max(0, int(y) - r), min(H, int(y) + r + 1)
        gx = np.exp(-0.5 * ((np.arange(x0, x1) - x) / s) ** 2)
        gy = np.exp(-0.5 * ((np.arange(y0, y1) - y) / s) ** 2)
        img[y0:y1, x0:x1] += a * np.outer(gy, gx)
    img += rng.uniform(0, 0.05, (H, W))
    return img.astype(np.float32)


def workload(seed=0, with_offset=False):
    """The 4096x4096 F32 blob field and the 31x31 template cut from it at a
    seeded offset (ty, tx); the exact match is output (tx + 15, ty + 15)."""
    S = blob_field(W_IMG, H_IMG, seed=seed)
    rng = np.random.default_rng(seed + 1)
    ty = int(rng.integers(0, H_IMG - T_SIDE))
    tx = int(rng.integers(0, W_IMG - T_SIDE))
    T = S[ty:ty + T_SIDE, tx:tx + T_SIDE].copy()
    return (S, T, (ty, tx)) if with_offset else (S, T)


def cfg1_images(seed=1):
    """512x512 U8 uniform 0-255, 16x16 template cut at a seeded offset plus
    round(N(0, 4^2)) noise, clipped to 0-255."""
    rng = np.random.default_rng(seed)
    S = rng.integers(0, 256, (512, 512), dtype=np.uint8)
    y, x = (int(v) for v in rng.integers(0, 512 - 16, 2))
    T = np.clip(S[y:y + 16, x:x + 16].astype(np.int32) + np.round(rng.normal(0, 4, (16, 16))),
                0, 255).astype(np.uint8)
    return S, T


def cfg5_images(dtype, seed=55):
    """3840x2160x4 multi-channel field: uniform noise plus a blob field (U8),
    or the blob field scaled to 0-65535 (U16); a 64x64x4 template cut at a
    seeded offset. Returns (S, T, (y, x))."""
    rng = np.random.default_rng(seed)
    field = np.stack([blob_field(3840, 2160, nblobs=60, seed=seed + 5 + c) for c in range(4)], -1)
    field = field / field.max()
    if dtype == np.uint8:
        S = np.clip(rng.integers(0, 128, field.shape) + 127 * field, 0, 255).astype(np.uint8)
    else:
        S = np.round(field * 65535).astype(np.uint16)
    y, x = 700, 1900
    return S, S[y:y + 64, x:x + 64].copy(), (y, x)


# ---- accuracy against the FP64 / exact oracle ----------------------------------------

def check_rows(H, th, n=256, match_row=None):
    """n output rows spread over the valid region, the first and last rows of
    the map, and the th rows around the match row (if given)."""
    rows = set(np.linspace(th // 2, H - th + th // 2, n).astype(int).tolist())
    rows |= {0, 1, H - 2, H - 1}
    if match_row is not None:
        rows |= set(range(max(0, match_row - th // 2), min(H, match_row + th // 2 + 1)))
    return sorted(rows)


def window_energy_rows(S, tw, th, rows):
    """Sum of S^2 over each output's window (zero padding), FP64, for the
    listed output rows: array (len(rows), W[, C])."""
    sq = S.astype(np.float64) ** 2
    H, W = S.shape[:2]
    ax, ay = tw // 2, th // 2
    pad = [(th, th), (tw, tw)] + ([(0, 0)] if S.ndim == 3 else [])
    ii = np.pad(sq, pad).cumsum(0).cumsum(1)  # ii[i, j] = sum over [0, i] x [0, j] of padded
    out = []
    xs = np.arange(W)
    for y in rows:
        # window rows y - ay .. y - ay + th - 1, columns x - ax .. x - ax + tw - 1
        r0, r1 = y - ay + th - 1, y - ay + 2 * th - 1  # padded index of the row before / last row
        c0, c1 = xs - ax + tw - 1, xs - ax + 2 * tw - 1
        out.append(ii[r1, c1] - ii[r0, c1] - ii[r1, c0] + ii[r0, c0])
    return np.array(out)


def scale_rows(measure, S, T, rows):
    """The scale each measure's error is stated against, per output:
    SqrDistance: sum S^2 + sum T^2 of the window (the terms that cancel to 0
    at a match); CrossCorr: sum |S| |T| (equal to the value for non-negative
    data; the bound of a dot product's rounding for signed data); the _Norm
    forms divide these by sqrt(sum S^2 sum T^2); AbsDistance: its value."""
    from oracle import oracle as O
    th, tw = T.shape[:2]
    es = window_energy_rows(S, tw, th, rows)
    t64 = T.astype(np.float64)
    et = (t64 ** 2).sum(axis=(0, 1))
    if measure in (0, 1):
        sc = es + et
    elif measure in (3, 4):
        sc = O.proximity_exact_rows(3, np.abs(S.astype(np.float64)), np.abs(t64), rows)
    else:
        return np.abs(O.proximity_exact_rows(2, S, T, rows))
    if measure in (1, 4):
        with np.errstate(divide="ignore", invalid="ignore"):
            sc = sc / np.sqrt(es * et)
    return sc


def error_rows(measure, S, T, got, rows, ex=None):
    """Errors of a computed map on the listed rows against the exact oracle:
    max_abs, max_rel (per output, against |exact|), max_scaled (against the
    measure's scale, scale_rows) and the share of outputs whose per-output
    relative error is within 1e-5."""
    from oracle import oracle as O
    if ex is None:
        ex = O.proximity_exact_rows(measure, S, T, rows)
    g = got[rows].astype(np.float64)
    sc = scale_rows(measure, S, T, rows)
    fin = np.isfinite(ex) & np.isfinite(sc)
    err = np.abs(g - ex)[fin]
    ref = np.abs(ex[fin])
    nz = ref > 0  # exact zeros (a perfect match) have no relative error
    rel = err[nz] / ref[nz]
    scaled = err / np.maximum(sc[fin], 1e-300)
    return {"max_abs": float(err.max()), "max_rel": float(rel.max()) if rel.size else 0.0,
            "max_scaled": float(scaled.max()),
            "within_1e-5_rel": round(float((rel <= 1e-5).mean()), 6) if rel.size else 1.0}


def valid_taps(W, H, tw, th, nch=1):
    return (W - tw + 1) * (H - th + 1) * tw * th * nch


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.path = os.path.join("/tmp", f"bench_clocks_{os.getpid()}.csv")
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
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
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return world, rank, local


def allreduce_max(x):
    """Max of x over the ranks (x on every rank when not distributed). The
    tensor lives where the backend wants it: GPU for NCCL, host for gloo."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized():
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank, world):
    """This rank's share of independent work items (images of a batch):
    every world-th item from `rank`. The shares are disjoint, cover the list
    and differ in size by at most one; the path needs no exchange between
    ranks."""
    items = list(items)
    return items[rank::world] if world > 1 else items


def barrier():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()


def run_ours(args, world, rank, local):
    import torch

    from openclipp_b200 import ocip

    S, T, (ty, tx) = workload(seed=1234 + rank, with_offset=True)
    H, W = S.shape
    MEASURES = args.measures
    taps_step = valid_taps(W, H, T_SIDE, T_SIDE) * len(MEASURES)

    ctx = ocip.Context(local)
    path = {"auto": ocip.PATH_AUTO, "plain": ocip.PATH_PLAIN, "tensor": ocip.PATH_TENSOR}[args.path]
    ctx.set_path(path)
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # Device-resident arm.
    Si, Ti = ocip.Image(S), ocip.Image(T)
    outs = [np.zeros((H, W), np.float32) for _ in MEASURES]
    Ds = [ocip.Image(o) for o in outs]
    Si.send()
    Ti.send()

    def timed_steps(n, measures, record=None):
        """n steps of `measures` (L2 flushed before each, not timed); per-measure
        CUDA-event times go to `record` (a dict) when given."""
        times = []
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(measures) + 1)]
            ev[0].record(stream)
            for i, m in enumerate(measures):
                ocip.check(ocip.proximity(m, Si, Ti, Ds[MEASURES.index(m)]), m)
                ev[i + 1].record(stream)
            ev[-1].synchronize()
            times.append(ev[0].elapsed_time(ev[-1]))
            if record is not None:
                for i, m in enumerate(measures):
                    record.setdefault(m, []).append(ev[i].elapsed_time(ev[i + 1]))
        return times

    timed_steps(args.warmup, MEASURES)
    paths_used = {}
    for m, D in zip(MEASURES, Ds):
        ocip.check(ocip.proximity(m, Si, Ti, D), m)
        paths_used[m] = {1: "plain", 2: "tensor"}[ctx.last_path()]
    ctx.finish()
    torch.cuda.synchronize()
    barrier()
    per_kernel = {}
    launches0 = ocip.launch_count()
    with Clocks(local) as clk:
        times = timed_steps(args.steps, MEASURES, per_kernel)
    launches = ocip.launch_count() - launches0
    torch.cuda.synchronize()
    barrier()
    ms_step = allreduce_max(float(np.mean(times)))
    clocks = clk.summary()

    # Accuracy of this run's maps against the exact oracle on full rows
    # (spread over the map, plus the template's rows around the match).
    rows = check_rows(H, T_SIDE, n=256, match_row=ty + T_SIDE // 2)
    acc = {}
    if rank == 0 and not args.no_accuracy:
        for D in Ds:
            D.read()
        acc[f"F32 {W}x{H} blob field, {T_SIDE}x{T_SIDE} ({args.path})"] = {
            "rows": f"{len(rows)} full rows: 256 spread over the map, its first/last two, "
                    f"rows {ty}-{ty + T_SIDE - 1} around the match",
            **{m: dict(error_rows(MEAS_ALL.index(m), S, T, outs[i], rows), path=paths_used[m])
               for i, m in enumerate(MEASURES)}}

    # The metric's comparison: the plain FP32 kernels (the drop-in) on the
    # same data, same step structure and L2 flush, for the product measures.
    product = [m for m in MEASURES if m != "AbsDistance"]
    per_kernel_plain = {}
    if product and not args.no_plain_arm:
        ctx.set_path(ocip.PATH_PLAIN)
        timed_steps(3, product)
        torch.cuda.synchronize()
        barrier()
        timed_steps(max(3, min(args.steps, 10)), product, per_kernel_plain)
        torch.cuda.synchronize()
        barrier()
        if rank == 0 and not args.no_accuracy:
            for m in product:
                Ds[MEASURES.index(m)].read()
            acc[f"F32 {W}x{H} blob field, {T_SIDE}x{T_SIDE} (plain FP32, reference arithmetic)"] = {
                m: error_rows(MEAS_ALL.index(m), S, T, outs[MEASURES.index(m)], rows)
                for m in product}
        ctx.set_path(path)
    if rank == 0 and not args.no_accuracy:
        acc.update(accuracy_suite(ocip, ctx, S, (ty, tx), product))
        ctx.set_path(path)

    # Best match of the step's CrossCorr_Norm map: ocipMaxIndx on a written map
    # against the reduction fused into the scoring epilogue (no map written).
    best = best_match_timing(ocip, torch, ctx, stream, flush, Si, Ti, Ds[MEASURES.index(
        "CrossCorr_Norm")]) if ("CrossCorr_Norm" in MEASURES and not args.no_plain_arm) else None
    ctx.set_path(path)

    # End-to-end arm: pinned host buffers, send + calls + reads per step.
    e2e_ms = run_e2e(args, ocip, torch, ctx, S, T, stream) if not args.no_e2e else float("nan")
    e2e_ms = allreduce_max(e2e_ms)
    e2e_pg_ms = (run_e2e(args, ocip, torch, ctx, S, T, stream, pinned=False)
                 if not args.no_e2e else float("nan"))
    e2e_pg_ms = allreduce_max(e2e_pg_ms)

    value = taps_step * world / (ms_step * 1e-3) / 1e9
    e2e_value = taps_step * world / (e2e_ms * 1e-3) / 1e9 if e2e_ms == e2e_ms else None

    # Roofline of the dominant tensor-core kernel (largest share of the step
    # among the measures served by the tensor path); the plain kernels that
    # remain in the step (AbsDistance has no product form) are reported beside
    # it against the FP32 ALU rate.
    med = {m: float(np.median(v)) for m, v in per_kernel.items()}
    med_plain = {m: float(np.median(v)) for m, v in per_kernel_plain.items()}
    tensor_meas = [m for m in med if paths_used[m] == "tensor"] or list(med)
    dom = max(tensor_meas, key=med.get)
    peaks = load_peaks()
    taps_meas = valid_taps(W, H, T_SIDE, T_SIDE)
    same_taps = W * H * T_SIDE * T_SIDE
    tflops = 2.0 * same_taps / (med[dom] * 1e-3) / 1e12
    roof = {"kernel": f"{dom} ({paths_used[dom]})", "bound": "tensor", "achieved": round(tflops, 2),
            "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
            "frac": round(tflops / peaks["bf16_tflops"], 4),
            "traffic": ncu_traffic(dom, paths_used[dom]),
            "peak_source": peaks["source"],
            "flops_convention": "2 per tap (one multiply-add), same-size map "
                                f"{W}x{H}x{T_SIDE}x{T_SIDE} per launch"}
    plain_meas = [m for m in med if paths_used[m] == "plain"]
    roof_plain = {}
    for m in plain_meas:
        # FP32 lanes: 148 SMs x 128 lanes x 2 ops (sub, abs-add) per tap.
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        peak_taps = 148 * 128 * sm_mhz * 1e6 / 2.0
        got = same_taps / (med[m] * 1e-3)
        roof_plain[m] = {"bound": "alu (FP32 lanes)", "achieved_gtaps": round(got / 1e9, 1),
                         "peak_gtaps": round(peak_taps / 1e9, 1), "frac": round(got / peak_taps, 4),
                         "peak_source": "nominal: 148 SMs x 128 FP32 lanes x clock, 2 ops per tap"}

    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "Gtaps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded blob field, template cut from it)",
        "config": {"workload": f"{W}x{H} F32 1ch, {T_SIDE}x{T_SIDE} template, 5 measures per step",
                   "path": args.path, "paths_used": paths_used,
                   "taps_per_step": taps_step, "taps_counted": "valid region",
                   "l2": "flushed before every step (256 MiB write, outside the timed events)"},
        "per_measure_ms": {m: round(v, 4) for m, v in med.items()},
        "per_measure_gtaps": {m: round(taps_meas / (v * 1e-3) / 1e9, 1) for m, v in med.items()},
        "tensor_per_measure_ms": {m: round(med[m], 4) for m in product if m in med},
        "plain_per_measure_ms": {m: round(v, 4) for m, v in med_plain.items()},
        "tensor_over_plain": {m: round(med_plain[m] / med[m], 2) for m in med_plain
                              if paths_used.get(m) == "tensor"},
        "accuracy_vs_fp64": acc,
        "best_match": best,
        "roofline": roof,
        "roofline_plain": roof_plain,
        "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "Gtaps/s",
                "h2d_bytes_per_step": int(S.nbytes + T.nbytes),
                "d2h_bytes_per_step": int(sum(o.nbytes for o in outs)),
                "host_buffers": "page-locked (allocated pinned by the caller)"},
        "e2e_pageable": {
            "value": round(taps_step * world / (e2e_pg_ms * 1e-3) / 1e9, 2)
            if e2e_pg_ms == e2e_pg_ms else None, "unit": "Gtaps/s",
            "host_buffers": "numpy (malloc'd) arrays reused every step; the library page-locks "
                            "each after its fourth transfer (steady state measured)"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(S, T, budget_s=args.cpu_seconds)
    for D in Ds:
        D.release()
    Si.release()
    Ti.release()
    ctx.close()
    return result


MEAS_ALL = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]


def best_match_timing(ocip, torch, ctx, stream, flush, Si, Ti, Di, reps=10):
    """CUDA-event ms of the best match of CrossCorr_Norm (MaxIndx), tensor
    path: the map written then ocipMaxIndx, against ocipProximityIndx with
    the reduction in the scoring epilogue and no map. L2 flushed before each."""
    ctx.set_path(ocip.PATH_TENSOR)
    prog = ocip.prepare_statistics(Di)

    def map_then_index():
        ocip.check(ocip.proximity("CrossCorr_Norm", Si, Ti, Di), "CrossCorr_Norm")
        rc, v, x, y = ocip.index_reduce("MaxIndx", prog, Di)
        ocip.check(rc, "ocipMaxIndx")
        return v, x, y

    def fused():
        rc, v, x, y = ocip.proximity_index("CrossCorr_Norm", "MaxIndx", Si, Ti)
        ocip.check(rc, "ocipProximityIndx")
        return v, x, y

    out = {}
    answers = {}
    for name, fn in (("map_then_index_ms", map_then_index), ("fused_no_map_ms", fused)):
        for _ in range(3):
            answers[name] = fn()
        t = []
        for _ in range(reps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            t.append(e0.elapsed_time(e1))
        out[name] = round(float(np.median(t)), 4)
    prog.release()
    out["same_answer"] = answers["map_then_index_ms"] == answers["fused_no_map_ms"]
    out["answer"] = list(answers["fused_no_map_ms"])
    out["measure"], out["reduction"] = "CrossCorr_Norm", "MaxIndx"
    return out


def _run_maps(ocip, ctx, path, measures, S, T, out_dtype=np.float32):
    """Each measure of (S, T) on the given path; returns {measure: map} and the
    paths that served them."""
    ctx.set_path(path)
    Si, Ti = ocip.Image(S), ocip.Image(T)
    maps, used = {}, {}
    for m in measures:
        out = np.zeros(S.shape, out_dtype)
        D = ocip.Image(out)
        ocip.check(ocip.proximity(m, Si, Ti, D), m)
        D.read()
        used[m] = {1: "plain", 2: "tensor"}[ctx.last_path()]
        D.release()
        maps[m] = out
    Si.release()
    Ti.release()
    return maps, used


def accuracy_suite(ocip, ctx, S, off, product):
    """Error reports per measure and dtype beyond the timed workload:
    the zero-mean (signed) variant of the 4096^2 F32 field on both paths,
    the 512^2 U8 config (bit-exact count against the reference's own kernel
    source), and the 3840x2160x4 U8/U16 config with a 64x64x4 template."""
    from oracle import oracle as O
    rep = {}
    ty, tx = off
    H, W = S.shape
    rows = check_rows(H, T_SIDE, n=64, match_row=ty + T_SIDE // 2)
    S0 = (S - np.float32(S.mean(dtype=np.float64))).astype(np.float32)
    T0 = S0[ty:ty + T_SIDE, tx:tx + T_SIDE].copy()
    for name, path in (("tensor", ocip.PATH_TENSOR), ("plain FP32, reference arithmetic",
                                                      ocip.PATH_PLAIN)):
        maps, used = _run_maps(ocip, ctx, path, product, S0, T0)
        rep[f"F32 {W}x{H} zero-mean blob field, {T_SIDE}x{T_SIDE} ({name})"] = {
            "rows": f"{len(rows)} full rows incl. the match's", "note":
                "signed data: per-output relative error is unbounded where a sum cancels; "
                "max_scaled states it against sum |S||T| (CrossCorr) or sum S^2 + sum T^2 "
                "(SqrDistance), over sqrt(sum S^2 sum T^2) for _Norm",
            **{m: dict(error_rows(MEAS_ALL.index(m), S0, T0, maps[m], rows), path=used[m])
               for m in product}}
    # 512x512 U8, 16x16 template: integer scores, bit-exact against the
    # reference's own kernel source (built for the host).
    S1, T1 = cfg1_images()
    for name, path in (("tensor", ocip.PATH_TENSOR), ("plain", ocip.PATH_PLAIN)):
        maps, used = _run_maps(ocip, ctx, path, MEAS_ALL[:], S1, T1)
        r = {}
        for m in MEAS_ALL:
            want = (O.proximity_reference(m, S1, T1) if O.ref_available()
                    else O.proximity_refexact(m, S1, T1))
            r[m] = {"unequal_to_reference": int((~((maps[m] == want) |
                                                   (np.isnan(maps[m]) & np.isnan(want)))).sum()),
                    "outputs": int(want.size), "path": used[m]}
        rep[f"U8 512x512, 16x16 ({name})"] = r
    # 3840x2160x4 U8 and U16, 64x64x4 template, _Norm measures on the tensor path.
    for dt, label in ((np.uint8, "U8"), (np.uint16, "U16")):
        S5, T5, (y5, _) = cfg5_images(dt)
        rows5 = sorted({0, 1, 2158, 2159, y5 + 32} |
                       set(np.linspace(32, 2160 - 33, 6).astype(int).tolist()))
        maps, used = _run_maps(ocip, ctx, ocip.PATH_TENSOR, ["SqrDistance_Norm", "CrossCorr_Norm"],
                               S5, T5)
        rep[f"{label} 3840x2160x4, 64x64x4 (tensor)"] = {
            "rows": f"{len(rows5)} full rows (all 4 channels) incl. the match row",
            **{m: dict(error_rows(MEAS_ALL.index(m), S5, T5, maps[m], rows5), path=used[m])
               for m in maps}}
    return rep


def run_e2e(args, ocip, torch, ctx, S, T, stream, pinned=True):
    """Mean ms of a step through the C ABI from host buffers: send the
    source and template, the measures, read every map. pinned=False uses
    plain numpy (malloc'd) buffers as a reference program passes them; the
    library page-locks a reused buffer after its fourth transfer, and the
    warm-up covers those, so this is the steady state of a caller that
    reuses its buffers."""
    MEASURES = args.measures
    H, W = S.shape
    if pinned:
        hS = torch.empty((H, W), dtype=torch.float32, pin_memory=True).numpy()
        hT = torch.empty(T.shape, dtype=torch.float32, pin_memory=True).numpy()
        houts = [torch.empty((H, W), dtype=torch.float32, pin_memory=True).numpy()
                 for _ in MEASURES]
    else:
        hS = np.empty((H, W), np.float32)
        hT = np.empty(T.shape, np.float32)
        houts = [np.empty((H, W), np.float32) for _ in MEASURES]
    hS[:] = S
    hT[:] = T
    Si, Ti = ocip.Image(hS), ocip.Image(hT)
    Ds = [ocip.Image(o) for o in houts]

    def step():
        Si.send()
        Ti.send()
        for m, D in zip(MEASURES, Ds):
            ocip.check(ocip.proximity(m, Si, Ti, D), m)
        for D in Ds:
            D.read()

    for _ in range(max(4, min(args.warmup, 6))):
        step()
    times = []
    for _ in range(max(1, min(args.steps, 5))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    for D in Ds:
        D.release()
    Si.release()
    Ti.release()
    return float(np.mean(times))


def ncu_traffic(measure, path):
    """DRAM bytes (read + write) per launch of the given kernel from the
    committed ncu summary, or None when that kernel was not captured."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(f"{measure} ({path})")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "source": "measured (MEASURED_PEAKS.json, burst)"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def cpu_reference_time(S, T, rows):
    """Seconds for the reference kernel source (host build, all threads) on
    output rows [0, rows) for the five measures."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    for i in range(len(MEASURES)):
        O.proximity_reference(i, S, T, rows=(0, rows))
    return time.perf_counter() - t0


def cpu_baseline(S, T, budget_s=15.0):
    from oracle import oracle as O
    if not O.ref_available():
        return {"value": None, "unit": "Gtaps/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "reference kernels not built"}
    rows = 8
    dt = cpu_reference_time(S, T, rows)
    rows = int(max(8, min(S.shape[0], rows * budget_s / max(dt, 1e-3))))
    dt = cpu_reference_time(S, T, rows)
    H, W = S.shape
    taps = rows * (W - T_SIDE + 1) * T_SIDE * T_SIDE * len(MEASURES)
    return {"value": round(taps / dt / 1e9, 4), "unit": "Gtaps/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
            "kind": "reference",
            "sample": f"output rows 0-{rows} of the {W}x{H} map, 5 measures, "
                      f"cl-files/ImageProximity.cl built for the host (OpenMP), {dt:.1f} s"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    from oracle import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (no reference sources)"}
    S, T = workload(seed=1234)
    H, W = S.shape
    rows = 4
    dt = cpu_reference_time(S, T, rows)
    budget = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    rows = int(max(4, min(H, rows * budget / max(dt, 1e-3))))
    taps = rows * (W - T_SIDE + 1) * T_SIDE * T_SIDE * len(MEASURES)
    for _ in range(args.warmup):
        cpu_reference_time(S, T, max(1, rows // 8))
    times = [cpu_reference_time(S, T, rows) for _ in range(args.steps)]
    value = taps / float(np.mean(times)) / 1e9
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    sample = (f"output rows 0-{rows} of the {W}x{H} map per step, 5 measures, "
              "cl-files/ImageProximity.cl built for the host (OpenMP)")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Gtaps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(float(np.mean(times)) * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded blob field, template cut from it)",
            "config": {"workload": f"{W}x{H} F32 1ch, {T_SIDE}x{T_SIDE} template, 5 measures per step",
                       "taps_counted": "valid region"},
            "cpu_baseline": {"value": round(value, 4), "unit": "Gtaps/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "Gtaps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


BATCH_SIDES = [8, 12, 16, 24, 32, 48, 64]


def batch_workload(seed=31, n_img=16, n_tpl=64, side=2048):
    """16 U8 images of 2048x2048 (uniform 0-255) and 64 square U8 templates of
    sides drawn from {8, 12, 16, 24, 32, 48, 64}, each cut from a random image
    at a random offset with +-8 intensity noise (seeded)."""
    rng = np.random.default_rng(seed)
    imgs = [rng.integers(0, 256, (side, side), dtype=np.uint8) for _ in range(n_img)]
    tmpls = []
    for s in rng.choice(BATCH_SIDES, n_tpl):
        s = int(s)
        k = int(rng.integers(0, n_img))
        y, x = (int(v) for v in rng.integers(0, side - s, 2))
        t = imgs[k][y:y + s, x:x + s].astype(np.int32) + rng.integers(-8, 9, (s, s))
        tmpls.append(np.clip(t, 0, 255).astype(np.uint8))
    return imgs, tmpls


def run_batch_bench(args, world, rank, local):
    """Batched uneven templates: CrossCorr and SqrDistance for every (image,
    template) pair, each measure one persistent launch replayed from a CUDA
    graph. One step = both launches. Work is split by image across ranks."""
    import torch

    from openclipp_b200 import ocip

    imgs, tmpls = batch_workload()
    mine = shard(imgs, rank, world)
    side = imgs[0].shape[0]
    taps_meas = sum(len(mine) * (side - t.shape[0] + 1) ** 2 * t.size for t in tmpls)
    measures = ["CrossCorr", "SqrDistance"]
    ctx = ocip.Context(local)
    ctx.set_path(ocip.PATH_TENSOR)
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    Si = [ocip.Image(a) for a in mine]
    Ti = [ocip.Image(t) for t in tmpls]
    Ds = [ocip.Image(shape=(side, side), dtype=np.float32) for _ in range(len(mine) * len(tmpls))]
    t0 = time.time()
    batches = [ocip.prepare_batch(m, Si, Ti, Ds) for m in measures]
    prep_s = time.time() - t0
    nitems = batches[0].info()[0]
    bh = {s: batches[0].info(s, s)[1] for s in BATCH_SIDES}

    def step():
        for b in batches:
            ocip.check(b.run(), "ocipRunProximityBatch")

    def timed(n):
        out = []
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return out

    timed(args.warmup)
    torch.cuda.synchronize()
    barrier()
    launches0 = ocip.launch_count()
    with Clocks(local) as clk:
        times = timed(args.steps)
    launches = ocip.launch_count() - launches0
    torch.cuda.synchronize()
    barrier()
    ms_step = allreduce_max(float(np.mean(times)))

    # Exactness check: a batch over 256x256 crops of two images and four of
    # the templates (host-backed maps) equals the int64 oracle.
    from oracle import oracle as O
    crops = [np.ascontiguousarray(mine[k][:256, :256]) for k in range(min(2, len(mine)))]
    sub = tmpls[:4]
    outs = [np.zeros((256, 256), np.float32) for _ in crops for _ in sub]
    Ci, Ui, Oi = [ocip.Image(c) for c in crops], [ocip.Image(t) for t in sub], [ocip.Image(o) for o in outs]
    cb = ocip.prepare_batch("CrossCorr", Ci, Ui, Oi)
    ocip.check(cb.run(), "ocipRunProximityBatch")
    for o in Oi:
        o.read()
    exact = all(np.array_equal(outs[i * len(sub) + j], O.proximity_exact(3, c, t).astype(np.float32))
                for i, c in enumerate(crops) for j, t in enumerate(sub))
    cb.release()
    for x in Ci + Ui + Oi:
        x.release()
    # Plain path on the same pairs (one measure, timed once).
    ctx.set_path(ocip.PATH_PLAIN)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(len(mine)):
        for j in range(len(tmpls)):
            ocip.check(ocip.proximity("CrossCorr", Si[i], Ti[j], Ds[i * len(tmpls) + j]), "plain")
    ev1.record(stream)
    ev1.synchronize()
    plain_ms = ev0.elapsed_time(ev1)
    for b in batches:
        b.release()
    for x in Si + Ti + Ds:
        x.release()
    ctx.close()
    value = 2 * taps_meas * world / (ms_step * 1e-3) / 1e9
    peaks = load_peaks()
    # i8 MMA: one multiply-add per tap = 2 int ops; against the bf16 dense
    # peak doubled (the i8 rate of the same tensor pipe).
    tops = 2.0 * 2 * taps_meas / (ms_step * 1e-3) / 1e12
    return {
        "metric": "batched match-score Gtaps/s (i8 MMA, bit-exact)", "value": round(value, 2),
        "unit": "Gtaps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded uniform U8 images, templates cut with +-8 noise)",
        "config": {"workload": f"{len(imgs)} x {side}x{side} U8 images x {len(tmpls)} templates "
                               "(sides 8-64), CrossCorr + SqrDistance per step",
                   "taps_per_step": 2 * taps_meas, "taps_counted": "valid region",
                   "work_items": nitems, "band_heights": bh, "prepare_s": round(prep_s, 2),
                   "l2": "flushed before every step (256 MiB write, outside the timed events)"},
        "plain_crosscorr_ms": round(plain_ms, 2),
        "plain_crosscorr_gtaps": round(taps_meas / (plain_ms * 1e-3) / 1e9, 1),
        "batch_crosscorr_exact_vs_int64_oracle": exact,
        "roofline": {"kernel": "prox_tensor_kernel<U8> (batch)", "bound": "tensor",
                     "achieved": round(tops, 2), "peak": 2 * peaks["bf16_tflops"],
                     "unit": "TOPS (i8)", "frac": round(tops / (2 * peaks["bf16_tflops"]), 4),
                     "traffic": None, "peak_source": peaks["source"] + ", x2 for i8"},
        "e2e": {"value": None, "unit": "Gtaps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "not measured: 32 GB of score maps per step"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }


def run_backward_bench(args, world, rank, local):
    """Differentiation workload: 32 F32 images of 1024x1024 (blob field), each
    with a 32x32 template (its seeded crop + N(0, 0.02)). Forward =
    CrossCorr_Norm and SqrDistance of every pair; backward = the gradients of
    sum G1 SqrDistance + sum G2 CrossCorr_Norm (G ~ N(0, 1)) with respect to
    the image and the template. Reports both times and their ratio."""
    import torch

    from openclipp_b200 import ocip
    n_img, side, ts = 32, 1024, 32
    rng = np.random.default_rng(41)
    ctx = ocip.Context(local)
    ctx.set_path(ocip.PATH_TENSOR)
    stream = torch.cuda.ExternalStream(ctx.stream())
    imgs, tps, g1s, g2s, sqs, ccs, dss, dts = [], [], [], [], [], [], [], []
    for k in range(rank, n_img, world):
        S = blob_field(side, side, nblobs=60, seed=400 + k)
        y, x = (int(v) for v in rng.integers(0, side - ts, 2))
        T = (S[y:y + ts, x:x + ts] + rng.normal(0, 0.02, (ts, ts))).astype(np.float32)
        imgs.append(ocip.Image(S))
        tps.append(ocip.Image(T))
        g1s.append(ocip.Image(rng.standard_normal((side, side)).astype(np.float32)))
        g2s.append(ocip.Image(rng.standard_normal((side, side)).astype(np.float32)))
        sqs.append(ocip.Image(shape=(side, side), dtype=np.float32))
        ccs.append(ocip.Image(shape=(side, side), dtype=np.float32))
        dss.append(ocip.Image(shape=(side, side), dtype=np.float32))
        dts.append(ocip.Image(shape=(ts, ts), dtype=np.float32))
    for x in imgs + tps + g1s + g2s:
        x.send()

    def forward():
        for i in range(len(imgs)):
            ocip.check(ocip.sqr_distance(imgs[i], tps[i], sqs[i]), "fwd")
            ocip.check(ocip.cross_corr_norm(imgs[i], tps[i], ccs[i]), "fwd")

    def backward():
        for i in range(len(imgs)):
            ocip.check(ocip.proximity_backward(imgs[i], tps[i], g1s[i], g2s[i], ccs[i], dss[i],
                                               dts[i]), "bwd")

    def timed(fn, n):
        out = []
        for _ in range(n):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return out

    for _ in range(args.warmup):
        forward()
        backward()
    torch.cuda.synchronize()
    barrier()
    with Clocks(local) as clk:
        f_ms = allreduce_max(float(np.mean(timed(forward, args.steps))))
        b_ms = allreduce_max(float(np.mean(timed(backward, args.steps))))
    taps = n_img * (side - ts + 1) ** 2 * ts * ts  # per measure, valid region
    # Gradient check on a crop of the first pair against the long-double adjoint.
    from oracle import oracle as O
    crop = np.ascontiguousarray(blob_field(side, side, nblobs=60, seed=400 + rank)[:192, :192])
    rng2 = np.random.default_rng(3)
    Tc = (crop[40:72, 60:92] + rng2.normal(0, 0.02, (ts, ts))).astype(np.float32)
    G1 = rng2.standard_normal(crop.shape).astype(np.float32)
    G2 = rng2.standard_normal(crop.shape).astype(np.float32)
    Ci, Ti = ocip.Image(crop), ocip.Image(Tc)
    N = np.zeros(crop.shape, np.float32)
    Ni = ocip.Image(N)
    ocip.check(ocip.cross_corr_norm(Ci, Ti, Ni), "fwd")
    dS = np.zeros(crop.shape, np.float32)
    dT = np.zeros((ts, ts), np.float32)
    G1i, G2i, dSi, dTi = ocip.Image(G1), ocip.Image(G2), ocip.Image(dS), ocip.Image(dT)
    ocip.check(ocip.proximity_backward(Ci, Ti, G1i, G2i, Ni, dSi, dTi), "bwd")
    dSi.read()
    dTi.read()
    a0, b0 = O.proximity_backward(0, crop, Tc, G1)
    a4, b4 = O.proximity_backward(4, crop, Tc, G2)
    err_s = float(np.abs(dS - (a0 + a4)).max() / np.abs(a0 + a4).max())
    err_t = float(np.abs(dT - (b0 + b4)).max() / np.abs(b0 + b4).max())
    for x in imgs + tps + g1s + g2s + sqs + ccs + dss + dts + [Ci, Ti, Ni, G1i, G2i, dSi, dTi]:
        x.release()
    ctx.close()
    return {
        "metric": "backward / forward time, CrossCorr_Norm + SqrDistance (tensor path)",
        "value": round(b_ms / f_ms, 3), "unit": "ratio", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(b_ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded blob fields, templates cut with N(0, 0.02) noise)",
        "config": {"workload": f"{n_img} x {side}x{side} F32 images, {ts}x{ts} templates; "
                               "forward = SqrDistance + CrossCorr_Norm, backward = dS and dT "
                               "of both in one pass"},
        "forward_ms": round(f_ms, 3), "backward_ms": round(b_ms, 3),
        "forward_gtaps": round(2 * taps * world / (f_ms * 1e-3) / 1e9, 1),
        "adjoint_rel_err_vs_fp64": {"dS": err_s, "dT": err_t},
        "clocks": clk.summary(),
    }


def run_sad_bench(args, world, rank, local):
    """U8 AbsDistance workload: a 4096x4096 U8 image (uniform noise plus the
    blob field scaled to 0-255) against a 31x31 template cut from it, on the
    packed-byte SAD kernel. Taps counted over the valid region; the peak is
    four taps per vabsdiff4 at 64 lanes per clock per SM."""
    import torch

    from openclipp_b200 import ocip
    from oracle import oracle as O

    H = W = 4096
    ts = 31
    rng = np.random.default_rng(77 + rank)
    S = np.clip(blob_field(W, H, seed=77 + rank) * 200 + rng.integers(0, 56, (H, W)),
                0, 255).astype(np.uint8)
    T = S[1000:1000 + ts, 2000:2000 + ts].copy()
    ctx = ocip.Context(local)
    ctx.set_path(ocip.PATH_PLAIN)
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = np.zeros((H, W), np.float32)
    Si, Ti, Di = ocip.Image(S), ocip.Image(T), ocip.Image(out)
    Si.send()
    Ti.send()

    def timed(n):
        t = []
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ocip.check(ocip.proximity("AbsDistance", Si, Ti, Di), "AbsDistance")
            e1.record(stream)
            e1.synchronize()
            t.append(e0.elapsed_time(e1))
        return t

    timed(args.warmup)
    torch.cuda.synchronize()
    barrier()
    steps = max(args.steps, 1000)
    launches0 = ocip.launch_count()
    with Clocks(local) as clk:
        times = timed(steps)
    launches = ocip.launch_count() - launches0
    ms = allreduce_max(float(np.mean(times)))
    clocks = clk.summary()
    taps = valid_taps(W, H, ts, ts)
    value = taps * world / (ms * 1e-3) / 1e9
    # Exactness on a band of rows against the exact integer sums.
    Di.read()
    band = np.ascontiguousarray(S[:96])
    ex = O.proximity_exact(2, band, T)[:96 - ts]
    exact = bool(np.array_equal(out[:96 - ts], ex[:96 - ts].astype(np.float32)))

    # End to end: pinned host source in, score map out, every step.
    hS = torch.empty((H, W), dtype=torch.uint8, pin_memory=True).numpy()
    hS[:] = S
    hO = torch.empty((H, W), dtype=torch.float32, pin_memory=True).numpy()
    hSi, hDi = ocip.Image(hS), ocip.Image(hO)

    def e2e_step():
        hSi.send()
        ocip.check(ocip.proximity("AbsDistance", hSi, Ti, hDi), "AbsDistance")
        hDi.read()

    for _ in range(3):
        e2e_step()
    et = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        et.append(e0.elapsed_time(e1))
    e2e_ms = allreduce_max(float(np.mean(et)))
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    peak = 148 * 64 * 4 * sm_mhz * 1e6 / 1e9  # Gtaps/s
    same = W * H * ts * ts / (ms * 1e-3) / 1e9
    result = {
        "metric": "U8 AbsDistance Gtaps/s (packed-byte SAD)", "value": round(value, 1),
        "unit": "Gtaps/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (blob field x 200 + uniform 0-55, template cut from it)",
        "config": {"workload": f"{W}x{H} U8 1ch, {ts}x{ts} template, AbsDistance",
                   "taps_counted": "valid region",
                   "l2": "flushed before every step (256 MiB write, outside the timed events)"},
        "exact_vs_integer_oracle": exact,
        "roofline": {"bound": "alu (vabsdiff4, 4 taps per instruction)",
                     "achieved": round(same, 1), "peak": round(peak, 1), "unit": "Gtaps/s",
                     "frac": round(same / peak, 4), "traffic": None,
                     "peak_source": "nominal: 148 SMs x 64 lanes x clock x 4 taps "
                                    "(a probe of vabsdiff4 chains measured 73.7 T taps/s)",
                     "taps_convention": "same-size map per launch"},
        "e2e": {"value": round(taps * world / (e2e_ms * 1e-3) / 1e9, 1), "unit": "Gtaps/s",
                "h2d_bytes_per_step": int(S.nbytes), "d2h_bytes_per_step": int(out.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline and O.ref_available():
        # A trial band sizes a sample of about args.cpu_seconds.
        rows = 32
        t0 = time.perf_counter()
        O.proximity_reference(2, S, T, rows=(0, rows))
        dt = time.perf_counter() - t0
        rows = int(max(32, min(H, rows * args.cpu_seconds / max(dt, 1e-3))))
        t0 = time.perf_counter()
        O.proximity_reference(2, S, T, rows=(0, rows))
        dt = time.perf_counter() - t0
        result["cpu_baseline"] = {
            "value": round(rows * (W - ts + 1) * ts * ts / dt / 1e9, 3), "unit": "Gtaps/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())), "kind": "reference",
            "sample": f"output rows 0-{rows}, cl-files/ImageProximity.cl AbsDistance built for "
                      f"the host (OpenMP), {dt:.2f} s"}
    for x in (Si, Ti, Di, hSi, hDi):
        x.release()
    ctx.close()
    return result


def run_integral_bench(args, world, rank, local):
    """Integral scan workload: Integral and SqrIntegral of the 4096x4096 F32
    blob field into F64 tables, one of each per step. Algorithmic bytes per
    table: the source read once (4 B/px) and the table written once (8 B/px).
    The tables are checked against the exact integral of the oracle."""
    import torch

    from openclipp_b200 import ocip
    from oracle import oracle as O

    S = workload(seed=1234 + rank)[0]
    H, W = S.shape
    ctx = ocip.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    Si = ocip.Image(S)
    outs = [np.zeros((H, W), np.float64) for _ in range(2)]
    Ds = [ocip.Image(o) for o in outs]
    Si.send()
    prog = ocip.prepare_integral(Si)
    per_table = {0: [], 1: []}

    def timed(n, record=False):
        times = []
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(stream)
            for sqr in (0, 1):
                ocip.integral(prog, Si, Ds[sqr], sqr=bool(sqr))
                ev[sqr + 1].record(stream)
            ev[2].synchronize()
            times.append(ev[0].elapsed_time(ev[2]))
            if record:
                for sqr in (0, 1):
                    per_table[sqr].append(ev[sqr].elapsed_time(ev[sqr + 1]))
        return times

    timed(args.warmup)
    torch.cuda.synchronize()
    barrier()
    # A step is ~0.15 ms: at least 2000 steps so that the clock sampler
    # (100 ms period) sees the timed region.
    steps = max(args.steps, 2000)
    launches0 = ocip.launch_count()
    with Clocks(local) as clk:
        times = timed(steps, record=True)
    launches = ocip.launch_count() - launches0
    ms_step = allreduce_max(float(np.mean(times)))

    exact = True
    if rank == 0:
        for sqr in (0, 1):
            Ds[sqr].read()
            ex = O.integral_exact(S, sqr)
            rel = float(np.abs(outs[sqr] - ex).max() / np.abs(ex).max())
            exact = exact and rel < 1e-12

    # End-to-end: pinned host source in, both tables out, every step.
    hS = torch.empty((H, W), dtype=torch.float32, pin_memory=True).numpy()
    hS[:] = S
    houts = [torch.empty((H, W), dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    hSi = ocip.Image(hS)
    hDs = [ocip.Image(o) for o in houts]

    def e2e_step():
        hSi.send()
        for sqr in (0, 1):
            ocip.integral(prog, hSi, hDs[sqr], sqr=bool(sqr))
        for D in hDs:
            D.read()

    for _ in range(3):
        e2e_step()
    e2e_t = []
    for _ in range(max(1, min(args.steps, 5))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_t.append(e0.elapsed_time(e1))
    e2e_ms = allreduce_max(float(np.mean(e2e_t)))

    bytes_table = W * H * (4 + 8)
    bytes_step = 2 * bytes_table
    peaks = load_peaks()
    med = {k: float(np.median(v)) for k, v in per_table.items()}
    dom = max(med, key=med.get)
    gbs = bytes_table / (med[dom] * 1e-3) / 1e9
    result = {
        "metric": "integral table throughput (Integral + SqrIntegral, F32 -> F64)",
        "value": round(bytes_step * world / (ms_step * 1e-3) / 1e9, 1), "unit": "GB/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded blob field)",
        "config": {"workload": f"{W}x{H} F32 1ch -> F64 Integral and SqrIntegral per step",
                   "bytes_per_step": bytes_step,
                   "bytes_counted": "source read once + table written once, per table",
                   "l2": "flushed before every step (256 MiB write, outside the timed events)"},
        "per_table_ms": {"Integral": round(med[0], 4), "SqrIntegral": round(med[1], 4)},
        "exact_vs_oracle": exact,
        "roofline": {"kernel": ["Integral", "SqrIntegral"][dom] + " (3 launches)",
                     "bound": "hbm", "achieved": round(gbs, 1), "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": round(gbs / peaks["hbm_gbs"], 4),
                     "traffic": ncu_traffic("Integral", "3 launches"),
                     "traffic_note": "DRAM bytes of the three Integral launches, ncu with cold "
                                     "caches (profiles/integral_f32_to_f64_4096x4096.md)",
                     "peak_source": peaks["source"]},
        "e2e": {"value": round(bytes_step * world / (e2e_ms * 1e-3) / 1e9, 1), "unit": "GB/s",
                "h2d_bytes_per_step": int(S.nbytes),
                "d2h_bytes_per_step": int(sum(o.nbytes for o in houts))},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline and O.ref_available():
        # A trial band sizes a sample of about args.cpu_seconds.
        rows = 256
        t0 = time.perf_counter()
        for sqr in (0, 1):
            O.integral_reference(np.ascontiguousarray(S[:rows]), sqr, True)
        dt = time.perf_counter() - t0
        rows = int(max(256, min(H, rows * args.cpu_seconds / max(dt, 1e-3))))
        t0 = time.perf_counter()
        for sqr in (0, 1):
            O.integral_reference(np.ascontiguousarray(S[:rows]), sqr, True)
        dt = time.perf_counter() - t0
        result["cpu_baseline"] = {
            "value": round(2 * rows * W * 12 / dt / 1e9, 3), "unit": "GB/s", "cores": 1,
            "kind": "reference",
            "sample": f"rows 0-{rows} of the {W}x{H} source, Integral + SqrIntegral, "
                      f"cl-files/Integral.cl pipeline built for the host, {dt:.2f} s"}
    for D in Ds + hDs + [Si, hSi, prog]:
        D.release()
    ctx.close()
    return result


def side_workloads(args, world, rank, local):
    """Short runs of the other workloads beside the headline (batch, backward,
    integral, sad), so that one default run records each of them: 5 timed
    steps after 3 warm-up steps, no CPU baselines, each with its own checks
    against the oracle. A workload that fails records its error instead of
    ending the run."""
    import copy
    import gc

    import torch

    out = {}
    for name, fn in (("batch", run_batch_bench), ("backward", run_backward_bench),
                     ("integral", run_integral_bench), ("sad", run_sad_bench)):
        a = copy.copy(args)
        a.steps, a.warmup, a.no_cpu_baseline = 5, 3, True
        t0 = time.time()
        try:
            r = fn(a, world, rank, local)
            r = {k: v for k, v in r.items() if k not in ("n_gpus", "higher_is_better", "scaling",
                                                         "vs_baseline", "cpu_baseline")}
        except Exception as e:  # recorded, so that the headline line still prints
            r = {"error": f"{type(e).__name__}: {e}"}
        r["wall_s"] = round(time.time() - t0, 1)
        out[name] = r
        gc.collect()
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--path", choices=["auto", "tensor", "plain"], default="tensor")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--measures", default=",".join(MEASURES),
                    help="comma-separated subset of the five measures (profiling)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end arm (profiling)")
    ap.add_argument("--no-plain-arm", action="store_true",
                    help="skip timing the plain FP32 kernels beside the tensor path (profiling)")
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="skip the short runs of the batch, backward, integral and sad "
                         "workloads that a default single-GPU run adds to its line")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the error reports against the oracle (profiling)")
    ap.add_argument("--workload", choices=["single", "batch", "backward", "integral", "sad"],
                    default="single",
                    help="single: 4096^2 F32, 31x31, five measures (the headline); batch: 16 x "
                         "2048^2 U8 x 64 uneven templates in persistent launches; backward: "
                         "32 x 1024^2 F32 with 32x32 templates, gradients vs forward time; "
                         "integral: 4096^2 F32 Integral + SqrIntegral into F64 tables; "
                         "sad: 4096^2 U8 AbsDistance with a 31x31 template")
    args = ap.parse_args()
    args.measures = [m for m in args.measures.split(",") if m]
    assert all(m in MEASURES for m in args.measures), args.measures
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, world, rank)
        if res is not None:
            print(json.dumps(res))
        return
    world, rank, local = dist_setup()
    if args.workload == "batch":
        res = run_batch_bench(args, world, rank, local)
    elif args.workload == "backward":
        res = run_backward_bench(args, world, rank, local)
    elif args.workload == "integral":
        res = run_integral_bench(args, world, rank, local)
    elif args.workload == "sad":
        res = run_sad_bench(args, world, rank, local)
    else:
        res = run_ours(args, world, rank, local)
        if world == 1 and not args.no_side_workloads:
            res["side_workloads"] = side_workloads(args, world, rank, local)
    if rank == 0:
        print(json.dumps(res))
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
