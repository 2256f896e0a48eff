"""Benchmark of the projector pair on the parallel-beam FBP/SQS workload.

Workload (one step): parallel-beam distance-driven forward projection, the
normalised back projection, the Hann ramp filter and the FBP-weighted back
projection of a batch of 16 slices of 512 x 512 pixels at 0.8 mm, 720 views
over pi, 768 detector cells of 0.8 mm (seeded synthetic ellipse phantoms).

Metric: FP+BP GB/s against the HBM roofline -- the algorithmic bytes of the
step (per projector: one operand fetch per operator nonzero plus compulsory
input and output; the filter: its input and output) divided by the step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --op OP --workload NAME [--repeat N]     # one operation, for ncu

Under torchrun every rank processes its own batch (weak scaling, no
collective on the data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("parallel-beam DD FP + BP + ramp_filter(hann) + FBP BP, 16 x 512 x 512 at 0.8 mm, 720 views over pi, "
            "768 cells of 0.8 mm")
METRIC = "FP+BP GB/s vs HBM roofline; served recons/s, p50/p99 latency at <=1e-4 rel L2"
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 512 << 20


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def max_over_ranks(x: float, device) -> float:
    """The largest of every rank's ``x`` (the step time of the slowest rank);
    ``x`` itself without an initialised process group."""
    import torch
    import torch.distributed as tdist

    if not (tdist.is_available() and tdist.is_initialized()) or tdist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- workload
def workload_inputs(seed_index: int = 0):
    from ctprojector_b200 import synthetic as S

    scan, ang, nb = S.config2()
    rng = np.random.default_rng(S.seed_for(2, seed_index))
    img = np.stack([S.ellipse_phantom(rng, scan.nx, scan.ny, scan.dx, scan.dy)[None] for _ in range(nb)])
    return scan, ang, img.astype(np.float32)


def algorithmic_bytes(nnz_slice: int, nb: int, scan) -> dict:
    n_img = nb * scan.nz * scan.ny * scan.nx
    n_prj = nb * scan.nview * scan.nv * scan.nu
    proj = 4 * (nnz_slice * nb + n_img + n_prj)
    return {"fp": proj, "bp": proj, "filter": 4 * 2 * n_prj, "bp_fbp": proj}


# ours: launches of our own kernels per step (FP: edge table, view order,
# transpose, row and column line tables, streamed sweep; BP: gather; filter:
# one FFT row convolution over every row; FBP BP: gather)
OUR_LAUNCHES_PER_STEP = 6 + 1 + 1 + 1

# The filter of the step runs in exact mode: FP64 arithmetic in one launch
# (conv_rows_kernel).  The default mode replays the reference's FP32
# construction and transforms (bit-identical to it, 0.83 ms at this size);
# that FP32 rounding leaves the reference's filter 1.2-2.2e-5 from the exact
# result at 700-900 cells, the exact mode about 1e-7.
FILTER_NOTE = ("hann ramp filter in exact mode (FP64 arithmetic, one launch; ~1e-7 from the exact result, where the "
               "reference's FP32 filter is 1.2-2.2e-5 from it)")

# the launches behind each timed projector operation (the roofline names the dominant one)
ROOFLINE_KERNEL = {
    "fp": "dd2d_fp_stream_kernel (with its edge-table, view-order, transpose and line-table launches)",
    "bp": "dd2d_bp_par_fast_kernel",
    "bp_fbp": "dd2d_bp_par_fast_kernel (FBP weighting)",
}

# served streams: seeded Poisson arrivals of reconstruction jobs
SERVED_JOBS = 150  # 2D jobs only
SERVED_MIX_JOBS = 40  # the full mix, a third of it helical cone volumes
SERVED_RATE_HZ = 50.0
SERVED_SEED = 5
SERVED_MIX_SEED = 7
SERVED_STORAGE = ("sinograms in 16-bit affine storage on the device (uint16 codes, one FP32 offset and step per "
                  "view: half the bytes of FP32); iterate, projections and sums FP32")
SERVED_ACCURACY = ("q16 results within 1e-4 relative L2 of the FP64 oracle reconstruction of the FP32 sinograms "
                   "(tests/test_gpu_serving.py, tests/test_gpu_lowp.py); BF16 / FP16 sinograms measured at 6e-3 / "
                   "7e-4 (FBP) and 7e-4-1.3e-3 / 0.9-1.6e-4 (20 SQS-TV iterations) from it, so not served")


def run_ours(args, rank, world, local):
    import torch

    from ctprojector_b200.projector import _device as D
    from ctprojector_b200.projector.cupy import parallel as P
    from ctprojector_b200.projector.cupy.ct_projector import ct_projector
    from ctprojector_b200.projector.numpy import parallel as NP
    from ctprojector_b200.projector.numpy.ct_projector import ct_projector as np_ct_projector

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    scan, ang, img = workload_inputs(rank)
    nb = img.shape[0]
    p = scan.projector(ct_projector)
    timg = torch.tensor(img, device=dev)
    tang = torch.tensor(ang, device=dev)
    nnz = D.dd_nnz(p, tang, 1)
    ab = algorithmic_bytes(nnz, nb, scan)
    step_bytes = sum(ab.values())
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    ops = ["fp", "bp", "filter", "bp_fbp"]
    ev = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for k in ops}

    def step(record):
        e = ev["fp"]
        if record:
            e[0].record()
        prj = P.distance_driven_fp(p, timg, tang)
        if record:
            e[1].record()
            ev["bp"][0].record()
        bp = P.distance_driven_bp(p, prj, tang)
        if record:
            ev["bp"][1].record()
            ev["filter"][0].record()
        fprj = P.ramp_filter(p, prj, "hann", exact=True)
        if record:
            ev["filter"][1].record()
            ev["bp_fbp"][0].record()
        rec = P.distance_driven_bp(p, fprj, tang, True)
        if record:
            ev["bp_fbp"][1].record()
        return bp, rec

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()

    dist = world > 1
    if dist:
        import torch.distributed as tdist
    op_ms = {k: [] for k in ops}
    step_ms = []
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the step events)
            s0.record()
            step(True)
            s1.record()
            torch.cuda.synchronize()
            step_ms.append(s0.elapsed_time(s1))
            for k in ops:
                op_ms[k].append(ev[k][0].elapsed_time(ev[k][1]))
        torch.cuda.synchronize()
        if dist:
            tdist.barrier()
    ms = max_over_ranks(float(np.mean(step_ms)), dev)
    value = world * step_bytes / (ms * 1e-3) / 1e9

    # roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    op_avg = {k: float(np.mean(v)) for k, v in op_ms.items()}
    proj_ops = ["fp", "bp", "bp_fbp"]
    dom = max(proj_ops, key=lambda k: op_avg[k])
    achieved = ab[dom] / (op_avg[dom] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(f"dd2d_{dom}_cfg2")

    # end to end through the host-array API (numpy modules, c* entries)
    pinned = torch.empty(img.shape, dtype=torch.float32, pin_memory=True)
    pinned.copy_(torch.from_numpy(img))
    himg = pinned.numpy()
    pn = scan.projector(np_ct_projector)

    def e2e_step():
        prj = NP.distance_driven_fp(pn, himg, ang)
        bp = NP.distance_driven_bp(pn, prj, ang)
        fprj = NP.ramp_filter(pn, prj, "hann", exact=True)
        rec = NP.distance_driven_bp(pn, fprj, ang, True)
        return prj, bp, fprj, rec

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if dist:
        tdist.barrier()
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = max_over_ranks(float(np.mean(e2e_ms)), dev)
    n_img, n_prj = img.size, nb * scan.nview * scan.nv * scan.nu
    h2d = 4 * (n_img + n_prj + n_prj + n_prj) + 3 * 4 * len(ang)
    d2h = 4 * (n_prj + n_img + n_prj + n_img)

    cpu = cpu_baseline(scan, ang, img) if rank == 0 else None
    clocks = clk.summary()
    served = run_served(dev) if (rank == 0 and not args.no_served) else None
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipse phantoms)",
        "config": {"workload": WORKLOAD, "batch_per_gpu": nb, "nnz_per_slice": nnz,
                   "algorithmic_bytes_per_step": step_bytes, "l2": "flushed between steps (512 MiB write)",
                   "filter": FILTER_NOTE,
                   "parallelism": f"replicas x{world}", "op_ms": {k: round(v, 4) for k, v in op_avg.items()}},
        "roofline": {"bound": "hbm", "kernel": ROOFLINE_KERNEL.get(dom, dom), "achieved": round(achieved, 2),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic,
                     "achieved_meaning": "algorithmic bytes (one operand fetch per operator nonzero, served from "
                                         "shared memory and L2, plus compulsory I/O) per CUDA-event second",
                     "limiter": "SM instruction issue and shared-memory wavefronts, not DRAM "
                                "(profiles/dd2d_fp_stream_par512x16.md)",
                     "dram_gbs": None if traffic is None else round(traffic / (op_avg[dom] * 1e-3) / 1e9, 2),
                     "dram_frac": None if traffic is None else round(traffic / (op_avg[dom] * 1e-3) / 1e9 / peak, 4),
                     "compulsory_gbs": round((ab[dom] - 4 * nnz * nb) / (op_avg[dom] * 1e-3) / 1e9, 2)},
        "e2e": {"value": round(world * step_bytes / (e2e * 1e-3) / 1e9, 3), "unit": "GB/s", "ms_per_step": round(e2e, 3),
                "api": "ctprojector_b200.projector.numpy.parallel (host arrays, c* entries)",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "cpu_baseline": cpu,
        "gpu_launches": OUR_LAUNCHES_PER_STEP * args.steps,
        "clocks": clocks,
        "served": served,
    }
    return line


def _serve_stream(dev, n_jobs, mix, seed, label):
    """One seeded Poisson stream of ``n_jobs`` jobs drawn from ``mix`` at
    SERVED_RATE_HZ: through the reconstruction server with q16 sinograms
    (16-bit codes, one FP32 offset and step per view; iterate and sums FP32),
    then the same jobs and arrivals through the plain FP32 per-call path (one
    public-API call per operation, one job at a time).  Latency is arrival to
    result on the host; recons/s is jobs over the time to the last result; GPU
    busy is the union of the CUDA-event intervals of the work over the wall
    time of the run."""
    import torch

    from ctprojector_b200 import quant
    from ctprojector_b200.serving import Engine
    from ctprojector_b200.serving import workload as W
    from ctprojector_b200.serving.per_call import reconstruct, run_per_call

    p32 = W.catalog(storage="float32")
    plp = W.catalog(storage="q16")
    stream = W.arrivals(n_jobs, SERVED_RATE_HZ, seed, mix)
    names = sorted({n for _, n, _ in stream})
    pools32 = {n: W.sinogram_pool(p32[n], 2, 16, seed=i) for i, n in enumerate(names)}
    poolslp = {n: [quant.quantize(t.cuda()).cpu().pin_memory() for t in v] for n, v in pools32.items()}
    jobs = W.make_jobs(plp, stream, poolslp)
    eng = Engine(device=dev, track_busy=True)
    t0 = time.perf_counter()
    eng.warmup([plp[n] for n in names])
    warm = time.perf_counter() - t0
    served = eng.run(jobs, realtime=True)
    eng.close()
    del eng
    jobs32 = W.same_jobs(jobs, p32, pools32)
    for n in names:  # first-call costs (filter tables, kernel attributes) outside the stream
        reconstruct(next(j for j in jobs32 if j.protocol.name == n))
    torch.cuda.synchronize()
    per_call = run_per_call(jobs32, realtime=True, track_busy=True)
    by = {}
    for j in jobs:
        by.setdefault(j.protocol.name, []).append(j.latency)
    counts = {n: sum(1 for _, m, _ in stream if m == n) for n in names}
    r = lambda x: round(x, 3)  # noqa: E731
    return {
        "recons_per_s": r(served["recons_per_s"]), "p50_ms": r(served["p50_ms"]), "p99_ms": r(served["p99_ms"]),
        "jobs": served["jobs"], "arrival_rate_hz": SERVED_RATE_HZ, "gpu_busy_frac": r(served["gpu_busy_frac"]),
        "per_call_fp32": {"recons_per_s": r(per_call["recons_per_s"]), "p50_ms": r(per_call["p50_ms"]),
                          "p99_ms": r(per_call["p99_ms"]), "gpu_busy_frac": r(per_call["gpu_busy_frac"])},
        "served_over_per_call": r(served["recons_per_s"] / per_call["recons_per_s"]),
        "p50_ms_by_protocol": {k: r(1e3 * float(np.median(v))) for k, v in sorted(by.items())},
        "jobs_by_protocol": counts,
        "mix": f"{label}; FBP or 20 SQS-TV iterations; 1-16 slices per 2D job; Poisson arrivals, seed {seed}",
        "warmup_s": r(warm),
    }


def run_served(dev):
    """The reconstruction server on two seeded streams: SERVED_JOBS 2D jobs
    (fan 256^2 and 512^2, parallel 512^2), and SERVED_MIX_JOBS jobs of the full
    mix with helical cone 64 x 512^2 volumes."""
    out = _serve_stream(dev, SERVED_JOBS, _mix("2d"), SERVED_SEED,
                        "2D: fan 256^2 (360 views) and 512^2 (984 views), parallel 512^2 (720 views)")
    out["with_cone"] = _serve_stream(dev, SERVED_MIX_JOBS, _mix("all"), SERVED_MIX_SEED,
                                     "full mix: the 2D protocols and helical cone 64 x 512^2 (360 views, 736 x 64 "
                                     "panel; SQS only)")
    out["storage"] = SERVED_STORAGE
    out["accuracy"] = SERVED_ACCURACY
    return out


def _mix(which):
    from ctprojector_b200.serving import mix as M

    return M.MIX_2D if which == "2d" else M.MIX


def cpu_baseline(scan, ang, img):
    """The FP64 oracle (all host threads) on one slice of the batch: the same
    four operators, scaled to GB/s with that slice's algorithmic bytes."""
    from oracle import oracle as O

    O.build()
    sl = img[:1]
    t0 = time.perf_counter()
    prj = O.dd_fp(scan, sl, ang, "parallel")
    O.dd_bp(scan, prj, ang, "parallel")
    fprj = O.ramp_filter(scan, prj, "hann", "parallel")
    O.dd_bp(scan, fprj, ang, "parallel", is_fbp=True)
    dt = time.perf_counter() - t0
    nnz = O.dd_nnz(scan, ang, "parallel")
    b = sum(algorithmic_bytes(nnz, 1, scan).values())
    return {"value": round(b / dt / 1e9, 4), "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
            "seconds": round(dt, 2), "sample": "1 of the 16 slices: FP, BP, hann ramp filter, FBP BP (FP64 oracle)"}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank, world, local):
    """The reference library built from its own sources for sm_100a
    (oracle/_ref/libprojector.so) through its host-pointer C entries, with the
    argument conventions of its numpy wrappers, on the same workload."""
    import ctypes
    from ctypes import c_float, c_int, c_ulong, c_void_p

    path = os.path.join(ROOT, "oracle", "_ref", "libprojector.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "oracle/_ref/libprojector.so was not built from the reference "
                "sources (needs the reference tree at build time)"}
    L = ctypes.CDLL(path)
    scan, ang, img = workload_inputs(0)
    nb = img.shape[0]
    p = scan

    def g(nb_, prj_shape):
        nview, nv, nu = prj_shape
        return [c_ulong(nb_), c_ulong(p.nx), c_ulong(p.ny), c_ulong(p.nz), c_float(p.dx), c_float(p.dy),
                c_float(p.dz), c_float(p.cx), c_float(p.cy), c_float(p.cz), c_ulong(nu), c_ulong(nv),
                c_ulong(nview)]

    P = lambda a: c_void_p(a.ctypes.data)  # noqa: E731
    shape = (len(ang), p.nv, p.nu)

    def fp(x):  # parallel.py:133-189
        out = np.zeros([nb, *shape], np.float32)
        rc = L.cDistanceDrivenParallelProjection(P(out), P(x), P(ang), *g(nb, shape), c_float(p.du), c_float(p.dv),
                                                 c_float(p.off_u), c_float(p.off_v), c_int(0))
        assert rc == 0, rc
        return out

    def bp(y, fbp):  # parallel.py:192-254
        out = np.zeros([nb, p.nz, p.ny, p.nx], np.float32)
        rc = L.cDistanceDrivenParallelBackprojection(P(out), P(y), P(ang), *g(nb, shape), c_float(p.du),
                                                     c_float(p.dv), c_float(p.off_u), c_float(p.off_v),
                                                     c_int(1 if fbp else 0))
        assert rc == 0, rc
        return out

    def filt(y):  # parallel.py:20-71
        out = np.zeros(y.shape, np.float32)
        rc = L.cfbpParallelFilter(P(out), P(y), c_int(nb), c_ulong(p.nu), c_ulong(p.nv), c_ulong(len(ang)),
                                  c_float(p.du), c_float(p.dv), c_float(p.off_u), c_float(p.off_v), c_int(2))
        assert rc == 0, rc
        return out

    import torch

    pinned = torch.empty(img.shape, dtype=torch.float32, pin_memory=True)
    pinned.copy_(torch.from_numpy(img))
    himg = pinned.numpy()

    def step():
        prj = fp(himg)
        bp(prj, False)
        fprj = filt(prj)
        bp(fprj, True)

    for _ in range(args.warmup):
        step()
    ts = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            step()
            ts.append((time.perf_counter() - t0) * 1e3)
    ms = float(np.mean(ts))
    from oracle import oracle as O  # the operator's nonzero count, on the CPU (nothing of ours on this arm)

    O.build()
    nnz = O.dd_nnz(scan, ang, "parallel")
    step_bytes = sum(algorithmic_bytes(nnz, nb, scan).values())
    value = step_bytes / (ms * 1e-3) / 1e9
    n_prj = nb * len(ang) * p.nv * p.nu
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipse phantoms)",
        "config": {"workload": WORKLOAD, "batch_per_gpu": nb, "nnz_per_slice": nnz,
                   "algorithmic_bytes_per_step": step_bytes,
                   "implementation": "reference libprojector.so built from its sources for sm_100a, "
                                     "host-pointer c* entries as called by its numpy modules"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": 1, "kind": "reference",
                         "sample": "full workload; the reference's only implementation of the path is its CUDA "
                                   "library, driven from one host thread"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "copies_inside_reference_calls_bytes": 4 * (img.size + 3 * n_prj) + 4 * (2 * n_prj + 2 * img.size)},
        "clocks": clk.summary(),
        "served": None if args.no_served else run_reference_served(),
    }


class _RefDD:
    """The reference library's device-pointer DD entries and filters for one
    2D protocol, called with the argument conventions of its cupy wrappers
    (fan_equiangular.py:19-256, parallel.py:19-254): outputs allocated
    zero-filled per call, back projections accumulate into them."""

    def __init__(self, L, scan, kind, angles):
        import torch

        self.L, self.s, self.fan = L, scan, kind == "fan"
        self.ang = torch.tensor(angles, device="cuda")

    def _geo(self, nb, nu, nview):
        from ctypes import c_float, c_ulong

        s = self.s
        g = [c_ulong(nb), c_ulong(s.nx), c_ulong(s.ny), c_ulong(1), c_float(s.dx), c_float(s.dy), c_float(s.dz),
             c_float(s.cx), c_float(s.cy), c_float(s.cz), c_ulong(nu), c_ulong(1), c_ulong(nview)]
        if self.fan:
            return g + [c_float(s.du / s.dsd), c_float(s.dv), c_float(s.off_u), c_float(s.off_v), c_float(s.dsd),
                        c_float(s.dso)]
        return g + [c_float(s.du), c_float(s.dv), c_float(s.off_u), c_float(s.off_v)]

    def fp(self, x):
        import torch
        from ctypes import c_int, c_void_p

        nb, nview = x.shape[0], self.ang.numel()
        out = torch.zeros(nb, nview, 1, self.s.nu, device="cuda")
        f = self.L.cupyDistanceDrivenFanProjection if self.fan else self.L.cupyDistanceDrivenParallelProjection
        rc = f(c_void_p(out.data_ptr()), c_void_p(x.data_ptr()), c_void_p(self.ang.data_ptr()),
               *self._geo(nb, self.s.nu, nview), c_int(0))
        assert rc == 0, rc
        return out

    def bp(self, y, fbp=False):
        import torch
        from ctypes import c_int, c_void_p

        nb, nview = y.shape[0], y.shape[1]
        out = torch.zeros(nb, 1, self.s.ny, self.s.nx, device="cuda")
        f = self.L.cupyDistanceDrivenFanBackprojection if self.fan else self.L.cupyDistanceDrivenParallelBackprojection
        rc = f(c_void_p(out.data_ptr()), c_void_p(y.data_ptr()), c_void_p(self.ang.data_ptr()),
               *self._geo(nb, y.shape[3], nview), c_int(1 if fbp else 0))
        assert rc == 0, rc
        return out

    def filt(self, y):
        import torch
        from ctypes import c_float, c_int, c_ulong, c_void_p

        s = self.s
        out = torch.zeros_like(y)
        head = [c_void_p(out.data_ptr()), c_void_p(y.data_ptr()), c_int(y.shape[0]), c_ulong(y.shape[3]),
                c_ulong(y.shape[2]), c_ulong(y.shape[1])]
        if self.fan:  # fan_equiangular.py:19-71, 'hann' = 2
            rc = self.L.cupyfbpFanFilter(*head, c_float(s.du / s.dsd), c_float(s.dv), c_float(s.off_u),
                                         c_float(s.off_v), c_float(s.dsd), c_float(s.dso), c_int(2))
        else:  # parallel.py:19-71
            rc = self.L.cupyfbpParallelFilter(*head, c_float(s.du), c_float(s.dv), c_float(s.off_u), c_float(s.off_v),
                                              c_int(2))
        assert rc == 0, rc
        return out


class _RefCone:
    """The reference library's device-pointer Siddon cone entries for one
    helical protocol, with the argument conventions of its cupy cone module
    (cone.py:15-170): outputs zero-filled per call, both accumulate."""

    def __init__(self, L, scan, cone):
        import torch

        self.L, self.s = L, scan
        self.geo = [torch.tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda") for a in cone]
        self.nview = int(cone[0].shape[0])

    def _args(self):
        from ctypes import c_float, c_ulong, c_void_p

        s = self.s
        return ([c_void_p(g.data_ptr()) for g in self.geo] +
                [c_ulong(1), c_ulong(s.nx), c_ulong(s.ny), c_ulong(s.nz), c_float(s.dx), c_float(s.dy), c_float(s.dz),
                 c_float(s.cx), c_float(s.cy), c_float(s.cz), c_ulong(s.nu), c_ulong(s.nv), c_ulong(self.nview),
                 c_float(s.du), c_float(s.dv), c_float(s.off_u), c_float(s.off_v)])

    def fp(self, x):
        import torch
        from ctypes import c_void_p

        out = torch.zeros(1, self.nview, self.s.nv, self.s.nu, device="cuda")
        rc = self.L.cupySiddonConeProjectionArbitrary(c_void_p(out.data_ptr()), c_void_p(x.data_ptr()), *self._args())
        assert rc == 0, rc
        return out

    def bp(self, y):
        import torch
        from ctypes import c_void_p

        out = torch.zeros(1, self.s.nz, self.s.ny, self.s.nx, device="cuda")
        rc = self.L.cupySiddonConeBackprojectionArbitrary(c_void_p(out.data_ptr()), c_void_p(y.data_ptr()),
                                                          *self._args())
        assert rc == 0, rc
        return out


def _ref_serve_stream(L, T, n_jobs, mix, seed):
    """A served stream of the ours arm (same seeded arrivals, mix and slice
    counts; sinograms made here with the reference's own projectors and the
    same noise model) through the reference's per-call path: its cupy entries
    for FP, BP and the filters and its TV prior (cupyTVSQS3D), FP32, array
    arithmetic in between, one job at a time."""
    import torch
    from ctypes import c_float, c_ulong, c_void_p
    from types import SimpleNamespace

    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.serving import mix as W
    from ctprojector_b200.serving.scheduler import LatencyStats

    protos = {n: SimpleNamespace(**d) for n, d in W.protocol_specs().items()}
    stream = W.arrivals(n_jobs, SERVED_RATE_HZ, seed, mix)
    names = sorted({n for _, n, _ in stream})
    ops = {n: (_RefCone(L, protos[n].scan, protos[n].cone) if protos[n].kind == "cone"
               else _RefDD(L, protos[n].scan, protos[n].kind, protos[n].angles)) for n in names}
    pools = {}
    for i, n in enumerate(names):
        rng = np.random.default_rng(i)
        sc = protos[n].scan
        pools[n] = []
        for _ in range(2):
            if protos[n].kind == "cone":
                vol = S.ellipsoid_phantom(rng, int(sc.nz), int(sc.ny), int(sc.nx), sc.dz, sc.dy, sc.dx,
                                          supersample=1)[None]
                y = ops[n].fp(torch.tensor(vol, device="cuda")).cpu().numpy()
            else:
                img = np.stack([S.ellipse_phantom(rng, sc.nx, sc.ny, sc.dx, sc.dy)[None] for _ in range(16)])
                y = ops[n].fp(torch.tensor(img, device="cuda")).cpu().numpy()
            pools[n].append(torch.tensor(S.poisson_log(y, 1e5, rng)).pin_memory())
    rng = np.random.default_rng(0)
    jobs = [(t, n, nz, pools[n][int(rng.integers(2))] if protos[n].kind == "cone"
             else pools[n][int(rng.integers(2))][:nz]) for t, n, nz in stream]

    def tv(x, w, eps):  # prior/cupy/recon_prior.py:85-135
        s1, s2, var = torch.zeros_like(x), torch.zeros_like(x), torch.zeros_like(x)
        rc = T.cupyTVSQS3D(c_void_p(s1.data_ptr()), c_void_p(s2.data_ptr()), c_void_p(var.data_ptr()),
                           c_void_p(x.data_ptr()), c_float(w[2]), c_float(w[1]), c_float(w[0]), c_ulong(x.shape[0]),
                           c_ulong(x.shape[3]), c_ulong(x.shape[2]), c_ulong(x.shape[1]), c_float(eps))
        assert rc == 0, rc
        return s1, s2

    def reconstruct(n, ysino):
        pr, op = protos[n], ops[n]
        y = ysino.cuda()
        sc = pr.scan
        if pr.algo == "fbp":
            return op.bp(op.filt(y), True).cpu()
        if pr.kind == "cone":
            shape = (1, int(sc.nz), int(sc.ny), int(sc.nx))
            norm = op.bp(op.fp(torch.ones(shape, device="cuda")))
        else:
            shape = (y.shape[0], 1, sc.ny, sc.nx)
            norm = op.bp(op.fp(torch.ones(1, 1, sc.ny, sc.nx, device="cuda")))
        x = torch.zeros(shape, device="cuda")
        vol = (1, -1, int(sc.ny), int(sc.nx))
        for _ in range(pr.n_iter):
            g = op.bp(op.fp(x) - y)
            s1, s2 = tv(x.reshape(vol).contiguous(), pr.tv_weights, pr.eps)
            x = x - (g + pr.beta * s1.reshape(x.shape)) / (norm + pr.beta * s2.reshape(x.shape))
        return x.cpu()

    for n in names:  # first-call costs outside the stream
        reconstruct(n, pools[n][0] if protos[n].kind == "cone" else pools[n][0][:1])
    torch.cuda.synchronize()
    stats = LatencyStats()
    t0 = time.perf_counter()
    for t, n, nz, ysino in jobs:
        wait = t - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        reconstruct(n, ysino)
        torch.cuda.synchronize()
        done = time.perf_counter() - t0
        stats.add(done - t, done)
    sm = stats.summary(0.0)
    r = lambda x: round(x, 3)  # noqa: E731
    return {"recons_per_s": r(sm["recons_per_s"]), "p50_ms": r(sm["p50_ms"]), "p99_ms": r(sm["p99_ms"]),
            "jobs": sm["jobs"], "arrival_rate_hz": SERVED_RATE_HZ, "seed": seed,
            "jobs_by_protocol": {n: sum(1 for _, m, _ in stream if m == n) for n in names},
            "path": "reference libprojector.so + libprior.so (built from its sources for sm_100a), cupy entries, "
                    "FP32, one call per operation, one job at a time"}


def run_reference_served():
    """The served streams of the ours arm through the reference's per-call path."""
    import ctypes

    lp = os.path.join(ROOT, "oracle", "_ref", "libprojector.so")
    tp = os.path.join(ROOT, "oracle", "_ref", "libprior.so")
    if not (os.path.exists(lp) and os.path.exists(tp)):
        return {"unavailable": "oracle/_ref/libprojector.so or libprior.so not built"}
    L, T = ctypes.CDLL(lp), ctypes.CDLL(tp)
    out = _ref_serve_stream(L, T, SERVED_JOBS, _mix("2d"), SERVED_SEED)
    out["with_cone"] = _ref_serve_stream(L, T, SERVED_MIX_JOBS, _mix("all"), SERVED_MIX_SEED)
    return out


# ----------------------------------------------------------------------------- one operation, for profilers
OP_WORKLOADS = {
    "par512x16": "parallel 16 x 512^2 at 0.8 mm, 720 views over pi, 768 cells",
    "fan512x4": "fan 4 x 512^2 at 0.8 mm, 984 views over 2 pi, 888 cells",
    "fan256": "fan 1 x 256^2 at 1.0 mm, 360 views over 2 pi, 736 cells",
    "cone64": "helical cone 1 x 64 x 512^2 at 0.7 x 0.7 x 1.0 mm, 360 views, 736 x 64 panel",
    "tomo64": "tomosynthesis 1 x 64 x 256 x 512 (z, y, x) at 0.4 x 0.4 x 1.0 mm, 25 views over 30 degrees, "
              "1024 x 512 detector of 0.25 mm cells 20 mm below the volume centre, source arc radius 650 mm",
}
OPS = ("fp", "bp", "bp_fbp", "bp_adjoint", "filter", "filter_exact", "siddon_fp", "siddon_bp", "tomo_fp",
       "tomo_bp")


def _op_workload(name):
    from ctprojector_b200 import synthetic as S

    if name == "par512x16":
        scan, ang, nb = S.config2()
        return "parallel", scan, ang, nb
    if name == "fan512x4":
        scan, ang, nb = S.config4()
        return "fan", scan, ang, nb
    if name == "fan256":
        scan, ang, nb = S.config1()
        return "fan", scan, ang, nb
    if name == "cone64":
        scan = S.Scan(512, 512, 64, 0.7, 0.7, 1.0, 736, 64, 1.2858, 1.0, 360)
        geo = S.helical(360, 1.0, scan.dso, scan.dsd, 64 * scan.dso / scan.dsd)
        return "cone", scan, geo, 1
    if name == "tomo64":
        scan = S.Scan(512, 256, 64, 0.4, 0.4, 1.0, 1024, 512, 0.25, 0.25, 25)
        dc, src = S.tomo_geometry(25, 30.0, 650.0, -52.0)
        return "tomo", scan, (dc, src), 1
    raise SystemExit(f"unknown workload {name!r}; one of {sorted(OP_WORKLOADS)}")


def run_op(op: str, workload: str, repeat: int) -> int:
    """One projector operation of a named workload (OP_WORKLOADS) on seeded
    uniform random inputs of its shapes (the cost does not depend on the
    values): once untimed, then ``repeat`` times, so that ``ncu -k <kernel> -s 1
    -c 1`` captures a warm launch."""
    import torch

    from ctprojector_b200.projector import _device as D

    kind, scan, geo, nb = _op_workload(workload)
    rng = np.random.default_rng(0)
    dev = torch.device("cuda")
    u = lambda *shape: torch.tensor(rng.uniform(0, 1, shape).astype(np.float32), device=dev)  # noqa: E731
    if kind in ("tomo", "cone"):
        g = [torch.tensor(x, device=dev) for x in geo]
        img, prj = u(nb, scan.nz, scan.ny, scan.nx), u(nb, len(geo[0]), scan.nv, scan.nu)
        ops = {"tomo_fp": lambda: D.tomo_fp(scan, img, *g), "tomo_bp": lambda: D.tomo_bp(scan, prj, *g)} \
            if kind == "tomo" else \
            {"siddon_fp": lambda: D.siddon_fp(scan, img, *g), "siddon_bp": lambda: D.siddon_bp(scan, prj, *g)}
    else:
        code = 0 if kind == "fan" else 1
        ang = torch.tensor(geo, device=dev)
        img, prj = u(nb, 1, scan.ny, scan.nx), u(nb, len(geo), 1, scan.nu)
        ops = {"fp": lambda: D.dd_fp(scan, img, ang, code),
               "bp": lambda: D.dd_bp(scan, prj, ang, code),
               "bp_fbp": lambda: D.dd_bp(scan, prj, ang, code, is_fbp=True),
               "bp_adjoint": lambda: D.dd_bp(scan, prj, ang, code, adjoint=True),
               "filter": lambda: D.ramp_filter(scan, prj, "hann", code),
               "filter_exact": lambda: D.ramp_filter(scan, prj, "hann", code, exact=True)}
    if op not in ops:
        raise SystemExit(f"op {op!r} is not defined for workload {workload!r}")
    ops[op]()
    times = []
    for _ in range(max(0, repeat)):
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        ops[op]()
        t1.record()
        t1.synchronize()
        times.append(t0.elapsed_time(t1))
    torch.cuda.synchronize()
    tail = f", median {float(np.median(times)):.4f} ms over {len(times)} warm calls (CUDA events)" if times else ""
    print(f"{op} {workload}: ok{tail}")
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream measurement")
    ap.add_argument("--op", choices=OPS, default=None,
                    help="run only this operation of --workload (for profilers) and print no JSON line")
    ap.add_argument("--workload", choices=sorted(OP_WORKLOADS), default="par512x16")
    ap.add_argument("--repeat", type=int, default=1, help="with --op: warm launches after the first")
    args = ap.parse_args(argv)
    if args.op:
        return run_op(args.op, args.workload, args.repeat)
    rank, world, local = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args, rank, world, local)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
    try:
        line = run_ours(args, rank, world, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as tdist

            tdist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
