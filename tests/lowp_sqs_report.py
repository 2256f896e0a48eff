"""Per-iterate error of reduced-precision SQS-TV against the FP64 oracle.

The reduced-precision fan workload: 512 x 512 slices at 0.8 mm, 984 views over
2 pi, 888 cells (SID 595, SDD 1085.6), seeded ellipse phantoms, Poisson noise
at 2e4 photons before -log.  50 SQS-TV iterations from zero run on the GPU
with the measured sinogram and the image copy read by the forward projector
stored in fp32, bf16 or fp16; projections, back projections, the TV terms and
the iterate itself are accumulated and kept in FP32.  Every iterate is
compared with the same iterate of the FP64 oracle reconstruction of the
float32 sinogram (so the storage rounding of the input counts as error).

The views start half a view step past 0, so none lies exactly on a 45 degree
diagonal (there the reference's axis switch, which the GPU kernels replay with
the same fast intrinsics, and the oracle's exact trigonometry may pick
different axes; that case is tested separately).

    python tests/lowp_sqs_report.py [--slices 1] [--iters 50] [--json out.json]
    python tests/lowp_sqs_report.py --oracle-out ref.npz    # CPU only: data + FP64 iterates
    python tests/lowp_sqs_report.py --oracle-in ref.npz     # GPU part against saved iterates

Test infrastructure (it runs the oracle); the GPU part needs a CUDA device.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

BETA, EPS, WEIGHTS = 2e-4, 1e-6, (1.0, 1.0, 1.0)
PHOTONS = 2e4
STORAGES = ("float32", "bfloat16", "float16")


def gpu_iterates(scan, ang, y32, storage, iters):
    """Every iterate of the GPU SQS-TV loop with the given storage type."""
    import torch

    from ctprojector_b200.projector import _device as D
    from ctprojector_b200.recon import sqs_tv_update

    dt = {"float32": torch.float32, "bfloat16": torch.bfloat16, "float16": torch.float16}[storage]
    ns = y32.shape[0]
    tang = torch.tensor(ang, device="cuda")
    y = torch.tensor(y32, device="cuda").to(dt)
    one = torch.ones(1, 1, scan.ny, scan.nx, device="cuda")
    norm = D.dd_bp(scan, D.dd_fp(scan, one, tang, 0), tang, 0).reshape(1, scan.ny, scan.nx).contiguous()
    zl = torch.zeros(ns, dtype=torch.uint8, device="cuda")
    if ns > 1:
        zl[1:] |= 1
        zl[:-1] |= 2
    x = torch.zeros(ns, 1, scan.ny, scan.nx, device="cuda")
    xlp = x.to(dt) if dt != torch.float32 else None
    out = []
    for _ in range(iters):
        fp = D.dd_fp(scan, xlp if xlp is not None else x, tang, 0, dtype=torch.float32)
        fp.sub_(y)
        bp = D.dd_bp(scan, fp, tang, 0)
        x = sqs_tv_update(x, bp, norm, BETA, WEIGHTS, EPS, zlink=zl, x_lp=xlp)
        out.append(x.reshape(ns, scan.ny, scan.nx).cpu().numpy().astype(np.float64))
    return out


def angles(nview):
    import numpy as np

    from ctprojector_b200 import synthetic as S

    return (S.angles(nview, 2 * np.pi) + np.float32(np.pi / nview)).astype(np.float32)


def oracle_part(slices, iters):
    """Seeded phantom, FP64 projection with Poisson noise, and every iterate of
    the FP64 oracle reconstruction (float32 copies)."""
    from ctprojector_b200 import synthetic as S
    from oracle import oracle as O
    from oracle import recon as R

    O.build()
    scan, _, _ = S.config4()
    ang = angles(scan.nview)
    rng = np.random.default_rng(S.seed_for(4, 0))
    img = np.stack([S.ellipse_phantom(rng, scan.nx, scan.ny, scan.dx, scan.dy)[None] for _ in range(slices)])
    p = O.dd_fp(R._proj2d(scan), img.astype(np.float64), ang, "fan")
    y32 = S.poisson_log(p, PHOTONS, rng)
    its = []
    t0 = time.perf_counter()
    R.sqs_tv(scan, "fan", y32.astype(np.float64), ang, iters, BETA, WEIGHTS, EPS,
             callback=lambda k, x: its.append(x.astype(np.float32)))
    return y32, np.stack(its), ang, time.perf_counter() - t0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--slices", type=int, default=1)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--json", default=None)
    ap.add_argument("--oracle-out", default=None, help="compute the oracle part only and save it here")
    ap.add_argument("--oracle-in", default=None, help="read the oracle part saved by --oracle-out")
    args = ap.parse_args(argv)

    from ctprojector_b200 import synthetic as S

    if args.oracle_in:
        z = np.load(args.oracle_in)
        y32, ref_its, ang, t_oracle = z["y32"], z["iterates"], z["angles"], float(z["seconds"])
    else:
        y32, ref_its, ang, t_oracle = oracle_part(args.slices, args.iters)
        if args.oracle_out:
            np.savez(args.oracle_out, y32=y32, iterates=ref_its, angles=ang, seconds=t_oracle)
            print(f"saved {args.oracle_out}: {ref_its.shape[0]} iterates, oracle {t_oracle:.0f} s")
            return 0
    iters, slices = ref_its.shape[0], y32.shape[0]
    scan, _, _ = S.config4()
    ref = {k + 1: ref_its[k].astype(np.float64) for k in range(iters)}
    rows = {}
    for storage in STORAGES:
        its = gpu_iterates(scan, ang, y32, storage, iters)
        rows[storage] = [(float(np.linalg.norm(x - ref[k + 1]) / np.linalg.norm(ref[k + 1])),
                          float(np.abs(x - ref[k + 1]).max())) for k, x in enumerate(its)]
    peak = float(max(np.abs(ref[iters]).max(), 1e-30))
    print(f"# reduced-precision SQS-TV, fan 512^2, 984 views (half-step offset), 888 cells, {slices} slice(s), "
          f"{iters} iterations; FP64 oracle {t_oracle:.0f} s; max |x| of the last oracle iterate {peak:.4g}")
    print("| iterate | fp32 rel L2 | fp32 max abs | bf16 rel L2 | bf16 max abs | fp16 rel L2 | fp16 max abs |")
    print("|---|---|---|---|---|---|---|")
    for k in range(iters):
        cells = " | ".join(f"{rows[s][k][0]:.3e} | {rows[s][k][1]:.3e}" for s in STORAGES)
        print(f"| {k + 1} | {cells} |")
    if args.json:
        with open(args.json, "w") as f:
            json.dump({"iters": iters, "slices": slices, "peak": peak, "rows": rows}, f)
    return 0


if __name__ == "__main__":
    sys.exit(main())
