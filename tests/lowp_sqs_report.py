"""Per-iterate error of reduced-precision SQS-TV against the FP64 oracle.

The reduced-precision fan workload: 512 x 512 slices at 0.8 mm, 984 views over
2 pi, 888 cells (SID 595, SDD 1085.6), seeded ellipse phantoms, Poisson noise
at 2e4 photons before -log.  50 SQS-TV iterations from zero run on the GPU
with the measured sinogram and the image copy read by the forward projector
stored in fp32, bf16 or fp16; projections, back projections, the TV terms and
the iterate itself are accumulated and kept in FP32.  Every iterate is
compared with the same iterate of the FP64 oracle reconstruction of the
float32 sinogram (so the storage rounding of the input counts as error).

    python tests/lowp_sqs_report.py [--slices 1] [--iters 50] [--json out.json]

Test infrastructure (it runs the oracle); needs a CUDA device.
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


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--slices", type=int, default=1)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--json", default=None)
    args = ap.parse_args(argv)

    import torch

    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.projector import _device as D
    from oracle import oracle as O
    from oracle import recon as R

    O.build()
    scan, ang, _ = S.config4()
    rng = np.random.default_rng(S.seed_for(4, 0))
    img = np.stack([S.ellipse_phantom(rng, scan.nx, scan.ny, scan.dx, scan.dy)[None] for _ in range(args.slices)])
    p = D.dd_fp(scan, torch.tensor(img, device="cuda"), torch.tensor(ang, device="cuda"), 0).cpu().numpy()
    y32 = S.poisson_log(p, PHOTONS, rng)

    t0 = time.perf_counter()
    ref = {}
    R.sqs_tv(scan, "fan", y32.astype(np.float64), ang, args.iters, BETA, WEIGHTS, EPS,
             callback=lambda k, x: ref.__setitem__(k, x.copy()))
    t_oracle = time.perf_counter() - t0
    rows = {}
    for storage in STORAGES:
        its = gpu_iterates(scan, ang, y32, storage, args.iters)
        rows[storage] = [(float(np.linalg.norm(x - ref[k + 1]) / np.linalg.norm(ref[k + 1])),
                          float(np.abs(x - ref[k + 1]).max())) for k, x in enumerate(its)]
    peak = float(max(np.abs(ref[args.iters]).max(), 1e-30))
    print(f"# reduced-precision SQS-TV, fan 512^2, 984 views, 888 cells, {args.slices} slice(s), "
          f"{args.iters} iterations; FP64 oracle {t_oracle:.0f} s; max |x| of the last oracle iterate {peak:.4g}")
    print("| iterate | fp32 rel L2 | fp32 max abs | bf16 rel L2 | bf16 max abs | fp16 rel L2 | fp16 max abs |")
    print("|---|---|---|---|---|---|---|")
    for k in range(args.iters):
        cells = " | ".join(f"{rows[s][k][0]:.3e} | {rows[s][k][1]:.3e}" for s in STORAGES)
        print(f"| {k + 1} | {cells} |")
    if args.json:
        with open(args.json, "w") as f:
            json.dump({"iters": args.iters, "slices": args.slices, "peak": peak, "rows": rows}, f)
    return 0


if __name__ == "__main__":
    sys.exit(main())
