"""Run one projector operation of a named workload, for profilers.

    python -m ctprojector_b200.workloads <op> <workload> [--repeat N]

op: fp, bp, bp_fbp, bp_adjoint, filter, siddon_fp, siddon_bp, tomo_fp, tomo_bp
workload:
  par512x16   parallel 16 x 512^2 at 0.8 mm, 720 views over pi, 768 cells
  fan512x4    fan 4 x 512^2 at 0.8 mm, 984 views over 2 pi, 888 cells
  fan256      fan 1 x 256^2 at 1.0 mm, 360 views over 2 pi, 736 cells
  cone64      helical cone 1 x 64 x 512^2 at 0.7 x 0.7 x 1.0 mm, 360 views, 736 x 64 panel
  tomo64      tomosynthesis 1 x 64 x 256 x 512 (z, y, x) at 0.4 x 0.4 x 1.0 mm, 25 views over 30 degrees,
              1024 x 512 detector of 0.25 mm cells 20 mm below the volume centre, source arc radius 650 mm

Inputs are seeded uniform random arrays of the workload's shapes (the
operations' cost does not depend on the values).  The operation runs once
untimed and then ``--repeat`` times, so ``ncu -k <kernel> -s 1 -c 1`` captures a
warm launch.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def _workload(name):
    from . import synthetic as S

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
    raise SystemExit(f"unknown workload {name!r}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("op")
    ap.add_argument("workload")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)

    import torch

    from .projector import _device as D

    kind, scan, geo, nb = _workload(a.workload)
    rng = np.random.default_rng(0)
    dev = torch.device("cuda")
    if kind == "tomo":
        g = [torch.tensor(x, device=dev) for x in geo]
        img = torch.tensor(rng.uniform(0, 1, (nb, scan.nz, scan.ny, scan.nx)).astype(np.float32), device=dev)
        prj = torch.tensor(rng.uniform(0, 1, (nb, len(geo[0]), scan.nv, scan.nu)).astype(np.float32), device=dev)
        ops = {"tomo_fp": lambda: D.tomo_fp(scan, img, *g), "tomo_bp": lambda: D.tomo_bp(scan, prj, *g)}
    elif kind == "cone":
        g = [torch.tensor(x, device=dev) for x in geo]
        img = torch.tensor(rng.uniform(0, 1, (nb, scan.nz, scan.ny, scan.nx)).astype(np.float32), device=dev)
        prj = torch.tensor(rng.uniform(0, 1, (nb, len(geo[0]), scan.nv, scan.nu)).astype(np.float32), device=dev)
        ops = {"siddon_fp": lambda: D.siddon_fp(scan, img, *g), "siddon_bp": lambda: D.siddon_bp(scan, prj, *g)}
    else:
        code = 0 if kind == "fan" else 1
        ang = torch.tensor(geo, device=dev)
        img = torch.tensor(rng.uniform(0, 1, (nb, 1, scan.ny, scan.nx)).astype(np.float32), device=dev)
        prj = torch.tensor(rng.uniform(0, 1, (nb, len(geo), 1, scan.nu)).astype(np.float32), device=dev)
        ops = {"fp": lambda: D.dd_fp(scan, img, ang, code),
               "bp": lambda: D.dd_bp(scan, prj, ang, code),
               "bp_fbp": lambda: D.dd_bp(scan, prj, ang, code, is_fbp=True),
               "bp_adjoint": lambda: D.dd_bp(scan, prj, ang, code, adjoint=True),
               "filter": lambda: D.ramp_filter(scan, prj, "hann", code)}
    if a.op not in ops:
        raise SystemExit(f"op {a.op!r} is not defined for workload {a.workload!r}")
    for _ in range(1 + max(0, a.repeat)):
        ops[a.op]()
    torch.cuda.synchronize()
    print(f"{a.op} {a.workload}: ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
