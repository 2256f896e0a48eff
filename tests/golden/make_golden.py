"""Generate the golden fixtures tests/golden/*.npz from the reference itself.

Runs the reference projector library -- oracle/_ref/libprojector.so, built
from the reference sources for sm_100a by ``make -f oracle/ref.mk`` -- through
its host-pointer C entries with the argument conventions of its numpy
wrappers (ct_projector/projector/numpy/*.py), on the seeded cases of
cases.py, and stores inputs and outputs.  Needs a GPU:

    python tests/golden/make_golden.py [--out DIR] [--only CASE ...]   # default: tests/golden
    python tests/golden/make_golden.py --branchless [--out DIR]         # branchless_*.npz

This script is test infrastructure; the product never runs the reference.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys
from ctypes import c_float, c_int, c_ulong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libprojector.so")


def ptr(a):
    return c_void_p(a.ctypes.data)


def geom(p, nb, img_shape, prj_shape):
    nz, ny, nx = img_shape
    nview, nv, nu = prj_shape
    return [c_ulong(nb), c_ulong(nx), c_ulong(ny), c_ulong(nz), c_float(p.dx), c_float(p.dy), c_float(p.dz),
            c_float(p.cx), c_float(p.cy), c_float(p.cz), c_ulong(nu), c_ulong(nv), c_ulong(nview)]


class Ref:
    def __init__(self, path):
        self.L = ctypes.CDLL(path)

    def call(self, name, *args):
        f = getattr(self.L, name)
        f.restype = c_int
        rc = f(*args)
        if rc != 0:
            raise RuntimeError(f"{name} returned {rc}")

    # fan_equiangluar.py:241-299
    def dd_fp(self, p, img, ang, fan, type_=0):
        prj = np.zeros([img.shape[0], len(ang), p.nv, p.nu], np.float32)
        if fan:
            self.call("cDistanceDrivenFanProjection", ptr(prj), ptr(img), ptr(ang),
                      *geom(p, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du / p.dsd), c_float(p.dv),
                      c_float(p.off_u), c_float(p.off_v), c_float(p.dsd), c_float(p.dso), c_int(type_))
        else:
            self.call("cDistanceDrivenParallelProjection", ptr(prj), ptr(img), ptr(ang),
                      *geom(p, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                      c_float(p.off_u), c_float(p.off_v), c_int(type_))
        return prj

    # fan_equiangluar.py:302-366, parallel.py:192-254
    def dd_bp(self, p, prj, ang, fan, type_=0):
        img = np.zeros([prj.shape[0], p.nz, p.ny, p.nx], np.float32)
        if fan:
            self.call("cDistanceDrivenFanBackprojection", ptr(img), ptr(prj), ptr(ang),
                      *geom(p, prj.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du / p.dsd), c_float(p.dv),
                      c_float(p.off_u), c_float(p.off_v), c_float(p.dsd), c_float(p.dso), c_int(type_))
        else:
            self.call("cDistanceDrivenParallelBackprojection", ptr(img), ptr(prj), ptr(ang),
                      *geom(p, prj.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                      c_float(p.off_u), c_float(p.off_v), c_int(type_))
        return img

    # fan_equiangluar.py:19-67, parallel.py:20-71
    def ramp(self, p, prj, fan, ifilter):
        out = np.zeros(prj.shape, np.float32)
        nb, nview, nv, nu = prj.shape
        if fan:
            self.call("cfbpFanFilter", ptr(out), ptr(prj), c_int(nb), c_ulong(nu), c_ulong(nv), c_ulong(nview),
                      c_float(p.du / p.dsd), c_float(p.dv), c_float(p.off_u), c_float(p.off_v), c_float(p.dsd),
                      c_float(p.dso), c_int(ifilter))
        else:
            self.call("cfbpParallelFilter", ptr(out), ptr(prj), c_int(nb), c_ulong(nu), c_ulong(nv), c_ulong(nview),
                      c_float(p.du), c_float(p.dv), c_float(p.off_u), c_float(p.off_v), c_int(ifilter))
        return out

    # fan_equiangluar.py:75-123
    def fbp_bp(self, p, prj, ang):
        img = np.zeros([prj.shape[0], p.nz, p.ny, p.nx], np.float32)
        self.call("cfbpFanBackprojection", ptr(img), ptr(prj), ptr(ang),
                  *geom(p, prj.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du / p.dsd), c_float(p.dv),
                  c_float(p.off_u), c_float(p.off_v), c_float(p.dsd), c_float(p.dso))
        return img

    # cone.py:19-93
    def siddon_fp(self, p, img, dc, du, dv, src):
        prj = np.zeros([img.shape[0], dc.shape[0], p.nv, p.nu], np.float32)
        self.call("cSiddonConeProjectionArbitrary", ptr(prj), ptr(img), ptr(dc), ptr(du), ptr(dv), ptr(src),
                  *geom(p, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                  c_float(p.off_u), c_float(p.off_v))
        return prj

    def siddon_bp(self, p, prj, dc, du, dv, src):
        img = np.zeros([prj.shape[0], p.nz, p.ny, p.nx], np.float32)
        self.call("cSiddonConeBackprojectionArbitrary", ptr(img), ptr(prj), ptr(dc), ptr(du), ptr(dv), ptr(src),
                  *geom(p, prj.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                  c_float(p.off_u), c_float(p.off_v))
        return img

    # tomo.py:19-164
    def tomo_fp(self, p, img, dc, src):
        prj = np.zeros([img.shape[0], dc.shape[0], p.nv, p.nu], np.float32)
        self.call("cDistanceDrivenTomoProjection", ptr(prj), ptr(img), ptr(dc), ptr(src),
                  *geom(p, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                  c_float(p.off_u), c_float(p.off_v), c_int(0))
        return prj

    def tomo_bp(self, p, prj, dc, src):
        img = np.zeros([prj.shape[0], p.nz, p.ny, p.nx], np.float32)
        self.call("cDistanceDrivenTomoBackprojection", ptr(img), ptr(prj), ptr(dc), ptr(src),
                  *geom(p, prj.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                  c_float(p.off_u), c_float(p.off_v), c_int(0))
        return img


    # fan_equiangluar.py:131-238 (numpy module): nBatches passed as an unsigned long
    def siddon_fan(self, p, x, ang, fp):
        if fp:
            out = np.zeros([x.shape[0], len(ang), p.nv, p.nu], np.float32)
            shapes = (x.shape[1:], out.shape[1:])
        else:
            out = np.zeros([x.shape[0], p.nz, p.ny, p.nx], np.float32)
            shapes = (out.shape[1:], x.shape[1:])
        self.call("cSiddonFanProjection" if fp else "cSiddonFanBackprojection", ptr(out), ptr(x), ptr(ang),
                  *geom(p, x.shape[0], *shapes), c_float(p.du / p.dsd), c_float(p.dv), c_float(p.off_u),
                  c_float(p.off_v), c_float(p.dsd), c_float(p.dso))
        return out

    # parallel.py:75-130 (numpy module)
    def pixel_bp(self, p, prj, ang):
        img = np.zeros([prj.shape[0], p.nz, p.ny, p.nx], np.float32)
        self.call("cfbpParallelBackprojection", ptr(img), ptr(prj), ptr(ang),
                  *geom(p, prj.shape[0], img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv),
                  c_float(p.off_u), c_float(p.off_v), c_int(0))
        return img

    # tomo.py:157-221: the reference has only the device entry, called with device buffers
    def tomo_filter(self, p, prj, dc, src, ifilter, cutoff_x, cutoff_z):
        import torch

        t = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
        dp, ddc, dsr = t(prj), t(dc), t(src)
        out = torch.zeros_like(dp)
        self.call("cupyFbpTomoFilter", c_void_p(out.data_ptr()), c_void_p(dp.data_ptr()), c_void_p(ddc.data_ptr()),
                  c_void_p(dsr.data_ptr()), c_ulong(prj.shape[0]), c_ulong(prj.shape[3]), c_ulong(prj.shape[2]),
                  c_ulong(prj.shape[1]), c_float(p.du), c_float(p.dx), c_float(p.dz), c_int(ifilter),
                  c_float(cutoff_x), c_float(cutoff_z))
        torch.cuda.synchronize()
        return out.cpu().numpy()


TOMO_FILTERS = (("hann", 2, 1.0, 1.0), ("hamming_cut", 1, 0.8, 0.6), ("ramlak", 0, 1.0, 1.0))


def run_case(ref: Ref, fn):
    name, p, inp = fn()
    out = {}
    if name in ("fan_basic", "fan_offsets", "par_basic", "par_offsets", "par_wide", "fan_45", "fan_wide"):
        fan = name.startswith("fan")
        img, ang = inp["img"], inp["angles"]
        prj = ref.dd_fp(p, img, ang, fan)
        out["fp"] = prj
        out["bp"] = ref.dd_bp(p, prj, ang, fan, 0)
        for fname, code in (("hann", 2), ("hamming", 1), ("cosine", 3), ("ramlak", 0)):
            out[f"filter_{fname}"] = ref.ramp(p, prj, fan, code)
        out["bp_fbp"] = ref.dd_bp(p, out["filter_hann"], ang, fan, 1)
        if fan:
            out["fbp_bp"] = ref.fbp_bp(p, out["filter_hann"], ang)
            out["siddon_fp"] = ref.siddon_fan(p, img, ang, True)
            out["siddon_bp"] = ref.siddon_fan(p, out["siddon_fp"], ang, False)
        else:
            out["pixel_bp"] = ref.pixel_bp(p, out["filter_hann"], ang)
    elif name == "kat":
        out["fp"] = ref.dd_fp(p, inp["img"], inp["angles"], False)
        out["bp_fbp"] = ref.dd_bp(p, inp["prj"], inp["angles"], False, 1)
    elif name == "siddon":
        a = (inp["det_center"], inp["det_u"], inp["det_v"], inp["src"])
        prj = ref.siddon_fp(p, inp["img"], *a)
        out["fp"] = prj
        out["bp"] = ref.siddon_bp(p, prj, *a)
    elif name == "tomo":
        prj = ref.tomo_fp(p, inp["img"], inp["det_center"], inp["src"])
        out["fp"] = prj
        out["bp"] = ref.tomo_bp(p, prj, inp["det_center"], inp["src"])
        for fname, code, cx, cz in TOMO_FILTERS:
            out[f"filter_{fname}"] = ref.tomo_filter(p, prj, inp["det_center"], inp["src"], code, cx, cz)
    geom_attrs = {f"geom_{k}": np.asarray(v) for k, v in p.as_dict().items()}
    return name, {**{f"in_{k}": v for k, v in inp.items()}, **{f"ref_{k}": v for k, v in out.items()}, **geom_attrs}


# the branchless distance-driven modes (typeProjector bit 1 of the 2D entries,
# distanceDriven2D.cu:18-19; typeProjector 1 of the tomo entries, which the
# reference's tomo modules set for branchless=True, tomo.py:48-51)
BRANCHLESS_CASES = ("fan_basic", "fan_offsets", "par_basic", "par_offsets", "par_wide", "fan_wide", "tomo")


def run_branchless(ref: Ref, fn):
    """The reference's branchless outputs on a case's inputs.  Tomo: batch item
    0 only, and the back projection of one view, because the reference's tomo
    branchless path indexes a one-item accumulation buffer by the batch item
    (distanceDriven3DBranchless.cu:209) and pre-weights only view 0
    (distanceDriven3DBranchless.cu:347)."""
    name, p, inp = fn()
    out = {}
    if name == "tomo":
        img = inp["img"][:1]
        dc, src = inp["det_center"], inp["src"]
        prj = np.zeros([1, dc.shape[0], p.nv, p.nu], np.float32)
        ref.call("cDistanceDrivenTomoProjection", ptr(prj), ptr(img), ptr(dc), ptr(src),
                 *geom(p, 1, img.shape[1:], prj.shape[1:]), c_float(p.du), c_float(p.dv), c_float(p.off_u),
                 c_float(p.off_v), c_int(1))
        out["fp"] = prj
        dc1, src1 = np.ascontiguousarray(dc[:1]), np.ascontiguousarray(src[:1])
        prj1 = np.ascontiguousarray(prj[:, :1])
        bimg = np.zeros([1, p.nz, p.ny, p.nx], np.float32)
        ref.call("cDistanceDrivenTomoBackprojection", ptr(bimg), ptr(prj1), ptr(dc1), ptr(src1),
                 *geom(p, 1, bimg.shape[1:], prj1.shape[1:]), c_float(p.du), c_float(p.dv), c_float(p.off_u),
                 c_float(p.off_v), c_int(1))
        out["bp_view0"] = bimg
        inp = dict(inp, img=img)
    else:
        fan = name.startswith("fan")
        img, ang = inp["img"], inp["angles"]
        prj = ref.dd_fp(p, img, ang, fan, 2)
        out["fp"] = prj
        out["bp"] = ref.dd_bp(p, prj, ang, fan, 2)
        out["bp_fbp"] = ref.dd_bp(p, prj, ang, fan, 3)
    geom_attrs = {f"geom_{k}": np.asarray(v) for k, v in p.as_dict().items()}
    return f"branchless_{name}", {**{f"in_{k}": v for k, v in inp.items()},
                                  **{f"ref_{k}": v for k, v in out.items()}, **geom_attrs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--only", nargs="*", default=None, help="case names to (re)generate")
    ap.add_argument("--branchless", action="store_true", help="write the branchless fixtures only")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    ref = Ref(REF_LIB)
    for fn in cases.ALL:
        if a.only and fn.__name__[5:] not in a.only:
            continue
        if a.branchless:
            if fn.__name__[5:] not in BRANCHLESS_CASES:
                continue
            name, arrays = run_branchless(ref, fn)
        else:
            name, arrays = run_case(ref, fn)
        path = os.path.join(a.out, f"{name}.npz")
        np.savez_compressed(path, **arrays)
        print(f"wrote {path}: " + ", ".join(f"{k}{list(v.shape)}" for k, v in arrays.items() if k.startswith("ref_")))


if __name__ == "__main__":
    main()
