"""The C ABI: libctp.so loads and exports every entry point declared in
include/ctp.h, the ctypes binding covers the same set, and argument checks
answer without touching a GPU."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ctp.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\s*\*)\s+([A-Za-z_]\w*)\s*\(", src, flags=re.M)))


def test_header_declares_reference_entries():
    names = set(declared())
    reference = {
        "SetDevice", "cupyDistanceDrivenFanProjection", "cDistanceDrivenFanProjection",
        "cupyDistanceDrivenParallelProjection", "cDistanceDrivenParallelProjection",
        "cupyDistanceDrivenFanBackprojection", "cDistanceDrivenFanBackprojection",
        "cupyDistanceDrivenParallelBackprojection", "cDistanceDrivenParallelBackprojection",
        "cupyDistanceDrivenTomoProjection", "cDistanceDrivenTomoProjection",
        "cupyDistanceDrivenTomoBackprojection", "cDistanceDrivenTomoBackprojection",
        "cupySiddonConeProjectionArbitrary", "cSiddonConeProjectionArbitrary",
        "cupySiddonConeBackprojectionArbitrary", "cSiddonConeBackprojectionArbitrary",
        "cupyfbpFanFilter", "cfbpFanFilter", "cupyfbpParallelFilter", "cfbpParallelFilter",
        "cupyfbpFanBackprojection", "cfbpFanBackprojection",
    }
    assert reference <= names


def test_library_exports_every_declared_symbol():
    from ctprojector_b200._lib import LIB_PATH

    L = ctypes.CDLL(LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing


def test_binding_matches_header():
    from ctprojector_b200._lib import declared_symbols

    assert sorted(declared_symbols()) == declared()


def test_version_and_error_string():
    from ctprojector_b200._lib import last_error_string, lib

    assert b"sm_100a" in lib().ctpVersion()
    assert isinstance(last_error_string(), str)


def test_null_geometry_is_rejected_on_host():
    from ctprojector_b200._lib import CTP_ERR_INVALID_ARGUMENT, last_error_string, lib

    rc = lib().ctp_dd2d_fp(None, None, None, None, 0, 0, 0, None, 0, None)
    assert rc == CTP_ERR_INVALID_ARGUMENT
    assert "geometry" in last_error_string()


def test_zero_extent_is_rejected_on_host():
    from ctprojector_b200._lib import CTP_ERR_INVALID_ARGUMENT, Geometry, lib

    g = Geometry(1, 0, 4, 1, 1, 1, 1, 0, 0, 0, 8, 1, 4, 1, 1, 0, 0, 1000, 500)
    assert lib().ctp_dd2d_fp(1, 1, 1, ctypes.byref(g), 1, 0, 0, None, 0, None) == CTP_ERR_INVALID_ARGUMENT


def test_workspace_queries_need_no_gpu():
    from ctprojector_b200._lib import Geometry, lib

    g = Geometry(16, 512, 512, 1, 0.8, 0.8, 1, 0, 0, 0, 768, 1, 720, 0.8, 1, 0, 0, 1000, 500)
    fp = lib().ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0)
    assert fp >= 16 * 512 * 512 * 4
    assert lib().ctp_dd2d_bp_workspace(ctypes.byref(g), 1, 0, 0) == 0
    assert lib().ctp_tomo_bp_workspace(ctypes.byref(g)) >= 16 * 720 * 768 * 4


def _align(x, a=256):
    return (x + a - 1) // a * a


def test_bp_workspace_holds_view_parts():
    """One 256 x 256 fan slice gives the fast back projector 64 tiles, fewer
    than the SMs, so its views are split into parts with FP32 partial
    volumes in the workspace (besides the pre-weighted sinogram).  A
    16-slice 256^2 fan stack (512 CTAs of two slices: 1.7 waves of 2 per SM
    on 148 SMs) takes the 4 parts that fill the waves best; the 16-slice
    512^2 parallel batch (1024 CTAs of four slices, 3.5 waves) takes none.
    Host-side sizing only: no GPU."""
    from ctprojector_b200._lib import Geometry, lib

    da = 1.2858 / 1085.6
    one = Geometry(1, 256, 256, 1, 1.0, 1.0, 1, 0, 0, 0, 736, 1, 360, da, 1, 0, 0, 1085.6, 595.0)
    stack = Geometry(16, 256, 256, 1, 1.0, 1.0, 1, 0, 0, 0, 736, 1, 360, da, 1, 0, 0, 1085.6, 595.0)
    pre = 360 * 736 * 4
    assert lib().ctp_dd2d_bp_workspace(ctypes.byref(one), 0, 0, 0) >= pre + 2 * 256 * 256 * 4
    stack_ws = lib().ctp_dd2d_bp_workspace(ctypes.byref(stack), 0, 0, 0)
    assert stack_ws == _align(16 * pre) + _align(4 * 16 * 256 * 256 * 4)
    par = Geometry(16, 512, 512, 1, 0.8, 0.8, 1, 0, 0, 0, 768, 1, 720, 0.8, 1, 0, 0, 1000, 500)
    assert lib().ctp_dd2d_bp_workspace(ctypes.byref(par), 1, 0, 0) == 0


def test_fp_workspace_line_tables_up_to_128_edge_groups():
    """The fast forward projectors serve detectors of up to 128 groups of 31
    cells (3937 cells): their workspace holds the streamed line tables (per
    line of 256 cells, 258 FP64 and 260 FP32 entries; rows and columns of a
    256 x 256 slice); wider detectors take the general kernel, whose
    workspace has none."""
    from ctprojector_b200._lib import Geometry, lib

    def ws(nu):
        g = Geometry(1, 256, 256, 1, 1.0, 1.0, 1, 0, 0, 0, nu, 1, 40, 0.4 / 1085.6, 1, 0, 0, 1085.6, 595.0)
        return lib().ctp_dd2d_fp_workspace(ctypes.byref(g), 0, 0, 0)

    def edge_table(nu, nview=40):
        return (2 * (2 * nview * (nu + 1) + nview * nu) + 5 * nview) * 4

    line_tables = 2 * 256 * (258 * 8 + 260 * 4)
    image = 256 * 256 * 4
    assert ws(3000) >= edge_table(3000) + image + line_tables
    assert ws(4000) < edge_table(4000) + image + line_tables


def test_fp_workspace_follows_the_stream_chunk():
    """The streamed forward projector runs in chunks of slices, each chunk's
    transposed slices and line tables rebuilt in one buffer.  For the
    16-slice 512 x 512, 720-view, 768-cell batch the query returns one chunk
    of all 16 slices; capped at 4 slices per chunk (ctp_set_fp_stream_slices)
    a quarter of that; with the streamed path off (cap 0), the staged
    kernel's edge table and transposed stack.  Host-side sizing only: no GPU."""
    from ctprojector_b200._lib import Geometry, lib

    L = lib()
    nb, n, nview, nu = 16, 512, 720, 768
    g = Geometry(nb, n, n, 1, 0.8, 0.8, 1, 0, 0, 0, nu, 1, nview, 0.8, 1, 0, 0, 1000.0, 500.0)
    edge = _align((2 * (2 * nview * (nu + 1) + nview * nu) + 5 * nview) * 4) + _align(nview * 4)
    line = (n + 2) * 8 + (n + 4) * 4  # FP64 and FP32 entries of one line's table, each padded
    slice_tables = 2 * n * line
    slice_px = n * n * 4

    def stream(chunk):
        return edge + _align(chunk * slice_px) + _align(chunk * slice_tables)

    try:
        assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) == stream(16)
        assert L.ctp_set_fp_stream_slices(4) == 0
        assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) == stream(4)
        assert L.ctp_set_fp_stream_slices(3) == 0  # 16 slices in chunks of at most 3: 6 chunks of 3 or fewer
        assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) == stream(3)
        assert L.ctp_set_fp_stream_slices(0) == 0
        assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) == edge + _align(nb * slice_px)
    finally:
        assert L.ctp_set_fp_stream_slices(-1) == 0
    assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) == stream(16)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import ctprojector_b200._lib as L
    from ctprojector_b200.errors import CTProjectorError

    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "libctp.so"))
    with pytest.raises(CTProjectorError):
        L.lib()


def test_workspace_queries_return_on_degenerate_geometry():
    """The workspace queries run before any geometry validation, so zero
    extents must not send their shape search into an endless loop (checked
    in a child process with a time limit)."""
    import subprocess
    import sys

    code = (
        "from ctypes import byref\n"
        "from ctprojector_b200._lib import Geometry, lib\n"
        "for nu, nview, n in ((0, 90, 64), (96, 0, 64), (96, 90, 0), (0, 0, 0)):\n"
        "    g = Geometry(1, n, n, 1, 1.0, 1.0, 1.0, 0, 0, 0, nu, 1, nview, 1.0, 1.0, 0, 0, 1000.0, 500.0)\n"
        "    for geom in (0, 1):\n"
        "        lib().ctp_dd2d_fp_workspace(byref(g), geom, 0, 0)\n"
        "        lib().ctp_dd2d_bp_workspace(byref(g), geom, 0, 0)\n"
        "print('ok')\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr
