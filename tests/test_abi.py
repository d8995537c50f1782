"""The C ABI library loads and exports every entry point include/*.h
declares; host-only paths (size checks, error statuses) work without a GPU."""
import ctypes as ct
import pathlib
import re

import pytest

from homogenenousshearturbulence_b200 import hst

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(hst_gpu_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = hst.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bad_sizes_are_rejected_without_a_device():
    p = hst.Params()
    p.nx, p.ny, p.nz = 15, 31, 15           # odd ny: unsupported, refused before any CUDA call
    p.alfa0, p.beta0, p.ly, p.re = 1.0, 1.0, 2.0, 100.0
    h = ct.c_void_p()
    rc = hst.lib().hst_gpu_create(ct.byref(p), ct.byref(h))
    assert rc == -1 and not h.value
    assert hst.lib().hst_gpu_device_bytes(ct.byref(p)) == 0.0


def test_device_bytes_of_the_benchmark_workloads():
    # the 768^2 x 512 workload must fit in one B200's 180 GB with room to spare
    b3 = hst.device_bytes(nx=255, ny=512, nz=256, alfa0=1.0, beta0=1.0, ly=6.283185307179586)
    assert 20e9 < b3 < 60e9
    b1 = hst.device_bytes(nx=31, ny=64, nz=32, alfa0=1.0, beta0=1.0, ly=6.283185307179586)
    assert b1 < 1e9


def test_null_context_calls_fail_cleanly():
    L = hst.lib()
    assert L.hst_gpu_destroy(None) == -1
    assert L.hst_gpu_sync(None) == -1
    assert L.hst_gpu_upload(None, 0, None) == -1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(hst, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(hst, "_lib", None)
    with pytest.raises(hst.HstError):
        hst.lib()


def test_stokes_layer_deck_is_refused(golden):
    """The Stokes-layer forcing is outside the GPU substep: a deck that uses
    it is refused (HstError) before any device work, not run without it."""
    deck = hst.read_deck(golden / "small_stokes.in")
    assert deck["sl_amplitude"] == 0.5
    with pytest.raises(hst.HstError):
        hst.Solver(deck)


def test_async_io_and_noalloc_reject_bad_arguments():
    L = hst.lib()
    assert L.hst_gpu_upload_async(None, 0, None) == -1
    assert L.hst_gpu_download_async(None, 0, None) == -1
    assert L.hst_gpu_wait_io(None) == -1
    f = L.hst_gpu_line_solve_noalloc
    d, i, vp = ct.c_double, ct.c_int, ct.c_void_p
    f.restype = i
    f.argtypes = [i, i, i, d, d, d, i, d, vp, vp, vp, d, d, vp, ct.c_char_p, i]
    msg = ct.create_string_buffer(128)
    # sizes are checked before any CUDA call
    assert f(15, 4096, 15, 1.0, 1.0, 100.0, 1, 1.0, 16, 32, 64, 0.0, 0.0, None, msg, 128) == -1
    assert b"scratch" in msg.value
    assert f(15, 31, 15, 1.0, 1.0, 100.0, 1, 1.0, 16, 32, 64, 0.0, 0.0, None, msg, 128) == -1
    # overlaps of dst with src or with der are refused before any CUDA call
    # (the addresses are never dereferenced)
    field = 16 * 16 * 31 * 36
    base = 1 << 32
    assert f(15, 32, 15, 1.0, 1.0, 100.0, 1, 1.0, base, base + 2 * field, base + 2 * field + 256, 0.0, 0.0, None, msg,
             128) == -1
    assert b"src and dst" in msg.value
    assert f(15, 32, 15, 1.0, 1.0, 100.0, 1, 1.0, base + 2 * field + 1024, base, base + 2 * field, 0.0, 0.0, None,
             msg, 128) == -1
    assert b"der and dst" in msg.value


def test_mixed_precision_rejects_uncompiled_sizes():
    """HST_PREC_MIXED needs 2 nxd and nzd in {96, 192, 384, 768} and ny a
    multiple of 32; anything else is refused before any CUDA call."""
    for nx, ny, nz in ((15, 32, 15), (31, 48, 32), (31, 64, 20)):
        p = hst.Params()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.alfa0, p.beta0, p.ly, p.re = 1.0, 1.0, 2.0, 100.0
        p.precision = hst.PREC_MIXED
        h = ct.c_void_p()
        assert hst.lib().hst_gpu_create(ct.byref(p), ct.byref(h)) == -1 and not h.value
        assert hst.lib().hst_gpu_device_bytes(ct.byref(p)) == 0.0
    p.precision = 7
    assert hst.lib().hst_gpu_device_bytes(ct.byref(p)) == 0.0
