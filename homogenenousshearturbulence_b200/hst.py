"""Python host side of the hst substep on a B200: a thin ctypes binding of the
C ABI in include/hst_gpu.h (libhst_gpu.so, built in this directory), with the
names and argument meanings of the reference's Fortran interfaces:

  Solver.timestep()                          hst_equations::timestep (src/hst_equations.f90:56-87)
  Solver.line_solve(kind, lam, src, dst)     hst_linsolve::line_solve (src/hst_linsolve.f90:147-233)
  Solver.fill_ghosts(field[, sx, sz])        hst_derivatives::fill_ghosts[_field] (:134-157)
  Solver.compute_cfl()                       hst_transforms::compute_cfl (src/hst_transforms.f90:163-179)
  Solver.shear_shifts(t), s2_of, s2_integral hst_derivatives (:85-128)

Fields are numpy complex128 arrays of shape (nx+1, 2nz+1, ny+4), i.e. the
reference's V(iy, iz, ix) with iy fastest.  There is no CPU fallback: the
library must be built (build.py) and a CUDA device present.
"""
from __future__ import annotations

import ctypes as ct
import math
import os
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
# HST_GPU_LIB: another build of the library (e.g. one compiled with other
# launch bounds, to compare); the in-tree build by default
LIB_PATH = pathlib.Path(os.environ.get("HST_GPU_LIB", str(PKG / "libhst_gpu.so")))

V1, V2, V3, OLD1, OLD2, RHS1, RHS2 = range(7)
KIND_D2V, KIND_ETA, KIND_POISSON, KIND_D0, KIND_DY = 1, 2, 3, 4, 5
# transform buffers of the per-piece path, FFT kinds, layout changes (include/hst_gpu.h)
BUF_VVDZ, BUF_VVDX, BUF_VVDP = 0, 1, 2
FFT_FFT, FFT_IFT, FFT_RFT, FFT_HFT = 1, 2, 3, 4
Z_TO_X, X_TO_Z = 0, 1


def id_buf(buf, m):
    """the registry id of component m (1..3) of a transform buffer"""
    return 8 + 3 * buf + m - 1


# RK_rai (src/hst_params.f90:108-111), one row per substep
RK_RAI = ((120.0 / 32.0, 2.0, 0.0), (120.0 / 8.0, 50.0 / 8.0, 34.0 / 8.0), (120.0 / 20.0, 90.0 / 20.0, 50.0 / 20.0))
PI = 3.141592653589793


class HstError(RuntimeError):
    """A failed call of the C ABI; `code` is its HST_E* status (0 when the
    failure was found on the host side of this module)."""

    def __init__(self, msg, code=0):
        super().__init__(msg)
        self.code = code


# status classes (include/hst_gpu.h)
EARG, ENOMEM, ECUDA, ETIMEOUT, EFINITE = -1, -2, -3, -4, -5


class Params(ct.Structure):
    """hst_gpu_params (include/hst_gpu.h)."""
    _fields_ = [
        ("nx", ct.c_int), ("ny", ct.c_int), ("nz", ct.c_int),
        ("nxd", ct.c_int), ("nzd", ct.c_int),
        ("alfa0", ct.c_double), ("beta0", ct.c_double), ("ly", ct.c_double), ("ystretch", ct.c_double),
        ("re", ct.c_double), ("S", ct.c_double),
        ("linear", ct.c_int), ("exact_shift", ct.c_int),
        ("s2_mean", ct.c_double), ("s2_amplitude", ct.c_double), ("s2_period", ct.c_double), ("s2_start", ct.c_double),
        ("damp_kpar", ct.c_double), ("damp_kperp", ct.c_double), ("damp_rate", ct.c_double),
        ("damp_edge", ct.c_double), ("damp_norm", ct.c_double), ("damp_angle", ct.c_double),
        ("damp_hard", ct.c_int), ("damp_mean", ct.c_int), ("damp_follow", ct.c_int),
        ("device", ct.c_int),
        ("precision", ct.c_int),
    ]


_lib = None


def lib():
    """Loads libhst_gpu.so; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise HstError(f"{LIB_PATH} is missing: build it with `python -m homogenenousshearturbulence_b200.build`")
        L = ct.CDLL(str(LIB_PATH))
        P = ct.POINTER
        d, i, vp = ct.c_double, ct.c_int, ct.c_void_p
        sig = {
            "hst_gpu_create": (i, [P(Params), P(vp)]),
            "hst_gpu_create_batch": (i, [P(Params), i, P(vp)]),
            "hst_gpu_select_member": (i, [vp, i]),
            "hst_gpu_members": (i, [vp]),
            "hst_gpu_destroy": (i, [vp]),
            "hst_gpu_last_error": (ct.c_char_p, [vp]),
            "hst_gpu_device_bytes": (d, [P(Params)]),
            "hst_gpu_set_tables": (i, [vp, P(d), P(d), P(d)]),
            "hst_gpu_get_tables": (i, [vp, P(d), P(d), P(d)]),
            "hst_gpu_upload": (i, [vp, i, P(d)]),
            "hst_gpu_download": (i, [vp, i, P(d)]),
            "hst_gpu_timestep": (i, [vp, P(d), d, P(d)]),
            "hst_gpu_timesteps": (i, [vp, i, P(d), d]),
            "hst_gpu_line_solve": (i, [vp, i, d, i, i, i, d, d, d]),
            "hst_gpu_fill_ghosts": (i, [vp, i, d, d]),
            "hst_gpu_fill_ghosts_at": (i, [vp, i, d]),
            "hst_gpu_compute_cfl": (i, [vp, P(d)]),
            "hst_gpu_sync": (i, [vp]),
            "hst_gpu_shear_shifts": (i, [vp, d, P(d), P(d)]),
            "hst_gpu_s2_of": (d, [vp, d]),
            "hst_gpu_s2_integral": (d, [vp, d, d]),
            "hst_gpu_launch_count": (ct.c_longlong, [vp]),
            "hst_gpu_set_profiling": (i, [vp, i]),
            "hst_gpu_kernel_times": (i, [vp, P(d), P(ct.c_longlong)]),
            "hst_gpu_reset_kernel_times": (i, [vp]),
            "hst_gpu_stream": (vp, [vp]),
            "hst_gpu_upload_async": (i, [vp, i, vp]),
            "hst_gpu_download_async": (i, [vp, i, vp]),
            "hst_gpu_wait_io": (i, [vp]),
            "hst_gpu_outstats": (i, [vp, d, P(d)]),
            "hst_gpu_outstats_sums": (i, [vp, d, P(d), P(d)]),
            "hst_gpu_fft": (i, [vp, i, i]),
            "hst_gpu_transpose": (i, [vp, i, i]),
            "hst_gpu_transform_to_physical": (i, [vp]),
            "hst_gpu_build_products": (i, [vp, i]),
            "hst_gpu_products_to_spectral": (i, [vp]),
            "hst_gpu_vvdz_to_field": (i, [vp, i, i]),
            "hst_gpu_buildrhs_prepare": (i, [vp, P(d), d, d]),
            "hst_gpu_buildrhs": (i, [vp, P(d), i]),
            "hst_gpu_damping_update": (i, [vp, d]),
            "hst_gpu_damping_mask": (i, [vp]),
            "hst_gpu_shear_shift": (i, [vp, d, d]),
            "hst_gpu_linsolve": (i, [vp, d, d]),
            "hst_gpu_buffer_upload": (i, [vp, i, i, vp]),
            "hst_gpu_buffer_download": (i, [vp, i, i, vp]),
            "hst_gpu_buffer_pointer": (i, [vp, i, P(vp), P(ct.c_size_t)]),
            "hst_gpu_register_host": (i, [vp, vp, ct.c_size_t, i]),
            "hst_gpu_unregister_host": (i, [vp, vp]),
            "hst_gpu_host_id": (i, [vp, vp]),
            "hst_gpu_upload_host": (i, [vp, vp]),
            "hst_gpu_download_host": (i, [vp, vp]),
            "hst_gpu_line_solve_host": (i, [vp, i, d, vp, vp, i, d, d, d]),
            "hst_gpu_fill_ghosts_host": (i, [vp, vp, d, d]),
            "hst_gpu_vvdz_to_field_host": (i, [vp, vp, i]),
            "hst_gpu_pressure": (i, [vp, d, i]),
            "hst_gpu_autotune": (i, [vp, d, i, ct.c_char_p, i]),
            "hst_gpu_write_restart": (i, [vp, ct.c_char_p, d, d, d, d, d]),
            "hst_gpu_read_restart": (i, [vp, ct.c_char_p, P(d)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


# ------------------------------------------------------------------ deck ----
DECK_DEFAULTS = dict(  # src/hst_input.f90:26-42
    nx=63, ny=128, nz=63, alfa0=2.0 * PI / 3.0, beta0=2.0 * PI, ly=2.0, ystretch=0.0,
    re=1000.0, S=1.0, linear=False, exact_shift=False,
    s2_mean=0.0, s2_amplitude=0.0, s2_period=0.0, s2_start=0.0,
    deltat=0.0, cflmax=1.0, t_max=100.0, nstep=1000000, time=0.0,
    amplitude=1.0e-3, seed=1, kpeak=4.0,
    damp_kpar=0.0, damp_kperp=0.0, damp_rate=0.0, damp_hard=False, damp_edge=0.0, damp_norm=2.0,
    damp_mean=False, damp_follow=True, damp_angle=0.0,
    # the Stokes-layer forcing (src/hst_input.f90, &physics sl_*): read so
    # that a deck using it is refused, not run without it
    sl_amplitude=0.0, sl_period=0.0, sl_delta=0.0, sl_start=0.0, sl_bodyforce=False, sl_ramp=False,
)
PREC_FP64, PREC_MIXED = 0, 1  # hst_gpu_params.precision


def read_deck(path) -> dict:
    """Reads the namelist groups of an hst.in deck (the subset the path uses)."""
    text = []
    for line in pathlib.Path(path).read_text().splitlines():
        out, q = [], None
        for ch in line:
            if ch in "'\"":
                q = None if q == ch else (ch if q is None else q)
            if ch == "!" and q is None:
                break
            out.append(ch)
        text.append("".join(out))
    body = "\n".join(text)
    deck = dict(DECK_DEFAULTS)
    keys = {k.lower(): k for k in deck}
    for grp in body.split("&")[1:]:
        grp = grp.split("/")[0]
        parts = grp.split(None, 1)
        if len(parts) < 2:
            continue
        items = parts[1]
        import re as _re
        for m in _re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*=\s*('[^']*'|\"[^\"]*\"|[^,\n]+)", items):
            k, v = m.group(1).lower(), m.group(2).strip()
            if k not in keys:
                continue
            name = keys[k]
            ref = DECK_DEFAULTS[name]
            if isinstance(ref, bool):
                deck[name] = v.lower().strip(".") in ("true", "t")
            elif isinstance(ref, int):
                deck[name] = int(float(v.replace("d", "e").replace("D", "e")))
            elif isinstance(ref, float):
                deck[name] = float(v.replace("d", "e").replace("D", "e"))
            else:
                deck[name] = v.strip("'\"")
    return deck


def fft_fit(n: int) -> bool:
    """A power of two times at most one factor three (src/hst_input.f90:107-115)."""
    j = n
    while j % 2 == 0:
        j //= 2
    return j in (1, 3)


def padded_sizes(nx, nz, nxd=0, nzd=0):
    """nxd, nzd as read_input derives them (src/hst_input.f90:97-98)."""
    if nxd <= 0:
        nxd = 3 * (nx + 1) // 2
        while not fft_fit(nxd):
            nxd += 1
    if nzd <= 0:
        nzd = 3 * nz
        while not fft_fit(nzd):
            nzd += 1
    return nxd, nzd


# --------------------------------------------------------------- solver ----
class Solver:
    """One field resident on one GPU (one hst_ctx); with members > 1 an
    ensemble of independent realisations of the deck advanced together
    (hst_gpu_create_batch): timestep() runs every member, and the field calls
    act on the member chosen with select()."""

    def __init__(self, deck: dict | None = None, device: int = 0, members: int = 1, **kw):
        cfg = dict(DECK_DEFAULTS)
        if deck:
            cfg.update(deck)
        cfg.update(kw)
        if float(cfg.get("sl_amplitude", 0.0)) != 0.0:
            raise HstError("the Stokes-layer forcing (sl_amplitude != 0) is not part of the GPU substep")
        self.cfg = cfg
        p = Params()
        p.nx, p.ny, p.nz = int(cfg["nx"]), int(cfg["ny"]), int(cfg["nz"])
        p.nxd, p.nzd = int(cfg.get("nxd", 0)), int(cfg.get("nzd", 0))
        p.alfa0, p.beta0, p.ly, p.ystretch = cfg["alfa0"], cfg["beta0"], cfg["ly"], cfg["ystretch"]
        p.re, p.S = cfg["re"], cfg["S"]
        p.linear, p.exact_shift = int(bool(cfg["linear"])), int(bool(cfg["exact_shift"]))
        p.s2_mean, p.s2_amplitude = cfg["s2_mean"], cfg["s2_amplitude"]
        p.s2_period, p.s2_start = cfg["s2_period"], cfg["s2_start"]
        p.damp_kpar, p.damp_kperp, p.damp_rate = cfg["damp_kpar"], cfg["damp_kperp"], cfg["damp_rate"]
        p.damp_edge, p.damp_norm, p.damp_angle = cfg["damp_edge"], cfg["damp_norm"], cfg["damp_angle"]
        p.damp_hard, p.damp_mean, p.damp_follow = int(bool(cfg["damp_hard"])), int(bool(cfg["damp_mean"])), int(
            bool(cfg["damp_follow"]))
        p.device = int(device)
        prec = cfg.get("precision", PREC_FP64)
        p.precision = {"fp64": PREC_FP64, "mixed": PREC_MIXED}.get(prec, prec) if isinstance(prec, str) else int(prec)
        self.params = p
        self._h = ct.c_void_p()
        self.members = int(members)
        if self.members > 1:
            rc = lib().hst_gpu_create_batch(ct.byref(p), self.members, ct.byref(self._h))
        else:
            rc = lib().hst_gpu_create(ct.byref(p), ct.byref(self._h))
        if rc != 0:
            raise HstError(f"hst_gpu_create failed ({rc}) for nx={p.nx} ny={p.ny} nz={p.nz}", rc)
        self.nx, self.ny, self.nz = p.nx, p.ny, p.nz
        self.nxd, self.nzd = padded_sizes(p.nx, p.nz, p.nxd, p.nzd)
        self.shape = (self.nx + 1, 2 * self.nz + 1, self.ny + 4)
        self.time = float(cfg.get("time", 0.0))
        self.deltat = float(cfg.get("deltat", 0.0))
        self.cfl = 0.0
        self._tables()

    def _tables(self):
        ny = self.ny
        der = np.zeros(20 * ny)
        y = np.zeros(ny + 4)
        dyl = np.zeros(ny)
        P = ct.POINTER(ct.c_double)
        lib().hst_gpu_get_tables(self._h, der.ctypes.data_as(P), y.ctypes.data_as(P), dyl.ctypes.data_as(P))
        self.der = der.reshape(5, 4, ny)  # der[j+2, n, iy] = der(iy, n, j)
        self.y = y
        self.dyl = dyl

    def select(self, member: int):
        """the member the field calls act on (an ensemble context)"""
        self._check(lib().hst_gpu_select_member(self._h, int(member)), "select_member")

    def close(self):
        if self._h:
            lib().hst_gpu_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            msg = lib().hst_gpu_last_error(self._h)
            raise HstError(f"{what} failed ({rc}): {msg.decode() if msg else ''}", rc)

    # ---- fields
    def upload(self, field: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        if a.shape != self.shape:
            raise ValueError(f"field shape {a.shape}, expected {self.shape}")
        self._check(lib().hst_gpu_upload(self._h, field, a.ctypes.data_as(ct.POINTER(ct.c_double))), "upload")

    def download(self, field: int) -> np.ndarray:
        a = np.empty(self.shape, np.complex128)
        self._check(lib().hst_gpu_download(self._h, field, a.ctypes.data_as(ct.POINTER(ct.c_double))), "download")
        return a

    def set_velocity(self, V: np.ndarray):
        """V: (3, nx+1, 2nz+1, ny+4) u, v, w; ghost rows are refilled at self.time."""
        for c in range(3):
            self.upload(c, V[c])
            self.fill_ghosts(c)

    def velocity(self) -> np.ndarray:
        return np.stack([self.download(c) for c in range(3)])

    def set_tables(self, der=None, y=None, dyl=None):
        P = ct.POINTER(ct.c_double)
        args = []
        for a, n in ((der, 20 * self.ny), (y, self.ny + 4), (dyl, self.ny)):
            if a is None:
                args.append(None)
            else:
                a = np.ascontiguousarray(a, np.float64).ravel()
                assert a.size == n
                args.append(a)
        self._check(lib().hst_gpu_set_tables(self._h, *[a.ctypes.data_as(P) if a is not None else None for a in args]),
                    "set_tables")
        self._tables()

    # ---- the path
    def timestep(self, deltat: float | None = None) -> float:
        dt = self.deltat if deltat is None else float(deltat)
        t = ct.c_double(self.time)
        c = ct.c_double(0.0)
        self._check(lib().hst_gpu_timestep(self._h, ct.byref(t), dt, ct.byref(c)), "timestep")
        self.time = t.value
        self.cfl = c.value
        return self.cfl

    def timesteps(self, n: int, deltat: float | None = None):
        dt = self.deltat if deltat is None else float(deltat)
        t = ct.c_double(self.time)
        self._check(lib().hst_gpu_timesteps(self._h, int(n), ct.byref(t), dt), "timesteps")
        self.time = t.value

    def line_solve(self, kind, lam, src, dst, shift=None, time=None):
        t = self.time if time is None else float(time)
        if shift is None:
            rc = lib().hst_gpu_line_solve(self._h, kind, float(lam), src, dst, 0, 0.0, 0.0, t)
        else:
            rc = lib().hst_gpu_line_solve(self._h, kind, float(lam), src, dst, 1, float(shift[0]), float(shift[1]), t)
        self._check(rc, "line_solve")

    def fill_ghosts(self, field, sx=None, sz=None):
        if sx is None:
            self._check(lib().hst_gpu_fill_ghosts_at(self._h, field, self.time), "fill_ghosts")
        else:
            self._check(lib().hst_gpu_fill_ghosts(self._h, field, float(sx), float(sz)), "fill_ghosts")

    def compute_cfl(self) -> float:
        c = ct.c_double(0.0)
        self._check(lib().hst_gpu_compute_cfl(self._h, ct.byref(c)), "compute_cfl")
        self.cfl = c.value
        return c.value

    def sync(self):
        self._check(lib().hst_gpu_sync(self._h), "sync")

    def shear_shifts(self, t):
        sx, sz = ct.c_double(), ct.c_double()
        lib().hst_gpu_shear_shifts(self._h, float(t), ct.byref(sx), ct.byref(sz))
        return sx.value, sz.value

    def s2_of(self, t):
        return lib().hst_gpu_s2_of(self._h, float(t))

    def s2_integral(self, t1, t2):
        return lib().hst_gpu_s2_integral(self._h, float(t1), float(t2))

    KERNEL_CLASSES = ("zinv", "xprod", "zfwd", "column", "line_solve", "ghosts", "rhs", "shift")

    def set_profiling(self, on: bool):
        self._check(lib().hst_gpu_set_profiling(self._h, int(bool(on))), "set_profiling")

    def kernel_times(self) -> dict:
        """{class: (total ms, launches)} since the last reset (waits for the stream)."""
        n = len(self.KERNEL_CLASSES)
        ms = (ct.c_double * n)()
        cnt = (ct.c_longlong * n)()
        self._check(lib().hst_gpu_kernel_times(self._h, ms, cnt), "kernel_times")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    def reset_kernel_times(self):
        self._check(lib().hst_gpu_reset_kernel_times(self._h), "reset_kernel_times")

    def upload_ptr(self, field: int, ptr: int):
        """upload from a host address (e.g. pinned memory) holding one field"""
        self._check(lib().hst_gpu_upload(self._h, field, ct.cast(ct.c_void_p(ptr), ct.POINTER(ct.c_double))), "upload")

    def download_ptr(self, field: int, ptr: int):
        self._check(lib().hst_gpu_download(self._h, field, ct.cast(ct.c_void_p(ptr), ct.POINTER(ct.c_double))),
                    "download")

    def outstats(self, time=None) -> dict:
        """outstats (src/hst_stats.f90:136-285) on the device: energy,
        dissipation, uv, vw, uu, vv, ww, uw of the resident field."""
        t = self.time if time is None else float(time)
        out = np.zeros(8)
        self._check(lib().hst_gpu_outstats(self._h, t, out.ctypes.data_as(ct.POINTER(ct.c_double))), "outstats")
        return dict(zip(["energy", "diss", "uv", "vw", "uu", "vv", "ww", "uw"], out))

    # ---- the substep one piece at a time (reference-layout buffers)
    def buffer_shape(self, buf):
        """numpy shape of one component of a buffer: VVdz(nzd, nx+1, rows) is
        (rows, nx+1, nzd); VVdx, VVdp(nxd+1, nzd, rows) are (rows, nzd, nxd+1)
        complex128 (2(nxd+1) reals along the last axis in their real view)"""
        rows = self.ny + 4
        return (rows, self.nx + 1, self.nzd) if buf == BUF_VVDZ else (rows, self.nzd, self.nxd + 1)

    def buffer_download(self, buf, m) -> np.ndarray:
        a = np.empty(self.buffer_shape(buf), np.complex128)
        self._check(lib().hst_gpu_buffer_download(self._h, buf, m, a.ctypes.data), "buffer_download")
        return a

    def buffer_upload(self, buf, m, a):
        a = np.ascontiguousarray(a, np.complex128)
        if a.shape != self.buffer_shape(buf):
            raise ValueError(f"buffer shape {a.shape}, expected {self.buffer_shape(buf)}")
        self._check(lib().hst_gpu_buffer_upload(self._h, buf, m, a.ctypes.data), "buffer_upload")

    def buffer_pointer(self, buf):
        """(device address, bytes) of a whole buffer"""
        ptr, n = ct.c_void_p(), ct.c_size_t()
        self._check(lib().hst_gpu_buffer_pointer(self._h, buf, ct.byref(ptr), ct.byref(n)), "buffer_pointer")
        return ptr.value, n.value

    def fft(self, kind, m):
        self._check(lib().hst_gpu_fft(self._h, kind, m), "fft")

    def transpose(self, direction, m):
        self._check(lib().hst_gpu_transpose(self._h, direction, m), "transpose")

    def transform_to_physical(self):
        self._check(lib().hst_gpu_transform_to_physical(self._h), "transform_to_physical")

    def build_products(self, g):
        self._check(lib().hst_gpu_build_products(self._h, int(g)), "build_products")

    def products_to_spectral(self):
        self._check(lib().hst_gpu_products_to_spectral(self._h), "products_to_spectral")

    def vvdz_to_field(self, field, m):
        self._check(lib().hst_gpu_vvdz_to_field(self._h, field, m), "vvdz_to_field")

    def buildrhs_prepare(self, ode, deltat=None, time=None):
        dt = self.deltat if deltat is None else float(deltat)
        t = self.time if time is None else float(time)
        o = (ct.c_double * 3)(*[float(x) for x in ode])
        self._check(lib().hst_gpu_buildrhs_prepare(self._h, o, dt, t), "buildrhs_prepare")

    def buildrhs(self, ode, g):
        o = (ct.c_double * 3)(*[float(x) for x in ode])
        self._check(lib().hst_gpu_buildrhs(self._h, o, int(g)), "buildrhs")

    def damping_update(self, time=None):
        t = self.time if time is None else float(time)
        self._check(lib().hst_gpu_damping_update(self._h, t), "damping_update")

    def damping_mask(self):
        self._check(lib().hst_gpu_damping_mask(self._h), "damping_mask")

    def shear_shift(self, dt_sub, time=None):
        t = self.time if time is None else float(time)
        self._check(lib().hst_gpu_shear_shift(self._h, float(dt_sub), t), "shear_shift")

    def linsolve(self, lam, time=None):
        t = self.time if time is None else float(time)
        self._check(lib().hst_gpu_linsolve(self._h, float(lam), t), "linsolve")

    def timestep_by_pieces(self, deltat=None, product_hook=None):
        """timestep() (src/hst_equations.f90:56-87) called piece by piece, as
        the reference's loop calls its module procedures; product_hook(g), if
        given, runs between build_products(g) and products_to_spectral() (the
        place tests/test_conservation.f90 edits the products).  Returns the
        CFL number of the third substep."""
        dt = self.deltat if deltat is None else float(deltat)
        linear = bool(self.cfg.get("linear"))
        cfl = 0.0
        for i in range(3):
            ode = RK_RAI[i]
            if not linear or i == 2:
                self.transform_to_physical()
            if i == 2:
                cfl = self.compute_cfl()
            self.damping_update(self.time)
            self.buildrhs_prepare(ode, dt, self.time)
            if not linear:
                for g in (1, 2):
                    self.build_products(g)
                    if product_hook is not None:
                        product_hook(g)
                    self.products_to_spectral()
                    self.buildrhs(ode, g)
            self.damping_mask()
            dt_sub = 2.0 / ode[0] * dt
            self.shear_shift(dt_sub, self.time)
            self.time = self.time + dt_sub
            self.linsolve(ode[0] / dt, self.time)
        self.cfl = cfl
        return cfl

    # ---- host address registry (what a Fortran shim uses)
    def register_host(self, addr: int, nbytes: int, ident: int):
        self._check(lib().hst_gpu_register_host(self._h, ct.c_void_p(addr), nbytes, ident), "register_host")

    def unregister_host(self, addr: int):
        self._check(lib().hst_gpu_unregister_host(self._h, ct.c_void_p(addr)), "unregister_host")

    def host_id(self, addr: int) -> int:
        return int(lib().hst_gpu_host_id(self._h, ct.c_void_p(addr)))

    SUM_NAMES = ("eps", "uv", "uu", "vv", "ww", "vw", "uw", "mfx", "mfz", "q_in", "q_out", "e_in", "e_out", "ed", "pd",
                 "ncol_damped")

    def outstats_sums(self, time=None):
        """The reductions of outstats as the reference's `sums` array holds
        them (src/hst_stats.f90:242; box-height integrals before the mean
        correction) and the column energies exz as an (nx+1, 2nz+1) array
        (exz[ix, iz + nz] = sum_y w |u|^2, :225-240).  RHS1 is overwritten."""
        t = self.time if time is None else float(time)
        sums = np.zeros(16)
        exz = np.zeros((self.nx + 1, 2 * self.nz + 1))
        P = ct.POINTER(ct.c_double)
        self._check(lib().hst_gpu_outstats_sums(self._h, t, sums.ctypes.data_as(P), exz.ctypes.data_as(P)),
                    "outstats_sums")
        return dict(zip(self.SUM_NAMES, sums)), exz

    def autotune(self, deltat=None, steps: int = 3) -> str:
        """Pick the fastest line-solver group width and FFT plans for this
        context's sizes (the fields are left as they were); returns the report."""
        dt = self.deltat if deltat is None else float(deltat)
        buf = ct.create_string_buffer(4096)
        self._check(lib().hst_gpu_autotune(self._h, dt, int(steps), buf, 4096), "autotune")
        return buf.value.decode()

    def pressure(self, dst: int = 6, time=None) -> np.ndarray:
        """compute_pressure (src/hst_pressure.f90:35-110) into field dst
        (RHS2 by default, as write_pressure); returns that field."""
        t = self.time if time is None else float(time)
        self._check(lib().hst_gpu_pressure(self._h, t, int(dst)), "pressure")
        return self.download(dst)

    def write_restart(self, path, deltat=None, t_max=0.0, dt_field=0.0, dt_save=0.0):
        """restart_write: V in the reference's CPL field file (Dati.cart)."""
        dt = self.deltat if deltat is None else float(deltat)
        self._check(lib().hst_gpu_write_restart(self._h, str(path).encode(), self.time, dt, float(t_max),
                                                float(dt_field), float(dt_save)), "write_restart")

    def read_restart(self, path) -> float:
        """restart_read of a file of this mesh; sets and returns its time."""
        t = ct.c_double()
        self._check(lib().hst_gpu_read_restart(self._h, str(path).encode(), ct.byref(t)), "read_restart")
        self.time = t.value
        return t.value

    def upload_async_ptr(self, field: int, ptr: int):
        """queue the upload of V1..V3 from a pinned host address (see wait_io)"""
        self._check(lib().hst_gpu_upload_async(self._h, field, ct.c_void_p(ptr)), "upload_async")

    def download_async_ptr(self, field: int, ptr: int):
        """queue the download of V1..V3 as it is now into a pinned host address"""
        self._check(lib().hst_gpu_download_async(self._h, field, ct.c_void_p(ptr)), "download_async")

    def wait_io(self):
        """wait for every queued asynchronous upload and download"""
        self._check(lib().hst_gpu_wait_io(self._h), "wait_io")

    @property
    def launches(self) -> int:
        return int(lib().hst_gpu_launch_count(self._h))

    @property
    def stream(self) -> int:
        return int(lib().hst_gpu_stream(self._h) or 0)


class ColumnSpectrum:
    """The running average of the column energies that spectrum_write
    (src/hst_stats.f90:110-134) keeps between its calls: add() every outstats
    sample (the sums and exz of Solver.outstats_sums), energies() the
    average E(ix, iz) = exz_acc / nacc / 2, the (0,0) column taken about the
    box mean (the squared box means of the mean-flow profiles removed)."""

    def __init__(self, dyl, t0=0.0):
        self.ly_w = float(np.sum(dyl))
        self.reset(t0)

    def reset(self, t0=0.0):
        self.acc = None
        self.nacc = 0
        self.mean_acc = 0.0
        self.t0 = t0

    def add(self, sums: dict, exz: np.ndarray):
        self.acc = exz.copy() if self.acc is None else self.acc + exz
        self.nacc += 1
        self.mean_acc += (sums["mfx"] ** 2 + sums["mfz"] ** 2) / self.ly_w

    def energies(self) -> np.ndarray:
        """(nx+1, 2nz+1): 0.5 times the averaged column energies."""
        if not self.nacc:
            raise HstError("no samples")
        full = self.acc / self.nacc
        nz = (full.shape[1] - 1) // 2
        full[0, nz] -= self.mean_acc / self.nacc
        return 0.5 * full

    def write(self, path, time, alfa0, beta0):
        """The text file of spectrum_write: one line per column, ix, iz, kx,
        kz, E; restarts the average."""
        e = self.energies()
        nx, nzT = e.shape
        nz = (nzT - 1) // 2
        with open(path, "w") as f:
            f.write(f"# column energies ly/2 sum_y |u|^2 averaged over t = {self.t0:12.5f} .. {time:12.5f} "
                    f"({self.nacc} samples);  ix  iz  kx  kz  E\n")
            for ix in range(nx):
                for iz in range(-nz, nz + 1):
                    f.write(f"{ix:5d} {iz:5d} {alfa0 * ix:15.7E} {beta0 * iz:15.7E} {e[ix, iz + nz]:15.7E}\n")
        self.reset(time)


def device_bytes(**deck) -> float:
    cfg = dict(DECK_DEFAULTS)
    cfg.update(deck)
    p = Params()
    p.nx, p.ny, p.nz = int(cfg["nx"]), int(cfg["ny"]), int(cfg["nz"])
    p.nxd, p.nzd = int(cfg.get("nxd", 0)), int(cfg.get("nzd", 0))
    p.alfa0, p.beta0, p.ly, p.re = cfg["alfa0"], cfg["beta0"], cfg["ly"], cfg["re"]
    prec = cfg.get("precision", PREC_FP64)
    p.precision = {"fp64": PREC_FP64, "mixed": PREC_MIXED}.get(prec, prec) if isinstance(prec, str) else int(prec)
    return float(lib().hst_gpu_device_bytes(ct.byref(p)))


# ------------------------------------------------------ initial fields ----
def uniform_from_key(seed, component, iy, iz, ix):
    """The keyed uniform deviate of src/hst_initial.f90:139-159, vectorised."""
    M = np.uint64(0xFFFFFFFF)
    h = (np.int64(seed) + np.int64(2654435761) * np.asarray(component, np.int64)
         + np.int64(2246822519) * np.asarray(iy, np.int64) + np.int64(3266489917) * np.asarray(iz, np.int64)
         + np.int64(668265263) * np.asarray(ix, np.int64))
    h = h.astype(np.uint64) & M
    h = h ^ (h >> np.uint64(16))
    h = (h * np.uint64(2146121005)) & M
    h = h ^ (h >> np.uint64(13))
    h = (h * np.uint64(2032289749)) & M
    h = h ^ (h >> np.uint64(16))
    return h.astype(np.float64) * (1.0 / 4294967296.0)


def random_field(nx, ny, nz, alfa0, beta0, ly, y, seed=1, k0=4.0, energy=0.1, envelope="gauss", amplitude=1.0):
    """A seeded divergence-free field: the curl of a keyed random vector
    potential (src/hst_initial.f90:27-67,113-133: modes |m| <= ny/3 in y,
    (0,0) column zero, the ix = 0 plane Hermitian).  envelope 'gauss' is
    exp(-(k/k0)^2) on the potential, i.e. E(k) ~ k^4 exp(-2 (k/k0)^2); 'hst'
    is the reference's (k/k0)^2 exp(1 - (k/k0)^2).  With energy set, the
    field is rescaled so that <u_i u_i>/2 = energy (box mean, as
    src/hst_stats.f90:257-269 reports it).  Returns (3, nx+1, 2nz+1, ny+4)."""
    mmax = ny // 3
    # both envelopes are below their 1e-8 cut beyond k = 5 k0, so only the
    # modes of that box are drawn (the 1536^2 x 512 field in seconds)
    kcut = 5.0 * k0
    nxb = min(nx, int(kcut / abs(alfa0)))
    nzb = min(nz, int(kcut / abs(beta0)))
    mb = min(mmax, int(kcut * ly / (2.0 * PI)))
    ix = np.arange(nxb + 1)[:, None, None]
    iz = np.arange(-nzb, nzb + 1)[None, :, None]
    m = np.arange(-mb, mb + 1)[None, None, :]
    kx = alfa0 * ix
    kz = beta0 * iz
    ky = 2.0 * PI * m / ly
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    q = k / k0
    with np.errstate(divide="ignore", invalid="ignore"):
        env = np.exp(-q * q) if envelope == "gauss" else q * q * np.exp(1.0 - q * q)
    env = np.where((k == 0.0) | (env < 1e-8) | (q > 5.0), 0.0, env)
    env = np.where((ix == 0) & (iz == 0), 0.0, env)
    mirror = (ix == 0) & ((iz < 0) | ((iz == 0) & (m < 0)))
    jz = np.where(mirror, -iz, iz)
    jm = np.where(mirror, -m, m)
    a = []
    for c in range(1, 4):
        r = uniform_from_key(seed, c, jm, jz, ix)
        ph = 2.0 * PI * uniform_from_key(seed, c + 3, jm, jz, ix)
        ac = r * np.exp(1j * ph)
        del r, ph
        a.append(np.where(mirror, np.conj(ac), ac) * amplitude * env)
        del ac
    del k, q, env, mirror, jz, jm
    I = 1j
    E = np.exp(I * ky[0, 0, :, None] * y[None, :])  # (modes in y, ny+4)
    # one velocity component at a time, projected on the y grid by one
    # complex matrix product; the modes outside the box stay zero
    V = np.zeros((3, nx + 1, 2 * nz + 1, len(y)), np.complex128)
    for c in range(3):
        if c == 0:
            uc = I * (ky * a[2] - kz * a[1])
        elif c == 1:
            uc = I * (kz * a[0] - kx * a[2])
        else:
            uc = I * (kx * a[1] - ky * a[0])
        V[c, :nxb + 1, nz - nzb:nz + nzb + 1] = (uc.reshape(-1, E.shape[0]) @ E).reshape(nxb + 1, 2 * nzb + 1, len(y))
        del uc
    del a
    if energy is not None:
        e = box_energy(V, ly, y)
        if e > 0:
            V *= math.sqrt(energy / e)
    return V


def box_energy(V, ly, y):
    """<u_i u_i>/2 box mean from the spectral field (Parseval, weights dyl)."""
    ny = V.shape[-1] - 4
    dyl = 0.5 * (y[3:ny + 3] - y[1:ny + 1])
    w = np.full(V.shape[1], 2.0)
    w[0] = 1.0
    q = 0.0
    for c in range(V.shape[0]):  # a component at a time: bounded temporaries at large sizes
        q += float((np.abs(V[c, :, :, 2:ny + 2]) ** 2 * w[:, None, None] * dyl[None, None, :]).sum())
    return 0.5 * q / ly
