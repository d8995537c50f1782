"""ctypes binding of the hst oracle (oracle/hst_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  The oracle is the CPU FP64 restatement of the
reference's substep; tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it as the checker.  The product never imports it.
Parity pin: the oracle reproduces the reference's stored regression fields
tests/golden/small*.fld at the reference's 1e-10 tolerance
(tests/test_oracle_golden.py).
"""
from __future__ import annotations

import ctypes as ct
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
EXE = HERE / "_build" / "hst_oracle"

D2V, ETA, POISSON, D0, DY = 1, 2, 3, 4, 5
V1, V2, V3, OLD1, OLD2, RHS1, RHS2 = range(7)
# RK_rai (src/hst_params.f90:108-111), one row per substep
RK = np.array([[120.0 / 32.0, 2.0, 0.0], [120.0 / 8.0, 50.0 / 8.0, 34.0 / 8.0],
               [120.0 / 20.0, 90.0 / 20.0, 50.0 / 20.0]])


class Params(ct.Structure):
    _fields_ = [
        ("nx", ct.c_int), ("ny", ct.c_int), ("nz", ct.c_int),
        ("alfa0", ct.c_double), ("beta0", ct.c_double), ("ly", ct.c_double), ("ystretch", ct.c_double),
        ("re", ct.c_double), ("S", ct.c_double),
        ("linear", ct.c_int), ("exact_shift", ct.c_int),
        ("s2_mean", ct.c_double), ("s2_amplitude", ct.c_double), ("s2_period", ct.c_double), ("s2_start", ct.c_double),
        ("sl_amplitude", ct.c_double), ("sl_period", ct.c_double), ("sl_delta", ct.c_double), ("sl_start", ct.c_double),
        ("sl_bodyforce", ct.c_int), ("sl_ramp", ct.c_int),
        ("deltat", ct.c_double), ("cflmax", ct.c_double), ("t_max", ct.c_double),
        ("nstep", ct.c_long),
        ("time", ct.c_double),
        ("time_from_restart", ct.c_int), ("restart_from_file", ct.c_int),
        ("restart_file", ct.c_char * 256),
        ("initial_condition", ct.c_char * 32),
        ("amplitude", ct.c_double), ("kpeak", ct.c_double),
        ("seed", ct.c_int),
        ("tg_amplitude", ct.c_double),
        ("tg_mode", ct.c_int),
        ("damp_kpar", ct.c_double), ("damp_kperp", ct.c_double), ("damp_rate", ct.c_double),
        ("damp_edge", ct.c_double), ("damp_norm", ct.c_double), ("damp_angle", ct.c_double),
        ("damp_hard", ct.c_int), ("damp_mean", ct.c_int), ("damp_follow", ct.c_int),
    ]


def build():
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ct.CDLL(str(LIB))
        P = ct.POINTER
        d, i, vp = ct.c_double, ct.c_int, ct.c_void_p
        sig = {
            "ora_default_params": (None, [P(Params)]),
            "ora_read_deck": (i, [ct.c_char_p, P(Params)]),
            "ora_create": (vp, [P(Params)]),
            "ora_destroy": (None, [vp]),
            "ora_set_threads": (None, [i]),
            "ora_nxd": (i, [vp]), "ora_nzd": (i, [vp]),
            "ora_field_size": (ct.c_long, [vp]),
            "ora_field": (P(d), [vp, i]),
            "ora_der": (P(d), [vp]), "ora_y": (P(d), [vp]), "ora_dyl": (P(d), [vp]),
            "ora_gdamp": (P(d), [vp]), "ora_products": (P(d), [vp]), "ora_rvvdx": (P(d), [vp]),
            "ora_vvdz": (P(d), [vp]),
            "ora_get_time": (d, [vp]), "ora_set_time": (None, [vp, d]),
            "ora_get_deltat": (d, [vp]), "ora_set_deltat": (None, [vp, d]),
            "ora_get_cfl": (d, [vp]),
            "ora_set_physics": (None, [vp, d, d, i]),
            "ora_generate_initial_field": (None, [vp]),
            "ora_fill_ghosts": (None, [vp, i, d, d]),
            "ora_fill_ghosts_now": (None, [vp, i]),
            "ora_shear_shifts": (None, [vp, d, P(d), P(d)]),
            "ora_s2_of": (d, [vp, d]), "ora_s2_integral": (d, [vp, d, d]),
            "ora_transform_to_physical": (None, [vp]),
            "ora_compute_cfl": (d, [vp]),
            "ora_build_products": (None, [vp, i]),
            "ora_products_to_spectral": (None, [vp]),
            "ora_vvdz_to_field": (None, [vp, i, P(d)]),
            "ora_buildrhs_prepare": (None, [vp, P(d)]),
            "ora_buildrhs": (None, [vp, P(d), i]),
            "ora_shear_shift": (None, [vp, d]),
            "ora_linsolve": (None, [vp, d]),
            "ora_damping_update": (None, [vp, d]),
            "ora_damping_mask": (None, [vp]),
            "ora_damping_active": (i, [vp]),
            "ora_line_solve": (None, [vp, i, d, i, i, i, d, d]),
            "ora_timestep": (None, [vp]),
            "ora_substep": (None, [vp, i]),
            "ora_start": (None, [vp]),
            "ora_run": (ct.c_long, [vp, ct.c_long]),
            "ora_outstats": (None, [vp, P(d)]),
            "ora_outstats_sums": (None, [vp, P(d), P(d)]),
            "ora_compute_pressure": (None, [vp, ct.c_int]),
            "ora_restart_write": (i, [vp, ct.c_char_p]),
            "ora_restart_read": (i, [vp, ct.c_char_p]),
            "ora_uniform_from_key": (d, [i, i, i, i, i]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def default_params() -> Params:
    p = Params()
    lib().ora_default_params(ct.byref(p))
    return p


def params_from_deck(deck: dict) -> Params:
    """Oracle parameters from a deck dict (the keys of the hst.in
    namelists, as hst.read_deck returns them); no restart file is read."""
    p = default_params()
    for k in ("nx", "ny", "nz", "seed", "tg_mode"):
        if k in deck:
            setattr(p, k, int(deck[k]))
    for k in ("alfa0", "beta0", "ly", "ystretch", "re", "S", "s2_mean", "s2_amplitude", "s2_period", "s2_start",
              "deltat", "cflmax", "t_max", "time", "amplitude", "kpeak", "damp_kpar", "damp_kperp", "damp_rate",
              "damp_edge", "damp_norm", "damp_angle"):
        if k in deck:
            setattr(p, k, float(deck[k]))
    for k in ("linear", "exact_shift", "damp_hard", "damp_mean", "damp_follow"):
        if k in deck:
            setattr(p, k, int(bool(deck[k])))
    p.restart_from_file = 0
    return p


def read_deck(path) -> Params:
    p = Params()
    rc = lib().ora_read_deck(str(path).encode(), ct.byref(p))
    if rc != 0:
        raise FileNotFoundError(path)
    return p


def uniform_from_key(seed, c, iy, iz, ix) -> float:
    return lib().ora_uniform_from_key(seed, c, iy, iz, ix)


def set_threads(n: int):
    lib().ora_set_threads(int(n))


class Sim:
    """One oracle run; fields are numpy complex128 views (iy fastest)."""

    def __init__(self, params: Params):
        self.p = params
        self.h = lib().ora_create(ct.byref(params))
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.nxd = lib().ora_nxd(self.h)
        self.nzd = lib().ora_nzd(self.h)
        self.shape = (self.nx + 1, 2 * self.nz + 1, self.ny + 4)  # (ix, iz, iy) C order

    def __del__(self):
        try:
            if self.h:
                lib().ora_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def field(self, fid) -> np.ndarray:
        n = lib().ora_field_size(self.h)
        ptr = lib().ora_field(self.h, fid)
        a = np.ctypeslib.as_array(ptr, shape=(2 * n,)).view(np.complex128)
        return a.reshape(self.shape)

    def der(self) -> np.ndarray:
        ptr = lib().ora_der(self.h)
        return np.ctypeslib.as_array(ptr, shape=(5 * 4 * self.ny,)).copy()

    def y(self) -> np.ndarray:
        return np.ctypeslib.as_array(lib().ora_y(self.h), shape=(self.ny + 4,)).copy()

    def dyl(self) -> np.ndarray:
        return np.ctypeslib.as_array(lib().ora_dyl(self.h), shape=(self.ny,)).copy()

    def gdamp(self) -> np.ndarray:
        return np.ctypeslib.as_array(lib().ora_gdamp(self.h), shape=((self.nx + 1) * (2 * self.nz + 1),)).reshape(
            self.nx + 1, 2 * self.nz + 1)

    @property
    def time(self):
        return lib().ora_get_time(self.h)

    @time.setter
    def time(self, t):
        lib().ora_set_time(self.h, float(t))

    @property
    def deltat(self):
        return lib().ora_get_deltat(self.h)

    @deltat.setter
    def deltat(self, dt):
        lib().ora_set_deltat(self.h, float(dt))

    def set_physics(self, S, ni, linear):
        lib().ora_set_physics(self.h, float(S), float(ni), int(linear))

    def generate_initial_field(self):
        lib().ora_generate_initial_field(self.h)

    def fill_ghosts(self, fid, sx=None, sz=None):
        if sx is None:
            lib().ora_fill_ghosts_now(self.h, fid)
        else:
            lib().ora_fill_ghosts(self.h, fid, float(sx), float(sz))

    def shear_shifts(self, t):
        sx, sz = ct.c_double(), ct.c_double()
        lib().ora_shear_shifts(self.h, float(t), ct.byref(sx), ct.byref(sz))
        return sx.value, sz.value

    def s2_of(self, t):
        return lib().ora_s2_of(self.h, float(t))

    def s2_integral(self, t1, t2):
        return lib().ora_s2_integral(self.h, float(t1), float(t2))

    def transform_to_physical(self):
        lib().ora_transform_to_physical(self.h)

    def compute_cfl(self):
        return lib().ora_compute_cfl(self.h)

    def physical(self) -> np.ndarray:
        """rVVdx as (3, ny+4, nzd, 2(nxd+1)) real, the reference layout."""
        n = 3 * (self.ny + 4) * self.nzd * 2 * (self.nxd + 1)
        a = np.ctypeslib.as_array(lib().ora_rvvdx(self.h), shape=(n,))
        return a.reshape(3, self.ny + 4, self.nzd, 2 * (self.nxd + 1))

    def products(self) -> np.ndarray:
        n = 3 * (self.ny + 4) * self.nzd * 2 * (self.nxd + 1)
        a = np.ctypeslib.as_array(lib().ora_products(self.h), shape=(n,))
        return a.reshape(3, self.ny + 4, self.nzd, 2 * (self.nxd + 1))

    def build_products(self, g):
        lib().ora_build_products(self.h, int(g))

    def products_to_spectral(self):
        lib().ora_products_to_spectral(self.h)

    def vvdz_to_field(self, m) -> np.ndarray:
        out = np.zeros(self.shape, np.complex128)
        lib().ora_vvdz_to_field(self.h, int(m), out.ctypes.data_as(ct.POINTER(ct.c_double)))
        return out

    def buildrhs_prepare(self, ode):
        o = np.ascontiguousarray(ode, np.float64)
        lib().ora_buildrhs_prepare(self.h, o.ctypes.data_as(ct.POINTER(ct.c_double)))

    def buildrhs(self, ode, g):
        o = np.ascontiguousarray(ode, np.float64)
        lib().ora_buildrhs(self.h, o.ctypes.data_as(ct.POINTER(ct.c_double)), int(g))

    def shear_shift(self, dt_sub):
        lib().ora_shear_shift(self.h, float(dt_sub))

    def linsolve(self, lam):
        lib().ora_linsolve(self.h, float(lam))

    def damping_update(self, t):
        lib().ora_damping_update(self.h, float(t))

    def damping_mask(self):
        lib().ora_damping_mask(self.h)

    def damping_active(self):
        return bool(lib().ora_damping_active(self.h))

    def line_solve(self, sys, lam, src, dst, shift=None):
        if shift is None:
            lib().ora_line_solve(self.h, sys, float(lam), src, dst, 0, 0.0, 0.0)
        else:
            lib().ora_line_solve(self.h, sys, float(lam), src, dst, 1, float(shift[0]), float(shift[1]))

    def timestep(self):
        lib().ora_timestep(self.h)

    def substep(self, i):
        """substep i (0, 1, 2) of timestep"""
        lib().ora_substep(self.h, int(i))

    def start(self):
        lib().ora_start(self.h)

    def run(self, max_steps):
        return lib().ora_run(self.h, int(max_steps))

    def outstats_sums(self):
        """outstats' 16 sums (eps, uv, uu, vv, ww, vw, uw, mfx, mfz, q_in,
        q_out, e_in, e_out, ed, pd, ncol_damped) and the column energies
        exz as an (nx+1, 2nz+1) array"""
        sums = np.zeros(16)
        exz = np.zeros((self.p.nx + 1, 2 * self.p.nz + 1))
        lib().ora_outstats_sums(self.h, sums.ctypes.data_as(ct.POINTER(ct.c_double)),
                                exz.ctypes.data_as(ct.POINTER(ct.c_double)))
        return sums, exz

    def outstats(self):
        out = np.zeros(8)
        lib().ora_outstats(self.h, out.ctypes.data_as(ct.POINTER(ct.c_double)))
        return dict(zip(["energy", "diss", "uv", "vw", "uu", "vv", "ww", "uw"], out))

    def compute_pressure(self, dst):
        lib().ora_compute_pressure(self.h, dst)

    def restart_write(self, path):
        return lib().ora_restart_write(self.h, str(path).encode())

    def restart_read(self, path):
        return lib().ora_restart_read(self.h, str(path).encode())


def read_cpl(path):
    """Reads a CPL velocity file: (time, array (nx+1, 2nz+1, ny+4, 3) complex in
    CPL component order (u, w, v)); as tests/compare_fields.py in the reference."""
    b = pathlib.Path(path).read_bytes()
    i = b.find(b"Vfield=\n")
    head = b[:i].decode("latin-1")
    sizes = {}
    for key in ("nx", "ny", "nz"):
        j = head.find(key + "=")
        sizes[key] = int(head[j + len(key) + 1:].split()[0])
    t = np.frombuffer(b[b.find(b"time=\n") + 6:][:8], np.float64)[0]
    nx, ny, nz = sizes["nx"], sizes["ny"], sizes["nz"]
    a = np.frombuffer(b[i + 8:], np.complex128).reshape((nx + 1, 2 * ny + 1, nz + 3, 3))
    return t, a


def cpl_compare(a, b):
    """Max-abs difference over the interior rows relative to max |a| (the
    reference's tests/compare_fields.py:51-57)."""
    d = np.abs(a[:, :, 2:-2] - b[:, :, 2:-2]).max()
    return d / np.abs(a).max()
