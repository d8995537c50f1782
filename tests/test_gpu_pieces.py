"""The substep one piece at a time (hst_gpu_transform_to_physical ...
hst_gpu_linsolve) on the reference-layout buffers, against the fused
substep, the oracle's pieces and the reference's own piece-by-piece tests
(tests/test_roundtrip.f90, tests/test_conservation.f90), all through the C
ABI; and the host address registry a Fortran shim uses."""
import ctypes as ct

import numpy as np
import pytest

import oracle
from homogenenousshearturbulence_b200 import hst
from tests.gpu_util import c1_deck, deck_to_oracle, make_pair, rel_l2, seeded_field

pytestmark = pytest.mark.gpu

VARIANTS = {
    "default": dict(),
    "exact_s2": dict(exact_shift=True, s2_amplitude=0.5, s2_period=0.3),
    "hard_damping": dict(damp_kpar=3.0, damp_kperp=2.0, damp_hard=True, s2_amplitude=0.4, s2_period=0.5),
    "soft_damping": dict(damp_kpar=3.0, damp_kperp=2.0, damp_rate=0.5, damp_edge=0.3, exact_shift=True),
    "linear": dict(linear=True),
}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_pieces_match_fused_and_oracle(variant):
    """10 time steps of the 96^2 x 64 deck run piece by piece as the
    reference's timestep calls its procedures (transform_to_physical,
    buildrhs_prepare, build_products / products_to_spectral / buildrhs per
    group, damping_mask, shear_shift, linsolve) against the fused
    hst_gpu_timestep and against the oracle: <= 1e-12 relative L2."""
    deck = c1_deck(**VARIANTS[variant])
    V0 = seeded_field(deck, seed=8, k0=4.0, energy=0.1)
    s, o = make_pair(deck, V0)
    f = hst.Solver(deck)
    f.time = 0.0
    f.set_velocity(V0)
    o.deltat = deck["deltat"]
    for _ in range(10):
        s.timestep_by_pieces(deck["deltat"])
        f.timestep(deck["deltat"])
        o.timestep()
    assert abs(s.time - o.time) <= 1e-15
    Vp, Vf = s.velocity(), f.velocity()
    Vo = np.stack([o.field(c).copy() for c in range(3)])
    assert abs(s.cfl - f.cfl) <= 1e-12 * f.cfl
    e_f, e_o = rel_l2(Vp, Vf), rel_l2(Vp, Vo)
    s.close()
    f.close()
    assert e_f <= 1e-12, e_f
    assert e_o <= 1e-12, e_o


def test_piece_buffers_match_oracle():
    """The buffers the pieces leave, in the reference's layouts, against the
    oracle's: rVVdx after transform_to_physical, products after
    build_products(g), VVdz (through vvdz_to_field) after
    products_to_spectral, every row; within 1e-13 of each buffer's largest
    entry.  On an uneven deck (nx = 20, nz = 11: 2 nxd = 64, nzd = 48)."""
    deck = c1_deck(nx=20, nz=11, ny=32, exact_shift=True, s2_amplitude=0.5, s2_period=0.7)
    V0 = seeded_field(deck, seed=3, k0=4.0, energy=0.1)
    s, o = make_pair(deck, V0)
    s.time = o.time = 0.37
    for c in range(3):
        s.fill_ghosts(c)
        o.fill_ghosts(c)
    NX = 2 * s.nxd

    def real_view(a):
        return a.view(np.float64)[..., :NX]

    s.transform_to_physical()
    o.transform_to_physical()
    ph = o.physical()
    for m in range(3):
        g = real_view(s.buffer_download(hst.BUF_VVDX, m + 1))
        assert np.abs(g - ph[m][..., :NX]).max() <= 1e-13 * np.abs(ph[m]).max(), m
    for grp in (1, 2):
        s.build_products(grp)
        o.build_products(grp)
        pr = o.products()
        for m in range(3):
            g = real_view(s.buffer_download(hst.BUF_VVDP, m + 1))
            assert np.abs(g - pr[m][..., :NX]).max() <= 1e-13 * np.abs(pr[m]).max(), (grp, m)
        s.products_to_spectral()
        o.products_to_spectral()
        for m in range(3):
            s.vvdz_to_field(hst.RHS1, m + 1)
            g = s.download(hst.RHS1)
            r = o.vvdz_to_field(m)
            assert np.abs(g - r).max() <= 1e-13 * np.abs(r).max(), (grp, m)
    s.close()


def test_roundtrip_through_the_pieces():
    """tests/test_roundtrip.f90 of the reference: spectral -> physical ->
    (products = rVVdx times factor) -> spectral returns the field to 1e-12 of
    its largest entry, every row, each component."""
    deck = c1_deck(nx=15, nz=16, ny=32)
    V0 = seeded_field(deck, seed=1, k0=4.0, energy=0.1)
    s = hst.Solver(deck)
    s.time = 0.0
    s.set_velocity(V0)
    V0 = s.velocity()
    s.transform_to_physical()
    factor = 1.0 / (2.0 * s.nxd * s.nzd)
    for m in (1, 2, 3):
        s.buffer_upload(hst.BUF_VVDP, m, s.buffer_download(hst.BUF_VVDX, m) * factor)
    s.products_to_spectral()
    vmax = np.abs(V0).max()
    for m in (1, 2, 3):
        s.vvdz_to_field(hst.RHS2, m)
        W = s.download(hst.RHS2)
        assert np.abs(W - V0[m - 1]).max() <= 1e-12 * vmax, m
    s.close()


def energy(V):
    """q2 = <u_i u_i> as tests/test_conservation.f90 sums it (weights 2 for
    ix > 0, interior rows, over ny)."""
    w = np.full(V.shape[1], 2.0)
    w[0] = 1.0
    return float(np.sum(w[None, :, None, None] * np.abs(V[..., 2:-2]) ** 2) / (V.shape[-1] - 4))


def test_conservation_product_by_product(golden):
    """tests/test_conservation.f90 of the reference on the GPU pieces: one
    inviscid step (S = 0, ni = 1e-12, dt = 1e-4) from the projected random
    field of the pressure deck with only one product kept (the others
    zeroed in the products buffer between build_products and
    products_to_spectral); the energy change rate over the energy of each of
    uu, vv, ww alone, and of uv + vw + uw, within the reference's 1e-2; the
    masked steps agree with the oracle doing the same to 1e-12."""
    deck = dict(hst.read_deck(golden / "pressure.in"), S=0.0, re=1.0e12, linear=False, deltat=1.0e-4)
    o0 = oracle.Sim(deck_to_oracle(deck))
    V0 = hst.random_field(deck["nx"], deck["ny"], deck["nz"], deck["alfa0"], deck["beta0"], deck["ly"], o0.y(),
                          seed=deck["seed"], k0=deck["kpeak"], energy=None, envelope="hst",
                          amplitude=deck["amplitude"])
    dt = deck["deltat"]
    rate = {}
    for mask in range(7):
        s, o = make_pair(deck, V0)
        zero = np.zeros(s.shape, np.complex128)
        for fld in (hst.OLD1, hst.OLD2):
            s.upload(fld, zero)
            o.field(fld)[...] = 0
        o.deltat = dt
        s.timestep(dt)
        o.timestep()
        q0 = energy(s.velocity())

        def gpu_hook(g):
            if mask == 0:
                return
            for p in (1, 2, 3):
                if 3 * (g - 1) + p != mask:
                    s.buffer_upload(hst.BUF_VVDP, p, np.zeros(s.buffer_shape(hst.BUF_VVDP), np.complex128))

        s.timestep_by_pieces(dt, product_hook=gpu_hook)
        # the same masked step on the oracle
        for i in range(3):
            ode = oracle.RK[i]
            o.transform_to_physical()
            o.buildrhs_prepare(ode)
            for g in (1, 2):
                o.build_products(g)
                if mask:
                    pr = o.products()
                    for p in (1, 2, 3):
                        if 3 * (g - 1) + p != mask:
                            pr[p - 1][...] = 0.0
                o.products_to_spectral()
                o.buildrhs(ode, g)
            dt_sub = 2.0 / ode[0] * dt
            o.shear_shift(dt_sub)
            o.time = o.time + dt_sub
            o.linsolve(ode[0] / dt)
        Vg = s.velocity()
        Vo = np.stack([o.field(c).copy() for c in range(3)])
        assert rel_l2(Vg, Vo) <= 1e-12, mask
        rate[mask] = (energy(Vg) - q0) / dt / q0
        s.close()
    assert max(abs(rate[k]) for k in range(4)) <= 1e-2, rate
    assert abs(rate[4] + rate[5] + rate[6]) <= 1e-2, rate


def test_host_registry():
    """hst_gpu_register_host and the calls that take host addresses: a
    registered numpy array round-trips through upload_host / download_host,
    line_solve_host equals line_solve by id, buffer components register and
    copy; a wrong size, an overlap and an unregistered address are refused
    with HST_EARG."""
    deck = c1_deck(nx=15, nz=16, ny=32)
    s = hst.Solver(deck)
    L = hst.lib()
    V0 = seeded_field(deck, seed=2, k0=4.0, energy=0.1)
    arrs = {hst.V2: np.ascontiguousarray(V0[1]), hst.RHS1: np.zeros(s.shape, np.complex128),
            hst.RHS2: np.zeros(s.shape, np.complex128)}
    for fid, a in arrs.items():
        s.register_host(a.ctypes.data, a.nbytes, fid)
        assert s.host_id(a.ctypes.data) == fid
    h = s._h
    assert L.hst_gpu_upload_host(h, ct.c_void_p(arrs[hst.V2].ctypes.data)) == 0
    assert L.hst_gpu_fill_ghosts_host(h, ct.c_void_p(arrs[hst.V2].ctypes.data), 0.1, 0.2) == 0
    assert L.hst_gpu_line_solve_host(h, hst.KIND_ETA, 50.0, ct.c_void_p(arrs[hst.V2].ctypes.data),
                                     ct.c_void_p(arrs[hst.RHS1].ctypes.data), 1, 0.1, 0.2, 0.0) == 0
    assert L.hst_gpu_download_host(h, ct.c_void_p(arrs[hst.RHS1].ctypes.data)) == 0
    s.line_solve(hst.KIND_ETA, 50.0, hst.V2, hst.RHS2, shift=(0.1, 0.2))
    assert np.array_equal(arrs[hst.RHS1], s.download(hst.RHS2))
    # a buffer component
    vz = np.zeros(s.buffer_shape(hst.BUF_VVDZ), np.complex128)
    s.register_host(vz.ctypes.data, vz.nbytes, hst.id_buf(hst.BUF_VVDZ, 2))
    s.transform_to_physical()
    assert L.hst_gpu_download_host(h, ct.c_void_p(vz.ctypes.data)) == 0
    assert np.array_equal(vz, s.buffer_download(hst.BUF_VVDZ, 2))
    # refusals
    bad = np.zeros(s.shape, np.complex128)
    with pytest.raises(hst.HstError) as e:
        s.register_host(bad.ctypes.data, bad.nbytes - 16, hst.V1)
    assert e.value.code == hst.EARG
    with pytest.raises(hst.HstError) as e:
        s.register_host(arrs[hst.V2].ctypes.data + 16, bad.nbytes, hst.V1)
    assert e.value.code == hst.EARG
    assert L.hst_gpu_upload_host(h, ct.c_void_p(bad.ctypes.data)) == hst.EARG
    assert L.hst_gpu_line_solve_host(h, hst.KIND_D0, 0.0, ct.c_void_p(vz.ctypes.data),
                                     ct.c_void_p(arrs[hst.RHS1].ctypes.data), 0, 0.0, 0.0, 0.0) == hst.EARG
    s.unregister_host(arrs[hst.V2].ctypes.data)
    assert s.host_id(arrs[hst.V2].ctypes.data) == hst.EARG
    s.close()
