"""hst_gpu_line_solve_noalloc against hst_gpu_line_solve: the same solves on
fields held in the caller's own device memory (torch tensors here), with no
context, two calls in a row per system kind.  Named to be collected last."""
import ctypes as ct

import numpy as np
import pytest

from homogenenousshearturbulence_b200 import hst
from tests.gpu_util import c1_deck, rel_l2, seeded_field

pytestmark = pytest.mark.gpu

TOL = 1e-14  # the same kernel on the same inputs: expected bit-identical


def noalloc():
    f = hst.lib().hst_gpu_line_solve_noalloc
    d, i, vp = ct.c_double, ct.c_int, ct.c_void_p
    f.restype = i
    f.argtypes = [i, i, i, d, d, d, i, d, vp, vp, vp, d, d, vp, ct.c_char_p, i]
    return f


def call(f, p, kind, lam, der, src, dst, shift, stream):
    msg = ct.create_string_buffer(256)
    rc = f(p["nx"], p["ny"], p["nz"], p["alfa0"], p["beta0"], p["re"], kind, lam, der.data_ptr(), src.data_ptr(),
           dst.data_ptr(), shift[0], shift[1], stream, msg, 256)
    return rc, msg.value.decode()


def test_noalloc_matches_context_line_solve():
    import torch

    deck = c1_deck()
    s = hst.Solver(deck)
    V0 = seeded_field(deck, seed=7)
    t = 0.37
    shift = s.shear_shifts(t)
    s.upload(hst.V2, V0[1])
    s.fill_ghosts(hst.V2, *shift)
    src_h = s.download(hst.V2)
    dev = torch.device("cuda:0")
    src = torch.from_numpy(src_h).to(dev)
    der = torch.from_numpy(np.ascontiguousarray(s.der).ravel()).to(dev)
    f = noalloc()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for kind, lams in ((hst.KIND_D2V, (2.5e4, 1.1e3)), (hst.KIND_ETA, (3.0e3, 7.0e2)), (hst.KIND_POISSON, (0.0, 0.0)),
                       (hst.KIND_D0, (0.0, 0.0)), (hst.KIND_DY, (0.0, 0.0))):
        want = []
        for lam in lams:
            s.line_solve(kind, lam, hst.V2, hst.RHS1, shift=shift)
            want.append(s.download(hst.RHS1))
        outs = [torch.zeros_like(src), torch.zeros_like(src)]
        for lam, out in zip(lams, outs):  # two calls in a row on one stream
            rc, msg = call(f, deck, kind, lam, der, src, out, shift, stream)
            assert rc == 0, msg
        torch.cuda.synchronize(dev)
        for w, out in zip(want, outs):
            err = rel_l2(out.cpu().numpy(), w)
            assert err <= TOL, (kind, err)
    s.close()


def test_noalloc_rejects_oversize_and_overlap():
    import torch

    deck = c1_deck()
    f = noalloc()
    dev = torch.device("cuda:0")
    src = torch.zeros((deck["nx"] + 1, 2 * deck["nz"] + 1, deck["ny"] + 4), dtype=torch.complex128, device=dev)
    der = torch.zeros(20 * deck["ny"], dtype=torch.float64, device=dev)
    big = dict(deck, ny=4096)
    rc, msg = call(f, big, hst.KIND_D0, 0.0, der, src, torch.zeros_like(src), (0.0, 0.0), None)
    assert rc == -1 and "scratch" in msg
    rc, msg = call(f, deck, hst.KIND_D0, 0.0, der, src, src, (0.0, 0.0), None)
    assert rc == -1 and "overlap" in msg


def test_noalloc_at_the_largest_size():
    """ny = 2048, the largest size the static scratch holds (all of it used,
    the widest solver group: 32 lanes of 64 rows), one Fourier column pair
    (nx = nz = 1): every kind against the context's hst_gpu_line_solve, two
    calls in a row."""
    import torch

    deck = dict(nx=1, ny=2048, nz=1, alfa0=1.0, beta0=1.0, ly=6.283185307179586, re=1000.0)
    s = hst.Solver(deck)
    t = 0.37
    shift = s.shear_shifts(t)
    rng = np.random.default_rng(11)
    V = rng.standard_normal(s.shape) + 1j * rng.standard_normal(s.shape)
    s.upload(hst.V2, V)
    s.fill_ghosts(hst.V2, *shift)
    src_h = s.download(hst.V2)
    dev = torch.device("cuda:0")
    src = torch.from_numpy(src_h).to(dev)
    der = torch.from_numpy(np.ascontiguousarray(s.der).ravel()).to(dev)
    f = noalloc()
    stream = torch.cuda.current_stream(dev).cuda_stream
    zero = np.zeros(s.shape, np.complex128)
    for kind, lam in ((hst.KIND_D2V, 2.5e4), (hst.KIND_ETA, 3.0e3), (hst.KIND_POISSON, 0.0), (hst.KIND_D0, 0.0),
                      (hst.KIND_DY, 0.0)):
        # KIND_POISSON leaves the (0,0) column of dst as it was: both paths
        # start from a zero dst
        s.upload(hst.RHS1, zero)
        s.line_solve(kind, lam, hst.V2, hst.RHS1, shift=shift)
        want = s.download(hst.RHS1)
        outs = [torch.zeros_like(src), torch.zeros_like(src)]
        for out in outs:
            rc, msg = call(f, deck, kind, lam, der, src, out, shift, stream)
            assert rc == 0, msg
        torch.cuda.synchronize(dev)
        for out in outs:
            err = rel_l2(out.cpu().numpy(), want)
            assert err <= TOL, (kind, err)
    s.close()
