"""kl_socs_forward_noalloc: SOCS imaging for callers that cannot allocate
device memory at run time (fixed memory budgets, frameworks that own the
allocator).  Its scratch is a static array inside the library, so this file
checks, through the C ABI, that two calls in a row -- with different clip
sizes, so the shared array is reused with a new layout -- give the same images
as the plan-based kl_socs_forward, and that an oversized request is refused.
Collected last on purpose: it must also pass after every other test has run.
"""
import ctypes

import numpy as np
import pytest

import klitho as K
import synth

pytestmark = pytest.mark.gpu
TOL_CF = 1e-5


def _noalloc():
    f = K.lib().kl_socs_forward_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _case(L, nclips, nk, seed):
    import torch
    src = K.createSource(41, "Annular", 0.6, 0.9)
    Nx, Ny = K.bandSize(synth.NA_IMMERSION, L, L, K.getOuterSigma(src))
    krn, sc = synth.random_kernels(nk, Nx, Ny, seed=seed)
    sc = (sc / sc.sum() * 0.9).astype(np.float32)  # clear field below 1
    masks = np.stack([synth.rect_mask(L, 10 + 3 * c, seed=seed + c) for c in range(nclips)])
    plan = K.SocsPlan(L, L, Nx, Ny, nk, max_clips=nclips)
    plan.set_kernels(0, krn, sc)
    md = torch.from_numpy(masks).cuda()
    ref = torch.empty((nclips, 1, L, L), dtype=torch.float32, device="cuda")
    plan.forward(md, ref)
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
    sd = torch.from_numpy(sc).cuda()
    out = torch.full((nclips, L, L), np.nan, dtype=torch.float32, device="cuda")
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    cf = float(np.sum(sc * np.abs(krn[:, c].astype(np.complex128)) ** 2))
    return dict(L=L, Nx=Nx, Ny=Ny, nk=nk, n=nclips, md=md, kd=kd, sd=sd, out=out, ref=ref,
                plan=plan, cf=cf)


def _call(f, c):
    rc = f(c["md"].data_ptr(), c["n"], c["L"], c["L"], c["Nx"], c["Ny"], c["kd"].data_ptr(),
           c["sd"].data_ptr(), c["nk"], c["out"].data_ptr(), None)
    assert rc == K.KL_OK, K.last_error()


def test_noalloc_matches_plan_path_twice(cuda):
    import torch
    f = _noalloc()
    first = _case(1024, 3, 24, seed=1)
    second = _case(512, 5, 16, seed=7)
    _call(f, first)
    _call(f, second)
    torch.cuda.synchronize()
    for c in (first, second):
        got = c["out"].cpu().numpy()
        want = c["ref"].cpu().numpy()[:, 0]
        assert np.isfinite(got).all()
        assert np.abs(got - want).max() <= TOL_CF * c["cf"]
    # and again on the first geometry, after the array held the second's data
    first["out"].fill_(np.nan)
    _call(f, first)
    torch.cuda.synchronize()
    assert np.abs(first["out"].cpu().numpy() - first["ref"].cpu().numpy()[:, 0]).max() <= TOL_CF * first["cf"]


def test_noalloc_rejects_oversized_request(cuda):
    import torch
    f = _noalloc()
    L = 1024
    dummy = torch.zeros(1, dtype=torch.float32, device="cuda")
    rc = f(dummy.data_ptr(), 100000, L, L, 13, 13, dummy.data_ptr(), dummy.data_ptr(), 24,
           dummy.data_ptr(), None)
    assert rc == K.KL_ERR_INVALID
    assert "static workspace" in K.last_error()
