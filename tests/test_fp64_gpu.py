"""The plain FP64 GPU path against the oracle (the reference's FT_r2c,
calcSOCS + FI and calcImage + FT_c2r restated in FP64, pinned to the
reference build).  Tolerance 1e-12, relative to the spectrum's DC term or to
the clear-field intensity; the FP64 path keeps the reference's double image
(before its float store), so the comparison is made in double.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("L", [256, 1024])
def test_fp64_mask_spectrum_matches_ft_r2c(cuda, L):
    import torch
    m = synth.rect_mask(L, max(4, int(60 * (L / 1024) ** 2)), seed=L)
    md = torch.from_numpy(m).cuda()
    out = torch.empty((L, L, 2), dtype=torch.float64, device="cuda")
    K.fp64_mask_spectrum(md, out)
    got = out.cpu().numpy()
    got = got[..., 0] + 1j * got[..., 1]
    want = O.ft_r2c(m)
    assert np.abs(got - want).max() <= TOL * np.abs(want).max()


def _kernels(nk, Nx, Ny, seed):
    krn, sc = synth.random_kernels(nk, Nx, Ny, seed=seed)
    return krn.astype(np.complex64), (sc / sc.sum() * 0.95).astype(np.float32)


@pytest.mark.parametrize("L,nclips,nk", [(512, 3, 8), (1024, 2, 24), (2048, 1, 12)])
def test_fp64_socs_matches_oracle(cuda, L, nclips, nk):
    import torch
    src = K.createSource(41, "Annular", 0.6, 0.9)
    Nx, Ny = K.bandSize(synth.NA_IMMERSION, L, L, K.getOuterSigma(src))
    krn, sc = _kernels(nk, Nx, Ny, seed=L + nk)
    masks = np.stack([synth.rect_mask(L, max(4, int(60 * (L / 1024) ** 2)), seed=c + L) for c in range(nclips)])
    md = torch.from_numpy(masks).cuda()
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).copy()).cuda()
    sd = torch.from_numpy(sc).cuda()
    out = torch.full((nclips, L, L), np.nan, dtype=torch.float64, device="cuda")
    K.fp64_socs_forward(md, Nx, Ny, kd, sd, out)
    got = out.cpu().numpy()
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    cf = float(np.sum(sc.astype(np.float64) * np.abs(krn[:, c].astype(np.complex128)) ** 2))
    for i in range(nclips):
        want = O.socs_image(masks[i], krn, sc, Nx, Ny)
        assert np.abs(got[i] - want).max() <= TOL * cf


def test_fp64_socs_agrees_with_fast_path(cuda):
    # the mixed-precision fused path against the plain FP64 path: 1e-5 of clear field
    import torch
    L, nk = 1024, 24
    src = K.createSource(41, "Annular", 0.6, 0.9)
    Nx, Ny = K.bandSize(synth.NA_IMMERSION, L, L, K.getOuterSigma(src))
    krn, sc = _kernels(nk, Nx, Ny, seed=5)
    masks = np.stack([synth.rect_mask(L, 60, seed=s) for s in (21, 22)])
    md = torch.from_numpy(masks).cuda()
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).copy()).cuda()
    sd = torch.from_numpy(sc).cuda()
    d = torch.empty((2, L, L), dtype=torch.float64, device="cuda")
    K.fp64_socs_forward(md, Nx, Ny, kd, sd, d)
    plan = K.SocsPlan(L, L, Nx, Ny, nk, max_clips=2)
    plan.set_kernels(0, krn, sc)
    f = torch.empty((2, 1, L, L), dtype=torch.float32, device="cuda")
    plan.forward(md, f)
    torch.cuda.synchronize()
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    cf = float(np.sum(sc.astype(np.float64) * np.abs(krn[:, c].astype(np.complex128)) ** 2))
    assert np.abs(f.cpu().numpy()[:, 0] - d.cpu().numpy()).max() <= 1e-5 * cf


@pytest.mark.parametrize("L,kind,n,kw,NA,nm,df", [
    (512, "Annular", 41, dict(innerRadius=0.6, outerRadius=0.9), 1.35, 1.44, 0.0),
    (512, "Annular", 41, dict(innerRadius=0.5, outerRadius=0.8), 0.8, 1.0, 0.2),
])
def test_fp64_hopkins_matches_calcimage(cuda, L, kind, n, kw, NA, nm, df):
    import torch
    src = K.createSource(n, kind, **kw)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(NA, L, L, sig)
    tcc = O.calc_tcc(src, sig, NA, df, L, L, Nx, Ny, n_medium=nm)
    mask = synth.rect_mask(L, 16, seed=3)
    _, want = O.hopkins_image(mask, tcc, Nx, Ny)
    plan = K.TccPlan(src, NA, df, L, L, n_medium=nm, precision=K.PREC_FP64)
    md = torch.from_numpy(mask[None].copy()).cuda()
    out = torch.empty((1, L, L), dtype=torch.float64, device="cuda")
    plan.hopkins_fp64(md, out)
    torch.cuda.synchronize()
    cf = float(tcc[(tcc.shape[0] - 1) // 2, (tcc.shape[0] - 1) // 2].real)
    assert np.abs(out.cpu().numpy()[0] - want).max() <= TOL * cf


def test_fp64_rejects_non_power_of_two(cuda):
    import torch
    md = torch.zeros((1, 96, 96), dtype=torch.float32, device="cuda")
    kd = torch.zeros((1, 9, 2), dtype=torch.float32, device="cuda")
    sd = torch.ones(1, dtype=torch.float32, device="cuda")
    out = torch.empty((1, 96, 96), dtype=torch.float64, device="cuda")
    with pytest.raises(K.KLError, match="powers of two"):
        K.fp64_socs_forward(md, 1, 1, kd, sd, out)


def _vjp_case(L, nk, seed):
    from test_vjp_gpu import kernels
    _, Nx, Ny, krn, sc, _ = kernels(L, nk)
    masks = np.stack([synth.smooth_mask(L, seed=seed + c) for c in range(2)])
    tgts = np.stack([synth.rect_mask(L, int(60 * (L / 1024) ** 2) + 6, seed=seed + 10 + c) for c in range(2)])
    return Nx, Ny, krn, sc, masks, tgts


@pytest.mark.parametrize("L", [256, 512])
def test_fp64_vjp_matches_fp64_autograd(cuda, L):
    # the FP64 GPU adjoint (fields materialised) against torch complex128
    # autograd of the restated forward model: 1e-10 relative
    import torch
    Nx, Ny, krn, sc, masks, tgts = _vjp_case(L, 12, seed=L)
    md = torch.from_numpy(masks.astype(np.float32)).cuda()
    td = torch.from_numpy(tgts.astype(np.float32)).cuda()
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
    sd = torch.from_numpy(np.asarray(sc, dtype=np.float32)).cuda()
    grad = torch.empty((2, L, L), dtype=torch.float64, device="cuda")
    img = torch.empty((2, L, L), dtype=torch.float64, device="cuda")
    loss = torch.empty(2, dtype=torch.float64, device="cuda")
    K.fp64_socs_vjp(md, td, Nx, Ny, kd, sd, grad, loss, img)
    torch.cuda.synchronize()
    for c in range(2):
        l_ref, g_ref, I_ref, _ = O.socs_vjp_reference(masks[c].astype(np.float32), tgts[c], krn,
                                                      np.asarray(sc, dtype=np.float32), Nx, Ny)
        assert abs(loss[c].item() - l_ref) <= 1e-10 * l_ref
        assert np.abs(img[c].cpu().numpy() - I_ref).max() <= 1e-12
        assert np.abs(grad[c].cpu().numpy() - g_ref).max() <= 1e-10 * np.abs(g_ref).max()


def test_fused_vjp_agrees_with_fp64_path(cuda):
    import torch
    from test_vjp_gpu import run_vjp
    L = 1024
    Nx, Ny, krn, sc, masks, tgts = _vjp_case(L, 24, seed=40)
    _, g32, l32, _ = run_vjp(masks, tgts, [(krn, sc)], Nx, Ny, want_image=False)
    md = torch.from_numpy(masks.astype(np.float32)).cuda()
    td = torch.from_numpy(tgts.astype(np.float32)).cuda()
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
    sd = torch.from_numpy(np.asarray(sc, dtype=np.float32)).cuda()
    grad = torch.empty((2, L, L), dtype=torch.float64, device="cuda")
    loss = torch.empty(2, dtype=torch.float64, device="cuda")
    K.fp64_socs_vjp(md, td, Nx, Ny, kd, sd, grad, loss)
    torch.cuda.synchronize()
    g64, l64 = grad.cpu().numpy(), loss.cpu().numpy()
    assert np.abs(l32 - l64).max() <= 1e-5 * np.abs(l64).max()
    assert np.abs(g32 - g64).max() <= 1e-4 * np.abs(g64).max()
