"""GPU adjoint (kl_socs_vjp / kl_socs_vjp_source) against an FP64 reference
gradient (torch complex128 autograd of the restated forward model, CPU) and
central finite differences (h = 1e-3, 64 random pixels).

Workload shape of the differentiable-SOCS configuration: continuous masks in
[0, 1] (smooth noise through a sigmoid), binary rectangle targets, loss
sum (sigmoid(50 (I - 0.225)) - target)^2, physical kernels (NA 1.35 immersion
annular source).  Tolerances: loss relative 1e-5; gradient max error 1e-4 of
max |gradient| against the FP64 reference; finite differences 2e-3 relative
(the difference quotient itself carries O(h^2) error); source-weight gradient
1e-4 relative.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ALPHA, THR = 50.0, 0.225


def kernels(L, nk, defocus_nm=0.0):
    src = K.createSource(41, "Annular", 0.6, 0.9)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, L, L, sig)
    df = synth.defocus_arg(defocus_nm)
    tcc = O.calc_tcc(src, sig, 1.35, df, L, L, Nx, Ny, n_medium=1.44)
    krn, sc, _ = O.calc_kernels(tcc, nk)
    return src, Nx, Ny, krn.astype(np.complex64), sc, df


def run_vjp(masks, targets, sets, Nx, Ny, want_image=True, synthesis="auto"):
    import torch
    n, Ly, Lx = masks.shape
    nk = sets[0][0].shape[0]
    plan = K.SocsPlan(Lx, Ly, Nx, Ny, nk, nsets=len(sets), max_clips=n, adjoint=True)
    plan.set_synthesis(synthesis)
    for i, (k, s) in enumerate(sets):
        plan.set_kernels(i, k, s)
    md = torch.from_numpy(np.ascontiguousarray(masks, dtype=np.float32)).cuda()
    td = torch.from_numpy(np.ascontiguousarray(targets, dtype=np.float32)).cuda()
    grad = torch.empty_like(md)
    loss = torch.empty(n * len(sets), dtype=torch.float64, device="cuda")
    img = torch.empty((n, len(sets), Ly, Lx), dtype=torch.float32, device="cuda") if want_image else None
    plan.vjp(md, td, grad, loss, img, ALPHA, THR)
    torch.cuda.synchronize()
    return plan, grad.cpu().numpy(), loss.cpu().numpy(), (img.cpu().numpy() if want_image else None)


@pytest.mark.parametrize("L", [256, 512, 1024])
def test_vjp_matches_fp64_autograd(cuda, L):
    _, Nx, Ny, krn, sc, _ = kernels(L, 24 if L >= 512 else 12)
    mask = synth.smooth_mask(L, seed=L)
    tgt = synth.rect_mask(L, int(60 * (L / 1024) ** 2) + 6, seed=L + 1)
    _, grad, loss, img = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny)
    loss_ref, g_ref, I_ref, _ = O.socs_vjp_reference(mask, tgt, krn, sc, Nx, Ny, ALPHA, THR)
    assert abs(loss[0] - loss_ref) <= 1e-5 * loss_ref
    assert np.abs(img[0, 0] - I_ref).max() <= 1e-5
    assert np.abs(grad[0] - g_ref).max() <= 1e-4 * np.abs(g_ref).max()


def test_vjp_central_differences(cuda):
    L = 256
    _, Nx, Ny, krn, sc, _ = kernels(L, 12)
    mask = synth.smooth_mask(L, seed=3).astype(np.float64)
    tgt = synth.rect_mask(L, 8, seed=4)
    _, grad, _, _ = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny, want_image=False)
    rng = np.random.default_rng(64)
    h = 1e-3
    fd, gpu = [], []
    for y, x in rng.integers(0, L, size=(64, 2)):
        mp = mask.copy()
        mp[y, x] += h
        mm = mask.copy()
        mm[y, x] -= h
        fd.append((O.socs_loss(mp, tgt, krn, sc, Nx, Ny, ALPHA, THR) -
                   O.socs_loss(mm, tgt, krn, sc, Nx, Ny, ALPHA, THR)) / (2 * h))
        gpu.append(grad[0, y, x])
    fd, gpu = np.array(fd), np.array(gpu)
    assert np.abs(fd - gpu).max() <= 2e-3 * np.abs(fd).max()


def test_vjp_central_differences_config3(cuda):
    """The differentiable-SOCS configuration's clip: 1024^2, K = 24 physical
    kernels, continuous mask, binary target; central differences of the FP64
    loss (torch's FP64 FFTs on the GPU) at 64 random pixels where the
    gradient is not negligible."""
    L = 1024
    _, Nx, Ny, krn, sc, _ = kernels(L, 24)
    mask = synth.smooth_mask(L, seed=31).astype(np.float64)
    tgt = synth.rect_mask(L, 60, seed=32)
    _, grad, _, _ = run_vjp(mask[None].astype(np.float32), tgt[None], [(krn, sc)], Nx, Ny, want_image=False)
    _, g_ref, _, _ = O.socs_vjp_reference_chunked(mask, tgt, krn, sc, Nx, Ny, ALPHA, THR, device="cuda")
    assert np.abs(grad[0] - g_ref).max() <= 1e-4 * np.abs(g_ref).max()
    rng = np.random.default_rng(1024)
    cand = np.argwhere(np.abs(g_ref) >= 0.05 * np.abs(g_ref).max())
    pix = cand[rng.choice(len(cand), size=64, replace=False)]
    h = 1e-3
    fd, gpu = [], []
    for y, x in pix:
        mp = mask.copy()
        mp[y, x] += h
        mm = mask.copy()
        mm[y, x] -= h
        fd.append((O.socs_loss_chunked(mp, tgt, krn, sc, Nx, Ny, ALPHA, THR, device="cuda", chunk=24) -
                   O.socs_loss_chunked(mm, tgt, krn, sc, Nx, Ny, ALPHA, THR, device="cuda", chunk=24)) / (2 * h))
        gpu.append(grad[0, y, x])
    fd, gpu = np.array(fd), np.array(gpu)
    assert np.abs(fd - gpu).max() <= 2e-3 * np.abs(fd).max()


def test_vjp_two_focus_sets_sum(cuda):
    L = 256
    _, Nx, Ny, k0, s0, _ = kernels(L, 10, 0.0)
    _, _, _, k1, s1, _ = kernels(L, 10, 40.0)
    masks = np.stack([synth.smooth_mask(L, seed=s) for s in (5, 6)])
    tgts = np.stack([synth.rect_mask(L, 8, seed=s) for s in (7, 8)])
    _, grad, loss, _ = run_vjp(masks, tgts, [(k0, s0), (k1, s1)], Nx, Ny, want_image=False)
    for c in range(2):
        l0, g0, _, _ = O.socs_vjp_reference(masks[c], tgts[c], k0, s0, Nx, Ny, ALPHA, THR)
        l1, g1, _, _ = O.socs_vjp_reference(masks[c], tgts[c], k1, s1, Nx, Ny, ALPHA, THR)
        assert abs(loss[2 * c] - l0) <= 1e-5 * l0 and abs(loss[2 * c + 1] - l1) <= 1e-5 * l1
        g = g0 + g1
        assert np.abs(grad[c] - g).max() <= 1e-4 * np.abs(g).max()


def test_vjp_source_gradient_definition(cuda):
    import torch
    L = 256
    src, Nx, Ny, krn, sc, df = kernels(L, 12)
    mask = synth.smooth_mask(L, seed=9)
    tgt = synth.rect_mask(L, 8, seed=10)
    plan, _, _, _ = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny, want_image=False)
    tplan = K.TccPlan(src, 1.35, df, L, L, n_medium=1.44)
    gs = torch.zeros(src.size, dtype=torch.float32, device="cuda")
    plan.vjp_source(tplan, gs)
    got = gs.cpu().numpy()
    _, _, _, dLdI = O.socs_vjp_reference(mask, tgt, krn, sc, Nx, Ny, ALPHA, THR)
    P, ids, J = O.pupil_matrix(src, O.outer_sigma(src), 1.35, df, L, L, Nx, Ny, n_medium=1.44)
    want = O.source_gradient_reference(mask, dLdI, P, J, Nx, Ny)
    assert np.abs(got[ids] - want).max() <= 1e-4 * np.abs(want).max()
    mask_off = np.ones(src.size, bool)
    mask_off[ids] = False
    assert np.all(got[mask_off] == 0)


def test_vjp_source_gradient_finite_differences_hopkins(cuda):
    """With every nonzero eigenpair as a kernel the SOCS image is the Hopkins
    image, so the source gradient must match finite differences of the
    Hopkins model in the source weights."""
    import torch
    L = 256
    src = K.createSource(21, "Annular", 0.5, 0.9)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, L, L, sig)
    tcc = O.calc_tcc(src, sig, 1.35, 0.0, L, L, Nx, Ny, n_medium=1.44)
    N = tcc.shape[0]
    krn, sc, ev = O.calc_kernels(tcc, N)
    keep = ev > 1e-9 * ev[0]
    krn, sc = krn[keep].astype(np.complex64), sc[keep]
    mask = synth.smooth_mask(L, seed=12)
    tgt = synth.rect_mask(L, 8, seed=13)
    plan, _, _, _ = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny, want_image=False)
    tplan = K.TccPlan(src, 1.35, 0.0, L, L, n_medium=1.44)
    gs = torch.zeros(src.size, dtype=torch.float32, device="cuda")
    plan.vjp_source(tplan, gs)
    got = gs.cpu().numpy()
    P, ids, J = O.pupil_matrix(src, sig, 1.35, 0.0, L, L, Nx, Ny, n_medium=1.44)
    Jd = J.astype(np.float64)
    h = 1e-3 * Jd.max()
    rng = np.random.default_rng(1)
    for s in rng.choice(len(J), size=8, replace=False):
        jp, jm = Jd.copy(), Jd.copy()
        jp[s] += h
        jm[s] -= h
        fd = (O.hopkins_loss(mask, tgt, P, jp, Nx, Ny, ALPHA, THR) -
              O.hopkins_loss(mask, tgt, P, jm, Nx, Ny, ALPHA, THR)) / (2 * h)
        assert abs(got[ids[s]] - fd) <= 2e-3 * max(abs(fd), 1e-3 * np.abs(got).max()), (s, got[ids[s]], fd)


@pytest.mark.parametrize("engine", ["cuda", "tensor"])
def test_vjp_image_equals_forward(cuda, engine):
    # the adjoint's image is the forward pass's image, bit for bit, on either engine
    import torch
    L = 512
    _, Nx, Ny, krn, sc, _ = kernels(L, 16)
    mask = synth.smooth_mask(L, seed=14)
    tgt = synth.rect_mask(L, 10, seed=15)
    plan, _, _, img = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny, synthesis=engine)
    md = torch.from_numpy(mask[None].copy()).cuda()
    out = torch.empty((1, 1, L, L), dtype=torch.float32, device="cuda")
    plan.forward(md, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), img)


@pytest.mark.parametrize("L", [512, 1024])
def test_vjp_gradient_synthesis_engines_agree(cuda, L):
    # the adjoint on the tensor cores (default) and on the CUDA cores: same
    # loss and gradient within the FP32 tolerances
    _, Nx, Ny, krn, sc, _ = kernels(L, 24)
    masks = np.stack([synth.smooth_mask(L, seed=s) for s in (31, 32)])
    tgts = np.stack([synth.rect_mask(L, 20, seed=s) for s in (33, 34)])
    _, g_tc, loss_tc, _ = run_vjp(masks, tgts, [(krn, sc)], Nx, Ny, want_image=False)
    _, g_cu, loss_cu, _ = run_vjp(masks, tgts, [(krn, sc)], Nx, Ny, want_image=False, synthesis="cuda")
    assert np.allclose(loss_tc, loss_cu, rtol=1e-5, atol=0)  # the loss bar against FP64
    # (the resist's slope a/4 = 12.5 amplifies the engines' 1e-7-level image
    # differences; each engine is within 1e-4 of the FP64 gradient)
    assert np.abs(g_tc - g_cu).max() <= 5e-5 * np.abs(g_cu).max()
