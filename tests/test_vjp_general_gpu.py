"""GPU adjoint on the general-geometry pipeline (socs_gen_vjp.cu) against FP64
references: torch complex128 autograd of the restated forward model (run with
torch's FP64 FFTs on the GPU as an independent cross-check), central finite
differences of the FP64 loss (h = 1e-3, 64 pixels), and the Hopkins
definition of the source-weight gradient.

Covers the periods and bands only the general pipeline takes: 1000^2, odd and
non-square clips, 2048^2 (beyond the specialised adjoint's 1024^2), and the
4096^2 cross-quadrupole configuration (N = 53, K = 64 kernels computed by this
library's TCC + eigen path).  Tolerances as for the specialised adjoint: loss
relative 1e-5; image 1e-5 of clear field; gradient max error 1e-4 of
max |gradient|; finite differences 2e-3 relative.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ALPHA, THR = 50.0, 0.225


def phys_kernels(Lx, Ly, nk, kind="Annular", srcSize=41, defocus_nm=0.0, **kw):
    src = K.createSource(srcSize, kind, **(kw or dict(innerRadius=0.6, outerRadius=0.9)))
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, Lx, Ly, sig)
    df = synth.defocus_arg(defocus_nm)
    tcc = O.calc_tcc(src, sig, 1.35, df, Lx, Ly, Nx, Ny, n_medium=1.44)
    krn, sc, _ = O.calc_kernels(tcc, nk)
    return src, Nx, Ny, krn.astype(np.complex64), sc, df


def run_vjp(masks, targets, sets, Nx, Ny, want_image=True):
    import torch
    n, Ly, Lx = masks.shape
    nk = sets[0][0].shape[0]
    plan = K.SocsPlan(Lx, Ly, Nx, Ny, nk, nsets=len(sets), max_clips=n, adjoint=True)
    assert plan.engine == "general"
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


@pytest.mark.parametrize("Lx,Ly", [(1000, 1000), (1001, 999), (2048, 2048)])
def test_general_vjp_matches_fp64_autograd(cuda, Lx, Ly):
    _, Nx, Ny, krn, sc, _ = phys_kernels(Lx, Ly, 24)
    mask = synth.smooth_mask(Lx, seed=Lx, Ly=Ly)
    tgt = synth.rect_mask(Lx, int(60 * Lx * Ly / 1024 ** 2) + 6, seed=Lx + 1, Ly=Ly)
    _, grad, loss, img = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny)
    loss_ref, g_ref, I_ref, _ = O.socs_vjp_reference_chunked(mask, tgt, krn, sc, Nx, Ny, ALPHA, THR,
                                                             device="cuda")
    assert abs(loss[0] - loss_ref) <= 1e-5 * loss_ref
    assert np.abs(img[0, 0] - I_ref).max() <= 1e-5
    assert np.abs(grad[0] - g_ref).max() <= 1e-4 * np.abs(g_ref).max()


def test_general_vjp_two_sets_sum(cuda):
    L = 1000
    _, Nx, Ny, k0, s0, _ = phys_kernels(L, L, 12, defocus_nm=0.0)
    _, _, _, k1, s1, _ = phys_kernels(L, L, 12, defocus_nm=40.0)
    masks = np.stack([synth.smooth_mask(L, seed=s) for s in (5, 6)])
    tgts = np.stack([synth.rect_mask(L, 40, seed=s) for s in (7, 8)])
    _, grad, loss, _ = run_vjp(masks, tgts, [(k0, s0), (k1, s1)], Nx, Ny, want_image=False)
    for c in range(2):
        l0, g0, _, _ = O.socs_vjp_reference_chunked(masks[c], tgts[c], k0, s0, Nx, Ny, ALPHA, THR, device="cuda")
        l1, g1, _, _ = O.socs_vjp_reference_chunked(masks[c], tgts[c], k1, s1, Nx, Ny, ALPHA, THR, device="cuda")
        assert abs(loss[2 * c] - l0) <= 1e-5 * l0 and abs(loss[2 * c + 1] - l1) <= 1e-5 * l1
        g = g0 + g1
        assert np.abs(grad[c] - g).max() <= 1e-4 * np.abs(g).max()


def test_general_vjp_source_gradient(cuda):
    import torch
    L = 1000
    src, Nx, Ny, krn, sc, df = phys_kernels(L, L, 12)
    mask = synth.smooth_mask(L, seed=9)
    tgt = synth.rect_mask(L, 40, seed=10)
    plan, _, _, _ = run_vjp(mask[None], tgt[None], [(krn, sc)], Nx, Ny, want_image=False)
    tplan = K.TccPlan(src, 1.35, df, L, L, n_medium=1.44)
    gs = torch.zeros(src.size, dtype=torch.float32, device="cuda")
    plan.vjp_source(tplan, gs)
    got = gs.cpu().numpy()
    _, _, _, dLdI = O.socs_vjp_reference_chunked(mask, tgt, krn, sc, Nx, Ny, ALPHA, THR, device="cuda")
    P, ids, J = O.pupil_matrix(src, O.outer_sigma(src), 1.35, df, L, L, Nx, Ny, n_medium=1.44)
    want = O.source_gradient_reference(mask, dLdI, P, J, Nx, Ny)
    assert np.abs(got[ids] - want).max() <= 1e-4 * np.abs(want).max()


# ---------------------------------------------------------------------------
# the 4096^2 cross-quadrupole configuration: K = 64 kernels of the library's
# own TCC + eigen path (the parity checks below feed the same float32 kernels
# to the references)
# ---------------------------------------------------------------------------
_q4096 = {}


def quad4096():
    if not _q4096:
        src = K.createSource(81, "CrossQuadrupole", radius=0.12, offset=0.75)
        tp = K.TccPlan(src, 1.35, 0.0, 4096, 4096, n_medium=1.44)
        krn, sc, _, _ = tp.topk(64)
        _q4096.update(src=src, Nx=tp.Nx, Ny=tp.Ny, krn=krn.astype(np.complex64), sc=sc)
        tp.close()
    q = _q4096
    return q["src"], q["Nx"], q["Ny"], q["krn"], q["sc"]


def test_4096_forward_image_matches_oracle(cuda):
    import torch
    _, Nx, Ny, krn, sc = quad4096()
    assert (Nx, Ny) == (53, 53)
    mask = synth.rect_mask_fill(4096, seed=41, density=0.3)
    plan = K.SocsPlan(4096, 4096, Nx, Ny, 64)
    assert plan.engine == "general"
    plan.set_kernels(0, krn, sc)
    md = torch.from_numpy(mask[None].copy()).cuda()
    out = torch.empty((1, 1, 4096, 4096), dtype=torch.float32, device="cuda")
    plan.forward(md, out)
    torch.cuda.synchronize()
    want = O.socs_image(mask, krn.astype(np.complex128), sc, Nx, Ny)
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    cf = float(np.sum(sc.astype(np.float64) * np.abs(krn[:, c].astype(np.complex128)) ** 2))
    assert np.abs(out.cpu().numpy()[0, 0] - want).max() <= 1e-5 * cf


def test_4096_vjp_fp64_autograd_and_central_differences(cuda):
    _, Nx, Ny, krn, sc = quad4096()
    L = 4096
    mask = synth.smooth_mask(L, seed=44).astype(np.float64)
    tgt = synth.rect_mask_fill(L, seed=45, density=0.3)
    _, grad, loss, img = run_vjp(mask[None].astype(np.float32), tgt[None], [(krn, sc)], Nx, Ny)
    loss_ref, g_ref, I_ref, _ = O.socs_vjp_reference_chunked(mask, tgt, krn, sc, Nx, Ny, ALPHA, THR,
                                                             device="cuda", chunk=8)
    assert abs(loss[0] - loss_ref) <= 1e-5 * loss_ref
    assert np.abs(img[0, 0] - I_ref).max() <= 1e-5
    assert np.abs(grad[0] - g_ref).max() <= 1e-4 * np.abs(g_ref).max()
    # 64 random pixels where the gradient is not negligible (most of a 4096^2
    # clip sits far from any resist edge)
    rng = np.random.default_rng(4096)
    cand = np.argwhere(np.abs(g_ref) >= 0.05 * np.abs(g_ref).max())
    pix = cand[rng.choice(len(cand), size=64, replace=False)]
    h = 1e-3
    fd, gpu = [], []
    for y, x in pix:
        mp = mask.copy()
        mp[y, x] += h
        mm = mask.copy()
        mm[y, x] -= h
        fd.append((O.socs_loss_chunked(mp, tgt, krn, sc, Nx, Ny, ALPHA, THR, device="cuda", chunk=16) -
                   O.socs_loss_chunked(mm, tgt, krn, sc, Nx, Ny, ALPHA, THR, device="cuda", chunk=16)) / (2 * h))
        gpu.append(grad[0, y, x])
    fd, gpu = np.array(fd), np.array(gpu)
    assert np.abs(fd - gpu).max() <= 2e-3 * np.abs(fd).max()
