"""GPU parity of the fused FP32 SOCS imaging path against the FP64 oracle.

The oracle image is K-Litho-SOCS/klitho_socs.cpp's FT_r2c + calcSOCS + FI
restated in FP64 (oracle/klitho_oracle.c), fed the same float32 kernels and
eigenvalues the GPU gets.  Tolerance: 1e-5 of the clear-field intensity
(the mixed-precision bar), checked as max |gpu - oracle| over all pixels.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_CF = 1e-5


def physical_kernels(L, nk=24, kind="Annular", srcSize=41, NA=synth.NA_IMMERSION,
                     n_medium=synth.N_WATER, defocus_nm=0.0, **src_kw):
    src = K.createSource(srcSize, kind, **src_kw)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(NA, L, L, sig)
    tcc = O.calc_tcc(src, sig, NA, synth.defocus_arg(defocus_nm, NA), L, L, Nx, Ny,
                     n_medium=n_medium)
    krn, sc, _ = O.calc_kernels(tcc, nk)
    return krn.astype(np.complex64), sc, Nx, Ny


def clear_field(krn, sc, Nx, Ny):
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2  # DC index of the band
    return float(np.sum(sc.astype(np.float64) * np.abs(krn[:, c].astype(np.complex128)) ** 2))


def gpu_images(masks, kernel_sets, Nx, Ny):
    import torch
    Ly, Lx = masks.shape[-2:]
    nk = kernel_sets[0][0].shape[0]
    plan = K.SocsPlan(Lx, Ly, Nx, Ny, nk, nsets=len(kernel_sets), max_clips=masks.shape[0])
    for i, (k, s) in enumerate(kernel_sets):
        plan.set_kernels(i, k, s)
    md = torch.from_numpy(np.ascontiguousarray(masks)).cuda()
    out = torch.empty((masks.shape[0], len(kernel_sets), Ly, Lx), dtype=torch.float32,
                      device="cuda")
    plan.forward(md, out)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    return res


def oracle_image(mask, krn, sc, Nx, Ny):
    return O.socs_image(mask, krn.astype(np.complex128), sc, Nx, Ny)


@pytest.mark.parametrize("L", [512, 1024])
def test_socs_physical_kernels(cuda, L):
    krn, sc, Nx, Ny = physical_kernels(L)
    mask = synth.rect_mask(L, int(60 * (L / 1024) ** 2) + 4, seed=L)
    got = gpu_images(mask[None], [(krn, sc)], Nx, Ny)[0, 0]
    want = oracle_image(mask, krn, sc, Nx, Ny)
    cf = clear_field(krn, sc, Nx, Ny)
    err = np.abs(got - want).max()
    assert err <= TOL_CF * cf, (err, cf)


@pytest.mark.parametrize("Lx,Ly,Nx,Ny", [(256, 256, 3, 3), (512, 256, 6, 3), (256, 512, 3, 6),
                                         (1024, 1024, 13, 13), (2048, 2048, 27, 27),
                                         (768, 512, 9, 6)])
def test_socs_random_kernels(cuda, Lx, Ly, Nx, Ny):
    krn, sc = synth.random_kernels(7, Nx, Ny, seed=Lx + Ly)
    mask = synth.rect_mask(Lx, 12, seed=3, Ly=Ly)
    got = gpu_images(mask[None], [(krn, sc)], Nx, Ny)[0, 0]
    want = oracle_image(mask, krn, sc, Nx, Ny)
    cf = clear_field(krn, sc, Nx, Ny)
    assert np.abs(got - want).max() <= TOL_CF * cf


def test_socs_batch_and_sets(cuda):
    L, Nx = 512, 6
    sets = [synth.random_kernels(5, Nx, Nx, seed=s) for s in (1, 2)]
    masks = np.stack([synth.rect_mask(L, 8, seed=s) for s in range(3)])
    got = gpu_images(masks, sets, Nx, Nx)
    for c in range(3):
        for s, (k, sc) in enumerate(sets):
            want = oracle_image(masks[c], k, sc, Nx, Nx)
            assert np.abs(got[c, s] - want).max() <= TOL_CF * clear_field(k, sc, Nx, Nx)


def test_socs_empty_and_clear_field(cuda):
    L, Nx = 256, 3
    krn, sc = synth.random_kernels(4, Nx, Nx, seed=9)
    masks = np.stack([np.zeros((L, L), np.float32), np.ones((L, L), np.float32)])
    got = gpu_images(masks, [(krn, sc)], Nx, Nx)
    assert np.abs(got[0, 0]).max() == 0.0
    cf = clear_field(krn, sc, Nx, Nx)
    assert np.abs(got[1, 0] - cf).max() <= TOL_CF * cf


def test_mask_spectrum_band(cuda):
    import torch
    L, Nx = 512, 6
    mask = synth.rect_mask(L, 10, seed=5)
    krn, sc = synth.random_kernels(2, Nx, Nx, seed=1)
    plan = K.SocsPlan(L, L, Nx, Nx, 2)
    md = torch.from_numpy(mask[None].copy()).cuda()
    band = torch.empty((1, 2 * Nx + 1, 2 * (2 * Nx + 1)), dtype=torch.float32, device="cuda")
    plan.mask_spectrum(md, band)
    torch.cuda.synchronize()
    b = band.cpu().numpy()[0]
    got = b[:, 0::2] + 1j * b[:, 1::2]
    full = O.ft_r2c(mask)
    want = full[L // 2 - Nx:L // 2 + Nx + 1, L // 2 - Nx:L // 2 + Nx + 1]
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


def test_socs_host_entry_matches_device(cuda):
    L, Nx = 512, 6
    krn, sc = synth.random_kernels(3, Nx, Nx, seed=4)
    masks = np.stack([synth.rect_mask(L, 9, seed=s) for s in (11, 12)])
    plan = K.SocsPlan(L, L, Nx, Nx, 3, max_clips=2)
    plan.set_kernels(0, krn, sc)
    host = plan.forward_host(masks)
    dev = gpu_images(masks, [(krn, sc)], Nx, Nx)
    assert np.array_equal(host, dev)


def test_socs_host_entry_pipelined_chunks(cuda):
    # 18 clips go through the host entry in 4 chunks (copy-in, compute and
    # copy-out streams overlapping); images equal the device-entry ones up to
    # the summation order of kernel slices
    L, Nx = 512, 6
    sets = [synth.random_kernels(5, Nx, Nx, seed=s) for s in (7, 8)]
    masks = np.stack([synth.rect_mask(L, 9, seed=100 + s) for s in range(18)])
    plan = K.SocsPlan(L, L, Nx, Nx, 5, nsets=2, max_clips=18)
    for i, (k, sc) in enumerate(sets):
        plan.set_kernels(i, k, sc)
    host = plan.forward_host(masks)
    again = plan.forward_host(masks)
    dev = gpu_images(masks, sets, Nx, Nx)
    scale = np.abs(dev).max()
    assert np.abs(host - dev).max() <= 1e-6 * scale
    assert np.array_equal(host, again)


def test_socs_engine_choice(cuda):
    # the specialised kernels take the periods they were built for; any other
    # period goes to the general pipeline rather than failing
    assert K.SocsPlan(1024, 1024, 13, 13, 2).engine == "specialised"
    assert K.SocsPlan(300, 300, 3, 3, 2).engine == "general"
    assert K.SocsPlan(1024, 1024, 13, 13, 2, general=True).engine == "general"


def test_resist_contour_matches_numpy(cuda):
    """kl_resist_contour on SOCS images: the sigmoid resist (the adjoint's
    model), the printed pattern I >= TARGET_INTENSITY (klitho_tcc.cpp:442) and
    its contour (printed pixels with a non-printing 4-neighbour, periodic)
    against numpy on the same float32 images."""
    import torch
    krn, sc, Nx, Ny = physical_kernels(1024)
    masks = np.stack([synth.rect_mask_fill(1024, seed=s, density=0.3) for s in (61, 62)])
    img = gpu_images(masks, [(krn, sc)], Nx, Ny)[:, 0]
    dev = torch.from_numpy(img.copy()).cuda()
    res = torch.empty_like(dev)
    pr = torch.empty(dev.shape, dtype=torch.uint8, device="cuda")
    ed = torch.empty(dev.shape, dtype=torch.uint8, device="cuda")
    cnt = torch.empty(2, dtype=torch.int64, device="cuda")
    K.resist_contour(dev, 50.0, 0.225, res, pr, ed, cnt)
    torch.cuda.synchronize()
    want_r = 1.0 / (1.0 + np.exp(-50.0 * (img.astype(np.float64) - 0.225)))
    assert np.abs(res.cpu().numpy() - want_r).max() <= 2e-6
    p = img >= np.float32(0.225)
    assert np.array_equal(pr.cpu().numpy().astype(bool), p)
    nb = np.zeros_like(p)
    for ax, sh in ((1, 1), (1, -1), (2, 1), (2, -1)):
        nb |= ~np.roll(p, sh, axis=ax)
    e = p & nb
    assert np.array_equal(ed.cpu().numpy().astype(bool), e)
    assert list(cnt.cpu().numpy()) == [int(e[i].sum()) for i in range(2)]
    assert e.sum() > 1000  # the clips do print a pattern
