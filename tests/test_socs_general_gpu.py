"""GPU parity of the general-geometry SOCS pipeline (socs_gen.cu) against the
FP64 oracle.

The reference images any period Lx x Ly (K-Litho-SOCS/klitho_socs.cpp:256-270)
with any band (its SOCS grid is 4N+1, :199-200).  The plans here run on the
general pipeline whenever the specialised kernels do not cover the geometry:
periods with factors other than 2 and 3, odd and prime periods, and bands up
to 4N+1 <= 256 (4096^2 clips at NA 1.35: N = 53, grid 213).  Oracle:
FT_r2c + calcSOCS + FI restated in FP64 (oracle/klitho_oracle.c), fed the same
float32 kernels.  Tolerance: 1e-5 of the clear-field intensity, the mixed
precision bar, as max |gpu - oracle| over all pixels.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_CF = 1e-5


def clear_field(krn, sc, Nx, Ny):
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    return float(np.sum(sc.astype(np.float64) * np.abs(krn[:, c].astype(np.complex128)) ** 2))


def gpu_images(masks, kernel_sets, Nx, Ny, general=False):
    import torch
    Ly, Lx = masks.shape[-2:]
    nk = kernel_sets[0][0].shape[0]
    plan = K.SocsPlan(Lx, Ly, Nx, Ny, nk, nsets=len(kernel_sets), max_clips=masks.shape[0],
                      general=general)
    engine = plan.engine
    for i, (k, s) in enumerate(kernel_sets):
        plan.set_kernels(i, k, s)
    md = torch.from_numpy(np.ascontiguousarray(masks)).cuda()
    out = torch.empty((masks.shape[0], len(kernel_sets), Ly, Lx), dtype=torch.float32, device="cuda")
    plan.forward(md, out)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    return res, engine


def oracle_image(mask, krn, sc, Nx, Ny):
    return O.socs_image(mask, krn.astype(np.complex128), sc, Nx, Ny)


# periods the specialised kernels do not take: factors other than 2 and 3,
# odd and prime sizes, non-square clips, a band too wide for them, and a
# 4096 period with its NA 1.35 band
@pytest.mark.parametrize("Lx,Ly,Nx,Ny", [
    (1000, 1000, 13, 13), (2000, 2000, 26, 26), (1001, 999, 13, 12), (300, 300, 3, 3),
    (640, 480, 8, 6), (2048, 1000, 27, 13), (131, 97, 1, 2), (4096, 4096, 53, 53),
    (1024, 1024, 40, 40), (5000, 250, 12, 3)])
def test_general_random_kernels(cuda, Lx, Ly, Nx, Ny):
    nk = 4 if Lx * Ly > 8_000_000 else 7
    krn, sc = synth.random_kernels(nk, Nx, Ny, seed=Lx + 3 * Ly)
    mask = synth.rect_mask(Lx, max(4, int(12 * Lx * Ly / 1024 ** 2)), seed=Lx + Ly, Ly=Ly)
    got, engine = gpu_images(mask[None], [(krn, sc)], Nx, Ny)
    assert engine == "general"
    want = oracle_image(mask, krn, sc, Nx, Ny)
    cf = clear_field(krn, sc, Nx, Ny)
    err = np.abs(got[0, 0] - want).max()
    assert err <= TOL_CF * cf, (err, cf)


@pytest.mark.parametrize("L", [512, 1024, 2048])
def test_general_equals_specialised(cuda, L):
    # the two pipelines on a geometry both cover: each within the bar of the
    # oracle, so within twice the bar of each other
    Nx = int(1.35 * L * 1.9 / 193)
    krn, sc = synth.random_kernels(6, Nx, Nx, seed=L)
    mask = synth.rect_mask(L, int(30 * (L / 1024) ** 2) + 4, seed=L + 5)
    a, ea = gpu_images(mask[None], [(krn, sc)], Nx, Nx, general=False)
    b, eb = gpu_images(mask[None], [(krn, sc)], Nx, Nx, general=True)
    assert (ea, eb) == ("specialised", "general")
    cf = clear_field(krn, sc, Nx, Nx)
    assert np.abs(a - b).max() <= 2 * TOL_CF * cf
    want = oracle_image(mask, krn, sc, Nx, Nx)
    assert np.abs(b[0, 0] - want).max() <= TOL_CF * cf


def test_general_batch_sets_and_clear_field(cuda):
    # three clips (one empty, one clear) under two kernel sets, period 1000
    L, Nx = 1000, 13
    sets = [synth.random_kernels(5, Nx, Nx, seed=s) for s in (21, 22)]
    masks = np.stack([synth.rect_mask(L, 10, seed=7), np.zeros((L, L), np.float32),
                      np.ones((L, L), np.float32)])
    got, engine = gpu_images(masks, sets, Nx, Nx)
    assert engine == "general"
    for s, (k, sc) in enumerate(sets):
        cf = clear_field(k, sc, Nx, Nx)
        want = oracle_image(masks[0], k, sc, Nx, Nx)
        assert np.abs(got[0, s] - want).max() <= TOL_CF * cf
        assert np.abs(got[1, s]).max() <= 1e-7 * cf
        assert np.abs(got[2, s] - cf).max() <= TOL_CF * cf


def test_general_mask_spectrum_band(cuda):
    import torch
    Lx, Ly, Nx, Ny = 1000, 999, 13, 12
    mask = synth.rect_mask(Lx, 10, seed=5, Ly=Ly)
    plan = K.SocsPlan(Lx, Ly, Nx, Ny, 2)
    assert plan.engine == "general"
    md = torch.from_numpy(mask[None].copy()).cuda()
    band = torch.empty((1, 2 * Ny + 1, 2 * (2 * Nx + 1)), dtype=torch.float32, device="cuda")
    plan.mask_spectrum(md, band)
    torch.cuda.synchronize()
    b = band.cpu().numpy()[0]
    got = b[:, 0::2] + 1j * b[:, 1::2]
    full = O.ft_r2c(mask)
    cy, cx = Ly // 2, Lx // 2
    want = full[cy - Ny:cy + Ny + 1, cx - Nx:cx + Nx + 1]
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


def test_general_host_entry(cuda):
    L, Nx = 1000, 13
    krn, sc = synth.random_kernels(3, Nx, Nx, seed=4)
    masks = np.stack([synth.rect_mask(L, 9, seed=s) for s in (11, 12, 13, 14)])
    plan = K.SocsPlan(L, L, Nx, Nx, 3, max_clips=4)
    plan.set_kernels(0, krn, sc)
    host = plan.forward_host(masks)
    dev, _ = gpu_images(masks, [(krn, sc)], Nx, Nx)
    assert np.abs(host - dev).max() <= 1e-6 * np.abs(dev).max()


def test_band_beyond_grid_limit_is_an_error(cuda):
    with pytest.raises(K.KLError) as e:
        K.SocsPlan(8192, 8192, 70, 70, 2)
    assert e.value.code == K.KL_ERR_UNSUPPORTED
