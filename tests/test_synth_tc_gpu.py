"""GPU parity of the tensor-core image synthesis (FP16x3 split GEMM of the row
coefficients against a cos/sin basis) with the FP64 oracle and with the
CUDA-core synthesis of the same plan.

The oracle image is K-Litho-SOCS/klitho_socs.cpp's FT_r2c + calcSOCS + FI
restated in FP64 (oracle/klitho_oracle.c).  Tolerance: 1e-5 of the clear-field
intensity, max |gpu - oracle| over all pixels, as for the CUDA-core engine.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

from test_socs_gpu import clear_field, oracle_image, physical_kernels

pytestmark = pytest.mark.gpu

TOL_CF = 1e-5


def run_plan(masks, kernel_sets, Nx, Ny, mode, adjoint=False):
    import torch
    Ly, Lx = masks.shape[-2:]
    nk = kernel_sets[0][0].shape[0]
    plan = K.SocsPlan(Lx, Ly, Nx, Ny, nk, nsets=len(kernel_sets), max_clips=masks.shape[0],
                      adjoint=adjoint)
    assert plan.engine == "specialised"
    for i, (k, s) in enumerate(kernel_sets):
        plan.set_kernels(i, k, s)
    plan.set_synthesis(mode)
    assert plan.synthesis(masks.shape[0]) == mode
    md = torch.from_numpy(np.ascontiguousarray(masks)).cuda()
    out = torch.full((masks.shape[0], len(kernel_sets), Ly, Lx), float("nan"), dtype=torch.float32,
                     device="cuda")
    plan.forward(md, out)
    plan.status()
    res = out.cpu().numpy()
    plan.close()
    return res


@pytest.mark.parametrize("Lx,Ly,Nx,Ny", [(256, 256, 3, 3), (512, 256, 6, 3), (256, 512, 3, 6),
                                         (1024, 1024, 13, 13), (2048, 2048, 27, 27),
                                         (768, 512, 9, 6), (1024, 1024, 31, 20)])
def test_tc_synthesis_random_kernels(cuda, Lx, Ly, Nx, Ny):
    krn, sc = synth.random_kernels(7, Nx, Ny, seed=Lx + Ly)
    mask = synth.rect_mask(Lx, 12, seed=3, Ly=Ly)
    got = run_plan(mask[None], [(krn, sc)], Nx, Ny, "tensor")[0, 0]
    want = oracle_image(mask, krn, sc, Nx, Ny)
    cf = clear_field(krn, sc, Nx, Ny)
    assert np.isfinite(got).all()
    assert np.abs(got - want).max() <= TOL_CF * cf


@pytest.mark.parametrize("L", [512, 1024, 2048])
def test_tc_synthesis_physical_kernels(cuda, L):
    krn, sc, Nx, Ny = physical_kernels(L)
    mask = synth.rect_mask(L, int(60 * (L / 1024) ** 2) + 4, seed=L)
    got = run_plan(mask[None], [(krn, sc)], Nx, Ny, "tensor")[0, 0]
    want = oracle_image(mask, krn, sc, Nx, Ny)
    cf = clear_field(krn, sc, Nx, Ny)
    assert np.abs(got - want).max() <= TOL_CF * cf


def test_tc_synthesis_adjoint_plan_strips(cuda):
    # adjoint plans use taller strips (J >= 4Ny+1: 64 rows here, two strips a tile)
    L, Nx = 1024, 13
    krn, sc = synth.random_kernels(6, Nx, Nx, seed=5)
    mask = synth.rect_mask(L, 30, seed=8)
    got = run_plan(mask[None], [(krn, sc)], Nx, Nx, "tensor", adjoint=True)[0, 0]
    want = oracle_image(mask, krn, sc, Nx, Nx)
    assert np.abs(got - want).max() <= TOL_CF * clear_field(krn, sc, Nx, Nx)


def test_tc_synthesis_many_tiles_per_cta(cuda):
    # 150 clips x 2 sets of 256^2: 600 row tiles over at most 296 CTAs, so CTAs
    # run several tiles and cross image boundaries; compared with the CUDA-core
    # engine everywhere and with the oracle on a few images
    L, Nx = 256, 3
    sets = [synth.random_kernels(5, Nx, Nx, seed=s) for s in (1, 2)]
    masks = np.stack([synth.rect_mask(L, 6, seed=s) for s in range(150)])
    masks[7] *= 1000.0   # exponent of the power-of-two scale far from 1
    masks[8] = 0.0       # all-zero spectrum
    tc = run_plan(masks, sets, Nx, Nx, "tensor")
    cu = run_plan(masks, sets, Nx, Nx, "cuda")
    for s, (k, scl) in enumerate(sets):
        cf = clear_field(k, scl, Nx, Nx)
        peak = np.abs(cu[:, s]).reshape(150, -1).max(axis=1)
        err = np.abs(tc[:, s] - cu[:, s]).reshape(150, -1).max(axis=1)
        assert (err <= 2 * TOL_CF * np.maximum(cf, peak)).all()
        for c in (0, 7, 149):
            want = oracle_image(masks[c], k, scl, Nx, Nx)
            assert np.abs(tc[c, s] - want).max() <= TOL_CF * max(cf, np.abs(want).max())
    assert np.abs(tc[8]).max() == 0.0


def test_tc_synthesis_autotune_and_errors(cuda):
    import torch
    L, Nx = 512, 6
    krn, sc = synth.random_kernels(8, Nx, Nx, seed=4)
    masks = np.stack([synth.rect_mask(L, 8, seed=s) for s in range(4)])
    plan = K.SocsPlan(L, L, Nx, Nx, 8, max_clips=4)
    plan.set_kernels(0, krn, sc)
    md = torch.from_numpy(masks).cuda()
    out = torch.empty((4, 1, L, L), dtype=torch.float32, device="cuda")
    ns, spc = plan.autotune(md, out)
    assert plan.synthesis(4) == ("tensor" if spc < 0 else "cuda")
    plan.forward(md, out)
    plan.status()
    got = out.cpu().numpy()
    cf = clear_field(krn, sc, Nx, Nx)
    for c in range(4):
        assert np.abs(got[c, 0] - oracle_image(masks[c], krn, sc, Nx, Nx)).max() <= TOL_CF * cf
    plan.close()
    # no tensor-core synthesis for Ly not a multiple of 128, nor on the general pipeline
    odd = K.SocsPlan(256, 288, 3, 3, 4)
    assert odd.engine == "specialised"
    with pytest.raises(Exception):
        odd.set_synthesis("tensor")
    assert odd.synthesis(1) == "cuda"
    odd.close()
    gen = K.SocsPlan(1000, 1000, 7, 7, 4)
    assert gen.engine == "general"
    with pytest.raises(Exception):
        gen.set_synthesis("tensor")
    gen.close()


def test_tc_mask_range_reported(cuda):
    # mask values beyond the FP16 range of the tensor-core mask transform are
    # reported through the plan status, not silently imaged
    import torch
    L, Nx = 256, 3
    krn, sc = synth.random_kernels(4, Nx, Nx, seed=2)
    plan = K.SocsPlan(L, L, Nx, Nx, 4, max_clips=1)
    plan.set_kernels(0, krn, sc)
    plan.set_synthesis("tensor")
    mask = synth.rect_mask(L, 4, seed=1)
    mask[5, 7] = 1.0e6
    md = torch.from_numpy(mask[None].copy()).cuda()
    out = torch.empty((1, 1, L, L), dtype=torch.float32, device="cuda")
    plan.forward(md, out)
    with pytest.raises(Exception):
        plan.status()
    plan.status()  # cleared by the previous call
    plan.close()
