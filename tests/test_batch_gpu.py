"""Batched SOCS imaging: the launch-shape autotuner (kl_socs_autotune) and
graph-captured batches of plans (kl_socs_batch_*).  Both change only how the
work is launched, so their images must equal the plain kl_socs_forward images
(up to the summation order of kernel slices: 1e-6 of clear field) and, through
those, the oracle (1e-5 of clear field, checked on one clip per size)."""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _setup(L, nclips, nsets, nk, seed):
    import torch
    src = K.createSource(41, "Annular", 0.6, 0.9)
    Nx, Ny = K.bandSize(synth.NA_IMMERSION, L, L, K.getOuterSigma(src))
    sets = []
    for s in range(nsets):
        krn, sc = synth.random_kernels(nk, Nx, Ny, seed=seed + s)
        sets.append((krn.astype(np.complex64), (sc / sc.sum() * 0.9).astype(np.float32)))
    plan = K.SocsPlan(L, L, Nx, Ny, nk, nsets=nsets, max_clips=nclips)
    for s, (k, sc) in enumerate(sets):
        plan.set_kernels(s, k, sc)
    masks = np.stack([synth.rect_mask(L, max(4, int(60 * (L / 1024) ** 2)), seed=seed + 10 + c)
                      for c in range(nclips)])
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    cf = max(float(np.sum(sc.astype(np.float64) * np.abs(k[:, c].astype(np.complex128)) ** 2))
             for k, sc in sets)
    return plan, torch.from_numpy(masks).cuda(), sets, Nx, Ny, cf


def _eager(plan, md):
    import torch
    out = torch.empty((md.shape[0], plan.nsets, plan.Ly, plan.Lx), dtype=torch.float32, device="cuda")
    plan.forward(md, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_autotune_keeps_images(cuda):
    import torch
    plan, md, sets, Nx, Ny, cf = _setup(1024, 6, 2, 24, seed=3)
    ref = _eager(plan, md)
    out = torch.full((6, 2, 1024, 1024), np.nan, dtype=torch.float32, device="cuda")
    ns, spc = plan.autotune(md, out)
    torch.cuda.synchronize()
    assert ns in (1, 2, 4, 8) and -2 <= spc <= 16  # spc < 0: the tensor-core engine
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-6 * cf
    again = _eager(plan, md)  # kl_socs_forward now uses the tuned shape
    assert np.abs(again - ref).max() <= 1e-6 * cf
    want = O.socs_image(md[0].cpu().numpy(), sets[1][0], sets[1][1], Nx, Ny)
    assert np.abs(again[0, 1] - want).max() <= 1e-5 * cf


def test_batch_graph_replays_and_recaptures(cuda):
    import torch
    cases = [(512, 5, 2, 16, 21), (1024, 3, 2, 24, 31), (2048, 2, 1, 24, 41)]
    plans, masks, cfs = [], [], []
    for L, n, ns, nk, seed in cases:
        p, md, sets, Nx, Ny, cf = _setup(L, n, ns, nk, seed)
        plans.append(p)
        masks.append(md)
        cfs.append(cf)
    plans[1].autotune(masks[1], torch.empty((3, 2, 1024, 1024), dtype=torch.float32, device="cuda"))
    batch = K.SocsBatch(plans)
    outs = [torch.full((m.shape[0], p.nsets, p.Ly, p.Lx), np.nan, dtype=torch.float32, device="cuda")
            for p, m in zip(plans, masks)]
    for _ in range(3):  # direct run + capture, then two replays
        batch.forward(masks, outs)
    torch.cuda.synchronize()
    assert batch.graph_builds() == 1
    for p, m, o, cf in zip(plans, masks, outs, cfs):
        assert np.abs(o.cpu().numpy() - _eager(p, m)).max() <= 1e-6 * cf
    # new mask contents in the same buffers: the replayed graph sees them
    for i, m in enumerate(masks):
        m.copy_(torch.flip(m, dims=[1]))
        outs[i].fill_(np.nan)
    batch.forward(masks, outs)
    torch.cuda.synchronize()
    assert batch.graph_builds() == 1
    for p, m, o, cf in zip(plans, masks, outs, cfs):
        assert np.abs(o.cpu().numpy() - _eager(p, m)).max() <= 1e-6 * cf
    # fewer clips for one plan: a new graph
    counts = [m.shape[0] for m in masks]
    counts[0] = 2
    outs[0].fill_(np.nan)
    batch.forward(masks, outs, nclips=counts)
    torch.cuda.synchronize()
    assert batch.graph_builds() == 2
    got = outs[0].cpu().numpy()
    assert np.isfinite(got[:2]).all() and np.isnan(got[2:]).all()
    batch.close()


def test_batch_stage_timing(cuda):
    import torch
    p, md, *_ = _setup(512, 4, 1, 12, seed=5)
    batch = K.SocsBatch([p])
    batch.enable_timing(True)
    out = torch.empty((4, 1, 512, 512), dtype=torch.float32, device="cuda")
    batch.forward([md], [out])
    batch.forward([md], [out])
    ms = batch.stage_times(0)
    assert len(ms) == 3 and all(t > 0 for t in ms)
    batch.close()


def test_batch_rejects_oversized_count(cuda):
    import torch
    p, md, *_ = _setup(512, 2, 1, 8, seed=6)
    batch = K.SocsBatch([p])
    out = torch.empty((2, 1, 512, 512), dtype=torch.float32, device="cuda")
    with pytest.raises(K.KLError, match="max_clips"):
        batch.forward([md], [out], nclips=[3])
    batch.close()
