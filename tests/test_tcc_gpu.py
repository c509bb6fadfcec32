"""GPU parity of TCC assembly, top-K SOCS kernels and the Hopkins image.

Oracle: klitho_tcc.cpp's calcTCC / calcKernels (LAPACK zheevr) / calcImage
restated in FP64 (oracle/klitho_oracle.c, pinned to the reference build).
Tolerances:
  fast path  -- TCC relative Frobenius error <= 3e-5 (3-term BF16 split:
                each product keeps ~17 bits, ~3 * 2^-18 relative,
                FP32 accumulate); eigenvalues relative <= 1e-6; weighted
                projector sum_k lam_k v_k v_k^H relative <= 1e-5; Hopkins
                image <= 1e-5 of clear-field intensity.
  FP64 path  -- TCC max abs error <= 1e-12 of max |TCC|; eigenvalues
                relative <= 1e-10.
Kernels are compared as projectors: eigenvector phases (and rotations inside
degenerate pairs) are arbitrary.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = {
    # name: (L, source type, srcSize, source kwargs, NA, n_medium, defocus arg, nk)
    "annular512": (512, "Annular", 41, dict(innerRadius=0.6, outerRadius=0.9), 1.35, 1.44, 0.0, 24),
    "annular1024": (1024, "Annular", 41, dict(innerRadius=0.6, outerRadius=0.9), 1.35, 1.44,
                    synth.defocus_arg(25.0), 24),
    "dipole2048": (2048, "Dipole", 61, dict(radius=0.15, offset=0.7, onXAxis=1), 1.35, 1.44,
                   synth.defocus_arg(-50.0), 32),
    "dry_na08": (512, "Annular", 41, dict(innerRadius=0.5, outerRadius=0.8), 0.8, 1.0, 0.2, 12),
    "quad512": (512, "CrossQuadrupole", 41, dict(radius=0.12, offset=0.75), 1.35, 1.44, 0.0, 16),
    # 196 source points: the one-step Gram solve on a thread-block cluster
    "quad81_512": (512, "CrossQuadrupole", 81, dict(radius=0.12, offset=0.75), 1.35, 1.44,
                   synth.defocus_arg(30.0), 32),
}

_oracle_cache = {}


def oracle_case(name):
    if name not in _oracle_cache:
        L, kind, n, kw, NA, nm, df, nk = CASES[name]
        src = K.createSource(n, kind, **kw)
        sig = O.outer_sigma(src)
        Nx, Ny = O.band(NA, L, L, sig)
        tcc = O.calc_tcc(src, sig, NA, df, L, L, Nx, Ny, n_medium=nm)
        krn, sc, ev = O.calc_kernels(tcc, nk)
        _oracle_cache[name] = (src, Nx, Ny, tcc, krn, sc, ev)
    return _oracle_cache[name]


def tensor_to_complex(T):
    a = T.cpu().numpy()
    return a[..., 0] + 1j * a[..., 1]


def weighted_projector(krn, ev):
    # kernels are index-reversed eigenvectors: undo the reversal first
    V = np.asarray(krn, dtype=np.complex128)[:, ::-1].T  # N x K
    return (V * np.asarray(ev, dtype=np.float64)[None, :]) @ V.conj().T


@pytest.mark.parametrize("name", list(CASES))
def test_tcc_fast_matches_oracle(cuda, name):
    L, kind, n, kw, NA, nm, df, nk = CASES[name]
    src, Nx, Ny, tcc_ref, *_ = oracle_case(name)
    plan = K.TccPlan(src, NA, df, L, L, n_medium=nm)
    assert (plan.Nx, plan.Ny) == (Nx, Ny)
    T = tensor_to_complex(plan.build())
    rel = np.linalg.norm(T - tcc_ref) / np.linalg.norm(tcc_ref)
    assert rel <= 3e-5, rel
    assert np.array_equal(T, T.conj().T)  # exactly Hermitian by construction
    mm = plan.minmax(plan.build())
    assert abs(mm[0] - tcc_ref.real.max()) <= 3e-5 * abs(tcc_ref.real.max())


@pytest.mark.parametrize("name", ["annular512", "dry_na08", "quad512"])
def test_tcc_fp64_matches_oracle(cuda, name):
    L, kind, n, kw, NA, nm, df, nk = CASES[name]
    src, Nx, Ny, tcc_ref, *_ = oracle_case(name)
    plan = K.TccPlan(src, NA, df, L, L, n_medium=nm, precision=K.PREC_FP64)
    T = tensor_to_complex(plan.build())
    err = np.abs(T - tcc_ref).max()
    assert err <= 1e-12 * np.abs(tcc_ref).max(), err


@pytest.mark.parametrize("name", list(CASES))
def test_topk_fast_matches_zheevr(cuda, name):
    L, kind, n, kw, NA, nm, df, nk = CASES[name]
    src, Nx, Ny, tcc_ref, krn_ref, sc_ref, ev_ref = oracle_case(name)
    plan = K.TccPlan(src, NA, df, L, L, n_medium=nm)
    krn, sc, ev, it = plan.topk(nk)
    rel_ev = np.abs(ev - ev_ref) / np.abs(ev_ref).max()
    assert rel_ev.max() <= 1e-6, (rel_ev.max(), it)
    P = weighted_projector(krn, ev)
    Pr = weighted_projector(krn_ref, ev_ref)
    assert np.linalg.norm(P - Pr) / np.linalg.norm(Pr) <= 1e-5
    # kernels are unit vectors
    assert np.allclose(np.linalg.norm(krn.astype(np.complex128), axis=1), 1.0, atol=1e-6)


@pytest.mark.parametrize("name", ["annular512", "dry_na08"])
def test_topk_fp64_matches_zheevr(cuda, name):
    L, kind, n, kw, NA, nm, df, nk = CASES[name]
    src, Nx, Ny, tcc_ref, krn_ref, sc_ref, ev_ref = oracle_case(name)
    plan = K.TccPlan(src, NA, df, L, L, n_medium=nm, precision=K.PREC_FP64)
    krn, sc, ev, it = plan.topk(nk)
    assert np.abs(ev - ev_ref).max() <= 1e-10 * np.abs(ev_ref).max()
    P = weighted_projector(krn, ev)
    Pr = weighted_projector(krn_ref, ev_ref)
    # float32 kernel output limits the projector agreement
    assert np.linalg.norm(P - Pr) / np.linalg.norm(Pr) <= 1e-6


@pytest.mark.parametrize("name", ["annular512", "dry_na08", "annular1024"])
def test_hopkins_image_matches_calcimage(cuda, name):
    import torch
    L, kind, n, kw, NA, nm, df, nk = CASES[name]
    src, Nx, Ny, tcc_ref, *_ = oracle_case(name)
    plan = K.TccPlan(src, NA, df, L, L, n_medium=nm)
    mask = synth.rect_mask(L, int(60 * (L / 1024) ** 2) + 6, seed=11)
    md = torch.from_numpy(mask[None].copy()).cuda()
    img = torch.empty((1, 1, L, L), dtype=torch.float32, device="cuda")
    plan.hopkins(md, img)
    torch.cuda.synchronize()
    got = img.cpu().numpy()[0, 0]
    _, want = O.hopkins_image(mask, tcc_ref, Nx, Ny)
    cf = float(tcc_ref[(tcc_ref.shape[0] - 1) // 2, (tcc_ref.shape[0] - 1) // 2].real)
    assert np.abs(got - want).max() <= 1e-5 * cf


def test_topk_beyond_rank_is_zero(cuda):
    # a single point source has a rank-1 TCC: one kernel = the pupil, rest zero
    src = K.createSource(21, "Point", ptX=0.3, ptY=-0.2)
    plan = K.TccPlan(src, 0.8, 0.0, 256, 256)
    krn, sc, ev, it = plan.topk(3)
    assert ev[0] > 0 and np.all(ev[1:] == 0) and np.all(krn[1:] == 0)


def test_topk_batch_focus_sweep(cuda):
    # one plan per focus value, solved in one call; each must agree with its
    # single-plan solve and with zheevr on the oracle TCC
    L, nk = 512, 32
    src = K.createSource(61, "Dipole", radius=0.15, offset=0.7, onXAxis=1)
    focus = [-50.0, 0.0, 35.0]
    plans = [K.TccPlan(src, 1.35, synth.defocus_arg(f), L, L, n_medium=1.44) for f in focus]
    kb, sb, eb, itb = K.TccPlan.topk_batch(plans, nk)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, L, L, sig)
    for i, f in enumerate(focus):
        k1, s1, e1, _ = plans[i].topk(nk)
        assert np.abs(eb[i] - e1).max() <= 1e-12 * np.abs(e1).max()
        assert np.linalg.norm(weighted_projector(kb[i], eb[i]) - weighted_projector(k1, e1)) <= \
            1e-6 * np.linalg.norm(weighted_projector(k1, e1))
        tcc = O.calc_tcc(src, sig, 1.35, synth.defocus_arg(f), L, L, Nx, Ny, n_medium=1.44)
        kr, _, er = O.calc_kernels(tcc, nk)
        assert np.abs(eb[i] - er).max() <= 1e-6 * np.abs(er).max()
        Pr = weighted_projector(kr, er)
        assert np.linalg.norm(weighted_projector(kb[i], eb[i]) - Pr) / np.linalg.norm(Pr) <= 1e-5
        assert 0 < itb[i] < 40  # iterations of the one Gram solve (1 for the tridiagonal solver)


def eig_residual(krn, ev, tcc):
    """max_k ||T v_k - lam_k v_k|| / lam_0 over the returned kernels."""
    V = np.asarray(krn, dtype=np.complex128)[:, ::-1].T  # N x K
    R = tcc @ V - V * np.asarray(ev, dtype=np.float64)[None, :]
    return np.linalg.norm(R, axis=0).max() / abs(ev[0])


def gap_cut(w, hi, rel=1e-3):
    """largest n <= hi with lam_{n-1} - lam_n > rel lam_0 (a unique top-n projector)."""
    return max(n for n in range(1, hi + 1) if w[n - 1] - w[n] > rel * w[0])


def test_topk_batch_cluster_gram(cuda):
    # 196 source points: each focus value's 196 x 196 Gram eigensolve runs on
    # one thread-block cluster (the tridiagonal reduction), three in one launch
    L, nk = 512, 48
    src = K.createSource(71, "CrossQuadrupole", radius=0.12, offset=0.75)
    assert int((np.asarray(src) > 0).sum()) == 196
    focus = [-40.0, 10.0, 60.0]
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, L, L, sig)
    plans = [K.TccPlan(src, 1.35, synth.defocus_arg(f), L, L, n_medium=1.44) for f in focus]
    kb, sb, eb, itb = K.TccPlan.topk_batch(plans, nk)
    for i, f in enumerate(focus):
        tcc = O.calc_tcc(src, sig, 1.35, synth.defocus_arg(f), L, L, Nx, Ny, n_medium=1.44)
        kr, _, er = O.calc_kernels(tcc, nk)
        assert np.abs(eb[i] - er).max() <= 1e-6 * np.abs(er).max()
        # eigenpairs of the TCC whatever the degenerate pairs (BF16x3 TCC: ~3e-5)
        assert eig_residual(kb[i], eb[i], tcc) <= 1e-4
        n = gap_cut(np.linalg.eigvalsh(tcc)[::-1], nk)
        Pr = weighted_projector(kr[:n], er[:n])
        assert np.linalg.norm(weighted_projector(kb[i][:n], eb[i][:n]) - Pr) / np.linalg.norm(Pr) <= 1e-5
        assert np.allclose(np.linalg.norm(kb[i].astype(np.complex128), axis=1), 1.0, atol=1e-6)
        assert 0 < itb[i] < 40


def test_topk_subspace_cluster_block(cuda):
    # 572 source points (subspace iteration) with an 80-kernel request: the
    # 120-wide Rayleigh-Ritz blocks are solved by the cluster Jacobi
    L, nk = 1024, 80
    src = K.createSource(41, "Annular", 0.6, 0.9)
    plan = K.TccPlan(src, 1.35, synth.defocus_arg(20.0), L, L, n_medium=1.44)
    krn, sc, ev, it = plan.topk(nk)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, L, L, sig)
    tcc = O.calc_tcc(src, sig, 1.35, synth.defocus_arg(20.0), L, L, Nx, Ny, n_medium=1.44)
    kr, _, er = O.calc_kernels(tcc, nk)
    assert np.abs(ev - er).max() <= 1e-6 * np.abs(er).max(), it
    assert eig_residual(krn, ev, tcc) <= 1e-4
    n = gap_cut(np.linalg.eigvalsh(tcc)[::-1], nk)
    Pr = weighted_projector(kr[:n], er[:n])
    assert np.linalg.norm(weighted_projector(krn[:n], ev[:n]) - Pr) / np.linalg.norm(Pr) <= 1e-5


@pytest.mark.parametrize("precision", [K.PREC_FAST, K.PREC_FP64])
def test_topk_batch_sequential_paths(cuda, precision):
    # more than 128 source points (subspace iteration) or FP64 plans: the batch
    # is solved plan by plan and must equal the single-plan results
    L, nk = 512, 16
    src = K.createSource(41, "Annular", 0.6, 0.9)
    plans = [K.TccPlan(src, 1.35, synth.defocus_arg(f), L, L, n_medium=1.44, precision=precision)
             for f in (-25.0, 25.0)]
    kb, sb, eb, itb = K.TccPlan.topk_batch(plans, nk)
    for i in range(2):
        k1, s1, e1, it1 = plans[i].topk(nk)
        assert np.abs(eb[i] - e1).max() <= 1e-12 * np.abs(e1).max()
        assert itb[i] == it1


def test_topk_batch_rejects_mixed_band(cuda):
    src = K.createSource(41, "Annular", 0.6, 0.9)
    a = K.TccPlan(src, 1.35, 0.0, 512, 512, n_medium=1.44)
    b = K.TccPlan(src, 1.35, 0.0, 1024, 1024, n_medium=1.44)
    with pytest.raises(RuntimeError, match="same N"):
        K.TccPlan.topk_batch([a, b], 8)


def custom_source(S, size=41, seed=0):
    """A source map of exactly S points (uniform weights) inside 0.9 of the pupil radius."""
    rng = np.random.default_rng(seed)
    sh = (size - 1) // 2
    cand = [(p, q) for q in range(-sh, sh + 1) for p in range(-sh, sh + 1) if p * p + q * q <= (0.9 * sh) ** 2]
    pick = rng.choice(len(cand), size=S, replace=False)
    src = np.zeros((size, size), dtype=np.float32)
    for i in pick:
        p, q = cand[i]
        src[q + sh, p + sh] = 1.0 / S
    return src


@pytest.mark.parametrize("S", [63, 64, 250])
def test_topk_gram_size_boundaries(cuda, S):
    # Gram orders at the solver's boundaries: 63 (one CTA), 64 (the smallest
    # cluster, 4 indices per group) and 250 (padded to 256: 16 per group, the
    # largest cluster layout, with padding indices)
    L, nk = 1024, 24
    src = custom_source(S, seed=S)
    sig = O.outer_sigma(src)
    assert O.source_point_count(src, sig) == S
    Nx, Ny = O.band(1.35, L, L, sig)
    plan = K.TccPlan(src, 1.35, synth.defocus_arg(15.0), L, L, n_medium=1.44)
    assert plan.S == S
    krn, sc, ev, it = plan.topk(nk)
    tcc = O.calc_tcc(src, sig, 1.35, synth.defocus_arg(15.0), L, L, Nx, Ny, n_medium=1.44)
    kr, _, er = O.calc_kernels(tcc, nk)
    assert np.abs(ev - er).max() <= 1e-6 * np.abs(er).max(), it
    assert eig_residual(krn, ev, tcc) <= 1e-4
    n = gap_cut(np.linalg.eigvalsh(tcc)[::-1], nk)
    Pr = weighted_projector(kr[:n], er[:n])
    assert np.linalg.norm(weighted_projector(krn[:n], ev[:n]) - Pr) / np.linalg.norm(Pr) <= 1e-5
    assert 0 < it < 40


def principal_angles_at_gaps(kf, kr, ev, rel_gap=1e-4):
    """Largest principal angle between the spans of the first m kernels of two
    solves, at every cut m where the reference spectrum has a gap."""
    qa, _ = np.linalg.qr(np.asarray(kf, np.complex128).T)
    qb, _ = np.linalg.qr(np.asarray(kr, np.complex128).T)
    out = []
    for m in range(1, qa.shape[1]):
        if (ev[m - 1] - ev[m]) / ev[0] > rel_gap:
            sv = np.linalg.svd(qa[:, :m].conj().T @ qb[:, :m], compute_uv=False)
            out.append((m, float(np.arccos(np.clip(sv.min(), -1.0, 1.0)))))
    return out


def test_config4_fast_vs_fp64_gpu_path(cuda):
    """The stress configuration (4096^2, cross-quadrupole 0.75/0.12 on 81^2,
    NA 1.35 water: N = 11449, S = 196, K = 64): the fast path's TCC, eigenvalues
    and kernels against the plain FP64 GPU path, which the tests above pin to
    zheevr at sizes the CPU oracle handles.  Kernels are compared as weighted
    projectors and by principal angles at every spectral-gap cut."""
    import torch
    src = K.createSource(81, "CrossQuadrupole", radius=0.12, offset=0.75)
    df = synth.defocus_arg(25.0)
    tf = K.TccPlan(src, 1.35, df, 4096, 4096, n_medium=1.44)
    t64 = K.TccPlan(src, 1.35, df, 4096, 4096, n_medium=1.44, precision=K.PREC_FP64)
    assert (tf.N, tf.S) == (11449, 196)
    kf, sf, evf, _ = tf.topk(64)
    k64, s64, ev64, _ = t64.topk(64)
    assert np.max(np.abs(evf - ev64)) <= 1e-6 * ev64[0]
    cuts = principal_angles_at_gaps(kf, k64, ev64)
    assert len(cuts) >= 8
    assert max(a for _, a in cuts) <= 1e-3, cuts
    # weighted projectors through K x K Gram products
    w = np.sqrt(np.maximum(ev64, 0))
    A = np.asarray(kf, np.complex128).T * w[None, :]
    B = np.asarray(k64, np.complex128).T * w[None, :]
    aa, bb, ab = A.conj().T @ A, B.conj().T @ B, A.conj().T @ B
    d2 = np.real(np.trace(aa @ aa) + np.trace(bb @ bb) - 2 * np.trace(ab @ ab.conj().T))
    assert np.sqrt(max(d2, 0.0)) <= 1e-5 * np.sqrt(np.real(np.trace(bb @ bb)))
    # the materialised TCC: tcgen05 BF16x3 against the FP64 accumulation
    Tf = tf.build()
    T64 = t64.build()
    num = torch.linalg.norm(Tf.double() - T64)
    assert float(num / torch.linalg.norm(T64)) <= 3e-5
    del Tf, T64
    tf.close()
    t64.close()


def test_topk_planes_and_interleaved_agree(cuda):
    # kl_topk_eig (two float planes, the CLI's layout) and kl_topk_eig_c64
    # (interleaved, behind TccPlan.topk) return the same kernels bit for bit,
    # including the zero kernels beyond the rank (nk > S)
    import ctypes
    src = K.createSource(71, "CrossQuadrupole", radius=0.12, offset=0.75)
    plan = K.TccPlan(src, 1.35, synth.defocus_arg(-20.0), 1024, 1024, n_medium=1.44)
    nk, N = plan.S + 4, plan.N
    assert nk <= N  # rank S < nk: the last four kernels are zero
    krn, sc, ev, it = plan.topk(nk)
    re = np.empty(nk * N, np.float32)
    im = np.empty(nk * N, np.float32)
    sc2 = np.zeros(nk, np.float32)
    ev2 = np.zeros(nk, np.float64)
    it2 = ctypes.c_int()
    K.check(K.lib().kl_topk_eig(plan._h, nk, 0, re.ctypes.data_as(K._c_float_p), im.ctypes.data_as(K._c_float_p),
                                sc2.ctypes.data_as(K._c_float_p), ev2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                ctypes.byref(it2)), "kl_topk_eig")
    plan.close()
    assert np.array_equal(krn.real.ravel(), re) and np.array_equal(krn.imag.ravel(), im)
    assert np.array_equal(sc, sc2) and np.array_equal(ev, ev2) and it == it2.value
    assert np.all(krn[-4:] == 0) and np.all(ev[-4:] == 0)


def test_topk_batch_mixed_gram_orders(cuda):
    # two sources with the same outer sigma (same band N) but 120 and 200 points:
    # one batched launch holds Gram solves of different orders; each must equal
    # the plan's own solve
    sh = 20
    far = (sh, 0)  # the same farthest point in both sources fixes sigma_o

    def src_with(S, seed):
        rng = np.random.default_rng(seed)
        cand = [(p, q) for q in range(-sh, sh + 1) for p in range(-sh, sh + 1)
                if p * p + q * q <= (0.8 * sh) ** 2]
        pick = rng.choice(len(cand), size=S - 1, replace=False)
        src = np.zeros((2 * sh + 1, 2 * sh + 1), dtype=np.float32)
        for i in pick:
            p, q = cand[i]
            src[q + sh, p + sh] = 1.0
        src[far[1] + sh, far[0] + sh] = 1.0
        return src

    L, nk = 1024, 24
    srcs = [src_with(120, 1), src_with(200, 2)]
    plans = [K.TccPlan(s, 1.35, synth.defocus_arg(10.0), L, L, n_medium=1.44) for s in srcs]
    assert [p.S for p in plans] == [120, 200] and plans[0].N == plans[1].N
    kb, sb, eb, itb = K.TccPlan.topk_batch(plans, nk)
    for i, p in enumerate(plans):
        k1, s1, e1, it1 = p.topk(nk)
        assert np.abs(eb[i] - e1).max() <= 1e-12 * np.abs(e1).max()
        assert np.linalg.norm(weighted_projector(kb[i], eb[i]) - weighted_projector(k1, e1)) <= \
            1e-10 * np.linalg.norm(weighted_projector(k1, e1))
        p.close()
