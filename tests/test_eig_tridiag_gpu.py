"""GPU tests of the Hermitian top-K eigensolver behind the Gram step of
kl_topk_eig (tridiagonal reduction on a thread-block cluster, bisection,
inverse iteration): kl_hermitian_topk against numpy's eigh (LAPACK) on
matrices whose spectra stress each stage -- random, exactly degenerate,
rank-deficient, already diagonal or tridiagonal, and the Gram matrix of a
real TCC factor (one dominant eigenvalue, degenerate symmetric pairs).

Tolerances (FP64 throughout): eigenvalues within 1e-12 ||H||, residuals
||H v - lam v|| within 1e-12 ||H||, orthonormality within 1e-12, and the
projector onto every group of eigenvalues closer than 1e-5 ||H|| within 1e-10
of LAPACK's.
"""
import numpy as np
import pytest

import klitho as K
import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def solve(H, k):
    import torch
    B = H.shape[0]
    Hd = torch.from_numpy(np.ascontiguousarray(H, dtype=np.complex128)).cuda()
    ev = torch.full((k,), float("nan"), dtype=torch.float64, device="cuda")
    V = torch.full((B, k), complex("nan"), dtype=torch.complex128, device="cuda")
    K.hermitian_topk(Hd, k, ev, V)
    torch.cuda.synchronize()
    assert np.array_equal(Hd.cpu().numpy(), H)  # the input is left alone
    return ev.cpu().numpy(), V.cpu().numpy()


def check(H, k, proj_tol=1e-10):
    ev, V = solve(H, k)
    w, Q = np.linalg.eigh(H)
    w, Q = w[::-1], Q[:, ::-1]
    nh = np.abs(w).max()
    assert np.isfinite(ev).all() and np.isfinite(V).all()
    assert np.all(np.diff(ev) <= 1e-12 * nh)  # descending
    assert np.abs(ev - w[:k]).max() <= 1e-12 * nh
    assert np.linalg.norm(H @ V - V * ev[None, :], axis=0).max() <= 1e-12 * nh
    assert np.abs(V.conj().T @ V - np.eye(k)).max() <= 1e-12
    # projectors onto groups of eigenvalues closer than 1e-5 ||H|| (within a group the
    # vectors are determined only up to rotation) that lie wholly inside the top k
    start = 0
    for i in range(1, k + 1):
        if i == k or w[i - 1] - w[i] > 1e-5 * nh:
            if i == k and k < len(w) and w[k - 1] - w[k] <= 1e-5 * nh:
                break  # the cluster continues past the cut
            Pa = V[:, start:i] @ V[:, start:i].conj().T
            Pb = Q[:, start:i] @ Q[:, start:i].conj().T
            assert np.abs(Pa - Pb).max() <= proj_tol, (start, i)
            start = i
    return ev, V


def random_hermitian(B, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, B)) + 1j * rng.standard_normal((B, B))
    return (X + X.conj().T) / 2


def with_spectrum(lam, seed):
    rng = np.random.default_rng(seed)
    B = len(lam)
    X = rng.standard_normal((B, B)) + 1j * rng.standard_normal((B, B))
    U, _ = np.linalg.qr(X)
    H = (U * np.asarray(lam, dtype=np.float64)[None, :]) @ U.conj().T
    return (H + H.conj().T) / 2


@pytest.mark.parametrize("B,k", [(64, 64), (64, 1), (97, 24), (196, 64), (255, 40), (256, 256)])
def test_random_hermitian(cuda, B, k):
    check(random_hermitian(B, seed=B + k), k)


def test_degenerate_and_clustered_spectrum(cuda):
    B = 150
    lam = np.linspace(1.0, 0.01, B)
    lam[3:5] = 0.8                     # an exact pair
    lam[10:15] = 0.5                   # a five-fold eigenvalue
    lam[20:22] = [0.3, 0.3 + 1e-13]    # a pair closer than the solver's cluster tolerance
    lam[30:32] = [0.2, 0.2 + 1e-6]     # a pair just outside it
    check(with_spectrum(lam, seed=3), 40)


def test_rank_deficient_gram(cuda):
    # 70 x 70 Gram of a 70 x 30 factor: 40 zero eigenvalues in one cluster
    rng = np.random.default_rng(7)
    A = rng.standard_normal((30, 70)) + 1j * rng.standard_normal((30, 70))
    G = A.conj().T @ A
    G = (G + G.conj().T) / 2
    ev, V = check(G, 30)
    ev2, V2 = solve(G, 70)  # all of them, the null space included
    assert np.abs(V2.conj().T @ V2 - np.eye(70)).max() <= 1e-12
    assert np.abs(np.sort(ev2)[::-1] - np.linalg.eigvalsh(G)[::-1]).max() <= 1e-12 * ev2[0]


def test_diagonal_and_tridiagonal_inputs(cuda):
    B = 80
    rng = np.random.default_rng(11)
    D = np.diag(rng.standard_normal(B)).astype(np.complex128)  # every reflector is the identity
    check(D, 20)
    T = np.diag(rng.standard_normal(B)).astype(np.complex128)
    off = rng.standard_normal(B - 1) + 1j * rng.standard_normal(B - 1)
    off[[9, 40, 41]] = 0.0  # the tridiagonal splits into blocks
    T += np.diag(off, -1) + np.diag(off.conj(), 1)
    check(T, 30)


def test_tcc_gram_matrix(cuda):
    # G = A^H A of the pupil factor of a cross-quadrupole source (196 points)
    src = K.createSource(71, "CrossQuadrupole", radius=0.12, offset=0.75)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, 512, 512, sig)
    P, _, J = O.pupil_matrix(src, sig, 1.35, synth.defocus_arg(30.0), 512, 512, Nx, Ny, n_medium=1.44)
    A = P * np.sqrt(J.astype(np.float64))[None, :]
    G = A.conj().T @ A
    G = (G + G.conj().T) / 2
    assert G.shape == (196, 196)
    check(G, 64)


def test_rejects_bad_sizes(cuda):
    import torch
    for B, k in [(63, 8), (257, 8), (64, 0), (64, 65)]:
        H = torch.zeros((B, B), dtype=torch.complex128, device="cuda")
        ev = torch.zeros((max(k, 1),), dtype=torch.float64, device="cuda")
        V = torch.zeros((B, max(k, 1)), dtype=torch.complex128, device="cuda")
        with pytest.raises(RuntimeError):
            K.hermitian_topk(H, k, ev, V)
