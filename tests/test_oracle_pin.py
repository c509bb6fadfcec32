"""Pin the restated FP64 oracle to the reference's own code, bit for bit.

oracle/_ref holds the UNMODIFIED K-Litho functions compiled with the
project's FFT shim and zheevr forwarder; oracle/_build/libklitho_oracle.so is
the restatement the GPU tests compare against.  On NA <= 1 inputs (where the
reference is defined) every output must be identical: TCC, centred mask
spectrum, Hopkins image, LAPACK kernels and SOCS image.  Also pinned: the
n_medium extension reduces to the reference at n_medium = 1.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
SRC101 = os.path.join(HERE, "golden", "src_test1_size101.bin")

SOURCES = [
    ("Annular", 41, dict(inner=0.6, outer=0.9)),
    ("Annular", 31, dict(inner=0.3, outer=1.0)),
    ("Dipole", 41, dict(radius=0.2, offset=0.6, onx=1)),
    ("Dipole", 40, dict(radius=0.25, offset=0.5, onx=0)),
    ("CrossQuadrupole", 31, dict(radius=0.15, offset=0.7)),
    ("Point", 21, dict(ptx=0.3, pty=-0.2)),
    ("Import", 101, dict(path=SRC101)),
]


def mask_for(L, msize, seed):
    rng = np.random.default_rng(seed)
    m = np.zeros((msize, msize), np.float32)
    for _ in range(8):
        w, h = rng.integers(6, 30, size=2)
        x, y = rng.integers(0, msize - w), rng.integers(0, msize - h)
        m[y:y + h, x:x + w] = 1.0
    full = np.zeros((L, L), np.float32)
    o = (L - msize) // 2
    full[o:o + msize, o:o + msize] = m
    return full


@pytest.mark.parametrize("kind,n,kw", SOURCES)
def test_source_and_sigma_match_reference(ref_built, kind, n, kw):
    src = O.ref_create_source(n, kind, **kw)
    assert O.outer_sigma(src) == O.ref_outer_sigma(src)


@pytest.mark.parametrize("kind,n,kw", SOURCES)
@pytest.mark.parametrize("NA,defocus", [(0.8, 0.2), (0.6, 0.0), (0.95, -0.4)])
def test_tcc_bit_exact(ref_built, kind, n, kw, NA, defocus):
    src = O.ref_create_source(n, kind, **kw)
    sig = O.outer_sigma(src)
    L = 200
    Nx, Ny = O.band(NA, L, L, sig)
    before = O.out_of_band_count()
    a = O.ref_calc_tcc(src, sig, NA, defocus, L, L, Nx, Ny)
    b = O.calc_tcc(src, sig, NA, defocus, L, L, Nx, Ny, n_medium=1.0)
    assert np.array_equal(a, b)
    assert O.out_of_band_count() == before


@pytest.mark.parametrize("L", [128, 160, 127, 130])
def test_mask_spectrum_bit_exact(ref_built, L):
    m = mask_for(L, L - 20, seed=L)
    assert np.array_equal(O.ref_ft_r2c(m), O.ft_r2c(m))


@pytest.mark.parametrize("L,NA,defocus", [(192, 0.8, 0.2), (191, 0.7, -0.1), (256, 0.9, 0.0)])
def test_hopkins_kernels_socs_bit_exact(ref_built, L, NA, defocus):
    src = O.ref_create_source(41, "Annular", inner=0.6, outer=0.9)
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(NA, L, L, sig)
    tcc = O.calc_tcc(src, sig, NA, defocus, L, L, Nx, Ny)
    m = mask_for(L, L // 2, seed=3)
    img_ref = O.ref_hopkins_image(m, tcc, Nx, Ny)
    img_f32, _ = O.hopkins_image(m, tcc, Nx, Ny)
    assert np.array_equal(img_ref, img_f32)
    nk = 6
    k_ref, s_ref = O.ref_calc_kernels(tcc, Nx, Ny, nk)
    k, s, _ = O.calc_kernels(tcc, nk)
    assert np.array_equal(k_ref, k) and np.array_equal(s_ref, s)
    kr, ki = k.real.astype(np.float32), k.imag.astype(np.float32)
    socs_ref = O.ref_socs_image(m, kr, ki, s, Nx, Ny)
    socs = O.socs_image(m, kr.astype(np.float64) + 1j * ki.astype(np.float64), s, Nx, Ny)
    assert np.array_equal(socs_ref, socs.astype(np.float32))


def test_n_medium_extension_defined_beyond_na1():
    src = O.ref_create_source(41, "Annular", inner=0.6, outer=0.9) if O.ref_available() else None
    if src is None:
        pytest.skip("reference build not present")
    sig = O.outer_sigma(src)
    Nx, Ny = O.band(1.35, 256, 256, sig)
    t = O.calc_tcc(src, sig, 1.35, 0.3, 256, 256, Nx, Ny, n_medium=1.44)
    assert np.isfinite(t).all()
    assert np.allclose(t, t.conj().T)
    # clear field: TCC(0,0) = sum of source weights inside the pupil = 1
    c = (t.shape[0] - 1) // 2
    assert abs(t[c, c] - 1.0) < 1e-6


def test_known_answers():
    """Reference-independent self checks: Hermitian TCC, trace = sum of all
    eigenvalues, point source -> rank-one TCC, clear field image = TCC(0,0)."""
    from oracle.oracle import ref_available
    if not ref_available():
        pytest.skip("reference build not present")
    src = O.ref_create_source(31, "Annular", inner=0.5, outer=0.9)
    sig = O.outer_sigma(src)
    L = 160
    Nx, Ny = O.band(0.8, L, L, sig)
    t = O.calc_tcc(src, sig, 0.8, 0.25, L, L, Nx, Ny)
    N = t.shape[0]
    assert np.array_equal(t, t.conj().T)
    _, _, ev = O.calc_kernels(t, N)
    assert abs(ev.sum() - np.trace(t).real) < 1e-10 * abs(np.trace(t))
    pt = O.ref_create_source(21, "Point", ptx=0.4, pty=0.1)
    tp = O.calc_tcc(pt, O.outer_sigma(pt), 0.8, 0.1, L, L, *O.band(0.8, L, L, O.outer_sigma(pt)))
    assert np.linalg.matrix_rank(tp, tol=1e-9) == 1
    img, _ = O.hopkins_image(np.ones((L, L), np.float32), t, Nx, Ny)
    c = (N - 1) // 2
    assert np.abs(img - t[c, c].real).max() < 1e-6
