"""Golden vectors: the restated oracle must reproduce the reference's outputs
stored in tests/golden (made by tests/golden/make_golden.py from the reference
build), and the reference's shipped sample files must parse.
"""
import glob
import os

import numpy as np
import pytest

import klitho as K
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TCC_FILES = sorted(glob.glob(os.path.join(GOLDEN, "tcc_*.npz")))
SOCS_FILES = sorted(glob.glob(os.path.join(GOLDEN, "socs_*.npz")))


def test_golden_files_present():
    assert len(TCC_FILES) >= 4 and len(SOCS_FILES) >= 5


@pytest.mark.parametrize("path", TCC_FILES, ids=os.path.basename)
def test_oracle_reproduces_reference_tcc_chain(path):
    g = np.load(path)
    src, L, NA, df = g["src"], int(g["L"]), float(g["NA"]), float(g["defocus"])
    sig = O.outer_sigma(src)
    assert np.float32(sig) == g["sigma"]
    Nx, Ny = O.band(NA, L, L, sig)
    assert (Nx, Ny) == (int(g["Nx"]), int(g["Ny"]))
    tcc = O.calc_tcc(src, sig, NA, df, L, L, Nx, Ny)
    assert np.array_equal(tcc, g["tcc"])
    img, _ = O.hopkins_image(g["mask"], tcc, Nx, Ny)
    assert np.array_equal(img, g["hopkins"])
    k, s, _ = O.calc_kernels(tcc, g["krn"].shape[0])
    assert np.array_equal(s, g["scales"])
    assert np.array_equal(k, g["krn"])


@pytest.mark.parametrize("path", SOCS_FILES, ids=os.path.basename)
def test_oracle_reproduces_reference_socs(path):
    g = np.load(path)
    k = g["krn_r"].astype(np.float64) + 1j * g["krn_i"].astype(np.float64)
    img = O.socs_image(g["mask"], k, g["scales"], int(g["Nx"]), int(g["Ny"]))
    assert np.array_equal(img.astype(np.float32), g["image"])


def test_shipped_kernel_files_parse():
    d = os.path.join(GOLDEN, "shipped_kernels")
    kx, ky, nk, sc = K.readKernelInfo(os.path.join(d, "kernel_info.txt"))
    assert (kx, ky, nk) == (33, 33, 3)
    assert np.allclose(sc, [78.9658, 37.2823, 37.2823])
    for i in range(nk):
        re, n = K.readFloatArray(os.path.join(d, f"krn_{i}_r.bin"), kx * ky)
        im, _ = K.readFloatArray(os.path.join(d, f"krn_{i}_i.bin"), kx * ky)
        assert n == kx * ky
        # eigenvectors are unit vectors
        assert abs(np.sum(re.astype(np.float64) ** 2 + im.astype(np.float64) ** 2) - 1.0) < 1e-5


def test_shipped_source_imports():
    src = K.createSource(101, "Import", sourceFile=os.path.join(GOLDEN, "src_test1_size101.bin"))
    assert np.count_nonzero(src) == 1576
    # normalised with a float running sum (source.cpp:89-103): ~1e-5 off
    assert abs(float(src.sum(dtype=np.float64)) - 1.0) < 1e-4
    # annulus of radius 20..30 pixels around the centre -> sigma_o = 30/50
    assert abs(K.getOuterSigma(src) - 0.6) < 1e-6
