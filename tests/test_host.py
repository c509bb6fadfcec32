"""Host-side inputs of the product (k-litho_b200/csrc/kl_host.cpp) against the
reference's own createSource / createMask / getOuterSigma / file I/O
(oracle/_ref), bit for bit; plus the on-disk formats."""
import os

import numpy as np
import pytest

import klitho as K
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("kind,n,kw", [
    ("Annular", 41, dict(innerRadius=0.6, outerRadius=0.9)),
    ("Annular", 61, dict(innerRadius=0.0, outerRadius=1.0)),
    ("Annular", 40, dict(innerRadius=0.55, outerRadius=0.95)),
    ("Dipole", 61, dict(radius=0.15, offset=0.7, onXAxis=1)),
    ("Dipole", 60, dict(radius=0.2, offset=0.5, onXAxis=0)),
    ("CrossQuadrupole", 81, dict(radius=0.12, offset=0.75)),
    ("CrossQuadrupole", 30, dict(radius=0.3, offset=0.6)),
    ("Point", 21, dict(ptX=0.6, ptY=0.2)),
    ("Point", 20, dict(ptX=-0.35, ptY=-0.5)),
    ("Point", 41, dict(ptX=0.0, ptY=0.0)),
    ("Bogus", 11, dict()),
])
def test_create_source_bit_exact(ref_built, kind, n, kw):
    ours = K.createSource(n, kind, **kw)
    ref = O.ref_create_source(n, kind, inner=kw.get("innerRadius", 0.6),
                              outer=kw.get("outerRadius", 0.9), radius=kw.get("radius", 0.1),
                              offset=kw.get("offset", 0.5), onx=kw.get("onXAxis", 1),
                              ptx=kw.get("ptX", 0.6), pty=kw.get("ptY", 0.2))
    assert np.array_equal(ours, ref)
    assert K.getOuterSigma(ours) == O.ref_outer_sigma(ref)


def test_import_source_bit_exact(ref_built):
    p = os.path.join(GOLDEN, "src_test1_size101.bin")
    assert np.array_equal(K.createSource(101, "Import", sourceFile=p),
                          O.ref_create_source(101, "Import", path=p))


@pytest.mark.parametrize("Lx,Ly,msx,msy,lw,sw,hz", [(256, 256, 128, 128, 20, 30, 0),
                                                    (300, 256, 101, 77, 7, 9, 1),
                                                    (64, 64, 64, 64, 1, 1, 0)])
def test_linespace_mask_bit_exact(ref_built, Lx, Ly, msx, msy, lw, sw, hz):
    ours = K.createMask(Lx, Ly, msx, msy, "LineSpace", lw, sw, hz)
    ref = O.ref_create_mask(Lx, Ly, msx, msy, "LineSpace", lw, sw, hz)
    assert np.array_equal(ours, ref)


@pytest.mark.parametrize("ext,count", [("bin", 100 * 80), ("bin", 5000), ("bin", 9000),
                                       ("txt", 100 * 80), ("txt", 4000)])
def test_import_mask_bit_exact(ref_built, tmp_path, ext, count):
    rng = np.random.default_rng(count)
    vals = rng.random(count).astype(np.float32)
    path = str(tmp_path / f"m.{ext}")
    if ext == "bin":
        vals.tofile(path)
    else:
        np.savetxt(path, vals.reshape(-1, 10) if count % 10 == 0 else vals, fmt="%.9g")
    ours = K.createMask(256, 200, 100, 80, "Import", maskFile=path, dose=1.0)
    ref = O.ref_create_mask(256, 200, 100, 80, "Import", path=path)
    assert np.array_equal(ours, ref)


def test_band_size_matches_oracle():
    for NA in (0.5, 0.8, 1.0, 1.35):
        for L in (256, 1000, 1024, 2048, 4096):
            for s in (0.3, 0.8333333, 0.9, 1.0, 1.2):
                assert K.bandSize(NA, L, L, s) == O.band(NA, L, L, s)


def test_kernel_info_text_identical(ref_built, tmp_path):
    sc = np.array([69.024139, 27.891796, 27.891796, 6.8732, 1e-7, 123456789.0], np.float32)
    a, b = str(tmp_path / "ours.txt"), str(tmp_path / "ref.txt")
    K.writeKernelInfo(a, 27, 29, sc)
    O.ref_tcc().kref_write_kernel_info(b.encode(), 27, 29, len(sc),
                                       sc.ctypes.data_as(O._c_float_p))
    assert open(a).read() == open(b).read()
    kx, ky, nk, got = K.readKernelInfo(a)
    assert (kx, ky, nk) == (27, 29, 6)
    assert np.allclose(got, sc, rtol=1e-5)


def test_float_file_roundtrip_and_short_file(tmp_path):
    p = str(tmp_path / "x.bin")
    v = np.arange(10, dtype=np.float32)
    K.writeFloatArray(p, v)
    got, n = K.readFloatArray(p, 10)
    assert n == 10 and np.array_equal(got, v)
    got, n = K.readFloatArray(p, 16)  # short file: zero padded, warning on stderr
    assert n == 10 and np.array_equal(got[:10], v) and np.all(got[10:] == 0)


def test_missing_file_is_io_error(tmp_path):
    with pytest.raises(K.KLError) as e:
        K.readFloatArray(str(tmp_path / "nope.bin"), 4)
    assert e.value.code == K.KL_ERR_IO
