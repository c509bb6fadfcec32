"""Generate the golden vectors under tests/golden/ from the reference build.

Run in a checkout where the reference sources are available and
`make -C oracle ref` has produced oracle/_ref (the unmodified K-Litho
functions compiled with the project's FFT shim and LAPACK forwarder):

    python tests/golden/make_golden.py

Each case stores inputs and the reference's outputs (NA <= 1, where the
reference itself is defined):
  tcc_<case>.npz   : source map, optics, Nx/Ny, TCC (complex128), top-k kernels
                     and eigenvalues (zheevr), Hopkins image (float32)
  socs_<case>.npz  : mask, kernels (float32 planes), eigenvalues, SOCS image
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "k-litho_b200")]

from oracle import oracle as O  # noqa: E402

TCC_CASES = {
    # name: (L, msize, source args, NA, defocus, nk)
    "annular_na08_df02": (256, 128, ("Annular", 41, dict(inner=0.6, outer=0.9)), 0.8, 0.2, 8),
    "dipole_na09": (256, 192, ("Dipole", 41, dict(radius=0.2, offset=0.6, onx=1)), 0.9, 0.0, 6),
    "quad_na075_df-03": (256, 200, ("CrossQuadrupole", 31, dict(radius=0.15, offset=0.7)), 0.75, -0.3, 6),
    "import101_na08": (256, 128, ("Import", 101, dict(path=os.path.join(HERE, "src_test1_size101.bin"))), 0.8, 0.2, 3),
}


def rect_mask(n, count, seed):
    rng = np.random.default_rng(seed)
    m = np.zeros((n, n), np.float32)
    for _ in range(count):
        w, h = rng.integers(8, 40, size=2)
        x, y = rng.integers(0, n - w), rng.integers(0, n - h)
        m[y:y + h, x:x + w] = 1.0
    return m


def main():
    assert O.ref_available(), "build the reference first: make -C oracle ref"
    for name, (L, ms, (kind, n, kw), NA, df, nk) in TCC_CASES.items():
        src = O.ref_create_source(n, kind, **kw)
        sig = O.ref_outer_sigma(src)
        Nx, Ny = O.band(NA, L, L, sig)
        tcc = O.ref_calc_tcc(src, sig, NA, df, L, L, Nx, Ny)
        krn, sc = O.ref_calc_kernels(tcc, Nx, Ny, nk)
        small = rect_mask(ms, 10, seed=len(name))
        mfile = os.path.join("/tmp", f"golden_mask_{name}.bin")
        small.tofile(mfile)
        mask = O.ref_create_mask(L, L, ms, ms, "Import", path=mfile)
        img = O.ref_hopkins_image(mask, tcc, Nx, Ny)
        np.savez_compressed(os.path.join(HERE, f"tcc_{name}.npz"), src=src, sigma=np.float32(sig),
                            L=L, NA=NA, defocus=df, Nx=Nx, Ny=Ny, tcc=tcc, krn=krn, scales=sc,
                            mask=mask, hopkins=img)
        # SOCS with these kernels, as klitho_socs reads them (float32 planes)
        kr = krn.real.astype(np.float32)
        ki = krn.imag.astype(np.float32)
        socs = O.ref_socs_image(mask, kr, ki, sc, Nx, Ny)
        np.savez_compressed(os.path.join(HERE, f"socs_{name}.npz"), mask=mask, krn_r=kr, krn_i=ki,
                            scales=sc, Nx=Nx, Ny=Ny, image=socs)
        print(name, "N", tcc.shape[0], "eig", sc)
    # the reference's shipped kernels on a synthetic mask
    kdir = os.path.join(HERE, "shipped_kernels")
    kx, ky = 33, 33
    sc = np.array([78.9658, 37.2823, 37.2823], np.float32)
    kr = np.stack([np.fromfile(os.path.join(kdir, f"krn_{i}_r.bin"), np.float32) for i in range(3)])
    ki = np.stack([np.fromfile(os.path.join(kdir, f"krn_{i}_i.bin"), np.float32) for i in range(3)])
    small = rect_mask(160, 14, seed=99)
    small.tofile("/tmp/golden_mask_shipped.bin")
    mask = O.ref_create_mask(256, 256, 160, 160, "Import", path="/tmp/golden_mask_shipped.bin")
    socs = O.ref_socs_image(mask, kr, ki, sc, 16, 16)
    np.savez_compressed(os.path.join(HERE, "socs_shipped_kernels.npz"), mask=mask, krn_r=kr,
                        krn_i=ki, scales=sc, Nx=16, Ny=16, image=socs)
    print("shipped kernels ok")


if __name__ == "__main__":
    main()
