"""Seeded synthetic workloads for the K-Litho imaging path.

The reference's sample masks (ICCAD-2013 T1..T10) are not distributed with
it, so benchmarks and tests use generated stand-ins with the shapes, sizes
and value distributions of the benchmark configurations:

* binary masks: unions of axis-aligned rectangles, widths/heights uniform in
  [40, 120] nm snapped to the 1 nm grid, positions uniform;
* continuous masks: Gaussian-filtered white noise through a sigmoid, in [0, 1];
* optics: lambda = 193 nm, NA = 1.35 with an immersion medium n = 1.44.
"""
from __future__ import annotations

import numpy as np

LAMBDA_NM = 193.0
NA_IMMERSION = 1.35
N_WATER = 1.44


def rect_mask(L: int, n_rects: int, seed: int, wmin: int = 40, wmax: int = 120,
              Ly: int | None = None) -> np.ndarray:
    """Union of `n_rects` random rectangles on an L x Ly float32 grid."""
    Ly = L if Ly is None else Ly
    rng = np.random.default_rng(seed)
    m = np.zeros((Ly, L), dtype=np.float32)
    w = rng.integers(wmin, wmax + 1, size=n_rects)
    h = rng.integers(wmin, wmax + 1, size=n_rects)
    x0 = rng.integers(0, np.maximum(L - w, 1))
    y0 = rng.integers(0, np.maximum(Ly - h, 1))
    for i in range(n_rects):
        m[y0[i]:y0[i] + h[i], x0[i]:x0[i] + w[i]] = 1.0
    return m


def rect_mask_density(L: int, seed: int, density: float) -> np.ndarray:
    """Random-rectangle mask whose fill fraction is close to `density`: rectangles
    are added until the target is reached."""
    rng = np.random.default_rng(seed)
    m = np.zeros((L, L), dtype=np.float32)
    area = float(L * L)
    filled = 0.0
    while filled / area < density:
        w, h = rng.integers(40, 121, size=2)
        x0 = rng.integers(0, max(L - w, 1))
        y0 = rng.integers(0, max(L - h, 1))
        m[y0:y0 + h, x0:x0 + w] = 1.0
        filled = float(m.sum())
    return m


def rect_mask_fill(L: int, seed: int, density: float) -> np.ndarray:
    """Random-rectangle mask with about `density` fill: the rectangle count
    follows the Poisson coverage law 1 - exp(-R a / L^2) for mean area a."""
    mean_area = 80.0 * 80.0
    R = max(1, int(round(-np.log(1.0 - density) * L * L / mean_area)))
    return rect_mask(L, R, seed)


def smooth_mask(L: int, seed: int, sigma_px: float = 12.0, gain: float = 6.0,
                Ly: int | None = None) -> np.ndarray:
    """Continuous mask in [0, 1]: periodic Gaussian-filtered noise through a
    sigmoid, L x Ly (square by default)."""
    Ly = L if Ly is None else Ly
    rng = np.random.default_rng(seed)
    n = rng.standard_normal((Ly, L))
    fx, fy = np.fft.fftfreq(L), np.fft.fftfreq(Ly)
    g = np.exp(-2.0 * (np.pi * sigma_px) ** 2 * (fy[:, None] ** 2 + fx[None, :] ** 2))
    s = np.real(np.fft.ifft2(np.fft.fft2(n) * g))
    s /= s.std() + 1e-30
    return (1.0 / (1.0 + np.exp(-gain * s))).astype(np.float32)


def random_kernels(nk: int, Nx: int, Ny: int, seed: int):
    """Random complex kernels in the kernel-file layout with decaying weights
    (stand-ins where only the data flow matters)."""
    rng = np.random.default_rng(seed)
    nb = (2 * Nx + 1) * (2 * Ny + 1)
    k = (rng.standard_normal((nk, nb)) + 1j * rng.standard_normal((nk, nb))) / np.sqrt(2 * nb)
    sc = (np.geomspace(1.0, 1e-3, nk) * 50.0).astype(np.float32)
    return k.astype(np.complex64), sc


def defocus_arg(defocus_nm: float, NA: float = NA_IMMERSION) -> float:
    """klitho_tcc's normalised defocus argument for a defocus in nm
    (dz = defocus * lambda / NA^2, klitho_tcc.cpp:191)."""
    return defocus_nm * NA * NA / LAMBDA_NM
