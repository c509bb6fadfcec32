"""CPU oracle for the K-Litho Hopkins/SOCS path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this module, and only to check (or to time as the CPU
baseline) the GPU product.  The product itself never imports it.

Two libraries are wrapped:

* ``_build/libklitho_oracle.so`` -- the restated FP64 oracle (klitho_oracle.c),
  step-for-step restatements of K-Litho-TCC/klitho_tcc.cpp:52-377 and
  K-Litho-SOCS/klitho_socs.cpp:158-241 with the ``n_medium`` generalisation of
  the defocus phase (klitho_tcc.cpp:220) so NA > 1 is defined.
* ``_ref/libkref_tcc.so`` / ``_ref/libkref_socs.so`` -- the reference's own,
  unmodified functions compiled with the project's FFT shim and zheevr
  forwarder (built by ``oracle/Makefile``; optional at run time).

The restated oracle is pinned bit-for-bit to the reference build on NA <= 1
inputs by tests/test_oracle_pin.py, and to committed golden vectors by
tests/test_golden.py.

It also holds the FP64 numpy reference of the SOCS adjoint (VJP), which has no
counterpart in the reference.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LAMBDA_NM = 193.0  # klitho_tcc.cpp:439

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_double_p = ctypes.POINTER(ctypes.c_double)

_LIB = None
_REF_TCC = None
_REF_SOCS = None


def _fp(a):
    return a.ctypes.data_as(_c_float_p)


def _dp(a):
    return a.ctypes.data_as(_c_double_p)


def _ip(a):
    return a.ctypes.data_as(_c_int_p)


def build_if_missing() -> None:
    """Compile the restated oracle (and the reference build when the
    reference checkout is present) with oracle/Makefile."""
    import subprocess

    path = os.path.join(HERE, "_build", "libklitho_oracle.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        build_if_missing()
        L = ctypes.CDLL(os.path.join(HERE, "_build", "libklitho_oracle.so"))
        L.kor_outer_sigma.restype = ctypes.c_float
        L.kor_outer_sigma.argtypes = [_c_float_p, ctypes.c_int]
        L.kor_band.restype = None
        L.kor_band.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                               ctypes.c_float, _c_int_p, _c_int_p]
        L.kor_calc_tcc.restype = ctypes.c_int
        L.kor_calc_tcc.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_double_p]
        L.kor_source_point_count.restype = ctypes.c_int
        L.kor_source_point_count.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_float]
        L.kor_pupil_matrix.restype = ctypes.c_int
        L.kor_pupil_matrix.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       _c_double_p, _c_int_p, _c_float_p, ctypes.c_int]
        L.kor_ft_r2c.restype = None
        L.kor_ft_r2c.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_int, _c_double_p]
        L.kor_ft_c2r_d.restype = None
        L.kor_ft_c2r_d.argtypes = [_c_double_p, ctypes.c_int, ctypes.c_int, _c_double_p]
        L.kor_calc_image.restype = None
        L.kor_calc_image.argtypes = [_c_double_p, ctypes.c_int, ctypes.c_int, _c_double_p,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_double_p]
        L.kor_calc_kernels.restype = ctypes.c_int
        L.kor_calc_kernels.argtypes = [_c_double_p, ctypes.c_int, ctypes.c_int, _c_double_p,
                                       _c_float_p, _c_double_p]
        L.kor_calc_socs.restype = None
        L.kor_calc_socs.argtypes = [_c_double_p, ctypes.c_int, ctypes.c_int, _c_double_p,
                                    _c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    _c_double_p]
        L.kor_socs_small_grid.restype = None
        L.kor_socs_small_grid.argtypes = L.kor_calc_socs.argtypes
        L.kor_out_of_band_count.restype = ctypes.c_long
        L.kor_out_of_band_count.argtypes = []
        _LIB = L
    return _LIB


# ---------------------------------------------------------------------------
# Restated oracle
# ---------------------------------------------------------------------------

def outer_sigma(src: np.ndarray) -> float:
    """getOuterSigma (klitho_tcc.cpp:52-67), before main's clamp to 1."""
    s = np.ascontiguousarray(src, dtype=np.float32)
    n = int(round(np.sqrt(s.size)))
    return float(lib().kor_outer_sigma(_fp(s), n))


def band(NA: float, Lx: int, Ly: int, sigma: float) -> tuple[int, int]:
    """Nx, Ny as klitho_tcc.cpp:479-486 computes them (sigma clamped to 1)."""
    nx, ny = ctypes.c_int(), ctypes.c_int()
    lib().kor_band(float(NA), int(Lx), int(Ly), float(sigma), float(LAMBDA_NM),
                   ctypes.byref(nx), ctypes.byref(ny))
    return nx.value, ny.value


def calc_tcc(src, sigma, NA, defocus, Lx, Ly, Nx, Ny, n_medium=1.0) -> np.ndarray:
    """calcTCC (klitho_tcc.cpp:186-267): N x N complex128 TCC."""
    s = np.ascontiguousarray(src, dtype=np.float32)
    n = int(round(np.sqrt(s.size)))
    N = (2 * Nx + 1) * (2 * Ny + 1)
    out = np.zeros((N, N), dtype=np.complex128)
    sig = min(float(sigma), 1.0)
    lib().kor_calc_tcc(_fp(s), n, sig, LAMBDA_NM, float(NA), float(defocus), float(n_medium),
                       int(Lx), int(Ly), int(Nx), int(Ny), _dp(out.view(np.float64)))
    return out


def source_point_count(src, sigma) -> int:
    s = np.ascontiguousarray(src, dtype=np.float32)
    n = int(round(np.sqrt(s.size)))
    return int(lib().kor_source_point_count(_fp(s), n, min(float(sigma), 1.0)))


def pupil_matrix(src, sigma, NA, defocus, Lx, Ly, Nx, Ny, n_medium=1.0):
    """Pupil values P[f, s] for active source points s (raster order of
    klitho_tcc.cpp:202-205); returns (P N x S complex128, src_ids, J)."""
    s = np.ascontiguousarray(src, dtype=np.float32)
    n = int(round(np.sqrt(s.size)))
    sig = min(float(sigma), 1.0)
    S = source_point_count(s, sig)
    N = (2 * Nx + 1) * (2 * Ny + 1)
    P = np.zeros((N, max(S, 1)), dtype=np.complex128)
    ids = np.zeros(max(S, 1), dtype=np.int32)
    J = np.zeros(max(S, 1), dtype=np.float32)
    lib().kor_pupil_matrix(_fp(s), n, sig, LAMBDA_NM, float(NA), float(defocus),
                           float(n_medium), int(Lx), int(Ly), int(Nx), int(Ny),
                           _dp(P.view(np.float64)), _ip(ids), _fp(J), S)
    return P[:, :S].copy(), ids[:S].copy(), J[:S].copy()


def ft_r2c(mask: np.ndarray) -> np.ndarray:
    """FT_r2c (klitho_tcc.cpp:97-148): centred, 1/(Lx*Ly)-scaled spectrum."""
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    out = np.zeros((Ly, Lx), dtype=np.complex128)
    lib().kor_ft_r2c(_fp(m), Lx, Ly, _dp(out.view(np.float64)))
    return out


def hopkins_image(mask, tcc, Nx, Ny) -> tuple[np.ndarray, np.ndarray]:
    """klitho_tcc's image.bin path: FT_r2c, calcImage, FT_c2r
    (klitho_tcc.cpp:510,534,537).  Returns (float32 as written, float64)."""
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    mf = ft_r2c(m)
    t = np.ascontiguousarray(tcc, dtype=np.complex128)
    N = t.shape[0]
    imgf = np.zeros((Ly, Lx), dtype=np.complex128)
    lib().kor_calc_image(_dp(mf.view(np.float64)), Lx, Ly, _dp(t.view(np.float64)), N,
                         int(Nx), int(Ny), _dp(imgf.view(np.float64)))
    img = np.zeros((Ly, Lx), dtype=np.float64)
    lib().kor_ft_c2r_d(_dp(imgf.view(np.float64)), Lx, Ly, _dp(img))
    return img.astype(np.float32), img


def calc_kernels(tcc: np.ndarray, nk: int):
    """calcKernels (klitho_tcc.cpp:300-377) through LAPACK zheevr.
    Returns (kernels nk x N complex128, scales float32, eigenvalues float64)."""
    t = np.ascontiguousarray(tcc, dtype=np.complex128)
    N = t.shape[0]
    nk = min(int(nk), N)
    k = np.zeros((nk, N), dtype=np.complex128)
    sc = np.zeros(nk, dtype=np.float32)
    ev = np.zeros(nk, dtype=np.float64)
    info = lib().kor_calc_kernels(_dp(t.view(np.float64)), N, nk, _dp(k.view(np.float64)),
                                  _fp(sc), _dp(ev))
    if info != 0:
        raise RuntimeError(f"zheevr info={info}")
    return k, sc, ev


def socs_image(mask, krns, scales, Nx, Ny) -> np.ndarray:
    """klitho_socs's image: FT_r2c then calcSOCS + FI (klitho_socs.cpp:338,343),
    in float64 (the reference stores the float32 cast of this array)."""
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    mf = ft_r2c(m)
    kk = np.ascontiguousarray(krns, dtype=np.complex128)
    sc = np.ascontiguousarray(scales, dtype=np.float32)
    out = np.zeros((Ly, Lx), dtype=np.float64)
    lib().kor_calc_socs(_dp(mf.view(np.float64)), Lx, Ly, _dp(kk.view(np.float64)), _fp(sc),
                        len(sc), int(Nx), int(Ny), _dp(out))
    return out


def socs_small_grid(mask, krns, scales, Nx, Ny) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    mf = ft_r2c(m)
    kk = np.ascontiguousarray(krns, dtype=np.complex128)
    sc = np.ascontiguousarray(scales, dtype=np.float32)
    out = np.zeros((4 * Ny + 1, 4 * Nx + 1), dtype=np.float64)
    lib().kor_socs_small_grid(_dp(mf.view(np.float64)), Lx, Ly, _dp(kk.view(np.float64)),
                              _fp(sc), len(sc), int(Nx), int(Ny), _dp(out))
    return out


def out_of_band_count() -> int:
    return int(lib().kor_out_of_band_count())


# ---------------------------------------------------------------------------
# The reference's own functions (oracle/_ref), when built
# ---------------------------------------------------------------------------

def ref_available() -> bool:
    return all(os.path.exists(os.path.join(HERE, "_ref", f))
               for f in ("libkref_tcc.so", "libkref_socs.so", "klitho_tcc", "klitho_socs"))


def ref_tcc():
    global _REF_TCC
    if _REF_TCC is None:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libkref_tcc.so"))
        L.kref_create_source.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_char_p, _c_float_p]
        L.kref_create_mask.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_char_p, ctypes.c_float, _c_float_p]
        L.kref_outer_sigma.restype = ctypes.c_float
        L.kref_outer_sigma.argtypes = [_c_float_p, ctypes.c_int]
        L.kref_calc_tcc.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, _c_double_p]
        L.kref_ft_r2c.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_int, _c_double_p]
        L.kref_hopkins_image.argtypes = [_c_float_p, _c_double_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _c_float_p]
        L.kref_calc_kernels.argtypes = [_c_double_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _c_double_p, _c_float_p]
        L.kref_write_kernel_info.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, _c_float_p]
        L.kref_read_kernel_info.argtypes = [ctypes.c_char_p, _c_int_p, _c_int_p, _c_int_p,
                                            _c_float_p, ctypes.c_int]
        L.kref_read_float_file.argtypes = [ctypes.c_char_p, ctypes.c_int, _c_float_p]
        L.kref_write_png.argtypes = [ctypes.c_char_p, _c_float_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_int]
        _REF_TCC = L
    return _REF_TCC


def ref_write_png(path, data, mn, mx, mode) -> None:
    """The reference's PNG writers (common/file_io.cpp:7-135; mode 0 grey,
    1 seven colours, 2 continuous) on a float32 array (rows x columns)."""
    d = np.ascontiguousarray(data, dtype=np.float32)
    ref_tcc().kref_write_png(str(path).encode(), _fp(d), d.shape[1], d.shape[0], float(mn), float(mx),
                             int(mode))


def ref_socs():
    global _REF_SOCS
    if _REF_SOCS is None:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libkref_socs.so"))
        L.kref_socs_image.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_int, _c_float_p,
                                      _c_float_p, _c_float_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _c_float_p]
        _REF_SOCS = L
    return _REF_SOCS


def ref_create_source(srcSize, kind, inner=0.6, outer=0.9, radius=0.1, offset=0.5, onx=1,
                      ptx=0.6, pty=0.2, path="") -> np.ndarray:
    out = np.zeros(srcSize * srcSize, dtype=np.float32)
    ref_tcc().kref_create_source(int(srcSize), kind.encode(), inner, outer, radius, offset,
                                 int(onx), ptx, pty, path.encode(), _fp(out))
    return out.reshape(srcSize, srcSize)


def ref_create_mask(Lx, Ly, msx, msy, kind, lw=128, sw=128, horiz=0, path="",
                    dose=1.0) -> np.ndarray:
    out = np.zeros(Lx * Ly, dtype=np.float32)
    ref_tcc().kref_create_mask(int(Lx), int(Ly), int(msx), int(msy), kind.encode(), int(lw),
                               int(sw), int(horiz), path.encode(), float(dose), _fp(out))
    return out.reshape(Ly, Lx)


def ref_outer_sigma(src) -> float:
    s = np.ascontiguousarray(src, dtype=np.float32)
    n = int(round(np.sqrt(s.size)))
    return float(ref_tcc().kref_outer_sigma(_fp(s), n))


def ref_calc_tcc(src, sigma, NA, defocus, Lx, Ly, Nx, Ny) -> np.ndarray:
    s = np.ascontiguousarray(src, dtype=np.float32)
    n = int(round(np.sqrt(s.size)))
    N = (2 * Nx + 1) * (2 * Ny + 1)
    out = np.zeros((N, N), dtype=np.complex128)
    ref_tcc().kref_calc_tcc(_fp(s), n, min(float(sigma), 1.0), LAMBDA_NM, float(NA),
                            float(defocus), int(Lx), int(Ly), int(Nx), int(Ny),
                            _dp(out.view(np.float64)))
    return out


def ref_ft_r2c(mask) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    out = np.zeros((Ly, Lx), dtype=np.complex128)
    ref_tcc().kref_ft_r2c(_fp(m), Lx, Ly, _dp(out.view(np.float64)))
    return out


def ref_hopkins_image(mask, tcc, Nx, Ny) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    t = np.ascontiguousarray(tcc, dtype=np.complex128)
    out = np.zeros((Ly, Lx), dtype=np.float32)
    ref_tcc().kref_hopkins_image(_fp(m), _dp(t.view(np.float64)), Lx, Ly, int(Nx), int(Ny),
                                 _fp(out))
    return out


def ref_calc_kernels(tcc, Nx, Ny, nk):
    t = np.ascontiguousarray(tcc, dtype=np.complex128)
    N = t.shape[0]
    k = np.zeros((nk, N), dtype=np.complex128)
    sc = np.zeros(nk, dtype=np.float32)
    info = ref_tcc().kref_calc_kernels(_dp(t.view(np.float64)), N, int(Nx), int(Ny), int(nk),
                                       _dp(k.view(np.float64)), _fp(sc))
    if info != 0:
        raise RuntimeError(f"zheevr info={info}")
    return k, sc


def ref_socs_image(mask, krn_r, krn_i, scales, Nx, Ny) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.float32)
    Ly, Lx = m.shape
    kr = np.ascontiguousarray(krn_r, dtype=np.float32)
    ki = np.ascontiguousarray(krn_i, dtype=np.float32)
    sc = np.ascontiguousarray(scales, dtype=np.float32)
    out = np.zeros((Ly, Lx), dtype=np.float32)
    ref_socs().kref_socs_image(_fp(m), Lx, Ly, _fp(kr), _fp(ki), _fp(sc), len(sc), int(Nx),
                               int(Ny), _fp(out))
    return out


# ---------------------------------------------------------------------------
# FP64 reference of the SOCS adjoint (no counterpart in the reference):
# the forward model restated with torch complex128 FFTs on the CPU, the loss
# L = sum (sigmoid(alpha (I - c)) - t)^2, gradients by autograd.
# ---------------------------------------------------------------------------

def _band_index(L, N):
    import torch
    return torch.arange(-N, N + 1) % L


def socs_fields_torch(mask, krn, Nx, Ny):
    """Coherent fields E_k on the full Lx x Ly grid (complex128), the
    band-limited evaluation the reference's calcSOCS + FI produces.  Runs on
    the device of `mask` when it is a torch tensor (CPU otherwise)."""
    import torch
    m = mask if isinstance(mask, torch.Tensor) else torch.as_tensor(mask, dtype=torch.float64)
    dev = m.device
    Ly, Lx = m.shape
    D = torch.fft.fft2(m.to(torch.float64))
    iy, ix = _band_index(Ly, Ny).to(dev), _band_index(Lx, Nx).to(dev)
    M = D[iy][:, ix] / (Lx * Ly)
    H = torch.as_tensor(np.asarray(krn, dtype=np.complex128), device=dev).reshape(-1, 2 * Ny + 1, 2 * Nx + 1)
    # odd periods: the reference's shifts place the image one pixel later
    dy, dx = 2 * ((Ly + 1) // 2) - Ly, 2 * ((Lx + 1) // 2) - Lx
    fy = torch.arange(-Ny, Ny + 1, dtype=torch.float64, device=dev)[:, None]
    fx = torch.arange(-Nx, Nx + 1, dtype=torch.float64, device=dev)[None, :]
    ph = torch.exp(-2j * np.pi * (fy * dy / Ly + fx * dx / Lx))
    C = H * (M * ph)[None]
    full = torch.zeros((H.shape[0], Ly, Lx), dtype=torch.complex128, device=dev)
    full[:, iy[:, None], ix[None, :]] = C
    return torch.fft.ifft2(full) * (Lx * Ly)


def socs_vjp_reference_chunked(mask, target, krn, scales, Nx, Ny, alpha=50.0, thr=0.225,
                               device="cpu", chunk=8):
    """(loss, dL/dmask, image, dL/dI) in FP64 like socs_vjp_reference, with the
    kernels taken `chunk` at a time (the image first, then one
    vector-Jacobian product per chunk), so large clips with many kernels fit
    in memory.  `device` may be a CUDA device: torch's FP64 FFTs then serve as
    the cross-check."""
    import torch
    krn = np.asarray(krn)
    lam = np.asarray(scales, dtype=np.float64)
    m = torch.as_tensor(np.asarray(mask, dtype=np.float64), device=device)
    t = torch.as_tensor(np.asarray(target, dtype=np.float64), device=device)
    nk = krn.shape[0]
    with torch.no_grad():
        I = torch.zeros_like(m)
        for k0 in range(0, nk, chunk):
            E = socs_fields_torch(m, krn[k0:k0 + chunk], Nx, Ny)
            lk = torch.as_tensor(lam[k0:k0 + chunk], device=device)
            I += (lk[:, None, None] * (E.real ** 2 + E.imag ** 2)).sum(0)
            del E
        s = torch.sigmoid(alpha * (I - thr))
        loss = float(((s - t) ** 2).sum())
        G = 2.0 * (s - t) * s * (1.0 - s) * alpha
    grad = torch.zeros_like(m)
    for k0 in range(0, nk, chunk):
        mm = m.clone().requires_grad_(True)
        E = socs_fields_torch(mm, krn[k0:k0 + chunk], Nx, Ny)
        lk = torch.as_tensor(lam[k0:k0 + chunk], device=device)
        Ic = (lk[:, None, None] * (E.real ** 2 + E.imag ** 2)).sum(0)
        (Ic * G).sum().backward()
        grad += mm.grad
        del E, Ic, mm
    return loss, grad.cpu().numpy(), I.cpu().numpy(), G.cpu().numpy()


def socs_loss_chunked(mask, target, krn, scales, Nx, Ny, alpha=50.0, thr=0.225, device="cpu", chunk=8):
    """FP64 loss of socs_vjp_reference_chunked (for finite differences)."""
    import torch
    krn = np.asarray(krn)
    lam = np.asarray(scales, dtype=np.float64)
    with torch.no_grad():
        m = torch.as_tensor(np.asarray(mask, dtype=np.float64), device=device)
        t = torch.as_tensor(np.asarray(target, dtype=np.float64), device=device)
        I = torch.zeros_like(m)
        for k0 in range(0, krn.shape[0], chunk):
            E = socs_fields_torch(m, krn[k0:k0 + chunk], Nx, Ny)
            lk = torch.as_tensor(lam[k0:k0 + chunk], device=device)
            I += (lk[:, None, None] * (E.real ** 2 + E.imag ** 2)).sum(0)
            del E
        s = torch.sigmoid(alpha * (I - thr))
        return float(((s - t) ** 2).sum())


def socs_image_torch(mask, krn, scales, Nx, Ny):
    import torch
    E = socs_fields_torch(mask, krn, Nx, Ny)
    lam = torch.as_tensor(np.asarray(scales, dtype=np.float64))
    return (lam[:, None, None] * (E.real ** 2 + E.imag ** 2)).sum(0)


def resist_loss_torch(I, target, alpha=50.0, thr=0.225):
    import torch
    t = torch.as_tensor(np.asarray(target, dtype=np.float64))
    s = torch.sigmoid(alpha * (I - thr))
    return ((s - t) ** 2).sum()


def socs_vjp_reference(mask, target, krn, scales, Nx, Ny, alpha=50.0, thr=0.225):
    """(loss, dL/dmask, image, dL/dI) in FP64."""
    import torch
    m = torch.as_tensor(np.asarray(mask, dtype=np.float64)).clone().requires_grad_(True)
    I = socs_image_torch(m, krn, scales, Nx, Ny)
    I.retain_grad()
    L = resist_loss_torch(I, target, alpha, thr)
    L.backward()
    return float(L.detach()), m.grad.numpy(), I.detach().numpy(), I.grad.numpy()


def socs_loss(mask, target, krn, scales, Nx, Ny, alpha=50.0, thr=0.225):
    import torch
    with torch.no_grad():
        I = socs_image_torch(torch.as_tensor(np.asarray(mask, dtype=np.float64)), krn, scales, Nx, Ny)
        return float(resist_loss_torch(I, target, alpha, thr))


def source_gradient_reference(mask, dLdI, P, J, Nx, Ny):
    """dL/dJ_s = sum_x dL/dI(x) |E_s(x)|^2 with E_s from conj(P[:, s]) (the
    Hopkins/Abbe fields of calcImage's convention)."""
    E = socs_fields_torch(mask, np.conj(P).T, Nx, Ny).numpy()
    return np.einsum("yx,syx->s", dLdI, E.real ** 2 + E.imag ** 2)


def hopkins_loss(mask, target, P, J, Nx, Ny, alpha=50.0, thr=0.225):
    """Loss of the full Hopkins image sum_s J_s |E_s|^2 (for finite differences
    of the source weights)."""
    import torch
    with torch.no_grad():
        E = socs_fields_torch(mask, np.conj(P).T, Nx, Ny)
        I = (torch.as_tensor(np.asarray(J, dtype=np.float64))[:, None, None] *
             (E.real ** 2 + E.imag ** 2)).sum(0)
        return float(resist_loss_torch(I, target, alpha, thr))
