"""ctypes binding of libklitho_gpu (include/klitho_gpu.h).

The Python-side mirror of the K-Litho imaging interface: the same function
names and argument meanings as the reference's C++ functions (createSource,
createMask, getOuterSigma, calcSOCS, ...), backed by the B200 library.  It
loads ``lib/libklitho_gpu.so`` from this directory and raises if it is
missing -- there is no CPU fallback.  Device buffers are torch CUDA tensors
(PyTorch provides allocation and streams only); every computation runs in
the library's own CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libklitho_gpu.so")

KL_OK = 0
KL_ERR_INVALID = 1
KL_ERR_CUDA = 2
KL_ERR_NOMEM = 3
KL_ERR_UNSUPPORTED = 4
KL_ERR_NOT_CONVERGED = 5
KL_ERR_IO = 6
KL_SOCS_ADJOINT = 1
KL_SOCS_GENERAL = 2
KL_SYNTH_AUTO = 0
KL_SYNTH_CUDA_CORES = 1
KL_SYNTH_TENSOR_CORES = 2

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_float_p = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p

_LIB = None


class KLError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load the library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; run `make -C k-litho_b200` "
                              "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        L.kl_version.restype = ctypes.c_int
        L.kl_last_error.restype = ctypes.c_char_p
        L.kl_create_source.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_char_p, _c_float_p]
        L.kl_create_mask.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_char_p, ctypes.c_float, _c_float_p]
        L.kl_outer_sigma.restype = ctypes.c_float
        L.kl_outer_sigma.argtypes = [_c_float_p, ctypes.c_int]
        L.kl_band_size.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                   _c_int_p, _c_int_p]
        L.kl_source_point_count.argtypes = [_c_float_p, ctypes.c_int, ctypes.c_float]
        L.kl_read_float_file.argtypes = [ctypes.c_char_p, ctypes.c_int, _c_float_p, _c_int_p]
        L.kl_write_float_file.argtypes = [ctypes.c_char_p, _c_float_p, ctypes.c_int]
        L.kl_write_kernel_info.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _c_float_p]
        L.kl_read_kernel_info.argtypes = [ctypes.c_char_p, _c_int_p, _c_int_p, _c_int_p,
                                          _c_float_p, ctypes.c_int]
        L.kl_socs_plan_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int]
        L.kl_socs_plan_create_ex.argtypes = L.kl_socs_plan_create.argtypes + [ctypes.c_int]
        L.kl_socs_plan_engine.argtypes = [_vp]
        L.kl_socs_set_synthesis.argtypes = [_vp, ctypes.c_int]
        L.kl_socs_synthesis.argtypes = [_vp, ctypes.c_int]
        L.kl_socs_plan_status.argtypes = [_vp]
        L.kl_socs_plan_destroy.argtypes = [_vp]
        L.kl_resist_contour.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                        ctypes.c_float, _vp, _vp, _vp, _vp, _vp]
        L.kl_socs_set_kernels.argtypes = [_vp, ctypes.c_int, _c_float_p, _c_float_p, _c_float_p]
        L.kl_socs_forward.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp]
        L.kl_socs_forward_host.argtypes = [_vp, _c_float_p, ctypes.c_int, _c_float_p, _vp]
        L.kl_mask_spectrum.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp]
        L.kl_tcc_plan_create.argtypes = [ctypes.POINTER(_vp), _c_float_p, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.kl_tcc_plan_destroy.argtypes = [_vp]
        L.kl_tcc_plan_info.argtypes = [_vp, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_float_p]
        L.kl_tcc_factor.argtypes = [_vp, _vp, _vp]
        L.kl_hermitian_topk.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]
        L.kl_factor_gram.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp]
        L.kl_tcc_build.argtypes = [_vp, _vp, _vp]
        L.kl_tcc_minmax.argtypes = [_vp, _vp, ctypes.POINTER(ctypes.c_double), _vp]
        L.kl_topk_eig.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _c_float_p, _c_float_p,
                                  _c_float_p, ctypes.POINTER(ctypes.c_double), _c_int_p]
        L.kl_topk_eig_batch.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _c_float_p, _c_float_p, _c_float_p,
                                        ctypes.POINTER(ctypes.c_double), _c_int_p]
        L.kl_topk_eig_c64.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _c_float_p, _c_float_p,
                                      ctypes.POINTER(ctypes.c_double), _c_int_p]
        L.kl_topk_eig_batch_c64.argtypes = [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            _c_float_p, _c_float_p, ctypes.POINTER(ctypes.c_double), _c_int_p]
        L.kl_hopkins_image.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp]
        L.kl_fp64_hopkins_image.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp]
        L.kl_fp64_socs_forward.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp]
        L.kl_fp64_mask_spectrum.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp]
        L.kl_fp64_socs_vjp.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double, _vp, _vp, _vp, _vp]
        L.kl_socs_plan_create_adjoint.argtypes = L.kl_socs_plan_create.argtypes
        L.kl_socs_vjp.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                  _vp, _vp, _vp, _vp]
        L.kl_socs_vjp_source.argtypes = [_vp, _vp, _vp, _vp]
        L.kl_write_png.argtypes = [ctypes.c_char_p, _c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_int]
        L.kl_socs_autotune.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp, _c_int_p, _c_int_p]
        L.kl_socs_batch_create.argtypes = [ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.c_int]
        L.kl_socs_batch_destroy.argtypes = [_vp]
        L.kl_socs_batch_forward.argtypes = [_vp, ctypes.POINTER(_vp), _c_int_p, ctypes.POINTER(_vp), _vp]
        L.kl_socs_batch_enable_timing.argtypes = [_vp, ctypes.c_int]
        L.kl_socs_batch_stage_times.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.kl_socs_batch_graph_builds.argtypes = [_vp]
        L.kl_socs_enable_timing.argtypes = [_vp, ctypes.c_int]
        L.kl_socs_stage_times.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), _c_int_p]
        _LIB = L
    return _LIB


def last_error() -> str:
    return lib().kl_last_error().decode(errors="replace")


def check(rc: int, where: str) -> None:
    if rc != KL_OK:
        raise KLError(rc, where, last_error())


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_c_float_p)


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


def _dev_ptr(t) -> int:
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError("expected a contiguous CUDA tensor")
    return int(t.data_ptr())


# ---------------------------------------------------------------------------
# host-side inputs (mirrors of source.cpp / mask.cpp / file_io.cpp)
# ---------------------------------------------------------------------------

def createSource(srcSize: int, srcType: str, innerRadius=0.6, outerRadius=0.9, radius=0.1,
                 offset=0.5, onXAxis=1, ptX=0.6, ptY=0.2, sourceFile="") -> np.ndarray:
    out = np.zeros(srcSize * srcSize, dtype=np.float32)
    check(lib().kl_create_source(int(srcSize), srcType.encode(), innerRadius, outerRadius,
                                 radius, offset, int(onXAxis), ptX, ptY, sourceFile.encode(),
                                 _fp(out)), "kl_create_source")
    return out.reshape(srcSize, srcSize)


def createMask(Lx, Ly, maskSizeX, maskSizeY, maskType="LineSpace", lineWidth=128,
               spaceWidth=128, isHorizontal=0, maskFile="", dose=1.0) -> np.ndarray:
    out = np.zeros(Lx * Ly, dtype=np.float32)
    check(lib().kl_create_mask(int(Lx), int(Ly), int(maskSizeX), int(maskSizeY),
                               maskType.encode(), int(lineWidth), int(spaceWidth),
                               int(isHorizontal), maskFile.encode(), float(dose), _fp(out)),
          "kl_create_mask")
    return out.reshape(Ly, Lx)


def getOuterSigma(src: np.ndarray) -> float:
    s = np.ascontiguousarray(src, dtype=np.float32)
    return float(lib().kl_outer_sigma(_fp(s), int(s.shape[0])))


def bandSize(NA: float, Lx: int, Ly: int, outerSigma: float) -> tuple[int, int]:
    nx, ny = ctypes.c_int(), ctypes.c_int()
    check(lib().kl_band_size(float(NA), int(Lx), int(Ly), float(outerSigma), ctypes.byref(nx),
                             ctypes.byref(ny)), "kl_band_size")
    return nx.value, ny.value


def sourcePointCount(src: np.ndarray, outerSigma: float) -> int:
    s = np.ascontiguousarray(src, dtype=np.float32)
    return int(lib().kl_source_point_count(_fp(s), int(s.shape[0]), float(outerSigma)))


def readFloatArray(path: str, size: int) -> tuple[np.ndarray, int]:
    out = np.zeros(size, dtype=np.float32)
    cnt = ctypes.c_int()
    check(lib().kl_read_float_file(path.encode(), int(size), _fp(out), ctypes.byref(cnt)),
          "kl_read_float_file")
    return out, cnt.value


def writeFloatArray(path: str, data: np.ndarray) -> None:
    d = np.ascontiguousarray(data, dtype=np.float32).ravel()
    check(lib().kl_write_float_file(path.encode(), _fp(d), int(d.size)), "kl_write_float_file")


def writeKernelInfo(path: str, kx: int, ky: int, scales) -> None:
    s = np.ascontiguousarray(scales, dtype=np.float32)
    check(lib().kl_write_kernel_info(path.encode(), int(kx), int(ky), int(s.size), _fp(s)),
          "kl_write_kernel_info")


def readKernelInfo(path: str, cap: int = 4096):
    kx, ky, nk = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    sc = np.zeros(cap, dtype=np.float32)
    check(lib().kl_read_kernel_info(path.encode(), ctypes.byref(kx), ctypes.byref(ky),
                                    ctypes.byref(nk), _fp(sc), cap), "kl_read_kernel_info")
    return kx.value, ky.value, nk.value, sc[: max(nk.value, 0)].copy()


# ---------------------------------------------------------------------------
# SOCS imaging plan
# ---------------------------------------------------------------------------

class SocsPlan:
    """GPU SOCS imaging for clips of one period (calcSOCS + FI on device)."""

    def __init__(self, Lx: int, Ly: int, Nx: int, Ny: int, nk: int, nsets: int = 1,
                 max_clips: int = 1, adjoint: bool = False, general: bool = False):
        """`general` puts the plan on the general-geometry pipeline even where
        the specialised kernels cover the period (kl_socs_plan_create_ex)."""
        self.Lx, self.Ly, self.Nx, self.Ny = int(Lx), int(Ly), int(Nx), int(Ny)
        self.nk, self.nsets, self.max_clips = int(nk), int(nsets), int(max_clips)
        h = _vp()
        flags = (KL_SOCS_ADJOINT if adjoint else 0) | (KL_SOCS_GENERAL if general else 0)
        check(lib().kl_socs_plan_create_ex(ctypes.byref(h), self.Lx, self.Ly, self.Nx, self.Ny,
                                           self.nk, self.nsets, self.max_clips, flags),
              "kl_socs_plan_create")
        self._h = h

    @property
    def engine(self) -> str:
        """'specialised' or 'general' (kl_socs_plan_engine)."""
        return "general" if lib().kl_socs_plan_engine(self._h) == 1 else "specialised"

    def set_synthesis(self, mode: str) -> None:
        """'auto', 'cuda' or 'tensor' engine of the image synthesis
        (kl_socs_set_synthesis)."""
        m = {"auto": KL_SYNTH_AUTO, "cuda": KL_SYNTH_CUDA_CORES, "tensor": KL_SYNTH_TENSOR_CORES}[mode]
        check(lib().kl_socs_set_synthesis(self._h, m), "kl_socs_set_synthesis")

    def synthesis(self, nclips: int) -> str:
        """'cuda' or 'tensor': the engine a forward of nclips clips uses."""
        return "tensor" if lib().kl_socs_synthesis(self._h, int(nclips)) == KL_SYNTH_TENSOR_CORES else "cuda"

    def status(self) -> None:
        """Raise if a tensor-core pipeline wait timed out (kl_socs_plan_status)."""
        check(lib().kl_socs_plan_status(self._h), "kl_socs_plan_status")

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().kl_socs_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_kernels(self, set_index: int, krn: np.ndarray, scales: np.ndarray) -> None:
        """krn: nk x (2Ny+1)(2Nx+1) complex (kernel-file layout)."""
        k = np.asarray(krn)
        re = np.ascontiguousarray(k.real, dtype=np.float32)
        im = np.ascontiguousarray(k.imag, dtype=np.float32)
        sc = np.ascontiguousarray(scales, dtype=np.float32)
        check(lib().kl_socs_set_kernels(self._h, int(set_index), _fp(re), _fp(im), _fp(sc)),
              "kl_socs_set_kernels")

    def forward(self, masks_dev, images_dev, nclips: int | None = None, stream=None) -> None:
        n = masks_dev.shape[0] if nclips is None else nclips
        check(lib().kl_socs_forward(self._h, _dev_ptr(masks_dev), int(n), _dev_ptr(images_dev),
                                    _stream_ptr(stream)), "kl_socs_forward")

    def forward_host(self, masks: np.ndarray, images: np.ndarray | None = None,
                     stream=None) -> np.ndarray:
        m = np.ascontiguousarray(masks, dtype=np.float32)
        n = m.shape[0]
        if images is None:
            images = np.empty((n, self.nsets, self.Ly, self.Lx), dtype=np.float32)
        check(lib().kl_socs_forward_host(self._h, _fp(m), int(n), _fp(images),
                                         _stream_ptr(stream)), "kl_socs_forward_host")
        return images

    def vjp(self, masks_dev, targets_dev, grad_dev, loss_dev, images_dev=None, alpha=50.0,
            threshold=0.225, nclips: int | None = None, stream=None) -> None:
        """Adjoint of imaging + sigmoid resist + L2 loss (kl_socs_vjp)."""
        n = masks_dev.shape[0] if nclips is None else nclips
        check(lib().kl_socs_vjp(self._h, _dev_ptr(masks_dev), _dev_ptr(targets_dev), int(n),
                                float(alpha), float(threshold),
                                _dev_ptr(images_dev) if images_dev is not None else None,
                                _dev_ptr(grad_dev), _dev_ptr(loss_dev), _stream_ptr(stream)),
              "kl_socs_vjp")

    def vjp_source(self, tcc_plan, grad_src_dev, stream=None) -> None:
        check(lib().kl_socs_vjp_source(self._h, tcc_plan._h, _dev_ptr(grad_src_dev),
                                       _stream_ptr(stream)), "kl_socs_vjp_source")

    def autotune(self, masks_dev, images_dev, nclips: int | None = None, stream=None):
        """Pick the fastest launch shape for batches of nclips clips
        (kl_socs_autotune); returns (kernel slices, strips per CTA)."""
        n = masks_dev.shape[0] if nclips is None else nclips
        ns, spc = ctypes.c_int(), ctypes.c_int()
        check(lib().kl_socs_autotune(self._h, _dev_ptr(masks_dev), int(n), _dev_ptr(images_dev),
                                     _stream_ptr(stream), ctypes.byref(ns), ctypes.byref(spc)),
              "kl_socs_autotune")
        return ns.value, spc.value

    def enable_timing(self, on: bool = True) -> None:
        check(lib().kl_socs_enable_timing(self._h, int(bool(on))), "kl_socs_enable_timing")

    def stage_times(self):
        """(ms[3], launches[3]) for the forward, spectral and inverse kernels."""
        ms = (ctypes.c_double * 3)()
        n = (ctypes.c_int * 3)()
        check(lib().kl_socs_stage_times(self._h, ms, n), "kl_socs_stage_times")
        return list(ms), list(n)

    def mask_spectrum(self, masks_dev, band_dev, nclips: int | None = None, stream=None) -> None:
        n = masks_dev.shape[0] if nclips is None else nclips
        check(lib().kl_mask_spectrum(self._h, _dev_ptr(masks_dev), int(n), _dev_ptr(band_dev),
                                     _stream_ptr(stream)), "kl_mask_spectrum")


class SocsBatch:
    """Several SOCS plans imaged as concurrent branches of one CUDA graph
    (kl_socs_batch_*); the plans must stay open while the batch is used."""

    def __init__(self, plans):
        self.plans = list(plans)
        h = _vp()
        arr = (_vp * len(self.plans))(*[p._h for p in self.plans])
        check(lib().kl_socs_batch_create(ctypes.byref(h), arr, len(self.plans)), "kl_socs_batch_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().kl_socs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, masks_list, images_list, nclips=None, stream=None) -> None:
        n = len(self.plans)
        counts = [m.shape[0] for m in masks_list] if nclips is None else list(nclips)
        m = (_vp * n)(*[_dev_ptr(t) for t in masks_list])
        o = (_vp * n)(*[_dev_ptr(t) for t in images_list])
        c = (ctypes.c_int * n)(*counts)
        check(lib().kl_socs_batch_forward(self._h, m, c, o, _stream_ptr(stream)), "kl_socs_batch_forward")

    def enable_timing(self, on: bool = True) -> None:
        check(lib().kl_socs_batch_enable_timing(self._h, int(bool(on))), "kl_socs_batch_enable_timing")

    def stage_times(self, i: int):
        ms = (ctypes.c_double * 3)()
        check(lib().kl_socs_batch_stage_times(self._h, int(i), ms), "kl_socs_batch_stage_times")
        return list(ms)

    def graph_builds(self) -> int:
        return int(lib().kl_socs_batch_graph_builds(self._h))


# ---------------------------------------------------------------------------
# TCC, SOCS kernels and the Hopkins image (klitho_tcc's numerics)
# ---------------------------------------------------------------------------

PREC_FAST = 0
PREC_FP64 = 1


class TccPlan:
    """GPU TCC of one optical setting (calcTCC / calcKernels / calcImage)."""

    def __init__(self, src: np.ndarray, NA: float, defocus: float, Lx: int, Ly: int,
                 n_medium: float = 1.0, precision: int = PREC_FAST):
        s = np.ascontiguousarray(src, dtype=np.float32)
        h = _vp()
        check(lib().kl_tcc_plan_create(ctypes.byref(h), _fp(s), int(s.shape[0]), float(NA),
                                       float(defocus), float(n_medium), int(Lx), int(Ly),
                                       int(precision)), "kl_tcc_plan_create")
        self._h = h
        self.precision = precision
        self.Lx, self.Ly = int(Lx), int(Ly)
        nx, ny, n, S = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        sig = ctypes.c_float()
        check(lib().kl_tcc_plan_info(h, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(n),
                                     ctypes.byref(S), ctypes.byref(sig)), "kl_tcc_plan_info")
        self.Nx, self.Ny, self.N, self.S = nx.value, ny.value, n.value, S.value
        self.outer_sigma = sig.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().kl_tcc_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factor(self, stream=None):
        import torch
        A = torch.empty((self.N, self.S, 2), dtype=torch.float32, device="cuda")
        check(lib().kl_tcc_factor(self._h, _dev_ptr(A), _stream_ptr(stream)), "kl_tcc_factor")
        return A

    def build(self, stream=None):
        """The N x N TCC as a torch tensor (..., 2) of float32 (fast) or float64 (FP64)."""
        import torch
        dt = torch.float32 if self.precision == PREC_FAST else torch.float64
        T = torch.empty((self.N, self.N, 2), dtype=dt, device="cuda")
        check(lib().kl_tcc_build(self._h, _dev_ptr(T), _stream_ptr(stream)), "kl_tcc_build")
        return T

    def minmax(self, T, stream=None):
        out = (ctypes.c_double * 4)()
        check(lib().kl_tcc_minmax(self._h, _dev_ptr(T), out, _stream_ptr(stream)), "kl_tcc_minmax")
        return list(out)

    def topk(self, nk: int, block: int = 0):
        """(kernels nk x N complex64 in the reference layout, scales float32,
        eigenvalues float64, iterations)."""
        krn = np.empty((nk, self.N), dtype=np.complex64)  # every entry is written
        sc = np.zeros(nk, dtype=np.float32)
        ev = np.zeros(nk, dtype=np.float64)
        it = ctypes.c_int()
        check(lib().kl_topk_eig_c64(self._h, int(nk), int(block), krn.ctypes.data_as(_c_float_p), _fp(sc),
                                    ev.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    ctypes.byref(it)), "kl_topk_eig_c64")
        return krn, sc, ev, it.value

    @staticmethod
    def topk_batch(plans, nk: int, block: int = 0):
        """kl_topk_eig over several plans sharing N (e.g. a focus sweep) in one
        call: lists of (kernels, scales, eigenvalues, iterations) per plan."""
        n, N = len(plans), plans[0].N
        k = np.empty((n, nk, N), dtype=np.complex64)  # every entry is written
        sc = np.zeros(n * nk, dtype=np.float32)
        ev = np.zeros(n * nk, dtype=np.float64)
        it = np.zeros(n, dtype=np.int32)
        hs = (_vp * n)(*[p._h for p in plans])
        check(lib().kl_topk_eig_batch_c64(hs, n, int(nk), int(block), k.ctypes.data_as(_c_float_p), _fp(sc),
                                          ev.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          it.ctypes.data_as(_c_int_p)), "kl_topk_eig_batch_c64")
        return ([k[i] for i in range(n)], list(sc.reshape(n, nk)), list(ev.reshape(n, nk)),
                [int(x) for x in it])

    def hopkins_fp64(self, masks_dev, images_dev, nclips: int | None = None, stream=None) -> None:
        """Plain FP64 Hopkins image (plans of PREC_FP64); images_dev float64."""
        n = masks_dev.shape[0] if nclips is None else nclips
        check(lib().kl_fp64_hopkins_image(self._h, _dev_ptr(masks_dev), int(n), _dev_ptr(images_dev),
                                          _stream_ptr(stream)), "kl_fp64_hopkins_image")

    def hopkins(self, masks_dev, images_dev, nclips: int | None = None, stream=None) -> None:
        n = masks_dev.shape[0] if nclips is None else nclips
        check(lib().kl_hopkins_image(self._h, _dev_ptr(masks_dev), int(n), _dev_ptr(images_dev),
                                     _stream_ptr(stream)), "kl_hopkins_image")


def resist_contour(images_dev, alpha: float = 50.0, threshold: float = 0.225, resist_dev=None,
                   printed_dev=None, edges_dev=None, edge_count_dev=None, stream=None) -> None:
    """Resist image, printed pattern and its contour of images (..., Ly, Lx)
    float32 on the device (kl_resist_contour); outputs are optional tensors of
    the same shape (float32 / uint8 / uint8) and edge_count_dev int64 per image."""
    Ly, Lx = images_dev.shape[-2:]
    n = images_dev.numel() // (Lx * Ly)
    p = lambda t: _dev_ptr(t) if t is not None else None
    check(lib().kl_resist_contour(_dev_ptr(images_dev), int(n), int(Lx), int(Ly), float(alpha),
                                  float(threshold), p(resist_dev), p(printed_dev), p(edges_dev),
                                  p(edge_count_dev), _stream_ptr(stream)), "kl_resist_contour")


def fp64_socs_forward(masks_dev, Nx: int, Ny: int, kernels_dev, scales_dev, images_dev, stream=None) -> None:
    """Plain FP64 SOCS image (FT_r2c + calcSOCS + FI with full FFTs): masks
    (n, Ly, Lx) float32, kernels (nk, N, 2) float32, scales (nk,) float32 on the
    device; images_dev (n, Ly, Lx) float64."""
    n, Ly, Lx = masks_dev.shape
    nk = scales_dev.shape[0]
    check(lib().kl_fp64_socs_forward(_dev_ptr(masks_dev), int(n), int(Lx), int(Ly), int(Nx), int(Ny),
                                     _dev_ptr(kernels_dev), _dev_ptr(scales_dev), int(nk),
                                     _dev_ptr(images_dev), _stream_ptr(stream)), "kl_fp64_socs_forward")


def factor_gram(A_dev, G_dev, stream=None) -> None:
    """G = A^H A (S, S) complex128 of a factor A (N, S) complex64 on the device."""
    N, S = A_dev.shape
    check(lib().kl_factor_gram(_dev_ptr(A_dev), int(N), int(S), _dev_ptr(G_dev), _stream_ptr(stream)),
          "kl_factor_gram")


def hermitian_topk(H_dev, K: int, evals_dev, vecs_dev, stream=None) -> None:
    """Top-K eigenpairs of the Hermitian H (B, B) complex128 on the device,
    64 <= B <= 256: eigenvalues descending into evals (K,) float64, eigenvector j
    into vecs[:, j] of vecs (B, K) complex128."""
    B = H_dev.shape[0]
    check(lib().kl_hermitian_topk(_dev_ptr(H_dev), int(B), int(K), _dev_ptr(evals_dev), _dev_ptr(vecs_dev),
                                  _stream_ptr(stream)), "kl_hermitian_topk")


def fp64_mask_spectrum(mask_dev, spectrum_dev, stream=None) -> None:
    """FT_r2c in FP64: mask (Ly, Lx) float32 -> spectrum (Ly, Lx, 2) float64."""
    Ly, Lx = mask_dev.shape[-2:]
    check(lib().kl_fp64_mask_spectrum(_dev_ptr(mask_dev), int(Lx), int(Ly), _dev_ptr(spectrum_dev),
                                      _stream_ptr(stream)), "kl_fp64_mask_spectrum")


def fp64_socs_vjp(masks_dev, targets_dev, Nx: int, Ny: int, kernels_dev, scales_dev, grad_dev, loss_dev,
                  images_dev=None, alpha: float = 50.0, threshold: float = 0.225, stream=None) -> None:
    """Plain FP64 loss and dL/dmask (float64 outputs) of the sigmoid resist
    L2 loss of the SOCS image; masks/targets (n, Ly, Lx) float32."""
    n, Ly, Lx = masks_dev.shape
    nk = scales_dev.shape[0]
    check(lib().kl_fp64_socs_vjp(_dev_ptr(masks_dev), _dev_ptr(targets_dev), int(n), int(Lx), int(Ly),
                                 int(Nx), int(Ny), _dev_ptr(kernels_dev), _dev_ptr(scales_dev), int(nk),
                                 float(alpha), float(threshold),
                                 None if images_dev is None else _dev_ptr(images_dev),
                                 _dev_ptr(grad_dev), _dev_ptr(loss_dev), _stream_ptr(stream)),
          "kl_fp64_socs_vjp")
