/*
 * klitho_gpu.h -- C ABI of the B200-native K-Litho Hopkins/SOCS imaging path.
 *
 * The reference (LithoSimulator/K-Litho) is two single-threaded C++ programs
 * whose imaging functions take std::vector arguments and are called only
 * from their own main()s; it has no library boundary.  This header
 * re-expresses those functions as plain-C entry points (pointers, sizes,
 * int status) so that a host program -- the drop-in klitho_tcc/klitho_socs
 * CLIs shipped here, or a ctypes/cgo/JNI caller -- can bind them.  Each entry
 * point names the reference function it replaces (file:line).
 *
 * Conventions
 *  - Return value: KL_OK (0) on success, a KL_ERR_* code otherwise;
 *    kl_last_error() returns a thread-local message for the last failure.
 *  - "_dev" pointers are device (cudaMalloc'd) memory owned by the caller;
 *    "_host" pointers are host memory.  Complex arrays are interleaved
 *    (re, im) float32 ("c64") or float64 ("c128").
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *    default stream.  Device entry points are stream-ordered and do not
 *    synchronise unless they return host results.
 *  - Arrays are row-major with x fastest, as in the reference.  Band arrays
 *    ("kernel layout") are (2Ny+1) x (2Nx+1) with frequency (ky, kx) at
 *    [(ky+Ny)(2Nx+1) + kx+Nx], the layout of krn_<i>_{r,i}.bin.
 *  - One handle per host thread; handles are not thread-safe.
 */
#ifndef KLITHO_GPU_H
#define KLITHO_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KL_OK 0
#define KL_ERR_INVALID 1        /* bad argument or size                     */
#define KL_ERR_CUDA 2           /* CUDA runtime / launch failure            */
#define KL_ERR_NOMEM 3          /* device or host allocation failed         */
#define KL_ERR_UNSUPPORTED 4    /* geometry outside the compiled kernels    */
#define KL_ERR_NOT_CONVERGED 5  /* eigen-solver hit its iteration cap       */
#define KL_ERR_IO 6             /* file could not be opened / read / written */

/* Library version (major*10000 + minor*100 + patch). */
int kl_version(void);
/* Message describing the most recent failure on this thread ("" if none). */
const char* kl_last_error(void);

/* ------------------------------------------------------------------------- */
/* Host-side inputs (no GPU needed)                                            */
/* ------------------------------------------------------------------------- */

/* createSource: K-Litho-TCC/source.cpp:105-142 (shapes :5-88, point :122-129,
 * import :130-139, normalisation to sum 1 :89-103,141).  `type` is one of
 * "Annular", "Dipole", "CrossQuadrupole", "Point", "Import".  `out` holds
 * srcSize*srcSize floats. */
int kl_create_source(int srcSize, const char* type, float innerRadius, float outerRadius,
                     float radius, float offset, int onXAxis, float ptX, float ptY,
                     const char* sourceFile, float* out);

/* createMask: common/mask.cpp:31-60 (line/space :5-29, import :42-52, centred
 * embedding times dose :53-59).  `type` is "LineSpace" or "Import"; `out`
 * holds Lx*Ly floats. */
int kl_create_mask(int Lx, int Ly, int maskSizeX, int maskSizeY, const char* type, int lineWidth,
                   int spaceWidth, int isHorizontal, const char* maskFile, float dose, float* out);

/* getOuterSigma: K-Litho-TCC/klitho_tcc.cpp:52-67 (before main's clamp). */
float kl_outer_sigma(const float* src_host, int srcSize);

/* Band half-widths Nx, Ny: K-Litho-TCC/klitho_tcc.cpp:479-486 (outerSigma is
 * clamped to 1 as at :480-483).  lambda is 193 nm (:439). */
int kl_band_size(double NA, int Lx, int Ly, float outerSigma, int* Nx, int* Ny);

/* Number of source pixels that enter the TCC (klitho_tcc.cpp:202-205). */
int kl_source_point_count(const float* src_host, int srcSize, float outerSigma);

/* readFloatArrayFromBinary / readFloatArrayFromTxt: common/file_io.cpp:204-260.
 * Reads up to `size` floats ('.bin' raw little-endian, else whitespace text);
 * a short file is zero-padded and, like the reference, a size mismatch is
 * reported as a warning on stderr.  *count receives the number of floats the
 * file held. */
int kl_read_float_file(const char* path, int size, float* out, int* count);
/* writeFloatArrayToBinary: common/file_io.cpp:137-150 */
int kl_write_float_file(const char* path, const float* data, int size);

/* writeKernelInfo / readKernelInfo: common/file_io.cpp:262-307 (same text). */
int kl_write_kernel_info(const char* path, int krnSizeX, int krnSizeY, int nk,
                         const float* scales);
/* scales receives up to `cap` eigenvalues; *nk the declared kernel count. */
int kl_read_kernel_info(const char* path, int* krnSizeX, int* krnSizeY, int* nk, float* scales,
                        int cap);

/* writeFloatArrayToPNGWithGrayscale / ...With7Colors / ...WithContinuousColor:
 * common/file_io.cpp:7-135.  colormap 0 = grey, 1 = seven colours, 2 =
 * continuous colour, each over [min, max] with the reference's pixel
 * arithmetic; data is sizeY rows of sizeX floats.  The file is encoded by
 * the library (zlib deflate), so only the decoded pixels equal the
 * reference's. */
#define KL_PNG_GRAY 0
#define KL_PNG_7COLORS 1
#define KL_PNG_CONTINUOUS 2
int kl_write_png(const char* path, const float* data, int sizeX, int sizeY, float min, float max,
                 int colormap);

/* ------------------------------------------------------------------------- */
/* SOCS imaging: K-Litho-SOCS/klitho_socs.cpp:196-241 (calcSOCS) + :158-194   */
/* (FI), fed by FT_r2c :70-121.  Fused single-precision path.                 */
/* ------------------------------------------------------------------------- */

typedef struct kl_socs_plan_s* kl_socs_plan;
typedef struct kl_tcc_plan_s* kl_tcc_plan; /* see the TCC section below */

/* Plan for clips of period Lx x Ly imaged with `nsets` kernel sets (e.g. one
 * per focus) of `nk` kernels of band (2Nx+1) x (2Ny+1), for batches of up to
 * `max_clips` clips.  Allocates the plan's device workspace on the current
 * device.  Any period is accepted, as the reference accepts any Lx, Ly
 * (K-Litho-SOCS/klitho_socs.cpp:256-270): periods whose pixels split into 32
 * lanes of 8, 16 or 32 (Lx in {256, 512, 768, 1024, 1536, 2048, 3072}, Ly a
 * multiple of the strip height) with 4N+1 <= 128 run on the specialised
 * kernels, every other period and bands up to 4*max(Nx,Ny)+1 <= 256 (4096^2
 * at NA 1.35) on the general pipeline.  Returns KL_ERR_UNSUPPORTED (with a
 * message) beyond that, or when the SOCS grid 4N+1 exceeds half the period. */
int kl_socs_plan_create(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk, int nsets,
                        int max_clips);
int kl_socs_plan_destroy(kl_socs_plan plan);

/* kl_socs_plan_create with options: KL_SOCS_ADJOINT makes the plan that
 * kl_socs_plan_create_adjoint makes; KL_SOCS_GENERAL puts the plan on the
 * general pipeline even where the specialised kernels cover the geometry
 * (same results within the FP32 tolerance; for cross-checks and timing).
 * No counterpart in the reference. */
#define KL_SOCS_ADJOINT 1
#define KL_SOCS_GENERAL 2
int kl_socs_plan_create_ex(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk, int nsets,
                           int max_clips, int flags);
/* 0 if the plan runs on the specialised kernels, 1 on the general pipeline. */
int kl_socs_plan_engine(kl_socs_plan plan);

/* Engine of the mask transform (FT_r2c) and the image synthesis (the FI step)
 * on the specialised kernels: KL_SYNTH_CUDA_CORES, per-lane DFTs of each row;
 * KL_SYNTH_TENSOR_CORES, the same sums as FP16x3 split matrix products on the
 * tensor cores (periods with Lx, Ly multiples of 128 and 2(2Nx+1) <= 128;
 * image error of the same order as the CUDA-core engine's; mask values within
 * +-2^15, others are reported by kl_socs_plan_status); KL_SYNTH_AUTO
 * (the default), the engine kl_socs_autotune picked, else the CUDA cores.
 * kl_socs_vjp runs its image, resist and gradient syntheses on the tensor
 * cores wherever the geometry allows, unless KL_SYNTH_CUDA_CORES is set, and
 * its mask transform there only with KL_SYNTH_TENSOR_CORES.
 * Returns KL_ERR_UNSUPPORTED for the tensor-core engine on other geometries
 * and on general-pipeline plans.  No counterpart in the reference. */
#define KL_SYNTH_AUTO 0
#define KL_SYNTH_CUDA_CORES 1
#define KL_SYNTH_TENSOR_CORES 2
int kl_socs_set_synthesis(kl_socs_plan plan, int mode);
/* The engine the next kl_socs_forward of nclips clips uses (KL_SYNTH_CUDA_CORES
 * or KL_SYNTH_TENSOR_CORES; KL_SYNTH_CUDA_CORES on the general pipeline). */
int kl_socs_synthesis(kl_socs_plan plan, int nclips);
/* Synchronises the device and returns KL_OK, or KL_ERR_CUDA (with a message)
 * if a tensor-core pipeline wait of the plan's kernels has timed out since
 * the last call (the affected images are incomplete); clears the status. */
int kl_socs_plan_status(kl_socs_plan plan);

/* Upload kernel set `set`: nk planes of the kernel layout, real and imaginary
 * parts separately (as krn_<i>_r.bin / krn_<i>_i.bin hold them), and nk
 * eigenvalues (kernel_info.txt).  Host pointers; synchronous. */
int kl_socs_set_kernels(kl_socs_plan plan, int set, const float* krn_re_host,
                        const float* krn_im_host, const float* scales_host);

/* images_dev[c][s] (nclips x nsets x Ly x Lx float32) from masks_dev
 * (nclips x Ly x Lx float32, already embedded in the period as createMask
 * does).  Stream-ordered. */
int kl_socs_forward(kl_socs_plan plan, const float* masks_dev, int nclips, float* images_dev,
                    void* stream);

/* Same computation from and to host memory: copies the masks in, images
 * out, and synchronises `stream` before returning. */
int kl_socs_forward_host(kl_socs_plan plan, const float* masks_host, int nclips,
                         float* images_host, void* stream);

/* ------------------------------------------------------------------------- */
/* Batched imaging: launch-shape autotuning and graph-captured batches.       */
/* No counterpart in the reference, which images one clip per process.       */
/* ------------------------------------------------------------------------- */

/* Times the plan's launch shapes for batches of nclips clips (kernel slices of
 * the spectral stage: 1, 2, 4, 8; image strips per CTA of the synthesis stage:
 * 1 .. 16; the tensor-core synthesis where the geometry allows it) with CUDA
 * events on `stream` and keeps the fastest; later calls of kl_socs_forward
 * with nclips clips use it.  Writes images_dev (the images of the chosen
 * shape).  Synchronous.  The chosen shape is returned in *nsplit / *spc when
 * those are not NULL (*spc = -1: the tensor-core synthesis, -2: the tensor-core
 * synthesis and mask transform). */
int kl_socs_autotune(kl_socs_plan plan, const float* masks_dev, int nclips, float* images_dev,
                     void* stream, int* nsplit, int* spc);

typedef struct kl_socs_batch_s* kl_socs_batch;
/* A batch of plans (e.g. one per clip size, each holding one kernel set per
 * focus value) imaged together: kl_socs_batch_forward runs the plans as
 * concurrent branches of one CUDA graph, so the on-chip stage of one plan
 * overlaps the memory-bound stages of the others.  The plans must outlive the
 * batch. */
int kl_socs_batch_create(kl_socs_batch* batch, const kl_socs_plan* plans, int nplans);
int kl_socs_batch_destroy(kl_socs_batch batch);
/* masks_dev[i] / images_dev[i] / nclips[i] for plan i (layouts as in
 * kl_socs_forward).  The first call for a given set of buffers and counts
 * runs the work directly and captures it as a graph; later calls with the
 * same buffers and counts replay the graph (buffer contents may change).
 * Ordered after earlier work on `stream`; later work on `stream` waits for it. */
int kl_socs_batch_forward(kl_socs_batch batch, const float* const* masks_dev, const int* nclips,
                          float* const* images_dev, void* stream);
/* Per-stage timing inside the graph (recaptures on change); stage times of
 * plan `plan` in the last completed call: ms[0] forward, ms[1] spectral,
 * ms[2] synthesis. */
int kl_socs_batch_enable_timing(kl_socs_batch batch, int enable);
int kl_socs_batch_stage_times(kl_socs_batch batch, int plan, double* ms);
/* Number of graphs captured so far (for checking that replays reuse one). */
int kl_socs_batch_graph_builds(kl_socs_batch batch);

/* ------------------------------------------------------------------------- */
/* Adjoint (VJP) of SOCS imaging under a sigmoid resist and an L2 loss.       */
/* No counterpart in the reference.                                            */
/* ------------------------------------------------------------------------- */

/* A SOCS plan that also supports kl_socs_vjp (taller strips so the band of
 * dL/dI fits).  Clips up to 1024^2 at NA 1.35 run on the specialised
 * kernels, larger bands and other periods on the general pipeline, with the
 * limits of kl_socs_plan_create.  Its kl_socs_forward gives the same images
 * as kl_socs_plan_create's within the FP32 tolerance. */
int kl_socs_plan_create_adjoint(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk,
                                int nsets, int max_clips);

/* loss[c*nsets+s] = sum_x (sigmoid(alpha (I - threshold)) - target)^2 for the
 * SOCS image I of clip c under kernel set s, and grad_dev[c] = dL/dmask
 * summed over the sets (nclips x Ly x Lx float32).  images_dev may be NULL
 * (the image is then not written).  The K coherent fields are recomputed on
 * chip, never stored.  Stream-ordered; loss_dev is device memory.
 * targets_dev must be 16-byte aligned (any cudaMalloc or torch allocation is). */
int kl_socs_vjp(kl_socs_plan plan, const float* masks_dev, const float* targets_dev, int nclips,
                float alpha, float threshold, float* images_dev, float* grad_dev,
                double* loss_dev, void* stream);

/* dL/dJ for the source map of `tcc` (srcSize^2 float32, zero where the map
 * has no TCC source point), from the last kl_socs_vjp on this plan, summed
 * over its clips.  Defined through the TCC factor A = sqrt(J) P (the Hopkins
 * model): dL/dJ_s = sum_x dL/dI(x) |E_s(x)|^2.  One kernel set per plan;
 * synchronous. */
int kl_socs_vjp_source(kl_socs_plan plan, kl_tcc_plan tcc, float* grad_src_dev, void* stream);

/* Stage timing for diagnostics and roofline accounting.  While enabled, every
 * kl_socs_forward records CUDA events on its stream around its three kernels
 * (mask forward transform, spectral core, image synthesis).
 * kl_socs_stage_times synchronises on those events, returns the summed
 * milliseconds and launch counts per stage (ms[3], launches[3]) and clears
 * them.  No reference counterpart (the reference prints wall time only,
 * klitho_socs.cpp:355-361). */
int kl_socs_enable_timing(kl_socs_plan plan, int enable);
int kl_socs_stage_times(kl_socs_plan plan, double* ms, int* launches);

/* SOCS images without any memory allocation.  No counterpart in the
 * reference.  For callers that may not allocate device memory at run time
 * (a fixed memory budget handed over at start-up, a framework that owns the
 * allocator, code where cudaMalloc would synchronise or fail): the caller
 * passes every buffer -- masks (nclips x Ly x Lx float32), kernels in the
 * kernel layout as interleaved c64 (nk x (2Ny+1)(2Nx+1)), nk float scales,
 * images (nclips x Ly x Lx float32), all device memory -- and the scratch
 * comes from one static 8 MiB device array inside the library (about 38 clips
 * of 1024^2 per call; larger requests return KL_ERR_INVALID with the sizes in
 * kl_last_error).  The first call on each device looks up that array's
 * device address; make it before any stream capture.  The address is looked
 * up again when the device's primary context has changed since (after a
 * cudaDeviceReset); make the first call after such a reset outside a capture
 * as well.  Calls share the array,
 * so calls that overlap on the GPU race and must be serialised by the
 * caller.  Same results as kl_socs_forward with one kernel set. */
int kl_socs_forward_noalloc(const float* masks_dev, int nclips, int Lx, int Ly, int Nx, int Ny,
                            const float* kernels_dev, const float* scales_dev, int nk,
                            float* images_dev, void* stream);

/* Resist image and printed contour of nimg aerial images (Lx x Ly float32
 * each, e.g. kl_socs_forward's output).  The reference uses its threshold
 * TARGET_INTENSITY = 0.225 (K-Litho-TCC/klitho_tcc.cpp:442) only as the top
 * of image_s.png's colour scale (:547); here it defines, per pixel,
 *   resist_dev  = 1 / (1 + exp(-alpha (I - threshold)))   (the adjoint's resist model)
 *   printed_dev = I >= threshold ? 1 : 0                   (bytes)
 *   edges_dev   = 1 where a printed pixel has a 4-neighbour (periodic over the
 *                 clip) that does not print: the contour of the pattern
 * and edge_count_dev[i] the number of contour pixels of image i (unsigned
 * 64-bit).  Any output may be NULL.  Device memory; stream-ordered; rows up to
 * 5120 pixels. */
int kl_resist_contour(const float* images_dev, int nimg, int Lx, int Ly, float alpha, float threshold,
                      float* resist_dev, unsigned char* printed_dev, unsigned char* edges_dev,
                      unsigned long long* edge_count_dev, void* stream);

/* The band of FT_r2c (K-Litho-TCC/klitho_tcc.cpp:97-148): centred spectrum
 * scaled by 1/(Lx Ly), cropped to the kernel band; band_dev receives nclips
 * c64 arrays in the kernel layout.  Stream-ordered. */
int kl_mask_spectrum(kl_socs_plan plan, const float* masks_dev, int nclips, float* band_dev,
                     void* stream);

/* ------------------------------------------------------------------------- */
/* Plain FP64 path: the reference's FFT-based chain restated in FP64 on the   */
/* GPU (full L x L FFTs, the K fields of calcSOCS materialised), for FP64      */
/* parity and as the baseline of the fused path.  Lx, Ly powers of two.       */
/* ------------------------------------------------------------------------- */

/* FT_r2c (K-Litho-SOCS/klitho_socs.cpp:70-121) in FP64: spectrum_dev receives
 * Lx*Ly complex128 (interleaved doubles), DC at [Ly/2][Lx/2], scaled by
 * 1/(Lx Ly).  Synchronous. */
int kl_fp64_mask_spectrum(const float* mask_dev, int Lx, int Ly, double* spectrum_dev, void* stream);
/* FT_r2c + calcSOCS + FI (klitho_socs.cpp:338-343, :196-241, :158-194) in FP64
 * for nclips masks; kernels_dev nk x (2Nx+1)(2Ny+1) complex64 interleaved (the
 * krn_*.bin contents), scales_dev nk floats; images_dev nclips x Ly x Lx
 * doubles (the reference's image before its float store).  Stream-ordered;
 * allocates its scratch per call. */
int kl_fp64_socs_forward(const float* masks_dev, int nclips, int Lx, int Ly, int Nx, int Ny,
                         const float* kernels_dev, const float* scales_dev, int nk, double* images_dev,
                         void* stream);
/* kl_socs_vjp's loss and mask gradient (one kernel set) in FP64 with the
 * fields materialised: loss_dev[c], grad_dev (nclips x Ly x Lx doubles) and,
 * if images_dev is not NULL, the FP64 image.  The plain-path counterpart of
 * the fused adjoint; no reference counterpart.  Stream-ordered. */
int kl_fp64_socs_vjp(const float* masks_dev, const float* targets_dev, int nclips, int Lx, int Ly, int Nx,
                     int Ny, const float* kernels_dev, const float* scales_dev, int nk, double alpha,
                     double threshold, double* images_dev, double* grad_dev, double* loss_dev, void* stream);

/* ------------------------------------------------------------------------- */
/* TCC assembly, SOCS kernels, Hopkins image: K-Litho-TCC/klitho_tcc.cpp      */
/* ------------------------------------------------------------------------- */

#define KL_PREC_FAST 0 /* FP32 pupil factor, 3-term BF16 tensor-core TCC, FP64 Rayleigh-Ritz */
#define KL_PREC_FP64 1 /* plain FP64 GPU path (pupil table from the host libm, FP64 TCC)    */

/* Optical setting of one TCC: source map (createSource output, host), NA,
 * defocus in the reference's normalised units (argv[21], dz = defocus *
 * lambda / NA^2, klitho_tcc.cpp:191), immersion index n_medium (1 reproduces
 * klitho_tcc.cpp:220; NA > 1 needs n_medium >= NA), period Lx x Ly.
 * Computes outer sigma and the band (klitho_tcc.cpp:479-486), the source
 * points (:202-211) and the pupil factor A[f][s] = sqrt(J_s) P(f, s)
 * (:201-228) on the current device. */
int kl_tcc_plan_create(kl_tcc_plan* plan, const float* src_host, int srcSize, double NA,
                       double defocus, double n_medium, int Lx, int Ly, int precision);
int kl_tcc_plan_destroy(kl_tcc_plan plan);
/* Band half-widths, TCC size N = (2Nx+1)(2Ny+1), source point count S, sigma_o. */
int kl_tcc_plan_info(kl_tcc_plan plan, int* Nx, int* Ny, int* N, int* S, float* outerSigma);
/* Copy the FP32 factor A (N x S c64, row-major) to A_dev (fast path only). */
int kl_tcc_factor(kl_tcc_plan plan, float* A_dev, void* stream);

/* G = A^H A (S x S complex128, row-major) of a TCC factor A (N x S complex64,
 * row-major, e.g. from kl_tcc_factor) on the device: the Gram step of
 * kl_topk_eig.  Exact products of the FP32 factor in FP64 -- integer digits on
 * the tensor cores for S <= 256 and N <= 500000 on B200, FP64 CUDA cores
 * otherwise.  Synchronous (reports pipeline timeouts). */
int kl_factor_gram(const void* A_dev, int N, int S, void* G_dev, void* stream);

/* Top-K eigenpairs of a Hermitian B x B complex128 matrix on the device
 * (row-major, 64 <= B <= 256, 1 <= K <= B): the eigensolve behind kl_topk_eig's
 * Gram step, the part of zheevr (klitho_tcc.cpp:300-377) that remains once the
 * TCC is reduced to its source span.  Householder tridiagonalisation on a
 * cluster of 8 CTAs, bisection, inverse iteration; eigenvalues descending into
 * evals_dev (K doubles), eigenvector j into column j of vecs_dev (B x K
 * complex128, row-major).  H_dev is not modified.  The reduction forms sums of
 * squares of the entries without rescaling: entries should lie within about
 * 1e-150 .. 1e150 in magnitude (a Gram matrix of a TCC factor is far inside).
 * Synchronous (reports a timed-out exchange of the reduction). */
int kl_hermitian_topk(const void* H_dev, int B, int K, double* evals_dev, void* vecs_dev, void* stream);

/* calcTCC (klitho_tcc.cpp:186-267): the N x N Hermitian TCC, row-major, into
 * tcc_dev -- c64 on the fast path (tcgen05 tensor cores, BF16x3 split, FP32
 * accumulate), c128 on the FP64 path.  Synchronous on the fast path (reports
 * pipeline timeouts). */
int kl_tcc_build(kl_tcc_plan plan, void* tcc_dev, void* stream);
/* {max re, min re, max im, min im} of a TCC built by kl_tcc_build (the
 * "Max. TCC Real/Imag Value" lines of klitho_tcc.cpp:521-528). */
int kl_tcc_minmax(kl_tcc_plan plan, const void* tcc_dev, double* out4, void* stream);
/* Build the TCC into library-owned device memory, return its min/max as above
 * and release it (what klitho_tcc prints; the TCC itself is not an output of
 * the reference program). */
int kl_tcc_build_minmax(kl_tcc_plan plan, double* out4);
/* The TCC as two host float planes (N x N each, row f1, column f2): the
 * tccReal / tccImag arrays klitho_tcc.cpp:517-529 turns into tcc_r.png /
 * tcc_i.png.  Synchronous. */
int kl_tcc_build_host(kl_tcc_plan plan, float* re_host, float* im_host);

/* calcKernels (klitho_tcc.cpp:300-377): top-nk eigenpairs of the TCC, in
 * descending order.  Fast plans with S <= 256 source points take one exact
 * Rayleigh-Ritz step on the source span: G = A^H A (kl_factor_gram), its
 * top-nk by the tridiagonal solver (kl_hermitian_topk; Jacobi below order 64),
 * U = A V diag(w)^-1/2; `iterations` is 1.  Otherwise blocked subspace
 * iteration (block `block`, 0 = automatic) with FP64 CholeskyQR2 and
 * Rayleigh-Ritz, returning KL_ERR_NOT_CONVERGED if the iteration cap is
 * reached.  Kernels in the reference layout krn[k][j] = v_k[N-1-j] as float
 * planes (nk x N each), scales = eigenvalues as float, evals_host (optional)
 * in double. */
int kl_topk_eig(kl_tcc_plan plan, int nk, int block, float* krn_re_host, float* krn_im_host,
                float* scales_host, double* evals_host, int* iterations);
/* kl_topk_eig for nplans plans that share the pupil band N (e.g. one per
 * focus value of a focus-exposure sweep; no counterpart in the reference,
 * whose klitho_tcc handles one focus per run).  Outputs are the per-plan
 * outputs of kl_topk_eig back to back: plan i's kernels at
 * krn_re_host + i*nk*N, its scales at scales_host + i*nk, evals_host (optional)
 * likewise, iterations (optional) at iterations[i].  On the fast path with
 * S <= 256 source points the Rayleigh-Ritz step on span(A) is exact and the
 * plans' eigensolves run concurrently in one batch of launches; otherwise (or
 * for FP64 plans) the plans are solved one after another. */
int kl_topk_eig_batch(const kl_tcc_plan* plans, int nplans, int nk, int block, float* krn_re_host,
                      float* krn_im_host, float* scales_host, double* evals_host, int* iterations);
/* kl_topk_eig / kl_topk_eig_batch with the kernels as interleaved complex64
 * (re, im pairs: nk x N x 2 floats per plan) in one host buffer, for callers
 * that hold kernels as complex arrays: one copy instead of two planes. */
int kl_topk_eig_c64(kl_tcc_plan plan, int nk, int block, float* krn_host, float* scales_host,
                    double* evals_host, int* iterations);
int kl_topk_eig_batch_c64(const kl_tcc_plan* plans, int nplans, int nk, int block, float* krn_host,
                          float* scales_host, double* evals_host, int* iterations);

/* Hopkins image (calcImage + FT_c2r, klitho_tcc.cpp:269-290, :150-183) of
 * nclips masks: sum_s J_s |IFFT(P(.,s) conj . M)|^2, the source-point form
 * of the TCC contraction (identical in exact arithmetic), computed by the
 * fused SOCS pipeline with the columns of A as kernels.  Fast path only. */
int kl_hopkins_image(kl_tcc_plan plan, const float* masks_dev, int nclips, float* images_dev,
                     void* stream);
/* One Hopkins image from and to host memory (Lx*Ly floats each); synchronous. */
int kl_hopkins_image_host(kl_tcc_plan plan, const float* mask_host, float* image_host);
/* calcImage + FT_c2r (klitho_tcc.cpp:269-290, :150-183) in FP64 on the plan's
 * FP64 TCC (built on first use) with full L x L FFTs: the plain FP64 path of
 * the Hopkins image, in double (before the reference's float store).  Plans
 * of KL_PREC_FP64 precision only. */
int kl_fp64_hopkins_image(kl_tcc_plan plan, const float* masks_dev, int nclips, double* images_dev,
                          void* stream);
/* One FP64 Hopkins image from and to host memory, stored as float as the
 * reference stores image.bin (klitho_tcc.cpp:537-544); KL_PREC_FP64 plans,
 * Lx and Ly powers of two.  Synchronous. */
int kl_fp64_hopkins_image_host(kl_tcc_plan plan, const float* mask_host, float* image_host);

#ifdef __cplusplus
}
#endif
#endif /* KLITHO_GPU_H */
