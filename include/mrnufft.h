/*
 * mrnufft -- B200 (sm_100a) Kaiser-Bessel NUFFT for MRI reconstruction.
 *
 * C ABI of libmrnufft.so. Every pointer argument is DEVICE memory owned by the
 * caller unless stated otherwise; every call is asynchronous on the given
 * CUDA stream (a cudaStream_t passed as void*, NULL = legacy default stream)
 * and returns MRN_OK (0) or a negative MRN_ERR_* code. No C++ exception
 * crosses this boundary. A plan is not thread-safe: use one plan per stream.
 *
 * Data conventions (those of mr_recon's triton_nufft, src/mr_recon/fourier.py):
 *   complex values  : complex64, interleaved re/im (torch.view_as_real layout)
 *   image           : slice-major, per slice [C][N0][N1][N2] (last axis fastest)
 *   k-space samples : per slice [C][M]
 *   trajectory      : per slice [M][ndim] float32, grid units k_i in [-N_i/2, N_i/2)
 *   oversampled grid: per slice [C][Nos0][Nos1][Nos2], Nos_i = ceil(os * N_i),
 *                     centred (DC at index Nos_i//2), as forward_FT_only returns
 * A "plan" holds n_slices independent NUFFT problems that share ndim, width,
 * oversampling and beta but may differ in image size, sample count and coil
 * count (uneven batches); slices are laid out back to back in every buffer,
 * at the offsets reported by mrn_plan_offsets().
 */
#ifndef MRNUFFT_H
#define MRNUFFT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MRN_OK 0
#define MRN_ERR_ARG (-1)      /* bad argument: shape, dims, null pointer, layout */
#define MRN_ERR_WIDTH (-2)    /* kernel width outside [1, 15] (mirrors the ValueError of
                                 ungrid.py:132-143 get_block_width for too-wide kernels) */
#define MRN_ERR_CUDA (-3)     /* CUDA runtime error (see mrn_last_cuda_error) */
#define MRN_ERR_CUFFT (-4)    /* cuFFT error */
#define MRN_ERR_NOMEM (-5)    /* device allocation failed */
#define MRN_ERR_STATE (-6)    /* plan used before mrn_plan_set_traj */
#define MRN_ERR_UNSUPPORTED (-7)
#define MRN_ERR_SCRATCH (-8)  /* problem larger than the fixed scratch of mrn_interp_noalloc */

/* Plan flags */
#define MRN_PLAN_RAW 1        /* im_size is the grid size itself; trajectories are grid
                                 coordinates used as-is (reference ungrid/grid,
                                 triton_interp/ungrid.py:34, grid.py:32); no FFT stage */
#define MRN_PLAN_NO_APOD 2    /* apodize=False (fourier.py:366) */

typedef struct mrn_plan mrn_plan;

const char* mrn_version(void);
const char* mrn_error_string(int code);
int mrn_last_cuda_error(void);

/*
 * Create a plan. Replaces triton_nufft.__init__ (fourier.py:361-374) plus the
 * per-call shape preparation of prep_ungrid_shapes / prep_grid_shapes
 * (ungrid.py:851-894, grid.py:508-553), hoisted to once per geometry.
 *   ndim       1, 2 or 3
 *   im_size    [n_slices * ndim] image size per slice (grid size with MRN_PLAN_RAW)
 *   n_pts      [n_slices] samples per slice
 *   n_coil     [n_slices] image batch (coils) per slice
 *   width      kernel width per dimension, [ndim] (reference `width` tuple)
 *   beta       KB shape parameter; beta <= 0 selects the reference default
 *              pi*sqrt((W/os*(os-0.5))^2 - 0.8) of fourier.py:372
 *   tile       [ndim] tile edge in grid cells, or NULL for the built-in choice
 *   coil_group coils per CTA, 0 = built-in choice
 *   max_chunk  maximum samples per work item, 0 = built-in choice
 * Host arrays: im_size, n_pts, n_coil, width, tile. Allocates device memory.
 */
int mrn_plan_create(mrn_plan** plan, int ndim, int n_slices, const int* im_size,
                    const int64_t* n_pts, const int* n_coil, double oversamp,
                    const double* width, double beta, int flags, const int* tile,
                    int coil_group, int max_chunk, int device);
int mrn_plan_destroy(mrn_plan* plan);

/* Host-side layout query: writes n_slices entries to each non-NULL array
 * (element offsets, in complex64 units for img/ksp/grid, float units for trj). */
int mrn_plan_offsets(const mrn_plan* plan, int64_t* img_off, int64_t* ksp_off,
                     int64_t* grid_off, int64_t* trj_off);
/* Totals: [0] image elems, [1] ksp elems, [2] grid elems, [3] trj floats,
 * [4] number of tiles, [5] oversampled size dim0, [6] dim1, [7] dim2 (slice 0). */
int mrn_plan_sizes(const mrn_plan* plan, int64_t* out8);
/* Number of interp and gridding work items, gridding entries, and split
 * (multi-item) gridding tiles of the bound trajectory, in out4 (all zero
 * before mrn_plan_set_traj). Synchronises the plan's device to read them. */
int mrn_plan_stats(mrn_plan* plan, int64_t* out4);

/* Which FFT the plan's transforms run (no counterpart in the reference):
 * 0 cuFFT for every grid size, 1 the native per-axis passes for every grid
 * size (MRN_OPT_NATIVE_FFT), 2 native for some FFT groups and cuFFT for the
 * others; a negative MRN_ERR_* code for a null plan. */
int mrn_plan_fft_kind(const mrn_plan* plan);

/* Plan options (no counterpart in the reference).
 * MRN_OPT_FAST_KERNELS (default 1): use the unrolled fixed-width tile kernels
 * where they apply (2D/3D, equal width in [4, 8) per dimension); 0 forces the
 * general kernels. Both compute the same taps and weights. */
#define MRN_OPT_FAST_KERNELS 1
/* MRN_OPT_WARP_GRIDDING (default 1): 2D gridding with one warp per output tile
 * (no atomics, reproducible summation order) where the fast kernels apply; 0
 * uses the shared-memory-atomic tile kernel (whose shared-memory float atomics
 * add in a run-dependent order). On every path, tiles split over several
 * work items are combined by adding their partial tiles in item order. */
#define MRN_OPT_WARP_GRIDDING 2
/* MRN_OPT_WEIGHT_TABLES (default 0): in 2D, mrn_plan_set_traj evaluates the KB
 * weights of every sample once and stores them (~80 bytes per sample and per
 * gridding entry); interpolation and gridding then read them instead of
 * re-evaluating the kernel on every call. Set before mrn_plan_set_traj. */
#define MRN_OPT_WEIGHT_TABLES 3
/* Work decomposition (each takes effect at the next mrn_plan_set_traj):
 * MRN_OPT_INTERP_CHUNK / MRN_OPT_GRID_CHUNK: samples per interpolation work
 * item and gridding entries per gridding work item (defaults: 256 / 256 in
 * 2D, 1024 / 4096 in 3D, 1024 in 1D); MRN_OPT_INTERP_TILE / MRN_OPT_GRID_TILE:
 * tile edge in grid cells, every dimension (defaults: 10 / 8 in 2D, 4 / 8 in
 * 3D, 256 in 1D). */
#define MRN_OPT_INTERP_CHUNK 4
#define MRN_OPT_GRID_CHUNK 5
#define MRN_OPT_INTERP_TILE 6
#define MRN_OPT_GRID_TILE 7
/* MRN_OPT_REG_GRIDDING (default 1): 2D gridding tiles of at most 8x8 cells
 * keep their accumulator in registers (two warps per tile, lane = coil);
 * 0 keeps it in shared memory. Each gives the same bits from run to run. */
#define MRN_OPT_REG_GRIDDING 8
/* MRN_OPT_REG_INTERP (default 1): 2D and 3D interpolation with one lane per
 * coil over the tile region staged as [cell][coil] (packed two-lane FMAs); 0
 * uses the coil-plane kernel. */
#define MRN_OPT_REG_INTERP 9
/* MRN_OPT_GRID_LANES (default 0): lanes of one coil group in the 2D
 * register gridding, 8, 16 or 32 (0: the plan's coil group rounded up). A
 * group of fewer lanes than 32 splits a warp into entry streams whose partial
 * tiles are added at the end, so the summation order depends on it; a
 * one-slice plan given the lane count of a larger uneven plan (the lanes its
 * widest slice needs) adds every cell in the same order as that plan. */
#define MRN_OPT_GRID_LANES 10
/* MRN_OPT_ENTRY_MAJOR (default 1): in 2D, mrn_plan_set_traj also builds the
 * map from samples to gridding entries and a sample buffer of 8 * (largest
 * coil count) bytes per gridding entry (about 2.7x the k-space at width 6),
 * so that mrn_sense_normal keeps its samples in entry order between the
 * interpolation and the gridding (contiguous rows instead of per-coil
 * gathers; the same bits). 0 skips both; set before mrn_plan_set_traj. */
#define MRN_OPT_ENTRY_MAJOR 11
/* MRN_OPT_NATIVE_FFT (default 1): the FFT stage as the library's own passes
 * (one per axis, Stockham in shared memory, radices 2, 3, 4, 5, 8, 16) with the apodize /
 * zero-pad folded into the first forward pass and the crop / deapodize into
 * the last adjoint pass, the zero-padded lines skipped; used when every slice
 * has the same image and grid size and every grid size is a product of 2, 3
 * and 5 of at most 1024. 0 (or any other plan) uses cuFFT between separate
 * pad and crop kernels. The two agree to float32 rounding, not bitwise. */
#define MRN_OPT_NATIVE_FFT 12
int mrn_plan_set_option(mrn_plan* plan, int option, int value);

/* Kaiser-Bessel beta per dimension for a raw (MRN_PLAN_RAW) plan, beta[0..ndim),
 * the per-axis kernel parameter sigpy's interpolate/gridding take and the
 * type-3 NUFFT passes (mr_recon linops.py:258-262, 312-319). Dimensions with
 * different betas run the generic tile kernels. The trajectory must be bound
 * again afterwards (MRN_ERR_STATE until then). Non-raw plans: MRN_ERR_ARG. */
int mrn_plan_set_beta(mrn_plan* plan, const double* beta);

/* Stage timing, a profiling aid with no counterpart in the reference (which
 * only prints wall-clock, recons.py:127-133). When on, every call records a
 * CUDA event pair around each stage on the launching stream (not for use
 * under stream capture). mrn_plan_timing waits for the recorded events,
 * writes per-stage total milliseconds and counts for the 8 stages
 *   0 pre-FFT  1 FFT  2 interpolation  3 gridding  4 post-iFFT
 *   5 layout copy  6 trajectory gradient  7 CG vector ops
 * and clears the record. */
int mrn_plan_enable_timing(mrn_plan* plan, int on);
int mrn_plan_timing(mrn_plan* plan, double* ms8, int64_t* count8);

/*
 * Bind a trajectory (device, float32, all slices back to back). Scales it
 * (triton_nufft._scale_trj, fourier.py:420-430), wraps it circularly
 * (torch.remainder, ungrid.py:873), and sorts the samples into spatial tiles
 * for both interpolation and gridding. Must be called again when the
 * trajectory values change. NOT asynchronous and not for use under stream
 * capture: it waits for the stream once, to read back the number of gridding
 * entries, and may allocate device memory when that number (or the work-item
 * or partial-tile capacity derived from it) outgrows the plan's buffers.
 * Everything else (sorts, work items, their longest-first order) stays on the
 * device. Plans are limited to fewer than 2^31 samples and 2^31 gridding
 * entries (2^d entries per sample at most): mrn_plan_create returns
 * MRN_ERR_UNSUPPORTED beyond that.
 */
int mrn_plan_set_traj(mrn_plan* plan, const float* trj, void* stream);

/* Full NUFFT. forward: triton_nufft.forward = forward_interp_only(forward_FT_only)
 * (fourier.py:230-252, 432-503). adjoint: adjoint_iFT_only(adjoint_grid_only)
 * (fourier.py:254-276, 505-550). img/ksp in the slice layout above. */
int mrn_forward(mrn_plan* plan, const void* img, void* ksp, void* stream);
int mrn_adjoint(mrn_plan* plan, const void* ksp, void* img, void* stream);

/* Split stages with the reference's centred grid layout.
 * forward_ft  : triton_nufft.forward_FT_only   (fourier.py:432-468)
 * interp      : triton_nufft.forward_interp_only (fourier.py:470-503), output * scale
 * grid        : triton_nufft.adjoint_grid_only (fourier.py:527-550), output * scale
 * adjoint_ift : triton_nufft.adjoint_iFT_only  (fourier.py:505-525)
 * With MRN_PLAN_RAW, interp/grid are ungrid/grid of triton_interp (ungrid.py:34,
 * grid.py:32) with pad_mode='circular', norm='1', kernel='kaiser_bessel'. */
int mrn_forward_ft(mrn_plan* plan, const void* img, void* grid, void* stream);
int mrn_interp(mrn_plan* plan, const void* grid, void* ksp, float scale, void* stream);
int mrn_grid(mrn_plan* plan, const void* ksp, void* grid, float scale, void* stream);
int mrn_adjoint_ift(mrn_plan* plan, const void* grid, void* img, void* stream);

/*
 * Trajectory gradient (no counterpart in the reference: InterpolateFn.backward,
 * triton_interp/interp.py:51-74, returns grad_locs=None). For the centred grid
 * G (as mrn_forward_ft writes) and sample weights S (both complex64), writes
 * grad[p, i] = scale * Re sum_c conj(S[c,p]) * sum_j dW(u_p - j)/du_i * G[c,j]
 * times d u_i / d k_i, i.e. the derivative of Re<S, interp(G)> w.r.t. the
 * trajectory k (float32, slice layout [M][ndim]).
 */
int mrn_traj_grad(mrn_plan* plan, const void* grid, const void* samples, float* grad,
                  float scale, void* stream);

/*
 * SENSE operator of sense_linop (linops.py:1041-1308) with identity
 * spatial/temporal functions, one image per slice:
 *   forward: ksp[c] = NUFFT(mps[c] * x)                   (linops.py:1134-1178)
 *   adjoint: x = sum_c conj(mps[c]) NUFFT^H(dcf * ksp[c])  (linops.py:1180-1228)
 *   normal : out = adjoint(forward(x)) * out_scale + lam * x (linops.py:1230-1247)
 * x/out: per slice [N...]; mps: per slice [C][N...] (image layout); dcf: per
 * slice [M] float32 or NULL. With pap != NULL, normal also accumulates
 * Re<x, out> per slice into pap[slice * pap_stride] (float64, caller zeroes
 * it; pass the CG state + 1 with stride 8 to feed mrn_cg_step directly).
 */
int mrn_sense_forward(mrn_plan* plan, const void* x, const void* mps, void* ksp, void* stream);
int mrn_sense_adjoint(mrn_plan* plan, const void* ksp, const float* dcf, const void* mps,
                      void* x, float out_scale, void* stream);
int mrn_sense_normal(mrn_plan* plan, const void* x, const void* mps, const float* dcf,
                     void* out, float out_scale, float lam, double* pap, int pap_stride,
                     void* stream);

/*
 * Low-rank SENSE operators: time-segmented off-resonance models with any
 * temporal interpolators (sense_linop with spatial_funcs / temporal_funcs,
 * linops.py:1134-1228, e.g. alpha_segementation's least-squares h_l(t),
 * imperfections/field.py:272-369) and subspace models (subspace_linop,
 * linops.py:1496-1772; subspace_linop_new, 1379-1495). The plan's slices are
 * the J components (a segment, or a subspace coefficient and segment): all
 * slices have the same image size, coil count C and sample count M, and the
 * same trajectory (bound once per slice, back to back). x / out hold one
 * component image per slice (b_l times the coefficient volume, the caller's
 * elementwise product), mps per slice [C][N...], w per slice [M] complex64
 * (the component's temporal weight h_l(t) phi_k(t)); ksp is one [C][M] block.
 *   mrn_lr_forward: ksp[c][t] = sum_j w[j][t] NUFFT_j(mps[j][c] x[j])[t]
 *                   (components summed in order)
 *   mrn_lr_adjoint: x[j] = out_scale sum_c conj(mps[j][c]) NUFFT_j^H(conj(w[j]) ksp[c])
 *                   (fold a density compensation into w: it is real)
 *   mrn_lr_normal : out[j] = out_scale lr_adjoint(lr_forward(x; w_fwd); w_adj)[j] + lam x[j]
 * MRN_ERR_ARG when the slices differ in coil or sample count.
 */
int mrn_lr_forward(mrn_plan* plan, const void* x, const void* mps, const void* w, void* ksp,
                   void* stream);
int mrn_lr_adjoint(mrn_plan* plan, const void* ksp, const void* w, const void* mps, void* x,
                   float out_scale, void* stream);
int mrn_lr_normal(mrn_plan* plan, const void* x, const void* mps, const void* w_fwd, const void* w_adj,
                  void* out, float out_scale, float lam, void* stream);

/*
 * Toeplitz (FFT-only) normal operator A^H A, for plans without MRN_PLAN_RAW.
 * Replaces NUFFT.normal_toeplitz (fourier.py:302-352) and the Toeplitz branch
 * of sense_linop.normal (linops.py:1249-1308) for one image per slice and no
 * time segmentation. The kernel is what calc_teoplitz_kernels
 * (fourier.py:552-582) returns: per slice the centred complex64 kernel on the
 * padded grid pad_size[s * ndim + i] (normally twice the image size; pad_size
 * - im_size must be even, the centred pad of PadLast), slices back to back.
 * mrn_plan_set_toeplitz copies it into the plan (reordered for the FFT, with
 * the 1 / prod(pad) of the two orthonormal FFTs folded in), allocating the
 * padded grids and their cuFFT plans when the sizes change; it needs no
 * trajectory. Then, with centred orthonormal FFTs on the padded grid:
 *   mrn_toeplitz_normal      : out[c] = crop(IFFT(K * FFT(pad(img[c]))))
 *                              (img/out in the image layout [C][N...])
 *   mrn_sense_normal_toeplitz: out = out_scale * sum_c conj(mps[c])
 *                              crop(IFFT(K * FFT(pad(mps[c] x)))) + lam x,
 *                              pap as in mrn_sense_normal (fixed-order sum)
 * Both return MRN_ERR_STATE before mrn_plan_set_toeplitz.
 */
int mrn_plan_set_toeplitz(mrn_plan* plan, const int* pad_size, const void* kern, void* stream);
int mrn_toeplitz_normal(mrn_plan* plan, const void* img, void* out, void* stream);
int mrn_sense_normal_toeplitz(mrn_plan* plan, const void* x, const void* mps, void* out, float out_scale,
                              float lam, double* pap, int pap_stride, void* stream);

/*
 * Conjugate-gradient vector steps for n_slices independent systems (the loop
 * body of conjugate_gradient, algs.py:779-872), complex64 vectors with
 * float64 dot products and norms. Every float64 sum is taken in a fixed order
 * (per-block partials added in block order), so a solve gives the same bits
 * on every run, eager or replayed from a CUDA graph; per-slice scalars stay on
 * the device, so a whole solve can be captured. Vectors use the per-slice
 * image layout (one image per slice). state: float64 [n_slices * 8] owned by
 * the caller:
 *   [0] rz  [1] pAp (accumulated)  [2] rr (accumulated)  [3] done  [4] tol^2
 *   [5] iterations  [6] last alpha  [7] last beta
 * mrn_cg_init : zero state; r = b - Ab (Ab given), p = r, x = b, rz = |r|^2
 * per iteration: Ap = (A^H A + lam) p accumulating pAp into state[1]
 *                (mrn_sense_normal with pap = state + 1, pap_stride = 8), then
 * mrn_cg_step : alpha = rz/pAp; x += alpha p; r -= alpha Ap; rr = |r|^2
 * mrn_cg_dir  : done |= rr < tol^2; beta = rr/rz; p = r + beta p; rz = rr;
 *               pAp = rr = 0 for the next iteration
 * Once a slice is done its vectors are left unchanged (the reference breaks
 * out of the loop at the same point, algs.py:859-860).
 */
int mrn_cg_init(mrn_plan* plan, const void* b, const void* Ab, void* x, void* r, void* p,
                double* state, double tol, void* stream);
int mrn_cg_step(mrn_plan* plan, void* x, void* r, const void* p, const void* Ap,
                double* state, void* stream);
int mrn_cg_dir(mrn_plan* plan, const void* r, void* p, double* state, void* stream);
/* Per-slice Re<a, b> in float64 (fixed summation order), accumulated into
 * out[slice] (caller zeroes). */
int mrn_cg_dot(mrn_plan* plan, const void* a, const void* b, double* out, void* stream);

/*
 * Type-2 interpolation that allocates nothing (no counterpart in the
 * reference). For callers that cannot call cudaMalloc when they interpolate:
 * work issued while a CUDA graph is being captured (allocation is not allowed
 * there), real-time loops whose device memory is reserved up front, or hosts
 * whose framework allocator owns all device memory. It needs no plan; its
 * scratch is one fixed 32 MiB array in device memory that every GPU loading
 * libmrnufft.so holds until the process exits.
 * Result: the same as mrn_interp on an MRN_PLAN_RAW plan of this grid with
 * scale 1 (ungrid, triton_interp/ungrid.py:34, kernel='kaiser_bessel',
 * norm='1', pad_mode='circular'): grid [n_coil][grid_size...] complex64,
 * locs [n_pts][ndim] float32 grid coordinates (wrapped), out [n_coil][n_pts].
 * Limit: n_pts * ndim * (1 + K) * 4 bytes (+ 256) <= 32 MiB, K = floor(max
 * width) + 1 -- about 524,000 samples for 2D width 6; larger calls return
 * MRN_ERR_SCRATCH without launching anything. Calls share the scratch: calls
 * that overlap on the GPU race and must be serialised by the caller. The
 * first call on each device looks up the scratch's device address (with
 * that device current); make that first call before any stream capture.
 */
int mrn_interp_noalloc(int ndim, const int* grid_size, int n_coil, int64_t n_pts,
                       const double* width, double beta, const void* grid, const float* locs,
                       void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MRNUFFT_H */
