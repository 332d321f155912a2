/*
 * monalisa_gpu.h -- C ABI of libmonalisa_gpu.so, the B200 (sm_100a)
 * implementation of Monalisa's non-Cartesian gridding hot path.
 *
 * Conventions
 *  - Every function returns an int status: MLG_OK (0) or a negative
 *    MLG_ERR_* code.  mlg_last_error() gives a message for the calling
 *    thread's last failure.  Invalid arguments are rejected before any launch.
 *  - Host-buffer entry points ("MEX equivalents") take and return the exact
 *    argument layouts of the reference MEX kernels they replace: MATLAB
 *    column-major arrays, complex values as separate real/imaginary float
 *    arrays, int32 indices, and outputs written into caller-owned buffers.
 *    They are synchronous, like a MEX call.
 *  - Device-resident objects sit behind opaque handles (mlg_matrix_t,
 *    mlg_plan_t).  *_dev entry points take device pointers and a cudaStream_t
 *    (passed as void*, NULL = default stream) and are stream-ordered.  A
 *    handle may be used by one host thread at a time.
 *  - Device data layouts: complex64 = interleaved float2.  Images are
 *    [prod(n_u)] with x fastest (MATLAB column order).  Gridded data on the
 *    device are coil-fastest [prod(N_u)][nCh] (one cell's coils adjacent).
 *    k-space data on the device are coil-fastest [nPt][nCh] ("point
 *    layout").
 *
 * Reference paths in the comments are relative to the Monalisa source tree.
 */
#ifndef MONALISA_GPU_H
#define MONALISA_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* exported even when the library is compiled with -fvisibility=hidden */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define MLG_OK 0
#define MLG_ERR_ARG -1         /* invalid argument (sizes, NULL, bad matrix)   */
#define MLG_ERR_OOM -2         /* device memory could not be obtained           */
#define MLG_ERR_CUDA -3        /* a CUDA / cuFFT call failed                    */
#define MLG_ERR_TIMEOUT -4     /* a bounded device wait gave up                 */
#define MLG_ERR_STATE -5       /* handle used in a wrong state                  */
#define MLG_ERR_UNSUPPORTED -6 /* configuration not implemented                 */
#define MLG_ERR_NO_DEVICE -7   /* no CUDA device visible                        */

#define MLG_KERNEL_GAUSS 0
#define MLG_KERNEL_KAISER 1

typedef struct mlg_matrix_s* mlg_matrix_t;
typedef struct mlg_plan_s* mlg_plan_t;

/* ---- library ------------------------------------------------------------ */
int mlg_version(void);
const char* mlg_status_string(int status);
const char* mlg_last_error(void);
/* Device used by subsequent calls of this host thread (default: current). */
int mlg_set_device(int device);
/* Number of launches of this library's kernels since load (all threads). */
long long mlg_kernel_launch_count(void);

/* ---- adjoint gridding, host buffers (MEX equivalents) ------------------- */

/* Replaces bmGridder_n2u_leight{1,2,3}_mex
 * (src/gridding123/mex/bmGridder_n2u_leight3/bmGridder_n2u_leight3_mex.cpp:39
 * gateway, :116 kernel; leight2 :36/:108; leight1 :34/:100), as called by
 * src/gridding123/m/bmGridder_n2u_leight.m:125-131.
 * aReal/aImag [nCh, nPt]; tx,ty,tz [nPt] 1-based grid coordinates (ty/tz
 * ignored below imDim); Dn [nPt]; out bReal/bImag [nCh, Nx*Ny*Nz].
 * Gaussian window sigma = kernelParam_1; kernelParam_2 is unused, as in the
 * reference. */
int mlg_gridder_n2u_leight(int imDim, const float* aReal, const float* aImag,
                           const float* tx, const float* ty, const float* tz,
                           const float* Dn, int nCh, int nPt, int Nx, int Ny,
                           int Nz, int nWin, float kernelParam_1,
                           float kernelParam_2, float* bReal, float* bImag);

/* The gridder of mlg_gridder_n2u_leight for callers that cannot allocate
 * device memory while they run: a program that reserved the GPU's memory for
 * its own pool at start-up (an allocation would fail, or take memory the
 * pool counts on), or an embedding that forbids allocation after
 * initialisation.  No counterpart in the reference: it is an addition of
 * this library.
 *  - Inputs and outputs are device pointers owned by the caller, in the same
 *    layouts as mlg_gridder_n2u_leight: aReal/aImag [nCh, nPt], tx/ty/tz/Dn
 *    [nPt], bReal/bImag [nCh, Nx*Ny*Nz].  Work is ordered on `stream`
 *    (NULL = default stream).
 *  - The call waits on the host once: after its counting kernels it
 *    synchronises `stream` (so it also waits for all work queued there
 *    before it) and reads seven bin totals into host memory, then queues the
 *    gridding kernels and returns; the outputs are ready when the stream
 *    reaches that point.
 *  - Nothing is allocated: all scratch comes from one fixed 32 MiB array in
 *    device memory that every GPU loading the library holds until exit.  A
 *    problem whose counters or bins do not fit, or whose (tile, sample)
 *    pairs could exceed 2^31 - 1, is rejected with MLG_ERR_ARG and a message
 *    giving the bytes or pairs it would need, before anything is launched.
 *  - The first call on a device does the set-up: it looks up the array's
 *    device address and loads the gridding kernels (under CUDA's lazy module
 *    loading the array and the kernels take their device memory then).  Make
 *    that first call before any stream capture, and before reserving the
 *    GPU's memory for a pool (or set CUDA_MODULE_LOADING=EAGER).
 *  - All calls share the array, which keeps the last call's contents: calls
 *    that overlap on the GPU (other threads, other streams) race.  Each call
 *    clears the counters it relies on. */
int mlg_gridder_n2u_leight_noalloc(int imDim, const float* aReal,
                                   const float* aImag, const float* tx,
                                   const float* ty, const float* tz,
                                   const float* Dn, int nCh, int nPt, int Nx,
                                   int Ny, int Nz, int nWin,
                                   float kernelParam_1, float kernelParam_2,
                                   float* bReal, float* bImag, void* stream);

/* Replaces bmGridder_n2u_mex
 * (src/gridding123/mex/bmGridder_n2u/bmGridder_n2u_mex.cpp:23 gateway, :72
 * kernel), as called by src/gridding123/m/bmGridder_n2u.m:203.
 * w [nNb*nPt] weights; nJump [nNb*nPt] jump-coded 0-based target cells (first
 * entry absolute); out [nCh, Nu_tot]. */
int mlg_gridder_n2u(const float* aReal, const float* aImag, const float* w,
                    const int* nJump, int nCh, int nNb, int nPt, int Nu_tot,
                    float* bReal, float* bImag);

/* ---- sparse gridding matrices ------------------------------------------- */

/* Replaces bmSparseMat_cC_oBlock_omp_mex / bmSparseMat_cC_oBlock_mex
 * (src/sparseMat/mex/bmSparseMat_vec/bmSparseMat_cC_oBlock_omp/
 * bmSparseMat_cC_oBlock_omp_mex.cpp:26 gateway, :106 kernel), as dispatched
 * by src/sparseMat/m/bmSparseMat_vec.m:183-240.
 * The matrix is the cpp_prepared 'one_block' jump format of
 * src/sparseMat/m/bmSparseMat.m:100-188; l_jump == NULL means no row
 * squeezing.  v [r_size, nVec] -> w [l_size, nVec] (column layout). */
int mlg_sparsemat_vec_cC(int r_size, const int* r_jump, const int* r_nJump,
                         const float* m_val, int l_size, const int* l_jump,
                         int l_nJump, const float* vReal, const float* vImag,
                         int nVec, float* wReal, float* wImag);

/* Replaces bmSparseMat_cR_oBlock_mex (…/bmSparseMat_cR_oBlock_mex.cpp:14
 * gateway, :82 kernel): row layout v [nVec, r_size] -> w [nVec, l_size]. */
int mlg_sparsemat_vec_cR(int r_size, const int* r_jump, const int* r_nJump,
                         const float* m_val, int l_size, const int* l_jump,
                         int l_nJump, const float* vReal, const float* vImag,
                         int nVec, float* wReal, float* wImag);

/* Replaces bmSparseMat_rC_oBlock(_omp)_mex (…/bmSparseMat_rC_oBlock_mex.cpp):
 * real column layout. */
int mlg_sparsemat_vec_rC(int r_size, const int* r_jump, const int* r_nJump,
                         const float* m_val, int l_size, const int* l_jump,
                         int l_nJump, const float* v, int nVec, float* w);

/* Replaces bmSparseMat_rR_oBlock_mex
 * (…/bmSparseMat_rR_oBlock/bmSparseMat_rR_oBlock_mex.cpp:13 gateway): real
 * row layout v [nVec, r_size] -> w [nVec, l_size]. */
int mlg_sparsemat_vec_rR(int r_size, const int* r_jump, const int* r_nJump,
                         const float* m_val, int l_size, const int* l_jump,
                         int l_nJump, const float* v, int nVec, float* w);

/* Every product of src/sparseMat/m/bmSparseMat_vec.m:120-240 in one entry
 * point: layout MLG_LAYOUT_CC (complex, column layout v [r_size, nVec], split
 * real/imaginary), _CR (complex row layout [nVec, r_size]), _RC (real
 * column), _RR (real row).  nBlock = 0: the one-block jump format; nBlock >
 * 0: the multi-block format of bmSparseMat.m:100-188 (running sums restart
 * at every block; block_length, l_block_start [nBlock] int32,
 * m_block_start [nBlock] int64), as the *_nBlock_omp_mex kernels read it
 * (…/bmSparseMat_cR_nBlock_omp_mex.cpp:19-95, bmSparseMat_rR_nBlock_omp_mex.cpp:20-85).
 * vI / wI are ignored for the real layouts. */
#define MLG_LAYOUT_CC 0
#define MLG_LAYOUT_CR 1
#define MLG_LAYOUT_RC 2
#define MLG_LAYOUT_RR 3
int mlg_sparsemat_vec(int layout, int r_size, const int* r_jump,
                      const int* r_nJump, const float* m_val, int l_size,
                      const int* l_jump, int l_nJump, int nBlock,
                      const int* block_length, const int* l_block_start,
                      const long long* m_block_start, const float* vR,
                      const float* vI, int nVec, float* wR, float* wI);

/* Replaces bmSparseMat_r_nJump2index_mex
 * (…/bmSparseMat_r_nJump2index/bmSparseMat_r_nJump2index_mex.cpp:12,70):
 * out[out_length] = 0-based row index of every stored entry. */
int mlg_sparsemat_r_nJump2index(int l_size, const int* r_nJump,
                                long long out_length, int* out);

/* Uploads a cpp_prepared bmSparseMat (host arrays, jump format of
 * bmSparseMat.m:100-188) to the device as absolute-index CSR with a dense
 * row pointer over l_size.  Column and row indices are validated. */
int mlg_matrix_create(int r_size, const int* r_jump, const int* r_nJump,
                      const float* m_val, int l_size, const int* l_jump,
                      int l_nJump, mlg_matrix_t* out);
/* Same for a matrix prepared with argMode 'multi_block' (block arrays as for
 * mlg_sparsemat_vec; nBlock = 0 is mlg_matrix_create). */
int mlg_matrix_create_blocks(int r_size, const int* r_jump, const int* r_nJump,
                             const float* m_val, int l_size, const int* l_jump,
                             int l_nJump, int nBlock, const int* block_length,
                             const int* l_block_start,
                             const long long* m_block_start, mlg_matrix_t* out);
int mlg_matrix_destroy(mlg_matrix_t m);
int mlg_matrix_info(mlg_matrix_t m, long long* nnz, int* r_size, int* l_size);
/* Rows holding at least one entry, and rows handled by the split long-row
 * kernel (more than 256 entries). */
int mlg_matrix_row_stats(mlg_matrix_t m, int* nonempty_rows, int* long_rows);
/* Downloads the matrix back to jump format (sizes from mlg_matrix_info;
 * l_nJump_out receives the number of non-empty rows written to r_nJump). */
int mlg_matrix_download(mlg_matrix_t m, int* r_jump, int* r_nJump,
                        float* m_val, int* l_jump, int* l_nJump_out);

/* w = M v on the device, complex64 point layout: v [r_size][nVec],
 * w [l_size][nVec]. */
int mlg_matrix_spmm_dev(mlg_matrix_t m, const void* v, int nVec, void* w,
                        void* stream);

/* GPU form of src/gridding123/m/bmTraj2SparseMat.m:12-314 (Gu and Gut):
 * t [imDim, nPt] (column-major, physical units), ve [nPt], N_u [imDim],
 * dK_u [imDim]; kernelType MLG_KERNEL_GAUSS (params sigma, K_max) or
 * MLG_KERNEL_KAISER (tau, alpha, K_max).  Rows normalised to sum 1, periodic
 * wrap, samples outside the grid keep empty rows; Gut = Gu^T with empty rows
 * squeezed.  Either output pointer may be NULL. */
int mlg_traj2sparsemat(int imDim, int nPt, const double* t, const double* ve,
                       const int* N_u, const double* dK_u, int kernelType,
                       int nWin, const double* kernelParam, mlg_matrix_t* Gu,
                       mlg_matrix_t* Gut);
/* The three-output form [Gn, Gu, Gut] = bmTraj2SparseMat(...) (nargout 3,
 * bmTraj2SparseMat.m:245-297).  Gn [prod(N_u), nPt]: weight * Dn with Dn =
 * ve / prod(dK_u), rows (grid cells) normalised to sum 1, empty rows
 * squeezed, entries of a row in ascending sample order.  Any output pointer
 * may be NULL; ve is needed for Gn. */
int mlg_traj2sparsemat3(int imDim, int nPt, const double* t, const double* ve,
                        const int* N_u, const double* dK_u, int kernelType,
                        int nWin, const double* kernelParam, mlg_matrix_t* Gn,
                        mlg_matrix_t* Gu, mlg_matrix_t* Gut);

/* GPU form of src/gridding123/m/bmImDeformField2SparseMat.m:14-146 (weights
 * of bmImDeformField2sparseMat_ind_weight.m): the image-deformation matrices
 * of a displacement field v [imDim, prod(N_u)] (column-major, pixel units;
 * pixel p moves to its 1-based position + v(:, p)).  Each pixel's row holds
 * the bump weights exp(-1/(1-d^2)) (d < 1) of the 2^imDim cells
 * floor(t) + {0, 1}, periodic wrap, normalised to sum 1; a pixel moved
 * outside [1, N_u] keeps an empty row unless torus_flag.  Gu [prod(N_u),
 * prod(N_u)] (the Tu of bmTevaMorphosia_chain), Gut = Gu^T (Tut), Gn:
 * weight * Dn per cell, rows normalised (needs Dn [prod(N_u)]).  Any output
 * pointer may be NULL. */
int mlg_deform2sparsemat(int imDim, const int* N_u, const double* v,
                         const double* Dn, int torus_flag, mlg_matrix_t* Gn,
                         mlg_matrix_t* Gu, mlg_matrix_t* Gut);

/* ---- deapodisation ------------------------------------------------------ */

/* src/fourier123/prep_function/bmK.m:6-156 for one coil: K [prod(N_u)]
 * (column order), computed in FP64 and rounded to single. */
int mlg_deapodization(int imDim, const int* N_u, const double* dK_u,
                      int kernelType, int nWin, const double* kernelParam,
                      float* K);
/* The same K computed on the device (K: device buffer of prod(N_u) floats),
 * bit-identical to mlg_deapodization; stream-ordered, returns after the
 * kernels finished.  (No reference counterpart: a device form of bmK.) */
int mlg_deapodization_dev(int imDim, const int* N_u, const double* dK_u,
                          int kernelType, int nWin,
                          const double* kernelParam, float* K, void* stream);

/* ---- volume elements ---------------------------------------------------- */

/* Volume elements of a full radial trajectory on the device, FP64:
 * imDim 3 as src/geom3/bmVolumeElement_full_radial3.m, imDim 2 as
 * src/geom2/bmVolumeElement_voronoi_full_radial2.m.  t: device
 * [imDim][nPt] (row-major), lines of N samples (line l = samples l*N ..
 * l*N+N-1, through the centre at sample N/2); v: device [nPt].  Radial
 * lengths are the 1-D Voronoi lengths along each line in the first line's
 * order (bmVolumeElement1); the centre samples share one ball (3-D) or disc
 * (2-D) element.  Stream-ordered. */
int mlg_volume_element_radial_dev(int imDim, int nPt, int N, const double* t,
                                  double* v, void* stream);

/* ---- fused operators (NUFFT plan) --------------------------------------- */

/* A plan holds the FFT pass tables, the sign-folded copies of Gu/Gut used by
 * the fused operators, KFC and KFC_conj ([prod(n_u), nCh] column layout, host
 * arrays as produced by src/fourier123/prep_function/bmKF.m and
 * bmKF_conj.m) and work buffers.  N_u and n_u must be even; n_u <= N_u.
 * Gu / Gut stay owned by the caller and must outlive the plan. */
int mlg_plan_create(int imDim, const int* N_u, const int* n_u, int nCh,
                    mlg_matrix_t Gu, mlg_matrix_t Gut, const float* KFC_re,
                    const float* KFC_im, const float* KFCc_re,
                    const float* KFCc_im, mlg_plan_t* out);
/* MLG_ERR_STATE while plans created by mlg_plan_create_sharing borrow from p. */
int mlg_plan_destroy(mlg_plan_t p);
/* A plan over other matrices on base's grid (another frame bin or another
 * trajectory with the same N_u, n_u, coils and KFC): it borrows base's KFC,
 * KFC_conj, grid buffers, FFT tables, dK_u and stream, so its operators run
 * in the order of base's stream and it costs only the matrices'
 * sign-folded copies.  The frame bins of bmTevaMorphosia_chain.m:56-57 all
 * use one KFC.  No reference counterpart (the reference recomputes its FFT
 * buffers per call). */
int mlg_plan_create_sharing(mlg_plan_t base, mlg_matrix_t Gu, mlg_matrix_t Gut,
                            mlg_plan_t* out);
/* k-space grid step dK_u [imDim] (default 1): sets the image-space volume
 * element HX = prod((1/dK_u)/N_u) used by the solvers
 * (src/fourier123/solver_function/imDim/nonCartesian/bmSensa.m:26-27). */
int mlg_plan_set_dk(mlg_plan_t p, const double* dK_u);
/* Device bytes held by the plan (excluding the caller's matrices). */
int mlg_plan_device_bytes(mlg_plan_t p, long long* bytes);

/* Synchronises the plan's stream and reports whether a bounded wait inside
 * one of its device passes ran out since the last check (MLG_ERR_TIMEOUT;
 * the results of that work are invalid) -- MLG_OK otherwise.  The flag is
 * one per device and is cleared by the check; the synchronous host-buffer
 * calls check it themselves.  No counterpart in the reference: the
 * reference has no device code. */
int mlg_plan_status(mlg_plan_t p);

/* bmShanna (src/fourier123/map_function/nonCartesian/bmShanna_MATLAB.m:6-56)
 * on device buffers: x [prod(n_u)] (or [prod(n_u)][nCh], coil fastest, if
 * x_per_coil) -> y [nPt][nCh]. */
int mlg_shanna_dev(mlg_plan_t p, const void* x, int x_per_coil, void* y,
                   void* stream);
/* bmNakatsha with C_flag = true (bmNakatsha_MATLAB.m:6-58): y [nPt][nCh] ->
 * x [prod(n_u)] (coil-summed).  Optional row weights HY [nPt] (NULL = 1) are
 * applied to y first and the result is multiplied by `scale`. */
int mlg_nakatsha_dev(mlg_plan_t p, const void* y, const float* HY, float scale,
                     void* x, void* stream);

/* Host-buffer fused operators with the argument layouts fixed by the
 * reference's call sites of its (absent) CUFFT MEX files:
 * bmShanna{1,2,3}_CUFFT_omp_mex
 * (src/fourier123/map_function/nonCartesian/bmShanna_CUFFT_omp.m:15-35) and
 * bmNakatsha{1,2,3}_CUFFT_omp_mex (…/bmNakatsha_CUFFT_omp.m:17-36).
 * x [prod(n_u), x_nCol] with x_nCol = 1 or nCh, KFC [prod(n_u), nCh],
 * y [nPt, nCh]; G is the cpp_prepared jump format.  n_u == NULL means
 * n_u = N_u (the reference's only supported case); otherwise zero-filling and
 * cropping are fused. */
int mlg_shanna(int imDim, const int* N_u, const int* n_u, int nCh,
               const float* xR, const float* xI, int x_nCol,
               const float* KFC_R, const float* KFC_I, int r_size,
               const int* r_jump, const int* r_nJump, const float* m_val,
               int l_size, const int* l_jump, int l_nJump, float* yR,
               float* yI);
int mlg_nakatsha(int imDim, const int* N_u, const int* n_u, int nCh,
                 const float* yR, const float* yI, const float* KFCc_R,
                 const float* KFCc_I, int r_size, const int* r_jump,
                 const int* r_nJump, const float* m_val, int l_size,
                 const int* l_jump, int l_nJump, float* xR, float* xI);

/* bmIDF{1,2,3}_CUFFT_mex (called at
 * src/fourier123/map_function/nonCartesian/bmMathilda.m:85-102):
 * fftshift(ifft(ifftshift(x))) * prod(N_u)*prod(dK_u) over the first imDim
 * dimensions of x [N_u..., nCol]. */
int mlg_idf(int imDim, const int* N_u, const float* dK_u, int nCol,
            const float* xR, const float* xI, float* yR, float* yI);

/* How the adjoint (Nakatsha) feeds its first inverse FFT pass with the Gut
 * product: MLG_ADJ_FULL_GRID writes every grid cell and streams the grid;
 * MLG_ADJ_FUSED gathers the Gut rows inside the pass (2-D/3-D);
 * MLG_ADJ_MASKED writes only the non-empty Gut rows and reads a cell only if
 * its occupancy bit is set (even nCh).  All give the same values up to
 * floating-point summation order of the long rows.  Tuning API; no reference
 * counterpart. */
#define MLG_ADJ_FULL_GRID 0
#define MLG_ADJ_FUSED 1
#define MLG_ADJ_MASKED 2
int mlg_plan_set_adjoint(mlg_plan_t p, int mode);
int mlg_plan_get_adjoint(mlg_plan_t p, int* mode);
/* Autotuner: times every valid adjoint strategy on the plan's own matrices
 * (`reps` runs each after a warm-up, CUDA events on the plan's stream) and
 * keeps the fastest.  ms (may be NULL) receives 3 times in milliseconds,
 * negative for strategies the plan cannot run. */
int mlg_plan_autotune(mlg_plan_t p, int reps, double* ms);
/* Kernel variants of a plan, with different launch shapes, that compute the
 * same values bit for bit: pass_buffers = 2 or 3 moves the line-FFT bundles
 * with the TMA unit (a producer warp and that many bundle buffers per CTA:
 * 3 CTAs per SM with 2 buffers, 2 with 3, at 256-point lines of 16 coils),
 * 0 with per-thread cp.async copies; gut_records = 1 reads Gut's short rows
 * from 32-byte row records (masked adjoint, even coil count), 0 from the
 * CSR; fwd_masked_store = 1 lets the last forward TMA pass store only the
 * 32-row chunks of grid lines that hold cells Gu reads (the grid's other
 * cells then keep stale values, which no operator reads; allowed when every
 * Gu column is an occupied cell of Gut, checked at plan creation), 0 stores
 * the whole grid.  Defaults: 2 buffers, records where built, masked stores
 * where allowed.  Set them before a chain is created over the plan.
 * mlg_plan_autotune_variants times them for the plan's adjoint strategy and
 * keeps the fastest: ms[6] (may be NULL) = forward + adjoint with 2 / 3
 * buffers and with cp.async passes, adjoint with CSR / record Gut rows,
 * forward + adjoint storing the whole grid at the chosen buffer count (-1:
 * not timed).  No counterpart in the reference (its kernels are CPU code). */
int mlg_plan_set_variant(mlg_plan_t p, int pass_buffers, int gut_records, int fwd_masked_store);
int mlg_plan_get_variant(mlg_plan_t p, int* pass_buffers, int* gut_records, int* fwd_masked_store);
int mlg_plan_autotune_variants(mlg_plan_t p, int reps, double* ms);

/* Precision of the plan's CG-SENSE solver (mlg_sensa_dev / mlg_sensa).
 * MLG_PRECISION_FP32: FP32 data and matrix values, FP64 scalars (the
 * reference's single-precision arithmetic).  MLG_PRECISION_MIXED: FP16 matrix
 * values (copies of Gu/Gut made once) and, where the plan's passes support
 * it (mlg_plan_get_half_intermediate), 16-bit storage of the 3-D
 * transforms' intermediate and of the forward grid inside the CG steps (FP16
 * times a power of two bounding it from the forward x pass's or the Gut
 * product's largest value); FP32 k-space vectors (M p and
 * the residual), FP32 sums and FFT arithmetic, FP64 scalars; the caller's y
 * and x stay complex64.  Mixed precision turns the fused-gather adjoint
 * strategy off (it reads FP32 k-space).  The operator entry points
 * (mlg_shanna_dev, mlg_nakatsha_dev) of a mixed plan read the FP16 values
 * but keep their complex64 k-space buffers.  No reference counterpart. */
#define MLG_PRECISION_FP32 0
#define MLG_PRECISION_MIXED 1
/* FP16 matrix values only; the k-space work vectors stay FP32. */
#define MLG_PRECISION_FP16_VALUES 2
int mlg_plan_set_precision(mlg_plan_t p, int precision);
int mlg_plan_get_precision(mlg_plan_t p, int* precision);
/* *on != 0 when a mixed solve of this plan keeps the intermediate of its
 * 3-D transforms (after the forward y pass, after the adjoint z pass) in
 * scaled FP16 inside the CG steps: MLG_PRECISION_MIXED, 3-D, a multiple of 4
 * coils, no fused adjoint gather, and TMA line passes for those shapes (bit
 * 0); bit 1 set when the forward grid is stored in scaled FP16 as well (the
 * last forward pass writes it, Gu's gathers read it: even coil count, no Gu
 * row longer than 256 entries); 0 otherwise.  No reference counterpart. */
int mlg_plan_get_half_intermediate(mlg_plan_t p, int* on);

/* Times the stages of one Shanna and one Nakatsha on the plan's stream with
 * CUDA events, averaged over `iters` repetitions after one warm-up:
 * ms[0..2] forward x, y, z FFT passes (x pass fused with x .* KFC),
 * ms[3] Gu product, ms[4] Gut product, ms[5..7] inverse z, y, x FFT passes
 * (x pass fused with .* KFC_conj and the coil sum).  Passes a 2-D / 1-D
 * plan does not run read 0.  A mixed-precision plan's stages run as inside
 * its CG steps (the FP16 transform intermediate where
 * mlg_plan_get_half_intermediate says so).  Inputs are zeros.  Measurement
 * helper; no reference counterpart. */
int mlg_plan_profile(mlg_plan_t p, int iters, double* ms);

/* ---- reconstructions ---------------------------------------------------- */

/* bmMathilda-style leight gridding on device buffers (stream-ordered): the
 * arguments of mlg_gridder_n2u_leight with aReal/aImag [nPt][nCh],
 * tx/ty/tz/Dn [nPt], bReal/bImag [prod(N)][nCh] device pointers; scratch
 * from the library's stream-ordered pool.  No reference counterpart (the
 * reference's gridder takes MATLAB arrays). */
int mlg_gridder_n2u_leight_dev(int imDim, const float* aReal, const float* aImag,
                               const float* tx, const float* ty, const float* tz,
                               const float* Dn, int nCh, int nPt, int Nx, int Ny,
                               int Nz, int nWin, float kernelParam_1,
                               float kernelParam_2, float* bReal, float* bImag,
                               void* stream);

/* The tail of the gridded reconstructions bmMathilda.m:76-121 and
 * bmNasha.m:48-88 on device buffers:
 *   x = coil_pinv(crop_{n_u}(K .* bmIDF(grid)))
 * grid [prod(N_u)][nCh] point layout: interleaved complex (grid_split = 0,
 * grid_a) or split (grid_split = 1, grid_a = real, grid_b = imaginary
 * parts); K [prod(N_u)] float (mlg_deapodization); C [prod(n_u)][nCh]
 * complex or NULL.  x [prod(n_u)] complex with C, else [nCh][prod(n_u)]
 * (every coil's image, the column layout of [prod(n_u), nCh]).  N_u even. */
int mlg_gridded_tail_dev(int imDim, const int* N_u, const int* n_u,
                         const float* dK_u, int nCh, int grid_split,
                         const void* grid_a, const void* grid_b, const float* K,
                         const void* C, void* x, void* stream);

/* CG-SENSE, src/fourier123/solver_function/imDim/nonCartesian/bmSensa.m:6-96:
 * nIter outer iterations (the convergence condition's iteration cap), each
 * a CG run of at most nCGD x-updates restarted from the current x.
 * y [nPt][nCh] k-space (device, point layout), ve [nPt] (device), ve_max <=
 * 0 means max(ve).  x [prod(n_u)] device image, in: initial guess, out:
 * reconstruction.  residual (host, may be NULL) receives nIter values of
 * ||y - Mx||^2_HY.  Dot products, norms and step sizes are FP64. */
int mlg_sensa_dev(mlg_plan_t p, const void* y, const float* ve, float ve_max,
                  int nIter, int nCGD, void* x, double* residual,
                  void* stream);
/* Same with host buffers in MATLAB layouts: yR/yI [nPt, nCh], ve [nPt],
 * xR/xI [prod(n_u)] in/out.  Copies in and out are part of the call. */
int mlg_sensa(mlg_plan_t p, const float* yR, const float* yI, const float* ve,
              float ve_max, int nIter, int nCGD, float* xR, float* xI,
              double* residual);

/* Frame bins of a temporal reconstruction: one plan per frame (same device,
 * N_u, n_u, nCh; each with Gu and Gut; typically plans 1.. created with
 * mlg_plan_create_sharing from plan 0).  HX comes from plan 0's dK_u.  The
 * chain holds the solver's work arrays over all frames; the plans stay the
 * caller's, must outlive the chain and must not be used while a chain call
 * runs. */
typedef struct mlg_chain_s* mlg_chain_t;
int mlg_chain_create(int nFr, const mlg_plan_t* plans, mlg_chain_t* out);
int mlg_chain_destroy(mlg_chain_t c);
/* nFr, the total k-space rows sum(nPt_f) and the pixels per frame. */
int mlg_chain_info(mlg_chain_t c, int* nFr, long long* rows, long long* pixels);
/* Deformation fields of the temporal sparsifier (the Tu, Tut arguments of
 * bmTevaMorphosia_chain.m, applied as bmImDeform / bmImDeformT with K = []):
 * Tu[f], Tut[f] for f < nFr, each [pixels x pixels] (e.g. from
 * mlg_deform2sparsemat) or NULL (identity for that frame); NULL arrays: no
 * deformation.  F x_f = Tu_f x_f - x_{f-1}, F* z_f = (1/HX)(Tut_f (HZ z_f)
 * - HZ z_{f+1}).  The matrices stay the caller's and must outlive the
 * chain's runs. */
int mlg_chain_set_deform(mlg_chain_t c, const mlg_matrix_t* Tu, const mlg_matrix_t* Tut);

#define MLG_REGUL_NORMAL 0 /* delta, rho from linspace(first, last, nIter) */
#define MLG_REGUL_ADAPT 1  /* delta = factor * regul / dafi, rho = factor * delta */
/* Temporal-TV ADMM,
 * src/fourier123/solver_function/imDim_morphosia/nonCartesian/
 * bmTevaMorphosia_chain.m:6-195, with Tu = Tut = [] (no deformation):
 *   min sum_f 0.5 |y_f - M_f x_f|^2_HY + delta sum_f |x_f - x_{f-1}|_1
 * with circular frame differences.  nIter ADMM iterations, each a CG run of
 * at most nCGD x-updates.  Device buffers: y [sum nPt_f][nCh] (frames in
 * order), ve [sum nPt_f], x, z, u [nFr][prod(n_u)] (x in: initial guess,
 * out: result; z, u in/out, set to F x and 0 first when init_zu).  delta and
 * rho are {first, last} of their per-iteration lists (equal values for a
 * constant).  history (host, may be NULL) receives per iteration
 * {0.5 dafi + 0.5 delta regul, dafi, regul} (:172-178).  Norms and step sizes
 * are FP64. */
int mlg_tevamorphosia_dev(mlg_chain_t c, const void* y, const float* ve,
                          float ve_max, const float* delta, const float* rho,
                          int regul_mode, int nIter, int nCGD, void* x,
                          void* z, void* u, int init_zu, double* history,
                          void* stream);
/* Same with host buffers in MATLAB layouts: y{f} [nPt_f, nCh] column-major,
 * frames concatenated (yR, yI), ve{f} concatenated, x [prod(n_u), nFr]
 * (xR, xI in/out).  z and u start as F x and 0 (the reference's defaults). */
int mlg_tevamorphosia(mlg_chain_t c, const float* yR, const float* yI,
                      const float* ve, float ve_max, const float* delta,
                      const float* rho, int regul_mode, int nIter, int nCGD,
                      float* xR, float* xI, double* history);

/* Spatial-TV ADMM of one image,
 * src/fourier123/solver_function/imDim/nonCartesian/bmSteva.m:6-138, on a
 * chain of one frame:
 *   min 0.5 |y - M x|^2_HY + delta |G x|_1
 * with G the backward gradient along each image axis scaled by 1/dX_u
 * (src/optim/bmBackGradient_n.m).  Device buffers: y [nPt][nCh], ve [nPt],
 * x [prod(n_u)] in/out, z, u [imDim][prod(n_u)] in/out (set to G x and 0
 * first when init_zu).  ve_max <= 0 means max(ve) (bmSteva.m:25-27).
 * delta, rho as for mlg_tevamorphosia_dev.  history (host, may be NULL)
 * receives per iteration {R = |y - Mx|^2_HY, TV = HZ |G x|_1}
 * (bmSteva.m:117-125). */
int mlg_steva_dev(mlg_chain_t c, const void* y, const float* ve, float ve_max,
                  const float* delta, const float* rho, int nIter, int nCGD,
                  void* x, void* z, void* u, int init_zu, double* history,
                  void* stream);
/* Same with host buffers: yR/yI [nPt, nCh] column-major, ve [nPt], xR/xI
 * [prod(n_u)] in/out; z and u start as G x and 0. */
int mlg_steva(mlg_chain_t c, const float* yR, const float* yI, const float* ve,
              float ve_max, const float* delta, const float* rho, int nIter,
              int nCGD, float* xR, float* xI, double* history);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* MONALISA_GPU_H */
