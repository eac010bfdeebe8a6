/*
 * gpawb200.h -- C ABI of libgpawb200.so, the B200 (sm_100a) implementation of
 * GPAW's real-space finite-difference Kohn-Sham hot path.
 *
 * Every entry point:
 *   - takes plain pointers (device pointers for grid data), sizes and an
 *     opaque cudaStream_t passed as void* (NULL = legacy default stream);
 *   - returns an int status: GB_OK (0) or a negative GB_E* code, with a
 *     message available from gb_last_error() (per host thread);
 *   - never allocates its outputs: callers own every input/output buffer
 *     (the reference's ownership rule, c/_gpaw.h objects borrow caller arrays).
 *
 * Grid arrays are C-contiguous (nbatch, n0, n1, n2) of one of the GB_DTYPE_*
 * element types; complex arrays are interleaved (re, im).
 *
 * Each declaration cites the reference interface it replaces
 * (path:line inside the GPAW source tree).
 */
#ifndef GPAWB200_H
#define GPAWB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GB_OK               0
#define GB_E_INVALID       -1   /* bad argument: shape, dtype, null pointer   */
#define GB_E_UNSUPPORTED   -2   /* valid request this build does not handle   */
#define GB_E_CUDA          -3   /* CUDA runtime/launch error                  */
#define GB_E_NOMEM         -4   /* host/device allocation for an object failed */
#define GB_E_TIMEOUT       -5   /* a bounded device-side wait gave up          */

/* ---- element types ----------------------------------------------------- */
#define GB_DTYPE_F64   0   /* double                        (numpy float)      */
#define GB_DTYPE_F32   1   /* float                         (FP32 batched form) */
#define GB_DTYPE_C128  2   /* double complex, interleaved   (numpy complex)    */
#define GB_DTYPE_C64   3   /* float complex, interleaved                      */

/* Message for the last failing call on this host thread ("" if none). */
const char* gb_last_error(void);
/* Library version string. */
const char* gb_version(void);
/* Number of SMs of the current device (used by the host-side autotuner). */
int gb_device_sm_count(int* sm_count);

/* ======================================================================
 * FD operator (stencil)  -- replaces _gpaw.Operator
 *   reference: c/operators.c:384-425 (NewOperatorObject),
 *              c/operators.c:250-321 (Operator_apply),
 *              c/operators.c:324-337 (get_diagonal_element),
 *              c/bmgs/fd.c:9-33 (bmgs_fd), c/bc.c:146-308 (halo / BCs)
 * ==================================================================== */
typedef struct gb_operator gb_operator;

/* coef_p[np], offset_p[np]: linear offsets in the array padded by `range`
 * on each side (offset = o0*M1*M2 + o1*M2 + o2, M = n + 2*range), exactly
 * as gpaw/fd_operators.py:55-57 builds them.  neighbor_cd[3][2]: -1 = zero
 * boundary on that side, >= 0 = periodic (single domain).  `real` selects
 * float vs complex data; `cfd` is the reference's central-FD flag (all
 * offsets on the axes). */
int gb_operator_new(const double* coef_p, const int64_t* offset_p, int np,
                    const int64_t size_c[3], int range,
                    const int64_t neighbor_cd[6], int real, int cfd,
                    gb_operator** out);
/* out = stencil(in) for nin stacked grids.  phase_cd: 3x2 complex Bloch
 * phases as 12 doubles (re, im), required for complex dtypes, ignored for
 * real ones (c/operators.c:270-273). */
int gb_operator_apply(const gb_operator* op, const void* in, void* out,
                      int64_t nin, int dtype, const double* phase_cd,
                      void* stream);
/* out = op(in) + vt * in for nin stacked grids: the local part of the
 * pseudo-Hamiltonian (kinetic stencil plus local potential) in one pass.
 * vt is one real grid of the operator's shape (device memory, FP64 for
 * f64/c128 data, FP32 for f32/c64), shared by all grids.  No single
 * counterpart: fuses Operator.apply with the potential multiply of
 * gpaw/wavefunctions/fd.py:82-88 / gpaw/hamiltonian.py:437-443. */
int gb_operator_apply_potential(const gb_operator* op, const void* in,
                                void* out, int64_t nin, int dtype,
                                const void* vt, const double* phase_cd,
                                void* stream);
/* Weighted-Jacobi relaxation sweeps (relax_method 2) used by the FD Poisson
 * solver: c/operators.c:55-97, c/bmgs/relax.c:7-66.  Real FP64 only. */
/* A batch of nk k-points in one launch: the nin grids are nk equal groups of
 * bands (k-point major), group k taking the Bloch phases
 * phase_kcd[k * 12 .. k * 12 + 11] (the (3, 2) complex phase_cd of that
 * k-point, re/im interleaved); vt (optional, NULL for none) adds the local
 * potential as gb_operator_apply_potential does.  nk <= 8.  This is the
 * loop over kpt_u of gpaw/eigensolvers/eigensolver.py:136-144 folded into
 * the launch; it has no single counterpart in the reference. */
int gb_operator_apply_k(const gb_operator* op, const void* in, void* out,
                        int64_t nin, int dtype, int nk,
                        const double* phase_kcd, const void* vt, void* stream);

int gb_operator_relax(const gb_operator* op, int relax_method, double* f_g,
                      const double* s_g, int nrelax, double w, void* stream);
int gb_operator_get_diagonal_element(const gb_operator* op, double* d);
/* Stencil kernel selection (no reference counterpart; for tests and
 * benchmarks): 0 = automatic (TMA pipeline where the layout allows it,
 * cp.async kernel otherwise), 1 = cp.async kernel only, 2 = TMA required. */
int gb_set_stencil_path(int mode);
/* Device-side error code left by a bounded wait that gave up (0 = none);
 * clear != 0 resets it. */
int gb_device_errors(int clear, int* code);
int gb_operator_free(gb_operator* op);

/* ======================================================================
 * Transformer (restriction / interpolation)  -- replaces _gpaw.Transformer
 *   reference: c/transformers.c:202-252 (NewTransformerObject),
 *              c/transformers.c:44-164 (apply), c/bmgs/restrict.c:136-155,
 *              c/bmgs/interpolate.c:227-257, gpaw/transformers.py:27-77
 * ==================================================================== */
typedef struct gb_transformer gb_transformer;

/* Arguments as in gpaw/transformers.py:71-77: size_in/size_out = gdin.n_c /
 * gdout.n_c, k = 2*nn (2, 4, 6, 8), pad_cd/npad_cd/skip_cd [3][2],
 * neighbor_cd [3][2] of the input grid, interpolate = 0 (restrict) / 1. */
int gb_transformer_new(const int64_t size_in[3], const int64_t size_out[3],
                       int k, const int64_t pad_cd[6], const int64_t npad_cd[6],
                       const int64_t skip_cd[6], const int64_t neighbor_cd[6],
                       int real, int interpolate, gb_transformer** out);
int gb_transformer_apply(const gb_transformer* t, const void* in, void* out,
                         int64_t nin, int dtype, const double* phase_cd,
                         void* stream);
/* out = alpha * T(in) (+ gamma * y for an interpolation, y shaped like out):
 * the same transfer with a fused scale and addend (no reference counterpart;
 * the V-cycle's own kernels and the learned preconditioner's skip
 * connection use it). */
int gb_transformer_apply_axpy(const gb_transformer* t, const void* in,
                              void* out, int64_t nin, int dtype,
                              const double* phase_cd, double alpha,
                              const void* y, double gamma, void* stream);
/* nk k-point groups of bands in one launch, phases as gb_operator_apply_k */
int gb_transformer_apply_k(const gb_transformer* t, const void* in, void* out,
                           int64_t nin, int dtype, int nk,
                           const double* phase_kcd, void* stream);
int gb_transformer_free(gb_transformer* t);

/* ======================================================================
 * Multigrid preconditioner V-cycle  -- replaces _gpaw.fd_precond
 *   reference: c/fd_preconditioner.c:108-353, gpaw/preconditioner.py:59-93
 * Work arrays as in the reference: d0,q0 (nin, level-0 grid); r1,d1,q1
 * (nin, level-1); r2,d2,q2 (nin, level-2).  The result is written to d0.
 * nresiduals may be NULL (the negation is done on the fly).
 * ==================================================================== */
int gb_fd_precond(const gb_transformer* rest0, const gb_transformer* rest1,
                  const gb_transformer* intp1, const gb_transformer* intp2,
                  const gb_operator* kin0, const gb_operator* kin1,
                  const gb_operator* kin2,
                  void* d0, void* q0, void* r1, void* d1, void* q1,
                  void* r2, void* d2, void* q2,
                  const void* residuals, const void* nresiduals,
                  double step, int64_t nin, int dtype,
                  const double* phase_cd, void* stream);

/* The V-cycle for nk k-point groups of bands in one chain of launches,
 * phases as gb_operator_apply_k (work arrays sized for all nin grids). */
int gb_fd_precond_k(const gb_transformer* rest0, const gb_transformer* rest1,
                    const gb_transformer* intp1, const gb_transformer* intp2,
                    const gb_operator* kin0, const gb_operator* kin1,
                    const gb_operator* kin2,
                    void* d0, void* q0, void* r1, void* d1, void* q1,
                    void* r2, void* d2, void* q2,
                    const void* residuals, double step, int64_t nin,
                    int dtype, int nk, const double* phase_kcd, void* stream);

/* The same V-cycle for callers that cannot allocate device memory while
 * they run: a C or Fortran host program that owns only the residual and
 * result buffers it passes in, or a process whose device-memory budget is
 * fixed at start-up.  It has no counterpart in the reference.  The work grids
 * come from one 64 MiB array inside the library (held by every GPU that
 * loads it); a call needing more -- about 1.41 x nin x level-0 points x
 * element size -- fails with GB_E_INVALID.  Nothing is allocated or freed.
 * The first call on a device looks up the array's address: make it before
 * any stream capture.  Under CUDA's lazy module loading (the default) that
 * look-up is also what places the array in device memory, so a caller with
 * a budget fixed at start-up makes one call then: nin = 0 does the look-up
 * and launches nothing.  The address is kept per device and goes stale
 * after cudaDeviceReset: do not call this entry point on that device again.
 * Calls share the array, so calls whose launches can overlap on the GPU
 * race: keep them on one stream.  Result in d0, as gb_fd_precond. */
int gb_fd_precond_noalloc(const gb_transformer* rest0,
                          const gb_transformer* rest1,
                          const gb_transformer* intp1,
                          const gb_transformer* intp2,
                          const gb_operator* kin0, const gb_operator* kin1,
                          const gb_operator* kin2, void* d0,
                          const void* residuals, double step, int64_t nin,
                          int dtype, const double* phase_cd, void* stream);

/* ======================================================================
 * Radial splines and spline_to_grid  -- replace _gpaw.Spline and
 * _gpaw.spline_to_grid
 *   reference: c/spline.c (NewSplineObject), c/bmgs/spline.c:11-75
 *              (natural cubic spline, value and slope), c/lfc.c:887-977
 *              (spline_to_grid), c/bmgs/spherical_harmonics.h:5-48
 *   called from gpaw/spline.py:19-31 and gpaw/lfc.py:94-97 (Sphere)
 * gb_spline_new: f_g holds nbins + 1 host values on r = 0 .. rmax (the
 *   last one is taken as given; Spline.from_data zeroes it); l <= 2.
 * gb_spline_to_grid: f(r) r^l Y_lm on the box beg_c <= g < end_c (global
 *   grid indices) around pos_v (Bohr), h_cv row-major, n_c the local grid
 *   and gdcorner_c its first global index.  Device outputs: A_gm rows for
 *   every point with r < rmax, rows (g0, g1) in order and g2 increasing
 *   within each (capacity: box points x (2l + 1) doubles), and G_B the
 *   [start, end) flat local indices of the runs along g2 (capacity: 2 x box
 *   rows ints).  *ng_out points and *nB_out entries of G_B are written
 *   back (the call waits for its stream).
 * ==================================================================== */
typedef struct gb_spline gb_spline;
int gb_spline_new(int l, double rmax, int nbins, const double* f_g,
                  gb_spline** out);
int gb_spline_free(gb_spline* s);
int gb_spline_get(const gb_spline* s, int* l, double* rmax, int* nbins);
int gb_spline_to_grid(const gb_spline* s, const int64_t beg_c[3],
                      const int64_t end_c[3], const double pos_v[3],
                      const double h_cv[9], const int64_t n_c[3],
                      const int64_t gdcorner_c[3], double* A_gm, int* G_B,
                      int64_t* ng_out, int64_t* nB_out, void* stream);

/* ======================================================================
 * Localized functions (LFC)  -- replaces _gpaw.LFC
 *   reference: c/lfc.c:146-257 (NewLFCObject), c/lfc.c:818-885 (add),
 *              c/lfc.c:432-505 (integrate), c/lfc.h:79-130 (GRID_LOOP),
 *              gpaw/lfc.py:259-374 (_update builds the arguments)
 * The arguments are the reference's, flattened to plain arrays (host
 * memory): the nW volumes' A_gm blocks concatenated row-major in A_all
 * (ngm_W[W] rows of nm_W[W] values each), M_W, the sorted boundary list
 * G_B/W_B (W >= 0 enters volume W, -W-1 leaves it), dv, and phase_qW as
 * nq*nW complex numbers (re, im) (nq = 0: Gamma point / real).  nG is the
 * number of grid points per band, nM the length of c_xM rows.
 * add:       a_xG[x] += sum_W conj(phase_qW) sum_m c_xM[x][M_W+m] A_W
 * integrate: c_xM[x][M_W+m] += dv sum_G phase_qW a_xG[x][G] A_W[g][m]
 *            (accumulates, like the reference; callers zero c_xM)
 * q = -1 for real data / no Bloch phase.  Device arrays for a_xG / c_xM.
 * ==================================================================== */
typedef struct gb_lfc gb_lfc;
int gb_lfc_new(int nW, const double* A_all, const int64_t* ngm_W,
               const int* nm_W, const int* M_W, int nB, const int* G_B,
               const int* W_B, double dv, int nq, const double* phase_qW,
               int64_t nG, int nM, gb_lfc** out);
int gb_lfc_add(const gb_lfc* lfc, const void* c_xM, void* a_xG, int64_t nx,
               int dtype, int q, void* stream);
int gb_lfc_integrate(const gb_lfc* lfc, const void* a_xG, void* c_xM,
                     int64_t nx, int dtype, int q, void* stream);
int gb_lfc_free(gb_lfc* lfc);
/* FP32 real data (q = -1): where every volume has at most 8 functions, nG
 * is a multiple of 4 and no 32-point chunk of the grid meets more than 16
 * function groups, add and integrate run chunk-tiled and keep a work space
 * on the object (nM x 256 floats for add, a few MB of partial sums for
 * integrate).  It grows on the first call of a larger band count, which
 * must not be inside stream capture; calls on one object are ordered on
 * one stream.  gb_lfc_tiled returns 1 when the object has that path (a
 * query of this implementation; no reference counterpart). */
int gb_lfc_tiled(const gb_lfc* lfc);
/* add / integrate over nk k-point groups of the nx rows in one launch:
 * row x takes the Bloch phases of k-point q = x / (nx / nk) (complex
 * dtypes; nk <= nq). */
int gb_lfc_add_k(const gb_lfc* lfc, const void* c_xM, void* a_xG, int64_t nx,
                 int dtype, int nk, void* stream);
int gb_lfc_integrate_k(const gb_lfc* lfc, const void* a_xG, void* c_xM,
                       int64_t nx, int dtype, int nk, void* stream);

/* LFC.derivative (c/lfc.c:1449-1601, called from gpaw/lfc.py:680-682):
 *   c_xMv[x][M][v] += dv sum_G a_xG[x][G] phase_qW d/dr_v Phi_M(r_G - R_W)
 * computed on the fly from the radial splines; arguments as the
 * reference's: h_cv row-major, n_c / beg_c the local grid and its first
 * global index, spline_M one spline per M (each function's spline
 * repeated 2l + 1 times), pos_Wv the centre of every volume the object was
 * built with (nW x 3, Bohr), q the k-point (-1 for real data).  Volumes of
 * at most 16 functions; c_xMv (nx, nM, 3) accumulates like integrate.
 * d/dR = -d/dr is left to the caller, as in the reference. */
int gb_lfc_derivative(const gb_lfc* lfc, const void* a_xG, void* c_xMv,
                      int64_t nx, const double h_cv[9], const int64_t n_c[3],
                      const gb_spline* const* spline_M, const int64_t beg_c[3],
                      const double* pos_Wv, int q, int dtype, void* stream);

/* ======================================================================
 * Exchange-correlation on the grid  -- replaces _gpaw.XCFunctional.calculate
 *   reference: c/xc/xc.c:73-227 (spin-paired / polarised drivers),
 *              c/xc/pbe.c (PBE exchange + PW92/PBE correlation),
 *              c/xc/rpbe.c, gpaw/xc/kernel.py:6-58 (codes)
 * code: -1 LDA, 0 PBE, 1 revPBE, 2 RPBE.  FP64 device arrays of ng points:
 * e_g [ng] (overwritten), n_sg [nspins][ng], v_sg [nspins][ng] (ADDED to,
 * as in the reference), sigma_xg / dedsigma_xg [2*nspins-1][ng] (GGA only;
 * dedsigma overwritten).
 * ==================================================================== */
int gb_xc_calculate(int code, int nspins, int64_t ng, double* e_g,
                    const double* n_sg, double* v_sg, const double* sigma_xg,
                    double* dedsigma_xg, void* stream);

/* ======================================================================
 * Density accumulation  -- replaces _gpaw.add_to_density
 *   reference: c/utilities.c:313- (one band per call),
 *              gpaw/wavefunctions/fd.py:95-100 (the loop over bands)
 * nt_G[G] += sum_n f_n[n] |psit_nG[n][G]|^2 for all nb bands in one launch;
 * f_n (nb doubles) and nt_G (FP64) are device arrays.
 * ==================================================================== */
int gb_add_to_density(int64_t nb, const double* f_n, const void* psit_nG,
                      int dtype, int64_t nG, double* nt_G, void* stream);

/* ======================================================================
 * 3x3x3 convolutions of the learned preconditioner (no reference
 * counterpart: the network stands in for the multigrid V-cycle of
 * c/fd_preconditioner.c inside RMM-DIIS).  x, y: FP32 (nb, C, n0, n1, n2);
 * w: BF16 [cout][cin][27] (offsets o = (k/9-1, (k/3)%3-1, k%3-1)); FP32
 * accumulation; pbc_c: 1 = periodic, 0 = zero padding per axis.
 * forward: y (=|+=) conv(x); backward_weight: dw (FP32) += dL/dw.
 * Channel pairs: (1,1), (1,16), (16,16), (16,1).
 * ==================================================================== */
int gb_conv3d_forward(const float* x, const void* w_bf16, float* y,
                      int64_t nb, int cin, int cout, const int64_t n_c[3],
                      const int pbc_c[3], int accumulate, void* stream);
/* y = conv(x0, w[0][0]) + conv(x1, w[0][1]) for single-channel x0, x1, y
 * (nb, n0, n1, n2) FP32 and BF16 w [1][2][27]: the network's two level-0
 * convolutions in one pass. */
int gb_conv3d_forward_pair(const float* x0, const float* x1, const void* w_bf16,
                           float* y, int64_t nb, const int64_t n_c[3],
                           const int pbc_c[3], void* stream);
/* dw += dL/dw summed in a fixed order (bit-identical on repeats); the
 * per-block partial sums live in stream-ordered memory from a pool of this
 * library that keeps what it frees (GB_E_NOMEM if that allocation fails). */
int gb_conv3d_backward_weight(const float* x, const float* dy, float* dw,
                              int64_t nb, int cin, int cout,
                              const int64_t n_c[3], const int pbc_c[3],
                              void* stream);
/* Folded inference of the (linear) network on periodic grids of even size,
 * FP32, composite weights from the caller:
 *   fine:   y[p] = sum_{|d|<=rh} F[d] xf[p + d]
 *                + sum_{c<cc} sum_{e in {-1,0,1}^3} G[c][(p%2) - 2e + 2] xc[c][p/2 + e]
 *           F: (2rh+1)^3, G: cc x 6^3 ([c][tx][ty][tz]); (rh, cc) in
 *           {(1, 1), (2, 16)}; xc (nb, cc, n/2) per axis; n2 >= 10;
 *           y must not overlap xf or xc (for (2, 16) the fine part is
 *           written first and the coarse part added by a second launch);
 *           an overlapping y is refused with GB_E_INVALID
 *   stride: y[c][I] = sum_{|d|<=2} Q[d][c] x[2I + d], 16 channels out,
 *           Q [125][16], y (nb, 16, n/2) per axis */
int gb_learned_fold_fine(const float* xf, const float* F, int rh, const float* xc,
                         const float* G, int cc, float* y, int64_t nb,
                         const int64_t n_c[3], void* stream);
int gb_learned_fold_stride(const float* x, const float* Q, float* y, int64_t nb,
                           const int64_t n_c[3], void* stream);

/* ======================================================================
 * Per-band inner products of RMM-DIIS -- the gd.integrate(a_nG, b_nG) /
 * np.dot calls of gpaw/eigensolvers/rmmdiis.py:133-145 (<R|R>, <dR|R>,
 * <dR|dR>) and 175-190 (the DIIS matrix <R_i|R_j>), all bands per launch,
 * FP64 accumulation for every storage dtype (no dv factor):
 *   dots: out[n] = Re sum_G conj(a[n*lda + G]) b[n*ldb + G], G < N
 *   gram: out[n][i][j] = Re sum_G conj(X[n*ldn + i*ldi + G]) X[n*ldn + j*ldi + G],
 *         i, j < k <= 5 (band-major or vector-major strides, no overlap)
 * ==================================================================== */
int gb_band_dots(int64_t nb, int64_t N, const void* a, int64_t lda,
                 const void* b, int64_t ldb, int dtype, double* out,
                 void* stream);
int gb_band_gram(int64_t nb, int k, int64_t N, const void* X, int64_t ldn,
                 int64_t ldi, int dtype, double* out, void* stream);
/* ====================================================================
 * Band-space GEMMs of the eigensolver on the tcgen05 tensor cores, FP32
 * wave functions, FP32 accuracy by the three-product TF32 split
 * (x = hi + lo, a b ~ hi hi + hi lo + lo hi).  Replace the GEMMs of
 * gpaw/wavefunctions/fdpw.py:394-424 (overlap + inverse-Cholesky
 * rotation), gpaw/eigensolvers/eigensolver.py:174-236 (H_nn and the
 * subspace rotation) and gpaw/matrix.py:229-260 (the BLAS calls behind
 * them).  Rows are 16-byte aligned (ld % 4 == 0, 16-byte aligned bases);
 * other layouts return GB_E_UNSUPPORTED.
 *   gram:   C[i*ldc + j] = alpha sum_{G<K} A[i*lda + G] B[j*ldb + G]
 *           (FP64 out; `work` of gb_band_gram_tc_workspace bytes holds the
 *           per-CTA FP64 partial sums, combined in a fixed order)
 *   split:  hi/lo TF32 parts (FP32 containers) of an FP64 matrix,
 *           rows x cols, zero-padded to ldd columns
 *   rotate: Y[n*ldy + G] = sum_{k<nk} U[n][k] X[k*ldx + G]
 *                          + beta Z[n*ldz + G]   (Z optional, may be X),
 *           U given as its split parts Uhi/Ulo (nn x nk, leading dim ldu);
 *           Y must not alias X or Z.  FP32 additions in the tensor core
 *           truncate (~1e-6 relative shrink of a 160-term sum): rotating by
 *           U - I with Z = X keeps that bias in the correction only
 * ==================================================================== */
int gb_band_gram_tc_workspace(int64_t na, int64_t nb, int64_t K, int64_t* bytes);
int gb_band_gram_tc(int64_t na, int64_t nb, int64_t K, const float* A, int64_t lda,
                    const float* B, int64_t ldb, double alpha, double* C, int64_t ldc,
                    void* work, int64_t work_bytes, void* stream);
int gb_tf32_split(int64_t rows, int64_t cols, const double* x, int64_t lds,
                  float* hi, float* lo, int64_t ldd, void* stream);
int gb_band_rotate_tc(int64_t nn, int64_t nk, int64_t K, const float* Uhi,
                      const float* Ulo, int64_t ldu, const float* X, int64_t ldx,
                      float beta, const float* Z, int64_t ldz, float* Y, int64_t ldy,
                      void* stream);
/* nb independent n x n FP64 systems A[s] x[s] = b[s] (n <= 8), the DIIS
 * solves of gpaw/eigensolvers/rmmdiis.py:175-190 and of the density mixer
 * (gpaw/mixer.py); partial pivoting; a singular system gives info[s] = 1 and
 * x[s] = 0; no host synchronisation (info may be NULL). */
int gb_small_solve(int64_t nb, int n, const double* A, const double* b,
                   double* x, int* info, void* stream);
/* Per-band linear combinations of RMM-DIIS (gpaw/eigensolvers/rmmdiis.py:
 * 150-200: R -= eps psi, psi += lambda dpsi, the DIIS recombinations):
 * out[n*ldo + G] = sum_{i<k} coef[n*k + i] x[i][n*ldx[i] + G], G < N, k <= 4,
 * coef FP64 on the device; out may be one of the inputs.  x and ldx are host
 * arrays of k entries. */
int gb_band_combine(int64_t nb, int64_t N, int k, const double* coef,
                    const void* const* x, const int64_t* ldx, void* out,
                    int64_t ldo, int dtype, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GPAWB200_H */
