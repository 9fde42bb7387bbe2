/*
 * piro.h -- C ABI of piro_b200, a B200 (sm_100a) implementation of PIRO's
 * sparse finite-difference time-stepping path.
 *
 * Two layers:
 *   1. Kernel entry points on caller-owned device memory (plain pointers and
 *      sizes, asynchronous on the given CUDA stream, which may be NULL for the
 *      legacy default stream).  Each replaces one reference routine, cited as
 *      file:line in the PIRO source tree.
 *   2. A context API (piro_open ... piro_close) mirroring PIRO's operator API
 *      (process::ddt_r / laplacian / gradient / vector, operator&, operator=,
 *      scalarMatrix::Solve, Piro::solve) and its .ini case format; the library
 *      owns all device memory of a context.
 *
 * Conventions, as in the reference: grid sizes nx, ny, nz include one ghost
 * layer per side (src/preprocess.cpp:72-74); the linear index is
 * i = x + y*nx + z*nx*ny (src/mathoperations.cpp:38-40); fields are float[N];
 * a vector field is float[3N] stored x block, y block, z block (src/ic.cpp:84-95);
 * CSR index arrays are int32.
 *
 * Every function returns a status code (PIRO_OK on success); no C++ exception
 * crosses this boundary.  piro_last_error() gives a message for the calling
 * thread's last failure.  Calls on one context are not thread-safe; separate
 * contexts may be used from separate threads.
 */
#ifndef PIRO_H
#define PIRO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PIRO_OK 0
#define PIRO_ERR_ARG 1          /* invalid argument or size                     */
#define PIRO_ERR_CONFIG 2       /* .ini missing a key or holding a bad value     */
#define PIRO_ERR_DATATYPE 3     /* [Solve] Data not supported for this operator  */
#define PIRO_ERR_TABLE_FULL 4   /* hash insert found no free slot (methods.cpp:106-116 exits) */
#define PIRO_ERR_TABLE_SIZE 5   /* hash table size <= 0 (reference formula below N~18.6k only) */
#define PIRO_ERR_CUDA 6         /* a CUDA runtime call failed                    */
#define PIRO_STATUS_STALLED 7   /* iterative solve stopped making progress       */
#define PIRO_ERR_NOT_CONVERGED 8 /* iteration cap reached                        */
#define PIRO_ERR_SCHEME 9       /* TIMESCHEME / SOLVERSCHEME / space scheme unsupported */
#define PIRO_ERR_NOMEM 10       /* device allocation failed                      */
#define PIRO_ERR_STATE 11       /* call out of order (e.g. operator not built)  */
#define PIRO_ERR_ZERO_PIVOT 12  /* elimination without pivoting met a zero pivot */

typedef void *piro_stream_t; /* a cudaStream_t */

const char *piro_status_string(int status);
const char *piro_last_error(void);
/* Version string of the library build. */
const char *piro_version(void);

/* Polls that a bounded device wait makes before it gives up (the grid
 * barriers of piro_be_solve's persistent kernel and of piro_batch_step, the
 * stage waits of piro_stencil_fe_step's staged kernel).  A wait that runs out
 * sets an error flag, every block leaves the kernel, and the call (or
 * piro_stencil_check) returns PIRO_ERR_CUDA; the CUDA context stays usable.
 * Negative restores the built-in bound (about 2 s of polling).  Process-wide,
 * read at each launch.  No counterpart in the reference, which never waits
 * on the device (it blocks on clFinish).  For tests of the failure path. */
int piro_set_wait_limit(long long polls);

/* ========================================================================
 * 1. Kernel entry points (device pointers; asynchronous on `stream`)
 * ======================================================================== */

/* -- assembly ------------------------------------------------------------ */

/* nnz of the 7-point Laplacian, 7N - 2(nx*ny + ny*nz + nx*nz), for every
 * space scheme (the uw/dw duplicates and the 10.0 entries add no entries). */
int piro_laplacian_nnz(int nx, int ny, int nz, int64_t *nnz);

/* CSR Laplacian, bit-exact with CSR::stencils::laplacian_{uw,dw,cd}
 * (src/stencils.cpp:233-429) called from CSR::laplacian
 * (src/operatorlaplacian.cpp:14-63): per row self -6/norm then x-, x+, y-, y+,
 * z-, z+ at +1/norm; scheme 1 (uw) replaces "+" columns by the row, scheme 2
 * (dw) the "-" columns; the first occurrence of each boundary column is 10.0
 * (stencils.cpp:278-291).  norm is the float (l0/(n0-2))^2 of
 * operatorlaplacian.cpp:33.  rowptr[N+1], col/val[nnz]. */
int piro_csr_laplacian(int nx, int ny, int nz, int space_scheme, float norm, int32_t *rowptr, int32_t *col,
                       float *val, piro_stream_t stream);

/* COO Laplacian, bit-exact with COO::stencils::laplacian_* (src/stencils.cpp:572-795)
 * via COO::laplacian (src/operatorlaplacian.cpp:105-153): same entries and
 * order as CSR with an explicit row array. */
int piro_coo_laplacian(int nx, int ny, int nz, int space_scheme, float norm, int32_t *rows, int32_t *col,
                       float *val, piro_stream_t stream);

/* nnz of one gradient matrix: 2N - 2N/n_axis. */
int piro_gradient_nnz(int nx, int ny, int nz, int axis, int64_t *nnz);

/* One CSR gradient matrix (axis 0 x, 1 y, 2 z), bit-exact with
 * CSR::stencils::gradient_{uw,dw,cd}_{x,y,z} (src/stencils.cpp:7-231) via
 * CSR::gradient (src/operatorgradient.cpp:13-117, norm = 2*(l0/(n0-2)), :25). */
int piro_csr_gradient(int nx, int ny, int nz, int space_scheme, int axis, float norm, int32_t *rowptr,
                      int32_t *col, float *val, piro_stream_t stream);
/* Rows row0 .. row0+nrows-1 of one axis's gradient matrix with columns
 * shifted down by col_shift (col_shift <= row0 - nx*ny when row0 > 0): the
 * rows a z-slab owns, with its local column numbering; the entries of each
 * row exactly as piro_csr_gradient gives them. */
int piro_gradient_nnz_rows(int nx, int ny, int nz, int axis, int64_t row0, int64_t nrows, int64_t *nnz);
int piro_csr_gradient_rows(int nx, int ny, int nz, int space_scheme, int axis, float norm, int64_t row0, int64_t nrows,
                           int64_t col_shift, int32_t *rowptr, int32_t *col, float *val, piro_stream_t stream);

/* val[k] *= s[row(k)]: the row scale diag(s)*M that kernelmethods::csrscale
 * (src/kernelcsrgeam.cpp:208-234) intends through SpMDSM.cl:20-31. */
int piro_csr_rowscale(int64_t nrows, const int32_t *rowptr, float *val, const float *s, piro_stream_t stream);

/* -- hash-table (HT) format ---------------------------------------------- */

/* Table size.  policy 0: the reference formula of
 * src/operatorlaplacian.cpp:184-185, (int)(nnz / ((a*N^b + c) * lf)) with
 * float/double arithmetic as written (may be <= 0 above N ~ 18.6k, in which
 * case PIRO_ERR_TABLE_SIZE is returned); policy 1: the smallest prime >=
 * ceil(nnz/lf). */
int piro_ht_table_size(int64_t nnz, int64_t N, int policy, float a, float b, float c, float lf, int64_t *ts);

/* Bytes of device workspace piro_ht_build needs for a table of ts slots. */
int piro_ht_build_workspace(int64_t ts, size_t *bytes);

/* Insert a CSR matrix into an open-addressing table: key = row*N + col (int64;
 * equal to the reference's int32 key while N <= 46340), slot = key % ts,
 * linear probing, a repeated key keeps its first slot and takes the last
 * value.  Slots match the reference's sequential row-major methods::sethash
 * (src/methods.cpp:74-118, src/operatorlaplacian.cpp:190-203) exactly: keys
 * are inserted in parallel with atomicCAS under insertion-time priority (a
 * probe that meets a later-inserted key takes its slot and carries it on),
 * which converges to the first-come-first-served layout whatever the thread
 * interleaving.  keys[ts] get -1 for empty slots.  Returns PIRO_ERR_TABLE_FULL (synchronously checked) when an
 * insert finds no slot. */
int piro_ht_build(int64_t N, const int32_t *rowptr, const int32_t *col, const float *val, int64_t nnz, int64_t ts,
                  int64_t *keys, float *vals, void *work, size_t work_bytes, piro_stream_t stream);

/* -- time-step kernels ---------------------------------------------------- */

/* SpMVCSR.cl:12-39 as launched by kernelsolve::CSR::TIMESCHEME_11
 * (src/kernelprocess.cpp:10-40): for interior rows
 * out[r] = u[r] + sum_k (dt*val[k])*u[col[k]], summed in storage order with
 * no fused multiply-add; boundary rows of out are not written. */
int piro_csr_fe_step(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val, float dt,
                     const float *u, float *out, piro_stream_t stream);
/* One whole forward-Euler step of Solve(): a zero-filled result, the
 * SpMVCSR update of the interior rows, and setBC of the face cells from bc
 * (bc::opencl_setBC; NULL: no [BC], faces stay 0), in one pass.  Face cells
 * are the cells with exactly one coordinate on the boundary, which is the
 * union of bc::initbc's six lists; edges and corners are 0.  Same result bit
 * for bit as memset + piro_csr_fe_step + piro_set_bc. */
int piro_csr_fe_step_bc(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val, float dt,
                        const float *u, const float *bc, float *out, piro_stream_t stream);

/* SpMVCSR_I1.cl:12-36 (backward-Euler residual form): interior rows get
 * out[r] = u[r] - sum_k (dt*val[k])*u[col[k]]; boundary rows untouched. */
int piro_csr_i1(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val, float dt,
                const float *u, float *out, piro_stream_t stream);

/* SpMVCOO.cl:12-24 semantics with a warp-segmented reduction: out[r] =
 * dt * sum of vals*u[cols] over the entries of row r, for every row (rows
 * without entries get dt*0).  rows must be sorted ascending (the Laplacian
 * assembly order); ids outside [0, N) or unsorted rows return PIRO_ERR_ARG
 * (the call synchronizes the stream to read the check).  Summation order
 * differs from the sequential kernel (results agree to FP32 rounding) but is
 * fixed: results do not vary from run to run.  With 16-byte aligned arrays
 * the step is finished inside the reduction (no accumulator pass). */
int piro_coo_spmv(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals, float dt,
                  const float *u, float *out, piro_stream_t stream);

/* kernelsolve::COO::TIMESCHEME_11 (src/kernelprocess.cpp:93-120) fused:
 * out = u + dt*M*u on every row. */
int piro_coo_fe_step(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals, float dt,
                     const float *u, float *out, piro_stream_t stream);
/* COO with a row index, built once per operator: rowstart[r] = the first
 * entry of row r in the row-sorted arrays (int32[N+1]; PIRO_ERR_ARG if rows
 * are not sorted ascending or out of range; workspace >= 4 bytes; the call
 * synchronizes).  piro_coo_step_indexed then computes out = dt*(A u), or
 * u + dt*(A u) with fe = 1, on every row, each row's products summed in
 * storage order: the CSR row loop over cols/vals, without reading rows. */
int piro_coo_row_index(int64_t N, int64_t nnz, const int32_t *rows, int32_t *rowstart, void *work, size_t work_bytes,
                       piro_stream_t stream);
int piro_coo_step_indexed(int64_t N, const int32_t *rowstart, const int32_t *cols, const float *vals, float dt, int fe,
                          const float *u, float *out, piro_stream_t stream);

/* SpMVHT.cl:22-40 semantics: out[r] = dt * sum over present keys (r, c) of
 * H(r,c)*u[c] in ascending c, found by linear-probe lookups of the 7-point
 * stencil's candidate columns of row r (the only columns a Laplacian table
 * holds).  fe != 0 fuses addVectors: out = u + dt*H*u
 * (kernelsolve::HT::TIMESCHEME_11, src/kernelprocess.cpp:68-91). */
int piro_ht_spmv(int nx, int ny, int nz, const int64_t *keys, const float *vals, int64_t ts, float dt, int fe,
                 const float *u, float *out, piro_stream_t stream);
/* The same step with the rows taken in the order of their keys' home slot
 * (i*N + i) mod ts, as piro_ht_row_order gives it (int32 order[N], computed
 * once per table; workspace piro_ht_row_order_workspace bytes): the table is
 * then read as a window moving through it, not at random.  Same results bit
 * for bit (each row's sum is computed the same way). */
int piro_ht_row_order_workspace(int64_t N, int64_t ts, size_t *bytes);
int piro_ht_row_order(int64_t N, int64_t ts, int32_t *order, void *work, size_t work_bytes, piro_stream_t stream);
int piro_ht_spmv_ordered(int nx, int ny, int nz, const int64_t *keys, const float *vals, int64_t ts, float dt, int fe,
                         const int32_t *order, const float *u, float *out, piro_stream_t stream);
/* The same step in two passes over a caller-owned stage of
 * piro_ht_stage_bytes(N) bytes (32 per row, 16-byte aligned): the table is
 * read in home-slot order as above and each row's seven stencil values land
 * in a 32-byte record, then the rows are applied in index order, so that u
 * and out are read and written coalesced instead of at the scattered
 * home-slot rows.  Same results bit for bit; N < 2^31. */
int piro_ht_stage_bytes(int64_t N, size_t *bytes);
int piro_ht_spmv_staged(int nx, int ny, int nz, const int64_t *keys, const float *vals, int64_t ts, float dt, int fe,
                        const int32_t *order, void *stage, size_t stage_bytes, const float *u, float *out,
                        piro_stream_t stream);

/* Scheme 27 (TIMESCHEME 12 + solver 27) on a table built by piro_ht_build
 * (int64 keys, -1 empty; -2 marks a deleted key).  piro_ht_lu_reference is
 * PIRO's factorization (src/matrixoperations.cpp:10-104, lu_decompHT.cl) in
 * place, resident on the device: per pivot row the fill-in (explicit zeros
 * inserted in the reference's order) and the elimination round, with entries
 * below 1e-6 deleted -- the multipliers included, so no solve follows, as in
 * the reference.  Each round's items read the pre-round factor.  Returns
 * PIRO_ERR_TABLE_FULL when the fill-in does not fit.  N <= 46340 (int32 keys
 * in the reference).
 * piro_ht_lu_factor / piro_ht_lu_solve give scheme 27 a solution, which the
 * reference does not compute (its lu_decompHT.cl eliminates in FP32 without
 * pivoting and never substitutes).  The factor reads the table once and
 * writes shift*I + scale*M (M the table's matrix) in FP64 into a band of
 * bandwidth bw (nx*ny for the 7-point grid), then factorizes it by Gaussian
 * elimination with partial pivoting in FP64, as LAPACK's banded LU (dgbtrf):
 * P A = L U with U's upper bandwidth 2bw, the first row of largest magnitude
 * chosen on a tie, by panels of 16 columns (8 or 4 for bands wider than
 * about 1 600); the environment variable PIRO_LU_UNBLOCKED=1 selects the
 * column-by-column form, which gives the same bits.  band is a device buffer
 * of piro_ht_lu_band_bytes bytes (band, multipliers, pivots, the panels'
 * multipliers and the solve's workspace).  PIRO_ERR_ARG when a
 * table entry lies outside the band; PIRO_ERR_ZERO_PIVOT when a column has no
 * nonzero at or below the diagonal (a singular matrix).  piro_ht_lu_solve
 * solves A x = b (b, x device float[N]) in FP64 -- the row exchanges and
 * Gauss transforms, then back substitution -- and rounds x to FP32.
 * The solve runs by 16-row panels with y in a shared-memory ring of 2bw + 16
 * rows (bands up to about 10 000 wide; wider ones, or PIRO_LU_NO_RING=1, keep
 * y in global memory, same bits).
 * piro_ht_lu_pivots copies the pivot rows (0-based, LAPACK's ipiv - 1) to the
 * host. */
int piro_ht_lu_reference(int64_t N, int64_t *keys, float *vals, int64_t ts, piro_stream_t stream);
int piro_ht_lu_band_bytes(int64_t N, int64_t bw, size_t *bytes);
int piro_ht_lu_factor(int64_t N, int64_t bw, const int64_t *keys, const float *vals, int64_t ts, float shift,
                      float scale, void *band, size_t band_bytes, piro_stream_t stream);
int piro_ht_lu_solve(int64_t N, int64_t bw, void *band, size_t band_bytes, const float *b, float *x,
                     piro_stream_t stream);
int piro_ht_lu_pivots(int64_t N, int64_t bw, const void *band, size_t band_bytes, int32_t *piv_host);

/* DENSE format (Data 1).  piro_dense_laplacian: Piro::DENSE::stencils::
 * laplacian_* (src/stencils.cpp:431-570) into A (N x N row-major floats,
 * a_bytes >= 4*N*N; zeroed here), values -6/norm and 1/norm in float, uw/dw
 * assignments in the reference's order.  piro_dense_fe_step:
 * kernelsolve::DENSE::TIMESCHEME_11 (src/kernelprocess.cpp:42-66,
 * SpMVDENSE.cl + addVectors.cl): out[r] = u[r] + dt*sum_k A[r][k]*u[k], every
 * row, the sum in ascending k as the kernel adds it. */
int piro_dense_laplacian(int nx, int ny, int nz, int scheme, float norm, float *A, size_t a_bytes,
                         piro_stream_t stream);
int piro_dense_fe_step(int64_t N, const float *A, float dt, const float *u, float *out, piro_stream_t stream);
/* Synchronizes the stream; PIRO_ERR_CUDA if a DENSE step's stage wait (a
 * bounded wait on the bulk copies, never expected to run out) gave up. */
int piro_dense_check(piro_stream_t stream);

/* Matrix-free 7-point step, the comparison point for CSR (laplacianscalar.cl:1-21
 * extended by alpha and the Euler update): interior cells
 * out = u + dt*(alpha*((u[x+1]+u[x-1]-2u)*idx2 + (..y..)*idy2 + (..z..)*idz2)),
 * boundary cells copied.  alpha may be NULL (1). */
int piro_stencil_fe_step(int nx, int ny, int nz, float idx2, float idy2, float idz2, float dt, const float *alpha,
                         const float *u, float *out, piro_stream_t stream);

/* Synchronizes the stream; PIRO_ERR_CUDA if a matrix-free step staged through
 * TMA (16 <= nx <= 256, nx a divisor of 2048 and a multiple of 4, 16-byte
 * aligned buffers) had a stage wait -- a bounded wait on its tile copies,
 * never expected to run out -- give up.  No reference counterpart (the
 * reference's laplacianscalar.cl is never launched). */
int piro_stencil_check(piro_stream_t stream);

/* setBC.cl (launched by bc::opencl_setBC, src/bc.cpp:38-65): dst[idx[i]] = src[idx[i]]. */
int piro_set_bc(int64_t q, const uint32_t *idx, const float *src, float *dst, piro_stream_t stream);

/* Face-interior index lists of bc::initbc (src/bc.cpp:107-146): faces 0 x=nx-1,
 * 1 x=0, 2 y=ny-1, 3 y=0, 4 z=0, 5 z=nz-1, each ascending, concatenated.
 * piro_face_count gives Q and the 7 face offsets (host only); piro_face_lists
 * writes idx[Q] on the device. */
int piro_face_count(int nx, int ny, int nz, int64_t *q, int64_t face_start[7]);
int piro_face_lists(int nx, int ny, int nz, uint32_t *idx, piro_stream_t stream);

/* Elementwise kernels of 0_kernels_math.txt (operatoroverload.cpp:125-307):
 * op 0 add (a = b + c), 1 subtract (b - c), 2 multiply, 3 divide. */
int piro_vec_op(int op, int64_t n, const float *b, const float *c, float *a, piro_stream_t stream);
/* *_constant.cl: op 0 a = s + c, 1 a = c - s, 2 a = s * c, 3 a = c / s. */
int piro_vec_op_scalar(int op, int64_t n, float s, const float *c, float *a, piro_stream_t stream);
/* addVectors_URF.cl: t = a; a += c*urf; c = a - t. */
int piro_vec_urf(int64_t n, float *a, float *c, float urf, piro_stream_t stream);

/* -- csrgeam ---------------------------------------------------------------- */

/* Workspace bytes for the count/scan passes over nrows rows. */
int piro_scan_workspace(int64_t nrows, size_t *bytes);

/* operator& (src/operatoroverload.cpp:102-123) -> kernelmethods::csrgeam
 * (src/kernelcsrgeam.cpp:9-86; csrgeam_1.cl, prefixsum.cl, csrgeam_3.cl):
 * D = diag(v_x)*A (+) diag(v_y)*B (+) diag(v_z)*C as concatenated rows: a
 * three-way column merge (ties A, B, C) while all three rows have entries,
 * then the tails of A, B, C appended unmerged.  v is the 3N SoA vector.
 * nnz(D) = nnz(A)+nnz(B)+nnz(C).  The N serial scan launches of the
 * reference become one device scan. */
int piro_csrgeam3(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA, const int32_t *rpB,
                  const int32_t *cB, const float *vB, const int32_t *rpC, const int32_t *cC, const float *vC,
                  const float *v, int32_t *rpD, int32_t *cD, float *vD, void *work, size_t work_bytes,
                  piro_stream_t stream);

/* piro_csrgeam3 for callers that cannot allocate device memory (a host that
 * fixes its whole device-memory budget before the time loop, or one that only
 * owns the buffers it passes in).  No counterpart in the reference: it is an
 * addition of this library.  Same arguments and results as piro_csrgeam3,
 * without the workspace: the scan scratch is a fixed 36 KB array inside the
 * library, held on every GPU that loads it until exit.  Serves 1 to 16,777,216
 * rows (PIRO_ERR_ARG beyond).  Allocates nothing.  All calls share the array:
 * calls whose GPU work overlaps (other streams or threads on the same device)
 * race and must be serialised by the caller.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; under CUDA's lazy module loading that first call is also where the
 * driver loads the array onto the device.  Make one small call per device at
 * start-up, before fixing the device-memory budget and before starting any
 * stream capture; later calls allocate nothing.  Arguments are checked before
 * any device work. */
int piro_csrgeam3_noalloc(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA, const int32_t *rpB,
                          const int32_t *cB, const float *vB, const int32_t *rpC, const int32_t *cC, const float *vC,
                          const float *v, int32_t *rpD, int32_t *cD, float *vD, piro_stream_t stream);

/* D = A + beta*B, one union row per row with ascending columns; a column in
 * both rows is A's value + beta*B's value.  Builds the backward-Euler matrix
 * I - dt*diag(alpha)*L (no counterpart kernel in the reference, whose JLI
 * applies dt inside SpMVCSR_I1.cl).  Two calls: _count writes rpD[N+1]
 * (read rpD[N] for nnz), _fill writes cD/vD. */
int piro_csrgeam2_count(int64_t N, const int32_t *rpA, const int32_t *cA, const int32_t *rpB, const int32_t *cB,
                        int32_t *rpD, void *work, size_t work_bytes, piro_stream_t stream);
int piro_csrgeam2_fill(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA, float beta,
                       const int32_t *rpB, const int32_t *cB, const float *vB, const int32_t *rpD, int32_t *cD,
                       float *vD, piro_stream_t stream);

/* Identity CSR of N rows (the A of A + beta*B). */
int piro_csr_identity(int64_t N, int32_t *rowptr, int32_t *col, float *val, piro_stream_t stream);

/* -- norms and dots (FP64 accumulation, deterministic) -------------------- */

/* Workspace bytes for a reduction over n elements. */
int piro_reduce_workspace(int64_t n, size_t *bytes);
/* *out (device double) = sum x[i]*y[i]; y == x gives the squared norm, which
 * replaces the host sum of squares of extras.cpp:24-30. */
int piro_dot_f64(int64_t n, const float *x, const float *y, double *out, void *work, size_t work_bytes,
                 piro_stream_t stream);

/* -- backward Euler (TIMESCHEME 12) ----------------------------------------- */

typedef struct piro_be_solver piro_be_solver;

typedef struct piro_be_info {
    int status;            /* PIRO_OK, PIRO_STATUS_STALLED or PIRO_ERR_NOT_CONVERGED */
    int outer_iterations;  /* FP64 refinement sweeps                               */
    int inner_iterations;  /* FP32 Krylov iterations summed over sweeps            */
    int fallbacks;         /* learned-preconditioner sweeps that reverted to Jacobi */
    double rel_residual;   /* ||b - A x||_2 / ||b||_2 over interior rows, FP64     */
} piro_be_info;

/* Preconditioner kinds for piro_be_set_preconditioner. */
#define PIRO_PRECOND_JACOBI 0
#define PIRO_PRECOND_LEARNED 1
#define PIRO_PRECOND_JACOBI_FLEX 2 /* Jacobi inside the flexible-CG iteration (checks that path) */

/* Create a solver for A x = b with A = I - dt*diag(alpha)*L given as CSR over
 * all N rows (device pointers, which must stay valid).  Interior rows are the
 * unknowns; boundary values are held at b (Dirichlet).  The system is solved
 * in its symmetric form diag(alpha)^-1 A on the interior (requires L
 * symmetric there: space scheme 3), by FP32 Jacobi-PCG inside FP64 iterative
 * refinement.  Replaces kernelsolve::CSR::TIMESCHEME_12_40
 * (src/kernelprocess.cpp:123-209), whose Richardson iteration diverges for
 * dt*lambda_max > 2.  The solver allocates its own workspace. */
int piro_be_create(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                   const float *alpha, piro_stream_t stream, piro_be_solver **out);
/* As piro_be_create, for A built as I - dt*diag(alpha)*L from the central
 * 7-point Laplacian of the given norm (space scheme 3).  The inner Krylov
 * operator is then applied matrix-free (alpha, dt and norm instead of the
 * CSR stream: 20 instead of ~60 bytes per row) after a device check that A's
 * interior block holds exactly those coefficients; if it does not, the CSR
 * operator is used.  The FP64 residual is always that of the assembled A:
 * the CSR itself, or the checked stencil plus A's interior-boundary entries
 * copied from the CSR. */
int piro_be_create_stencil(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                           const float *alpha, float dt, float norm, piro_stream_t stream, piro_be_solver **out);
/* Inner operator in use: 0 CSR SpMV (graph-launched CG), 1 matrix-free
 * 7-point stencil (graph-launched CG), 2 matrix-free stencil with the whole
 * solve in one persistent cooperative launch (FP64 refinement and CG phases
 * separated by a grid barrier whose waits are bounded), 3 the same launch
 * with each block's p, d, q resident in shared memory (r formed from z where
 * it is needed).  The environment
 * variable PIRO_BE_PERSISTENT, read at creation, forces kind <= 1 ("0") or
 * keeps kind 2 instead of 3 ("g"). */
int piro_be_inner_operator(piro_be_solver *s, int *kind);
/* Algorithmic bytes moved by the persistent launches counted in
 * piro_be_kernel_stats (since its last reset). */
int piro_be_persistent_bytes(piro_be_solver *s, double *bytes);
/* Solve: b, x device float[N]; x receives the FP32 solution (boundary = b).
 * Stops when the FP64 relative residual <= rtol.  info may be NULL. */
int piro_be_solve(piro_be_solver *s, const float *b, float *x, double rtol, int max_outer, int max_inner,
                  piro_be_info *info);
/* FP64 copy of the last solution (device double[N]) for error reporting. */
int piro_be_solution_f64(piro_be_solver *s, const double **x64);
/* Live timing of the solver's dominant kernel -- the CG SpMV q = A p, or the
 * persistent solve kernel when inner operator kind 2 is in use: CUDA events
 * recorded around each launch give the launches since the last reset and
 * their summed device time in ms; kernel_launches counts every kernel the
 * solver launched.  Any output pointer may be NULL. */
int piro_be_kernel_stats(piro_be_solver *s, int reset, long long *spmv_launches, double *spmv_ms,
                         long long *kernel_launches);
int piro_be_destroy(piro_be_solver *s);

/* -- learned preconditioner (flexible CG inside the backward-Euler solve) -----
 *
 * A 3-D convolutional net z = M(r, f): four 3x3x3 convolutions, channels
 * 2 -> 16 -> 16 -> 16 -> 1, GELU (tanh form) after the first three, zero padding outside
 * the interior, BF16 weights and activations with FP32 accumulation.  Input
 * channels per cell: the residual r (scaled to unit RMS over the interior by
 * the solver) and r*f with the feature f = log(dt * alpha / h^2); output: an
 * approximation of the error A^-1 r.  With no biases M(0) = 0.  It is trained on the device with the library's own
 * forward and backward kernels (masked MSE against the error, Adam).  PIRO has
 * no learned component: this extends TIMESCHEME 12
 * (src/kernelprocess.cpp:123-209), with Jacobi-PCG kept as the fallback. */
typedef struct piro_pcnet piro_pcnet;

/* Number of parameters (one flat FP32 vector: per layer W[tap][ci][co],
 * tap = (dz+1)*9 + (dy+1)*3 + (dx+1); the convolutions have no bias, so a
 * zero residual maps to a zero correction). */
int piro_pcnet_num_params(int64_t *n);
/* New network with deterministic He-normal weights from `seed`. */
int piro_pcnet_create(uint64_t seed, piro_pcnet **out);
/* Host copies of the parameters: FP32 master values, or (rounded != 0) the
 * BF16-rounded values the kernels use.  set_params also resets Adam. */
int piro_pcnet_get_params(piro_pcnet *n, float *host, int64_t count, int rounded);
int piro_pcnet_set_params(piro_pcnet *n, const float *host, int64_t count);
/* out[b][c] = M(r[b], feat[b]) over `batch` grids of nx*ny*nz cells (device
 * float arrays, batch-major; feat may be NULL = 0).  Boundary outputs are 0. */
int piro_pcnet_forward(piro_pcnet *n, int batch, int nx, int ny, int nz, const float *r, const float *feat,
                       float *out, piro_stream_t stream);
/* Forward + backward: loss = sum mask*(M(r,f) - target)^2 / sum mask; the
 * parameter gradient is kept on the device for piro_pcnet_adam_step.  loss
 * (host double) and grad (host float[num_params]) may be NULL; when either is
 * given the call synchronizes the stream. */
int piro_pcnet_loss_grad(piro_pcnet *n, int batch, int nx, int ny, int nz, const float *r, const float *feat,
                         const float *target, const float *mask, double *loss, float *grad, piro_stream_t stream);
/* Adam (beta1 0.9, beta2 0.999, eps 1e-8) with the last computed gradient. */
int piro_pcnet_adam_step(piro_pcnet *n, float lr, piro_stream_t stream);
/* Engine of the network's kernels (default: tensor cores), for the
 * inference forward pass (piro_pcnet_forward and the solver's preconditioner
 * apply) and for training (piro_pcnet_loss_grad): CUDA-core kernels, or every
 * convolution on tcgen05 -- the forward passes and the data gradients as
 * implicit GEMMs (TMA-staged BF16 operands with the channels padded to 16,
 * FP32 accumulation in tensor memory), the weight gradients as GEMMs over the
 * cells with MN-major operands; in training the loss gradient enters the last
 * layer in BF16. */
#define PIRO_PCNET_CUDA_CORES 0
#define PIRO_PCNET_TENSOR_CORES 1
int piro_pcnet_set_engine(piro_pcnet *n, int engine);
/* Kernels launched by this network so far. */
int piro_pcnet_stats(piro_pcnet *n, long long *launches);
int piro_pcnet_destroy(piro_pcnet *n);

/* Select the inner preconditioner of a stencil solver (piro_be_create_stencil):
 * PIRO_PRECOND_JACOBI, or PIRO_PRECOND_LEARNED with a network (not owned; it
 * must outlive the solver's use of it).  With the learned preconditioner the
 * inner solve is flexible CG (Notay's FCG(1)): the network preconditions the
 * first iteration of each refinement sweep (graph-launched), Jacobi the rest
 * (one cooperative launch where the device allows it); a refinement sweep
 * that stalls (FP64 residual not halved) or breaks down reverts to
 * Jacobi-PCG for the rest of the solve (piro_be_info.fallbacks). */
int piro_be_set_preconditioner(piro_be_solver *s, int kind, piro_pcnet *net);
/* Live timing of the learned preconditioner: network applies since the last
 * reset and their summed device time in ms (CUDA events around each apply). */
int piro_be_pc_stats(piro_be_solver *s, int reset, long long *applies, double *ms);

/* -- z-slab decomposition of one grid over ranks ------------------------------
 *
 * A rank owns grid planes [z0, z1) and keeps arrays of planes z0-1 .. z1 (one
 * halo plane each side; local cell l = grid cell l + (z0-1)*nx*ny).  The host
 * exchanges halo planes between neighbouring ranks and all-reduces the FP64
 * partial sums these entry points return (device double[]); see
 * piro_b200/slab.py.  Forward Euler: the owned rows of the assembled CSR
 * matrix (column indices local) stepped exactly as SpMVCSR.cl, so a sharded
 * step equals the single-grid step bit for bit.  Backward Euler: the
 * single-grid solver's method (FP32 Jacobi-PCG in FP64 refinement on
 * A = I - dt*diag(alpha)*L, central scheme) with a matrix-free operator whose
 * couplings to boundary cells carry the stencil value. */
/* nnz of grid rows [row0, row0 + nrows) of the Laplacian. */
int piro_laplacian_nnz_rows(int nx, int ny, int nz, int64_t row0, int64_t nrows, int64_t *nnz);
/* Those rows of PIRO's CSR Laplacian (entries, order and 10.0 rule of
 * stencils.cpp:233-429): rowptr[nrows+1] from 0, columns minus col_shift. */
int piro_csr_laplacian_rows(int nx, int ny, int nz, int space_scheme, float norm, int64_t row0, int64_t nrows,
                            int64_t col_shift, int32_t *rowptr, int32_t *col, float *val, piro_stream_t stream);
/* SpMVCSR.cl on rows [row0, row0 + nrows): out[ubase + i] = u[ubase + i] +
 * sum_k (dt*val[k])*u[col[k]] for interior grid rows row0 + i. */
int piro_csr_fe_step_rows(int nx, int ny, int nz, int64_t row0, int64_t nrows, const int32_t *rowptr,
                          const int32_t *col, const float *val, float dt, const float *u, int64_t ubase, float *out,
                          piro_stream_t stream);
/* Doubles of the `work` array the slab solver kernels need. */
int piro_slab_workspace(int64_t *doubles);
/* r = b - A x64 (FP64), z = r / A_rr on owned interior cells; sums[4] =
 * |r64|^2, |b|^2, <r/alpha, z>, |r32|^2 over the owned interior. */
int piro_slab_be_residual(int nx, int ny, int nz, int z0, int z1, float dt, float norm, const float *alpha,
                          const float *b, const double *x64, float *r, float *z, double *work, double *sums,
                          piro_stream_t stream);
/* p_new = z + beta p_old (owned and halo planes), q = A p_new (owned);
 * sums[0] = <p_new, q/alpha>.  z's halo planes must be current. */
int piro_slab_cg_spmv(int nx, int ny, int nz, int z0, int z1, float dt, float norm, float beta, const float *alpha,
                      const float *z, const float *p_old, float *p_new, float *q, double *work, double *sums,
                      piro_stream_t stream);
/* d += a p, r -= a q, z = r / A_rr (owned); sums[0..1] = <r/alpha, z>, |r|^2. */
int piro_slab_cg_update(int nx, int ny, int nz, int z0, int z1, float dt, float norm, float a, const float *alpha,
                        const float *p, const float *q, float *d, float *r, float *z, double *work, double *sums,
                        piro_stream_t stream);
/* x64 += d, d = 0 on owned interior cells. */
int piro_slab_x_update(int nx, int ny, int nz, int z0, int z1, double *x64, float *d, piro_stream_t stream);
/* The CG steps with their scalars kept on the device, so that an iteration
 * needs no host round trip: state is a device double[8] -- 0 <r/alpha, z>,
 * 1 beta, 2 a, 3 the inner stop threshold (tol2 * rr0), 4 done, 5 iterations,
 * 6 |r|^2, 7 broken -- identical on every rank because it is formed from
 * all-reduced sums.  piro_slab_cg_spmv_dev is piro_slab_cg_spmv with beta
 * from state; piro_slab_cg_update_dev is piro_slab_cg_update with a =
 * state[0] / pq[0] (pq: the all-reduced sums of the spmv step); both return
 * at once when state says done.  piro_slab_cg_scalars (one thread) then
 * forms a, beta and the stop and breakdown tests from pq and up (the
 * all-reduced sums of the update step).  No counterpart in the reference,
 * which runs one grid in one process (src/solve.cpp:11-48). */
int piro_slab_cg_spmv_dev(int nx, int ny, int nz, int z0, int z1, float dt, float norm, const double *state,
                          const float *alpha, const float *z, const float *p_old, float *p_new, float *q,
                          double *work, double *sums, piro_stream_t stream);
int piro_slab_cg_update_dev(int nx, int ny, int nz, int z0, int z1, float dt, float norm, const double *state,
                            const double *pq, const float *alpha, const float *p, const float *q, float *d, float *r,
                            float *z, double *work, double *sums, piro_stream_t stream);
int piro_slab_cg_scalars(double *state, const double *pq, const double *up, piro_stream_t stream);

/* -- batched stepping: many independent problems in one persistent launch ----
 *
 * `count` independent heat problems, member k a constant-alpha cube of n[k]^3
 * ghost-inclusive cells (h = 1, homogeneous boundary values held fixed) with
 * its own dt and scheme (0: forward Euler as SpMVCSR.cl + setBC with the
 * matrix-free 7-point arithmetic; 1: backward Euler, (I - dt*alpha*L) u' = u
 * by FP32 CG inside FP64 iterative refinement to a relative residual).  The
 * fields sit back to back in one device array (member k at offset[k], offsets
 * 64-cell aligned).  One step advances every member with ONE cooperative
 * persistent kernel launch: forward-Euler members in its first pass, the
 * backward-Euler members as a lockstep state machine of FP64-residual and CG
 * phases separated by grid barriers (bounded waits), with per-member
 * reductions in a fixed order.  PIRO steps one grid per process
 * (src/solve.cpp:11-48); this is the build's batched form of that loop. */
typedef struct piro_batch piro_batch;
int piro_batch_create(int count, const int *n, const float *alpha, const float *dt, const int *scheme,
                      piro_stream_t stream, piro_batch **out);
/* offsets (int64[count], may be NULL) and the total cells of the field array. */
int piro_batch_layout(piro_batch *s, int64_t *offsets, int64_t *total_cells);
/* Copy all fields in (out): host (from_host/to_host != 0) or device memory. */
int piro_batch_set_fields(piro_batch *s, const float *u, int from_host);
int piro_batch_get_fields(piro_batch *s, float *u, int to_host);
/* Device pointer of the current fields (valid until the next step). */
int piro_batch_field_ptr(piro_batch *s, float **u);
/* Advance every member `steps` times (one launch per step); backward-Euler
 * members solve to the FP64 relative residual rtol.  *ms (may be NULL) gets
 * the device time (CUDA events). */
int piro_batch_step(piro_batch *s, int steps, double rtol, double *ms);
/* Per-member result of the last step (host arrays of count; any may be NULL):
 * status (PIRO_OK, PIRO_STATUS_STALLED, PIRO_ERR_NOT_CONVERGED), refinement
 * sweeps, CG iterations, FP64 relative residual (0 for forward Euler). */
int piro_batch_member_info(piro_batch *s, int *status, int *sweeps, int *inner, double *rel);
/* Autotuner: times one step from the current fields (result discarded) for
 * each tile size (2048 .. 16384 cells) and blocks-per-SM (1, 2, 4) the
 * occupancy allows and keeps the fastest. */
int piro_batch_autotune(piro_batch *s, double rtol, int *tile, int *blocks_per_sm);
/* Schedule of the step: 0 lockstep (k_batch_step: every backward-Euler
 * member advances one phase per grid-wide round), 1 grouped (k_batch_groups:
 * each large member on a group of CTAs of its own with group-local barriers,
 * small members packed onto the other CTAs; no grid-wide barrier).  The
 * autotuner picks the faster; piro_batch_set_schedule forces one, with the
 * given CTAs per SM.  Results agree to rounding (the same arithmetic per
 * member, sums over other partitions). */
int piro_batch_schedule(piro_batch *s, int *grouped);
int piro_batch_set_schedule(piro_batch *s, int grouped, int blocks_per_sm);
int piro_batch_destroy(piro_batch *s);

/* Reference JLI iteration (scheme 12 + solver 40, src/kernelprocess.cpp:123-209)
 * on the device: x = b; repeat r = b - (I - dt*L)x on interior rows (b on the
 * others), x += urf*r, r = dx; res = ||r||/sqrt(N); stop when
 * (res - res_old)^2 < tol.  Residual sums are FP64.  *iters receives the count. */
int piro_be_jli(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val, float dt,
                const float *b, float *x, float *r_work, float tol, float urf, int maxiter, int *iters,
                piro_stream_t stream);

/* ========================================================================
 * 2. Context API: PIRO's operator interface over a case .ini
 * ======================================================================== */

typedef struct piro_ctx piro_ctx;

/* A field handle (CLBuffer of operatoroverload.hpp:9-17): index of the field
 * in creation order (constants, scalars, vectors) and its length. */
typedef struct piro_buf {
    int32_t id;
    int64_t n;
} piro_buf;

/* An operator handle (the std::vector<CLBuffer> the reference returns). */
typedef struct piro_op {
    int32_t kind;
} piro_op;

#define PIRO_OP_LAPLACIAN 1
#define PIRO_OP_GRADIENT 2
#define PIRO_OP_DOT 3        /* vector & gradient (csrgeam result) */
#define PIRO_OP_DIV 4        /* div(var1, var2): csrgeam_2 of the divergence matrices */
#define PIRO_EQN_RESULT (-1) /* piro_buf id of the operator= result (partD) */

typedef struct piro_case_info {
    int32_t nx, ny, nz; /* ghost-inclusive */
    int64_t n_cells;
    int32_t timescheme, spacescheme, solverscheme, datatype, simindex;
    float timestep, totaltime;
    int64_t steps_done;
    int32_t n_fields;
    int64_t bc_cells;
} piro_case_info;

/* Piro::preprocess (src/preprocess.cpp:20-208) + bc::readbc: read
 * <assets_dir>/<case_name> ([File] [Mesh] [Simulation] [IC] [Schemes]
 * [Solve]), solver.ini ([JLI], when Solver = 40), Data/hashtable.ini ([Table],
 * when Data = 2), IC/distribution.ini and setup.ini ([BC]); add the ghost
 * layers; create the fields with their initial conditions (src/ic.cpp) on the
 * device; compute the boundary values of field 1 (src/bc.cpp:107-157).
 * PIRO_ERR_CONFIG names a missing or malformed key (the reference throws). */
int piro_open(const char *assets_dir, const char *case_name, piro_ctx **out);
void piro_close(piro_ctx *ctx);
int piro_ctx_query(piro_ctx *ctx, piro_case_info *info);
/* 0 (default): alpha applied as SpMDSM intends; 1: alpha dropped, as the
 * reference's csrscale actually behaves (src/kernelcsrgeam.cpp:224-231), and
 * likewise div's velocity scaling (SpMSCSR, kernelcsrgeam.cpp:100-130).
 * Must be set before the operator is assembled. */
int piro_set_alpha_mode(piro_ctx *ctx, int mode);
/* Scheme 27 (TIMESCHEME 12, solver 27, Data 2).  0 (default): backward Euler
 * solved directly -- A = I - dt*M (M the operator's table) factorized in a
 * dense band of bandwidth nx*ny on the first step (piro_ht_lu_factor), then
 * substitution every step (piro_ht_lu_solve).  1: as the reference
 * runs -- PIRO's factorization of the operator's own table on the first step
 * (piro_ht_lu_reference) and a zero result field
 * (src/operatoroverload.cpp:65-81).  Must be set before the first step. */
int piro_set_lu_mode(piro_ctx *ctx, int mode);

/* process::ddt_r / process::vector / matchscalartovar (src/process.cpp:20-58,
 * 154-166): the handle of the named field (field 0 when no name matches, as
 * in the reference). */
int piro_ddt_r(piro_ctx *ctx, const char *var, piro_buf *out);
int piro_vector(piro_ctx *ctx, const char *var, piro_buf *out);
int piro_field(piro_ctx *ctx, const char *var, piro_buf *out);
/* Host <-> device copies of a field (synchronous). */
int piro_field_upload(piro_ctx *ctx, piro_buf f, const float *host, int64_t n);
int piro_field_download(piro_ctx *ctx, piro_buf f, float *host, int64_t n);
int piro_field_device_ptr(piro_ctx *ctx, piro_buf f, float **dptr);

/* process::laplacian (src/process.cpp:60-122): assembled on the first call
 * per [Solve] Data (0 CSR, 1 DENSE (N x N floats), 2 HT, 3 COO) and cached;
 * for CSR the rows are scaled by the field named `coeff`. */
int piro_laplacian(piro_ctx *ctx, const char *var, const char *coeff, piro_op *out);
/* process::gradient (src/process.cpp:124-152): the three CSR matrices. */
int piro_gradient(piro_ctx *ctx, const char *var, piro_op *out);
/* operator& (src/operatoroverload.cpp:102-123): csrgeam of a vector field
 * with the gradient, merged once and cached. */
int piro_dot(piro_ctx *ctx, piro_buf v, piro_op grad, piro_op *out);
/* process::div (src/process.cpp:168-215): the divergence matrices (the
 * gradient stencils, operatordivergenceCSR.cpp:21-101) with matrix a's rows
 * scaled by component a of the vector field var2, merged as csrgeam_2
 * (kernelcsrgeam.cpp:88-207); CSR only.  Under piro_set_alpha_mode(1) the
 * rows stay unscaled, as the reference's SpMSCSR launches (int arguments set
 * with sizeof(cl_mem)) never run. */
int piro_div(piro_ctx *ctx, const char *var1, const char *var2, piro_op *out);
/* CLBuffer::operator= (src/operatoroverload.cpp:20-100): one time step of
 * lhs by [Schemes] Time: 11 forward Euler (CSR, DENSE, HT or COO), 12
 * backward Euler with Solver 40 (JLI, as written, CSR), 39 (FP32 PCG in FP64
 * refinement to 1e-8, CSR Laplacian) or 27 (HT LU, piro_set_lu_mode).  *out
 * is the new field (partD, PIRO_EQN_RESULT). */
int piro_assign(piro_ctx *ctx, piro_buf lhs, piro_op rhs, piro_buf *out);
/* scalarMatrix::Solve (src/process.cpp:221-236): copy the result into field
 * 1 and apply the Dirichlet face values (setBC). */
int piro_step_solve(piro_ctx *ctx, piro_buf eqn, float time);
/* Piro::solve (src/solve.cpp:11-48): while (time < TotalTime) with float
 * time, the equation of [File] simindex per step: 0 heat
 * ddt_r(T) = laplacian(T, Alpha), 1 advection ddt_r(U) = vector(v) &
 * gradient(U), 2 continuity ddt_r(rho) = div(rho, u). */
int piro_solve(piro_ctx *ctx, int64_t *steps_taken);
/* Download an assembled operator in CSR form (nnz only when rowptr is NULL). */
int piro_op_export_csr(piro_ctx *ctx, piro_op op, int32_t *rowptr, int32_t *col, float *val, int64_t cap,
                       int64_t *nnz);

/* -- ParaView output (Piro::paraview, src/paraview.cpp:12-137) ------------------
 *
 * piro_write_paraview writes <root>/<casename>/mesh/mesh_<ts>.vth and
 * .../mesh/level/<ts>_level_0.vti (ts zero-padded to 5 digits) with the bytes
 * PIRO writes: ASCII cell data of every scalar and vector field (constants
 * skipped; vectors as _x/_y/_z arrays), boundary cells removed, values
 * formatted as std::ostream formats a float.  The interior cells are gathered
 * on the device, so only they cross PCIe (the reference copies whole fields
 * and erases boundary entries one at a time).  [Mesh] index must be 1 per
 * level: the reference only has data for level data set 0.
 * piro_set_output sets the root (NULL disables output; [File] restart = 1
 * clears <root>/<casename> first, as Piro::init); piro_step_solve then writes
 * every Save steps as scalarMatrix::Solve does (src/process.cpp:236-247).
 * piro_interior_gather: dst[k*Ni + j] = src[k*N + interior cell j] for ncomp
 * components (Ni = (nx-2)(ny-2)(nz-2), x fastest). */
int piro_write_paraview(piro_ctx *c, const char *root, int timestep);
int piro_set_output(piro_ctx *c, const char *root);
int piro_interior_gather(int nx, int ny, int nz, int ncomp, const float *src, float *dst, piro_stream_t stream);


#ifdef __cplusplus
}
#endif
#endif /* PIRO_H */
