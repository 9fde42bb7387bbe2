/*
 * piro_oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * A plain-C CPU restatement of PIRO's sparse finite-difference time-stepping
 * path, used only as the checker: by tests/, by __graft_entry__.smoke() and by
 * bench.py's CPU baseline / reference arm.  Nothing in piro_b200/ links it.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths are relative to the PIRO source tree).  Parity is pinned by running
 * the reference's own host code and its .cl kernels (compiled as C++ through
 * oracle/ref_driver.cpp) against this file on small grids; the committed
 * fixtures in tests/golden/ hold those outputs.
 *
 * Conventions (as in the reference):
 *   - grid sizes nx, ny, nz include one ghost layer per side
 *     (src/preprocess.cpp:72-74);
 *   - linear index i = x + y*nx + z*nx*ny (src/mathoperations.cpp:38-40);
 *   - fields are float32[N]; vectors are float32[3N], x block, y block,
 *     z block (src/ic.cpp:84-95).
 * Floating-point expressions keep the reference's operation order; build with
 * -ffp-contract=off so that no multiply-add is fused.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR_ARG -1
#define OR_ERR_TABLE_FULL -2
#define OR_ERR_TABLE_SIZE -3

static inline int64_t idx3(int64_t x, int64_t y, int64_t z, int64_t nx, int64_t ny)
{
    /* src/mathoperations.cpp:38-40 */
    return x + y * nx + z * nx * ny;
}

static inline int is_boundary(int x, int y, int z, int nx, int ny, int nz)
{
    /* src/bc.cpp:169-178 (bc::isBoundaryPoint) */
    return x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Laplacian assembly: CSR (src/stencils.cpp:233-429), COO (:572-795) and the
 * row pushes the HT path uses (:797-993).  Per row, in this order: self
 * (-6/norm), x-, x+, y-, y+, z-, z+ (+1/norm), each only if that neighbour
 * exists.  Scheme 1 (uw) replaces every "+" neighbour column by the row itself,
 * scheme 2 (dw) every "-" neighbour column, scheme 3 (cd) keeps both.
 * For a boundary row i, std::find over the WHOLE column array sets the first
 * occurrence of column i to 10.0 (stencils.cpp:278-291).  first_pos[] records
 * the first push of each column, which is exactly what that std::find returns,
 * because columns are only ever appended.
 *
 * norm is float; the values are (float)(-6.0/(double)norm) and
 * (float)(1.0/(double)norm) because the literals are double (stencils.cpp:245,250).
 * rows may be NULL (CSR); rowptr may be NULL (COO).  Returns nnz, or -1.
 */
int64_t or_laplacian(int nx, int ny, int nz, int scheme, float norm,
                     int32_t *rowptr, int32_t *rows, int32_t *col, float *val)
{
    const int64_t N = (int64_t)nx * ny * nz;
    int64_t *first_pos = (int64_t *)malloc(sizeof(int64_t) * (size_t)N);
    if (!first_pos) return -1;
    for (int64_t i = 0; i < N; ++i) first_pos[i] = -1;
    if (rowptr) for (int64_t i = 0; i <= N; ++i) rowptr[i] = 0;
    if (scheme < 1 || scheme > 3) { free(first_pos); return 0; } /* operatorlaplacian.cpp:34-42: no stencil */

    const float v_self = (float)(-6.0 / (double)norm);
    const float v_nb = (float)(1.0 / (double)norm);
    int64_t k = 0;
#define PUSH(c, v)                                   \
    do {                                             \
        int64_t c_ = (c);                            \
        col[k] = (int32_t)c_;                        \
        val[k] = (v);                                \
        if (rows) rows[k] = (int32_t)i;              \
        if (first_pos[c_] < 0) first_pos[c_] = k;    \
        ++k;                                         \
    } while (0)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int64_t i = idx3(x, y, z, nx, ny);
                const int64_t xm = scheme == 2 ? i : idx3(x - 1, y, z, nx, ny);
                const int64_t xp = scheme == 1 ? i : idx3(x + 1, y, z, nx, ny);
                const int64_t ym = scheme == 2 ? i : idx3(x, y - 1, z, nx, ny);
                const int64_t yp = scheme == 1 ? i : idx3(x, y + 1, z, nx, ny);
                const int64_t zm = scheme == 2 ? i : idx3(x, y, z - 1, nx, ny);
                const int64_t zp = scheme == 1 ? i : idx3(x, y, z + 1, nx, ny);
                PUSH(i, v_self);
                if (x > 0) PUSH(xm, v_nb);
                if (x < nx - 1) PUSH(xp, v_nb);
                if (y > 0) PUSH(ym, v_nb);
                if (y < ny - 1) PUSH(yp, v_nb);
                if (z > 0) PUSH(zm, v_nb);
                if (z < nz - 1) PUSH(zp, v_nb);
                if (is_boundary(x, y, z, nx, ny, nz)) val[first_pos[i]] = 10.0f;
                if (rowptr) rowptr[i + 1] = (int32_t)k;
            }
#undef PUSH
    free(first_pos);
    return k;
}

/* Gradient assembly, CSR, one axis (src/stencils.cpp:7-231, called from
 * src/operatorgradient.cpp:35-104 with norm = 2*(l0/(n0-2)), :25).
 * uw: (i-e, -1/norm) if a>0, (i, +1/norm) if a<n-1; cd: (i-e, -), (i+e, +);
 * dw: (i, -) if a>0, (i+e, +) if a<n-1.  Values are float divisions
 * (-1/norm with int -1, stencils.cpp:17).  rowptr[i+1] is written only after
 * a push, so it must be passed in with its previous contents (zeros for x,
 * the x result for y, the y result for z: operatorgradient.cpp:26,51,77). */
int64_t or_gradient(int nx, int ny, int nz, int scheme, int axis, float norm,
                    int32_t *rowptr, int32_t *col, float *val)
{
    if (scheme < 1 || scheme > 3 || axis < 0 || axis > 2) return 0;
    const float vm = -1 / norm;
    const float vp = 1 / norm;
    int64_t k = 0;
    const int64_t e = axis == 0 ? 1 : axis == 1 ? nx : (int64_t)nx * ny;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int64_t i = idx3(x, y, z, nx, ny);
                const int a = axis == 0 ? x : axis == 1 ? y : z;
                const int na = axis == 0 ? nx : axis == 1 ? ny : nz;
                if (a > 0) {
                    col[k] = (int32_t)(scheme == 2 ? i : i - e);
                    val[k] = vm;
                    ++k;
                    rowptr[i + 1] = (int32_t)k;
                }
                if (a < na - 1) {
                    col[k] = (int32_t)(scheme == 1 ? i : i + e);
                    val[k] = vp;
                    ++k;
                    rowptr[i + 1] = (int32_t)k;
                }
            }
    return k;
}

/* ------------------------------------------------------------------------ */
/* Hash table (HT) format.  Table size: src/operatorlaplacian.cpp:184-185 with
 * the [Table] constants of assets/Data/hashtable.ini.  The expression mixes a
 * double pow() with float operands exactly like the C++ does:
 *   float load = a * pow(N, b) + c;            (double arithmetic, stored float)
 *   TS = (int)(sparsecount / (load * lf));     (float arithmetic)            */
int64_t or_ht_table_size_reference(int64_t sparsecount, int64_t N, float a, float b, float c, float lf)
{
    float load = (float)((double)a * pow((double)(int)N, (double)b) + (double)c);
    float denom = load * lf;
    float q = (float)(int)sparsecount / denom;
    return (int64_t)(int)q;
}

/* Linear-probing insert (src/methods.cpp:74-118, methods::sethash):
 * slot = key % TS; an existing key is overwritten; -1 is empty; the first -2
 * (tombstone) seen is reused when the probe reaches an empty slot.  Keys are
 * held in int64 here; the reference's int32 key row*N+col is the same number
 * while N <= 46340. */
int or_ht_sethash(int64_t key, float v, int64_t TS, int64_t *keys, float *vals)
{
    int64_t h = key % TS;
    int64_t attempts = 0, first_deleted = -1;
    while (attempts < TS) {
        if (keys[h] == key) { vals[h] = v; return OR_OK; }
        if (keys[h] == -1) {
            int64_t at = first_deleted != -1 ? first_deleted : h;
            keys[at] = key;
            vals[at] = v;
            return OR_OK;
        }
        if (keys[h] == -2 && first_deleted == -1) first_deleted = h;
        h = (h + 1) % TS;
        ++attempts;
    }
    if (first_deleted != -1) { keys[first_deleted] = key; vals[first_deleted] = v; return OR_OK; }
    return OR_ERR_TABLE_FULL; /* reference: logs and std::exit(1), methods.cpp:106-116 */
}

/* Row-major insertion of a CSR matrix (src/operatorlaplacian.cpp:190-203). */
int or_ht_build(int64_t N, const int32_t *rowptr, const int32_t *col, const float *val,
                int64_t TS, int64_t *keys, float *vals)
{
    if (TS <= 0) return OR_ERR_TABLE_SIZE;
    for (int64_t s = 0; s < TS; ++s) { keys[s] = -1; vals[s] = 0.0f; }
    for (int64_t i = 0; i < N; ++i)
        for (int64_t j = rowptr[i]; j < rowptr[i + 1]; ++j) {
            int rc = or_ht_sethash(i * N + col[j], val[j], TS, keys, vals);
            if (rc) return rc;
        }
    return OR_OK;
}

/* methods::lookup (src/methods.cpp:8-33): probe from key % TS over non-empty
 * slots; 0.0 when absent. */
float or_ht_lookup(int64_t key, int64_t TS, const int64_t *keys, const float *vals)
{
    int64_t h = key % TS, attempts = 0;
    while (keys[h] != -1 && keys[h] != key) {
        h = (h + 1) % TS;
        if (++attempts >= TS) return 0.0f;
    }
    return keys[h] == key ? vals[h] : 0.0f;
}

/* ------------------------------------------------------------------------ */
/* csrgeam (src/kernelcsrgeam.cpp:9-86 with csrgeam_1.cl, prefixsum.cl and
 * csrgeam_3.cl).  A, B, C are the x, y and z gradient matrices; v is the 3N
 * SoA vector.  Count = lenA+lenB+lenC (the dedup branch of csrgeam_1.cl:46-51
 * is unreachable).  Scan: rowptr[0] = 0, rowptr[i+1] = sum of counts up to i
 * (kernelcsrgeam.cpp:53-62 after the zero fill at :36-38).  Fill: three-way
 * merge by column while all three rows have entries, ties taken A then B then
 * C (csrgeam_3.cl:37-69), then the tails of A, B and C appended in that order
 * without merging (:71-88).  Values are val*v[row + comp*N].              */
void or_csrgeam3_count(int64_t N, const int32_t *rpA, const int32_t *rpB, const int32_t *rpC,
                       int32_t *count)
{
    for (int64_t r = 0; r < N; ++r)
        count[r] = (rpA[r + 1] - rpA[r]) + (rpB[r + 1] - rpB[r]) + (rpC[r + 1] - rpC[r]);
}

void or_scan_rowptr(int64_t N, const int32_t *count, int32_t *rowptr)
{
    rowptr[0] = 0;
    for (int64_t i = 0; i < N; ++i) rowptr[i + 1] = count[i] + rowptr[i];
}

void or_csrgeam3_fill(int64_t N,
                      const int32_t *rpA, const int32_t *cA, const float *vA,
                      const int32_t *rpB, const int32_t *cB, const float *vB,
                      const int32_t *rpC, const int32_t *cC, const float *vC,
                      const float *v, const int32_t *rpD, int32_t *cD, float *vD)
{
    for (int64_t row = 0; row < N; ++row) {
        int32_t i = rpA[row], ie = rpA[row + 1];
        int32_t j = rpB[row], je = rpB[row + 1];
        int32_t k = rpC[row], ke = rpC[row + 1];
        int64_t d = rpD[row];
        const float sa = v[row], sb = v[N + row], sc = v[2 * N + row];
        while (i < ie && j < je && k < ke) {
            int32_t a = cA[i], b = cB[j], c = cC[k];
            int32_t m = a < b ? a : b;
            m = m < c ? m : c;
            if (a == m) { cD[d] = a; vD[d] = vA[i] * sa; ++i; }
            else if (b == m) { cD[d] = b; vD[d] = vB[j] * sb; ++j; }
            else { cD[d] = c; vD[d] = vC[k] * sc; ++k; }
            ++d;
        }
        for (; i < ie; ++i, ++d) { cD[d] = cA[i]; vD[d] = vA[i] * sa; }
        for (; j < je; ++j, ++d) { cD[d] = cB[j]; vD[d] = vB[j] * sb; }
        for (; k < ke; ++k, ++d) { cD[d] = cC[k]; vD[d] = vC[k] * sc; }
    }
}

/* Row scale diag(s)*M: the intended effect of kernelmethods::csrscale
 * (src/kernelcsrgeam.cpp:208-234) through SpMDSM.cl:20-31, val[k] *= s[row(k)].
 * (The reference enqueues the wrong kernel there, so alpha is silently dropped;
 * the "compat" mode simply skips this call.) */
void or_csr_rowscale(int64_t N, const int32_t *rowptr, float *val, const float *s)
{
    for (int64_t r = 0; r < N; ++r)
        for (int32_t k = rowptr[r]; k < rowptr[r + 1]; ++k) val[k] *= s[r];
}

/* A + beta*B with one union row per row: columns ascending, a column present
 * in both is A's value plus beta*B's value; duplicate columns inside B are
 * summed in storage order.  This is the build's own operator for the
 * backward-Euler matrix I - dt*diag(alpha)*L (the reference has no such
 * kernel); count pass, then fill with the same rowptr. */
static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

static int64_t union_row(const int32_t *ca, int64_t na, const int32_t *cb, int64_t nb, int32_t *out)
{
    int64_t n = 0;
    for (int64_t t = 0; t < na; ++t) out[n++] = ca[t];
    for (int64_t t = 0; t < nb; ++t) out[n++] = cb[t];
    qsort(out, (size_t)n, sizeof(int32_t), cmp_i32);
    int64_t u = 0;
    for (int64_t t = 0; t < n; ++t)
        if (u == 0 || out[u - 1] != out[t]) out[u++] = out[t];
    return u;
}

void or_csrgeam2_count(int64_t N, const int32_t *rpA, const int32_t *cA,
                       const int32_t *rpB, const int32_t *cB, int32_t *count)
{
    int32_t buf[256];
    for (int64_t r = 0; r < N; ++r)
        count[r] = (int32_t)union_row(cA + rpA[r], rpA[r + 1] - rpA[r], cB + rpB[r], rpB[r + 1] - rpB[r], buf);
}

void or_csrgeam2_fill(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA, float beta,
                      const int32_t *rpB, const int32_t *cB, const float *vB,
                      const int32_t *rpD, int32_t *cD, float *vD)
{
    int32_t buf[256];
    for (int64_t r = 0; r < N; ++r) {
        int64_t u = union_row(cA + rpA[r], rpA[r + 1] - rpA[r], cB + rpB[r], rpB[r + 1] - rpB[r], buf);
        for (int64_t t = 0; t < u; ++t) {
            const int32_t c = buf[t];
            float acc = 0.0f;
            int have = 0;
            for (int32_t a = rpA[r]; a < rpA[r + 1]; ++a)
                if (cA[a] == c) { acc = have ? acc + vA[a] : vA[a]; have = 1; }
            for (int32_t b = rpB[r]; b < rpB[r + 1]; ++b)
                if (cB[b] == c) { float t2 = beta * vB[b]; acc = have ? acc + t2 : t2; have = 1; }
            cD[rpD[r] + t] = c;
            vD[rpD[r] + t] = acc;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* DENSE Laplacian (src/stencils.cpp:431-570, from src/operatorlaplacian.cpp:
 * 65-103): A is N x N row-major, zero except per row l, in this order,
 * A[l][l] = -6/norm, then for each existing neighbour (x-, x+, y-, y+, z-, z+)
 * A[l][nb] = 1/norm -- assignments, so where uw/dw replace a neighbour by l
 * itself the diagonal ends as 1/norm.  No 10.0 rule on this path.  The
 * constants are int / float: float divisions (stencils.cpp:439,445). */
void or_dense_laplacian(int nx, int ny, int nz, int scheme, float norm, float *A)
{
    const int64_t N = (int64_t)nx * ny * nz;
    memset(A, 0, sizeof(float) * (size_t)N * (size_t)N);
    if (scheme < 1 || scheme > 3) return;
    const float v_self = -6.0f / norm, v_nb = 1.0f / norm;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int64_t l = idx3(x, y, z, nx, ny);
                float *row = A + l * N;
                row[l] = v_self;
                if (x > 0) row[scheme == 2 ? l : idx3(x - 1, y, z, nx, ny)] = v_nb;
                if (x < nx - 1) row[scheme == 1 ? l : idx3(x + 1, y, z, nx, ny)] = v_nb;
                if (y > 0) row[scheme == 2 ? l : idx3(x, y - 1, z, nx, ny)] = v_nb;
                if (y < ny - 1) row[scheme == 1 ? l : idx3(x, y + 1, z, nx, ny)] = v_nb;
                if (z > 0) row[scheme == 2 ? l : idx3(x, y, z - 1, nx, ny)] = v_nb;
                if (z < nz - 1) row[scheme == 1 ? l : idx3(x, y, z + 1, nx, ny)] = v_nb;
            }
}

/* DENSE forward Euler (src/kernelprocess.cpp:42-66): SpMVDENSE.cl (P = 1)
 * C[r] = deltat * sum, sum += A[r][k]*B[k] over k ascending, every row; then
 * addVectors.cl: D = B + C. */
void or_fe_dense_step(int64_t N, const float *A, float dt, const float *B, float *C, float *D)
{
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < N; ++r) {
        float sum = 0.0f;
        const float *row = A + r * N;
        for (int64_t k = 0; k < N; ++k) sum += row[k] * B[k];
        C[r] = dt * sum;
        D[r] = B[r] + C[r];
    }
}

/* ------------------------------------------------------------------------ */
/* Interior mask used by SpMVCSR.cl:29-32 and SpMVCSR_I1.cl:28-31. */
static inline int interior_row(int64_t id, uint32_t nx, uint32_t ny, uint32_t size)
{
    uint32_t z = (uint32_t)(id / (nx * ny));
    uint32_t y = (uint32_t)((id / nx) % ny);
    uint32_t x = (uint32_t)(id % nx);
    return x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < (size / (nx * ny)) - 1;
}

/* SpMVCSR.cl:12-39 (R = 1): interior rows get B[r] + sum_k dt*val*B[col],
 * summed in storage order as result += (deltat*value_A)*B[col]; other rows of
 * C are left as they are. */
void or_spmv_csr_fe(int64_t N, int nx, int ny, const int32_t *rp, const int32_t *col, const float *val,
                    float dt, const float *B, float *C)
{
#pragma omp parallel for schedule(static)
    for (int64_t row = 0; row < N; ++row) {
        float result = 0.0f;
        for (int32_t i = rp[row]; i < rp[row + 1]; ++i) {
            float t = dt * val[i];
            result += t * B[col[i]];
        }
        if (interior_row(row, (uint32_t)nx, (uint32_t)ny, (uint32_t)N)) C[row] = result + B[row];
    }
}

/* SpMVCSR_I1.cl:12-36: interior rows get B[r] - sum_k dt*val*B[col]. */
void or_spmv_csr_i1(int64_t N, int nx, int ny, const int32_t *rp, const int32_t *col, const float *val,
                    float dt, const float *B, float *C)
{
#pragma omp parallel for schedule(static)
    for (int64_t row = 0; row < N; ++row) {
        float result = 0.0f;
        for (int32_t i = rp[row]; i < rp[row + 1]; ++i) {
            float t = dt * val[i];
            result += t * B[col[i]];
        }
        if (interior_row(row, (uint32_t)nx, (uint32_t)ny, (uint32_t)N)) C[row] = B[row] - result;
    }
}

/* SpMVCOO.cl:12-24: C[row] = dt * sum over entries with rows[ind]==row in
 * ascending ind of values*B[col], on every row.  One pass in ascending ind
 * gives every row the same summation order as the per-row scan. */
void or_spmv_coo(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals,
                 float dt, const float *B, float *C)
{
    float *acc = (float *)calloc((size_t)N, sizeof(float));
    for (int64_t k = 0; k < nnz; ++k) acc[rows[k]] += vals[k] * B[cols[k]];
    for (int64_t r = 0; r < N; ++r) C[r] = dt * acc[r];
    free(acc);
}

/* SpMVHT.cl:22-40: C[row] = dt * sum_{col=0..N-1} H(row,col)*B[col], with
 * lookup() returning 0 for absent keys (SpMVHT.cl:1-20).  Absent keys add
 * 0*B[col] = 0, so for finite B the sum equals the sum over present keys in
 * ascending column order, which is what is computed here: the table's keys
 * are gathered and sorted. */
static int cmp_i64pair(const void *a, const void *b)
{
    int64_t x = ((const int64_t *)a)[0], y = ((const int64_t *)b)[0];
    return (x > y) - (x < y);
}

void or_spmv_ht(int64_t N, int64_t TS, const int64_t *keys, const float *vals, float dt,
                const float *B, float *C)
{
    int64_t cnt = 0;
    for (int64_t s = 0; s < TS; ++s) cnt += keys[s] >= 0;
    int64_t *kv = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(cnt ? cnt : 1));
    int64_t m = 0;
    for (int64_t s = 0; s < TS; ++s)
        if (keys[s] >= 0) { kv[2 * m] = keys[s]; kv[2 * m + 1] = s; ++m; }
    qsort(kv, (size_t)m, 2 * sizeof(int64_t), cmp_i64pair);
    int64_t t = 0;
    for (int64_t r = 0; r < N; ++r) {
        float sum = 0.0f;
        while (t < m && kv[2 * t] / N == r) {
            int64_t c = kv[2 * t] % N;
            sum += vals[kv[2 * t + 1]] * B[c];
            ++t;
        }
        C[r] = dt * sum;
    }
    free(kv);
}

/* addVectors.cl, subtractVectors.cl, addVectors_URF.cl, setBC.cl and the
 * elementwise kernels of 0_kernels_math.txt (op: 0 add, 1 sub, 2 mul, 3 div). */
void or_vec_binary(int op, int64_t n, const float *B, const float *C, float *A)
{
    for (int64_t i = 0; i < n; ++i)
        A[i] = op == 0 ? B[i] + C[i] : op == 1 ? B[i] - C[i] : op == 2 ? B[i] * C[i] : B[i] / C[i];
}

/* *_constant.cl: add B + C, subtract C - B, multiply B * C, divide C / B. */
void or_vec_constant(int op, int64_t n, float b, const float *C, float *A)
{
    for (int64_t i = 0; i < n; ++i)
        A[i] = op == 0 ? b + C[i] : op == 1 ? C[i] - b : op == 2 ? b * C[i] : C[i] / b;
}

void or_urf(int64_t n, float *A, float *C, float urf)
{
    for (int64_t i = 0; i < n; ++i) {
        float t = A[i];
        A[i] += C[i] * urf;
        C[i] = A[i] - t;
    }
}

void or_setbc(int64_t q, const uint32_t *idx, const float *src, float *dst)
{
    for (int64_t i = 0; i < q; ++i) dst[idx[i]] = src[idx[i]];
}

/* Face-interior index lists (src/bc.cpp:113-146): faces 0 x=nx-1, 1 x=0,
 * 2 y=ny-1, 3 y=0, 4 z=0, 5 z=nz-1; edges and corners are excluded; each list
 * ascends in the linear index; the flat list concatenates faces 0..5
 * (bc.cpp:27-30).  face_start[7] receives the offsets.  Returns Q. */
int64_t or_face_lists(int nx, int ny, int nz, uint32_t *idx, int64_t *face_start)
{
    const int64_t N = (int64_t)nx * ny * nz;
    int64_t cnt[6] = {0, 0, 0, 0, 0, 0};
    for (int pass = 0; pass < 2; ++pass) {
        int64_t pos[6];
        if (pass == 1) {
            face_start[0] = 0;
            for (int f = 0; f < 6; ++f) face_start[f + 1] = face_start[f] + cnt[f];
            for (int f = 0; f < 6; ++f) pos[f] = face_start[f];
        }
        for (int64_t ind = 0; ind < N; ++ind) {
            uint32_t kd = (uint32_t)(ind / ((int64_t)ny * nx));
            uint32_t jd = (uint32_t)((ind % ((int64_t)ny * nx)) / nx);
            uint32_t id = (uint32_t)(ind % nx);
            int face[3] = {-1, -1, -1};
            int xi = id != 0 && id != (uint32_t)nx - 1, yi = jd != 0 && jd != (uint32_t)ny - 1,
                zi = kd != 0 && kd != (uint32_t)nz - 1;
            if (jd == 0 && xi && zi) face[0] = 3;
            else if (jd == (uint32_t)ny - 1 && xi && zi) face[0] = 2;
            if (kd == 0 && xi && yi) face[1] = 4;
            else if (kd == (uint32_t)nz - 1 && xi && yi) face[1] = 5;
            if (id == 0 && yi && zi) face[2] = 1;
            else if (id == (uint32_t)nx - 1 && yi && zi) face[2] = 0;
            for (int t = 0; t < 3; ++t)
                if (face[t] >= 0) {
                    if (pass == 0) cnt[face[t]]++;
                    else idx[pos[face[t]]++] = (uint32_t)ind;
                }
        }
    }
    return face_start[6];
}

/* Number of forward steps Piro::solve() takes: `while (time < totaltime)`
 * with float time += timestep (src/solve.cpp:17-18,45). */
int64_t or_step_count(float totaltime, float dt)
{
    float t = 0.0f;
    int64_t n = 0;
    while (t < totaltime) { t += dt; ++n; }
    return n;
}

/* One forward-Euler Solve() on CSR (src/operatoroverload.cpp:29-45,
 * src/kernelprocess.cpp:10-40, src/process.cpp:221-235): a zero-filled
 * partD, SpMVCSR over the interior, copy to the field, then setBC from the
 * saved initial values (memD, src/bc.cpp:31-32). */
void or_fe_csr_step(int64_t N, int nx, int ny, const int32_t *rp, const int32_t *col, const float *val,
                    float dt, float *u, int64_t q, const uint32_t *bc_idx, const float *bc_src, float *work)
{
    memset(work, 0, sizeof(float) * (size_t)N);
    or_spmv_csr_fe(N, nx, ny, rp, col, val, dt, u, work);
    memcpy(u, work, sizeof(float) * (size_t)N);
    or_setbc(q, bc_idx, bc_src, u);
}

/* COO and HT forward Euler (src/kernelprocess.cpp:68-120): C = dt*M*u on all
 * rows, u' = u + C (addVectors), then setBC. */
void or_fe_coo_step(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals,
                    float dt, float *u, int64_t q, const uint32_t *bc_idx, const float *bc_src, float *work)
{
    or_spmv_coo(N, nnz, rows, cols, vals, dt, u, work);
    for (int64_t i = 0; i < N; ++i) u[i] = u[i] + work[i];
    or_setbc(q, bc_idx, bc_src, u);
}

void or_fe_ht_step(int64_t N, int64_t TS, const int64_t *keys, const float *vals, float dt, float *u,
                   int64_t q, const uint32_t *bc_idx, const float *bc_src, float *work)
{
    or_spmv_ht(N, TS, keys, vals, dt, u, work);
    for (int64_t i = 0; i < N; ++i) u[i] = u[i] + work[i];
    or_setbc(q, bc_idx, bc_src, u);
}

/* Matrix-free 7-point forward Euler, the comparison point for the CSR path:
 * laplacianscalar.cl:1-21 gives dt*Lap(u) on interior cells as
 * ((u[+1]+u[-1]-2u)/dx^2 + (..y..)/dy^2 + (..z..)/dz^2); here the divisions are
 * multiplications by idx2 = 1/dx^2 etc., the sum is scaled by alpha[i] and
 * added to u, and boundary cells are copied through.  alpha may be NULL
 * (alpha = 1). */
void or_stencil_fe(int nx, int ny, int nz, float idx2, float idy2, float idz2, float dt, const float *alpha,
                   const float *B, float *C)
{
    const int64_t sxy = (int64_t)nx * ny;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                int64_t id = idx3(x, y, z, nx, ny);
                if (x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1) {
                    float c2 = 2.0f * B[id];
                    float lx = ((B[id + 1] + B[id - 1]) - c2) * idx2;
                    float ly = ((B[id + nx] + B[id - nx]) - c2) * idy2;
                    float lz = ((B[id + sxy] + B[id - sxy]) - c2) * idz2;
                    float lap = (lx + ly) + lz;
                    float a = alpha ? alpha[id] : 1.0f;
                    C[id] = B[id] + dt * (a * lap);
                } else {
                    C[id] = B[id];
                }
            }
}

/* Backward Euler "JLI" (scheme 12 + solver 40), src/kernelprocess.cpp:123-209:
 * x = b; repeat { r = 0; r[int] = x - dt*L*x (SpMVCSR_I1); r = b - r;
 * x += urf*r, r = x_new - x_old (addVectors_URF); res = sqrt(sum r^2)/sqrt(N)
 * (extras.cpp:24-30, float, sequential); stop when (res-res_old)^2 < tol }.
 * Returns the iteration count used (1-based). */
int or_be_jli(int64_t N, int nx, int ny, const int32_t *rp, const int32_t *col, const float *val, float dt,
              const float *b, float *x, float *r, float tol, float urf, int maxiter)
{
    memcpy(x, b, sizeof(float) * (size_t)N);
    float res_old = 0.0f;
    int it;
    for (it = 0; it < maxiter; ++it) {
        memset(r, 0, sizeof(float) * (size_t)N);
        or_spmv_csr_i1(N, nx, ny, rp, col, val, dt, x, r);
        for (int64_t i = 0; i < N; ++i) r[i] = b[i] - r[i];
        or_urf(N, x, r, urf);
        float s = 0.0f;
        for (int64_t i = 0; i < N; ++i) s += r[i] * r[i];
        float res = sqrtf(s) / sqrtf((float)N);
        float d = (res - res_old) * (res - res_old);
        if (d < tol) return it + 1;
        res_old = res;
    }
    return it;
}

/* ------------------------------------------------------------------------ */
/* FP64 reference solve for the backward-Euler step (the build's own
 * formulation; the reference's JLI diverges at large dt).  Interior rows r:
 *   sum_c A[r,c] u[c] = b[r], A = I - dt*diag(alpha)*L as assembled (FP32
 *   values, exact in FP64), boundary u held at b.
 * Solved as the SPD system diag(alpha)^-1 A_II d = diag(alpha)^-1 r by
 * Jacobi-preconditioned CG in FP64 until ||b - A u||_2 / ||b||_2 <= rtol over
 * interior rows.  A is passed as CSR over all N rows.  Returns iterations, or
 * -1 if maxiter is reached. */
static void csr_apply_interior_f64(int64_t N, const uint8_t *interior, const int32_t *rp, const int32_t *col,
                                   const float *val, const double *p, double *q)
{
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < N; ++r) {
        if (!interior[r]) { q[r] = 0.0; continue; }
        double s = 0.0;
        for (int32_t k = rp[r]; k < rp[r + 1]; ++k) s += (double)val[k] * p[col[k]];
        q[r] = s;
    }
}

static double dot_f64(int64_t n, const double *a, const double *b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

int or_be_cg_f64d(int64_t N, int nx, int ny, int nz, const int32_t *rp, const int32_t *col, const float *val,
                  const float *alpha, const double *b, double *u, double rtol, int maxiter, double *final_rel);

/* b in float32 (a field as the solvers receive it). */
int or_be_cg_f64(int64_t N, int nx, int ny, int nz, const int32_t *rp, const int32_t *col, const float *val,
                 const float *alpha, const float *b, double *u, double rtol, int maxiter, double *final_rel)
{
    double *bd = (double *)malloc((size_t)N * sizeof(double));
    for (int64_t i = 0; i < N; ++i) bd[i] = (double)b[i];
    const int it = or_be_cg_f64d(N, nx, ny, nz, rp, col, val, alpha, bd, u, rtol, maxiter, final_rel);
    free(bd);
    return it;
}

/* b in float64: the step of an FP64-only trajectory (the previous step's
 * FP64 solution as the right-hand side). */
int or_be_cg_f64d(int64_t N, int nx, int ny, int nz, const int32_t *rp, const int32_t *col, const float *val,
                  const float *alpha, const double *b, double *u, double rtol, int maxiter, double *final_rel)
{
    uint8_t *interior = (uint8_t *)malloc((size_t)N);
    double *r = (double *)calloc((size_t)N, sizeof(double));
    double *z = (double *)calloc((size_t)N, sizeof(double));
    double *p = (double *)calloc((size_t)N, sizeof(double));
    double *q = (double *)calloc((size_t)N, sizeof(double));
    double *dinv = (double *)calloc((size_t)N, sizeof(double));
    double *bb = (double *)calloc((size_t)N, sizeof(double));
    for (int64_t i = 0; i < N; ++i) {
        int x = (int)(i % nx), y = (int)((i / nx) % ny), zz = (int)(i / ((int64_t)nx * ny));
        interior[i] = !is_boundary(x, y, zz, nx, ny, nz);
        u[i] = b[i];
    }
    /* diag(S) = A_rr / alpha_r; S = diag(alpha)^-1 A on the interior block. */
    for (int64_t i = 0; i < N; ++i) {
        double d = 0.0;
        if (interior[i])
            for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
                if (col[k] == i) d += (double)val[k];
        dinv[i] = interior[i] && d != 0.0 ? (double)alpha[i] / d : 0.0;
    }
    /* ||b|| over interior rows; residual r = b - A u over interior rows. */
    csr_apply_interior_f64(N, interior, rp, col, val, u, q);
    double bnorm2 = 0.0;
    for (int64_t i = 0; i < N; ++i)
        if (interior[i]) {
            bb[i] = b[i];
            bnorm2 += bb[i] * bb[i];
            r[i] = bb[i] - q[i];
        }
    double bnorm = sqrt(bnorm2);
    if (bnorm == 0.0) bnorm = 1.0;
    /* CG on S = diag(1/alpha) A_II with rhs diag(1/alpha) r. */
    double *s = (double *)calloc((size_t)N, sizeof(double));
    for (int64_t i = 0; i < N; ++i) s[i] = interior[i] ? r[i] / (double)alpha[i] : 0.0;
    for (int64_t i = 0; i < N; ++i) { z[i] = dinv[i] * s[i]; p[i] = z[i]; }
    double rz = dot_f64(N, s, z);
    int it = 0, ok = 0;
    double rel = sqrt(dot_f64(N, r, r)) / bnorm;
    while (it < maxiter) {
        if (rel <= rtol) { ok = 1; break; }
        csr_apply_interior_f64(N, interior, rp, col, val, p, q); /* q = A p */
        double pq = 0.0;
#pragma omp parallel for reduction(+ : pq) schedule(static)
        for (int64_t i = 0; i < N; ++i)
            if (interior[i]) pq += p[i] * q[i] / (double)alpha[i];
        double a = rz / pq;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
            if (interior[i]) {
                u[i] += a * p[i];
                r[i] -= a * q[i];
                s[i] = r[i] / (double)alpha[i];
                z[i] = dinv[i] * s[i];
            }
        double rz2 = dot_f64(N, s, z);
        double beta = rz2 / rz;
        rz = rz2;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
        ++it;
        rel = sqrt(dot_f64(N, r, r)) / bnorm;
    }
    /* final true residual */
    csr_apply_interior_f64(N, interior, rp, col, val, u, q);
    double rr = 0.0;
    for (int64_t i = 0; i < N; ++i)
        if (interior[i]) { double t = bb[i] - q[i]; rr += t * t; }
    if (final_rel) *final_rel = sqrt(rr) / bnorm;
    free(interior); free(r); free(z); free(p); free(q); free(dinv); free(bb); free(s);
    return ok ? it : -1;
}

/* ------------------------------------------------------------------------ */
/* Initial conditions (src/ic.cpp:16-99), host float/double arithmetic as the
 * C++ evaluates it.  Coordinates are x*l0/(float)nx with ghost-inclusive n
 * (ic.cpp:53-55).  std::exp(float) is expf; std::pow with a double or int
 * argument is the double pow. */
void or_ic_gaussian(int nx, int ny, int nz, float l0, float l1, float l2, float scale, const float *sigma,
                    const float *mean, float *out)
{
    const float norm = (float)(1.0f / (pow(2.0f * M_PI, 1.5f) * sigma[0] * sigma[1] * sigma[2]));
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const float c0 = x * l0 / (float)nx, c1 = y * l1 / (float)ny, c2 = z * l2 / (float)nz;
                const float a = (c0 - mean[0]) / sigma[0], b = (c1 - mean[1]) / sigma[1], c = (c2 - mean[2]) / sigma[2];
                const float e = -0.5f * (a * a + b * b + c * c);
                out[idx3(x, y, z, nx, ny)] = scale * (norm * expf(e));
            }
}

void or_ic_coulomb(int nx, int ny, int nz, float l0, float l1, float l2, const float *center, float Z, double e,
                   double eps0, float *out)
{
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const float c0 = x * l0 / (float)nx, c1 = y * l1 / (float)ny, c2 = z * l2 / (float)nz;
                /* math_operations::calc_length_3d (src/mathoperations.cpp:42-46) */
                const float r = (float)pow(pow((double)(c0 - center[0]), 2.0) + pow((double)(c1 - center[1]), 2.0) +
                                               pow((double)(c2 - center[2]), 2.0),
                                           0.5);
                out[idx3(x, y, z, nx, ny)] =
                    (float)(-((double)Z * 1E15 * pow(e, 2.0)) / (4 * M_PI * eps0 * ((double)r + 1E-10)));
            }
}

/* UniformVector (ic.cpp:80-96): 3N values, block d = dir[d]*value. */
void or_ic_uniform_vector(int64_t N, const float *dir, float value, float *out)
{
    for (int d = 0; d < 3; ++d)
        for (int64_t i = 0; i < N; ++i) out[d * N + i] = dir[d] * value;
}
