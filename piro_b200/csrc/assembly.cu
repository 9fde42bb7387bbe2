// assembly.cu -- Laplacian / gradient assembly on the device, bit-exact with
// PIRO's serial host loops (src/stencils.cpp), plus the row scale, identity
// and boundary face lists.
//
// The reference builds a matrix by pushing entries row by row and, for the
// Laplacian, runs a std::find over the whole column array for every boundary
// row (O(nnz * boundary), stencils.cpp:278-291).  Here each thread owns one
// row: its rowptr comes from a closed-form prefix count of the 7-point
// pattern, so there is no scan, and the "first occurrence of column c" rule is
// decided locally from c's coordinates.  Rows are staged in shared memory per
// block so that col/val/rows leave the SM as coalesced stores.
#include "common.cuh"

namespace piro {
namespace {

constexpr int kRowsPerBlock = 256;
constexpr int kMaxPerRow = 7;

struct Grid {
    int nx, ny, nz;
    int64_t sxy;
    FastDiv fx, fxy;  // division by nx and nx*ny for cell indices below 2^31
};

Grid make_grid(int nx, int ny, int nz)
{
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.sxy = (int64_t)nx * ny;
    g.fx = FastDiv((uint32_t)nx);
    g.fxy = FastDiv((uint32_t)g.sxy);
    return g;
}

// Cell coordinates by multiply-shift division (every grid here has fewer
// than 2^31 cells), not 64-bit division.
__device__ __forceinline__ void coords(int64_t i, const Grid &g, int &x, int &y, int &z)
{
    const uint32_t u = (uint32_t)i;
    const uint32_t zz = g.fxy.div(u);
    const uint32_t rem = u - zz * (uint32_t)g.sxy;
    const uint32_t yy = g.fx.div(rem);
    z = (int)zz;
    y = (int)yy;
    x = (int)(rem - yy * (uint32_t)g.nx);
}

// Sum of 7-point row lengths over all rows before (x, y, z) in row-major
// order; a row has 7 - [x==0] - [x==nx-1] - [y==0] - [y==ny-1] - [z==0] - [z==nz-1]
// entries.
__host__ __device__ __forceinline__ int64_t lap_prefix(int x, int y, int z, const Grid &g)
{
    const int64_t nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t by = (y == 0) + (y == ny - 1);
    const int64_t bz = (z == 0) + (z == nz - 1);
    int64_t p = (int64_t)z * (7 * nx * ny - 2 * ny - 2 * nx) - nx * ny * (z > 0);
    p += (int64_t)y * (7 * nx - 2 - nx * bz) - nx * (y > 0);
    p += (int64_t)x * (7 - by - bz) - (x > 0);
    return p;
}

__device__ __forceinline__ bool is_bnd(int x, int y, int z, const Grid &g)
{
    return x == 0 || x == g.nx - 1 || y == 0 || y == g.ny - 1 || z == 0 || z == g.nz - 1;
}

// One row of the Laplacian: columns, values and count, in push order.  c and
// v point into the block's shared-memory stage (a thread-local array with a
// run-time count would live in local memory).
__device__ __forceinline__ int lap_row(int64_t i, const Grid &g, int scheme, float vself, float vnb, int32_t *c,
                                       float *v)
{
    int x, y, z;
    coords(i, g, x, y, z);
    const bool uw = scheme == 1, dw = scheme == 2;
    int n = 0;
    c[n] = (int32_t)i;
    v[n] = vself;
    // uw: the first occurrence of a boundary row's own column is its self
    // entry (lower rows never reference higher columns); cd/dw: only cell 0.
    if (is_bnd(x, y, z, g) && (uw || i == 0)) v[n] = 10.0f;
    ++n;
    if (x > 0) { c[n] = (int32_t)(dw ? i : i - 1); v[n] = vnb; ++n; }
    if (x < g.nx - 1) {
        c[n] = (int32_t)(uw ? i : i + 1);
        v[n] = vnb;
        // cd/dw: row i is the first referencer of column i+1 iff that cell
        // has no lower z- or y-neighbour (z == 0 and y == 0).
        if (!uw && z == 0 && y == 0 && is_bnd(x + 1, y, z, g)) v[n] = 10.0f;
        ++n;
    }
    if (y > 0) { c[n] = (int32_t)(dw ? i : i - g.nx); v[n] = vnb; ++n; }
    if (y < g.ny - 1) {
        c[n] = (int32_t)(uw ? i : i + g.nx);
        v[n] = vnb;
        if (!uw && z == 0 && is_bnd(x, y + 1, z, g)) v[n] = 10.0f;
        ++n;
    }
    if (z > 0) { c[n] = (int32_t)(dw ? i : i - g.sxy); v[n] = vnb; ++n; }
    if (z < g.nz - 1) {
        c[n] = (int32_t)(uw ? i : i + g.sxy);
        v[n] = vnb;
        if (!uw && is_bnd(x, y, z + 1, g)) v[n] = 10.0f;
        ++n;
    }
    return n;
}

// Block = kRowsPerBlock consecutive rows.  rowptr may be NULL (COO), rows may
// be NULL (CSR).  Rows [row0, row0 + N) of the grid's matrix: rowptr starts at
// 0, entries are stored from 0 and columns (and COO rows) are shifted by
// -col_shift (the whole matrix: row0 = 0, N = all rows, col_shift = 0).
__global__ void __launch_bounds__(kRowsPerBlock) k_laplacian(Grid g, int64_t N, int scheme, float vself, float vnb,
                                                             int32_t *__restrict__ rowptr,
                                                             int32_t *__restrict__ rows, int32_t *__restrict__ col,
                                                             float *__restrict__ val, int64_t row0,
                                                             int64_t col_shift)
{
    // staged at index (global entry index) mod 4 + position in the block, so
    // that shared and global indices agree mod 4 and both sides move as
    // aligned 16-byte vectors
    __shared__ __align__(16) int32_t s_col[kRowsPerBlock * kMaxPerRow + 4];
    __shared__ __align__(16) float s_val[kRowsPerBlock * kMaxPerRow + 4];
    __shared__ __align__(16) int32_t s_row[kRowsPerBlock * kMaxPerRow + 4];
    __shared__ int64_t s_end;
    int64_t base0;
    {
        int x, y, z;
        coords(row0, g, x, y, z);
        base0 = lap_prefix(x, y, z, g);
    }
    const int64_t R1 = row0 + N;
    const bool vec_ok = ((reinterpret_cast<uintptr_t>(col) | reinterpret_cast<uintptr_t>(val) |
                          reinterpret_cast<uintptr_t>(rows)) & 15) == 0;
    for (int64_t r0 = row0 + (int64_t)blockIdx.x * kRowsPerBlock; r0 < R1; r0 += (int64_t)gridDim.x * kRowsPerBlock) {
        const int64_t i = r0 + threadIdx.x;
        const int64_t rlast = (r0 + kRowsPerBlock < R1 ? r0 + kRowsPerBlock : R1) - 1;
        // the block's first entry, the same in every thread (no serial section)
        int64_t s_base;
        {
            int x, y, z;
            coords(r0, g, x, y, z);
            s_base = lap_prefix(x, y, z, g);
        }
        const int sh = vec_ok ? (int)((s_base - base0) & 3) : 0;  // shared index of the first entry
        if (i < R1) {
            int x, y, z;
            coords(i, g, x, y, z);
            const int64_t p = lap_prefix(x, y, z, g);
            const int off = (int)(p - s_base) + sh;
            const int n = lap_row(i, g, scheme, vself, vnb, s_col + off, s_val + off);
            if (col_shift)
                for (int t = 0; t < n; ++t) s_col[off + t] -= (int32_t)col_shift;
            if (rows)
                for (int t = 0; t < n; ++t) s_row[off + t] = (int32_t)(i - col_shift);
            if (rowptr) {
                rowptr[i - row0 + 1] = (int32_t)(p + n - base0);
                if (i == row0) rowptr[0] = 0;
            }
            if (i == rlast) s_end = p + n;
        }
        __syncthreads();
        // the block's entries leave as 16-byte stores (scalar head and tail)
        // when the arrays are 16-byte aligned
        const int cnt = (int)(s_end - s_base);
        const int64_t g0 = s_base - base0 - sh;                   // global index of shared index 0
        const int j0 = vec_ok ? (sh + 3) & ~3 : sh + cnt, j1 = vec_ok ? (sh + cnt) & ~3 : sh + cnt;
        const int head_end = j0 < sh + cnt ? j0 : sh + cnt;
        for (int j = sh + threadIdx.x; j < head_end; j += blockDim.x) {
            col[g0 + j] = s_col[j];
            val[g0 + j] = s_val[j];
            if (rows) rows[g0 + j] = s_row[j];
        }
        for (int j = j0 + 4 * threadIdx.x; j < j1; j += 4 * blockDim.x) {
            *reinterpret_cast<int4 *>(col + g0 + j) = *reinterpret_cast<const int4 *>(s_col + j);
            *reinterpret_cast<float4 *>(val + g0 + j) = *reinterpret_cast<const float4 *>(s_val + j);
            if (rows) *reinterpret_cast<int4 *>(rows + g0 + j) = *reinterpret_cast<const int4 *>(s_row + j);
        }
        for (int j = (j1 > head_end ? j1 : head_end) + threadIdx.x; j < sh + cnt; j += blockDim.x) {
            col[g0 + j] = s_col[j];
            val[g0 + j] = s_val[j];
            if (rows) rows[g0 + j] = s_row[j];
        }
        __syncthreads();
    }
}

// Gradient prefix: number of entries of rows before i for `axis`
// (each row has [a > 0] + [a < n_a - 1] entries).
__host__ __device__ __forceinline__ int64_t grad_prefix(int64_t i, int x, int y, int z, int axis, const Grid &g)
{
    int64_t c0, c1;  // rows before i with a == 0, with a == n_a - 1
    if (axis == 0) {
        int64_t r = (i - x) / g.nx;
        c0 = r + (x > 0);
        c1 = r;
    } else if (axis == 1) {
        c0 = (int64_t)g.nx * z + (y > 0 ? g.nx : x);
        c1 = (int64_t)g.nx * z + (y == g.ny - 1 ? x : 0);
    } else {
        c0 = z > 0 ? g.sxy : i;
        c1 = z == g.nz - 1 ? (int64_t)x + (int64_t)g.nx * y : 0;
    }
    return 2 * i - c0 - c1;
}

// Rows row0 .. row0+n-1 of one axis's matrix into local arrays: entry
// positions relative to row row0's first entry, columns shifted down by
// col_shift (the whole matrix: row0 = col_shift = 0, n = N).
__global__ void __launch_bounds__(kRowsPerBlock) k_gradient(Grid g, int64_t n, int scheme, int axis, float vm, float vp,
                                                            int32_t *__restrict__ rowptr, int32_t *__restrict__ col,
                                                            float *__restrict__ val, int64_t row0, int64_t p0,
                                                            int64_t col_shift)
{
    const int64_t e = axis == 0 ? 1 : axis == 1 ? g.nx : g.sxy;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = row0 + j;
        int x, y, z;
        coords(i, g, x, y, z);
        const int a = axis == 0 ? x : axis == 1 ? y : z;
        const int na = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
        int64_t p = grad_prefix(i, x, y, z, axis, g) - p0;
        if (a > 0) {
            col[p] = (int32_t)((scheme == 2 ? i : i - e) - col_shift);
            val[p] = vm;
            ++p;
        }
        if (a < na - 1) {
            col[p] = (int32_t)((scheme == 1 ? i : i + e) - col_shift);
            val[p] = vp;
            ++p;
        }
        rowptr[j + 1] = (int32_t)p;
        if (j == 0) rowptr[0] = 0;
    }
}

// grad_prefix at a row index on the host (row == N: every entry)
int64_t grad_prefix_host(int64_t i, int axis, const Grid &g, int64_t N)
{
    if (i >= N) {
        const int64_t na = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
        return 2 * N - 2 * (N / na);
    }
    const int z = (int)(i / g.sxy);
    const int64_t rem = i - (int64_t)z * g.sxy;
    const int y = (int)(rem / g.nx);
    return grad_prefix(i, (int)(rem - (int64_t)y * g.nx), y, z, axis, g);
}

__global__ void k_rowscale(int64_t nrows, const int32_t *__restrict__ rowptr, float *__restrict__ val,
                           const float *__restrict__ s)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += (int64_t)gridDim.x * blockDim.x) {
        const float f = s[r];
        for (int32_t k = rowptr[r]; k < rowptr[r + 1]; ++k) val[k] = __fmul_rn(val[k], f);
    }
}

__global__ void k_identity(int64_t N, int32_t *__restrict__ rowptr, int32_t *__restrict__ col, float *__restrict__ val)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        col[r] = (int32_t)r;
        val[r] = 1.0f;
        rowptr[r + 1] = (int32_t)(r + 1);
        if (r == 0) rowptr[0] = 0;
    }
}

// Face lists: faces 0/1 enumerate (z, y), 2/3 (z, x), 4/5 (y, x), each
// over the interior range [1, n-2].
__global__ void k_faces(Grid g, int64_t a, int64_t b, int64_t c, uint32_t *__restrict__ idx)
{
    const int64_t Q = 2 * (a + b + c);
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < Q; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t u = t;
        int face;
        if (u < 2 * a) { face = (int)(u / a); u -= face * a; }
        else if (u < 2 * a + 2 * b) { u -= 2 * a; face = 2 + (int)(u / b); u -= (face - 2) * b; }
        else { u -= 2 * a + 2 * b; face = 4 + (int)(u / c); u -= (face - 4) * c; }
        int x, y, z;
        if (face <= 1) {
            x = face == 0 ? g.nx - 1 : 0;
            z = 1 + (int)(u / (g.ny - 2));
            y = 1 + (int)(u % (g.ny - 2));
        } else if (face <= 3) {
            y = face == 2 ? g.ny - 1 : 0;
            z = 1 + (int)(u / (g.nx - 2));
            x = 1 + (int)(u % (g.nx - 2));
        } else {
            z = face == 4 ? 0 : g.nz - 1;
            y = 1 + (int)(u / (g.nx - 2));
            x = 1 + (int)(u % (g.nx - 2));
        }
        idx[t] = (uint32_t)(x + (int64_t)y * g.nx + (int64_t)z * g.sxy);
    }
}

bool grid_ok(int nx, int ny, int nz)
{
    return nx >= 3 && ny >= 3 && nz >= 3 && (int64_t)nx * ny * nz < (int64_t)INT32_MAX / 8;
}

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_laplacian_nnz(int nx, int ny, int nz, int64_t *nnz)
{
    PIRO_ARG(nnz && grid_ok(nx, ny, nz), "piro_laplacian_nnz: grid sizes must be >= 3 (ghost-inclusive)");
    const int64_t N = (int64_t)nx * ny * nz;
    *nnz = 7 * N - 2 * ((int64_t)nx * ny + (int64_t)ny * nz + (int64_t)nx * nz);
    return PIRO_OK;
}

static int launch_laplacian(int nx, int ny, int nz, int scheme, float norm, int32_t *rowptr, int32_t *rows,
                            int32_t *col, float *val, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz), "laplacian: grid sizes must be >= 3 (ghost-inclusive)");
    PIRO_ARG(col && val, "laplacian: null output");
    if (scheme < 1 || scheme > 3) {
        piro::set_error("laplacian: space scheme %d not in {1 uw, 2 dw, 3 cd}", scheme);
        return PIRO_ERR_SCHEME;
    }
    Grid g = make_grid(nx, ny, nz);
    const int64_t N = (int64_t)nx * ny * nz;
    // The literals are double in stencils.cpp:245,250: (float)(-6.0/norm).
    const float vself = (float)(-6.0 / (double)norm);
    const float vnb = (float)(1.0 / (double)norm);
    unsigned grid = grid_for(N, kRowsPerBlock, 4);
    k_laplacian<<<grid, kRowsPerBlock, 0, as_stream(stream)>>>(g, N, scheme, vself, vnb, rowptr, rows, col, val, 0,
                                                               0);
    PIRO_CHECK_LAUNCH("k_laplacian");
    return PIRO_OK;
}

extern "C" int piro_laplacian_nnz_rows(int nx, int ny, int nz, int64_t row0, int64_t nrows, int64_t *nnz)
{
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(nnz && grid_ok(nx, ny, nz) && row0 >= 0 && nrows >= 0 && row0 + nrows <= N,
             "piro_laplacian_nnz_rows: bad arguments");
    const Grid g = make_grid(nx, ny, nz);
    auto prefix = [&](int64_t i) -> int64_t {
        if (i >= N) return 7 * N - 2 * ((int64_t)nx * ny + (int64_t)ny * nz + (int64_t)nx * nz);
        const int z = (int)(i / g.sxy);
        const int64_t rem = i - (int64_t)z * g.sxy;
        const int y = (int)(rem / nx);
        return lap_prefix((int)(rem - (int64_t)y * nx), y, z, g);
    };
    *nnz = prefix(row0 + nrows) - prefix(row0);
    return PIRO_OK;
}

extern "C" int piro_csr_laplacian_rows(int nx, int ny, int nz, int space_scheme, float norm, int64_t row0,
                                       int64_t nrows, int64_t col_shift, int32_t *rowptr, int32_t *col, float *val,
                                       piro_stream_t stream)
{
    const int64_t N = (int64_t)nx * ny * nz;
    // columns of rows >= row0 reach down to row0 - nx*ny: local columns stay >= 0
    PIRO_ARG(grid_ok(nx, ny, nz) && rowptr && col && val && row0 >= 0 && nrows > 0 && row0 + nrows <= N &&
                 col_shift <= row0 - (row0 > 0 ? (int64_t)nx * ny : 0),
             "piro_csr_laplacian_rows: bad arguments");
    if (space_scheme < 1 || space_scheme > 3) {
        piro::set_error("laplacian: space scheme %d not in {1 uw, 2 dw, 3 cd}", space_scheme);
        return PIRO_ERR_SCHEME;
    }
    Grid g = make_grid(nx, ny, nz);
    const float vself = (float)(-6.0 / (double)norm);
    const float vnb = (float)(1.0 / (double)norm);
    unsigned grid = grid_for(nrows, kRowsPerBlock, 4);
    k_laplacian<<<grid, kRowsPerBlock, 0, as_stream(stream)>>>(g, nrows, space_scheme, vself, vnb, rowptr, nullptr,
                                                               col, val, row0, col_shift);
    PIRO_CHECK_LAUNCH("k_laplacian");
    return PIRO_OK;
}

extern "C" int piro_csr_laplacian(int nx, int ny, int nz, int space_scheme, float norm, int32_t *rowptr, int32_t *col,
                                  float *val, piro_stream_t stream)
{
    PIRO_ARG(rowptr, "piro_csr_laplacian: null rowptr");
    return launch_laplacian(nx, ny, nz, space_scheme, norm, rowptr, nullptr, col, val, stream);
}

extern "C" int piro_coo_laplacian(int nx, int ny, int nz, int space_scheme, float norm, int32_t *rows, int32_t *col,
                                  float *val, piro_stream_t stream)
{
    PIRO_ARG(rows, "piro_coo_laplacian: null rows");
    return launch_laplacian(nx, ny, nz, space_scheme, norm, nullptr, rows, col, val, stream);
}

extern "C" int piro_gradient_nnz(int nx, int ny, int nz, int axis, int64_t *nnz)
{
    PIRO_ARG(nnz && grid_ok(nx, ny, nz) && axis >= 0 && axis <= 2, "piro_gradient_nnz: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    const int64_t na = axis == 0 ? nx : axis == 1 ? ny : nz;
    *nnz = 2 * N - 2 * (N / na);
    return PIRO_OK;
}

extern "C" int piro_csr_gradient(int nx, int ny, int nz, int space_scheme, int axis, float norm, int32_t *rowptr,
                                 int32_t *col, float *val, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz) && axis >= 0 && axis <= 2, "piro_csr_gradient: bad grid or axis");
    PIRO_ARG(rowptr && col && val, "piro_csr_gradient: null output");
    if (space_scheme < 1 || space_scheme > 3) {
        piro::set_error("piro_csr_gradient: space scheme %d not in {1,2,3}", space_scheme);
        return PIRO_ERR_SCHEME;
    }
    Grid g = make_grid(nx, ny, nz);
    const int64_t N = (int64_t)nx * ny * nz;
    // -1/norm and 1/norm are float divisions (int operand promoted), stencils.cpp:17,24.
    const float vm = -1 / norm, vp = 1 / norm;
    k_gradient<<<grid_for(N, 256, 8), 256, 0, as_stream(stream)>>>(g, N, space_scheme, axis, vm, vp, rowptr, col, val,
                                                                   0, 0, 0);
    PIRO_CHECK_LAUNCH("k_gradient");
    return PIRO_OK;
}

extern "C" int piro_gradient_nnz_rows(int nx, int ny, int nz, int axis, int64_t row0, int64_t nrows, int64_t *nnz)
{
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(nnz && grid_ok(nx, ny, nz) && axis >= 0 && axis <= 2 && row0 >= 0 && nrows >= 0 && row0 + nrows <= N,
             "piro_gradient_nnz_rows: bad arguments");
    const Grid g = make_grid(nx, ny, nz);
    *nnz = grad_prefix_host(row0 + nrows, axis, g, N) - grad_prefix_host(row0, axis, g, N);
    return PIRO_OK;
}

extern "C" int piro_csr_gradient_rows(int nx, int ny, int nz, int space_scheme, int axis, float norm, int64_t row0,
                                      int64_t nrows, int64_t col_shift, int32_t *rowptr, int32_t *col, float *val,
                                      piro_stream_t stream)
{
    const int64_t N = (int64_t)nx * ny * nz;
    // columns of rows >= row0 reach down to row0 - nx*ny at most: local columns stay >= 0
    PIRO_ARG(grid_ok(nx, ny, nz) && axis >= 0 && axis <= 2 && rowptr && col && val && row0 >= 0 && nrows > 0 &&
                 row0 + nrows <= N && col_shift <= row0 - (row0 > 0 ? (int64_t)nx * ny : 0),
             "piro_csr_gradient_rows: bad arguments");
    if (space_scheme < 1 || space_scheme > 3) {
        piro::set_error("piro_csr_gradient_rows: space scheme %d not in {1,2,3}", space_scheme);
        return PIRO_ERR_SCHEME;
    }
    Grid g = make_grid(nx, ny, nz);
    const float vm = -1 / norm, vp = 1 / norm;
    const int64_t p0 = grad_prefix_host(row0, axis, g, N);
    k_gradient<<<grid_for(nrows, 256, 8), 256, 0, as_stream(stream)>>>(g, nrows, space_scheme, axis, vm, vp, rowptr,
                                                                       col, val, row0, p0, col_shift);
    PIRO_CHECK_LAUNCH("k_gradient");
    return PIRO_OK;
}

extern "C" int piro_csr_rowscale(int64_t nrows, const int32_t *rowptr, float *val, const float *s, piro_stream_t stream)
{
    PIRO_ARG(nrows >= 0 && rowptr && val && s, "piro_csr_rowscale: bad arguments");
    if (nrows == 0) return PIRO_OK;
    k_rowscale<<<grid_for(nrows, 256, 8), 256, 0, as_stream(stream)>>>(nrows, rowptr, val, s);
    PIRO_CHECK_LAUNCH("k_rowscale");
    return PIRO_OK;
}

extern "C" int piro_csr_identity(int64_t N, int32_t *rowptr, int32_t *col, float *val, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && rowptr && col && val, "piro_csr_identity: bad arguments");
    k_identity<<<grid_for(N, 256, 8), 256, 0, as_stream(stream)>>>(N, rowptr, col, val);
    PIRO_CHECK_LAUNCH("k_identity");
    return PIRO_OK;
}

extern "C" int piro_face_count(int nx, int ny, int nz, int64_t *q, int64_t face_start[7])
{
    PIRO_ARG(q && grid_ok(nx, ny, nz), "piro_face_count: bad arguments");
    const int64_t a = (int64_t)(ny - 2) * (nz - 2), b = (int64_t)(nx - 2) * (nz - 2), c = (int64_t)(nx - 2) * (ny - 2);
    const int64_t len[6] = {a, a, b, b, c, c};
    if (face_start) {
        face_start[0] = 0;
        for (int f = 0; f < 6; ++f) face_start[f + 1] = face_start[f] + len[f];
    }
    *q = 2 * (a + b + c);
    return PIRO_OK;
}

extern "C" int piro_face_lists(int nx, int ny, int nz, uint32_t *idx, piro_stream_t stream)
{
    PIRO_ARG(idx && grid_ok(nx, ny, nz), "piro_face_lists: bad arguments");
    Grid g = make_grid(nx, ny, nz);
    const int64_t a = (int64_t)(ny - 2) * (nz - 2), b = (int64_t)(nx - 2) * (nz - 2), c = (int64_t)(nx - 2) * (ny - 2);
    const int64_t Q = 2 * (a + b + c);
    k_faces<<<grid_for(Q, 256, 4), 256, 0, as_stream(stream)>>>(g, a, b, c, idx);
    PIRO_CHECK_LAUNCH("k_faces");
    return PIRO_OK;
}

namespace piro {
namespace {
// dst[k*Ni + j] = src[k*N + cell(j)] for the interior cells j (x fastest) of
// each of ncomp components.
__global__ void k_interior_gather(int nx, int ny, int nz, int ncomp, const float *__restrict__ src,
                                  float *__restrict__ dst)
{
    const int64_t ix = nx - 2, iy = ny - 2, iz = nz - 2;
    const int64_t Ni = ix * iy * iz, N = (int64_t)nx * ny * nz;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < Ni * ncomp;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / Ni, j = t - k * Ni;
        const int64_t z = j / (ix * iy), rem = j - z * ix * iy;
        const int64_t y = rem / ix, x = rem - y * ix;
        dst[t] = src[k * N + (x + 1) + (y + 1) * nx + (z + 1) * (int64_t)nx * ny];
    }
}
}  // namespace
}  // namespace piro

extern "C" int piro_interior_gather(int nx, int ny, int nz, int ncomp, const float *src, float *dst,
                                    piro_stream_t stream)
{
    PIRO_ARG(src && dst && grid_ok(nx, ny, nz) && ncomp >= 1, "piro_interior_gather: bad arguments");
    const int64_t total = (int64_t)(nx - 2) * (ny - 2) * (nz - 2) * ncomp;
    k_interior_gather<<<grid_for(total, 256, 4), 256, 0, as_stream(stream)>>>(nx, ny, nz, ncomp, src, dst);
    PIRO_CHECK_LAUNCH("k_interior_gather");
    return PIRO_OK;
}
