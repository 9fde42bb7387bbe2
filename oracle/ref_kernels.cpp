// ref_kernels.cpp -- TEST INFRASTRUCTURE, not product code.
//
// Compiles PIRO's own OpenCL C kernels (dependencies/assets/kernels/*.cl, read
// in place from the reference tree through -I, never copied) as C++ and runs
// each NDRange as a loop over the global id, so that the reference's device
// arithmetic can be executed on the host and compared with the oracle and the
// CUDA path.  Each kernel lives in its own namespace because several .cl files
// define a helper with the same name (lookup in SpMVHT.cl and lu_decompHT.cl).
//
// The loop runs work-items in ascending global id, sequentially.  For the one
// kernel with a cross-item race (prefixsum.cl:12, launched N times by
// kernelcsrgeam.cpp:55-62) ascending order is the order that yields the
// intended inclusive scan.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>

namespace clshim {
thread_local size_t g_gid = 0, g_gid1 = 0;
inline size_t get_global_id(int d) { return d == 0 ? g_gid : g_gid1; }
inline int min(int a, int b) { return a < b ? a : b; }
inline float fabs(float a) { return std::fabs(a); }
}  // namespace clshim

#define __kernel
#define __global
#define __local
typedef unsigned int uint;

#define CL_UNIT(ns, file) \
    namespace ns {        \
    using namespace clshim; \
    _Pragma("GCC diagnostic push") _Pragma("GCC diagnostic ignored \"-Wall\"")

CL_UNIT(k_spmvcsr, "SpMVCSR.cl")
#include "SpMVCSR.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_spmvcsr_i1, "SpMVCSR_I1.cl")
#include "SpMVCSR_I1.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_spmvcoo, "SpMVCOO.cl")
#include "SpMVCOO.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_spmvht, "SpMVHT.cl")
#include "SpMVHT.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_add, "addVectors.cl")
#include "addVectors.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_sub, "subtractVectors.cl")
#include "subtractVectors.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_urf, "addVectors_URF.cl")
#include "addVectors_URF.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_g1, "csrgeam_1.cl")
#include "csrgeam_1.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_ps, "prefixsum.cl")
#include "prefixsum.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_g3, "csrgeam_3.cl")
#include "csrgeam_3.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_g2, "csrgeam_2.cl")
#include "csrgeam_2.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_dense, "SpMVDENSE.cl")
#include "SpMVDENSE.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_spmdsm, "SpMDSM.cl")
#include "SpMDSM.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_setbc, "setBC.cl")
#include "setBC.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_lapsc, "laplacianscalar.cl")
#include "laplacianscalar.cl"
_Pragma("GCC diagnostic pop") }
CL_UNIT(k_lu, "lu_decompHT.cl")
#include "lu_decompHT.cl"
_Pragma("GCC diagnostic pop") }

#define NDRANGE(n, call)                                         \
    for (size_t gid_ = 0; gid_ < (size_t)(n); ++gid_) {          \
        clshim::g_gid = gid_;                                    \
        call;                                                    \
    }

// The same NDRange over the host's OpenMP threads, for kernels whose
// work-items write only their own row (the CPU baseline of the SpMV steps):
// each thread sets its own get_global_id (g_gid is thread-local).
#define NDRANGE_OMP(n, call)                                     \
    _Pragma("omp parallel for schedule(static)")                 \
    for (long gid_ = 0; gid_ < (long)(n); ++gid_) {              \
        clshim::g_gid = (size_t)gid_;                            \
        call;                                                    \
    }

#define NDRANGE2(n0, n1, call)                                   \
    for (size_t g1_ = 0; g1_ < (size_t)(n1); ++g1_)              \
        for (size_t g0_ = 0; g0_ < (size_t)(n0); ++g0_) {        \
            clshim::g_gid = g0_;                                 \
            clshim::g_gid1 = g1_;                                \
            call;                                                \
        }

extern "C" {

void refcl_spmvcsr(int M, const float *val, const int *col, const int *rp, float dt, float *B, float *C,
                   unsigned nx, unsigned ny, unsigned size)
{
    NDRANGE(M, k_spmvcsr::SpMVCSR(M, M, 1, val, col, rp, dt, B, C, nx, ny, size));
}

void refcl_spmvcsr_i1(int M, const float *val, const int *col, const int *rp, float dt, float *B, float *C,
                      unsigned nx, unsigned ny, unsigned size)
{
    // global size N, kernel guard `row > M` (SpMVCSR_I1.cl:14) never trips
    NDRANGE(M, k_spmvcsr_i1::SpMVCSR_I1(M, M, 1, val, col, rp, dt, B, C, nx, ny, size));
}

void refcl_spmvcoo(int M, int nnz, const float *val, const int *col, const int *rows, float dt, float *B,
                   float *C, unsigned nx, unsigned ny, unsigned size)
{
    NDRANGE(M, k_spmvcoo::SpMVCOO(M, M, nnz, val, col, rows, dt, B, C, nx, ny, size));
}

void refcl_spmvht(int *keys, float *vals, const float *B, float *C, int N, int TS, float dt)
{
    NDRANGE(N, k_spmvht::SpMVHT(keys, vals, B, C, N, TS, dt));
}

// The three SpMV kernels over all OpenMP threads (omp_set_num_threads picks
// the count): every work-item reads the shared inputs and writes C[gid] only.
void refcl_spmvcsr_par(int M, const float *val, const int *col, const int *rp, float dt, float *B, float *C,
                       unsigned nx, unsigned ny, unsigned size)
{
    NDRANGE_OMP(M, k_spmvcsr::SpMVCSR(M, M, 1, val, col, rp, dt, B, C, nx, ny, size));
}

void refcl_spmvcoo_par(int M, int nnz, const float *val, const int *col, const int *rows, float dt, float *B,
                       float *C, unsigned nx, unsigned ny, unsigned size)
{
    NDRANGE_OMP(M, k_spmvcoo::SpMVCOO(M, M, nnz, val, col, rows, dt, B, C, nx, ny, size));
}

void refcl_spmvht_par(int *keys, float *vals, const float *B, float *C, int N, int TS, float dt)
{
    NDRANGE_OMP(N, k_spmvht::SpMVHT(keys, vals, B, C, N, TS, dt));
}

void refcl_add(float *A, const float *B, const float *C, unsigned n) { NDRANGE(n, k_add::addVectors(A, B, C, n)); }
void refcl_sub(float *A, const float *B, const float *C, unsigned n) { NDRANGE(n, k_sub::subtractVectors(A, B, C, n)); }
void refcl_urf(float *A, float *C, float urf, unsigned n)
{
    // launched over N work-items (kernelprocess.cpp:184-189); guard `id > size`
    NDRANGE(n, k_urf::addVectors_URF(A, C, urf, n));
}

// kernelmethods::csrgeam (kernelcsrgeam.cpp:9-86): count, N scan launches,
// fill.  rpD must hold N+1 ints, cD/vD 3*nnz_x entries, all zero on entry.
void refcl_csrgeam(int N, const int *rpA, const int *cA, const float *vA, const int *rpB, const int *cB,
                   const float *vB, const int *rpC, const int *cC, const float *vC, const float *v, int *count,
                   int *rpD, int *cD, float *vD)
{
    NDRANGE(N, k_g1::csrgeam_1(cA, rpA, cB, rpB, cC, rpC, count, N));
    for (int i = 0; i < N; ++i) rpD[i + 1] = count[i];  // clEnqueueCopyBuffer, :53
    for (int row = 0; row < N; ++row) NDRANGE(N, k_ps::prefixsum(count, rpD, N, row));
    NDRANGE(N, k_g3::csrgeam_3(vA, cA, rpA, vB, cB, rpB, vC, cC, rpC, vD, cD, rpD, count, v, N));
}

// kernelmethods::csrgeam_2's merge (kernelcsrgeam.cpp:142-203): the same
// count and scan as csrgeam, then csrgeam_2.cl (no vector scaling).
void refcl_csrgeam2_merge(int N, const int *rpA, const int *cA, const float *vA, const int *rpB, const int *cB,
                          const float *vB, const int *rpC, const int *cC, const float *vC, int *rpD, int *cD,
                          float *vD, int *count)
{
    NDRANGE(N, k_g1::csrgeam_1(cA, rpA, cB, rpB, cC, rpC, count, N));
    rpD[0] = 0;
    for (int i = 0; i < N; ++i) rpD[i + 1] = count[i];
    for (int row = 0; row < N; ++row) NDRANGE(N, k_ps::prefixsum(count, rpD, N, row));
    NDRANGE(N, k_g2::csrgeam_2(vA, cA, rpA, vB, cB, rpB, vC, cC, rpC, vD, cD, rpD, count, N));
}

// kernelsolve::DENSE::TIMESCHEME_11 (kernelprocess.cpp:42-66): SpMVDENSE over
// the (N, N) range with P = 1 (only id(0) = 0 does work), then addVectors.
void refcl_fe_dense(int N, const float *A, float *B, float *C, float *D, float dt)
{
    NDRANGE2(N, N, k_dense::SpMVDENSE(A, B, C, (uint)N, (uint)N, 1u, dt));
    NDRANGE(N, k_add::addVectors(D, B, C, (unsigned)N));
}

void refcl_spmdsm(int nnz, int M, float *val, const int *col, const int *rp, const float *diag, int ind)
{
    // global size nnz; guard `index > nnz` (SpMDSM.cl:28) never trips
    NDRANGE(nnz, k_spmdsm::SpMDSM(nnz, M, val, col, rp, diag, ind));
}

void refcl_setbc(float *A, const float *B, unsigned *idx, unsigned q) { NDRANGE(q, k_setbc::setBC(A, B, idx, q)); }

void refcl_laplacianscalar(float *B, float *C, float dx, float dy, float dz, unsigned nx, unsigned ny, float dt,
                           unsigned size)
{
    NDRANGE(size, k_lapsc::laplacianscalar(B, C, dx, dy, dz, nx, ny, dt, size));
}

void refcl_lu_round(int *keys, float *vals, int N, int rowouter, int TS, int limit)
{
    // Work-items of one round run concurrently on a device.  The only
    // intra-round hazard is item (r, rowouter) rewriting a(r, rowouter), the
    // factor every other item of row r reads (lu_decompHT.cl:52-59).  Running
    // the ids in DESCENDING order gives every item the pre-round values, the
    // outcome the kernel intends.  Ids run 0..limit-1; the guard `gid > limit`
    // (:33) would also admit gid == limit, which addresses row N and is a no-op.
    for (long g = (long)limit - 1; g >= 0; --g) {
        clshim::g_gid = (size_t)g;
        k_lu::lu_decompHT(keys, vals, N, rowouter, TS, limit);
    }
}

}  // extern "C"
