// ref_driver.cpp -- TEST INFRASTRUCTURE, not product code.
//
// extern "C" entry points that call PIRO's own host code, linked from the
// reference's translation units (oracle/Makefile builds them in place from
// the reference tree into oracle/_ref/).  They set the singletons the
// reference functions read and call the stencil, hash and boundary routines
// directly; the OpenCL upload steps around them are skipped.  Used to pin the
// C restatement in piro_oracle.c and to generate tests/golden/ fixtures.
#include <filesystem>
#include <bc.hpp>
#include <ic.hpp>
#include <datatypes.hpp>
#include <fileutilities.hpp>
#include <methods.hpp>
#include <openclutilities.hpp>
#include <postprocess.hpp>
#include <stencils.hpp>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {
void set_grid(int nx, int ny, int nz)
{
    Piro::MeshParams &MP = Piro::MeshParams::getInstance();
    MP.setvalue(Piro::MeshParams::num_cells, std::vector<uint>{(uint)nx, (uint)ny, (uint)nz});
}
}  // namespace

extern "C" {

// fmt: 0 CSR, 2 HT row pushes, 3 COO (stencils.cpp:233-429, 797-993, 572-795)
// scheme: 1 uw, 2 dw, 3 cd.  Output arrays must hold 7N entries.
long long ref_laplacian(int fmt, int nx, int ny, int nz, int scheme, float norm, int *rowptr, int *rows, int *col,
                        float *val)
{
    set_grid(nx, ny, nz);
    std::vector<uint> n{(uint)nx, (uint)ny, (uint)nz};
    const int N = nx * ny * nz;
    Piro::CellData cd;
    cd.rowpointers.assign(N + 1, 0);  // operatorlaplacian.cpp:30
    if (fmt == 0) {
        if (scheme == 3) Piro::CSR::stencils::laplacian_cd(cd, n, norm);
        else if (scheme == 2) Piro::CSR::stencils::laplacian_dw(cd, n, norm);
        else if (scheme == 1) Piro::CSR::stencils::laplacian_uw(cd, n, norm);
    } else if (fmt == 2) {
        if (scheme == 3) Piro::HT::stencils::laplacian_cd(cd, n, norm);
        else if (scheme == 2) Piro::HT::stencils::laplacian_dw(cd, n, norm);
        else if (scheme == 1) Piro::HT::stencils::laplacian_uw(cd, n, norm);
    } else if (fmt == 3) {
        if (scheme == 3) Piro::COO::stencils::laplacian_cd(cd, n, norm);
        else if (scheme == 2) Piro::COO::stencils::laplacian_dw(cd, n, norm);
        else if (scheme == 1) Piro::COO::stencils::laplacian_uw(cd, n, norm);
    }
    const size_t nnz = cd.values.size();
    if (rowptr && fmt != 3) std::memcpy(rowptr, cd.rowpointers.data(), sizeof(int) * (N + 1));
    if (rows && fmt == 3) std::memcpy(rows, cd.rows.data(), sizeof(int) * nnz);
    std::memcpy(col, cd.columns.data(), sizeof(int) * nnz);
    std::memcpy(val, cd.values.data(), sizeof(float) * nnz);
    return (long long)nnz;
}

// The three gradient matrices in the order operatorgradient.cpp:35-104 builds
// them, sharing one rowpointers vector.  rp holds 3*(N+1) ints; col/val hold
// 3*2N entries; nnz3 receives the three counts.
void ref_gradient(int nx, int ny, int nz, int scheme, float norm, int *rp, int *col, float *val, long long *nnz3)
{
    set_grid(nx, ny, nz);
    std::vector<uint> n{(uint)nx, (uint)ny, (uint)nz};
    const int N = nx * ny * nz;
    Piro::CellData cd;
    cd.rowpointers.assign(N + 1, 0);
    size_t off = 0;
    for (int axis = 0; axis < 3; ++axis) {
        cd.columns.clear();
        cd.values.clear();
        if (axis == 0) {
            if (scheme == 3) Piro::CSR::stencils::gradient_cd_x(cd, n, norm);
            else if (scheme == 2) Piro::CSR::stencils::gradient_dw_x(cd, n, norm);
            else if (scheme == 1) Piro::CSR::stencils::gradient_uw_x(cd, n, norm);
        } else if (axis == 1) {
            if (scheme == 3) Piro::CSR::stencils::gradient_cd_y(cd, n, norm);
            else if (scheme == 2) Piro::CSR::stencils::gradient_dw_y(cd, n, norm);
            else if (scheme == 1) Piro::CSR::stencils::gradient_uw_y(cd, n, norm);
        } else {
            if (scheme == 3) Piro::CSR::stencils::gradient_cd_z(cd, n, norm);
            else if (scheme == 2) Piro::CSR::stencils::gradient_dw_z(cd, n, norm);
            else if (scheme == 1) Piro::CSR::stencils::gradient_uw_z(cd, n, norm);
        }
        std::memcpy(rp + axis * (N + 1), cd.rowpointers.data(), sizeof(int) * (N + 1));
        std::memcpy(col + off, cd.columns.data(), sizeof(int) * cd.columns.size());
        std::memcpy(val + off, cd.values.data(), sizeof(float) * cd.values.size());
        nnz3[axis] = (long long)cd.values.size();
        off += cd.values.size();
    }
}

// The three divergence matrices as Piro::CSR::div builds them
// (operatordivergenceCSR.cpp:21-101: div_*_x/y/z, one rowpointers vector,
// norm = 2*(l0/(n0-2))).  Same layout as ref_gradient.
void ref_div(int nx, int ny, int nz, int scheme, float norm, int *rp, int *col, float *val, long long *nnz3)
{
    set_grid(nx, ny, nz);
    std::vector<uint> n{(uint)nx, (uint)ny, (uint)nz};
    const int N = nx * ny * nz;
    Piro::CellData cd;
    cd.rowpointers.assign(N + 1, 0);
    size_t off = 0;
    for (int axis = 0; axis < 3; ++axis) {
        cd.columns.clear();
        cd.values.clear();
        if (axis == 0) {
            if (scheme == 3) Piro::CSR::stencils::div_cd_x(cd, n, norm);
            else if (scheme == 2) Piro::CSR::stencils::div_dw_x(cd, n, norm);
            else if (scheme == 1) Piro::CSR::stencils::div_uw_x(cd, n, norm);
        } else if (axis == 1) {
            if (scheme == 3) Piro::CSR::stencils::div_cd_y(cd, n, norm);
            else if (scheme == 2) Piro::CSR::stencils::div_dw_y(cd, n, norm);
            else if (scheme == 1) Piro::CSR::stencils::div_uw_y(cd, n, norm);
        } else {
            if (scheme == 3) Piro::CSR::stencils::div_cd_z(cd, n, norm);
            else if (scheme == 2) Piro::CSR::stencils::div_dw_z(cd, n, norm);
            else if (scheme == 1) Piro::CSR::stencils::div_uw_z(cd, n, norm);
        }
        std::memcpy(rp + axis * (N + 1), cd.rowpointers.data(), sizeof(int) * (N + 1));
        std::memcpy(col + off, cd.columns.data(), sizeof(int) * cd.columns.size());
        std::memcpy(val + off, cd.values.data(), sizeof(float) * cd.values.size());
        nnz3[axis] = (long long)cd.values.size();
        off += cd.values.size();
    }
}

// Piro::DENSE::stencils::laplacian_* (stencils.cpp:431-570) into A[N*N].
void ref_dense_laplacian(int nx, int ny, int nz, int scheme, float norm, float *A)
{
    set_grid(nx, ny, nz);
    std::vector<uint> n{(uint)nx, (uint)ny, (uint)nz};
    const size_t N = (size_t)nx * ny * nz;
    Piro::CellData cd;
    cd.matrix.resize(N * N);  // operatorlaplacian.cpp:79
    if (scheme == 3) Piro::DENSE::stencils::laplacian_cd(cd, n, norm);
    else if (scheme == 2) Piro::DENSE::stencils::laplacian_dw(cd, n, norm);
    else if (scheme == 1) Piro::DENSE::stencils::laplacian_uw(cd, n, norm);
    std::memcpy(A, cd.matrix.data(), sizeof(float) * N * N);
}

// Piro::methods::sethash on an int32 table (methods.cpp:74-118), fed in the
// row-major order of operatorlaplacian.cpp:190-203.  keys/vals hold TS.
int ref_ht_insert_all(int N, const int *rowptr, const int *col, const float *val, int TS, int *keys, float *vals)
{
    std::vector<int> k(TS, -1);
    std::vector<float> v(TS, 0.0f);
    for (int i = 0; i < N; i++)
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) Piro::methods::sethash(i * N + col[j], val[j], TS, k, v);
    std::memcpy(keys, k.data(), sizeof(int) * TS);
    std::memcpy(vals, v.data(), sizeof(float) * TS);
    return 0;
}

float ref_ht_lookup(int row, int coln, int N, const int *keys, const float *vals, int TS)
{
    std::vector<int> k(keys, keys + TS);
    std::vector<float> v(vals, vals + TS);
    return Piro::methods::lookup(row, coln, N, k, v, TS);
}

// methods::lookupandset (methods.cpp:35-72), used by the scheme-27 fill-in.
int ref_ht_lookupandset(int row, int coln, int N, float value, int *keys, float *vals, int TS)
{
    std::vector<int> k(keys, keys + TS);
    std::vector<float> v(vals, vals + TS);
    int rc = Piro::methods::lookupandset(row, coln, N, value, k, v, TS);
    std::memcpy(keys, k.data(), sizeof(int) * TS);
    std::memcpy(vals, v.data(), sizeof(float) * TS);
    return rc;
}

// bc::initbc (bc.cpp:107-157) for a case with one constant (index 0) and one
// scalar (index 1), reading [BC] from <assets_root>/assets/setup.ini exactly as
// the reference does.  idx receives the flat face list (Q entries, faces 0..5
// concatenated, bc.cpp:27-30); face_len[6] the per-face counts; field (N
// floats) the scalar after setbc() wrote the boundary values into it.
long long ref_initbc(int nx, int ny, int nz, const char *assets_root, const char *scalar_name, int *idx,
                     int *face_len, float *field)
{
    set_grid(nx, ny, nz);
    const int N = nx * ny * nz;
    Piro::file_utilities::current_path = std::string(assets_root);
    Piro::MeshParams &MP = Piro::MeshParams::getInstance();
    std::vector<Piro::AMR> amr(1);
    Piro::CellData c0, c1;
    c0.Scalars = "Alpha";
    c0.values.assign(N, 0.0f);
    c1.Scalars = scalar_name;
    c1.values.assign(N, 0.0f);
    amr[0].CD.push_back(c0);
    amr[0].CD.push_back(c1);
    MP.setvalue(Piro::MeshParams::AMR, amr);
    Piro::kernels::getInstance().setvalue(Piro::kernels::CONTEXT, (cl_context) nullptr);
    Piro::bc::initbc();
    Piro::bc::indices &indval = Piro::bc::indices::getInstance();
    auto lists = indval.getvalue<std::vector<std::vector<int>>>(Piro::bc::indices::IND);
    long long q = 0;
    for (int f = 0; f < 6; ++f) {
        face_len[f] = (int)lists[f].size();
        for (int e : lists[f]) idx[q++] = e;
    }
    auto &cd1 = MP.getvalue<std::vector<Piro::AMR>>(Piro::MeshParams::AMR)[0].CD[1];
    std::memcpy(field, cd1.values.data(), sizeof(float) * N);
    return q;
}

// Piro::initialcondition(0) (src/ic.cpp:34-99) for one field whose [IC]
// filename entry is `ic_name`, reading <assets_root>/assets/IC/distribution.ini.
// out must hold 3N floats; returns the number of values produced.
long long ref_initialcondition(int nx, int ny, int nz, float l0, float l1, float l2, const char *assets_root,
                               const char *ic_name, float *out)
{
    set_grid(nx, ny, nz);
    Piro::file_utilities::current_path = std::string(assets_root);
    Piro::MeshParams &MP = Piro::MeshParams::getInstance();
    MP.setvalue(Piro::MeshParams::L, std::vector<float>{l0, l1, l2});
    MP.setvalue(Piro::MeshParams::ICFILES, std::vector<std::string>{std::string(ic_name)});
    std::vector<float> v = Piro::initialcondition(0);
    std::memcpy(out, v.data(), sizeof(float) * v.size());
    return (long long)v.size();
}

// Piro::paraview::writevth (src/paraview.cpp:106-137) for a one-level mesh:
// the fields of AMR[0].CD (constants type 0, scalars type 1, vectors type 2,
// vectors holding 3N values), then the three operator slots preprocess.cpp
// appends; bc::prepbc() supplies the boundary cells to strip.  Files go under
// <dir>/<casename>/mesh/ (the directories must exist).
void ref_paraview(int nx, int ny, int nz, int ox, int oy, int oz, int sx, int sy, int sz, const char *dir,
                  const char *casename, int timestep, int nfields, const char *const *names, const int *types,
                  const float *const *values)
{
    set_grid(nx, ny, nz);
    const long long N = (long long)nx * ny * nz;
    Piro::file_utilities::current_path = std::string(dir);
    Piro::MeshParams &MP = Piro::MeshParams::getInstance();
    Piro::SolveParams &SP = Piro::SolveParams::getInstance();
    SP.setvalue(Piro::SolveParams::CASENAME, std::string(casename));
    MP.setvalue(Piro::MeshParams::LEVELS, 1);
    MP.setvalue(Piro::MeshParams::INDEX, std::vector<int>{1});
    int nvec = 0;
    Piro::AMR amr;
    amr.WholeExtent[0] = 0; amr.WholeExtent[1] = nx;
    amr.WholeExtent[2] = 0; amr.WholeExtent[3] = ny;
    amr.WholeExtent[4] = 0; amr.WholeExtent[5] = nz;
    amr.Origin[0] = ox; amr.Origin[1] = oy; amr.Origin[2] = oz;
    amr.Spacing[0] = sx; amr.Spacing[1] = sy; amr.Spacing[2] = sz;
    for (int f = 0; f < nfields; ++f) {
        Piro::CellData cd;
        cd.type = types[f];
        cd.Scalars = names[f];
        const long long cnt = types[f] == 2 ? 3 * N : N;
        cd.values.assign(values[f], values[f] + cnt);
        if (types[f] == 2) ++nvec;
        amr.CD.push_back(cd);
    }
    for (int k = 0; k < 3; ++k) amr.CD.push_back(Piro::CellData());
    MP.setvalue(Piro::MeshParams::VECTORNUM, nvec);
    MP.setvalue(Piro::MeshParams::AMR, std::vector<Piro::AMR>{amr, Piro::AMR()});
    Piro::bc::prepbc();
    Piro::paraview::writevth(timestep);
}

void refcl_lu_round(int *keys, float *vals, int N, int rowouter, int TS, int limit);

// Scheme 27's factorization (src/matrixoperations.cpp:37-99): per pivot row,
// the reference's host fill-in with methods::lookup / lookupandset on the
// table, then one lu_decompHT.cl round (refcl_lu_round, ids descending).  The
// reference's OpenCL upload/download around each round is an identity here.
// The table gets one spare slot before it: an item whose own key is absent
// writes slot -1 in the reference (lu_decompHT.cl:61-64), here that spare.
void ref_ht_lu(int N, int *keys, float *vals, int TS)
{
    std::vector<int> K(TS + 1, -1);
    std::vector<float> V(TS + 1, 0.0f);
    std::memcpy(K.data() + 1, keys, sizeof(int) * TS);
    std::memcpy(V.data() + 1, vals, sizeof(float) * TS);
    std::vector<int> k(K.begin() + 1, K.end());
    std::vector<float> v(V.begin() + 1, V.end());
    for (int ro = 0; ro < N - 1; ++ro) {
        std::vector<int> cols;
        for (int co = ro; co < N; co++)
            if (std::abs(Piro::methods::lookup(ro, co, N, k, v, TS)) > 1E-6) cols.push_back(co);
        for (int r = ro + 1; r < N; ++r) {
            if (Piro::methods::lookup(r, ro, N, k, v, TS) == 0.0) continue;
            for (int col : cols) Piro::methods::lookupandset(r, col, N, 0.0f, k, v, TS);
        }
        std::copy(k.begin(), k.end(), K.begin() + 1);
        std::copy(v.begin(), v.end(), V.begin() + 1);
        refcl_lu_round(K.data() + 1, V.data() + 1, N, ro, TS, (N - ro - 1) * (N - ro));
        std::copy(K.begin() + 1, K.end(), k.begin());
        std::copy(V.begin() + 1, V.end(), v.begin());
    }
    std::memcpy(keys, k.data(), sizeof(int) * TS);
    std::memcpy(vals, v.data(), sizeof(float) * TS);
}

}  // extern "C"
