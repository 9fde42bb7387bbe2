// context.cpp -- layer 2 of the C ABI: PIRO's operator API over a case .ini.
//
// One piro_ctx is one PIRO run: the .ini case file and its companion files
// are read the way src/preprocess.cpp:20-208 reads them, fields are created
// with their initial conditions (src/ic.cpp) and boundary values
// (src/bc.cpp:107-157), and the operator calls of src/solve.cpp
// -- ddt_r, laplacian, gradient, vector, operator&, operator=, Solve --
// map to piro_ddt_r ... piro_step_solve.  All device work goes through the
// layer-1 kernel entry points; the context owns every device buffer it uses
// (the reference leaks two N-float buffers per operator= call; here they are
// allocated once).  Host work is limited to parsing, the initial-condition
// and boundary-value setup (host float/double arithmetic as in the
// reference), and the control flow of the time loop.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "piro.h"

namespace piro {
void set_error(const char *fmt, ...);
}

namespace {

// ---------------------------------------------------------------- .ini
// IniReader semantics (src/fileutilities.cpp:124-183): trim spaces only,
// ';' or '#' lines are comments, "[section]" headers, key=value at the first
// '=', a later duplicate key replaces an earlier one.
using Ini = std::map<std::string, std::map<std::string, std::string>>;

std::string trim_spaces(const std::string &s)
{
    const size_t a = s.find_first_not_of(' ');
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(' ');
    return s.substr(a, b - a + 1);
}

bool read_ini(const std::string &path, Ini &ini)
{
    std::ifstream f(path);
    if (!f.is_open()) return false;
    std::string line, section;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        line = trim_spaces(line);
        if (line.empty() || line[0] == ';' || line[0] == '#') continue;
        if (line[0] == '[' && line.back() == ']') {
            section = line.substr(1, line.size() - 2);
        } else {
            const size_t eq = line.find('=');
            if (eq != std::string::npos) ini[section][trim_spaces(line.substr(0, eq))] = trim_spaces(line.substr(eq + 1));
        }
    }
    return true;
}

bool ini_get(const Ini &ini, const std::string &sec, const std::string &key, std::string &out)
{
    auto s = ini.find(sec);
    if (s == ini.end()) return false;
    auto k = s->second.find(key);
    if (k == s->second.end()) return false;
    out = k->second;
    return true;
}

// splitString(str, ' ') (src/stringutilities.cpp:9-20): single-space split.
std::vector<std::string> split_spaces(const std::string &s)
{
    std::vector<std::string> out;
    size_t a = 0, b;
    while ((b = s.find(' ', a)) != std::string::npos) {
        out.push_back(s.substr(a, b - a));
        a = b + 1;
    }
    out.push_back(s.substr(a));
    return out;
}

// convertStringVectorTo{Float,Int} (:22-75): tokens that do not parse are skipped.
template <class T>
std::vector<T> parse_list(const std::string &s)
{
    std::vector<T> out;
    for (const std::string &t : split_spaces(s)) {
        std::istringstream is(t);
        T v;
        if (is >> v) out.push_back(v);
    }
    return out;
}

int count_spaces(const std::string &s)
{
    int n = 0;
    for (char c : s) n += c == ' ';
    return n;
}

int count_words(const std::string &s)
{
    std::istringstream is(s);
    int n = 0;
    std::string w;
    while (is >> w) ++n;
    return n;
}

struct Field {
    std::string name;
    int kind = 0;  // 0 constant, 1 scalar, 2 vector
    int64_t n = 0;
    float *d = nullptr;
    std::vector<float> host;  // values after initial condition and setbc (CellData::values)
};

struct Csr {
    int32_t *rp = nullptr, *col = nullptr;
    float *val = nullptr;
    int64_t nnz = 0;
};

}  // namespace

// ------------------------------------------------------------------- context
struct piro_ctx {
    std::string assets;
    Ini cfg;
    int nx = 0, ny = 0, nz = 0;
    int64_t N = 0;
    std::vector<float> l;
    int timescheme = 0, spacescheme = 0, solverscheme = 0, simindex = 0, datatype = 0, save = 1;
    float timestep = 0.0f, totaltime = 0.0f;
    float jli_tol = 0.0f, jli_urf = 1.0f;
    int jli_maxiter = 0;
    float ht_a = 0, ht_b = 0, ht_c = 0, ht_lf = 0.7f;
    int alpha_mode = 0;  // 0 intended (SpMDSM row scale), 1 as the reference runs (alpha dropped)
    int lu_mode = 0;     // scheme 27: 0 solve by the banded LU, 1 as the reference runs (factor only, zero field)
    std::vector<Field> fields;
    int nconst = 0, nscalar = 0, nvector = 0;
    // boundary
    int64_t q = 0;
    uint32_t *bc_idx = nullptr;
    float *memD = nullptr;
    // operators (cached on first use, like the INIT flags of preprocess.hpp:105-122)
    bool lap_init = false, grad_init = false, dot_init = false, div_init = false;
    Csr lap, grad[3], dot, divm, be_A;
    float *dense = nullptr;  // DENSE Laplacian, N x N row-major (Data 1)
    int32_t *coo_rows = nullptr;
    int32_t *coo_rowstart = nullptr;  // first entry of each row (piro_coo_row_index)
    int64_t *ht_keys = nullptr;
    float *ht_vals = nullptr;
    int64_t ht_ts = 0;
    int32_t *ht_order = nullptr;  // rows by the home slot of their keys (piro_ht_row_order)
    float *ht_stage = nullptr;    // 32 bytes per row for piro_ht_spmv_staged
    // scheme 27: factorized once (INIT::RHS_INIT, operatoroverload.cpp:68-81)
    bool lu_done = false;
    void *lu_band = nullptr;
    size_t lu_band_bytes = 0;
    int64_t lu_bw = 0;
    int lap_coeff = -1;
    // equation result (partD) and scratch (partC)
    float *partD = nullptr, *partC = nullptr;
    piro_be_solver *be = nullptr;
    int64_t steps = 0;
    // ParaView output (Piro::paraview, src/paraview.cpp): [File] casename and
    // restart, [Mesh] o, s, levels, index; written when an output root is set
    std::string casename = "case", out_root;
    int restart = 0, levels = 1;
    int origin[3] = {0, 0, 0}, spacing[3] = {1, 1, 1};
    std::vector<int> index{1};
    cudaStream_t stream = nullptr;
    void *work = nullptr;
    size_t work_bytes = 0;
};

namespace {

int fail(int code, const char *fmt, const std::string &a = "", const std::string &b = "")
{
    piro::set_error(fmt, a.c_str(), b.c_str());
    return code;
}

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(PIRO_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define PK(call)                   \
    do {                           \
        int r_ = (call);           \
        if (r_ != PIRO_OK) return r_; \
    } while (0)

int need(const Ini &ini, const char *sec, const char *key, std::string &out)
{
    if (!ini_get(ini, sec, key, out))
        return fail(PIRO_ERR_CONFIG, "missing [%s] %s in the case files", sec, key);
    return PIRO_OK;
}

int need_int(const Ini &ini, const char *sec, const char *key, int &out)
{
    std::string s;
    PK(need(ini, sec, key, s));
    try {
        out = std::stoi(s);
    } catch (...) {
        return fail(PIRO_ERR_CONFIG, "[%s] %s is not an integer", sec, key);
    }
    return PIRO_OK;
}

int need_float(const Ini &ini, const char *sec, const char *key, float &out)
{
    std::string s;
    PK(need(ini, sec, key, s));
    try {
        out = std::stof(s);
    } catch (...) {
        return fail(PIRO_ERR_CONFIG, "[%s] %s is not a number", sec, key);
    }
    return PIRO_OK;
}

// Initial conditions (src/ic.cpp:34-99): coordinates x*l/(float)n with
// ghost-inclusive n; the float/double mix of calculategaussian and
// calculatecoulomb is kept.
int initial_condition(piro_ctx *c, const std::string &kind, std::vector<float> &v)
{
    Ini dist;
    if (!read_ini(c->assets + "/IC/distribution.ini", dist))
        return fail(PIRO_ERR_CONFIG, "cannot read %s/IC/distribution.ini", c->assets);
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const float l0 = c->l[0], l1 = c->l[1], l2 = c->l[2];
    auto at = [&](int x, int y, int z) { return (size_t)x + (size_t)y * nx + (size_t)z * nx * ny; };
    if (kind == "Gaussian") {
        float scale;
        std::string ss, sm;
        PK(need_float(dist, "Gaussian", "Scalefactor", scale));
        PK(need(dist, "Gaussian", "Sigma", ss));
        PK(need(dist, "Gaussian", "Median", sm));
        const std::vector<float> sg = parse_list<float>(ss), mn = parse_list<float>(sm);
        if (sg.size() < 3 || mn.size() < 3) return fail(PIRO_ERR_CONFIG, "[Gaussian] Sigma/Median need 3 values");
        v.assign((size_t)c->N, 0.0f);
        const float norm = (float)(1.0f / (std::pow(2.0f * M_PI, 1.5f) * sg[0] * sg[1] * sg[2]));
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    const float cx = x * l0 / (float)nx, cy = y * l1 / (float)ny, cz = z * l2 / (float)nz;
                    const float a = (cx - mn[0]) / sg[0], b = (cy - mn[1]) / sg[1], d = (cz - mn[2]) / sg[2];
                    const float e = -0.5f * (a * a + b * b + d * d);
                    v[at(x, y, z)] = scale * (norm * std::exp(e));
                }
        return PIRO_OK;
    }
    if (kind == "Coulomb") {
        std::string sc;
        float Z, ef, epsf;
        PK(need(dist, "Coulomb", "center", sc));
        PK(need_float(dist, "Coulomb", "Z", Z));
        PK(need_float(dist, "Coulomb", "e", ef));
        PK(need_float(dist, "Coulomb", "epsilon_0", epsf));
        const std::vector<float> ctr = parse_list<float>(sc);
        if (ctr.size() < 3) return fail(PIRO_ERR_CONFIG, "[Coulomb] center needs 3 values");
        const double e = ef, eps0 = epsf;
        v.assign((size_t)c->N, 0.0f);
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    const float cx = x * l0 / (float)nx, cy = y * l1 / (float)ny, cz = z * l2 / (float)nz;
                    const float r = (float)std::pow(std::pow((double)(cx - ctr[0]), 2.0) +
                                                        std::pow((double)(cy - ctr[1]), 2.0) +
                                                        std::pow((double)(cz - ctr[2]), 2.0),
                                                    0.5);
                    v[at(x, y, z)] =
                        (float)(-((double)Z * 1E15 * std::pow(e, 2.0)) / (4 * M_PI * eps0 * ((double)r + 1E-10)));
                }
        return PIRO_OK;
    }
    if (kind == "UniformVector") {
        std::string sd, sv;
        PK(need(dist, "Vector", "Direction", sd));
        PK(need(dist, "Vector", "Value", sv));
        const std::vector<float> dir = parse_list<float>(sd), val = parse_list<float>(sv);
        if (dir.size() < 3 || val.empty()) return fail(PIRO_ERR_CONFIG, "[Vector] Direction/Value malformed");
        v.assign((size_t)c->N * 3, 0.0f);
        for (int dd = 0; dd < 3; ++dd)
            for (int64_t i = 0; i < c->N; ++i) v[(size_t)(dd * c->N + i)] = dir[dd] * val[0];
        return PIRO_OK;
    }
    return fail(PIRO_ERR_CONFIG, "unknown initial condition '%s' (Gaussian, Coulomb, UniformVector)", kind);
}

// process::matchscalartovar (src/process.cpp:20-27): index of the field
// named `var`, 0 when there is none.
int match_field(const piro_ctx *c, const std::string &var)
{
    for (size_t i = 0; i < c->fields.size(); ++i)
        if (c->fields[i].name == var) return (int)i;
    return 0;
}

int ensure_work(piro_ctx *c, size_t bytes)
{
    if (c->work_bytes >= bytes) return PIRO_OK;
    cudaFree(c->work);
    c->work = nullptr;
    c->work_bytes = 0;
    CK(cudaMalloc(&c->work, bytes));
    c->work_bytes = bytes;
    return PIRO_OK;
}

int alloc_csr(Csr &m, int64_t N, int64_t nnz)
{
    CK(cudaMalloc(&m.rp, sizeof(int32_t) * (size_t)(N + 1)));
    CK(cudaMalloc(&m.col, sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1)));
    CK(cudaMalloc(&m.val, sizeof(float) * (size_t)(nnz > 0 ? nnz : 1)));
    m.nnz = nnz;
    return PIRO_OK;
}

void free_csr(Csr &m)
{
    cudaFree(m.rp);
    cudaFree(m.col);
    cudaFree(m.val);
    m = Csr();
}

// The host half of opening a case: the .ini files, the fields' initial
// values.  No CUDA call, so a malformed case reports PIRO_ERR_CONFIG on any
// machine.
int parse_case(piro_ctx *c, const std::string &case_name)
{
    if (!read_ini(c->assets + "/" + case_name, c->cfg))
        return fail(PIRO_ERR_CONFIG, "cannot read case file %s/%s", c->assets, case_name);
    const Ini &I = c->cfg;
    std::string s;
    PK(need_int(I, "Schemes", "Time", c->timescheme));
    PK(need_int(I, "Schemes", "Space", c->spacescheme));
    PK(need_int(I, "Schemes", "Solver", c->solverscheme));
    PK(need_int(I, "File", "simindex", c->simindex));
    PK(need(I, "Mesh", "n", s));
    const std::vector<unsigned> n = parse_list<unsigned>(s);
    PK(need(I, "Mesh", "l", s));
    c->l = parse_list<float>(s);
    if (n.size() < 3 || c->l.size() < 3) return fail(PIRO_ERR_CONFIG, "[Mesh] n and l need 3 values");
    // ghost layers (src/preprocess.cpp:72-74)
    c->nx = (int)n[0] + 2;
    c->ny = (int)n[1] + 2;
    c->nz = (int)n[2] + 2;
    c->N = (int64_t)c->nx * c->ny * c->nz;
    if (c->solverscheme == 40) {
        Ini sol;
        if (!read_ini(c->assets + "/solver.ini", sol)) return fail(PIRO_ERR_CONFIG, "cannot read %s/solver.ini", c->assets);
        PK(need_float(sol, "JLI", "tolerance", c->jli_tol));
        PK(need_float(sol, "JLI", "URF", c->jli_urf));
        PK(need_int(sol, "JLI", "max_iter", c->jli_maxiter));
    }
    // output settings: optional here (the reference throws on a missing key)
    if (ini_get(I, "File", "casename", s)) c->casename = s;
    if (ini_get(I, "File", "restart", s)) c->restart = std::atoi(s.c_str());
    if (ini_get(I, "Mesh", "o", s)) {
        const std::vector<float> o = parse_list<float>(s);
        for (int k = 0; k < 3 && k < (int)o.size(); ++k) c->origin[k] = (int)o[k];  // AMR::Origin is int
    }
    if (ini_get(I, "Mesh", "s", s)) {
        const std::vector<float> o = parse_list<float>(s);
        for (int k = 0; k < 3 && k < (int)o.size(); ++k) c->spacing[k] = (int)o[k];
    }
    if (ini_get(I, "Mesh", "levels", s)) c->levels = std::atoi(s.c_str());
    if (ini_get(I, "Mesh", "index", s)) c->index = parse_list<int>(s);
    PK(need_float(I, "Solve", "Timestep", c->timestep));
    PK(need_float(I, "Solve", "TotalTime", c->totaltime));
    PK(need_int(I, "Solve", "Save", c->save));
    PK(need_int(I, "Solve", "Data", c->datatype));
    if (c->datatype == 2) {
        Ini ht;
        if (!read_ini(c->assets + "/Data/hashtable.ini", ht))
            return fail(PIRO_ERR_CONFIG, "cannot read %s/Data/hashtable.ini", c->assets);
        PK(need_float(ht, "Table", "LoadFactor", c->ht_lf));
        PK(need_float(ht, "Table", "a", c->ht_a));
        PK(need_float(ht, "Table", "b", c->ht_b));
        PK(need_float(ht, "Table", "c", c->ht_c));
    }
    // fields: constants, scalars, vectors (src/preprocess.cpp:113-173)
    std::string sc, ss, sv = "", sicf;
    PK(need(I, "Simulation", "Constants", sc));
    PK(need(I, "Simulation", "Values", s));
    const std::vector<float> cval = parse_list<float>(s);
    PK(need(I, "Simulation", "Scalars", ss));
    ini_get(I, "Simulation", "Vectors", sv);
    PK(need(I, "IC", "filename", sicf));
    const std::vector<std::string> cnames = split_spaces(sc), snames = split_spaces(ss), vnames = split_spaces(sv),
                                   icf = split_spaces(sicf);
    c->nconst = count_spaces(sc) + 1;
    c->nscalar = count_spaces(ss) + 1;
    c->nvector = count_words(sv);
    const int64_t N = c->N;
    for (int i = 0; i < c->nconst; ++i) {
        if (i >= (int)cval.size()) return fail(PIRO_ERR_CONFIG, "[Simulation] Values has fewer entries than Constants");
        Field f;
        f.name = cnames[i];
        f.kind = 0;
        f.n = N;
        f.host.assign((size_t)N, cval[i]);
        c->fields.push_back(f);
    }
    for (int i = 0; i < c->nscalar; ++i) {
        if (i >= (int)icf.size()) return fail(PIRO_ERR_CONFIG, "[IC] filename has fewer entries than Scalars");
        Field f;
        f.name = snames[i];
        f.kind = 1;
        f.n = N;
        PK(initial_condition(c, icf[i], f.host));
        c->fields.push_back(f);
    }
    for (int i = 0; i < c->nvector; ++i) {
        // every vector takes the entry after the scalars (preprocess.cpp:160 passes scalar_idx)
        if (c->nscalar >= (int)icf.size()) return fail(PIRO_ERR_CONFIG, "[IC] filename has no entry for the vectors");
        Field f;
        f.name = vnames[i];
        f.kind = 2;
        f.n = 3 * N;
        PK(initial_condition(c, icf[c->nscalar], f.host));
        if ((int64_t)f.host.size() < 3 * N) f.host.resize((size_t)(3 * N), 0.0f);  // the reference reads past the end
        c->fields.push_back(f);
    }
    return PIRO_OK;
}

// The device half: upload, boundary conditions, work buffers.
int load_case(piro_ctx *c)
{
    const int64_t N = (int64_t)c->nx * c->ny * c->nz;
    // upload the initial values (before setbc, as clCreateBuffer copies them first)
    for (Field &f : c->fields) {
        CK(cudaMalloc(&f.d, sizeof(float) * (size_t)f.n));
        CK(cudaMemcpyAsync(f.d, f.host.data(), sizeof(float) * (size_t)f.n, cudaMemcpyHostToDevice, c->stream));
    }
    // boundary conditions (bc::readbc / initbc / setbc, src/bc.cpp:107-167): [BC] from setup.ini
    Ini setup;
    if (read_ini(c->assets + "/setup.ini", setup)) {
        std::string bt, bp, bv;
        if (ini_get(setup, "BC", "type", bt) && count_spaces(bt) > 1) {
            PK(need(setup, "BC", "property", bp));
            PK(need(setup, "BC", "values", bv));
            const std::vector<std::string> props = split_spaces(bp);
            const std::vector<float> vals = parse_list<float>(bv);
            int64_t fs[7];
            PK(piro_face_count(c->nx, c->ny, c->nz, &c->q, fs));
            std::vector<uint32_t> idx((size_t)c->q);
            // host copy of the face lists for setbc (same closed form as the device kernel)
            CK(cudaMalloc(&c->bc_idx, sizeof(uint32_t) * (size_t)(c->q > 0 ? c->q : 1)));
            PK(piro_face_lists(c->nx, c->ny, c->nz, c->bc_idx, c->stream));
            CK(cudaMemcpyAsync(idx.data(), c->bc_idx, sizeof(uint32_t) * (size_t)c->q, cudaMemcpyDeviceToHost,
                               c->stream));
            CK(cudaStreamSynchronize(c->stream));
            for (int face = 0; face < 6; ++face) {
                if (face >= (int)props.size() || face >= (int)vals.size()) break;
                Field &f = c->fields[match_field(c, props[face])];
                for (int64_t t = fs[face]; t < fs[face + 1]; ++t) f.host[idx[(size_t)t]] = vals[face];
            }
            // memD = CD[1].values after setbc (bc.cpp:31-32)
            if (c->fields.size() < 2) return fail(PIRO_ERR_CONFIG, "boundary conditions need at least two fields");
            CK(cudaMalloc(&c->memD, sizeof(float) * (size_t)N));
            CK(cudaMemcpyAsync(c->memD, c->fields[1].host.data(), sizeof(float) * (size_t)N, cudaMemcpyHostToDevice,
                               c->stream));
        }
    }
    CK(cudaMalloc(&c->partD, sizeof(float) * (size_t)N));
    CK(cudaMalloc(&c->partC, sizeof(float) * (size_t)N));
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}

float lap_norm(const piro_ctx *c)
{
    // pow((l[0] / float(n[0] - 2)), 2) stored as float (operatorlaplacian.cpp:33)
    return (float)std::pow((double)(c->l[0] / float(c->nx - 2)), 2.0);
}

}  // namespace

// ------------------------------------------------------------------- C ABI
extern "C" int piro_open(const char *assets_dir, const char *case_name, piro_ctx **out)
{
    if (!assets_dir || !case_name || !out) {
        piro::set_error("piro_open: null argument");
        return PIRO_ERR_ARG;
    }
    *out = nullptr;
    piro_ctx *c = new piro_ctx();
    c->assets = assets_dir;
    int rc = parse_case(c, case_name);
    if (!rc && cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        piro::set_error("piro_open: cannot create a stream");
        rc = PIRO_ERR_CUDA;
    }
    if (!rc) rc = load_case(c);
    if (rc) {
        piro_close(c);
        return rc;
    }
    *out = c;
    return PIRO_OK;
}

extern "C" void piro_close(piro_ctx *c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (Field &f : c->fields) cudaFree(f.d);
    free_csr(c->lap);
    for (Csr &g : c->grad) free_csr(g);
    free_csr(c->dot);
    free_csr(c->divm);
    free_csr(c->be_A);
    cudaFree(c->dense);
    cudaFree(c->coo_rows);
    cudaFree(c->coo_rowstart);
    cudaFree(c->ht_keys);
    cudaFree(c->ht_vals);
    cudaFree(c->ht_order);
    cudaFree(c->ht_stage);
    cudaFree(c->lu_band);
    cudaFree(c->bc_idx);
    cudaFree(c->memD);
    cudaFree(c->partD);
    cudaFree(c->partC);
    cudaFree(c->work);
    if (c->be) piro_be_destroy(c->be);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int piro_ctx_query(piro_ctx *c, piro_case_info *info)
{
    if (!c || !info) {
        piro::set_error("piro_ctx_query: null argument");
        return PIRO_ERR_ARG;
    }
    info->nx = c->nx;
    info->ny = c->ny;
    info->nz = c->nz;
    info->n_cells = c->N;
    info->timescheme = c->timescheme;
    info->spacescheme = c->spacescheme;
    info->solverscheme = c->solverscheme;
    info->datatype = c->datatype;
    info->simindex = c->simindex;
    info->timestep = c->timestep;
    info->totaltime = c->totaltime;
    info->steps_done = c->steps;
    info->n_fields = (int)c->fields.size();
    info->bc_cells = c->q;
    return PIRO_OK;
}

extern "C" int piro_set_alpha_mode(piro_ctx *c, int mode)
{
    if (!c || mode < 0 || mode > 1) {
        piro::set_error("piro_set_alpha_mode: mode must be 0 (intended) or 1 (as run by the reference)");
        return PIRO_ERR_ARG;
    }
    if (c->lap_init) {
        piro::set_error("piro_set_alpha_mode: the Laplacian is already assembled");
        return PIRO_ERR_STATE;
    }
    c->alpha_mode = mode;
    return PIRO_OK;
}

extern "C" int piro_set_lu_mode(piro_ctx *c, int mode)
{
    if (!c || mode < 0 || mode > 1) {
        piro::set_error("piro_set_lu_mode: mode must be 0 (solve) or 1 (as run by the reference)");
        return PIRO_ERR_ARG;
    }
    if (c->lu_done) {
        piro::set_error("piro_set_lu_mode: the LU is already factorized");
        return PIRO_ERR_STATE;
    }
    c->lu_mode = mode;
    return PIRO_OK;
}

extern "C" int piro_field(piro_ctx *c, const char *var, piro_buf *out)
{
    if (!c || !var || !out) {
        piro::set_error("piro_field: null argument");
        return PIRO_ERR_ARG;
    }
    out->id = match_field(c, var);
    out->n = c->fields[(size_t)out->id].n;
    return PIRO_OK;
}

extern "C" int piro_ddt_r(piro_ctx *c, const char *var, piro_buf *out) { return piro_field(c, var, out); }
extern "C" int piro_vector(piro_ctx *c, const char *var, piro_buf *out) { return piro_field(c, var, out); }

extern "C" int piro_field_upload(piro_ctx *c, piro_buf f, const float *host, int64_t n)
{
    if (!c || !host || f.id < 0 || f.id >= (int)c->fields.size() || n != c->fields[(size_t)f.id].n) {
        piro::set_error("piro_field_upload: bad field or size");
        return PIRO_ERR_ARG;
    }
    CK(cudaMemcpyAsync(c->fields[(size_t)f.id].d, host, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}

extern "C" int piro_field_download(piro_ctx *c, piro_buf f, float *host, int64_t n)
{
    if (!c || !host || f.id < 0 || f.id >= (int)c->fields.size() || n != c->fields[(size_t)f.id].n) {
        piro::set_error("piro_field_download: bad field or size");
        return PIRO_ERR_ARG;
    }
    CK(cudaMemcpyAsync(host, c->fields[(size_t)f.id].d, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}

extern "C" int piro_field_device_ptr(piro_ctx *c, piro_buf f, float **dptr)
{
    if (!c || !dptr || f.id < 0 || f.id >= (int)c->fields.size()) {
        piro::set_error("piro_field_device_ptr: bad field");
        return PIRO_ERR_ARG;
    }
    *dptr = c->fields[(size_t)f.id].d;
    return PIRO_OK;
}

extern "C" int piro_laplacian(piro_ctx *c, const char *var, const char *coeff, piro_op *out)
{
    (void)var;
    if (!c || !coeff || !out) {
        piro::set_error("piro_laplacian: null argument");
        return PIRO_ERR_ARG;
    }
    out->kind = PIRO_OP_LAPLACIAN;
    if (c->lap_init) return PIRO_OK;
    const int64_t N = c->N;
    const int coef = match_field(c, coeff);
    if (c->datatype == 1) {
        // Piro::DENSE::laplacian (operatorlaplacian.cpp:65-103): N x N, alpha never applied
        const size_t bytes = sizeof(float) * (size_t)N * (size_t)N;
        if (cudaMalloc(&c->dense, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            c->dense = nullptr;
            return fail(PIRO_ERR_NOMEM, "piro_laplacian: no device memory for the %s-byte DENSE matrix",
                        std::to_string(bytes));
        }
        PK(piro_dense_laplacian(c->nx, c->ny, c->nz, c->spacescheme, lap_norm(c), c->dense, bytes, c->stream));
        c->lap_coeff = coef;
        c->lap_init = true;
        CK(cudaStreamSynchronize(c->stream));
        return PIRO_OK;
    }
    if (c->datatype != 0 && c->datatype != 2 && c->datatype != 3) {
        piro::set_error("piro_laplacian: invalid Data %d", c->datatype);
        return PIRO_ERR_DATATYPE;
    }
    int64_t nnz = 0;
    PK(piro_laplacian_nnz(c->nx, c->ny, c->nz, &nnz));
    const float norm = lap_norm(c);
    if (c->datatype == 3) {
        PK(alloc_csr(c->lap, N, nnz));
        CK(cudaMalloc(&c->coo_rows, sizeof(int32_t) * (size_t)nnz));
        PK(piro_coo_laplacian(c->nx, c->ny, c->nz, c->spacescheme, norm, c->coo_rows, c->lap.col, c->lap.val,
                              c->stream));
        CK(cudaMalloc(&c->coo_rowstart, sizeof(int32_t) * (size_t)(N + 1)));
        PK(ensure_work(c, 256));
        PK(piro_coo_row_index(N, nnz, c->coo_rows, c->coo_rowstart, c->work, c->work_bytes, c->stream));
    } else {
        PK(alloc_csr(c->lap, N, nnz));
        PK(piro_csr_laplacian(c->nx, c->ny, c->nz, c->spacescheme, norm, c->lap.rp, c->lap.col, c->lap.val, c->stream));
        if (c->datatype == 0 && c->alpha_mode == 0)  // csrscale on the CSR path only (process.cpp:70-72)
            PK(piro_csr_rowscale(N, c->lap.rp, c->lap.val, c->fields[(size_t)coef].d, c->stream));
        if (c->datatype == 2) {
            int64_t ts = 0;
            PK(piro_ht_table_size(nnz, N, 0, c->ht_a, c->ht_b, c->ht_c, c->ht_lf, &ts));
            size_t wb = 0;
            PK(piro_ht_build_workspace(ts, &wb));
            PK(ensure_work(c, wb));
            CK(cudaMalloc(&c->ht_keys, sizeof(int64_t) * (size_t)ts));
            CK(cudaMalloc(&c->ht_vals, sizeof(float) * (size_t)ts));
            PK(piro_ht_build(N, c->lap.rp, c->lap.col, c->lap.val, nnz, ts, c->ht_keys, c->ht_vals, c->work,
                             c->work_bytes, c->stream));
            c->ht_ts = ts;
            PK(piro_ht_row_order_workspace(N, ts, &wb));
            PK(ensure_work(c, wb));
            CK(cudaMalloc(&c->ht_order, sizeof(int32_t) * (size_t)N));
            PK(piro_ht_row_order(N, ts, c->ht_order, c->work, c->work_bytes, c->stream));
            PK(piro_ht_stage_bytes(N, &wb));
            CK(cudaMalloc(&c->ht_stage, wb));
        }
    }
    c->lap_coeff = coef;
    c->lap_init = true;
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}

extern "C" int piro_gradient(piro_ctx *c, const char *var, piro_op *out)
{
    (void)var;
    if (!c || !out) {
        piro::set_error("piro_gradient: null argument");
        return PIRO_ERR_ARG;
    }
    out->kind = PIRO_OP_GRADIENT;
    if (c->grad_init) return PIRO_OK;
    if (c->datatype != 0) {
        piro::set_error("piro_gradient: only CSR (Data = 0), as in process.cpp:124-152");
        return PIRO_ERR_DATATYPE;
    }
    // norm = 2 * (l0 / float(n0 - 2)) in float (operatorgradient.cpp:25)
    const float norm = 2 * (c->l[0] / float(c->nx - 2));
    for (int a = 0; a < 3; ++a) {
        int64_t nnz = 0;
        PK(piro_gradient_nnz(c->nx, c->ny, c->nz, a, &nnz));
        PK(alloc_csr(c->grad[a], c->N, nnz));
        PK(piro_csr_gradient(c->nx, c->ny, c->nz, c->spacescheme, a, norm, c->grad[a].rp, c->grad[a].col,
                             c->grad[a].val, c->stream));
    }
    c->grad_init = true;
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}

extern "C" int piro_dot(piro_ctx *c, piro_buf v, piro_op grad, piro_op *out)
{
    if (!c || !out || grad.kind != PIRO_OP_GRADIENT || !c->grad_init || v.id < 0 || v.id >= (int)c->fields.size()) {
        piro::set_error("piro_dot: needs a vector field and an assembled gradient");
        return PIRO_ERR_STATE;
    }
    out->kind = PIRO_OP_DOT;
    if (c->dot_init) return PIRO_OK;  // DOT_INIT: merged once (kernelcsrgeam.cpp:12)
    const Field &f = c->fields[(size_t)v.id];
    if (f.n < 3 * c->N) {
        piro::set_error("piro_dot: field '%s' is not a vector field", f.name.c_str());
        return PIRO_ERR_ARG;
    }
    const int64_t nnz = c->grad[0].nnz + c->grad[1].nnz + c->grad[2].nnz;
    size_t wb = 0;
    PK(piro_scan_workspace(c->N, &wb));
    PK(ensure_work(c, wb));
    PK(alloc_csr(c->dot, c->N, nnz));
    PK(piro_csrgeam3(c->N, c->grad[0].rp, c->grad[0].col, c->grad[0].val, c->grad[1].rp, c->grad[1].col,
                     c->grad[1].val, c->grad[2].rp, c->grad[2].col, c->grad[2].val, f.d, c->dot.rp, c->dot.col,
                     c->dot.val, c->work, c->work_bytes, c->stream));
    c->dot_init = true;
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}

// process::div (src/process.cpp:168-215): Piro::CSR::div's three matrices
// (operatordivergenceCSR.cpp:21-101; the div_* stencils forward to the
// gradient ones, stencils.cpp:995-1003, with the same norm) merged by
// csrgeam_2 (kernelcsrgeam.cpp:88-207) after SpMSCSR scales matrix a's rows
// by component a of var2.  That merge is csrgeam3 with var2 as the vector.
// alpha_mode 1 keeps the reference's literal behaviour: its SpMSCSR launches
// set their int arguments with sizeof(cl_mem) (kernelcsrgeam.cpp:103-129) and
// never run, so the gradients are merged unscaled.  CSR only (the reference
// exits otherwise).
extern "C" int piro_div(piro_ctx *c, const char *var1, const char *var2, piro_op *out)
{
    (void)var1;
    if (!c || !var2 || !out) {
        piro::set_error("piro_div: null argument");
        return PIRO_ERR_ARG;
    }
    out->kind = PIRO_OP_DIV;
    if (c->div_init) return PIRO_OK;  // DIV_INIT
    if (c->datatype != 0) {
        piro::set_error("piro_div: only CSR (Data = 0), as in process.cpp:181-213");
        return PIRO_ERR_DATATYPE;
    }
    piro_op g;
    PK(piro_gradient(c, var1, &g));
    const Field &f = c->fields[(size_t)match_field(c, var2)];
    if (f.n < 3 * c->N) {
        piro::set_error("piro_div: field '%s' is not a vector field", f.name.c_str());
        return PIRO_ERR_ARG;
    }
    const float *v = f.d;
    float *ones = nullptr;
    if (c->alpha_mode == 1) {
        CK(cudaMalloc(&ones, sizeof(float) * 3 * (size_t)c->N));
        CK(cudaMemsetAsync(ones, 0, sizeof(float) * 3 * (size_t)c->N, c->stream));
        PK(piro_vec_op_scalar(0, 3 * c->N, 1.0f, ones, ones, c->stream));
        v = ones;
    }
    const int64_t nnz = c->grad[0].nnz + c->grad[1].nnz + c->grad[2].nnz;
    size_t wb = 0;
    int rc = piro_scan_workspace(c->N, &wb);
    if (rc == PIRO_OK) rc = ensure_work(c, wb);
    if (rc == PIRO_OK) rc = alloc_csr(c->divm, c->N, nnz);
    if (rc == PIRO_OK)
        rc = piro_csrgeam3(c->N, c->grad[0].rp, c->grad[0].col, c->grad[0].val, c->grad[1].rp, c->grad[1].col,
                           c->grad[1].val, c->grad[2].rp, c->grad[2].col, c->grad[2].val, v, c->divm.rp,
                           c->divm.col, c->divm.val, c->work, c->work_bytes, c->stream);
    if (rc == PIRO_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = PIRO_ERR_CUDA;
    cudaFree(ones);
    if (rc) return rc;
    c->div_init = true;
    return PIRO_OK;
}

static const Csr *op_csr(const piro_ctx *c, piro_op op)
{
    if (op.kind == PIRO_OP_LAPLACIAN && c->lap_init && c->datatype != 1) return &c->lap;
    if (op.kind == PIRO_OP_DOT && c->dot_init) return &c->dot;
    if (op.kind == PIRO_OP_DIV && c->div_init) return &c->divm;
    return nullptr;
}

// Backward Euler by FP32 PCG in FP64 refinement on A = I - dt*M (M the
// assembled operator, alpha already applied): solver 39.
static int be_pcg(piro_ctx *c, const Csr *M, const float *b, float *x)
{
    const int64_t N = c->N;
    if (!c->be) {
        Csr I;
        PK(alloc_csr(I, N, N));
        PK(piro_csr_identity(N, I.rp, I.col, I.val, c->stream));
        size_t wb = 0;
        PK(piro_scan_workspace(N, &wb));
        PK(ensure_work(c, wb));
        CK(cudaMalloc(&c->be_A.rp, sizeof(int32_t) * (size_t)(N + 1)));
        PK(piro_csrgeam2_count(N, I.rp, I.col, M->rp, M->col, c->be_A.rp, c->work, c->work_bytes, c->stream));
        int32_t nnz = 0;
        CK(cudaMemcpyAsync(&nnz, c->be_A.rp + N, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        CK(cudaMalloc(&c->be_A.col, sizeof(int32_t) * (size_t)nnz));
        CK(cudaMalloc(&c->be_A.val, sizeof(float) * (size_t)nnz));
        c->be_A.nnz = nnz;
        PK(piro_csrgeam2_fill(N, I.rp, I.col, I.val, -c->timestep, M->rp, M->col, M->val, c->be_A.rp, c->be_A.col,
                              c->be_A.val, c->stream));
        free_csr(I);
        const float *alpha = c->alpha_mode == 0 && c->lap_coeff >= 0 ? c->fields[(size_t)c->lap_coeff].d : nullptr;
        if (!alpha) {
            // the symmetric form needs a positive row weight; alpha = 1 when it was not applied
            CK(cudaMemsetAsync(c->partC, 0, sizeof(float) * (size_t)N, c->stream));
            PK(piro_vec_op_scalar(0, N, 1.0f, c->partC, c->partC, c->stream));
            alpha = c->partC;
        }
        int rc = c->spacescheme == 3
                     ? piro_be_create_stencil(c->nx, c->ny, c->nz, c->be_A.rp, c->be_A.col, c->be_A.val, alpha,
                                              c->timestep, lap_norm(c), c->stream, &c->be)
                     : piro_be_create(c->nx, c->ny, c->nz, c->be_A.rp, c->be_A.col, c->be_A.val, alpha, c->stream,
                                      &c->be);
        if (rc) return rc;
    }
    piro_be_info info;
    return piro_be_solve(c->be, b, x, 1e-8, 20, 20000, &info);
}

// Scheme 27 on the hash-table operator M (TIMESCHEME 12, solver 27, Data 2).
// Mode 1: PIRO's factorization of M's own table on the first step
// (matrix_operations::HT::lu_decomposition), the result field zero, as the
// reference returns it.  Mode 0: A = I - dt*M factorized in a dense band
// (bandwidth nx*ny) on the first step; every step then solves A x = u.
static int lu_step(piro_ctx *c, const float *u, float *x)
{
    const int64_t N = c->N;
    if (c->lu_mode == 1) {
        if (!c->lu_done) PK(piro_ht_lu_reference(N, c->ht_keys, c->ht_vals, c->ht_ts, c->stream));
        c->lu_done = true;
        return PIRO_OK;
    }
    if (!c->lu_done) {
        c->lu_bw = (int64_t)c->nx * c->ny;
        PK(piro_ht_lu_band_bytes(N, c->lu_bw, &c->lu_band_bytes));
        if (cudaMalloc(&c->lu_band, c->lu_band_bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            c->lu_band = nullptr;
            return fail(PIRO_ERR_NOMEM, "scheme 27: no device memory for the %s-byte band",
                        std::to_string(c->lu_band_bytes));
        }
        PK(piro_ht_lu_factor(N, c->lu_bw, c->ht_keys, c->ht_vals, c->ht_ts, 1.0f, -c->timestep, c->lu_band,
                             c->lu_band_bytes, c->stream));
        c->lu_done = true;
    }
    return piro_ht_lu_solve(N, c->lu_bw, c->lu_band, c->lu_band_bytes, u, x, c->stream);
}

extern "C" int piro_assign(piro_ctx *c, piro_buf lhs, piro_op rhs, piro_buf *out)
{
    if (!c || !out || lhs.id < 0 || lhs.id >= (int)c->fields.size()) {
        piro::set_error("piro_assign: bad arguments");
        return PIRO_ERR_ARG;
    }
    const int64_t N = c->N;
    float *u = c->fields[(size_t)lhs.id].d;
    const float dt = c->timestep;
    // partD starts from zeros on every call (operatoroverload.cpp:29-34)
    CK(cudaMemsetAsync(c->partD, 0, sizeof(float) * (size_t)N, c->stream));
    if (c->timescheme == 11) {
        if (c->datatype == 0) {
            const Csr *M = op_csr(c, rhs);
            if (!M) return fail(PIRO_ERR_STATE, "piro_assign: operator not assembled");
            PK(piro_csr_fe_step(c->nx, c->ny, c->nz, M->rp, M->col, M->val, dt, u, c->partD, c->stream));
        } else if (c->datatype == 1) {
            if (!c->dense || rhs.kind != PIRO_OP_LAPLACIAN)
                return fail(PIRO_ERR_STATE, "piro_assign: DENSE operator not assembled");
            PK(piro_dense_fe_step(N, c->dense, dt, u, c->partD, c->stream));
            PK(piro_dense_check(c->stream));
        } else if (c->datatype == 2) {
            if (!c->ht_keys) return fail(PIRO_ERR_STATE, "piro_assign: hash table not built");
            PK(piro_ht_spmv_staged(c->nx, c->ny, c->nz, c->ht_keys, c->ht_vals, c->ht_ts, dt, 1, c->ht_order,
                                   c->ht_stage, 32 * (size_t)N, u, c->partD, c->stream));
        } else if (c->datatype == 3) {
            if (!c->coo_rows) return fail(PIRO_ERR_STATE, "piro_assign: COO operator not assembled");
            PK(piro_coo_step_indexed(N, c->coo_rowstart, c->lap.col, c->lap.val, dt, 1, u, c->partD, c->stream));
        } else {
            return fail(PIRO_ERR_DATATYPE, "piro_assign: Data not supported on this path");
        }
    } else if (c->timescheme == 12 && c->solverscheme == 27) {
        if (c->datatype != 2) return fail(PIRO_ERR_DATATYPE, "piro_assign: solver 27 needs Data = 2 (hash table)");
        if (!c->ht_keys || rhs.kind != PIRO_OP_LAPLACIAN)
            return fail(PIRO_ERR_STATE, "piro_assign: hash table not built");
        PK(lu_step(c, u, c->partD));
    } else if (c->timescheme == 12) {
        const Csr *M = op_csr(c, rhs);
        if (c->datatype != 0 || !M) return fail(PIRO_ERR_DATATYPE, "piro_assign: backward Euler needs a CSR operator");
        if (c->solverscheme == 40) {
            int iters = 0;
            PK(piro_be_jli(c->nx, c->ny, c->nz, M->rp, M->col, M->val, dt, u, c->partD, c->partC, c->jli_tol,
                           c->jli_urf, c->jli_maxiter, &iters, c->stream));
        } else if (c->solverscheme == 39) {
            if (rhs.kind != PIRO_OP_LAPLACIAN)
                return fail(PIRO_ERR_SCHEME, "piro_assign: solver 39 (PCG) needs the symmetric Laplacian");
            PK(be_pcg(c, M, u, c->partD));
        } else {
            piro::set_error("piro_assign: Solver %d not available for TIMESCHEME 12 (40 JLI, 39 PCG, 27 LU)", c->solverscheme);
            return PIRO_ERR_SCHEME;
        }
    } else {
        piro::set_error("piro_assign: TIMESCHEME %d not available (11, 12)", c->timescheme);
        return PIRO_ERR_SCHEME;
    }
    out->id = PIRO_EQN_RESULT;
    out->n = N;
    return PIRO_OK;
}

// ---- ParaView output: Piro::paraview::writevth / writevti (src/paraview.cpp:12-137)
static std::string fmt_g(float v)
{
    char b[48];
    std::snprintf(b, sizeof b, "%g", (double)v);  // std::ostream << float (precision 6)
    return b;
}

static void append_values(std::string &out, const float *v, int64_t n)
{
    for (int64_t i = 0; i < n; ++i) {
        if (i) out += ' ';
        out += fmt_g(v[i]);
    }
}

// The .vti of one level: cell data of the scalar and vector fields with the
// boundary cells removed (bc::prepbc's list), gathered on the device.
static int vti_text(piro_ctx *c, std::string &out)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const int64_t Ni = (int64_t)(nx - 2) * (ny - 2) * (nz - 2);
    auto ext = [&]() {
        return "0 " + std::to_string(nx - 2) + " 0 " + std::to_string(ny - 2) + " 0 " + std::to_string(nz - 2);
    };
    out = "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\">\n";
    out += "<ImageData WholeExtent=\"" + ext() + "\" Origin=\"" + std::to_string(c->origin[0]) + " " +
           std::to_string(c->origin[1]) + " " + std::to_string(c->origin[2]) + "\" Spacing=\"" +
           std::to_string(c->spacing[0]) + " " + std::to_string(c->spacing[1]) + " " + std::to_string(c->spacing[2]) +
           "\">\n";
    out += "<Piece Extent=\"" + ext() + "\">\n";
    out += "<PointData Scalars=\"ScalarValues\">\n</PointData>\n<CellData>\n";
    float *d = nullptr;
    CK(cudaMalloc(&d, sizeof(float) * (size_t)(3 * Ni)));
    std::vector<float> h((size_t)(3 * Ni));
    int rc = PIRO_OK;
    for (const Field &f : c->fields) {
        if (f.kind == 0 || (f.kind == 2 && c->nvector <= 0)) continue;
        const int ncomp = f.kind == 2 ? 3 : 1;
        rc = piro_interior_gather(nx, ny, nz, ncomp, f.d, d, c->stream);
        if (rc) break;
        if (cudaMemcpyAsync(h.data(), d, sizeof(float) * (size_t)(ncomp * Ni), cudaMemcpyDeviceToHost, c->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess) {
            rc = fail(PIRO_ERR_CUDA, "paraview: device read failed");
            break;
        }
        static const char *suffix[3] = {"_x", "_y", "_z"};
        for (int k = 0; k < ncomp; ++k) {
            out += "<DataArray type=\"Float64\" Name=\"" + f.name + (ncomp == 3 ? suffix[k] : "") +
                   "\" format=\"ascii\">\n";
            append_values(out, h.data() + k * Ni, Ni);
            out += "</DataArray>\n";
        }
    }
    cudaFree(d);
    if (rc) return rc;
    out += "</CellData>\n</Piece>\n</ImageData>\n</VTKFile>\n";
    return PIRO_OK;
}

static int write_text(const std::string &path, const std::string &text)
{
    std::ofstream f(path);
    if (!f.is_open()) return fail(PIRO_ERR_CONFIG, "paraview: cannot write %s", path);
    f << text << std::endl;  // file_utilities::writefile appends a newline
    return f.good() ? PIRO_OK : fail(PIRO_ERR_CONFIG, "paraview: write failed for %s", path);
}

extern "C" int piro_write_paraview(piro_ctx *c, const char *root, int timestep)
{
    if (!c || !root || timestep < 0) {
        piro::set_error("piro_write_paraview: bad arguments");
        return PIRO_ERR_ARG;
    }
    for (int i = 0; i < c->levels; ++i)
        if (i >= (int)c->index.size() || c->index[i] != 1)
            return fail(PIRO_ERR_CONFIG, "paraview: [Mesh] index must be 1 per level (the reference writes "
                                         "only level data set 0)");
    const std::string base = std::string(root) + "/" + c->casename + "/mesh";
    std::error_code ec;
    std::filesystem::create_directories(base + "/level", ec);
    if (ec) return fail(PIRO_ERR_CONFIG, "paraview: cannot create %s/level", base);
    std::string ts = std::to_string(timestep);
    if (ts.size() < 5) ts = std::string(5 - ts.size(), '0') + ts;
    std::string vth = "<?xml version=\"1.0\"?>\n";
    vth += "<VTKFile type=\"vtkOverlappingAMR\" version=\"1.1\" byte_order=\"LittleEndian\" "
           "header_type=\"UInt32\">\n";
    vth += "<vtkOverlappingAMR origin=\"0 0 0\" grid_description=\"XYZ\">\n";
    std::string vti;
    PK(vti_text(c, vti));
    for (int i = 0; i < c->levels; ++i) {
        for (int j = 0; j < c->index[i]; ++j) {
            vth += "<Block level=\"" + std::to_string(i) + "\" spacing=\"1 1 1\">\n";
            vth += "<DataSet index=\"0\" amr_box=\"0 " + std::to_string(c->nx - 2) + " 0 " +
                   std::to_string(c->ny - 2) + " 0 " + std::to_string(c->nz - 2) + "\" file=\"level/" + ts +
                   "_level_" + std::to_string(j) + ".vti\">\n</DataSet>\n";
            PK(write_text(base + "/level/" + ts + "_level_" + std::to_string(j) + ".vti", vti));
        }
        vth += "</Block>\n";
    }
    vth += "</vtkOverlappingAMR>\n</VTKFile>\n";
    return write_text(base + "/mesh_" + ts + ".vth", vth);
}

extern "C" int piro_set_output(piro_ctx *c, const char *root)
{
    if (!c) {
        piro::set_error("piro_set_output: null context");
        return PIRO_ERR_ARG;
    }
    if (!root) {
        c->out_root.clear();
        return PIRO_OK;
    }
    c->out_root = root;
    // Piro::init (src/init.cpp:10-21): a restart clears the case directory
    const std::string dir = c->out_root + "/" + c->casename;
    std::error_code ec;
    if (c->restart) std::filesystem::remove_all(dir, ec);
    std::filesystem::create_directories(dir + "/mesh/level", ec);
    if (ec) return fail(PIRO_ERR_CONFIG, "piro_set_output: cannot create %s/mesh/level", dir);
    return PIRO_OK;
}

extern "C" int piro_step_solve(piro_ctx *c, piro_buf eqn, float time)
{
    if (!c || eqn.id != PIRO_EQN_RESULT || c->fields.size() < 2) {
        piro::set_error("piro_step_solve: needs the result of piro_assign and at least two fields");
        return PIRO_ERR_ARG;
    }
    // copy into VALUES_GPU[1] (index hard-coded in process.cpp:234), then setBC(1)
    const int64_t N = c->N;
    CK(cudaMemcpyAsync(c->fields[1].d, c->partD, sizeof(float) * (size_t)N, cudaMemcpyDeviceToDevice, c->stream));
    if (c->q > 0) PK(piro_set_bc(c->q, c->bc_idx, c->memD, c->fields[1].d, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    ++c->steps;
    // post-processing every Save steps (process.cpp:236-247), when an output root is set
    if (!c->out_root.empty() && c->save > 0) {
        const int ts = (int)(time / c->timestep);
        if ((ts + 1) % c->save == 0) PK(piro_write_paraview(c, c->out_root.c_str(), ts));
    }
    return PIRO_OK;
}

extern "C" int piro_solve(piro_ctx *c, int64_t *steps_taken)
{
    if (!c) {
        piro::set_error("piro_solve: null context");
        return PIRO_ERR_ARG;
    }
    // while (time < TotalTime) with float time (src/solve.cpp:17-18,45)
    float time = 0.0f;
    int64_t n = 0;
    while (time < c->totaltime) {
        piro_buf lhs, res;
        piro_op op;
        if (c->simindex == 0) {
            PK(piro_ddt_r(c, "T", &lhs));
            PK(piro_laplacian(c, "T", "Alpha", &op));
        } else if (c->simindex == 1) {
            piro_buf v;
            piro_op g;
            PK(piro_ddt_r(c, "U", &lhs));
            PK(piro_vector(c, "v", &v));
            PK(piro_gradient(c, "U", &g));
            PK(piro_dot(c, v, g, &op));
        } else if (c->simindex == 2) {
            PK(piro_ddt_r(c, "rho", &lhs));
            PK(piro_div(c, "rho", "u", &op));
        } else {
            piro::set_error("piro_solve: simindex %d invalid (0 heat, 1 advection, 2 continuity)", c->simindex);
            return PIRO_ERR_SCHEME;
        }
        PK(piro_assign(c, lhs, op, &res));
        PK(piro_step_solve(c, res, time));
        time += c->timestep;
        ++n;
    }
    if (steps_taken) *steps_taken = n;
    return PIRO_OK;
}

extern "C" int piro_op_export_csr(piro_ctx *c, piro_op op, int32_t *rowptr, int32_t *col, float *val, int64_t cap,
                                  int64_t *nnz)
{
    if (!c || !nnz) {
        piro::set_error("piro_op_export_csr: null argument");
        return PIRO_ERR_ARG;
    }
    const Csr *M = op_csr(c, op);
    if (!M || (c->datatype != 0 && op.kind == PIRO_OP_LAPLACIAN)) {
        piro::set_error("piro_op_export_csr: no CSR form of this operator");
        return PIRO_ERR_STATE;
    }
    *nnz = M->nnz;
    if (!rowptr) return PIRO_OK;
    if (cap < M->nnz) {
        piro::set_error("piro_op_export_csr: capacity %lld < nnz %lld", (long long)cap, (long long)M->nnz);
        return PIRO_ERR_ARG;
    }
    CK(cudaMemcpyAsync(rowptr, M->rp, sizeof(int32_t) * (size_t)(c->N + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(col, M->col, sizeof(int32_t) * (size_t)M->nnz, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(val, M->val, sizeof(float) * (size_t)M->nnz, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PIRO_OK;
}
