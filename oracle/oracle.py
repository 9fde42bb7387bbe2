"""Test infrastructure: numpy front end to the CPU oracle (oracle/piro_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module.  It is the checker, never part of the product path.

`Ref` wraps oracle/_ref/libpiro_ref.so, PIRO's own host code and .cl kernels
compiled for the CPU, which pins the restatement (see oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libpiro_ref.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")


def build(with_ref: bool = False) -> None:
    """Compile the oracle (and _ref, when PIRO_REF_DIR names the PIRO tree)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    ref = os.environ.get("PIRO_REF_DIR", "")
    if with_ref and ref and os.path.isdir(ref):
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref"])


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    i64, i32, f32, f64 = C.c_int64, C.c_int, C.c_float, C.c_double
    sig = {
        "or_num_threads": (i32, []),
        "or_set_threads": (None, [i32]),
        "or_laplacian": (i64, [i32, i32, i32, i32, f32, C.c_void_p, C.c_void_p, _i32p, _f32p]),
        "or_gradient": (i64, [i32, i32, i32, i32, i32, f32, _i32p, _i32p, _f32p]),
        "or_ht_table_size_reference": (i64, [i64, i64, f32, f32, f32, f32]),
        "or_ht_build": (i32, [i64, _i32p, _i32p, _f32p, i64, _i64p, _f32p]),
        "or_ht_lookup": (f32, [i64, i64, _i64p, _f32p]),
        "or_csrgeam3_count": (None, [i64, _i32p, _i32p, _i32p, _i32p]),
        "or_scan_rowptr": (None, [i64, _i32p, _i32p]),
        "or_csrgeam3_fill": (None, [i64, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                    _f32p, _i32p, _i32p, _f32p]),
        "or_csr_rowscale": (None, [i64, _i32p, _f32p, _f32p]),
        "or_csrgeam2_count": (None, [i64, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "or_csrgeam2_fill": (None, [i64, _i32p, _i32p, _f32p, f32, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p]),
        "or_spmv_csr_fe": (None, [i64, i32, i32, _i32p, _i32p, _f32p, f32, _f32p, _f32p]),
        "or_spmv_csr_i1": (None, [i64, i32, i32, _i32p, _i32p, _f32p, f32, _f32p, _f32p]),
        "or_spmv_coo": (None, [i64, i64, _i32p, _i32p, _f32p, f32, _f32p, _f32p]),
        "or_spmv_ht": (None, [i64, i64, _i64p, _f32p, f32, _f32p, _f32p]),
        "or_vec_binary": (None, [i32, i64, _f32p, _f32p, _f32p]),
        "or_vec_constant": (None, [i32, i64, f32, _f32p, _f32p]),
        "or_urf": (None, [i64, _f32p, _f32p, f32]),
        "or_setbc": (None, [i64, _u32p, _f32p, _f32p]),
        "or_face_lists": (i64, [i32, i32, i32, _u32p, _i64p]),
        "or_step_count": (i64, [f32, f32]),
        "or_fe_csr_step": (None, [i64, i32, i32, _i32p, _i32p, _f32p, f32, _f32p, i64, _u32p, _f32p, _f32p]),
        "or_fe_coo_step": (None, [i64, i64, _i32p, _i32p, _f32p, f32, _f32p, i64, _u32p, _f32p, _f32p]),
        "or_fe_ht_step": (None, [i64, i64, _i64p, _f32p, f32, _f32p, i64, _u32p, _f32p, _f32p]),
        "or_stencil_fe": (None, [i32, i32, i32, f32, f32, f32, f32, C.c_void_p, _f32p, _f32p]),
        "or_be_jli": (i32, [i64, i32, i32, _i32p, _i32p, _f32p, f32, _f32p, _f32p, _f32p, f32, f32, i32]),
        "or_be_cg_f64": (i32, [i64, i32, i32, i32, _i32p, _i32p, _f32p, _f32p, _f32p, _f64p, f64, i32,
                               C.POINTER(C.c_double)]),
        "or_be_cg_f64d": (i32, [i64, i32, i32, i32, _i32p, _i32p, _f32p, _f32p, _f64p, _f64p, f64, i32,
                                C.POINTER(C.c_double)]),
        "or_dense_laplacian": (None, [i32, i32, i32, i32, f32, _f32p]),
        "or_fe_dense_step": (None, [i64, _f32p, f32, _f32p, _f32p, _f32p]),
        "or_ic_gaussian": (None, [i32, i32, i32, f32, f32, f32, f32, _f32p, _f32p, _f32p]),
        "or_ic_coulomb": (None, [i32, i32, i32, f32, f32, f32, _f32p, f32, f64, f64, _f32p]),
        "or_ic_uniform_vector": (None, [i64, _f32p, f32, _f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------------- grid
def n_cells(nx, ny, nz):
    return int(nx) * int(ny) * int(nz)


def laplacian_norm(l0: float, n0: int) -> np.float32:
    """norm = (float)pow(l0/float(n0-2), 2) (src/operatorlaplacian.cpp:33)."""
    h = np.float32(np.float32(l0) / np.float32(n0 - 2))
    return np.float32(float(h) ** 2)


def gradient_norm(l0: float, n0: int) -> np.float32:
    """norm = 2 * (l0/float(n0-2)) in float (src/operatorgradient.cpp:25)."""
    return np.float32(np.float32(2) * np.float32(np.float32(l0) / np.float32(n0 - 2)))


def laplacian(nx, ny, nz, scheme, norm, fmt="csr"):
    """CSR -> (rowptr, col, val); COO -> (rows, col, val)."""
    N = n_cells(nx, ny, nz)
    cap = 7 * N
    col = np.zeros(cap, np.int32)
    val = np.zeros(cap, np.float32)
    rowptr = np.zeros(N + 1, np.int32) if fmt == "csr" else None
    rows = np.zeros(cap, np.int32) if fmt == "coo" else None
    nnz = lib().or_laplacian(nx, ny, nz, scheme, np.float32(norm), _ptr(rowptr), _ptr(rows), col, val)
    if fmt == "csr":
        return rowptr, col[:nnz].copy(), val[:nnz].copy()
    return rows[:nnz].copy(), col[:nnz].copy(), val[:nnz].copy()


def gradient3(nx, ny, nz, scheme, norm):
    """[(rowptr, col, val)] for x, y, z, sharing rowpointers as the reference does."""
    N = n_cells(nx, ny, nz)
    rp = np.zeros(N + 1, np.int32)
    out = []
    for axis in range(3):
        col = np.zeros(2 * N, np.int32)
        val = np.zeros(2 * N, np.float32)
        nnz = lib().or_gradient(nx, ny, nz, scheme, axis, np.float32(norm), rp, col, val)
        out.append((rp.copy(), col[:nnz].copy(), val[:nnz].copy()))
    return out


def dense_laplacian(nx, ny, nz, scheme, norm):
    """N x N row-major DENSE Laplacian (stencils.cpp:431-570)."""
    N = n_cells(nx, ny, nz)
    A = np.empty((N, N), np.float32)
    lib().or_dense_laplacian(nx, ny, nz, scheme, np.float32(norm), A.reshape(-1))
    return A


def fe_dense(A, dt, B):
    """One DENSE forward-Euler step (kernelprocess.cpp:42-66): (C, D = B + C)."""
    N = A.shape[0]
    C_ = np.zeros(N, np.float32)
    D = np.zeros(N, np.float32)
    lib().or_fe_dense_step(N, np.ascontiguousarray(A, np.float32).reshape(-1), np.float32(dt),
                           np.ascontiguousarray(B, np.float32), C_, D)
    return C_, D


def div3(nx, ny, nz, scheme, norm):
    """The three divergence matrices (operatordivergenceCSR.cpp:21-101): the
    gradient stencils (stencils.cpp:995-1003 forward to them) with the same norm."""
    return gradient3(nx, ny, nz, scheme, norm)


HT_A, HT_B, HT_C, HT_LF = 3.3608, -0.5552, -0.0143, 0.7  # assets/Data/hashtable.ini:3-7


def ht_table_size_reference(nnz, N, a=HT_A, b=HT_B, c=HT_C, lf=HT_LF):
    return int(lib().or_ht_table_size_reference(nnz, N, a, b, c, lf))


def ht_table_size_build(nnz):
    """Next prime >= ceil(nnz / 0.7): the build's policy where the reference
    formula is undefined (N above ~18.6k)."""
    t = max(2, int(np.ceil(nnz / 0.7)))

    def is_prime(n):
        if n < 2:
            return False
        if n % 2 == 0:
            return n == 2
        r = int(n ** 0.5)
        f = 3
        while f <= r:
            if n % f == 0:
                return False
            f += 2
        return True

    while not is_prime(t):
        t += 1
    return t


def ht_build(N, rowptr, col, val, TS):
    keys = np.zeros(TS, np.int64)
    vals = np.zeros(TS, np.float32)
    rc = lib().or_ht_build(N, rowptr, col, val, TS, keys, vals)
    if rc:
        raise RuntimeError(f"or_ht_build failed: {rc}")
    return keys, vals


def csrgeam3(N, A, B, Cm, v):
    rpA, cA, vA = A
    rpB, cB, vB = B
    rpC, cC, vC = Cm
    count = np.zeros(N, np.int32)
    lib().or_csrgeam3_count(N, rpA, rpB, rpC, count)
    rpD = np.zeros(N + 1, np.int32)
    lib().or_scan_rowptr(N, count, rpD)
    nnz = int(rpD[N])
    cD = np.zeros(max(nnz, 1), np.int32)
    vD = np.zeros(max(nnz, 1), np.float32)
    lib().or_csrgeam3_fill(N, rpA, cA, vA, rpB, cB, vB, rpC, cC, vC, np.ascontiguousarray(v, np.float32), rpD, cD, vD)
    return rpD, cD[:nnz], vD[:nnz]


def csr_rowscale(N, rowptr, val, s):
    out = val.copy()
    lib().or_csr_rowscale(N, rowptr, out, np.ascontiguousarray(s, np.float32))
    return out


def csrgeam2(N, A, beta, B):
    rpA, cA, vA = A
    rpB, cB, vB = B
    count = np.zeros(N, np.int32)
    lib().or_csrgeam2_count(N, rpA, cA, rpB, cB, count)
    rpD = np.zeros(N + 1, np.int32)
    lib().or_scan_rowptr(N, count, rpD)
    nnz = int(rpD[N])
    cD = np.zeros(max(nnz, 1), np.int32)
    vD = np.zeros(max(nnz, 1), np.float32)
    lib().or_csrgeam2_fill(N, rpA, cA, vA, np.float32(beta), rpB, cB, vB, rpD, cD, vD)
    return rpD, cD[:nnz], vD[:nnz]


def spmv_csr_fe(nx, ny, nz, A, dt, B, C_in=None):
    N = n_cells(nx, ny, nz)
    C_out = np.zeros(N, np.float32) if C_in is None else C_in.copy()
    lib().or_spmv_csr_fe(N, nx, ny, A[0], A[1], A[2], np.float32(dt), np.ascontiguousarray(B, np.float32), C_out)
    return C_out


def spmv_csr_i1(nx, ny, nz, A, dt, B, C_in=None):
    N = n_cells(nx, ny, nz)
    C_out = np.zeros(N, np.float32) if C_in is None else C_in.copy()
    lib().or_spmv_csr_i1(N, nx, ny, A[0], A[1], A[2], np.float32(dt), np.ascontiguousarray(B, np.float32), C_out)
    return C_out


def spmv_coo(N, coo, dt, B):
    rows, cols, vals = coo
    out = np.zeros(N, np.float32)
    lib().or_spmv_coo(N, len(vals), rows, cols, vals, np.float32(dt), np.ascontiguousarray(B, np.float32), out)
    return out


def spmv_ht(N, keys, vals, dt, B):
    out = np.zeros(N, np.float32)
    lib().or_spmv_ht(N, len(keys), keys, vals, np.float32(dt), np.ascontiguousarray(B, np.float32), out)
    return out


def face_lists(nx, ny, nz):
    N = n_cells(nx, ny, nz)
    idx = np.zeros(max(N, 1), np.uint32)
    fs = np.zeros(7, np.int64)
    q = lib().or_face_lists(nx, ny, nz, idx, fs)
    return idx[:q].copy(), fs


def step_count(total_time, dt):
    return int(lib().or_step_count(np.float32(total_time), np.float32(dt)))


def fe_csr(nx, ny, nz, A, dt, u0, steps, bc_idx=None, bc_src=None):
    """`steps` forward-Euler Solve() calls on CSR with setBC from bc_src."""
    N = n_cells(nx, ny, nz)
    u = np.ascontiguousarray(u0, np.float32).copy()
    if bc_idx is None:
        bc_idx, _ = face_lists(nx, ny, nz)
    if bc_src is None:
        bc_src = u.copy()
    work = np.zeros(N, np.float32)
    for _ in range(steps):
        lib().or_fe_csr_step(N, nx, ny, A[0], A[1], A[2], np.float32(dt), u, len(bc_idx), bc_idx,
                             np.ascontiguousarray(bc_src, np.float32), work)
    return u


def fe_coo(nx, ny, nz, coo, dt, u0, steps, bc_idx=None, bc_src=None):
    N = n_cells(nx, ny, nz)
    u = np.ascontiguousarray(u0, np.float32).copy()
    if bc_idx is None:
        bc_idx, _ = face_lists(nx, ny, nz)
    if bc_src is None:
        bc_src = u.copy()
    work = np.zeros(N, np.float32)
    for _ in range(steps):
        lib().or_fe_coo_step(N, len(coo[2]), coo[0], coo[1], coo[2], np.float32(dt), u, len(bc_idx), bc_idx,
                             np.ascontiguousarray(bc_src, np.float32), work)
    return u


def fe_ht(nx, ny, nz, keys, vals, dt, u0, steps, bc_idx=None, bc_src=None):
    N = n_cells(nx, ny, nz)
    u = np.ascontiguousarray(u0, np.float32).copy()
    if bc_idx is None:
        bc_idx, _ = face_lists(nx, ny, nz)
    if bc_src is None:
        bc_src = u.copy()
    work = np.zeros(N, np.float32)
    for _ in range(steps):
        lib().or_fe_ht_step(N, len(keys), keys, vals, np.float32(dt), u, len(bc_idx), bc_idx,
                            np.ascontiguousarray(bc_src, np.float32), work)
    return u


def stencil_fe(nx, ny, nz, dt, B, alpha=None, idx2=1.0, idy2=1.0, idz2=1.0):
    out = np.zeros(n_cells(nx, ny, nz), np.float32)
    a = None if alpha is None else np.ascontiguousarray(alpha, np.float32)
    lib().or_stencil_fe(nx, ny, nz, idx2, idy2, idz2, np.float32(dt), _ptr(a), np.ascontiguousarray(B, np.float32),
                        out)
    return out


def be_jli(nx, ny, nz, A, dt, b, tol=1e-5, urf=1.0, maxiter=1000):
    N = n_cells(nx, ny, nz)
    x = np.zeros(N, np.float32)
    r = np.zeros(N, np.float32)
    it = lib().or_be_jli(N, nx, ny, A[0], A[1], A[2], np.float32(dt), np.ascontiguousarray(b, np.float32), x, r,
                         np.float32(tol), np.float32(urf), maxiter)
    return x, it


def be_cg_f64(nx, ny, nz, A, alpha, b, rtol=1e-12, maxiter=100000):
    """FP64 Jacobi-PCG solve of the backward-Euler system (interior rows,
    boundary held at b).  A float64 b is used as is (a step of an FP64-only
    trajectory); any other b as float32.  Returns (u float64, iterations,
    final relative residual)."""
    N = n_cells(nx, ny, nz)
    u = np.zeros(N, np.float64)
    rel = C.c_double(0.0)
    al = np.ascontiguousarray(alpha, np.float32)
    if isinstance(b, np.ndarray) and b.dtype == np.float64:
        it = lib().or_be_cg_f64d(N, nx, ny, nz, A[0], A[1], A[2], al, np.ascontiguousarray(b), u, rtol, maxiter,
                                 C.byref(rel))
    else:
        it = lib().or_be_cg_f64(N, nx, ny, nz, A[0], A[1], A[2], al, np.ascontiguousarray(b, np.float32), u, rtol,
                                maxiter, C.byref(rel))
    return u, it, rel.value


def ic_gaussian(nx, ny, nz, l, scale, sigma, mean):
    out = np.zeros(n_cells(nx, ny, nz), np.float32)
    lib().or_ic_gaussian(nx, ny, nz, *map(np.float32, l), np.float32(scale), np.asarray(sigma, np.float32),
                         np.asarray(mean, np.float32), out)
    return out


def ic_coulomb(nx, ny, nz, l, center, Z, e, eps0):
    """e and eps0 as the reference holds them: parsed to float, widened to double."""
    out = np.zeros(n_cells(nx, ny, nz), np.float32)
    lib().or_ic_coulomb(nx, ny, nz, *map(np.float32, l), np.asarray(center, np.float32), np.float32(Z),
                        float(np.float32(e)), float(np.float32(eps0)), out)
    return out


def ic_uniform_vector(N, direction, value):
    out = np.zeros(3 * N, np.float32)
    lib().or_ic_uniform_vector(N, np.asarray(direction, np.float32), np.float32(value), out)
    return out


def set_threads(n):
    lib().or_set_threads(int(n))


def num_threads():
    return int(lib().or_num_threads())


# ----------------------------------------------------------------- reference
class Ref:
    """PIRO's own host functions and .cl kernels, built by `make -C oracle ref`."""

    def __init__(self, path: str = REF_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        i32, f32, ll = C.c_int, C.c_float, C.c_longlong
        vp = C.c_void_p
        L.ref_laplacian.restype = ll
        L.ref_laplacian.argtypes = [i32, i32, i32, i32, i32, f32, vp, vp, _i32p, _f32p]
        L.ref_gradient.restype = None
        L.ref_gradient.argtypes = [i32, i32, i32, i32, f32, _i32p, _i32p, _f32p, np.ctypeslib.ndpointer(np.int64)]
        L.ref_ht_insert_all.restype = i32
        L.ref_ht_insert_all.argtypes = [i32, _i32p, _i32p, _f32p, i32, _i32p, _f32p]
        L.ref_initialcondition.restype = ll
        L.ref_initialcondition.argtypes = [i32, i32, i32, f32, f32, f32, C.c_char_p, C.c_char_p, _f32p]
        L.ref_initbc.restype = ll
        L.ref_initbc.argtypes = [i32, i32, i32, C.c_char_p, C.c_char_p, _i32p, _i32p, _f32p]
        L.refcl_spmvcsr.argtypes = [i32, _f32p, _i32p, _i32p, f32, _f32p, _f32p, C.c_uint, C.c_uint, C.c_uint]
        L.refcl_spmvcsr_i1.argtypes = [i32, _f32p, _i32p, _i32p, f32, _f32p, _f32p, C.c_uint, C.c_uint, C.c_uint]
        L.refcl_spmvcoo.argtypes = [i32, i32, _f32p, _i32p, _i32p, f32, _f32p, _f32p, C.c_uint, C.c_uint, C.c_uint]
        L.refcl_spmvht.argtypes = [_i32p, _f32p, _f32p, _f32p, i32, i32, f32]
        L.refcl_spmvcsr_par.argtypes = L.refcl_spmvcsr.argtypes
        L.refcl_spmvcoo_par.argtypes = L.refcl_spmvcoo.argtypes
        L.refcl_spmvht_par.argtypes = L.refcl_spmvht.argtypes
        L.refcl_add.argtypes = [_f32p, _f32p, _f32p, C.c_uint]
        L.refcl_sub.argtypes = [_f32p, _f32p, _f32p, C.c_uint]
        L.refcl_urf.argtypes = [_f32p, _f32p, f32, C.c_uint]
        L.refcl_csrgeam.argtypes = [i32, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p, _f32p,
                                    _i32p, _i32p, _i32p, _f32p]
        L.refcl_spmdsm.argtypes = [i32, i32, _f32p, _i32p, _i32p, _f32p, i32]
        L.refcl_setbc.argtypes = [_f32p, _f32p, _u32p, C.c_uint]
        L.refcl_laplacianscalar.argtypes = [_f32p, _f32p, f32, f32, f32, C.c_uint, C.c_uint, f32, C.c_uint]
        L.refcl_lu_round.argtypes = [_i32p, _f32p, i32, i32, i32, i32]
        L.ref_div.restype = None
        L.ref_div.argtypes = [i32, i32, i32, i32, f32, _i32p, _i32p, _f32p, np.ctypeslib.ndpointer(np.int64)]
        L.ref_dense_laplacian.restype = None
        L.ref_dense_laplacian.argtypes = [i32, i32, i32, i32, f32, _f32p]
        L.refcl_csrgeam2_merge.argtypes = [i32, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                           _i32p, _i32p, _f32p, _i32p]
        L.refcl_fe_dense.argtypes = [i32, _f32p, _f32p, _f32p, _f32p, f32]
        for n in ("refcl_csrgeam2_merge", "refcl_fe_dense", "refcl_spmvcsr", "refcl_spmvcsr_i1", "refcl_spmvcoo", "refcl_spmvht",
                  "refcl_spmvcsr_par", "refcl_spmvcoo_par", "refcl_spmvht_par", "refcl_add", "refcl_sub",
                  "refcl_urf", "refcl_csrgeam", "refcl_spmdsm", "refcl_setbc", "refcl_laplacianscalar",
                  "refcl_lu_round"):
            getattr(L, n).restype = None

    def laplacian(self, nx, ny, nz, scheme, norm, fmt="csr"):
        N = n_cells(nx, ny, nz)
        cap = 7 * N
        col = np.zeros(cap, np.int32)
        val = np.zeros(cap, np.float32)
        rowptr = np.zeros(N + 1, np.int32)
        rows = np.zeros(cap, np.int32)
        code = {"csr": 0, "ht": 2, "coo": 3}[fmt]
        nnz = self.lib.ref_laplacian(code, nx, ny, nz, scheme, np.float32(norm), _ptr(rowptr), _ptr(rows), col, val)
        if fmt == "coo":
            return rows[:nnz].copy(), col[:nnz].copy(), val[:nnz].copy()
        return rowptr, col[:nnz].copy(), val[:nnz].copy()

    def gradient3(self, nx, ny, nz, scheme, norm):
        N = n_cells(nx, ny, nz)
        rp = np.zeros(3 * (N + 1), np.int32)
        col = np.zeros(6 * N, np.int32)
        val = np.zeros(6 * N, np.float32)
        nnz3 = np.zeros(3, np.int64)
        self.lib.ref_gradient(nx, ny, nz, scheme, np.float32(norm), rp, col, val, nnz3)
        out, off = [], 0
        for a in range(3):
            k = int(nnz3[a])
            out.append((rp[a * (N + 1):(a + 1) * (N + 1)].copy(), col[off:off + k].copy(), val[off:off + k].copy()))
            off += k
        return out

    def ht_insert_all(self, N, rowptr, col, val, TS):
        keys = np.zeros(TS, np.int32)
        vals = np.zeros(TS, np.float32)
        self.lib.ref_ht_insert_all(N, rowptr, col, val, TS, keys, vals)
        return keys, vals

    def initbc(self, nx, ny, nz, assets_root, scalar="T"):
        N = n_cells(nx, ny, nz)
        idx = np.zeros(N, np.int32)
        flen = np.zeros(6, np.int32)
        field = np.zeros(N, np.float32)
        q = self.lib.ref_initbc(nx, ny, nz, assets_root.encode(), scalar.encode(), idx, flen, field)
        return idx[:q].copy(), flen, field

    def paraview(self, nx, ny, nz, origin, spacing, out_dir, casename, timestep, fields):
        """Piro::paraview::writevth (src/paraview.cpp:106-137) on `fields`, a list
        of (name, type 0/1/2, float32 values): writes the .vth and level-0 .vti
        under out_dir/casename/mesh/ and returns (vth text, vti text)."""
        L = self.lib
        L.ref_paraview.restype = None
        mesh = os.path.join(out_dir, casename, "mesh")
        os.makedirs(os.path.join(mesh, "level"), exist_ok=True)
        names = (C.c_char_p * len(fields))(*[f[0].encode() for f in fields])
        types = (C.c_int * len(fields))(*[int(f[1]) for f in fields])
        arrs = [np.ascontiguousarray(f[2], np.float32) for f in fields]
        vals = (C.c_void_p * len(fields))(*[a.ctypes.data for a in arrs])
        L.ref_paraview(nx, ny, nz, *[int(v) for v in origin], *[int(v) for v in spacing], out_dir.encode(),
                       casename.encode(), int(timestep), len(fields), names, types, vals)
        ts = f"{int(timestep):05d}"
        with open(os.path.join(mesh, f"mesh_{ts}.vth")) as f:
            vth = f.read()
        with open(os.path.join(mesh, "level", f"{ts}_level_0.vti")) as f:
            vti = f.read()
        return vth, vti

    def initialcondition(self, nx, ny, nz, l, assets_root, ic_name):
        out = np.zeros(3 * n_cells(nx, ny, nz), np.float32)
        n = self.lib.ref_initialcondition(nx, ny, nz, *map(np.float32, l), assets_root.encode(), ic_name.encode(),
                                          out)
        return out[:n].copy()

    def spmvcsr(self, nx, ny, nz, A, dt, B, C_in):
        N = n_cells(nx, ny, nz)
        Cc = C_in.copy()
        Bc = np.ascontiguousarray(B, np.float32).copy()
        self.lib.refcl_spmvcsr(N, A[2], A[1], A[0], np.float32(dt), Bc, Cc, nx, ny, N)
        return Cc

    def spmvcsr_i1(self, nx, ny, nz, A, dt, B, C_in):
        N = n_cells(nx, ny, nz)
        Cc = C_in.copy()
        Bc = np.ascontiguousarray(B, np.float32).copy()
        self.lib.refcl_spmvcsr_i1(N, A[2], A[1], A[0], np.float32(dt), Bc, Cc, nx, ny, N)
        return Cc

    def spmvcoo(self, nx, ny, nz, coo, dt, B):
        N = n_cells(nx, ny, nz)
        Cc = np.zeros(N, np.float32)
        Bc = np.ascontiguousarray(B, np.float32).copy()
        self.lib.refcl_spmvcoo(N, len(coo[2]), coo[2], coo[1], coo[0], np.float32(dt), Bc, Cc, nx, ny, N)
        return Cc

    def spmvht(self, N, keys32, vals, dt, B):
        Cc = np.zeros(N, np.float32)
        self.lib.refcl_spmvht(keys32, vals, np.ascontiguousarray(B, np.float32), Cc, N, len(keys32), np.float32(dt))
        return Cc

    def spmv_par(self, kind, nx, ny, nz, op, dt, B, C_in=None):
        """One SpMVCSR / SpMVCOO / SpMVHT NDRange over the OpenMP threads
        (set_threads picks the count): the CPU baseline of the SpMV steps.
        op: CSR (rowptr, col, val), COO (rows, col, val), HT (keys32, vals)."""
        N = n_cells(nx, ny, nz)
        Bc = np.ascontiguousarray(B, np.float32)
        if kind == "csr":
            Cc = np.zeros(N, np.float32) if C_in is None else C_in.copy()
            self.lib.refcl_spmvcsr_par(N, op[2], op[1], op[0], np.float32(dt), Bc, Cc, nx, ny, N)
        elif kind == "coo":
            Cc = np.zeros(N, np.float32)
            self.lib.refcl_spmvcoo_par(N, len(op[2]), op[2], op[1], op[0], np.float32(dt), Bc, Cc, nx, ny, N)
        else:
            Cc = np.zeros(N, np.float32)
            self.lib.refcl_spmvht_par(op[0], op[1], Bc, Cc, N, len(op[0]), np.float32(dt))
        return Cc

    def csrgeam(self, N, A, B, Cm, v):
        nnz_x = len(A[2])
        count = np.zeros(N, np.int32)
        rpD = np.zeros(N + 1, np.int32)
        cD = np.zeros(3 * nnz_x, np.int32)
        vD = np.zeros(3 * nnz_x, np.float32)
        self.lib.refcl_csrgeam(N, A[0], A[1], A[2], B[0], B[1], B[2], Cm[0], Cm[1], Cm[2],
                               np.ascontiguousarray(v, np.float32), count, rpD, cD, vD)
        return rpD, cD, vD

    def spmdsm(self, N, A, diag, ind=0):
        v = A[2].copy()
        self.lib.refcl_spmdsm(len(v), N, v, A[1], A[0], np.ascontiguousarray(diag, np.float32), ind)
        return v

    def setbc(self, A, B, idx):
        Ac = A.copy()
        self.lib.refcl_setbc(Ac, np.ascontiguousarray(B, np.float32), idx.astype(np.uint32), len(idx))
        return Ac

    def add(self, B, Cc):
        A = np.zeros_like(B)
        self.lib.refcl_add(A, B, Cc, len(B))
        return A

    def sub(self, B, Cc):
        A = np.zeros_like(B)
        self.lib.refcl_sub(A, B, Cc, len(B))
        return A

    def urf(self, A, Cc, w):
        A2, C2 = A.copy(), Cc.copy()
        self.lib.refcl_urf(A2, C2, np.float32(w), len(A2))
        return A2, C2

    def laplacianscalar(self, nx, ny, nz, B, dt, dx=1.0, dy=1.0, dz=1.0):
        N = n_cells(nx, ny, nz)
        Cc = np.zeros(N, np.float32)
        self.lib.refcl_laplacianscalar(np.ascontiguousarray(B, np.float32).copy(), Cc, dx, dy, dz, nx, ny,
                                       np.float32(dt), N)
        return Cc

    def div3(self, nx, ny, nz, scheme, norm):
        N = n_cells(nx, ny, nz)
        rp = np.zeros(3 * (N + 1), np.int32)
        col = np.zeros(6 * N, np.int32)
        val = np.zeros(6 * N, np.float32)
        nnz3 = np.zeros(3, np.int64)
        self.lib.ref_div(nx, ny, nz, scheme, np.float32(norm), rp, col, val, nnz3)
        out, off = [], 0
        for a in range(3):
            k = int(nnz3[a])
            out.append((rp[a * (N + 1):(a + 1) * (N + 1)].copy(), col[off:off + k].copy(), val[off:off + k].copy()))
            off += k
        return out

    def csrgeam2_merge(self, N, A, B, Cm):
        """kernelmethods::csrgeam_2's merge of three matrices, unscaled."""
        nnz = len(A[2]) + len(B[2]) + len(Cm[2])
        count = np.zeros(N, np.int32)
        rpD = np.zeros(N + 1, np.int32)
        cD = np.zeros(max(nnz, 1), np.int32)
        vD = np.zeros(max(nnz, 1), np.float32)
        self.lib.refcl_csrgeam2_merge(N, A[0], A[1], A[2], B[0], B[1], B[2], Cm[0], Cm[1], Cm[2], rpD, cD, vD,
                                      count)
        k = int(rpD[N])
        return rpD, cD[:k], vD[:k]

    def dense_laplacian(self, nx, ny, nz, scheme, norm):
        N = n_cells(nx, ny, nz)
        A = np.zeros((N, N), np.float32)
        self.lib.ref_dense_laplacian(nx, ny, nz, scheme, np.float32(norm), A.reshape(-1))
        return A

    def fe_dense(self, A, dt, B):
        N = A.shape[0]
        Bc = np.ascontiguousarray(B, np.float32).copy()
        C_ = np.zeros(N, np.float32)
        D = np.zeros(N, np.float32)
        self.lib.refcl_fe_dense(N, np.ascontiguousarray(A, np.float32).reshape(-1), Bc, C_, D, np.float32(dt))
        return C_, D

    def ht_lu(self, N, keys32, vals, TS):
        """Scheme 27's factorization of the table (matrixoperations.cpp:37-99), in place."""
        self.lib.ref_ht_lu.restype = None
        self.lib.ref_ht_lu.argtypes = [C.c_int, _i32p, _f32p, C.c_int]
        self.lib.ref_ht_lu(N, keys32, vals, TS)

    def lu_round(self, keys32, vals, N, rowouter, TS):
        limit = (N - rowouter - 1) * (N - rowouter)
        self.lib.refcl_lu_round(keys32, vals, N, rowouter, TS, limit)


def ref_available() -> bool:
    return os.path.exists(REF_PATH)
