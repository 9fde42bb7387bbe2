"""Torch-facing wrappers of the C ABI (include/piro.h, layer 1).

Device memory comes from torch; every call goes through libpiro_b200.so on
torch's current CUDA stream.  Tensors must be contiguous CUDA tensors of the
documented dtype.  There is no CPU path: a non-CUDA tensor is an error.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import BeInfo, check, lib

i32, f32 = torch.int32, torch.float32


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _p(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("piro_b200 kernels take CUDA tensors only (no CPU fallback)")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


def _need(t: torch.Tensor, dtype: torch.dtype, n: int | None = None, name: str = "tensor") -> None:
    if t.dtype != dtype:
        raise TypeError(f"{name}: expected {dtype}, got {t.dtype}")
    if n is not None and t.numel() < n:
        raise ValueError(f"{name}: expected at least {n} elements, got {t.numel()}")


def cells(nx: int, ny: int, nz: int) -> int:
    return int(nx) * int(ny) * int(nz)


# ----------------------------------------------------------------- assembly
def laplacian_nnz(nx, ny, nz) -> int:
    v = C.c_int64()
    check(lib().piro_laplacian_nnz(nx, ny, nz, C.byref(v)), "piro_laplacian_nnz")
    return v.value


def gradient_nnz(nx, ny, nz, axis) -> int:
    v = C.c_int64()
    check(lib().piro_gradient_nnz(nx, ny, nz, axis, C.byref(v)), "piro_gradient_nnz")
    return v.value


def csr_laplacian(nx, ny, nz, scheme, norm, device="cuda"):
    N, nnz = cells(nx, ny, nz), laplacian_nnz(nx, ny, nz)
    rp = torch.empty(N + 1, dtype=i32, device=device)
    col = torch.empty(nnz, dtype=i32, device=device)
    val = torch.empty(nnz, dtype=f32, device=device)
    check(lib().piro_csr_laplacian(nx, ny, nz, scheme, float(norm), _p(rp), _p(col), _p(val), _stream()),
          "piro_csr_laplacian")
    return rp, col, val


def coo_laplacian(nx, ny, nz, scheme, norm, device="cuda"):
    nnz = laplacian_nnz(nx, ny, nz)
    rows = torch.empty(nnz, dtype=i32, device=device)
    col = torch.empty(nnz, dtype=i32, device=device)
    val = torch.empty(nnz, dtype=f32, device=device)
    check(lib().piro_coo_laplacian(nx, ny, nz, scheme, float(norm), _p(rows), _p(col), _p(val), _stream()),
          "piro_coo_laplacian")
    return rows, col, val


def csr_gradient(nx, ny, nz, scheme, axis, norm, device="cuda"):
    N, nnz = cells(nx, ny, nz), gradient_nnz(nx, ny, nz, axis)
    rp = torch.empty(N + 1, dtype=i32, device=device)
    col = torch.empty(nnz, dtype=i32, device=device)
    val = torch.empty(nnz, dtype=f32, device=device)
    check(lib().piro_csr_gradient(nx, ny, nz, scheme, axis, float(norm), _p(rp), _p(col), _p(val), _stream()),
          "piro_csr_gradient")
    return rp, col, val


def csr_rowscale(rowptr, val, s):
    """In place: val[k] *= s[row(k)]."""
    _need(rowptr, i32, name="rowptr")
    _need(val, f32, name="val")
    _need(s, f32, rowptr.numel() - 1, "s")
    check(lib().piro_csr_rowscale(rowptr.numel() - 1, _p(rowptr), _p(val), _p(s), _stream()), "piro_csr_rowscale")
    return val


def csr_identity(N, device="cuda"):
    rp = torch.empty(N + 1, dtype=i32, device=device)
    col = torch.empty(N, dtype=i32, device=device)
    val = torch.empty(N, dtype=f32, device=device)
    check(lib().piro_csr_identity(N, _p(rp), _p(col), _p(val), _stream()), "piro_csr_identity")
    return rp, col, val


# ---------------------------------------------------------------- hash table
HT_A, HT_B, HT_C, HT_LF = 3.3608, -0.5552, -0.0143, 0.7  # assets/Data/hashtable.ini


def ht_table_size(nnz, N, policy=0, a=HT_A, b=HT_B, c=HT_C, lf=HT_LF) -> int:
    v = C.c_int64()
    check(lib().piro_ht_table_size(nnz, N, policy, a, b, c, lf, C.byref(v)), "piro_ht_table_size")
    return v.value


def ht_build(N, rowptr, col, val, ts):
    keys = torch.empty(ts, dtype=torch.int64, device=rowptr.device)
    vals = torch.empty(ts, dtype=f32, device=rowptr.device)
    wb = C.c_size_t()
    check(lib().piro_ht_build_workspace(ts, C.byref(wb)), "piro_ht_build_workspace")
    work = torch.empty(wb.value, dtype=torch.uint8, device=rowptr.device)
    check(lib().piro_ht_build(N, _p(rowptr), _p(col), _p(val), val.numel(), ts, _p(keys), _p(vals), _p(work),
                              wb.value, _stream()), "piro_ht_build")
    return keys, vals


def ht_lu_reference(N, keys, vals, ts):
    """Scheme 27's factorization of the table, in place (PIRO's algorithm)."""
    check(lib().piro_ht_lu_reference(N, _p(keys), _p(vals), ts, _stream()), "piro_ht_lu_reference")


def dense_laplacian(nx, ny, nz, scheme, norm):
    """N x N DENSE Laplacian on the device (row-major float32)."""
    N = nx * ny * nz
    A = torch.empty((N, N), dtype=torch.float32, device="cuda")
    check(lib().piro_dense_laplacian(nx, ny, nz, scheme, norm, _p(A), A.numel() * 4, _stream()),
          "piro_dense_laplacian")
    return A


def dense_fe_step(A, dt, u, out=None):
    if out is None:
        out = torch.empty_like(u)
    check(lib().piro_dense_fe_step(u.numel(), _p(A), dt, _p(u), _p(out), _stream()), "piro_dense_fe_step")
    return out


def dense_check():
    check(lib().piro_dense_check(_stream()), "piro_dense_check")


class HtLu:
    """Scheme 27 with a solution: shift*I + scale*M (M the table's matrix)
    factorized in FP64 with partial pivoting in a band of bandwidth bw;
    solve(b) -> x (FP64 solve, x rounded to FP32)."""

    def __init__(self, N, bw, keys, vals, ts, shift=1.0, scale=1.0):
        n = C.c_size_t()
        check(lib().piro_ht_lu_band_bytes(N, bw, C.byref(n)), "piro_ht_lu_band_bytes")
        self.N, self.bw, self.nbytes = N, bw, n.value
        self.band = torch.empty(self.nbytes, dtype=torch.uint8, device="cuda")
        check(lib().piro_ht_lu_factor(N, bw, _p(keys), _p(vals), ts, shift, scale, _p(self.band), self.nbytes,
                                      _stream()), "piro_ht_lu_factor")

    def solve(self, b, x=None):
        if x is None:
            x = torch.empty_like(b)
        check(lib().piro_ht_lu_solve(self.N, self.bw, _p(self.band), self.nbytes, _p(b), _p(x), _stream()),
              "piro_ht_lu_solve")
        return x

    def pivots(self):
        """Pivot row of each elimination step (0-based), as numpy int32."""
        import numpy as np
        torch.cuda.synchronize()
        piv = np.empty(self.N, np.int32)
        check(lib().piro_ht_lu_pivots(self.N, self.bw, _p(self.band), self.nbytes, piv.ctypes.data_as(C.c_void_p)),
              "piro_ht_lu_pivots")
        return piv


# ----------------------------------------------------------------- steps
def csr_fe_step(nx, ny, nz, A, dt, u, out):
    check(lib().piro_csr_fe_step(nx, ny, nz, _p(A[0]), _p(A[1]), _p(A[2]), float(dt), _p(u), _p(out), _stream()),
          "piro_csr_fe_step")
    return out


def csr_i1(nx, ny, nz, A, dt, u, out):
    check(lib().piro_csr_i1(nx, ny, nz, _p(A[0]), _p(A[1]), _p(A[2]), float(dt), _p(u), _p(out), _stream()),
          "piro_csr_i1")
    return out


def coo_spmv(N, coo, dt, u, out, fe=False):
    fn = lib().piro_coo_fe_step if fe else lib().piro_coo_spmv
    check(fn(N, coo[2].numel(), _p(coo[0]), _p(coo[1]), _p(coo[2]), float(dt), _p(u), _p(out), _stream()),
          "piro_coo_spmv")
    return out


def ht_spmv(nx, ny, nz, keys, vals, dt, u, out, fe=False):
    check(lib().piro_ht_spmv(nx, ny, nz, _p(keys), _p(vals), keys.numel(), float(dt), int(fe), _p(u), _p(out),
                             _stream()), "piro_ht_spmv")
    return out


def coo_row_index(N, rows):
    """rowstart[N+1] of a row-sorted COO (built once per operator)."""
    rowstart = torch.empty(N + 1, dtype=i32, device="cuda")
    work = torch.empty(256, dtype=torch.uint8, device="cuda")
    check(lib().piro_coo_row_index(N, rows.numel(), _p(rows), _p(rowstart), _p(work), 256, _stream()),
          "piro_coo_row_index")
    return rowstart


def coo_step_indexed(N, rowstart, cols, vals, dt, u, out, fe=False):
    check(lib().piro_coo_step_indexed(N, _p(rowstart), _p(cols), _p(vals), float(dt), int(fe), _p(u), _p(out),
                                      _stream()), "piro_coo_step_indexed")
    return out


def csr_fe_step_bc(nx, ny, nz, A, dt, u, bc, out):
    """memset + SpMVCSR step + setBC from bc (None: faces 0) in one kernel."""
    check(lib().piro_csr_fe_step_bc(nx, ny, nz, _p(A[0]), _p(A[1]), _p(A[2]), float(dt), _p(u), _p(bc), _p(out),
                                    _stream()), "piro_csr_fe_step_bc")
    return out


def ht_row_order(N, ts):
    """Rows by the home slot of their keys (for ht_spmv(order=...))."""
    n = C.c_size_t()
    check(lib().piro_ht_row_order_workspace(N, ts, C.byref(n)), "piro_ht_row_order_workspace")
    work = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    order = torch.empty(N, dtype=i32, device="cuda")
    check(lib().piro_ht_row_order(N, ts, _p(order), _p(work), n.value, _stream()), "piro_ht_row_order")
    return order


def ht_spmv_ordered(nx, ny, nz, keys, vals, dt, order, u, out, fe=False):
    check(lib().piro_ht_spmv_ordered(nx, ny, nz, _p(keys), _p(vals), keys.numel(), float(dt), int(fe), _p(order),
                                     _p(u), _p(out), _stream()), "piro_ht_spmv_ordered")
    return out


def ht_stage(N):
    """The 32-byte-per-row stage piro_ht_spmv_staged writes and reads."""
    n = C.c_size_t()
    check(lib().piro_ht_stage_bytes(N, C.byref(n)), "piro_ht_stage_bytes")
    return torch.empty(n.value // 4, dtype=torch.float32, device="cuda")


def ht_spmv_staged(nx, ny, nz, keys, vals, dt, order, stage, u, out, fe=False):
    check(lib().piro_ht_spmv_staged(nx, ny, nz, _p(keys), _p(vals), keys.numel(), float(dt), int(fe), _p(order),
                                    _p(stage), stage.numel() * stage.element_size(), _p(u), _p(out), _stream()),
          "piro_ht_spmv_staged")
    return out


def stencil_fe_step(nx, ny, nz, dt, u, out, alpha=None, idx2=1.0, idy2=1.0, idz2=1.0):
    check(lib().piro_stencil_fe_step(nx, ny, nz, idx2, idy2, idz2, float(dt), _p(alpha), _p(u), _p(out), _stream()),
          "piro_stencil_fe_step")
    return out


def stencil_check():
    """Raise if a TMA-staged matrix-free step gave up on a stage wait."""
    check(lib().piro_stencil_check(_stream()), "piro_stencil_check")


def set_bc(idx, src, dst):
    check(lib().piro_set_bc(idx.numel(), _p(idx), _p(src), _p(dst), _stream()), "piro_set_bc")
    return dst


def face_lists(nx, ny, nz, device="cuda"):
    q = C.c_int64()
    fs = (C.c_int64 * 7)()
    check(lib().piro_face_count(nx, ny, nz, C.byref(q), fs), "piro_face_count")
    idx = torch.empty(q.value, dtype=torch.int32, device=device)  # uint32 bits
    check(lib().piro_face_lists(nx, ny, nz, _p(idx), _stream()), "piro_face_lists")
    return idx, list(fs)


def vec_op(op, b, c, out=None):
    out = torch.empty_like(b) if out is None else out
    check(lib().piro_vec_op(op, b.numel(), _p(b), _p(c), _p(out), _stream()), "piro_vec_op")
    return out


def vec_op_scalar(op, s, c, out=None):
    out = torch.empty_like(c) if out is None else out
    check(lib().piro_vec_op_scalar(op, c.numel(), float(s), _p(c), _p(out), _stream()), "piro_vec_op_scalar")
    return out


def vec_urf(a, c, urf):
    check(lib().piro_vec_urf(a.numel(), _p(a), _p(c), float(urf), _stream()), "piro_vec_urf")


# ----------------------------------------------------------------- csrgeam
def _scan_work(N, device):
    wb = C.c_size_t()
    check(lib().piro_scan_workspace(N, C.byref(wb)), "piro_scan_workspace")
    return torch.empty(wb.value, dtype=torch.uint8, device=device), wb.value


def csrgeam3(N, A, B, Cm, v):
    dev = A[0].device
    nnz = A[2].numel() + B[2].numel() + Cm[2].numel()
    rp = torch.empty(N + 1, dtype=i32, device=dev)
    col = torch.empty(nnz, dtype=i32, device=dev)
    val = torch.empty(nnz, dtype=f32, device=dev)
    work, wb = _scan_work(N, dev)
    check(lib().piro_csrgeam3(N, _p(A[0]), _p(A[1]), _p(A[2]), _p(B[0]), _p(B[1]), _p(B[2]), _p(Cm[0]), _p(Cm[1]),
                              _p(Cm[2]), _p(v), _p(rp), _p(col), _p(val), _p(work), wb, _stream()), "piro_csrgeam3")
    return rp, col, val


def csrgeam2(N, A, beta, B):
    dev = A[0].device
    rp = torch.empty(N + 1, dtype=i32, device=dev)
    work, wb = _scan_work(N, dev)
    check(lib().piro_csrgeam2_count(N, _p(A[0]), _p(A[1]), _p(B[0]), _p(B[1]), _p(rp), _p(work), wb, _stream()),
          "piro_csrgeam2_count")
    nnz = int(rp[N].item())
    col = torch.empty(nnz, dtype=i32, device=dev)
    val = torch.empty(nnz, dtype=f32, device=dev)
    check(lib().piro_csrgeam2_fill(N, _p(A[0]), _p(A[1]), _p(A[2]), float(beta), _p(B[0]), _p(B[1]), _p(B[2]),
                                   _p(rp), _p(col), _p(val), _stream()), "piro_csrgeam2_fill")
    return rp, col, val


# ----------------------------------------------------------------- reductions
class Reducer:
    """Reusable FP64 dot-product workspace."""

    def __init__(self, n, device="cuda"):
        wb = C.c_size_t()
        check(lib().piro_reduce_workspace(n, C.byref(wb)), "piro_reduce_workspace")
        self.work = torch.zeros(wb.value, dtype=torch.uint8, device=device)
        self.wb = wb.value
        self.out = torch.zeros(1, dtype=torch.float64, device=device)

    def dot(self, x, y):
        check(lib().piro_dot_f64(x.numel(), _p(x), _p(y), _p(self.out), _p(self.work), self.wb, _stream()),
              "piro_dot_f64")
        return self.out


def dot_f64(x, y):
    return float(Reducer(x.numel(), x.device).dot(x, y).item())


# ----------------------------------------------------------------- backward Euler
class BESolver:
    """FP32 Jacobi-PCG inside FP64 iterative refinement for A = I - dt*diag(alpha)*L."""

    def __init__(self, nx, ny, nz, A, alpha, stencil=None):
        """stencil=(dt, norm): A = I - dt*diag(alpha)*L(norm) from the central
        scheme; the inner operator then runs matrix-free when A matches."""
        self.keep = (A, alpha)
        h = C.c_void_p()
        if stencil is None:
            check(lib().piro_be_create(nx, ny, nz, _p(A[0]), _p(A[1]), _p(A[2]), _p(alpha), _stream(), C.byref(h)),
                  "piro_be_create")
        else:
            dt, norm = stencil
            check(lib().piro_be_create_stencil(nx, ny, nz, _p(A[0]), _p(A[1]), _p(A[2]), _p(alpha), float(dt),
                                               float(norm), _stream(), C.byref(h)), "piro_be_create_stencil")
        self.h = h
        self.N = cells(nx, ny, nz)

    @property
    def inner_operator(self):
        k = C.c_int()
        check(lib().piro_be_inner_operator(self.h, C.byref(k)), "piro_be_inner_operator")
        return ["csr", "stencil", "stencil-persistent", "stencil-persistent"][k.value]

    @property
    def persistent_variant(self):
        """'resident' (r, d, q in shared memory), 'global', or None (no persistent kernel)."""
        k = C.c_int()
        check(lib().piro_be_inner_operator(self.h, C.byref(k)), "piro_be_inner_operator")
        return {2: "global", 3: "resident"}.get(k.value)

    def persistent_bytes(self):
        v = C.c_double()
        check(lib().piro_be_persistent_bytes(self.h, C.byref(v)), "piro_be_persistent_bytes")
        return v.value

    def solve(self, b, x, rtol=1e-8, max_outer=20, max_inner=20000, strict=True):
        info = BeInfo()
        st = lib().piro_be_solve(self.h, _p(b), _p(x), rtol, max_outer, max_inner, C.byref(info))
        if strict:
            check(st, "piro_be_solve")
        return info

    def solution_f64(self):
        p = C.c_void_p()
        check(lib().piro_be_solution_f64(self.h, C.byref(p)), "piro_be_solution_f64")
        return p.value

    def set_preconditioner(self, net=None, flexible_jacobi=False):
        """Learned preconditioner (flexible CG) with a PCNet, or Jacobi with None
        (flexible_jacobi: Jacobi run through the flexible-CG iteration)."""
        if flexible_jacobi:
            check(lib().piro_be_set_preconditioner(self.h, 2, None), "piro_be_set_preconditioner")
            self.net = None
            return
        if net is None:
            check(lib().piro_be_set_preconditioner(self.h, 0, None), "piro_be_set_preconditioner")
            self.net = None
        else:
            check(lib().piro_be_set_preconditioner(self.h, 1, net.h), "piro_be_set_preconditioner")
            self.net = net  # keep the network alive while the solver may use it

    def pc_stats(self, reset=False):
        """(network applies, their total ms by CUDA events)."""
        n, ms = C.c_longlong(), C.c_double()
        check(lib().piro_be_pc_stats(self.h, int(reset), C.byref(n), C.byref(ms)), "piro_be_pc_stats")
        return n.value, ms.value

    def kernel_stats(self, reset=False):
        """(CG SpMV launches, their total ms by CUDA events, all kernel launches)."""
        n, ms, k = C.c_longlong(), C.c_double(), C.c_longlong()
        check(lib().piro_be_kernel_stats(self.h, int(reset), C.byref(n), C.byref(ms), C.byref(k)),
              "piro_be_kernel_stats")
        return n.value, ms.value, k.value

    def close(self):
        if self.h:
            lib().piro_be_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def be_jli(nx, ny, nz, A, dt, b, tol=1e-5, urf=1.0, maxiter=1000):
    x = torch.empty_like(b)
    r = torch.empty_like(b)
    it = C.c_int()
    check(lib().piro_be_jli(nx, ny, nz, _p(A[0]), _p(A[1]), _p(A[2]), float(dt), _p(b), _p(x), _p(r), float(tol),
                            float(urf), maxiter, C.byref(it), _stream()), "piro_be_jli")
    return x, it.value


# ----------------------------------------------------------------- learned preconditioner
class PCNet:
    """The learned preconditioner network (include/piro.h, piro_pcnet_*)."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        check(lib().piro_pcnet_create(int(seed), C.byref(h)), "piro_pcnet_create")
        self.h = h

    @staticmethod
    def num_params() -> int:
        n = C.c_int64()
        check(lib().piro_pcnet_num_params(C.byref(n)), "piro_pcnet_num_params")
        return n.value

    def get_params(self, rounded: bool = False):
        import numpy as np
        out = np.empty(self.num_params(), np.float32)
        check(lib().piro_pcnet_get_params(self.h, out.ctypes.data_as(C.c_void_p), out.size, int(rounded)),
              "piro_pcnet_get_params")
        return out

    def set_params(self, params) -> None:
        import numpy as np
        p = np.ascontiguousarray(params, np.float32)
        check(lib().piro_pcnet_set_params(self.h, p.ctypes.data_as(C.c_void_p), p.size), "piro_pcnet_set_params")

    def forward(self, nx, ny, nz, r, feat, out=None, batch=1):
        if out is None:
            out = torch.empty_like(r)
        check(lib().piro_pcnet_forward(self.h, batch, nx, ny, nz, _p(r), _p(feat), _p(out), _stream()),
              "piro_pcnet_forward")
        return out

    def loss_grad(self, nx, ny, nz, r, feat, target, mask, batch=1, want_loss=True, want_grad=False):
        """Forward + backward; returns (loss or None, gradient array or None)."""
        import numpy as np
        loss = C.c_double()
        g = np.empty(self.num_params(), np.float32) if want_grad else None
        check(lib().piro_pcnet_loss_grad(self.h, batch, nx, ny, nz, _p(r), _p(feat), _p(target), _p(mask),
                                         C.byref(loss) if want_loss else None,
                                         g.ctypes.data_as(C.c_void_p) if want_grad else None, _stream()),
              "piro_pcnet_loss_grad")
        return (loss.value if want_loss else None), g

    def set_engine(self, tensor_cores: bool) -> None:
        """Engine of inference and training: tcgen05 tensor cores (the default) or CUDA cores."""
        check(lib().piro_pcnet_set_engine(self.h, 1 if tensor_cores else 0), "piro_pcnet_set_engine")

    def adam_step(self, lr: float) -> None:
        check(lib().piro_pcnet_adam_step(self.h, float(lr), _stream()), "piro_pcnet_adam_step")

    def launches(self) -> int:
        n = C.c_longlong()
        check(lib().piro_pcnet_stats(self.h, C.byref(n)), "piro_pcnet_stats")
        return n.value

    def close(self):
        if getattr(self, "h", None):
            lib().piro_pcnet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------- batched stepping
class Batch:
    """Many independent heat problems stepped in one persistent launch per step
    (include/piro.h, piro_batch_*)."""

    def __init__(self, n, alpha, dt, scheme):
        import numpy as np
        self.n = np.ascontiguousarray(n, np.int32)
        self.alpha = np.ascontiguousarray(alpha, np.float32)
        self.dt = np.ascontiguousarray(dt, np.float32)
        self.scheme = np.ascontiguousarray(scheme, np.int32)
        self.count = int(self.n.size)
        h = C.c_void_p()
        vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        check(lib().piro_batch_create(self.count, vp(self.n), vp(self.alpha), vp(self.dt), vp(self.scheme),
                                      _stream(), C.byref(h)), "piro_batch_create")
        self.h = h
        self.offsets = np.empty(self.count, np.int64)
        tot = C.c_int64()
        check(lib().piro_batch_layout(self.h, vp(self.offsets), C.byref(tot)), "piro_batch_layout")
        self.total = tot.value

    def set_fields(self, u) -> None:
        """u: host numpy float32 array of total cells, or a CUDA tensor."""
        import numpy as np
        if isinstance(u, np.ndarray):
            a = np.ascontiguousarray(u, np.float32)
            check(lib().piro_batch_set_fields(self.h, a.ctypes.data_as(C.c_void_p), 1), "piro_batch_set_fields")
        else:
            check(lib().piro_batch_set_fields(self.h, _p(u), 0), "piro_batch_set_fields")

    def get_fields(self):
        import numpy as np
        out = np.empty(self.total, np.float32)
        check(lib().piro_batch_get_fields(self.h, out.ctypes.data_as(C.c_void_p), 1), "piro_batch_get_fields")
        return out

    def member(self, fields, k):
        n = int(self.n[k])
        o = int(self.offsets[k])
        return fields[o:o + n ** 3]

    def step(self, steps=1, rtol=1e-8) -> float:
        ms = C.c_double()
        check(lib().piro_batch_step(self.h, int(steps), float(rtol), C.byref(ms)), "piro_batch_step")
        return ms.value

    def member_info(self):
        import numpy as np
        st = np.empty(self.count, np.int32)
        sw = np.empty(self.count, np.int32)
        it = np.empty(self.count, np.int32)
        rel = np.empty(self.count, np.float64)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        check(lib().piro_batch_member_info(self.h, vp(st), vp(sw), vp(it), vp(rel)), "piro_batch_member_info")
        return dict(status=st, sweeps=sw, inner=it, rel=rel)

    def schedule(self):
        """'grouped' or 'lockstep' (piro_batch_schedule)."""
        g = C.c_int()
        check(lib().piro_batch_schedule(self.h, C.byref(g)), "piro_batch_schedule")
        return "grouped" if g.value else "lockstep"

    def set_schedule(self, grouped, blocks_per_sm=4):
        check(lib().piro_batch_set_schedule(self.h, int(bool(grouped)), int(blocks_per_sm)),
              "piro_batch_set_schedule")

    def autotune(self, rtol=1e-8):
        t, b = C.c_int(), C.c_int()
        check(lib().piro_batch_autotune(self.h, float(rtol), C.byref(t), C.byref(b)), "piro_batch_autotune")
        return t.value, b.value

    def close(self):
        if getattr(self, "h", None):
            lib().piro_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
