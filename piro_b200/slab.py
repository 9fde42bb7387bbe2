"""z-slab decomposition of one grid over ranks: one process per GPU, planes
split along z, one halo plane exchanged with each neighbour, FP64 sums
all-reduced.  PIRO runs one grid in one process (src/solve.cpp:11-48); this is
the path for a grid that should span several GPUs.

A rank owns grid planes [z0, z1) and keeps arrays of planes z0-1 .. z1 (local
cell l = grid cell l + (z0-1)*nx*ny); the halo planes outside the grid are
never read by an owned interior row.

- SlabFE: the owned rows of PIRO's assembled CSR matrix
  (piro_csr_laplacian_rows, columns local) stepped as SpMVCSR.cl after a halo
  exchange of u: a sharded forward-Euler step equals the single-grid step bit
  for bit.
- SlabAdvection: ddt_r(U) = vector(v) & gradient(U) on the slab: the owned
  rows of the three gradient matrices (piro_csr_gradient_rows, columns
  local) merged with the owned part of v by csrgeam (a row-local merge, so no
  shard needs another's row offsets), then stepped like SlabFE: bit for bit
  the single-grid advection step.
- SlabBE: the single-grid backward-Euler method -- FP32 Jacobi-PCG inside FP64
  iterative refinement on A = I - dt*diag(alpha)*L (central scheme) -- with a
  matrix-free operator on the slab: per CG iteration one halo exchange of z
  and two all-reduces (<p, Sp>; <r, z> with |r|^2), per refinement sweep one
  exchange of x64 and one all-reduce.

The orchestration is written once against two small interfaces: a
communicator (halo exchange, sum) and a backend (the slab kernels).
CudaBackend runs the kernels of libpiro_b200.so on torch CUDA tensors;
TorchComm uses torch.distributed (NCCL across GPUs, gloo on CPU); LocalComm
runs several slabs as threads of one process, meeting on the host.
"""
from __future__ import annotations

import ctypes as C
import math
import threading

import numpy as np


def split_planes(nz: int, world: int):
    """Contiguous, balanced z ranges [(z0, z1)] of the grid's planes."""
    if world > nz:
        raise ValueError(f"cannot split {nz} planes over {world} ranks")
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


# ------------------------------------------------------------------ communicators
class TorchComm:
    """Halo planes and sums over torch.distributed (the default process group)."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()

    def halo(self, t, plane: int) -> None:
        dist = self.dist
        nzl = t.numel() // plane
        ops = []
        if self.rank > 0:
            ops.append(dist.P2POp(dist.isend, t[plane:2 * plane], self.rank - 1))
            ops.append(dist.P2POp(dist.irecv, t[0:plane], self.rank - 1))
        if self.rank < self.world - 1:
            ops.append(dist.P2POp(dist.isend, t[(nzl - 2) * plane:(nzl - 1) * plane], self.rank + 1))
            ops.append(dist.P2POp(dist.irecv, t[(nzl - 1) * plane:nzl * plane], self.rank + 1))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def allsum(self, t):
        self.dist.all_reduce(t)
        return t


class LocalGroup:
    """Ranks emulated as threads of one process (all slabs on one device):
    halo copies and sums between the threads' own tensors, in rank order.  No
    kernel of one rank waits for another rank's: the threads meet on the host."""

    def __init__(self, world: int):
        self.world = world
        self.barrier = threading.Barrier(world, timeout=120)
        self.slot = [None] * world


class LocalComm:
    def __init__(self, group: LocalGroup, rank: int):
        self.g, self.rank, self.world = group, rank, group.world

    def halo(self, t, plane: int) -> None:
        g, r = self.g, self.rank
        g.slot[r] = t
        g.barrier.wait()
        nzl = t.numel() // plane
        if r > 0:
            lo = g.slot[r - 1]
            nl = lo.numel() // plane
            t[0:plane].copy_(lo[(nl - 2) * plane:(nl - 1) * plane])
        if r < self.world - 1:
            t[(nzl - 1) * plane:nzl * plane].copy_(g.slot[r + 1][plane:2 * plane])
        g.barrier.wait()

    def allsum(self, t):
        g, r = self.g, self.rank
        g.slot[r] = t.clone()
        g.barrier.wait()
        tot = g.slot[0].clone()
        for k in range(1, self.world):
            tot += g.slot[k]
        g.barrier.wait()
        t.copy_(tot)
        return t


# ------------------------------------------------------------------ CUDA backend
class CudaBackend:
    """Slab kernels of libpiro_b200.so on torch CUDA tensors."""

    def __init__(self):
        import torch

        from ._lib import check, lib
        from .ops import _p, _stream
        self.torch, self.lib, self.check, self._p, self._stream = torch, lib, check, _p, _stream
        n = C.c_int64()
        check(lib().piro_slab_workspace(C.byref(n)), "piro_slab_workspace")
        self.work = torch.empty(n.value, dtype=torch.float64, device="cuda")

    def empty(self, n, dtype="f32"):
        t = self.torch
        return t.zeros(n, dtype=t.float32 if dtype == "f32" else t.float64, device="cuda")

    def laplacian_rows(self, nx, ny, nz, scheme, norm, row0, nrows, col_shift):
        t, L = self.torch, self.lib()
        nnz = C.c_int64()
        self.check(L.piro_laplacian_nnz_rows(nx, ny, nz, row0, nrows, C.byref(nnz)), "piro_laplacian_nnz_rows")
        rp = t.empty(nrows + 1, dtype=t.int32, device="cuda")
        col = t.empty(nnz.value, dtype=t.int32, device="cuda")
        val = t.empty(nnz.value, dtype=t.float32, device="cuda")
        self.check(L.piro_csr_laplacian_rows(nx, ny, nz, scheme, float(norm), row0, nrows, col_shift, self._p(rp),
                                             self._p(col), self._p(val), self._stream()), "piro_csr_laplacian_rows")
        return rp, col, val

    def rowscale(self, A, s):
        from . import ops
        ops.csr_rowscale(A[0], A[2], s)

    def gradient_rows(self, nx, ny, nz, scheme, axis, norm, row0, nrows, col_shift):
        t, L = self.torch, self.lib()
        nnz = C.c_int64()
        self.check(L.piro_gradient_nnz_rows(nx, ny, nz, axis, row0, nrows, C.byref(nnz)), "piro_gradient_nnz_rows")
        rp = t.empty(nrows + 1, dtype=t.int32, device="cuda")
        col = t.empty(nnz.value, dtype=t.int32, device="cuda")
        val = t.empty(nnz.value, dtype=t.float32, device="cuda")
        self.check(L.piro_csr_gradient_rows(nx, ny, nz, scheme, axis, float(norm), row0, nrows, col_shift,
                                            self._p(rp), self._p(col), self._p(val), self._stream()),
                   "piro_csr_gradient_rows")
        return rp, col, val

    def geam3(self, nrows, G, v_owned):
        from . import ops
        return ops.csrgeam3(nrows, *G, v_owned)

    def fe_rows(self, nx, ny, nz, row0, nrows, A, dt, u, ubase, out):
        self.check(self.lib().piro_csr_fe_step_rows(nx, ny, nz, row0, nrows, self._p(A[0]), self._p(A[1]),
                                                    self._p(A[2]), float(dt), self._p(u), ubase, self._p(out),
                                                    self._stream()), "piro_csr_fe_step_rows")

    def _sums(self, n):
        return self.torch.zeros(n, dtype=self.torch.float64, device="cuda")

    def residual(self, S, alpha, b, x64, r, z):
        s = self._sums(4)
        self.check(self.lib().piro_slab_be_residual(*S, self._p(alpha), self._p(b), self._p(x64), self._p(r),
                                                    self._p(z), self._p(self.work), self._p(s), self._stream()),
                   "piro_slab_be_residual")
        return s

    def cg_spmv(self, S, beta, alpha, z, p_old, p_new, q):
        s = self._sums(1)
        self.check(self.lib().piro_slab_cg_spmv(*S, float(beta), self._p(alpha), self._p(z), self._p(p_old),
                                                self._p(p_new), self._p(q), self._p(self.work), self._p(s),
                                                self._stream()), "piro_slab_cg_spmv")
        return s

    def cg_update(self, S, a, alpha, p, q, d, r, z):
        s = self._sums(2)
        self.check(self.lib().piro_slab_cg_update(*S, float(a), self._p(alpha), self._p(p), self._p(q), self._p(d),
                                                  self._p(r), self._p(z), self._p(self.work), self._p(s),
                                                  self._stream()), "piro_slab_cg_update")
        return s

    def x_update(self, S, x64, d):
        nx, ny, nz, z0, z1 = S[:5]
        self.check(self.lib().piro_slab_x_update(nx, ny, nz, z0, z1, self._p(x64), self._p(d), self._stream()),
                   "piro_slab_x_update")

    # steps with the CG scalars on the device (state: double[8], see include/piro.h)
    def cg_spmv_dev(self, S, state, alpha, z, p_old, p_new, q, sums):
        self.check(self.lib().piro_slab_cg_spmv_dev(*S, self._p(state), self._p(alpha), self._p(z), self._p(p_old),
                                                    self._p(p_new), self._p(q), self._p(self.work), self._p(sums),
                                                    self._stream()), "piro_slab_cg_spmv_dev")

    def cg_update_dev(self, S, state, pq, alpha, p, q, d, r, z, sums):
        self.check(self.lib().piro_slab_cg_update_dev(*S, self._p(state), self._p(pq), self._p(alpha), self._p(p),
                                                      self._p(q), self._p(d), self._p(r), self._p(z),
                                                      self._p(self.work), self._p(sums), self._stream()),
                   "piro_slab_cg_update_dev")

    def cg_scalars(self, state, pq, up):
        self.check(self.lib().piro_slab_cg_scalars(self._p(state), self._p(pq), self._p(up), self._stream()),
                   "piro_slab_cg_scalars")


# ------------------------------------------------------------------ solvers
class SlabFE:
    """Forward Euler (TIMESCHEME 11, CSR) on this rank's slab."""

    def __init__(self, backend, comm, nx, ny, nz, z0, z1, scheme, norm, alpha_owned=None):
        self.b, self.comm = backend, comm
        self.nx, self.ny, self.nz, self.z0, self.z1 = nx, ny, nz, z0, z1
        self.plane = nx * ny
        self.row0 = z0 * self.plane
        self.nrows = (z1 - z0) * self.plane
        self.A = backend.laplacian_rows(nx, ny, nz, scheme, norm, self.row0, self.nrows, (z0 - 1) * self.plane)
        if alpha_owned is not None:
            backend.rowscale(self.A, alpha_owned)

    def local_cells(self) -> int:
        return (self.z1 - self.z0 + 2) * self.plane

    def step(self, u, out, dt) -> None:
        """out = u + dt*A u on the owned interior rows (u's halo planes are exchanged first)."""
        self.comm.halo(u, self.plane)
        self.b.fe_rows(self.nx, self.ny, self.nz, self.row0, self.nrows, self.A, dt, u, self.plane, out)


class SlabAdvection(SlabFE):
    """Advection (simindex 1, TIMESCHEME 11, CSR) on this rank's slab:
    vector(v) & gradient(U) over the owned rows.  v_owned is the owned part
    of the SoA vector field: three blocks of (z1-z0)*nx*ny values."""

    def __init__(self, backend, comm, nx, ny, nz, z0, z1, scheme, gnorm, v_owned):
        self.b, self.comm = backend, comm
        self.nx, self.ny, self.nz, self.z0, self.z1 = nx, ny, nz, z0, z1
        self.plane = nx * ny
        self.row0 = z0 * self.plane
        self.nrows = (z1 - z0) * self.plane
        shift = (z0 - 1) * self.plane
        G = [backend.gradient_rows(nx, ny, nz, scheme, a, gnorm, self.row0, self.nrows, shift) for a in range(3)]
        self.A = backend.geam3(self.nrows, G, v_owned)


class SlabBE:
    """Backward Euler (TIMESCHEME 12) on this rank's slab: FP32 Jacobi-PCG in
    FP64 refinement, matrix-free A = I - dt*diag(alpha)*L (central scheme)."""

    def __init__(self, backend, comm, nx, ny, nz, z0, z1, dt, norm, alpha_local):
        self.b, self.comm = backend, comm
        self.S = (nx, ny, nz, z0, z1, float(dt), float(norm))
        self.plane = nx * ny
        n = (z1 - z0 + 2) * self.plane
        self.n = n
        self.alpha = alpha_local
        self.r, self.z, self.q, self.d = (backend.empty(n) for _ in range(4))
        self.p = [backend.empty(n), backend.empty(n)]
        self.x64 = backend.empty(n, "f64")
        self.comm.halo(self.alpha, self.plane)

    def _sum(self, t):
        return self.comm.allsum(t).cpu().numpy().astype(np.float64)

    def solve(self, b, rtol=1e-8, max_outer=20, max_inner=20000, inner_floor=1e-6, device_scalars=False,
              check_every=8):
        """device_scalars: the CG step lengths, directions and stop test stay
        on the device (all-reduced into device buffers, read by the next
        kernel); the host looks at the done flag every `check_every`
        iterations, so an iteration costs no host round trip."""
        if device_scalars:
            return self._solve_dev(b, rtol, max_outer, max_inner, inner_floor, check_every)
        return self._solve_host(b, rtol, max_outer, max_inner, inner_floor)

    def _solve_dev(self, b, rtol, max_outer, max_inner, inner_floor, check_every):
        S, B = self.S, self.b
        self.comm.halo(b, self.plane)
        self.x64.copy_(b)
        self.d.zero_()
        state = B.empty(8, "f64")
        pq, up = B.empty(1, "f64"), B.empty(2, "f64")
        info = dict(status="not converged", outer=0, inner=0, rel=math.inf)
        prev = math.inf
        for outer in range(max_outer + 1):
            self.comm.halo(self.x64, self.plane)
            s = self._sum(B.residual(S, self.alpha, b, self.x64, self.r, self.z))  # one host sync per sweep
            bn = math.sqrt(s[1]) if s[1] > 0 else 1.0
            rel = math.sqrt(s[0]) / bn
            info["rel"] = rel
            if not math.isfinite(rel):
                info["status"] = "stalled"
                break
            if rel <= rtol:
                info["status"] = "ok"
                break
            if outer == max_outer or info["inner"] >= max_inner:
                break
            if outer > 0 and rel > 0.5 * prev:
                info["status"] = "stalled"
                break
            prev = rel
            info["outer"] = outer + 1
            itol = min(0.1, max(inner_floor, 0.5 * rtol / rel)) if rel > 0 else 1.0
            st = np.zeros(8)
            st[0], st[3] = s[2], itol * itol * s[3]
            st[4] = 1.0 if s[3] <= 0.0 else 0.0
            state.copy_(self.b_tensor(st, state))
            k, taken = 0, 0
            while True:
                for _ in range(check_every):
                    self.comm.halo(self.z, self.plane)
                    p_old, p_new = self.p[k & 1], self.p[(k + 1) & 1]
                    B.cg_spmv_dev(S, state, self.alpha, self.z, p_old, p_new, self.q, pq)
                    self.comm.allsum(pq)
                    B.cg_update_dev(S, state, pq, self.alpha, p_new, self.q, self.d, self.r, self.z, up)
                    self.comm.allsum(up)
                    B.cg_scalars(state, pq, up)
                    k += 1
                h = state.cpu().numpy()  # the host's look at the flags
                taken = int(h[5])
                if h[4] != 0.0 or info["inner"] + taken >= max_inner:
                    break
            info["inner"] += taken
            if h[7] != 0.0:
                info["status"] = "stalled"
                break
            B.x_update(S, self.x64, self.d)
        return self.x64, info

    @staticmethod
    def b_tensor(values, like):
        import torch
        return torch.as_tensor(values, dtype=torch.float64).to(like.device)

    def _solve_host(self, b, rtol=1e-8, max_outer=20, max_inner=20000, inner_floor=1e-6):
        """x64 (owned planes valid) for A x = b; b's halo planes are exchanged here."""
        S, B = self.S, self.b
        self.comm.halo(b, self.plane)
        self.x64.copy_(b)
        self.d.zero_()
        info = dict(status="not converged", outer=0, inner=0, rel=math.inf)
        prev = math.inf
        for outer in range(max_outer + 1):
            self.comm.halo(self.x64, self.plane)
            s = self._sum(B.residual(S, self.alpha, b, self.x64, self.r, self.z))
            bn = math.sqrt(s[1]) if s[1] > 0 else 1.0
            rel = math.sqrt(s[0]) / bn
            info["rel"] = rel
            if not math.isfinite(rel):
                info["status"] = "stalled"
                break
            if rel <= rtol:
                info["status"] = "ok"
                break
            if outer == max_outer or info["inner"] >= max_inner:
                break
            if outer > 0 and rel > 0.5 * prev:
                info["status"] = "stalled"
                break
            prev = rel
            info["outer"] = outer + 1
            itol = min(0.1, max(inner_floor, 0.5 * rtol / rel)) if rel > 0 else 1.0
            tol2, rr0, rz, beta = itol * itol, s[3], s[2], 0.0
            k = 0
            while info["inner"] < max_inner:
                self.comm.halo(self.z, self.plane)
                p_old, p_new = self.p[k & 1], self.p[(k + 1) & 1]
                pq = self._sum(B.cg_spmv(S, beta, self.alpha, self.z, p_old, p_new, self.q))[0]
                a = rz / pq if pq > 0 else math.nan
                if not math.isfinite(a):
                    info["status"] = "stalled"
                    break
                u = self._sum(B.cg_update(S, a, self.alpha, p_new, self.q, self.d, self.r, self.z))
                info["inner"] += 1
                k += 1
                beta, rz = u[0] / rz, u[0]
                if not math.isfinite(u[1]) or u[1] <= tol2 * rr0:
                    break
            if info["status"] == "stalled":
                break
            B.x_update(S, self.x64, self.d)
        return self.x64, info
