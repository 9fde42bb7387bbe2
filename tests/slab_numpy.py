"""Test infrastructure: the slab backend of piro_b200/slab.py restated on the
CPU (torch CPU tensors, numpy arithmetic) so that the multi-rank
orchestration runs under gloo without a GPU.  Assembly comes from the oracle
(rows of the whole grid's matrix); the forward-Euler rows keep SpMVCSR.cl's
sequential FP32 order, so a sharded step can be compared bit for bit."""
from __future__ import annotations

import numpy as np
import torch

from oracle import oracle as O


def _coef(alpha, dt, norm):
    a = alpha.astype(np.float32)
    vself = np.float32(-6.0 / float(norm))
    vnb = np.float32(1.0 / float(norm))
    mdt = np.float32(-dt)
    cd = np.float32(1.0) + mdt * (a * vself)
    co = mdt * (a * vnb)
    return cd.astype(np.float32), co.astype(np.float32)


class NumpyBackend:
    def empty(self, n, dtype="f32"):
        return torch.zeros(n, dtype=torch.float32 if dtype == "f32" else torch.float64)

    def laplacian_rows(self, nx, ny, nz, scheme, norm, row0, nrows, col_shift):
        rp, col, val = O.laplacian(nx, ny, nz, scheme, np.float32(norm), "csr")
        a, b = int(rp[row0]), int(rp[row0 + nrows])
        return (torch.from_numpy((rp[row0:row0 + nrows + 1] - rp[row0]).astype(np.int32)),
                torch.from_numpy((col[a:b] - col_shift).astype(np.int32)), torch.from_numpy(val[a:b].copy()))

    def gradient_rows(self, nx, ny, nz, scheme, axis, norm, row0, nrows, col_shift):
        rp, col, val = O.gradient3(nx, ny, nz, scheme, np.float32(norm))[axis]
        a, b = int(rp[row0]), int(rp[row0 + nrows])
        return (torch.from_numpy((rp[row0:row0 + nrows + 1] - rp[row0]).astype(np.int32)),
                torch.from_numpy((col[a:b] - col_shift).astype(np.int32)), torch.from_numpy(val[a:b].copy()))

    def geam3(self, nrows, G, v_owned):
        Gn = [tuple(t.numpy() for t in g) for g in G]
        rp, col, val = O.csrgeam3(nrows, *Gn, v_owned.numpy())
        return torch.from_numpy(rp), torch.from_numpy(col), torch.from_numpy(val)

    def rowscale(self, A, s):
        rp, val = A[0].numpy(), A[2].numpy()
        A[2].copy_(torch.from_numpy(O.csr_rowscale(len(rp) - 1, rp, val, s.numpy())))

    def fe_rows(self, nx, ny, nz, row0, nrows, A, dt, u, ubase, out):
        rp, col, val = (t.numpy() for t in A)
        un = u.numpy()
        acc = np.zeros(nrows, np.float32)
        lens = np.diff(rp)
        dt = np.float32(dt)
        for k in range(int(lens.max())):  # entry k of every row: the sequential order per row
            rows = np.nonzero(lens > k)[0]
            e = rp[rows] + k
            acc[rows] = acc[rows] + (dt * val[e]) * un[col[e]]
        g = np.arange(row0, row0 + nrows)
        z, rem = np.divmod(g, nx * ny)
        y, x = np.divmod(rem, nx)
        inter = (x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1)
        o = out.numpy()
        loc = ubase + np.arange(nrows)
        o[loc[inter]] = acc[inter] + un[loc[inter]]

    # ---- backward-Euler slab kernels (semantics of piro_b200/csrc/slab.cu)
    @staticmethod
    def _geom(S):
        nx, ny, nz, z0, z1, dt, norm = S
        plane = nx * ny
        nloc = (z1 - z0 + 2) * plane
        l = np.arange(nloc)
        g = l + (z0 - 1) * plane
        z, rem = np.divmod(g, plane)
        y, x = np.divmod(rem, nx)
        inter = ((x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1) & (g >= 0)
                 & (g < nx * ny * nz))
        own = (l >= plane) & (l < (z1 - z0 + 1) * plane)
        return plane, nx, inter, own

    @staticmethod
    def _nb(v, l, nx, plane):
        return ((v[l - 1] + v[l + 1]) + (v[l - nx] + v[l + nx])) + (v[l - plane] + v[l + plane])

    def residual(self, S, alpha, b, x64, r, z):
        plane, nx, inter, own = self._geom(S)
        cd, co = _coef(alpha.numpy(), S[5], S[6])
        l = np.nonzero(inter & own)[0]
        x, bb = x64.numpy(), b.numpy()
        ri = bb[l].astype(np.float64) - (cd[l].astype(np.float64) * x[l]
                                         + co[l].astype(np.float64) * self._nb(x, l, nx, plane))
        rf = ri.astype(np.float32)
        zf = (rf / cd[l]).astype(np.float32)
        rn, zn = r.numpy(), z.numpy()
        rn[own] = 0.0
        zn[own] = 0.0
        rn[l], zn[l] = rf, zf
        a = alpha.numpy()[l].astype(np.float64)
        return torch.tensor([(ri * ri).sum(), (bb[l].astype(np.float64) ** 2).sum(),
                             (rf.astype(np.float64) / a * zf).sum(), (rf.astype(np.float64) ** 2).sum()])

    def cg_spmv(self, S, beta, alpha, z, p_old, p_new, q):
        plane, nx, inter, own = self._geom(S)
        cd, co = _coef(alpha.numpy(), S[5], S[6])
        beta = np.float32(beta)
        pn = np.where(inter, z.numpy() + beta * p_old.numpy(), np.float32(0.0)).astype(np.float32)
        keep = np.zeros_like(inter)  # the owned planes and the halo planes inside the grid
        keep[(0 if S[3] > 0 else plane):len(keep) - (0 if S[4] < S[2] else plane)] = True
        p_new.numpy()[keep] = pn[keep]
        l = np.nonzero(inter & own)[0]
        qv = (cd[l] * pn[l] + co[l] * self._nb(pn, l, nx, plane)).astype(np.float32)
        q.numpy()[l] = qv
        a = alpha.numpy()[l].astype(np.float64)
        return torch.tensor([(pn[l].astype(np.float64) * qv / a).sum()])

    def cg_update(self, S, a, alpha, p, q, d, r, z):
        plane, nx, inter, own = self._geom(S)
        cd, _ = _coef(alpha.numpy(), S[5], S[6])
        l = np.nonzero(inter & own)[0]
        a = np.float32(a)
        dn, rn, zn = d.numpy(), r.numpy(), z.numpy()
        dn[l] = dn[l] + a * p.numpy()[l]
        rn[l] = rn[l] - a * q.numpy()[l]
        zn[l] = rn[l] / cd[l]
        al = alpha.numpy()[l].astype(np.float64)
        return torch.tensor([(rn[l].astype(np.float64) / al * zn[l]).sum(), (rn[l].astype(np.float64) ** 2).sum()])

    def x_update(self, S, x64, d):
        _, _, inter, own = self._geom(S)
        l = np.nonzero(inter & own)[0]
        x64.numpy()[l] += d.numpy()[l].astype(np.float64)
        d.numpy()[l] = 0.0

    # ---- the same steps with the CG scalars in a state vector (piro_slab_*_dev)
    def cg_spmv_dev(self, S, state, alpha, z, p_old, p_new, q, sums):
        st = state.numpy()
        if st[4] != 0.0:
            return
        sums.copy_(self.cg_spmv(S, float(np.float32(st[1])), alpha, z, p_old, p_new, q))

    def cg_update_dev(self, S, state, pq, alpha, p, q, d, r, z, sums):
        st, t = state.numpy(), float(pq.numpy()[0])
        if st[4] != 0.0:
            return
        a = st[0] / t if t != 0.0 else np.inf
        if not np.isfinite(a) or not t > 0.0:
            return
        sums.copy_(self.cg_update(S, float(np.float32(a)), alpha, p, q, d, r, z))

    def cg_scalars(self, state, pq, up):
        st, t = state.numpy(), float(pq.numpy()[0])
        if st[4] != 0.0:
            return
        a = st[0] / t if t != 0.0 else np.inf
        if not np.isfinite(a) or not t > 0.0:
            st[7] = st[4] = 1.0
            return
        st[2] = a
        rzn, rr = (float(v) for v in up.numpy()[:2])
        beta = rzn / st[0]
        st[5] += 1.0
        st[6] = rr
        if not np.isfinite(rr) or not np.isfinite(beta):
            st[7] = st[4] = 1.0
            return
        st[1], st[0] = beta, rzn
        if rr <= st[3]:
            st[4] = 1.0
