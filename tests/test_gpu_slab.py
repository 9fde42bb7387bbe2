"""z-slab decomposition with the CUDA slab kernels: 2 and 3 slabs on one GPU,
run as threads that meet on the host (piro_b200.slab.LocalComm; no kernel of
one slab waits for another's), against the single-grid kernels."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_ranks(world, fn):
    from piro_b200 import slab
    g = slab.LocalGroup(world)
    out, errs = [None] * world, []

    def body(r):
        import torch
        try:
            torch.cuda.set_device(0)
            out[r] = fn(r, slab.LocalComm(g, r))
        except BaseException as e:  # noqa: BLE001
            errs.append(e)
            g.barrier.abort()

    ts = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    return out


def _local(full, z0, z1, plane):
    lo, hi = (z0 - 1) * plane, (z1 + 1) * plane
    loc = np.zeros((z1 - z0 + 2) * plane, full.dtype)
    s0, s1 = max(lo, 0), min(hi, full.size)
    loc[s0 - lo:s1 - lo] = full[s0:s1]
    return loc


@pytest.mark.parametrize("world,scheme", [(2, 3), (3, 1)])
def test_slab_fe_bitexact(cuda, world, scheme):
    import torch
    from piro_b200 import ops, slab
    nx, ny, nz = 20, 17, 23
    N, plane = nx * ny * nz, nx * ny
    rng = np.random.default_rng(1)
    u = rng.random(N).astype(np.float32)
    alpha = (0.5 + rng.random(N)).astype(np.float32)
    A = ops.csr_laplacian(nx, ny, nz, scheme, 1.0)
    ops.csr_rowscale(A[0], A[2], torch.from_numpy(alpha).cuda())
    ref = torch.zeros(N, device="cuda")
    ops.csr_fe_step(nx, ny, nz, A, 0.01, torch.from_numpy(u).cuda(), ref)
    ref = ref.cpu().numpy()
    parts = slab.split_planes(nz, world)

    def fn(r, comm):
        z0, z1 = parts[r]
        be = slab.CudaBackend()
        fe = slab.SlabFE(be, comm, nx, ny, nz, z0, z1, scheme, 1.0,
                         alpha_owned=torch.from_numpy(alpha[z0 * plane:z1 * plane].copy()).cuda())
        ul = torch.from_numpy(_local(u, z0, z1, plane)).cuda()
        o = torch.zeros_like(ul)
        fe.step(ul, o, 0.01)
        torch.cuda.synchronize()
        return o.cpu().numpy()[plane:(z1 - z0 + 1) * plane]

    got = np.concatenate(_run_ranks(world, fn))
    idx = np.arange(N)
    z, rem = np.divmod(idx, plane)
    y, x = np.divmod(rem, nx)
    inter = (x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1)
    assert np.array_equal(got[inter], ref[inter])


@pytest.mark.parametrize("world,scheme", [(2, 1), (3, 3)])
def test_slab_advection_bitexact(cuda, world, scheme):
    import torch
    from piro_b200 import ops, slab
    nx, ny, nz = 20, 17, 23
    N, plane = nx * ny * nz, nx * ny
    rng = np.random.default_rng(2)
    u = rng.random(N).astype(np.float32)
    vel = rng.standard_normal(3 * N).astype(np.float32)
    G = [ops.csr_gradient(nx, ny, nz, scheme, a, 2.0) for a in range(3)]
    A = ops.csrgeam3(N, *G, torch.from_numpy(vel).cuda())
    ref = torch.zeros(N, device="cuda")
    ops.csr_fe_step(nx, ny, nz, A, 0.01, torch.from_numpy(u).cuda(), ref)
    ref = ref.cpu().numpy()
    parts = slab.split_planes(nz, world)

    def fn(r, comm):
        z0, z1 = parts[r]
        be = slab.CudaBackend()
        v_own = np.concatenate([vel[c * N + z0 * plane:c * N + z1 * plane] for c in range(3)])
        ad = slab.SlabAdvection(be, comm, nx, ny, nz, z0, z1, scheme, 2.0, torch.from_numpy(v_own).cuda())
        ul = torch.from_numpy(_local(u, z0, z1, plane)).cuda()
        o = torch.zeros_like(ul)
        ad.step(ul, o, 0.01)
        torch.cuda.synchronize()
        return o.cpu().numpy()[plane:(z1 - z0 + 1) * plane]

    got = np.concatenate(_run_ranks(world, fn))
    idx = np.arange(N)
    z, rem = np.divmod(idx, plane)
    y, x = np.divmod(rem, nx)
    inter = (x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1)
    assert np.array_equal(got[inter], ref[inter])


@pytest.mark.parametrize("world,device_scalars,n", [(2, False, 34), (3, False, 34), (2, True, 34), (3, True, 34),
                                                    (2, True, 36), (3, False, 36)])
def test_slab_be_matches_single_grid(cuda, world, device_scalars, n):
    """device_scalars: the CG scalars formed on the device from all-reduced
    sums (piro_slab_*_dev), the host looking at the done flag every 8
    iterations.  n = 36 (nx % 4 == 0) takes the operator kernel's 16-byte
    path, n = 34 its per-cell path; the update takes its 16-byte path in
    both (nx * ny % 4 == 0)."""
    import torch
    from piro_b200 import learned, ops, slab
    N, plane = n ** 3, n * n
    alpha, dt, b = learned.be_family(n, 204)
    a_t = torch.from_numpy(alpha).cuda()
    _, A = learned.assemble(ops, n, a_t, dt)
    sv = ops.BESolver(n, n, n, A, a_t, stencil=(float(dt), 1.0))
    x = torch.empty(N, device="cuda")
    sv.solve(torch.from_numpy(b).cuda(), x, rtol=1e-10)
    ref = x.double().cpu().numpy()
    sv.close()
    parts = slab.split_planes(n, world)

    def fn(r, comm):
        z0, z1 = parts[r]
        be = slab.CudaBackend()
        s = slab.SlabBE(be, comm, n, n, n, z0, z1, dt, 1.0, torch.from_numpy(_local(alpha, z0, z1, plane)).cuda())
        x64, info = s.solve(torch.from_numpy(_local(b, z0, z1, plane)).cuda(), rtol=1e-10,
                            device_scalars=device_scalars)
        assert info["status"] == "ok", info
        return x64.cpu().numpy()[plane:(z1 - z0 + 1) * plane]

    got = np.concatenate(_run_ranks(world, fn))
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-7, err
