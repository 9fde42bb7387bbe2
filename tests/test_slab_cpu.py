"""z-slab decomposition over world-size 2 and 3 gloo ranks on the CPU: the
orchestration of piro_b200/slab.py (halo exchange, all-reduced sums,
refinement) with the CPU backend of tests/slab_numpy.py, against the whole
grid computed by the oracle."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fields(nx, ny, nz, zero_boundary):
    """Seeded field and alpha.  The backward-Euler case holds the boundary at
    0: the slab operator couples to boundary cells with the stencil value,
    while PIRO's assembled A has 10.0-scaled entries there (stencils.cpp:278-291),
    which only meet nonzero boundary values."""
    rng = np.random.default_rng(5)
    u = rng.random(nx * ny * nz).astype(np.float32)
    alpha = (0.5 + rng.random(nx * ny * nz)).astype(np.float32)
    if zero_boundary:
        v = u.reshape(nz, ny, nx)
        v[0], v[-1] = 0, 0
        v[:, 0], v[:, -1] = 0, 0
        v[:, :, 0], v[:, :, -1] = 0, 0
    return u, alpha


def _velocity(nx, ny, nz):
    """Seeded SoA velocity field (x block, y block, z block)."""
    return np.random.default_rng(6).standard_normal(3 * nx * ny * nz).astype(np.float32)


def _rank_main(rank, world, port, task, out_dir):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from piro_b200 import slab
        from tests.slab_numpy import NumpyBackend
        kind, nx, ny, nz, arg = task
        z0, z1 = slab.split_planes(nz, world)[rank]
        plane = nx * ny
        comm = slab.TorchComm()
        be = NumpyBackend()
        full, alpha = _fields(nx, ny, nz, zero_boundary=(kind == "be"))
        lo, hi = (z0 - 1) * plane, (z1 + 1) * plane
        loc = np.zeros((z1 - z0 + 2) * plane, np.float32)
        a_loc = np.zeros_like(loc)
        s0, s1 = max(lo, 0), min(hi, nx * ny * nz)
        loc[s0 - lo:s1 - lo] = full[s0:s1]
        a_loc[s0 - lo:s1 - lo] = alpha[s0:s1]
        if kind == "adv":
            vel = _velocity(nx, ny, nz)
            N = nx * ny * nz
            v_own = np.concatenate([vel[c * N + z0 * plane:c * N + z1 * plane] for c in range(3)])
            ad = slab.SlabAdvection(be, comm, nx, ny, nz, z0, z1, arg, 2.0, torch.from_numpy(v_own))
            u = torch.from_numpy(loc)
            out = torch.zeros_like(u)
            ad.step(u, out, 0.01)
            res = out.numpy()[plane:(z1 - z0 + 1) * plane]
        elif kind == "fe":
            fe = slab.SlabFE(be, comm, nx, ny, nz, z0, z1, arg, 1.0,
                             alpha_owned=torch.from_numpy(alpha[z0 * plane:z1 * plane].copy()))
            u = torch.from_numpy(loc)
            out = torch.zeros_like(u)
            fe.step(u, out, 0.01)
            res = out.numpy()[plane:(z1 - z0 + 1) * plane]
        else:
            dt, dev = arg if isinstance(arg, tuple) else (arg, False)
            sv = slab.SlabBE(be, comm, nx, ny, nz, z0, z1, dt, 1.0, torch.from_numpy(a_loc))
            x64, info = sv.solve(torch.from_numpy(loc), rtol=1e-10, device_scalars=dev, check_every=3)
            assert info["status"] == "ok", info
            res = x64.numpy()[plane:(z1 - z0 + 1) * plane]
        np.save(os.path.join(out_dir, f"r{rank}.npy"), res)
    finally:
        dist.destroy_process_group()


def _run(world, task):
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), task, d), nprocs=world, join=True,
                           start_method="spawn")
        return np.concatenate([np.load(os.path.join(d, f"r{r}.npy")) for r in range(world)])


def _interior(nx, ny, nz):
    idx = np.arange(nx * ny * nz)
    z, rem = np.divmod(idx, nx * ny)
    y, x = np.divmod(rem, nx)
    return (x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1)


@pytest.mark.parametrize("world,scheme", [(2, 3), (3, 1), (2, 2)])
def test_slab_fe_matches_whole_grid(oracle, world, scheme):
    nx, ny, nz = 7, 6, 9
    got = _run(world, ("fe", nx, ny, nz, scheme))
    O = oracle
    u, alpha = _fields(nx, ny, nz, False)
    rp, col, val = O.laplacian(nx, ny, nz, scheme, np.float32(1.0), "csr")
    val = O.csr_rowscale(nx * ny * nz, rp, val, alpha)
    ref = O.spmv_csr_fe(nx, ny, nz, (rp, col, val), np.float32(0.01), u, np.zeros_like(u))
    inter = _interior(nx, ny, nz)
    assert np.array_equal(got[inter], ref[inter])  # bit for bit on every stepped row


@pytest.mark.parametrize("world,device_scalars", [(2, False), (3, False), (2, True), (3, True)])
def test_slab_be_matches_whole_grid(oracle, world, device_scalars):
    """device_scalars: the CG scalars stay in a device state vector formed from
    all-reduced sums (piro_slab_*_dev); the host looks at the flags every 3
    iterations and finished iterations are no-ops on every rank."""
    nx, ny, nz = 8, 7, 10
    dt = 2.0
    got = _run(world, ("be", nx, ny, nz, (dt, device_scalars)))
    O = oracle
    u, alpha = _fields(nx, ny, nz, True)
    N = nx * ny * nz
    rp, col, val = O.laplacian(nx, ny, nz, 3, np.float32(1.0), "csr")
    val = O.csr_rowscale(N, rp, val, alpha)
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = O.csrgeam2(N, I, np.float32(-dt), (rp, col, val))
    x64, _, _ = O.be_cg_f64(nx, ny, nz, A, alpha, u, rtol=1e-13)
    inter = _interior(nx, ny, nz)
    err = np.abs(got[inter] - x64[inter]).max() / np.abs(x64[inter]).max()
    assert err < 1e-8, err


@pytest.mark.parametrize("world,scheme", [(2, 1), (3, 3)])
def test_slab_advection_matches_whole_grid(oracle, world, scheme):
    """vector(v) & gradient(U) sharded by z-slabs: each rank merges its own
    gradient rows with its part of v; the step equals the whole grid's."""
    nx, ny, nz = 7, 6, 9
    got = _run(world, ("adv", nx, ny, nz, scheme))
    O = oracle
    u, _ = _fields(nx, ny, nz, False)
    A = O.csrgeam3(nx * ny * nz, *O.gradient3(nx, ny, nz, scheme, np.float32(2.0)), _velocity(nx, ny, nz))
    ref = O.spmv_csr_fe(nx, ny, nz, A, np.float32(0.01), u, np.zeros_like(u))
    inter = _interior(nx, ny, nz)
    assert np.array_equal(got[inter], ref[inter])
