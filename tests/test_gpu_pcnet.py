"""Learned preconditioner on the device: the network's forward and backward
kernels against the CPU oracle (oracle/pcnet_oracle.py), training on the
device, and flexible CG with the trained network against plain Jacobi-PCG."""
import numpy as np
import pytest

from oracle import pcnet_oracle as P

pytestmark = pytest.mark.gpu


def _inputs(seed, n, B):
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    N = nx * ny * nz
    r = rng.standard_normal((B, N)).astype(np.float32)
    f = (rng.standard_normal((B, N)) * 0.5).astype(np.float32)
    t = (rng.standard_normal((B, N)) * 0.1).astype(np.float32)
    m = (rng.random((B, N)) > 0.3).astype(np.float32)
    return r, f, t, m


@pytest.fixture(scope="module")
def net(cuda):
    from piro_b200 import ops
    h = ops.PCNet(seed=0)
    yield h
    h.close()


def test_param_count(net):
    assert net.num_params() == P.num_params()
    w = net.get_params(rounded=True)
    assert np.array_equal(w, P.bf16(net.get_params()).astype(np.float32))


@pytest.mark.parametrize("n,B", [((10, 9, 8), 2), ((7, 12, 9), 1)])
def test_forward_matches_oracle(cuda, net, n, B):
    import torch
    p = P.init_params(11).astype(np.float32)
    net.set_params(p)
    r, f, _, _ = _inputs(1, n, B)
    out = net.forward(*n, torch.from_numpy(r.reshape(-1)).cuda(), torch.from_numpy(f.reshape(-1)).cuda(), batch=B)
    ref = P.forward(p.astype(np.float64), n, r, f, emulate=True)
    got = out.cpu().numpy().reshape(B, -1).astype(np.float64)
    scale = np.abs(ref).max()
    assert scale > 0
    # same BF16 rounding points; only the FP32 vs FP64 accumulation order differs
    assert np.abs(got - ref).max() <= 2e-2 * scale
    assert np.sqrt(((got - ref) ** 2).sum() / (ref ** 2).sum()) < 5e-3
    nx, ny, nz = n
    b = ~P.interior(nx, ny, nz).reshape(-1)
    assert np.all(got[:, b] == 0.0)


@pytest.mark.parametrize("tensor_cores", [True, False])
@pytest.mark.parametrize("n,B", [((9, 8, 10), 2), ((20, 17, 13), 3)])
def test_gradient_matches_oracle(cuda, net, tensor_cores, n, B):
    """Loss and per-layer gradients of the device's training pass against the
    oracle's analytic gradient, on the tensor cores (tcgen05 forward, data
    gradient and weight gradient; the loss gradient enters the last layer in
    BF16) and on the CUDA cores."""
    import torch
    p = P.init_params(5).astype(np.float32)
    net.set_params(p)
    net.set_engine(tensor_cores)
    r, f, t, m = _inputs(2, n, B)
    T = lambda a: torch.from_numpy(a.reshape(-1)).cuda()  # noqa: E731
    loss, g = net.loss_grad(*n, T(r), T(f), T(t), T(m), batch=B, want_grad=True)
    rl, rg = P.loss_grad(p.astype(np.float64), n, r, f, t, m, emulate=True)
    assert abs(loss - rl) <= 1e-4 * abs(rl)
    wo, total = P.layout()
    ends = wo[1:] + [total]
    for l in range(4):
        a, b = g[wo[l]:ends[l]].astype(np.float64), rg[wo[l]:ends[l]]
        rel = np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))
        assert rel < 2e-2, (l, rel)
    net.set_engine(True)


@pytest.mark.parametrize("tensor_cores", [True, False])
def test_gradient_is_deterministic(cuda, net, tensor_cores):
    import torch
    n, B = (12, 11, 10), 3
    net.set_params(P.init_params(6).astype(np.float32))
    net.set_engine(tensor_cores)
    r, f, t, m = _inputs(3, n, B)
    T = lambda a: torch.from_numpy(a.reshape(-1)).cuda()  # noqa: E731
    _, g1 = net.loss_grad(*n, T(r), T(f), T(t), T(m), batch=B, want_grad=True)
    _, g2 = net.loss_grad(*n, T(r), T(f), T(t), T(m), batch=B, want_grad=True)
    assert np.array_equal(g1, g2)
    net.set_engine(True)


def test_tensor_core_and_cuda_core_gradients_agree(cuda, net):
    """The two training engines give the same gradient up to BF16 rounding of
    intermediate values (the tensor cores sum in another order and take the
    loss gradient in BF16)."""
    import torch
    n, B = (18, 14, 12), 2
    net.set_params(P.init_params(8).astype(np.float32))
    r, f, t, m = _inputs(6, n, B)
    T = lambda a: torch.from_numpy(a.reshape(-1)).cuda()  # noqa: E731
    out = []
    for tc in (True, False):
        net.set_engine(tc)
        out.append(net.loss_grad(*n, T(r), T(f), T(t), T(m), batch=B, want_grad=True))
    net.set_engine(True)
    (l1, g1), (l2, g2) = out
    assert abs(l1 - l2) <= 1e-3 * abs(l2)
    wo, total = P.layout()
    ends = wo[1:] + [total]
    for l in range(4):
        a, b = g1[wo[l]:ends[l]].astype(np.float64), g2[wo[l]:ends[l]].astype(np.float64)
        rel = np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))
        assert rel < 2e-2, (l, rel)


def test_training_reduces_loss(cuda):
    import torch
    from piro_b200 import learned, ops
    n, crop = 24, 12
    data = learned.make_dataset(torch, ops, n, range(100, 104), crop, 6)
    netw = ops.PCNet(seed=1)
    hist = learned.train(torch, ops, netw, data, crop, steps=200, batch=8, lr=3e-3, log_every=50)
    first, last = hist[0][1], hist[-1][1]
    assert np.isfinite(last) and last < 0.7 * first, hist
    netw.close()


def _family(n, seed):
    import torch
    from piro_b200 import learned, ops
    alpha, dt, b = learned.be_family(n, seed)
    a_t, b_t = torch.from_numpy(alpha).cuda(), torch.from_numpy(b).cuda()
    _, A = learned.assemble(ops, n, a_t, dt)
    return a_t, b_t, A, dt


def test_flexible_jacobi_is_pcg(cuda):
    """Jacobi run through the flexible-CG kernels takes the iterations of
    Jacobi-PCG (the FCG(1) direction update reduces to PCG's for a fixed
    linear preconditioner)."""
    import torch
    from piro_b200 import ops
    n = 28
    a_t, b_t, A, dt = _family(n, 202)
    its = []
    for flex in (False, True):
        sv = ops.BESolver(n, n, n, A, a_t, stencil=(float(dt), 1.0))
        if flex:
            sv.set_preconditioner(flexible_jacobi=True)
        x = torch.empty_like(b_t)
        info = sv.solve(b_t, x, rtol=1e-8)
        assert info.status == 0 and info.rel_residual <= 1e-8
        its.append(info.inner_iterations)
        sv.close()
    assert abs(its[0] - its[1]) <= 1, its


def test_fallback_to_jacobi(cuda):
    """A network whose output is not finite breaks flexible CG down at once;
    the solve discards that sweep's correction, reverts to Jacobi-PCG and still
    reaches the FP64 residual."""
    import torch
    from piro_b200 import ops
    n = 20
    a_t, b_t, A, dt = _family(n, 201)
    sv = ops.BESolver(n, n, n, A, a_t, stencil=(float(dt), 1.0))
    bad = ops.PCNet(seed=0)
    bad.set_params(np.full(ops.PCNet.num_params(), np.nan, np.float32))
    sv.set_preconditioner(bad)
    x = torch.empty_like(b_t)
    info = sv.solve(b_t, x, rtol=1e-8)
    assert info.status == 0 and info.rel_residual <= 1e-8 and info.fallbacks == 1
    assert torch.isfinite(x).all()
    sv.close()
    bad.close()


def test_learned_fcg_gains_over_jacobi(cuda):
    """A network trained on the device on seeds 100-115 cuts the inner
    iteration count of the backward-Euler solve on held-out fields (it
    preconditions the first iterations of each sweep), at the same FP64
    residual."""
    import torch
    from piro_b200 import learned, ops
    n, crop = 40, 20
    data = learned.make_dataset(torch, ops, n, range(100, 116), crop, 4)
    netw = ops.PCNet(seed=0)
    learned.train(torch, ops, netw, data, crop, steps=600, batch=8, lr=3e-3)
    rows = learned.compare(torch, ops, netw, n, [200, 201])
    for row in rows:
        assert row["learned"]["rel"] <= 1e-8 and row["jacobi"]["rel"] <= 1e-8
        assert row["learned"]["fallbacks"] == 0
        assert row["learned"]["iters"] < row["jacobi"]["iters"], rows
    netw.close()


@pytest.mark.parametrize("n,B", [((10, 9, 8), 2), ((7, 12, 9), 1), ((40, 33, 21), 1)])
def test_tensor_core_forward_matches_oracle(cuda, n, B):
    """The tcgen05 implicit-GEMM layers (TMA-staged BF16 operands, FP32 in
    tensor memory) give the oracle's network output to the same tolerance
    as the CUDA-core kernels."""
    import torch
    from piro_b200 import ops
    net = ops.PCNet(seed=0)
    p = P.init_params(12).astype(np.float32)
    net.set_params(p)
    net.set_engine(True)
    r, f, _, _ = _inputs(4, n, B)
    rt, ft = torch.from_numpy(r.reshape(-1)).cuda(), torch.from_numpy(f.reshape(-1)).cuda()
    got = net.forward(*n, rt, ft, batch=B).cpu().numpy().reshape(B, -1).astype(np.float64)
    ref = P.forward(p.astype(np.float64), n, r, f, emulate=True)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2e-2 * scale
    assert np.sqrt(((got - ref) ** 2).sum() / (ref ** 2).sum()) < 5e-3
    net.set_engine(False)
    cc = net.forward(*n, rt, ft, batch=B).cpu().numpy().reshape(B, -1).astype(np.float64)
    assert np.sqrt(((got - cc) ** 2).sum() / (cc ** 2).sum()) < 5e-3
    net.close()


def test_tensor_core_preconditioner_in_solver(cuda):
    """The solver with the tensor-core network converges like the CUDA-core one."""
    import torch
    from piro_b200 import ops
    n = 34
    a_t, b_t, A, dt = _family(n, 203)
    net = ops.PCNet(seed=3)
    its = []
    for tcore in (False, True):
        net.set_engine(tcore)
        sv = ops.BESolver(n, n, n, A, a_t, stencil=(float(dt), 1.0))
        sv.set_preconditioner(net)
        x = torch.empty_like(b_t)
        info = sv.solve(b_t, x, rtol=1e-8)
        assert info.status == 0 and info.rel_residual <= 1e-8
        its.append(info.inner_iterations)
        sv.close()
    assert abs(its[0] - its[1]) <= 2, its
    net.close()


def test_learned_solve_persistent_and_graph_launched_agree(cuda, monkeypatch):
    """The Jacobi flexible-CG iterations that follow the network's run either
    in one cooperative launch or as graph-launched chunks; both continue from
    the direction the network iteration left and take the same iterations to
    the same FP64 residual."""
    import torch
    from piro_b200 import ops
    n = 32
    a_t, b_t, A, dt = _family(n, 204)
    net = ops.PCNet(seed=3)
    its = []
    for persist in ("1", "0"):
        monkeypatch.setenv("PIRO_BE_PERSISTENT", persist)
        sv = ops.BESolver(n, n, n, A, a_t, stencil=(float(dt), 1.0))
        sv.set_preconditioner(net)
        x = torch.empty_like(b_t)
        info = sv.solve(b_t, x, rtol=1e-8)
        assert info.status == 0 and info.rel_residual <= 1e-8 and info.fallbacks == 0
        its.append(info.inner_iterations)
        sv.close()
    assert abs(its[0] - its[1]) <= 1, its
    net.close()


def test_learned_solution_matches_the_plain_solve(cuda, oracle):
    """The learned solve judges convergence by its own FP64 residual sweep
    (the matrix-free form with the solver's interior-boundary entries); its
    solution must equal the plain persistent solve's, and the FP64 oracle's,
    to the accuracy a 1e-8 residual allows."""
    import torch
    from piro_b200 import ops
    n = 30
    a_t, b_t, A, dt = _family(n, 205)
    net = ops.PCNet(seed=3)
    xs = []
    for learned_pc in (False, True):
        sv = ops.BESolver(n, n, n, A, a_t, stencil=(float(dt), 1.0))
        if learned_pc:
            sv.set_preconditioner(net)
        x = torch.empty_like(b_t)
        info = sv.solve(b_t, x, rtol=1e-8)
        assert info.status == 0 and info.rel_residual <= 1e-8
        xs.append(x.cpu().numpy().astype(np.float64))
        sv.close()
    Ah = tuple(t.cpu().numpy() for t in A)
    ref, _, _ = oracle.be_cg_f64(n, n, n, Ah, a_t.cpu().numpy(), b_t.cpu().numpy(), rtol=1e-13)
    scale = np.abs(ref).max()
    assert np.abs(xs[1] - xs[0]).max() <= 1e-6 * scale
    assert np.abs(xs[1] - ref).max() <= 1e-6 * scale
    net.close()
