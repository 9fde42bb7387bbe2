"""The learned-preconditioner network's CPU oracle (oracle/pcnet_oracle.py).

PIRO has no learned component, so nothing in the reference pins this oracle;
it is pinned here by central finite differences of its own loss (float64,
no rounding) and by the BF16 rounding rule it emulates.
"""
import numpy as np
import pytest

from oracle import pcnet_oracle as P


def _problem(seed, n=(6, 5, 7), B=2):
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    N = nx * ny * nz
    r = rng.standard_normal((B, N))
    f = rng.standard_normal((B, N)) * 0.5
    t = rng.standard_normal((B, N)) * 0.1
    m = (rng.random((B, N)) > 0.3).astype(np.float64)
    return n, r, f, t, m


def test_layout():
    assert P.num_params() == 27 * (2 * 16 + 16 * 16 + 16 * 16 + 16)
    wo, total = P.layout()
    assert wo == [0, 864, 864 + 6912, 864 + 2 * 6912] and total == wo[-1] + 432


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -3.14159, 0.0, 65504.0], np.float32)
    y = P.bf16(x)
    # 1 + 2^-9 is a tie between 1 and 1 + 2^-7... (bf16 keeps 7 fraction bits): ties go to even
    assert y[0] == 1.0 and y[3] == 1.0
    assert y[1] == 1.0  # 1 + 2^-8 < half ulp (2^-8 is exactly half of 2^-7: tie -> even = 1.0)
    assert y[2] == 1.0 + 2 ** -7
    assert abs(y[4] - (-3.140625)) < 1e-12
    assert y[5] == 0.0


@pytest.mark.parametrize("seed", [0, 1])
def test_gradient_matches_finite_differences(seed):
    n, r, f, t, m = _problem(seed)
    p = P.init_params(seed)
    loss, g = P.loss_grad(p, n, r, f, t, m, emulate=False)
    rng = np.random.default_rng(100 + seed)
    wo, total = P.layout()
    ends = wo[1:] + [total]
    # a few weights of every layer
    idx = []
    for l in range(4):
        idx += list(rng.integers(wo[l], ends[l], size=8))
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = P.loss_grad(pp, n, r, f, t, m, emulate=False)
        lm, _ = P.loss_grad(pm, n, r, f, t, m, emulate=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_zero_maps_to_zero():
    n, r, f, _, _ = _problem(4)
    p = P.init_params(4)
    out = P.forward(p, n, np.zeros_like(r), f, emulate=False)
    assert np.all(out == 0.0)


def test_zero_padding_and_boundary():
    n, r, f, t, m = _problem(3)
    p = P.init_params(3)
    out = P.forward(p, n, r, f, emulate=False)
    nx, ny, nz = n
    b = ~P.interior(nx, ny, nz).reshape(-1)
    assert np.all(out[:, b] == 0.0)
    # boundary input values do not reach the output (they are masked to zero)
    r2 = r.copy()
    r2[:, b] += 100.0
    assert np.array_equal(P.forward(p, n, r2, f, emulate=False), out)
