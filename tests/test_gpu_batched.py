"""Batched stepping (piro_batch_*): members of uneven sizes, forward and
backward Euler, one persistent launch per step, against the oracle."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _a64(n, alpha, dt):
    """FP64 A = I - dt*alpha*L (7-point, h = 1) on the interior unknowns and the
    interior-interior / interior-boundary split."""
    N = n ** 3
    idx = np.arange(N).reshape(n, n, n)
    inter = np.zeros((n, n, n), bool)
    inter[1:-1, 1:-1, 1:-1] = True
    rows, cols, vals = [], [], []
    ii = idx[inter]
    c = float(dt) * float(alpha)
    rows.append(ii); cols.append(ii); vals.append(np.full(ii.size, 1.0 + 6.0 * c))
    for ax in range(3):
        for s in (-1, 1):
            nb = np.roll(idx, -s, axis=ax)[inter]
            rows.append(ii); cols.append(nb); vals.append(np.full(ii.size, -c))
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    return A, inter.reshape(-1)


def _small_batch(seed=7, count=10):
    from piro_b200 import workloads as W
    return W.batched(seed=seed, count=count, lo=8, hi=22)


@pytest.mark.parametrize("schedule", ["lockstep", "grouped"])
def test_batch_matches_oracle(cuda, schedule):
    """Both schedules: the lockstep rounds of k_batch_step and the grouped
    k_batch_groups (each member on a CTA group of its own with group-local
    barriers, small members packed onto single CTAs)."""
    from piro_b200 import ops
    from piro_b200 import workloads as W
    cfg = _small_batch()
    assert set(cfg["scheme"]) == {0, 1}
    B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
    B.set_schedule(schedule == "grouped", 2)
    assert B.schedule() == schedule
    B.set_fields(W.pack_batch(cfg["fields"], B.offsets, B.total))
    B.step(2, rtol=1e-8)
    out = B.get_fields()
    info = B.member_info()
    for k in range(B.count):
        n, a, dt = int(cfg["n"][k]), cfg["alpha"][k], cfg["dt"][k]
        u = cfg["fields"][k]
        got = B.member(out, k)
        if cfg["scheme"][k] == 0:
            ref = u
            for _ in range(2):
                ref = O.stencil_fe(n, n, n, dt, ref, alpha=np.full(n ** 3, a, np.float32))
            assert np.array_equal(got, ref), k  # same arithmetic, bit for bit
        else:
            assert info["status"][k] == 0 and info["rel"][k] <= 1e-8, (k, info)
            A, inter = _a64(n, a, dt)
            x = u.astype(np.float64)
            for _ in range(2):
                b = x.copy()
                xi = spla.spsolve(A[inter][:, inter].tocsc(), b[inter] - A[inter][:, ~inter] @ b[~inter])
                x = b.copy()
                x[inter] = xi
            err = np.abs(got.astype(np.float64) - x).max() / np.abs(x).max()
            assert err < 1e-6, (k, err)


@pytest.mark.parametrize("schedule", ["lockstep", "grouped"])
def test_batch_is_deterministic(cuda, schedule):
    from piro_b200 import ops
    from piro_b200 import workloads as W
    cfg = _small_batch(seed=8, count=14)
    res = []
    for _ in range(2):
        B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
        B.set_schedule(schedule == "grouped", 4)
        B.set_fields(W.pack_batch(cfg["fields"], B.offsets, B.total))
        B.step(3)
        res.append(B.get_fields())
        B.close()
    assert np.array_equal(res[0], res[1])


def test_batch_autotune(cuda):
    from piro_b200 import ops
    from piro_b200 import workloads as W
    cfg = _small_batch(seed=9, count=16)
    B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
    u0 = W.pack_batch(cfg["fields"], B.offsets, B.total)
    B.set_fields(u0)
    B.step(1)
    ref = B.get_fields()
    B.set_fields(u0)
    tile, bps = B.autotune()
    assert tile in (2048, 4096, 8192, 16384) and bps in (1, 2, 4)
    assert B.schedule() in ("lockstep", "grouped")
    B.set_fields(u0)
    B.step(1)
    got = B.get_fields()
    info = B.member_info()
    assert np.all(info["status"] == 0)
    be = cfg["scheme"] == 1
    for k in range(B.count):
        a, b = B.member(got, k), B.member(ref, k)
        if be[k]:
            assert np.abs(a - b).max() <= 1e-6 * max(1e-30, np.abs(b).max())
        else:
            assert np.array_equal(a, b)


def test_grouped_schedule_large_members_vs_lockstep(cuda):
    """Members large enough to get CTA groups of their own (sides up to 60):
    the grouped step agrees with the lockstep one to rounding, forward-Euler
    members bit for bit, for two steps in a row."""
    from piro_b200 import ops
    from piro_b200 import workloads as W
    cfg = W.batched(seed=11, count=24, lo=12, hi=60)
    u0 = None
    out = {}
    for grouped in (False, True):
        B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
        u0 = W.pack_batch(cfg["fields"], B.offsets, B.total)
        B.set_schedule(grouped, 2)
        B.set_fields(u0)
        B.step(2)
        out[grouped] = (B.get_fields(), B.member_info())
        offs = B.offsets
        B.close()
    be = cfg["scheme"] == 1
    (a, ia), (b, ib) = out[False], out[True]
    assert np.all(ib["status"] == 0) and np.all(ib["rel"][be] <= 1e-8)
    for k in range(len(cfg["n"])):
        n3 = int(cfg["n"][k]) ** 3
        x, y = a[offs[k]:offs[k] + n3], b[offs[k]:offs[k] + n3]
        if be[k]:
            assert np.abs(x - y).max() <= 1e-6 * max(1e-30, np.abs(x).max()), k
        else:
            assert np.array_equal(x, y), k
