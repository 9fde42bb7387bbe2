"""Forward-Euler time loops (TIMESCHEME 11) on the device, one Solve() per
step as src/solve.cpp:18-46 runs them: a zero-filled result buffer, the
SpMV + update over the interior (SpMVCSR.cl), then setBC restoring the face
values saved at start-up -- all three in one kernel (piro_csr_fe_step_bc).  The per-step launches can be captured once in
a CUDA graph and replayed (graph=True), which removes the host from the loop
for small grids where a step is a few microseconds."""
from __future__ import annotations

import torch

from . import ops


class _Loop:
    def _setup_bc(self, u0: torch.Tensor) -> None:
        self.bc_idx, _ = ops.face_lists(self.nx, self.ny, self.nz)
        self.memD = u0.clone()  # face values at start-up (bc.cpp:31-32)

    def _step(self, u: torch.Tensor, out: torch.Tensor) -> None:
        # zero-filled result, SpMVCSR update, setBC of the faces: one kernel
        ops.csr_fe_step_bc(self.nx, self.ny, self.nz, self.A, self.dt, u, self.memD, out)

    def capture(self, u0: torch.Tensor):
        """Set up the boundary values and capture two steps in a CUDA graph
        once; returns replay(pairs) -> the field after 2*pairs steps from u0
        (each call restarts from u0)."""
        self._setup_bc(u0)
        bufs = [u0.clone(), torch.empty_like(u0)]
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            self._step(bufs[0], bufs[1])
            with torch.cuda.graph(g, stream=stream):
                self._step(bufs[0], bufs[1])
                self._step(bufs[1], bufs[0])
        torch.cuda.current_stream().wait_stream(stream)
        self._graph = g

        def replay(pairs: int) -> torch.Tensor:
            bufs[0].copy_(u0)
            for _ in range(pairs):
                g.replay()
            return bufs[0]

        return replay

    def run(self, u0: torch.Tensor, steps: int, graph: bool = False) -> torch.Tensor:
        self._setup_bc(u0)
        bufs = [u0.clone(), torch.empty_like(u0)]
        if not graph:
            for s in range(steps):
                self._step(bufs[s & 1], bufs[(s + 1) & 1])
            return bufs[steps & 1]
        # two steps per graph (buffers ping-pong), replayed steps//2 times
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            self._step(bufs[0], bufs[1])  # warm (non-captured) launch of every kernel
            bufs[0].copy_(u0)
            with torch.cuda.graph(g, stream=stream):
                self._step(bufs[0], bufs[1])
                self._step(bufs[1], bufs[0])
        torch.cuda.current_stream().wait_stream(stream)
        for _ in range(steps // 2):
            g.replay()
        if steps & 1:
            self._step(bufs[0], bufs[1])
            torch.cuda.synchronize()
            return bufs[1]
        torch.cuda.synchronize()
        return bufs[0]


class FeRunner(_Loop):
    """Heat equation: ddt_r(T) = laplacian(T, Alpha), central scheme, CSR,
    alpha applied as SpMDSM intends."""

    def __init__(self, nx, ny, nz, alpha: torch.Tensor, dt: float, norm: float = 1.0, scheme: int = 3):
        self.nx, self.ny, self.nz, self.dt = nx, ny, nz, dt
        rp, col, val = ops.csr_laplacian(nx, ny, nz, scheme, norm)
        self.A_unscaled_tens = val.clone()
        ops.csr_rowscale(rp, val, alpha)
        self.A = (rp, col, val)


class AdvectionRunner(_Loop):
    """Advection: ddt_r(U) = vector(v) & gradient(U), upwind, CSR."""

    def __init__(self, nx, ny, nz, v: torch.Tensor, dt: float, gnorm: float = 2.0, scheme: int = 1):
        self.nx, self.ny, self.nz, self.dt = nx, ny, nz, dt
        N = nx * ny * nz
        G = [ops.csr_gradient(nx, ny, nz, scheme, a, gnorm) for a in range(3)]
        self.A = ops.csrgeam3(N, *G, v)
