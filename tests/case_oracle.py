"""Test infrastructure: a PIRO case run composed from the CPU oracle.

Restates Piro::preprocess (src/preprocess.cpp:20-208), bc::initbc/setbc
(src/bc.cpp:107-157) and Piro::solve (src/solve.cpp:11-48) in Python on top of
the oracle's pinned building blocks (assembly, initial conditions, step
kernels), to check the context layer of the C ABI end to end.
"""
from __future__ import annotations

import os

import numpy as np

from oracle import oracle as O


def read_ini(path):
    """IniReader (src/fileutilities.cpp:124-183)."""
    out, sec = {}, ""
    with open(path) as f:
        for line in f:
            line = line.rstrip("\r\n").strip(" ")
            if not line or line[0] in ";#":
                continue
            if line[0] == "[" and line[-1] == "]":
                sec = line[1:-1]
            elif "=" in line:
                k, v = line.split("=", 1)
                out.setdefault(sec, {})[k.strip(" ")] = v.strip(" ")
    return out


def floats(s):
    out = []
    for t in s.split(" "):
        try:
            out.append(float(np.float32(t)))
        except ValueError:
            pass
    return out


def run_case(assets, case_name, alpha_mode=0, lu_mode=0):
    cfg = read_ini(os.path.join(assets, case_name))
    dist = read_ini(os.path.join(assets, "IC", "distribution.ini"))
    n = [int(v) for v in cfg["Mesh"]["n"].split(" ")]
    l = [np.float32(v) for v in floats(cfg["Mesh"]["l"])]
    nx, ny, nz = n[0] + 2, n[1] + 2, n[2] + 2
    N = nx * ny * nz
    ts, ss, solver = int(cfg["Schemes"]["Time"]), int(cfg["Schemes"]["Space"]), int(cfg["Schemes"]["Solver"])
    sim = int(cfg["File"]["simindex"])
    data = int(cfg["Solve"]["Data"])
    dt, total = np.float32(cfg["Solve"]["Timestep"]), np.float32(cfg["Solve"]["TotalTime"])

    def ic(kind):
        if kind == "Gaussian":
            g = dist["Gaussian"]
            return O.ic_gaussian(nx, ny, nz, l, np.float32(g["Scalefactor"]), floats(g["Sigma"]), floats(g["Median"]))
        if kind == "Coulomb":
            c = dist["Coulomb"]
            return O.ic_coulomb(nx, ny, nz, l, floats(c["center"]), np.float32(c["Z"]), np.float32(c["e"]),
                                np.float32(c["epsilon_0"]))
        v = dist["Vector"]
        return O.ic_uniform_vector(N, floats(v["Direction"]), floats(v["Value"])[0])

    sim_cfg = cfg["Simulation"]
    cnames, snames = sim_cfg["Constants"].split(" "), sim_cfg["Scalars"].split(" ")
    vnames = sim_cfg.get("Vectors", "").split()
    icf = cfg["IC"]["filename"].split(" ")
    cvals = floats(sim_cfg["Values"])
    names, host = [], []
    for i, nm in enumerate(cnames):
        names.append(nm)
        host.append(np.full(N, cvals[i], np.float32))
    for i, nm in enumerate(snames):
        names.append(nm)
        host.append(ic(icf[i]))
    for nm in vnames:
        names.append(nm)
        v = ic(icf[len(snames)])
        host.append(np.concatenate([v, np.zeros(max(0, 3 * N - len(v)), np.float32)])[:3 * N])
    # device values start from the initial conditions (before setbc)
    dev = [h[:N].copy() if i < len(cnames) + len(snames) else h.copy() for i, h in enumerate(host)]

    def match(var):
        return names.index(var) if var in names else 0

    bc_idx, memD = None, None
    setup = read_ini(os.path.join(assets, "setup.ini"))
    if "BC" in setup and setup["BC"]["type"].count(" ") > 1:
        props = setup["BC"]["property"].split(" ")
        vals = floats(setup["BC"]["values"])
        bc_idx, fs = O.face_lists(nx, ny, nz)
        for face in range(6):
            host[match(props[face])][bc_idx[fs[face]:fs[face + 1]]] = np.float32(vals[face])
        memD = host[1][:N].copy()

    def set_bc(u):
        if bc_idx is not None:
            u[bc_idx] = memD[bc_idx]

    norm = O.laplacian_norm(l[0], nx)
    op = None
    if sim == 0 and data == 1:
        op = ("dense", O.dense_laplacian(nx, ny, nz, ss, norm))
    elif sim == 0:
        if data == 3:
            rows, col, val = O.laplacian(nx, ny, nz, ss, norm, "coo")
            op = ("coo", (rows, col, val))
        else:
            rp, col, val = O.laplacian(nx, ny, nz, ss, norm, "csr")
            if data == 0 and alpha_mode == 0:
                val = O.csr_rowscale(N, rp, val, dev[match("Alpha")])
            op = ("csr", (rp, col, val))
            csr = (rp, col, val)
            if data == 2:
                tsz = O.ht_table_size_reference(len(val), N)
                keys, vals = O.ht_build(N, rp, col, val, tsz)
                op = ("ht", (keys, vals))
    elif sim == 1:
        G = O.gradient3(nx, ny, nz, ss, O.gradient_norm(l[0], nx))
        op = ("csr", O.csrgeam3(N, *G, dev[match("v")]))
    else:  # continuity: div(rho, u), the divergence matrices row-scaled by u (or not: alpha_mode 1)
        G = O.div3(nx, ny, nz, ss, O.gradient_norm(l[0], nx))
        vel = dev[match("u")] if alpha_mode == 0 else np.ones(3 * N, np.float32)
        op = ("csr", O.csrgeam3(N, *G, vel))
    lhs = match({0: "T", 1: "U", 2: "rho"}[sim])
    steps = O.step_count(total, dt)
    for _ in range(steps):
        u = dev[lhs]
        if ts == 11:
            if op[0] == "csr":
                part = O.spmv_csr_fe(nx, ny, nz, op[1], dt, u, np.zeros(N, np.float32))
            elif op[0] == "dense":
                part = O.fe_dense(op[1], dt, u)[1]
            elif op[0] == "coo":
                part = u + O.spmv_coo(N, op[1], dt, u)
            else:
                part = u + O.spmv_ht(N, op[1][0], op[1][1], dt, u)
        elif solver == 27:
            # lu_mode 1: the reference factorizes and returns a zero field
            # (operatoroverload.cpp:65-81); 0: FP64 solve of (I - dt*M) x = u
            part = np.zeros(N, np.float32)
            if lu_mode == 0:
                import scipy.sparse as sp
                import scipy.sparse.linalg as spl
                I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
                arp, acol, aval = O.csrgeam2(N, I, np.float32(-dt), csr)
                A = sp.csr_matrix((aval.astype(np.float64), acol, arp), shape=(N, N))
                part = spl.spsolve(A.tocsc(), u.astype(np.float64)).astype(np.float32)
        elif solver == 40:
            part, _ = O.be_jli(nx, ny, nz, op[1], dt, u)
        else:  # 39: FP64 solve of (I - dt*M) x = u on the interior
            M = op[1]
            I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
            A = O.csrgeam2(N, I, np.float32(-dt), M)
            alpha = dev[match("Alpha")] if alpha_mode == 0 else np.ones(N, np.float32)
            x64, _, _ = O.be_cg_f64(nx, ny, nz, A, alpha, u, rtol=1e-13)
            part = x64.astype(np.float32)
        part = part.astype(np.float32)
        dev[1] = part.copy()
        set_bc(dev[1])
    return dict(names=names, fields=dev, steps=steps, n=(nx, ny, nz))
