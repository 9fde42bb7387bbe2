"""PIRO's operator API in Python over the context layer of the C ABI.

    case = Case(assets_dir, "HeatEq.ini")
    solver = process(case)
    UEqn = scalarMatrix(solver.ddt_r("T").assign(solver.laplacian("T", "Alpha")))
    UEqn.Solve(time)

mirrors src/solve.cpp:22-37; `assign` stands for C++ operator= and `&` is
operator& (src/operatoroverload.cpp:20-123).  Every call goes through
libpiro_b200.so (piro_open, piro_laplacian, piro_assign, ...).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import Buf, CaseInfo, Op, check, lib


class Case:
    """One PIRO run (piro_ctx): a case .ini and its assets directory."""

    def __init__(self, assets_dir: str, case_name: str, alpha_mode: int = 0, lu_mode: int = 0):
        h = C.c_void_p()
        check(lib().piro_open(assets_dir.encode(), case_name.encode(), C.byref(h)), "piro_open")
        self.h = h
        if alpha_mode:
            check(lib().piro_set_alpha_mode(self.h, alpha_mode), "piro_set_alpha_mode")
        if lu_mode:
            check(lib().piro_set_lu_mode(self.h, lu_mode), "piro_set_lu_mode")

    @property
    def info(self) -> CaseInfo:
        i = CaseInfo()
        check(lib().piro_ctx_query(self.h, C.byref(i)), "piro_ctx_query")
        return i

    def handle(self, name: str) -> Buf:
        b = Buf()
        check(lib().piro_field(self.h, name.encode(), C.byref(b)), "piro_field")
        return b

    def get(self, name: str) -> np.ndarray:
        b = self.handle(name)
        out = np.empty(b.n, np.float32)
        check(lib().piro_field_download(self.h, b, out.ctypes.data_as(C.c_void_p), b.n), "piro_field_download")
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        b = self.handle(name)
        v = np.ascontiguousarray(values, np.float32)
        if v.size != b.n:
            raise ValueError(f"{name}: expected {b.n} values, got {v.size}")
        check(lib().piro_field_upload(self.h, b, v.ctypes.data_as(C.c_void_p), b.n), "piro_field_upload")

    def solve(self) -> int:
        """Piro::solve: the whole time loop of the case."""
        n = C.c_int64()
        check(lib().piro_solve(self.h, C.byref(n)), "piro_solve")
        return n.value

    def export_csr(self, op: "Operator"):
        nnz = C.c_int64()
        check(lib().piro_op_export_csr(self.h, op.op, None, None, None, 0, C.byref(nnz)), "piro_op_export_csr")
        N = self.info.n_cells
        rp = np.empty(N + 1, np.int32)
        col = np.empty(nnz.value, np.int32)
        val = np.empty(nnz.value, np.float32)
        check(lib().piro_op_export_csr(self.h, op.op, rp.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                       val.ctypes.data_as(C.c_void_p), nnz.value, C.byref(nnz)),
              "piro_op_export_csr")
        return rp, col, val

    def write_paraview(self, root: str, timestep: int) -> None:
        """Piro::paraview::writevth: <root>/<casename>/mesh/mesh_<ts>.vth and level/<ts>_level_0.vti."""
        check(lib().piro_write_paraview(self.h, root.encode(), int(timestep)), "piro_write_paraview")

    def set_output(self, root) -> None:
        """Write ParaView files every Save steps under root (None: no output)."""
        check(lib().piro_set_output(self.h, None if root is None else root.encode()), "piro_set_output")

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().piro_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Operator:
    def __init__(self, case: Case, op: Op):
        self.case, self.op = case, op


class Field:
    """A field handle (CLBuffer)."""

    def __init__(self, case: Case, buf: Buf):
        self.case, self.buf = case, buf

    def assign(self, rhs: Operator) -> "Field":
        """operator=: one time step of this field; returns the result (partD)."""
        out = Buf()
        check(lib().piro_assign(self.case.h, self.buf, rhs.op, C.byref(out)), "piro_assign")
        return Field(self.case, out)

    def __and__(self, grad: Operator) -> Operator:
        """operator&: the v.grad merge (csrgeam)."""
        out = Op()
        check(lib().piro_dot(self.case.h, self.buf, grad.op, C.byref(out)), "piro_dot")
        return Operator(self.case, out)


class process:
    """Piro::process (src/process.cpp)."""

    def __init__(self, case: Case):
        self.case = case

    def ddt_r(self, var: str) -> Field:
        b = Buf()
        check(lib().piro_ddt_r(self.case.h, var.encode(), C.byref(b)), "piro_ddt_r")
        return Field(self.case, b)

    def vector(self, var: str) -> Field:
        b = Buf()
        check(lib().piro_vector(self.case.h, var.encode(), C.byref(b)), "piro_vector")
        return Field(self.case, b)

    def laplacian(self, var: str, coeff: str) -> Operator:
        o = Op()
        check(lib().piro_laplacian(self.case.h, var.encode(), coeff.encode(), C.byref(o)), "piro_laplacian")
        return Operator(self.case, o)

    def gradient(self, var: str) -> Operator:
        o = Op()
        check(lib().piro_gradient(self.case.h, var.encode(), C.byref(o)), "piro_gradient")
        return Operator(self.case, o)

    def div(self, var1: str, var2: str) -> Operator:
        o = Op()
        check(lib().piro_div(self.case.h, var1.encode(), var2.encode(), C.byref(o)), "piro_div")
        return Operator(self.case, o)


class scalarMatrix:
    """Piro::scalarMatrix: Solve copies the result into field 1 and applies setBC."""

    def __init__(self, eqn: Field):
        self.eqn = eqn

    def Solve(self, time: float) -> None:
        check(lib().piro_step_solve(self.eqn.case.h, self.eqn.buf, float(time)), "piro_step_solve")
