"""C ABI checks that need no GPU: the library loads, exports every symbol
include/*.h declares, and its host-only entry points behave."""
import ctypes as C
import subprocess

import pytest

from piro_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) > 30
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported


def test_signatures_cover_header():
    # every declared function has a ctypes signature (and no stale extras)
    assert set(_lib.SIGNATURES) == set(_lib.declared_symbols())


def test_status_strings_and_version():
    L = _lib.lib()
    assert L.piro_status_string(0) == b"PIRO_OK"
    assert L.piro_status_string(4) == b"PIRO_ERR_TABLE_FULL"
    assert L.piro_status_string(999) == b"PIRO_ERR_UNKNOWN"
    assert b"sm_100a" in L.piro_version()


def test_nnz_closed_forms(oracle):
    L = _lib.lib()
    v = C.c_int64()
    for (nx, ny, nz) in [(3, 3, 3), (6, 5, 4), (32, 32, 32), (256, 256, 256), (130, 7, 9)]:
        assert L.piro_laplacian_nnz(nx, ny, nz, C.byref(v)) == 0
        N = nx * ny * nz
        assert v.value == 7 * N - 2 * (nx * ny + ny * nz + nx * nz)
        if N < 50000:
            assert v.value == len(oracle.laplacian(nx, ny, nz, 3, 1.0)[2])
            for a in range(3):
                assert L.piro_gradient_nnz(nx, ny, nz, a, C.byref(v)) == 0
                assert v.value == len(oracle.gradient3(nx, ny, nz, 1, 2.0)[a][2])
    assert L.piro_laplacian_nnz(2, 5, 5, C.byref(v)) == 1  # PIRO_ERR_ARG: grids include ghosts (>= 3)
    assert b"ghost" in L.piro_last_error()


def test_face_count(oracle):
    L = _lib.lib()
    q = C.c_int64()
    fs = (C.c_int64 * 7)()
    for n in [(3, 3, 3), (6, 5, 4), (12, 6, 9)]:
        assert L.piro_face_count(*n, C.byref(q), fs) == 0
        idx, ofs = oracle.face_lists(*n)
        assert q.value == len(idx) and list(fs) == list(ofs)


def test_ht_table_size_policies(oracle):
    L = _lib.lib()
    ts = C.c_int64()
    for N, nnz in [(125, 725), (120, 692), (343, 2107), (1000, 6400), (12 * 6 * 9, 4068)]:
        assert L.piro_ht_table_size(nnz, N, 0, 3.3608, -0.5552, -0.0143, 0.7, C.byref(ts)) == 0
        assert ts.value == oracle.ht_table_size_reference(nnz, N)
    # negative above N ~ 18.6k: a clear error instead of the reference's crash
    assert L.piro_ht_table_size(7 * 19683, 19683, 0, 3.3608, -0.5552, -0.0143, 0.7, C.byref(ts)) == 5
    assert L.piro_ht_table_size(117047296, 256 ** 3, 1, 0, 0, 0, 0.7, C.byref(ts)) == 0
    assert ts.value == oracle.ht_table_size_build(117047296)


def test_null_arguments_are_rejected_without_a_gpu():
    L = _lib.lib()
    assert L.piro_csr_laplacian(8, 8, 8, 3, 1.0, None, None, None, None) == 1
    assert L.piro_csr_fe_step(8, 8, 8, None, None, None, 0.1, None, None, None) == 1
    assert L.piro_csr_laplacian(8, 8, 8, 7, 1.0, 1, 1, 1, None) in (1, 9)
