"""The library's sparse interpolation matrices for level-dependent truncation numbers (host
code, CPU) against the oracle's restatement of the reference's Lagrange interpolation
(lib_sie_mlfmm.f90:268-610)."""
import ctypes as C

import numpy as np
import pytest


def _csr(lib, p, kc, kp, transpose):
    from scipy.sparse import csr_matrix
    f = lib.sie_internal_interp_csr
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, ip, ip, dp]
    rows, nnz = C.c_int(0), C.c_int(0)
    assert f(p, kc, kp, int(transpose), C.byref(rows), C.byref(nnz), None, None, None) == 0
    ptr = np.zeros(rows.value + 1, np.int32)
    col = np.zeros(nnz.value, np.int32)
    val = np.zeros(nnz.value)
    assert f(p, kc, kp, int(transpose), None, None, ptr.ctypes.data_as(ip), col.ctypes.data_as(ip),
             val.ctypes.data_as(dp)) == 0
    qc, qp = 2 * kc * kc + 2, 2 * kp * kp + 2
    shape = (2 * qc, 2 * qp) if transpose else (2 * qp, 2 * qc)
    return csr_matrix((val, col, ptr), shape=shape)


@pytest.mark.parametrize("kc,kp", [(12, 19), (16, 19), (19, 19), (19, 12)])
def test_matrix_applies_the_oracle_interpolation(gpu_lib, oracle_lib, kc, kp):
    m = _csr(gpu_lib, 3, kc, kp, False)
    qc = 2 * kc * kc + 2
    rng = np.random.default_rng(kc * 100 + kp)
    fa = rng.standard_normal(qc) + 1j * rng.standard_normal(qc)
    fb = rng.standard_normal(qc) + 1j * rng.standard_normal(qc)
    y = m @ np.concatenate([fa, fb])
    ga, gb = oracle_lib.lagrange_interp(3, kc, kp, fa, fb)
    ref = np.concatenate([ga, gb])
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()


def test_rows_and_poles(gpu_lib):
    kc, kp = 12, 19
    m = _csr(gpu_lib, 3, kc, kp, False)
    qc, qp = 2 * kc * kc + 2, 2 * kp * kp + 2
    per_row = np.diff(m.indptr)
    assert per_row.max() <= 72  # 36 taps, a pole-row tap reads two inputs
    for r, c in ((qp - 2, qc - 2), (qp - 1, qc - 1), (2 * qp - 2, 2 * qc - 2), (2 * qp - 1, 2 * qc - 1)):
        row = m.getrow(r)
        assert row.nnz == 1 and row.indices[0] == c and row.data[0] == 1.0
    # columns sorted within each row
    for r in range(0, m.shape[0], 97):
        cols = m.indices[m.indptr[r]:m.indptr[r + 1]]
        assert np.all(np.diff(cols) > 0)


def test_anterpolation_is_the_transpose(gpu_lib):
    m = _csr(gpu_lib, 3, 12, 19, False)
    mt = _csr(gpu_lib, 3, 12, 19, True)
    assert np.array_equal(mt.toarray(), m.toarray().T)


def test_bad_arguments_are_refused(gpu_lib):
    f = gpu_lib.sie_internal_interp_csr
    f.restype = C.c_int
    rows, nnz = C.c_int(0), C.c_int(0)
    assert f(0, 12, 19, 0, C.byref(rows), C.byref(nnz), None, None, None) != 0
    assert f(3, 3, 19, 0, C.byref(rows), C.byref(nnz), None, None, None) != 0
