"""ctypes loader for the oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the library in tsm_benchmark_b200/ never does.

  * ``lib()``  -> oracle/libtsm_oracle.so, the C restatement (tsm_oracle.c)
  * ``ref()``  -> oracle/_ref/libtsm_ref.so, the reference's own C++ compiled
                  in place against oracle/sycl_host (None where it was not
                  built, e.g. on a machine without the reference sources)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libtsm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtsm_ref.so")

P = ctypes.c_void_p
I64 = ctypes.c_int64
I = ctypes.c_int
D = ctypes.c_double

_lib = None
_ref = None


# The reference checkout whose sources oracle/Makefile compiles in place:
# TSM_REFERENCE_DIR from the environment, else the read-only checkout the
# project is built beside, when it is there (it is not on GPU hosts, which
# use the libraries built where it is).
REFERENCE_CHECKOUT = "/root/reference"


def reference_dir() -> str | None:
    d = os.environ.get("TSM_REFERENCE_DIR") or REFERENCE_CHECKOUT
    return d if os.path.exists(os.path.join(d, "main.cc")) else None


def make_args() -> list[str]:
    """REF_DIR=<checkout> for the Makefiles, or nothing without a checkout."""
    d = reference_dir()
    return [f"REF_DIR={d}"] if d else []


def build() -> None:
    """Runs oracle/Makefile (the reference part only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, *make_args()], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.tsm_oracle_naive_f64.argtypes = [I64, I, I, P, I64, P, I64, P, I64]
        L.tsm_oracle_naive_f32in.argtypes = [I64, I, I, P, I64, P, I64, P, I64]
        L.tsm_oracle_dot2_f64.argtypes = [I64, I, I, P, I64, P, I64, P, P, I64]
        L.tsm_oracle_check_f64.argtypes = [P, P, I, I, I64, D, D]
        L.tsm_oracle_check_f64.restype = I64
        L.tsm_oracle_normwise_f64.argtypes = [I64, I, I, P, I64, P, I64, P, P, I64, P]
        L.tsm_oracle_fill_uniform_f64.argtypes = [P, I64, ctypes.c_uint64, ctypes.c_uint64]
        L.tsm_oracle_fill_minstd_f64.argtypes = [P, P, I64, ctypes.c_uint32, D, D]
        L.tsm_oracle_v4_omp.argtypes = [I64, I, I, I, P, P, P]
        L.tsm_oracle_v4_omp.restype = I
        L.tsm_oracle_num_threads.restype = I
        L.tsm_oracle_tsmm_f64.argtypes = [I64, I, I, P, I64, P, I64, I64, P, I64, I]
        L.tsm_oracle_dot2_acc.argtypes = [I64, I, I, P, I64, P, I64, I, P, P, P, P]
        L.tsm_oracle_dot2_acc.restype = I
        L.tsm_oracle_dot2_uniform.argtypes = [I64, I64, I, I, ctypes.c_uint64, P, P, P, P]
        L.tsm_oracle_dot2_uniform.restype = I
        L.tsm_oracle_force_split.argtypes = [I]
        L.tsm_oracle_dot2_uniform_ex.argtypes = [I64, I64, I64, I, I, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.c_uint64, I, P, P, P, P]
        L.tsm_oracle_dot2_uniform_ex.restype = I
        _lib = L
    return _lib


def ref():
    """The reference's own code (or None when oracle/_ref was not built)."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        R = ctypes.CDLL(REF_SO)
        R.ref_compute_naive_f64.argtypes = [I, I, P, P, P]
        R.ref_is_correct_f64.argtypes = [P, P, I, D, D]
        R.ref_tsmttsm_f64.argtypes = [I, I, I, I, I, P, P, P, ctypes.POINTER(ctypes.c_uint64)]
        R.ref_generated_f64.argtypes = [ctypes.c_char_p, I, P, P, P, ctypes.POINTER(ctypes.c_uint64)]
        R.ref_fill_main_cc_f64.argtypes = [P, P, ctypes.c_long, ctypes.c_uint]
        R.ref_num_threads.restype = I
        _ref = R
    return _ref


def _p(a: np.ndarray):
    return a.ctypes.data_as(P)


def _rows(x: np.ndarray) -> tuple[int, int, int]:
    assert x.ndim == 2
    if x.shape[0] <= 1 or x.shape[1] <= 1:
        # strides of empty, single-row or single-column arrays carry no layout
        assert x.flags.c_contiguous or x.shape[1] <= 1 or x.shape[0] <= 1
        if x.shape[1] <= 1 and x.shape[0] > 1:
            return x.shape[0], x.shape[1], x.strides[0] // x.itemsize
        return x.shape[0], x.shape[1], max(1, x.shape[1])
    assert x.strides[1] == x.itemsize
    return x.shape[0], x.shape[1], x.strides[0] // x.itemsize


def naive(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """C = A^T B in compute_naive's order (main.cc:14-27), FP64."""
    n, m, lda = _rows(A)
    _, k, ldb = _rows(B)
    C = np.zeros((m, k), dtype=np.float64)
    if A.dtype == np.float32:
        lib().tsm_oracle_naive_f32in(n, m, k, _p(A), lda, _p(B), ldb, _p(C), k)
    else:
        lib().tsm_oracle_naive_f64(n, m, k, _p(A), lda, _p(B), ldb, _p(C), k)
    return C


def dot2(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """Compensated (double-double) A^T B, rounded to FP64."""
    n, m, lda = _rows(A)
    _, k, ldb = _rows(B)
    C = np.zeros((m, k), dtype=np.float64)
    lib().tsm_oracle_dot2_f64(n, m, k, _p(A), lda, _p(B), ldb, _p(C), None, k)
    return C


def check(ref_c: np.ndarray, got: np.ndarray, rel_tol: float = 1e-6, abs_tol: float = 1e-10) -> int:
    """is_correct's element rule (main.cc:29-41): index of the first failing
    entry, or -1."""
    ref_c = np.ascontiguousarray(ref_c, dtype=np.float64)
    got = np.ascontiguousarray(got, dtype=np.float64)
    m, k = ref_c.shape
    return int(lib().tsm_oracle_check_f64(_p(ref_c), _p(got), m, k, k, rel_tol, abs_tol))


def normwise(A: np.ndarray, B: np.ndarray, ref_c: np.ndarray, got: np.ndarray) -> dict:
    """||got - ref||_F and the bound 4 sqrt(n) 2^-53 ||A||_F ||B||_F."""
    n, m, lda = _rows(A)
    _, k, ldb = _rows(B)
    ref_c = np.ascontiguousarray(ref_c, dtype=np.float64)
    got = np.ascontiguousarray(got, dtype=np.float64)
    out = np.zeros(4)
    lib().tsm_oracle_normwise_f64(n, m, k, _p(A), lda, _p(B), ldb, _p(ref_c), _p(got), k, _p(out))
    return dict(err=out[0], normA=out[1], normB=out[2], bound=out[3])


def uniform(count: int, seed: int, stream: int = 0) -> np.ndarray:
    """The counter-based uniform[-1, 1) values (same bits as the device fill)."""
    x = np.empty(count, dtype=np.float64)
    lib().tsm_oracle_fill_uniform_f64(_p(x), count, seed, stream)
    return x


def operands(n: int, m: int, k: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """A (n x m) from stream 0 and B (n x k) from stream 1 under `seed`."""
    return uniform(n * m, seed, 0).reshape(n, m), uniform(n * k, seed, 1).reshape(n, k)


def main_cc_inputs(n: int, width: int, seed: int = 123) -> tuple[np.ndarray, np.ndarray]:
    """main.cc's inputs (single-engine path, main.cc:71-86), restated."""
    A = np.empty(n * width)
    B = np.empty(n * width)
    lib().tsm_oracle_fill_minstd_f64(_p(A), _p(B), n * width, seed, -1.0, 1.0)
    return A.reshape(n, width), B.reshape(n, width)


def v4_port(A: np.ndarray, B: np.ndarray, stride: int = 16384, tile: int = 4) -> np.ndarray:
    """The OpenMP restatement of tsmttsm4 (square widths)."""
    n, m = A.shape
    C = np.zeros((m, m))
    rc = lib().tsm_oracle_v4_omp(n, m, stride, tile, _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)), _p(C))
    if rc != 0:
        raise ValueError("launch shape not supported by tsmttsm4")
    return C


def tsmm(X: np.ndarray, W: np.ndarray, transpose_w: bool = False) -> np.ndarray:
    """Y = X W (or X W^T), the backward TSMM oracle."""
    n, p, ldx = _rows(X)
    Wc = np.ascontiguousarray(W, dtype=np.float64)
    if transpose_w:
        q = Wc.shape[0]
        w_row, w_col = 1, Wc.shape[1]
    else:
        q = Wc.shape[1]
        w_row, w_col = Wc.shape[1], 1
    Y = np.zeros((n, q))
    lib().tsm_oracle_tsmm_f64(n, p, q, _p(X), ldx, _p(Wc), w_row, w_col, _p(Y), q, 0)
    return Y


class Dot2Stream:
    """Compensated A^T B accumulated over row chunks (tsm_oracle_dot2_acc /
    tsm_oracle_dot2_uniform): the full-size checks feed it host chunks or let
    it generate the counter-based uniform operands itself, so no operand is
    ever held whole.  ``result()`` gives C rounded to FP64, the Frobenius
    norms of A and B, the normwise bound 4 sqrt(n) 2^-53 ||A||_F ||B||_F and,
    with ``with_abs``, sum_r |a_ri| |b_rj| per entry."""

    def __init__(self, m: int, k: int, with_abs: bool = False):
        self.m, self.k, self.rows = m, k, 0
        self.S = np.zeros(m * k)
        self.E = np.zeros(m * k)
        self.nrm = np.zeros(2)
        self.absC = np.zeros(m * k) if with_abs else None

    def _abs(self):
        return _p(self.absC) if self.absC is not None else None

    def add(self, A: np.ndarray, B: np.ndarray) -> None:
        n, m, lda = _rows(A)
        n2, k, ldb = _rows(B)
        assert (n, m, k) == (n2, self.m, self.k) and A.dtype == B.dtype
        f32 = 1 if A.dtype == np.float32 else 0
        assert f32 or A.dtype == np.float64
        rc = lib().tsm_oracle_dot2_acc(n, m, k, _p(A), lda, _p(B), ldb, f32, _p(self.S), _p(self.E), _p(self.nrm),
                                       self._abs())
        if rc != 0:
            raise MemoryError("oracle: host buffers")
        self.rows += n

    def add_uniform(self, seed: int, row0: int, rows: int, *, streams: tuple[int, int] = (0, 1),
                    col_major_n: int = 0) -> None:
        """Rows [row0, row0 + rows) of counter-based uniform operands: A from
        streams[0], B from streams[1] (equal streams and m == k: B is A).
        Row-major by default (operands(n, m, k, seed)'s values); with
        col_major_n = n, the values fill_uniform writes into A^T and B^T
        stored row-major (m x n and k x n)."""
        if streams[0] == streams[1] and self.m != self.k:
            raise ValueError("B is A only for m == k")
        rc = lib().tsm_oracle_dot2_uniform_ex(row0, rows, col_major_n or (row0 + rows), self.m, self.k, seed,
                                              streams[0], streams[1], 1 if col_major_n else 0, _p(self.S),
                                              _p(self.E), _p(self.nrm), self._abs())
        if rc != 0:
            raise MemoryError("oracle: host buffers")
        self.rows += rows

    def result(self) -> dict:
        C = (self.S + self.E).reshape(self.m, self.k)
        na, nb = float(np.sqrt(self.nrm[0])), float(np.sqrt(self.nrm[1]))
        out = dict(C=C, normA=na, normB=nb, rows=self.rows,
                   bound=4.0 * np.sqrt(float(self.rows)) * 2.0**-53 * na * nb)
        if self.absC is not None:
            out["absC"] = self.absC.reshape(self.m, self.k).copy()
        return out


def dot2_uniform(n: int, m: int, k: int, seed: int, with_abs: bool = False, *, gram: bool = False,
                 col_major: bool = False) -> dict:
    """Dot2Stream over all n rows of operands(n, m, k, seed), generated on
    the host as it goes; gram: B is A (stream 0); col_major: the values of
    A^T, B^T filled row-major."""
    d = Dot2Stream(m, k, with_abs)
    d.add_uniform(seed, 0, n, streams=(0, 0) if gram else (0, 1), col_major_n=n if col_major else 0)
    return d.result()
