"""CPU oracle for the CONQUEST block-sparse multiply -- TEST INFRASTRUCTURE ONLY.

This module wraps ``cq_oracle.cpp`` (a sequential restatement of the reference's
index layer and ``mat_mult``/``m_kern_max``/``m_kern_min``) with ctypes.  It is
imported only by ``tests/``, ``bench.py``'s CPU-baseline leg and
``__graft_entry__.smoke()`` as the checker; the product never imports it.

Parity status: the reference (Fortran + MPI) cannot be built in this image and
its own test-suite holds no vectors at this boundary, so the restatement is
pinned by known-answer tests (dense image-expanded products, brute-force
neighbour enumeration, dense eigh of the LNV problem) -- "parity unpinned" with
respect to reference outputs.

Reference files restated: see the header of ``cq_oracle.cpp``.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcq_oracle.so")
_lib = None
_blas = None


def build():
    """Compile the oracle library (g++ -fopenmp -ffp-contract=off)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def _load():
    global _lib, _blas
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    c_int, c_double, c_void_p, c_long = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_long
    P = ctypes.POINTER
    lib.orc_create.restype = c_void_p
    lib.orc_create.argtypes = [c_int, P(c_double), P(c_double), P(c_int), c_int, P(c_double), c_int, c_double, c_double]
    lib.orc_destroy.argtypes = [c_void_p]
    lib.orc_range_length.restype = c_int
    lib.orc_range_length.argtypes = [c_void_p, c_int]
    lib.orc_get_int.restype = c_long
    lib.orc_get_int.argtypes = [c_void_p, c_int, ctypes.c_char_p, P(ctypes.c_int64), c_long]
    lib.orc_get_double.restype = c_long
    lib.orc_get_double.argtypes = [c_void_p, c_int, ctypes.c_char_p, P(c_double), c_long]
    lib.orc_mat_mult.restype = c_int
    lib.orc_mat_mult.argtypes = [c_void_p, c_int, c_int, c_int, c_int, P(c_double), c_int, P(c_double), c_int,
                                 P(c_double), c_int, c_int, c_int]
    lib.orc_product_work.restype = c_int
    lib.orc_product_work.argtypes = [c_void_p, c_int, c_int, c_int, c_int, P(ctypes.c_int64), P(ctypes.c_int64)]
    lib.orc_matrix_add.argtypes = [c_void_p, c_double, P(c_double), c_int, c_double, P(c_double), c_int]
    lib.orc_matrix_transpose.argtypes = [c_void_p, c_int, P(c_double), P(c_double)]
    lib.orc_matrix_trace.restype = c_double
    lib.orc_matrix_trace.argtypes = [c_void_p, c_int, P(c_double)]
    lib.orc_vdot.restype = c_double
    lib.orc_vdot.argtypes = [c_long, P(c_double), P(c_double)]
    lib.orc_set_dgemm.argtypes = [c_void_p]
    lib.orc_exact_sum.restype = c_double
    lib.orc_exact_sum.argtypes = [c_long, P(c_double), P(c_double)]
    # scipy's bundled OpenBLAS provides the dgemm used by the ompGemm kernel (BLAS threads = 1)
    try:
        import scipy
        cands = glob.glob(os.path.join(os.path.dirname(scipy.__file__) + ".libs", "libscipy_openblas*.so"))
        if cands:
            _blas = ctypes.CDLL(cands[0])
            try:
                _blas.scipy_openblas_set_num_threads(1)
            except AttributeError:
                pass
            lib.orc_set_dgemm(ctypes.cast(_blas.scipy_dgemm_, c_void_p))
    except ImportError:
        pass
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleSystem:
    """One periodic system with one matrix index per range (all ranges share one cover set).

    ``rcuts`` lists the ranges; range ``r`` is addressed by its position in that list.
    """

    def __init__(self, coords, cell, nsf, rcuts, max_atoms_part=34, gap_threshold=None, avg_atomic_diameter=5.0):
        lib = _load()
        coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        n = coords.shape[0]
        cell = np.ascontiguousarray(cell, dtype=np.float64)
        nsf = np.ascontiguousarray(nsf, dtype=np.int32)
        rc = np.ascontiguousarray(rcuts, dtype=np.float64)
        if gap_threshold is None:
            gap_threshold = 2.0 * 7.0
        self.n_atoms = n
        self.rcuts = list(map(float, rcuts))
        self._h = lib.orc_create(n, _dp(coords), _dp(cell), nsf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 len(rc), _dp(rc), int(max_atoms_part), float(gap_threshold), float(avg_atomic_diameter))
        self._lib = lib

    def __del__(self):
        try:
            if self._h:
                self._lib.orc_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ---- index export -------------------------------------------------
    def geti(self, name, r=-1):
        n = self._lib.orc_get_int(self._h, r, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.int64)
        self._lib.orc_get_int(self._h, r, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n)
        return out

    def getd(self, name, r=-1):
        n = self._lib.orc_get_double(self._h, r, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        self._lib.orc_get_double(self._h, r, name.encode(), _dp(out), n)
        return out

    def length(self, r):
        return int(self._lib.orc_range_length(self._h, r))

    def blocklist(self, r, coords, cell):
        """Layout-agnostic description of range r (global atoms, periodic images, radii, offsets)."""
        from cq_b200.inputs import BlockList
        nnab = self.geti("n_nab", r)
        ig_prim = self.geti("ig_prim")
        ca = self.geti("icover_ibeg")[self.geti("i_part", r) - 1] + self.geti("i_seq", r) - 2   # 0-based cover atom
        ig_j = self.geti("ig_cover")[ca] - 1
        xcov = self.getd("xcover").reshape(-1, 3)
        c = np.asarray(coords, float)
        xw = c - np.floor((c + 1e-6) / cell) * cell
        shift = np.rint((xcov[ca] - xw[ig_j]) / cell).astype(np.int64)
        nd_i = np.repeat(self.geti("ndimi", r), nnab)
        nd_j = self.geti("ndimj", r)
        sizes = nd_i * nd_j
        off = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        return BlockList(np.repeat(ig_prim, nnab) - 1, ig_j, shift, self.getd("radius", r), nd_i, nd_j, off,
                         int(sizes.sum()))

    # ---- algebra -------------------------------------------------------
    def mat_mult(self, mult_type, ra, rb, rc, a, b, c, kernel="default", nthreads=0):
        """mat_mult(a, b, c) with mat_mult's own roles (multiply_module.f90:115).

        type 1: a = A (range ra), b = B (range rb), c = C (range rc) is overwritten.
        type 2: a = output (range ra) accumulates, b = B (range rb), c = input (range rc).
        kernel: "default" (multiply_kernel_default.f90, separate multiply and add), "ompGemm", "ompDoii",
        or "default_fma" (the default kernel's terms in its order, each multiply-add fused).
        """
        for arr in (a, b, c):
            assert arr.dtype == np.float64 and arr.flags.c_contiguous
        k = {"default": 0, "ompGemm": 1, "ompDoii": 2, "default_fma": 4}[kernel]
        st = self._lib.orc_mat_mult(self._h, mult_type, ra, rb, rc, _dp(a), a.size, _dp(b), b.size, _dp(c), c.size,
                                    k, int(nthreads))
        if st != 0:
            raise RuntimeError("oracle mat_mult failed (%d)" % st)

    def product_work(self, mult_type, ra, rb, rc):
        """(triples, flops) of one product: the (k, i, j) triples with a stored result and 2 nd1 nd2 nd3 each."""
        t, f = ctypes.c_int64(), ctypes.c_int64()
        self._lib.orc_product_work(self._h, mult_type, ra, rb, rc, ctypes.byref(t), ctypes.byref(f))
        return t.value, f.value

    def matrix_add(self, alpha, a, ra, beta, b, rb):
        self._lib.orc_matrix_add(self._h, float(alpha), _dp(a), ra, float(beta), _dp(b), rb)

    def transpose(self, r, a):
        at = np.zeros_like(a)
        self._lib.orc_matrix_transpose(self._h, r, _dp(np.ascontiguousarray(a)), _dp(at))
        return at

    def trace(self, r, a):
        return float(self._lib.orc_matrix_trace(self._h, r, _dp(a)))

    def vdot(self, x, y):
        """Sequential dot product (left to right)."""
        return float(self._lib.orc_vdot(x.size, _dp(x), _dp(y)))

    def exact_dot(self, x, y=None):
        """Order-independent dot product: exact fixed-point sum of the rounded products, rounded once."""
        x = np.ascontiguousarray(x, np.float64)
        if y is None:
            return float(self._lib.orc_exact_sum(x.size, _dp(x), None))
        y = np.ascontiguousarray(y, np.float64)
        return float(self._lib.orc_exact_sum(x.size, _dp(x), _dp(y)))
