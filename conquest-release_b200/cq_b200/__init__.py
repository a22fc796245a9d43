"""Python binding of libcqb200.so (B200 block-sparse multiply and LNV solver).

Thin ctypes layer over the C ABI declared in include/cq_b200.h: the product is
the CUDA library; this module only marshals arguments.  Device arrays are
passed as torch CUDA tensors (data_ptr) or raw integer device pointers.  There
is no CPU fallback: importing works without a GPU, but every call that needs
one raises if the library or the device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcqb200.so")
_lib = None

c_int, c_double, c_void_p, c_int64 = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64
P = ctypes.POINTER

# mirror of the status codes in include/cq_b200.h
(CQ_OK, CQ_ERR_ARG, CQ_ERR_OOM, CQ_ERR_CUDA, CQ_ERR_BOUNDS, CQ_ERR_TIMEOUT, CQ_ERR_STATE, CQ_ERR_NOT_CONVERGED,
 CQ_ERR_CALLBACK) = range(9)

# cq_h_rebuild_fn: (user, K_dev, H_dev, length, stream) -> status
H_REBUILD_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_void_p, c_void_p, c_int64, c_void_p)
# product arithmetic (cq_mat_mult precision)
PREC_FP64_FMA, PREC_FP64, PREC_BF16X3, PREC_BF16X6, PREC_FP64_TC = 0, 1, 2, 3, 4


class LNVParams(ctypes.Structure):
    """cq_lnv_params (include/cq_b200.h)."""
    _fields_ = [("n_L_iterations", c_int), ("tolerance", c_double), ("maxpulay", c_int), ("minpulaystep", c_double),
                ("maxpulaystep", c_double), ("lintol", c_double), ("global_tolerance", c_int), ("vary_mu", c_int),
                ("invs_max_steps", c_int), ("invs_delta_tol", c_double), ("invs_tol", c_double), ("exact", c_int),
                ("max_outer", c_int), ("mixed", c_int), ("mixed_tolerance", c_double), ("fp64_mcw_sweeps", c_int),
                ("graphs", c_int), ("mixed_mcw", c_int), ("fp64_continue", c_int), ("split_parts", c_int),
                ("mixed_max_outer", c_int), ("fp64_tensor", c_int)]


class LNVResult(ctypes.Structure):
    """cq_lnv_result (include/cq_b200.h)."""
    _fields_ = [("energy", c_double), ("electrons", c_double), ("residual", c_double), ("invs_omega", c_double),
                ("mcw_sweeps", c_int), ("early_iters", c_int), ("late_iters", c_int), ("ne_corrections", c_int),
                ("inflexions", c_int), ("converged", c_int), ("outer_iters", c_int), ("graph_launches", c_int64),
                ("n_products", c_int64),
                ("flops", c_int64),
                ("n_products_mixed", c_int64), ("flops_mixed", c_int64), ("split_restarts", c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# order of the ranges of the density-matrix chain (cq_lnv_create)
LNV_RANGE_NAMES = ("S", "H", "L", "T", "LS", "LH", "LSL", "SLS", "TS", "TH", "TL")


def lnv_ranges(rs, rh, rl, rt):
    """Range radii of the chain from the S, H, L and T ranges (src/dimens_module.f90:338-355)."""
    return {"S": rs, "H": rh, "L": rl, "T": rt, "LS": rl + rs, "LH": rl + rh, "LSL": 2 * rl + rs,
            "SLS": 2 * rs + rl, "TS": rt + rs, "TH": rt + rh, "TL": rt + rl}


class CQError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("cq_b200 error %d: %s" % (code, msg))
        self.code = code


def build():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.join(os.path.dirname(_HERE), "csrc")])


def lib():
    """Load libcqb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CQError(CQ_ERR_STATE, "libcqb200.so not built: run conquest-release_b200/csrc/Makefile")
    L = ctypes.CDLL(LIB_PATH)
    L.cq_last_error.restype = ctypes.c_char_p
    L.cq_version.restype = ctypes.c_char_p
    sigs = {
        "cq_system_create": [c_int, P(c_double), P(c_double), P(c_int), c_int, P(c_double), c_int, c_double, c_double,
                             P(c_void_p)],
        "cq_system_destroy": [c_void_p],
        "cq_range_length": [c_void_p, c_int, P(c_int64), P(c_int64)],
        "cq_export_index": [c_void_p, c_int, ctypes.c_char_p, P(c_int64), c_int64, P(c_int64)],
        "cq_export_radius": [c_void_p, c_int, P(c_double), c_int64, P(c_int64)],
        "cq_mat_mult": [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int],
        "cq_m_kern_defer": [c_int],
        "cq_m_kern_flush": [],
        "cq_mat_mult_batch": [c_int, P(c_void_p), P(c_int), P(c_int), P(c_int), P(c_int), P(c_void_p), P(c_void_p),
                              P(c_void_p), P(c_int)],
        "cq_mat_mult_host": [c_void_p, c_int, c_int, c_int, c_int, P(c_double), P(c_double), P(c_double), c_int],
        "cq_product_work": [c_void_p, c_int, c_int, c_int, c_int, P(c_int64), P(c_int64)],
        "cq_product_tuning": [c_void_p, c_int, c_int, c_int, c_int, P(c_int), P(ctypes.c_float), P(c_int),
                              P(ctypes.c_float)],
        "cq_product_tensor_work": [c_void_p, c_int, c_int, c_int, c_int, P(c_int64), P(c_int64), P(c_int)],
        "cq_matrix_sum": [c_void_p, c_int, c_void_p, c_double, c_int, c_void_p, c_double],
        "cq_matrix_transpose": [c_void_p, c_int, c_void_p, c_void_p],
        "cq_matrix_trace": [c_void_p, c_int, c_void_p, P(c_double)],
        "cq_matrix_product_trace": [c_void_p, c_int, c_void_p, c_void_p, P(c_double)],
        "cq_synchronize": [c_void_p],
        "cq_system_set_stream": [c_void_p, c_void_p],
        "cq_profile_enable": [c_void_p, c_int],
        "cq_profile_read": [c_void_p, P(c_int64), P(c_double), P(c_double), P(c_double)],
        "cq_launch_count": [c_void_p, P(c_int64)],
        "cq_lnv_solve": [c_void_p, P(LNVResult)],
        "cq_pulay_alphas": [c_int, P(c_double), c_int, c_int, P(c_double)],
        "cq_system_set_option": [c_void_p, c_int, c_int],
        "cq_generate_SH": [c_void_p, c_int, c_int, ctypes.c_uint64, c_void_p],
        "cq_dump_matrix": [c_void_p, c_int, c_void_p, ctypes.c_char_p, c_int],
        "cq_grab_matrix": [c_void_p, c_int, c_void_p, ctypes.c_char_p, P(c_int64)],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = c_int
    lnv_sigs = {
        "cq_lnv_params_default": [P(LNVParams)],
        "cq_lnv_create": [c_void_p, P(c_int), c_double, P(LNVParams), P(c_void_p)],
        "cq_lnv_destroy": [c_void_p],
        "cq_lnv_set_SH": [c_void_p, c_void_p, c_void_p, c_int],
        "cq_lnv_invert_S": [c_void_p, P(c_double)],
        "cq_lnv_find_min_dm": [c_void_p, c_int, P(LNVResult)],
        "cq_lnv_get": [c_void_p, ctypes.c_char_p, c_void_p, c_int64, c_int],
        "cq_lnv_put": [c_void_p, ctypes.c_char_p, c_void_p, c_int],
        "cq_lnv_solve_host": [c_void_p, P(c_double), P(c_double), P(c_double), P(c_double), P(LNVResult)],
        "cq_lnv_reduction_log": [c_void_p, c_int, P(c_double), c_int64, P(c_int64)],
        "cq_lnv_residual_history": [c_void_p, P(c_double), c_int64, P(c_int64)],
        "cq_lnv_force_matrices": [c_void_p, c_void_p, c_void_p, c_int],
    }
    for name, args in lnv_sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = c_int
    ip = P(c_int)
    kern = [c_int, c_int, ip, ip, ip, ip, ip, ip, P(c_double), P(c_double), P(c_double), ip, ip, ip, ip, ip, ip, ip, ip,
            c_int, ip, ip, ip, ip, c_int, c_int, c_int, c_int, c_int, c_int]
    for name in ("cq_m_kern_max", "cq_m_kern_min"):
        f = getattr(L, name)
        f.argtypes = kern
        f.restype = c_int
    _lib = L
    return L


def check(code):
    if code != CQ_OK:
        raise CQError(code, lib().cq_last_error().decode())


def _dp(a):
    return a.ctypes.data_as(P(c_double))


def _ip(a):
    return a.ctypes.data_as(P(c_int))


def _ptr(x):
    """Device pointer of a torch CUDA tensor or an integer."""
    if isinstance(x, int):
        return c_void_p(x)
    return c_void_p(x.data_ptr())


class System:
    """A periodic system with one block-sparse index per range, resident on the current GPU."""

    def __init__(self, coords, cell, nsf, rcuts, max_atoms_part=34, gap_threshold=14.0, avg_atomic_diameter=5.0):
        L = lib()
        coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        cell = np.ascontiguousarray(cell, dtype=np.float64)
        nsf = np.ascontiguousarray(nsf, dtype=np.int32)
        rc = np.ascontiguousarray(rcuts, dtype=np.float64)
        h = c_void_p()
        check(L.cq_system_create(coords.shape[0], _dp(coords), _dp(cell), _ip(nsf), len(rc), _dp(rc),
                                 int(max_atoms_part), float(gap_threshold), float(avg_atomic_diameter), ctypes.byref(h)))
        self._h = h
        self.n_atoms = coords.shape[0]
        self.rcuts = [float(x) for x in rcuts]
        # handles of the LNV solvers built on this system: close() destroys them first, whatever
        # order the garbage collector finalises the Python objects in
        self._lnvs = set()
        self._bound = {}          # matrix id -> host array bound to it (kept alive here)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            for h in list(getattr(self, "_lnvs", ())):
                lib().cq_lnv_destroy(c_void_p(h))
            self._lnvs = set()
            lib().cq_system_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def length(self, r):
        n, nb = c_int64(), c_int64()
        check(lib().cq_range_length(self._h, r, ctypes.byref(n), ctypes.byref(nb)))
        return n.value

    def n_blocks(self, r):
        n, nb = c_int64(), c_int64()
        check(lib().cq_range_length(self._h, r, ctypes.byref(n), ctypes.byref(nb)))
        return nb.value

    def geti(self, name, r=-1):
        n = c_int64()
        check(lib().cq_export_index(self._h, r, name.encode(), None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.int64)
        check(lib().cq_export_index(self._h, r, name.encode(), out.ctypes.data_as(P(c_int64)), n.value, ctypes.byref(n)))
        return out

    def radius(self, r):
        n = c_int64()
        check(lib().cq_export_radius(self._h, r, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value)
        check(lib().cq_export_radius(self._h, r, _dp(out), n.value, ctypes.byref(n)))
        return out

    # ---- products and algebra on device memory ------------------------------
    def mat_mult(self, mult_type, ra, rb, rc, a, b, c, exact=True, precision=None):
        """precision: PREC_FP64 (default kernel rounding), PREC_FP64_FMA, PREC_BF16X3 or PREC_BF16X6 (tensor cores,
        two- or three-part split), PREC_FP64_TC (FP64 on the tensor cores)."""
        prec = int(bool(exact)) if precision is None else int(precision)
        check(lib().cq_mat_mult(self._h, mult_type, ra, rb, rc, _ptr(a), _ptr(b), _ptr(c), prec))

    # ---- matrices by id (cq_matrix_*: the device side of mat_p(id)%matrix) ----------------
    def bind(self, mid, r, host=None):
        """Bind matrix id `mid` to range r: a zeroed device copy owned by the system.  `host` (a
        contiguous float64 array of the range's length, referenced here) is what upload() and
        download() copy from and to."""
        if host is not None and not (isinstance(host, np.ndarray) and host.dtype == np.float64
                                     and host.flags.c_contiguous and host.size == self.length(r)):
            raise ValueError("host must be a contiguous float64 array of the range's length")
        check(lib().cq_matrix_bind(self._h, int(mid), int(r), _dp(host) if host is not None else None))
        self._bound[int(mid)] = host

    def unbind(self, mid):
        check(lib().cq_matrix_unbind(self._h, int(mid)))
        self._bound.pop(int(mid), None)

    def upload(self, mid):
        check(lib().cq_matrix_upload(self._h, int(mid)))

    def download(self, mid):
        """Copy the device copy into the bound host array (synchronising) and return that array."""
        check(lib().cq_matrix_download(self._h, int(mid)))
        return self._bound[int(mid)]

    def device_ptr(self, mid):
        p, n = c_void_p(), c_int64()
        check(lib().cq_matrix_device(self._h, int(mid), ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def product_id(self, mult_type, ida, idb, idc, precision=PREC_FP64):
        check(lib().cq_matrix_product_id(self._h, int(mult_type), int(ida), int(idb), int(idc), int(precision)))

    def sum_id(self, ida, alpha, idb, beta):
        check(lib().cq_matrix_sum_id(self._h, int(ida), c_double(alpha), int(idb), c_double(beta)))

    def transpose_id(self, ida, idat):
        check(lib().cq_matrix_transpose_id(self._h, int(ida), int(idat)))

    def product_trace_id(self, ida, idb):
        v = c_double()
        check(lib().cq_matrix_product_trace_id(self._h, int(ida), int(idb), ctypes.byref(v)))
        return v.value

    def mat_mult_host(self, mult_type, ra, rb, rc, a, b, c, exact=True, precision=None):
        for arr in (a, b, c):
            assert arr.dtype == np.float64 and arr.flags.c_contiguous
        prec = int(bool(exact)) if precision is None else int(precision)
        check(lib().cq_mat_mult_host(self._h, mult_type, ra, rb, rc, _dp(a), _dp(b), _dp(c), prec))

    def product_work(self, mult_type, ra, rb, rc):
        t, f = c_int64(), c_int64()
        check(lib().cq_product_work(self._h, mult_type, ra, rb, rc, ctypes.byref(t), ctypes.byref(f)))
        return t.value, f.value

    def product_tuning(self, mult_type, ra, rb, rc, mixed=False):
        """FP64: (variant chosen by the autotuner or -1, {variant: timed ms}); mixed=True: (output blocks per
        warp chosen for the split-precision kernel or -1, {group size: timed ms})."""
        v, g = c_int(), c_int()
        ms, gms = (ctypes.c_float * 7)(), (ctypes.c_float * 4)()
        check(lib().cq_product_tuning(self._h, mult_type, ra, rb, rc, ctypes.byref(v), ms, ctypes.byref(g), gms))
        if mixed:
            return g.value, {gs: gms[i] for i, gs in enumerate((1, 2, 4, 8)) if gms[i] > 0}
        return v.value, {i: ms[i] for i in range(7) if ms[i] > 0}

    def product_tensor_work(self, mult_type, ra, rb, rc):
        """(tiles, issued tensor flops, usable) of the product's tcgen05 tile plan (cq_product_tensor_work)."""
        t, f, u = c_int64(), c_int64(), c_int()
        check(lib().cq_product_tensor_work(self._h, mult_type, ra, rb, rc, ctypes.byref(t), ctypes.byref(f),
                                           ctypes.byref(u)))
        return t.value, f.value, bool(u.value)

    def test_stall_next_tensor_product(self):
        """Test hook (CQ_OPT_TEST_STALL): the next tensor-core product's bounded waits run out."""
        check(lib().cq_system_set_option(self._h, 4, 1))

    def set_split_group(self, g):
        """Output blocks per warp of the mma.sync split-precision kernels: -1 = autotuned (default), 1, 2, 4
        or 8 (two-part split only); the same bits for every choice."""
        check(lib().cq_system_set_option(self._h, 5, int(g)))

    def set_mixed_kernel(self, k):
        """Kernel of the split-precision products: -1 = chosen per product by the tile plan's useful fraction
        (default), 0 = tcgen05 tiles, 1 = one block per mma.sync warp."""
        check(lib().cq_system_set_option(self._h, 3, int(k)))

    def matrix_sum(self, ra, a, alpha, rb, b, beta):
        check(lib().cq_matrix_sum(self._h, ra, _ptr(a), float(alpha), rb, _ptr(b), float(beta)))

    def transpose(self, r, a, at):
        check(lib().cq_matrix_transpose(self._h, r, _ptr(a), _ptr(at)))

    def trace(self, r, a):
        v = c_double()
        check(lib().cq_matrix_trace(self._h, r, _ptr(a), ctypes.byref(v)))
        return v.value

    def product_trace(self, r, a, b):
        v = c_double()
        check(lib().cq_matrix_product_trace(self._h, r, _ptr(a), _ptr(b), ctypes.byref(v)))
        return v.value

    def synchronize(self):
        check(lib().cq_synchronize(self._h))

    def set_stream(self, stream):
        """Enqueue on a cudaStream_t (int handle, e.g. torch.cuda.current_stream().cuda_stream); None = own."""
        check(lib().cq_system_set_stream(self._h, c_void_p(stream) if stream else None))

    def set_mult_variant(self, v):
        """FP64 4x4 product kernel: -1 = autotuned per product (default), 0 = one lane per output element,
        1 = one thread per output block, 2 = operand row staged in shared memory, 3 = warp-staged operand blocks,
        5 = four lanes per output block, 6 = operand blocks staged by bulk copies."""
        check(lib().cq_system_set_option(self._h, 1, int(v)))

    def profile(self, on=True):
        check(lib().cq_profile_enable(self._h, int(bool(on))))

    def profile_read(self):
        n, ms, by, fl = c_int64(), c_double(), c_double(), c_double()
        check(lib().cq_profile_read(self._h, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by), ctypes.byref(fl)))
        return {"launches": n.value, "ms": ms.value, "bytes": by.value, "flops": fl.value}

    def launch_count(self):
        n = c_int64()
        check(lib().cq_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def generate_SH(self, r, which, seed, out):
        """Synthetic S (which=0) or H (which=1) of range r into the device array `out`, stream-ordered."""
        check(lib().cq_generate_SH(self._h, int(r), int(which), int(seed), _ptr(out)))

    def dump_matrix(self, r, a, path, inode=1):
        """Write the device array `a` of range r as a matrix file of the reference's binary format."""
        check(lib().cq_dump_matrix(self._h, int(r), _ptr(a), os.fsencode(path), int(inode)))

    def grab_matrix(self, r, a, path):
        """Read a matrix file into the device array `a` of range r; returns the number of matched blocks."""
        m = c_int64()
        check(lib().cq_grab_matrix(self._h, int(r), _ptr(a), os.fsencode(path), ctypes.byref(m)))
        return m.value

    def set_blocking_sync(self, on=True):
        """Host waits for device scalars sleep on a blocking-sync event (many solvers per core)."""
        check(lib().cq_system_set_option(self._h, 2, int(bool(on))))

    def blocklist(self, r, coords, cell):
        """Layout-agnostic description of range r (global atoms, images, radii, offsets) for the input generators."""
        from .inputs import BlockList
        nnab = self.geti("n_nab", r)
        ig_prim = self.geti("ig_prim") - 1
        ig_j = self.geti("ig_j", r) - 1
        shift = self.geti("shift", r).reshape(-1, 3)
        nd_i = np.repeat(self.geti("ndimi", r), nnab)
        nd_j = self.geti("ndimj", r)
        elem = self.geti("elem", r)
        return BlockList(np.repeat(ig_prim, nnab), ig_j, shift, self.radius(r), nd_i, nd_j, elem, self.length(r))


def m_kern(kind, k_off, kpart, ib_nd_acc, ibaddr, nbnab, ibpart, ibseq, bndim2, a, b, c, ahalo, chalo, at,
           mx_absb=0, mx_part=0, mx_iprim=0):
    """Call cq_m_kern_max (kind='max') or cq_m_kern_min (kind='min') with Fortran-style int32 arrays.

    ahalo = dict(nh_part, j_beg, j_seq, ndimi, ndimj); chalo = dict(i_halo, i_hbeg, i_h2d, ni_in_halo);
    at = dict(i_prim, i_beg, i_nd_beg, n_hnab).  a, b, c are float64 numpy arrays (updated in place).
    """
    I = lambda x: np.ascontiguousarray(x, dtype=np.int32)
    arrs = [I(ib_nd_acc), I(ibaddr), I(nbnab), I(ibpart), I(ibseq), I(bndim2)]
    ah = [I(ahalo[k]) for k in ("nh_part", "j_beg", "j_seq", "ndimi", "ndimj")]
    ch = [I(chalo[k]) for k in ("i_halo", "i_hbeg", "i_h2d")]
    tr = [I(at[k]) for k in ("i_prim", "i_beg", "i_nd_beg", "n_hnab")]
    f = lib().cq_m_kern_max if kind == "max" else lib().cq_m_kern_min
    check(f(int(k_off), int(kpart), *[_ip(x) for x in arrs], _dp(a), _dp(b), _dp(c), *[_ip(x) for x in ah],
            *[_ip(x) for x in ch], int(chalo["ni_in_halo"]), *[_ip(x) for x in tr], int(mx_absb), int(mx_part),
            int(mx_iprim), a.size, b.size, c.size))


def m_kern_defer(np_in_halo):
    """cq_m_kern_defer: >0 = the following m_kern calls of one partition loop enqueue their work and the call
    with kpart == np_in_halo completes the loop; 0 = complete every call (flushes an open loop)."""
    check(lib().cq_m_kern_defer(int(np_in_halo)))


def m_kern_flush():
    check(lib().cq_m_kern_flush())


def mat_mult_batch(products):
    """cq_mat_mult_batch: products = [(system, mult_type, ra, rb, rc, a, b, c, precision), ...] with device
    operands (torch CUDA tensors or integer pointers) and precision PREC_FP64 or PREC_FP64_FMA; one
    persistent launch over all of them, bit-identical to separate mat_mult calls."""
    n = len(products)
    I = c_int * n
    V = c_void_p * n
    systems = V(*[p[0].handle.value for p in products])
    mt, ra, rb, rc = (I(*[int(p[k]) for p in products]) for k in (1, 2, 3, 4))
    a, b, c = (V(*[_ptr(p[k]).value for p in products]) for k in (5, 6, 7))
    prec = I(*[int(p[8]) for p in products])
    check(lib().cq_mat_mult_batch(n, systems, mt, ra, rb, rc, a, b, c, prec))


def lnv_params(**kw):
    p = LNVParams()
    check(lib().cq_lnv_params_default(ctypes.byref(p)))
    set_params(p, kw)
    return p


def set_params(p, kw):
    """Set cq_lnv_params fields by name; an unknown name is an error (ctypes would take it silently)."""
    names = {f for f, _ in LNVParams._fields_}
    for k, v in kw.items():
        if k not in names:
            raise TypeError("unknown cq_lnv_params field %r" % k)
        setattr(p, k, v)


class LNV:
    """Density-matrix solver on a System whose ranges include those of the chain.

    `range_ids` maps each name of LNV_RANGE_NAMES to a range index of the system.
    """

    def __init__(self, system, range_ids, ne_spin, **params):
        self.system = system
        ids = (c_int * 11)(*[int(range_ids[n]) for n in LNV_RANGE_NAMES])
        self._p = lnv_params(**params)
        h = c_void_p()
        check(lib().cq_lnv_create(system.handle, ids, float(ne_spin), ctypes.byref(self._p), ctypes.byref(h)))
        self._h = h
        system._lnvs.add(h.value)
        self.range_ids = dict(range_ids)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            # destroyed here unless the system's close() has already destroyed it
            if self._h.value in self.system._lnvs:
                self.system._lnvs.discard(self._h.value)
                lib().cq_lnv_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_SH(self, S, H):
        if isinstance(S, np.ndarray):
            S = np.ascontiguousarray(S, np.float64); H = np.ascontiguousarray(H, np.float64)
            check(lib().cq_lnv_set_SH(self._h, S.ctypes.data_as(c_void_p), H.ctypes.data_as(c_void_p), 0))
        else:
            check(lib().cq_lnv_set_SH(self._h, _ptr(S), _ptr(H), 1))

    def invert_S(self):
        w = c_double()
        check(lib().cq_lnv_invert_S(self._h, ctypes.byref(w)))
        return w.value

    def solve(self):
        """T = S^-1 and FindMinDM from the McWeeny start on the device-resident S and H."""
        r = LNVResult()
        check(lib().cq_lnv_solve(self._h, ctypes.byref(r)))
        return r.as_dict()

    def find_min_dm(self, resetL=True):
        r = LNVResult()
        check(lib().cq_lnv_find_min_dm(self._h, int(bool(resetL)), ctypes.byref(r)))
        return r.as_dict()

    def get(self, name):
        n = self.system.length(self.range_ids[{"L": "L", "K": "H", "T": "T", "S": "S", "H": "H", "phi": "L"}[name]])
        out = np.zeros(n)
        check(lib().cq_lnv_get(self._h, name.encode(), out.ctypes.data_as(c_void_p), n, 0))
        return out

    def put(self, name, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        check(lib().cq_lnv_put(self._h, name.encode(), arr.ctypes.data_as(c_void_p), 0))

    def reduction_log(self, enable=True, cap=1 << 20):
        """Trace values recorded since the last call, in call order; then clear the log and set recording."""
        out = np.zeros(cap)
        n = c_int64()
        check(lib().cq_lnv_reduction_log(self._h, int(bool(enable)), _dp(out), cap, ctypes.byref(n)))
        return out[:min(n.value, cap)]

    def residual_history(self):
        """Per earlyDM / lateDM iteration of the last solve: (residual, band energy, products so far,
        1.0 if split-precision, seconds since the solve started) rows of an (n, 5) array."""
        n = c_int64()
        check(lib().cq_lnv_residual_history(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 5))
        if n.value:
            check(lib().cq_lnv_residual_history(self._h, _dp(out), n.value, ctypes.byref(n)))
        return out

    def set_h_rebuild(self, fn):
        """Mixed-L self-consistency (minE.MixedLSelfConsistent): lateDM calls fn(K_ptr, H_ptr, length,
        stream) with the solver's device pointers of K and H (H range) at its start and after every
        Pulay step; fn writes the new H into H_ptr, ordered on `stream`, and returns 0.  None
        switches the coupling off."""
        if fn is None:
            self._h_cb = None
            check(lib().cq_lnv_set_h_rebuild(self._h, H_REBUILD_FN(), None))
            return

        def tramp(user, k, h, n, stream):
            try:
                return int(fn(k or 0, h or 0, int(n), stream or 0))
            except Exception:
                return -1
        self._h_cb = H_REBUILD_FN(tramp)      # kept alive while the solver may call it
        check(lib().cq_lnv_set_h_rebuild(self._h, self._h_cb, None))

    def force_matrices(self):
        """(M12 in the S range, M4 in the H range) of the current L, as host arrays."""
        M12 = np.zeros(self.system.length(self.range_ids["S"]))
        M4 = np.zeros(self.system.length(self.range_ids["H"]))
        check(lib().cq_lnv_force_matrices(self._h, M12.ctypes.data_as(c_void_p), M4.ctypes.data_as(c_void_p), 0))
        return M12, M4

    def solve_host(self, S, H, want_L=False, want_K=False):
        S = np.ascontiguousarray(S, np.float64); H = np.ascontiguousarray(H, np.float64)
        Lo = np.zeros(self.system.length(self.range_ids["L"])) if want_L else None
        Ko = np.zeros(self.system.length(self.range_ids["H"])) if want_K else None
        r = LNVResult()
        check(lib().cq_lnv_solve_host(self._h, _dp(S), _dp(H), _dp(Lo) if Lo is not None else None,
                                      _dp(Ko) if Ko is not None else None, ctypes.byref(r)))
        return r.as_dict(), Lo, Ko


def solve_cubic(a, b, c, guess):
    """SolveCubic root (host computation in libcqb200.so)."""
    x = c_double()
    check(lib().cq_solve_cubic(c_double(a), c_double(b), c_double(c), c_double(guess), ctypes.byref(x)))
    return x.value


def pulay_alphas(ipulay, Aij, n, max_n):
    """DoPulay2D_nospin mixing coefficients (host computation in libcqb200.so)."""
    A = np.zeros((max_n, max_n))
    A[:n, :n] = np.asarray(Aij)[:n, :n]
    Af = np.asfortranarray(A)
    al = np.zeros(max_n)
    check(lib().cq_pulay_alphas(int(ipulay), Af.ctypes.data_as(P(c_double)), int(n), int(max_n), _dp(al)))
    return al


# --------------------------------------------------------------------------
# serving loop (cq_server_*): continuous batching of independent solves
# --------------------------------------------------------------------------
class ServerConfig(ctypes.Structure):
    """cq_server_config (include/cq_b200.h)."""
    _fields_ = [("n_slots", c_int), ("hbm_budget", c_int64), ("max_bypass", c_int), ("blocking_sync", c_int),
                ("dry_run", c_int), ("dry_run_seconds", c_double), ("lnv", LNVParams), ("batch_products", c_int),
                ("batch_window_us", c_double)]


class Request(ctypes.Structure):
    """cq_request (include/cq_b200.h)."""
    _fields_ = [("n_atoms", c_int), ("coords", P(c_double)), ("cell", P(c_double)), ("nsf", P(c_int)),
                ("rs", c_double), ("rh", c_double), ("rl", c_double), ("rt", c_double), ("ne_spin", c_double),
                ("seed", ctypes.c_uint64), ("mixed", c_int), ("t_arrival", c_double)]


class RequestResult(ctypes.Structure):
    """cq_request_result (include/cq_b200.h)."""
    _fields_ = [("id", c_int64), ("status", c_int), ("n_atoms", c_int), ("converged", c_int), ("mixed", c_int),
                ("slot", c_int), ("energy", c_double), ("electrons", c_double), ("residual", c_double),
                ("n_products", c_int64), ("flops", c_int64), ("n_products_mixed", c_int64), ("flops_mixed", c_int64),
                ("t_arrival", c_double), ("t_admit", c_double), ("t_done", c_double), ("bytes_estimate", c_int64),
                ("bytes_peak", c_int64), ("message", ctypes.c_char * 128), ("split_restarts", c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["message"] = self.message.decode(errors="replace")
        d["latency"] = self.t_done - self.t_arrival
        return d


def _server_lib():
    L = lib()
    if not getattr(L, "_server_sigs", False):
        sigs = {
            "cq_server_config_default": [P(ServerConfig)],
            "cq_server_create": [P(ServerConfig), P(c_void_p)],
            "cq_server_submit": [c_void_p, P(Request), P(c_int64)],
            "cq_server_wait": [c_void_p, c_int64, c_double, P(RequestResult)],
            "cq_server_now": [c_void_p, P(c_double)],
            "cq_request_estimate": [P(Request), P(c_int64)],
            "cq_server_destroy": [c_void_p],
        }
        for name, args in sigs.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = c_int
        L._server_sigs = True
    return L


def _request(coords, cell, nsf, rs, rh, rl, rt, ne_spin, seed=0, mixed=False, t_arrival=-1.0):
    coords = np.ascontiguousarray(coords, np.float64).reshape(-1, 3)
    cell = np.ascontiguousarray(cell, np.float64)
    nsf = np.ascontiguousarray(np.broadcast_to(nsf, (len(coords),)), np.int32)
    r = Request(len(coords), _dp(coords), _dp(cell), _ip(nsf), rs, rh, rl, rt, float(ne_spin), int(seed),
                int(bool(mixed)), float(t_arrival))
    return r, (coords, cell, nsf)   # the arrays must stay alive while the request is read


def request_estimate(coords, cell, nsf, rs, rh, rl, rt, ne_spin=1.0, mixed=False):
    """Device bytes the server's admission reserves for this solve."""
    r, keep = _request(coords, cell, nsf, rs, rh, rl, rt, ne_spin, mixed=mixed)
    b = c_int64()
    check(_server_lib().cq_request_estimate(ctypes.byref(r), ctypes.byref(b)))
    return b.value


class Server:
    """Continuous-batching server of density-matrix solves (cq_server_*).

    Each request is one system given by its geometry and ranges; S and H are generated on the
    device from `seed`, and the result carries energy, electron count, work and latency.
    """

    def __init__(self, n_slots=8, hbm_budget=64 << 30, max_bypass=4, blocking_sync=True, dry_run=False,
                 dry_run_seconds=0.01, batch_products=False, batch_window_us=50.0, **lnv):
        L = _server_lib()
        c = ServerConfig()
        check(L.cq_server_config_default(ctypes.byref(c)))
        c.n_slots, c.hbm_budget, c.max_bypass = int(n_slots), int(hbm_budget), int(max_bypass)
        c.blocking_sync, c.dry_run, c.dry_run_seconds = int(bool(blocking_sync)), int(bool(dry_run)), float(dry_run_seconds)
        c.batch_products, c.batch_window_us = int(bool(batch_products)), float(batch_window_us)
        set_params(c.lnv, lnv)
        h = c_void_p()
        check(L.cq_server_create(ctypes.byref(c), ctypes.byref(h)))
        self._h = h

    def submit(self, coords, cell, nsf, rs, rh, rl, rt, ne_spin, seed=0, mixed=False, t_arrival=-1.0):
        r, keep = _request(coords, cell, nsf, rs, rh, rl, rt, ne_spin, seed, mixed, t_arrival)
        i = c_int64()
        check(_server_lib().cq_server_submit(self._h, ctypes.byref(r), ctypes.byref(i)))
        return i.value

    def wait(self, rid, timeout=-1.0):
        out = RequestResult()
        check(_server_lib().cq_server_wait(self._h, int(rid), float(timeout), ctypes.byref(out)))
        return out.as_dict()

    def now(self):
        t = c_double()
        check(_server_lib().cq_server_now(self._h, ctypes.byref(t)))
        return t.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _server_lib().cq_server_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NOALLOC_MAX_SUMS = 8   # CQ_NOALLOC_MAX_SUMS


def exact_dots_noalloc(xs, ys=None, stream=None):
    """cq_exact_dots_noalloc: exact dot products (plain sums where ys[k] is None) of device arrays,
    with the scratch in a static device array, for callers that cannot allocate device memory.
    Calls that overlap on the GPU share that scratch and must be serialised by the caller."""
    L = lib()
    f = L.cq_exact_dots_noalloc
    f.argtypes = [c_int, P(c_void_p), P(c_void_p), P(c_int64), c_void_p, P(c_double)]
    f.restype = c_int
    k = len(xs)
    xp = (c_void_p * max(k, 1))(*[_ptr(x).value for x in xs])
    yp = None
    if ys is not None:
        yp = (c_void_p * max(k, 1))(*[(_ptr(y).value if y is not None else None) for y in ys])
    ns = (c_int64 * max(k, 1))(*[int(x.numel()) for x in xs])
    out = (c_double * max(k, 1))()
    check(f(k, xp, yp, ns, c_void_p(stream) if stream else None, out))
    return [out[i] for i in range(k)]
