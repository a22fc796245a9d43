"""LNV / McWeeny density-matrix minimisation -- CPU ORACLE (test infrastructure only).

A line-by-line restatement, for one spin channel with nspin = 1 (spin_factor = 2),
of the reference's density-matrix chain on top of the oracle's ``mat_mult``:

  src/mult_module.f90     LNV_matrix_multiply 1478-1823, symmetrise_L 1856-1893,
                          matrix_product 2556-2606, matrix_sum 2677-2715
  src/DMMinModule.f90     FindMinDM 172-312, earlyDM 366-723, lateDM 809-1339,
                          lineMinL 1395-1614, correct_electron_number_fixspin 1676-1817,
                          SolveCubic 2072-2143
  src/McWeeny.f90         McWMin 107-272, InitMcW 340-570, McW_matrix_multiply_nonds 620-740,
                          McWXHX 908-946, McWRho0 961-987, GetHLimits 1020-1109
  src/Pulay.f90           DoPulay2D_nospin 188-262 (LAPACK dsytrf/dsytri via scipy)
  src/S_matrix_module.f90 Iter_Hott_InvS 746-963, HotInvS_mm 994-1032

Only tests/, bench.py's CPU baseline and smoke() use this module, as the checker.
Parity status: pinned by known-answer tests (dense purification / eigh), not by
reference outputs, which cannot be produced in this image.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg.lapack as lapack

RD_ERR = 1.0e-8

# product table (src/mult_module.f90:571-...) in mat_mult roles (type, a range, b range, c range)
MULTS = {
    "L_S_LS": (1, "L", "S", "LS"),
    "L_H_LH": (1, "L", "H", "LH"),
    "T_S_TS": (1, "T", "S", "TS"),
    "SL_S_SLS": (1, "LS", "S", "SLS"),      # SL range = LS range
    "LS_L_LSL": (1, "LS", "L", "LSL"),
    "HL_S_LSL": (1, "LH", "S", "LSL"),      # HL range = LH range
    "HLS_LS_L": (2, "L", "LS", "LSL"),      # = LSL_SL_L
    "SLS_LS_L": (2, "L", "LS", "SLS"),
    "LSL_SL_H": (2, "H", "LS", "LSL"),
    "TS_T_T": (2, "T", "T", "TS"),
    "TH_T_L": (2, "L", "T", "TH"),          # type 2 since rcut(TH) > rcut(L)
    "T_H_TH": (1, "T", "H", "TH"),
    "T_L_TL": (1, "T", "L", "TL"),
    "TL_T_L": (2, "L", "T", "TL"),
    "LH_L_SLS": (1, "LH", "L", "SLS"),      # type 1 while rcut(SLS) >= rcut(LH) (mult_module.f90:660-680)
    "LHL_SL_S": (2, "S", "LS", "SLS"),      # mult_module.f90:753-760
}


def bk_inverse(A):
    """Inverse of a small symmetric matrix by Bunch-Kaufman diagonal pivoting (LAPACK dsytf2 'U',
    alpha = (1 + sqrt(17)) / 8) and dsytri 'U'.  A is a list of rows (modified copy); returns the
    full inverse as a list of rows, or None when a pivot block is singular."""
    n = len(A)
    a = [row[:] for row in A]          # a[i][j], 0-based
    alpha = (1.0 + math.sqrt(17.0)) / 8.0
    ipiv = [0] * n
    k = n - 1
    while k >= 0:
        kstep = 1
        absakk = abs(a[k][k])
        imax, colmax = 0, 0.0
        for i in range(k):
            if abs(a[i][k]) > colmax:
                colmax = abs(a[i][k]); imax = i
        if max(absakk, colmax) == 0.0 or math.isnan(absakk):
            return None
        if absakk >= alpha * colmax:
            kp = k
        else:
            rowmax = 0.0
            for j in range(imax + 1, k + 1):
                rowmax = max(rowmax, abs(a[imax][j]))
            for j in range(imax):
                rowmax = max(rowmax, abs(a[j][imax]))
            if absakk >= alpha * colmax * (colmax / rowmax):
                kp = k
            elif abs(a[imax][imax]) >= alpha * rowmax:
                kp = imax
            else:
                kp = imax; kstep = 2
        kk = k - kstep + 1
        if kp != kk:
            for i in range(kp):
                a[i][kk], a[i][kp] = a[i][kp], a[i][kk]
            for j in range(kp + 1, kk):
                a[j][kk], a[kp][j] = a[kp][j], a[j][kk]
            a[kk][kk], a[kp][kp] = a[kp][kp], a[kk][kk]
            if kstep == 2:
                a[k - 1][k], a[kp][k] = a[kp][k], a[k - 1][k]
        if kstep == 1:
            r1 = 1.0 / a[k][k]
            for j in range(k - 1, -1, -1):
                f = -r1 * a[j][k]
                for i in range(j + 1):
                    a[i][j] += a[i][k] * f
            for i in range(k):
                a[i][k] *= r1
        elif k > 1:
            d12 = a[k - 1][k]
            d22 = a[k - 1][k - 1] / d12
            d11 = a[k][k] / d12
            t = 1.0 / (d11 * d22 - 1.0)
            d12 = t / d12
            for j in range(k - 2, -1, -1):
                wkm1 = d12 * (d11 * a[j][k - 1] - a[j][k])
                wk = d12 * (d22 * a[j][k] - a[j][k - 1])
                for i in range(j, -1, -1):
                    a[i][j] = a[i][j] - a[i][k] * wk - a[i][k - 1] * wkm1
                a[j][k] = wk
                a[j][k - 1] = wkm1
        if kstep == 1:
            ipiv[k] = kp + 1
        else:
            ipiv[k] = -(kp + 1); ipiv[k - 1] = -(kp + 1)
        k -= kstep
    for i in range(n - 1, -1, -1):
        if ipiv[i] > 0 and a[i][i] == 0.0:
            return None

    def inv_col(kc, m):
        work = [a[i][kc] for i in range(m)]
        y = []
        for i in range(m):
            s = 0.0
            for j in range(m):
                s += (a[i][j] if i <= j else a[j][i]) * work[j]
            y.append(s)
        for i in range(m):
            a[i][kc] = -y[i]
        s = 0.0
        for i in range(m):
            s += work[i] * a[i][kc]
        return s

    k = 0
    while k < n:
        if ipiv[k] > 0:
            a[k][k] = 1.0 / a[k][k]
            if k > 0:
                a[k][k] -= inv_col(k, k)
            kstep = 1
        else:
            t = abs(a[k][k + 1])
            ak = a[k][k] / t
            akp1 = a[k + 1][k + 1] / t
            akkp1 = a[k][k + 1] / t
            d = t * (ak * akp1 - 1.0)
            a[k][k] = akp1 / d
            a[k + 1][k + 1] = ak / d
            a[k][k + 1] = -akkp1 / d
            if k > 0:
                a[k][k] -= inv_col(k, k)
                s = 0.0
                for i in range(k):
                    s += a[i][k] * a[i][k + 1]
                a[k][k + 1] -= s
                a[k + 1][k + 1] -= inv_col(k + 1, k)
            kstep = 2
        kp = abs(ipiv[k]) - 1
        if kp != k:
            for i in range(kp):
                a[i][k], a[i][kp] = a[i][kp], a[i][k]
            for j in range(kp + 1, k):
                a[j][k], a[kp][j] = a[kp][j], a[j][k]
            a[k][k], a[kp][kp] = a[kp][kp], a[k][k]
            if kstep == 2:
                a[k][k + 1], a[kp][k + 1] = a[kp][k + 1], a[k][k + 1]
        k += kstep
    for i in range(n):
        for j in range(i + 1, n):
            a[j][i] = a[i][j]
    return a


class Params:
    def __init__(self, n_L_iterations=50, tolerance=1.0e-7, maxpulay=5, minpulaystep=1.0e-3, maxpulaystep=0.1,
                 lintol=0.1, global_tolerance=False, vary_mu=True, invs_max_steps=100, invs_delta_tol=1.0e-4,
                 invs_tol=1.0e-2):
        self.n_L_iterations = n_L_iterations
        self.tolerance = tolerance
        self.maxpulay = maxpulay
        self.minpulaystep = minpulaystep
        self.maxpulaystep = maxpulaystep
        self.lintol = lintol
        self.global_tolerance = global_tolerance
        self.vary_mu = vary_mu
        self.invs_max_steps = invs_max_steps
        self.invs_delta_tol = invs_delta_tol
        self.invs_tol = invs_tol


class Mat:
    __slots__ = ("rng", "v")

    def __init__(self, rng, v):
        self.rng = rng
        self.v = v


class OracleLNV:
    """Density-matrix chain on an OracleSystem whose ranges are named in `ridx` (name -> range index)."""

    def __init__(self, osys, ridx, S, H, ne_spin, n_orbitals, params=None, kernel="ompDoii", nthreads=0):
        self.o = osys
        self.ridx = dict(ridx)
        self.p = params or Params()
        self.kernel = kernel
        self.nthreads = nthreads
        self.ne = float(ne_spin)            # ne_spin_in_cell(1)
        self.n_o = float(n_orbitals)        # sum of nsf over atoms
        self.ni_in_cell = osys.n_atoms
        self.spin_factor = 2.0
        self.S = Mat("S", np.array(S, dtype=np.float64))
        self.H = Mat("H", np.array(H, dtype=np.float64))
        self.L = self.temp("L")
        self.T = self.temp("T")
        self.Ttran = self.temp("T")
        self.LS = self.temp("LS")
        self.SL = self.temp("LS")
        self.K = self.temp("H")
        self.phi = self.temp("L")
        self.delta_e = 0.0                  # `save` variable of FindMinDM
        self.n_products = 0
        self.flops = 0                      # algorithmic flops of the products run so far
        self._work = {}
        # optional: a callable run before every product (a bounded sample stops the chain by raising)
        self.before_product = None
        self.log = []
        self.rlog = []          # every trace / product-trace value in call order (chain comparison)
        # minE.MixedLSelfConsistent: callable(K values) -> new H values, run by lateDM
        self.h_rebuild = None
        self.h_rebuilds = 0

    # ---- matrix layer (mult_module) -------------------------------------
    def temp(self, rng):
        return Mat(rng, np.zeros(self.o.length(self.ridx[rng])))

    def product(self, A, B, C, mult):
        t, ra, rb, rc = MULTS[mult]
        if self.before_product is not None:
            self.before_product(self)
        self.n_products += 1
        key = (t, ra, rb, rc)
        if key not in self._work:
            self._work[key] = self.o.product_work(t, self.ridx[ra], self.ridx[rb], self.ridx[rc])[1]
        self.flops += self._work[key]
        if t == 1:
            assert A.rng == ra and B.rng == rb and C.rng == rc, mult
            self.o.mat_mult(1, self.ridx[ra], self.ridx[rb], self.ridx[rc], A.v, B.v, C.v, kernel=self.kernel,
                            nthreads=self.nthreads)
        else:
            assert C.rng == ra and B.rng == rb and A.rng == rc, mult
            C.v[:] = 0.0
            self.o.mat_mult(2, self.ridx[ra], self.ridx[rb], self.ridx[rc], C.v, B.v, A.v, kernel=self.kernel,
                            nthreads=self.nthreads)

    def msum(self, alpha, A, beta, B):
        """matrix_sum: same range -> scal + axpy, else matrix_add on the shared blocks."""
        if A.rng == B.rng:
            A.v *= alpha
            A.v += beta * B.v
        else:
            self.o.matrix_add(alpha, A.v, self.ridx[A.rng], beta, B.v, self.ridx[B.rng])

    def scale(self, alpha, A):
        A.v *= alpha

    def transpose(self, A, AT):
        AT.v[:] = self.o.transpose(self.ridx[A.rng], A.v)

    def ptrace(self, A, B):
        """matrix_product_trace: vdot over the storage, summed exactly (order independent)."""
        assert A.rng == B.rng
        v = self.o.exact_dot(A.v, B.v)
        self.rlog.append(v)
        return v

    def trace(self, A):
        v = self.o.trace(self.ridx[A.rng], A.v)
        self.rlog.append(v)
        return v

    def copy(self, A):
        return Mat(A.rng, A.v.copy())

    # ---- force matrices: the doM1 + doM2 and doM4 branches of LNV_matrix_multiply ----------
    def force_matrices(self):
        """M12 = 3 LHL - 2 LHLSL - 2 LSLHL (S range) and M4 = 12 LSL - 12 LSLSL (H range) of the current
        L (mult_module.f90:1564-1592, 1680-1726), the matrices the forces need from the density matrix."""
        L, S, H = self.L, self.S, self.H
        self.product(L, S, self.LS, "L_S_LS")
        self.transpose(self.LS, self.SL)
        LH = self.temp("LH")
        self.product(L, H, LH, "L_H_LH")
        LHL = self.temp("SLS")
        self.product(LH, L, LHL, "LH_L_SLS")
        LHLSL = self.temp("S"); LSLHL = self.temp("S")
        self.product(LHL, self.LS, LHLSL, "LHL_SL_S")
        self.transpose(LHLSL, LSLHL)
        LSL = self.temp("LSL"); LSLSL = self.temp("H")
        self.product(self.LS, L, LSL, "LS_L_LSL")
        self.product(LSL, self.LS, LSLSL, "LSL_SL_H")
        M12 = self.temp("S"); M4 = self.temp("H")
        self.msum(0.0, M4, 12.0, LSL)
        self.msum(1.0, M4, -12.0, LSLSL)
        self.msum(0.0, M12, 3.0, LHL)
        self.msum(1.0, M12, -2.0, LHLSL)
        self.msum(1.0, M12, -2.0, LSLHL)
        return M12.v, M4.v

    # ---- LNV_matrix_multiply (doM3, dophi, doE, doK; doM1/doM2/doM4: force_matrices) ----
    def lnv(self, doK=False, doM3=False, dophi=False, doE=False, M3=None, phi=None):
        L, S, H = self.L, self.S, self.H
        electrons = energy = None
        self.product(L, S, self.LS, "L_S_LS")
        self.transpose(self.LS, self.SL)
        if doM3:
            LH = self.temp("LH"); HL = self.temp("LH")
            self.product(L, H, LH, "L_H_LH")
            self.transpose(LH, HL)
            HLS = self.temp("LSL"); SLH = self.temp("LSL"); A = self.temp("LSL")
            B = self.temp("L"); C = self.temp("L")
            self.product(HL, S, HLS, "HL_S_LSL")
            self.product(HL, S, HLS, "HL_S_LSL")   # the reference computes this product twice (mult_module.f90:1609,1615)
            self.transpose(HLS, SLH)
            self.msum(0.0, A, 2.0, HLS)
            self.msum(1.0, A, 1.0, SLH)
            self.product(A, self.SL, B, "HLS_LS_L")
            self.transpose(B, C)
        if dophi:
            SLS = self.temp("SLS"); SLSLS = self.temp("L")
            self.product(self.SL, S, SLS, "SL_S_SLS")
            self.product(SLS, self.SL, SLSLS, "SLS_LS_L")
        if doK or doE:
            LSL = self.temp("LSL"); LSLSL = self.temp("H")
            self.product(self.LS, L, LSL, "LS_L_LSL")
            self.product(LSL, self.LS, LSLSL, "LSL_SL_H")
            self.msum(0.0, self.K, 3.0, LSL)
            self.msum(1.0, self.K, -2.0, LSLSL)
        if doE:
            energy = self.ptrace(H, self.K)
        if doM3:
            self.msum(0.0, M3, 3.0, HLS)
            self.msum(1.0, M3, 3.0, SLH)
            self.msum(1.0, M3, -1.0, B)
            self.msum(1.0, M3, -1.0, C)
        if dophi:
            self.msum(0.0, phi, 1.0, SLS)
            e1 = self.ptrace(L, phi)
            e2 = self.ptrace(L, SLSLS)
            electrons = 3.0 * e1 - 2.0 * e2
            self.msum(6.0, phi, -6.0, SLSLS)
        return electrons, energy

    def symmetrise_L(self):
        tmp = self.temp("L")
        self.transpose(self.L, tmp)
        self.msum(0.5, self.L, 0.5, tmp)

    def TMT(self, M, out, mat_temp, Tright):
        """T.M.T via T_L_TL then TL_T_L (earlyDM 450-451)."""
        self.product(self.T, M, mat_temp, "T_L_TL")
        self.product(mat_temp, Tright, out, "TL_T_L")

    def gsum_norm(self, A, B):
        g = self.spin_factor * self.ptrace(A, B)
        if not self.p.global_tolerance:
            g /= float(self.ni_in_cell)
        return g

    # ---- S^-1 by Hotelling (S_matrix_module.f90:746-1032) ----------------
    def iter_hott_invs(self):
        p = self.p
        n_orbs = self.n_o
        matI = self.temp("TS"); matT1 = self.temp("T"); matTold = self.temp("T"); matTM = self.temp("TS")
        onsite_I = self.o.geti("onsite", self.ridx["TS"])
        ndimi = self.o.geti("ndimi", self.ridx["TS"])
        onsite_T = self.o.geti("onsite", self.ridx["T"])
        for on, nd in zip(onsite_I, ndimi):
            for j in range(nd):
                matI.v[on - 1 + j * nd + j] = 1.0
        self.T.v[:] = 0.0
        for on, nd in zip(onsite_T, ndimi):
            for j in range(nd):
                self.T.v[on - 1 + j * nd + j] = 1.0
        # sum of squares of S, visited per block row orbital then column orbital (S_matrix_module.f90:834-850)
        rS = self.ridx["S"]
        ndj = self.o.geti("ndimj", rS)
        ndi_b = np.repeat(self.o.geti("ndimi", rS), self.o.geti("n_nab", rS))
        order = []
        pos = 0
        for a_, b_ in zip(ndi_b, ndj):
            blk = np.arange(pos, pos + a_ * b_).reshape(b_, a_)   # element (n1, n2) at n1 + a_*n2
            order.append(blk.T.ravel())
            pos += a_ * b_
        sq = self.S.v[np.concatenate(order)] ** 2
        tot = float(np.cumsum(sq)[-1])   # sequential left-to-right sum
        eps = 1.0 / tot
        self.scale(0.0, self.T)
        self.msum(0.0, self.T, eps, self.S)
        deltaomega = 0.0
        oldomega = 0.0
        omega = 0.0
        for n in range(1, p.invs_max_steps + 1):
            deltaomega = deltaomega * 0.5
            if n < 3 or abs(deltaomega) > p.invs_delta_tol:
                omega = self.hot_invs_mm(matI, matT1, matTM)
                deltaomega = omega - oldomega
                if omega > oldomega and oldomega != 0.0:
                    self.msum(0.0, self.T, 1.0, matTold)
                    omega = oldomega
                    break
                oldomega = omega
                self.msum(0.0, matTold, 1.0, self.T)
                self.msum(0.0, self.T, 1.0, matT1)
            else:
                break
        if omega / n_orbs > p.invs_tol:
            self.T.v[:] = 0.0
            for on, nd in zip(onsite_T, ndimi):
                for j in range(nd):
                    self.T.v[on - 1 + j * nd + j] = 1.0
        self.log.append(("invS", omega))
        return omega

    def hot_invs_mm(self, matI, matT1, matA):
        T0S = self.temp("TS"); Grad = self.temp("T")
        self.product(self.T, self.S, T0S, "T_S_TS")
        self.msum(0.0, matA, 1.0, matI)
        self.msum(1.0, matA, -1.0, T0S)
        self.product(T0S, self.T, Grad, "TS_T_T")
        self.msum(0.0, matT1, 2.0, self.T)
        self.msum(1.0, matT1, -1.0, Grad)
        return self.ptrace(matA, matA)

    # ---- McWeeny (McWeeny.f90) -------------------------------------------
    def get_h_limits(self):
        r = self.ridx["H"]
        nnab = self.o.geti("n_nab", r)
        iacc = self.o.geti("i_acc", r)
        inda = self.o.geti("i_nd_acc", r)
        ndimi = self.o.geti("ndimi", r)
        ndimj = self.o.geti("ndimj", r)
        onsite = self.o.geti("onsite", r)
        h = self.H.v
        minH, maxH = 1.0e30, -1.0e30
        for p_ in range(len(nnab)):
            nsfi = int(ndimi[p_])
            hmin = [0.0] * 64
            hmax = [0.0] * 64
            pos = int(inda[p_]) - 1
            for nb in range(int(nnab[p_])):
                e = int(iacc[p_]) - 1 + nb
                nsfj = int(ndimj[e])
                on = (pos + 1) == int(onsite[p_])
                for i in range(nsfj):
                    for j in range(nsfi):
                        v = abs(h[pos + i * nsfi + j])
                        if on:
                            hmin[i] += v
                        else:
                            hmin[i] -= v
                        hmax[i] += v
                pos += nsfi * nsfj
            for i in range(nsfi):
                minH = min(minH, hmin[i])
                maxH = max(maxH, hmax[i])
        return minH, maxH

    def mcw_xhx(self, matXHX, mat_temp):
        BA = self.temp("TH")
        self.product(self.T, self.H, BA, "T_H_TH")
        self.product(BA, self.T, matXHX, "TH_T_L")
        self.msum(0.0, mat_temp, 1.0, matXHX)

    def init_mcw(self):
        ne, n_o = self.ne, self.n_o
        TS = self.temp("TS")
        self.product(self.T, self.S, TS, "T_S_TS")
        SX = self.trace(TS)
        XHX = self.temp("L"); mat_temp = self.temp("S")
        self.mcw_xhx(XHX, mat_temp)
        SXHX = self.ptrace(self.S, mat_temp)
        hmin, hmax = self.get_h_limits()
        A = 1.0 - SX / n_o
        if n_o == ne:
            mubar = 0.0; lam = 0.0
        else:
            mu1 = SXHX / n_o + hmax * A
            mu2 = (hmin * A * ne / (n_o - ne) - SXHX / n_o) / (n_o * A / (n_o - ne) - 1.0)
            if (ne / (hmax - mu1)) < ((n_o - ne) / (mu1 - hmin)):
                mubar = mu1; lam = ne / (hmax - mu1)
            elif (ne / (hmax - mu2)) > ((n_o - ne) / (mu2 - hmin)):
                mubar = mu2; lam = (n_o - ne) / (mu2 - hmin)
            else:
                raise RuntimeError("InitMcW: Cannot find mubar.")
        self.log.append(("InitMcW", SX, SXHX, hmin, hmax, mubar, lam))
        # McWRho0: L = ((lam*mu + ne)/n_o) T - (lam/n_o) XHX
        self.msum(0.0, self.L, (lam * mubar + ne) / n_o, self.T)
        self.msum(1.0, self.L, -lam / n_o, XHX)

    def mcw_mm_nonds(self, RhoNew):
        L, S = self.L, self.S
        self.product(L, S, self.LS, "L_S_LS")
        LSL = self.temp("LSL"); LSLSL = self.temp("L"); top = self.temp("S"); bottom = self.temp("S")
        self.product(self.LS, L, LSL, "LS_L_LSL")
        self.product(LSL, self.LS, LSLSL, "HLS_LS_L")   # LSL_SL_L == HLS_LS_L
        self.msum(0.0, top, 1.0, LSL)
        self.msum(1.0, top, -1.0, LSLSL)
        c1 = self.ptrace(S, top)
        self.msum(0.0, bottom, 1.0, L)
        self.msum(1.0, bottom, -1.0, LSL)
        c2 = self.ptrace(S, bottom)
        if abs(c2) > 1e-15:
            cn = c1 / c2
        else:
            raise RuntimeError("McW_matrix_multiply: c2 is near zero")
        c = cn
        self.scale(0.0, RhoNew)
        self.msum(0.0, RhoNew, -1.0, LSLSL)
        self.msum(1.0, RhoNew, 1.0 + cn, LSL)
        if cn < 0.5:
            self.msum(1.0, RhoNew, 1.0 - 2.0 * cn, L)
            self.scale(1.0 / (1.0 - cn), RhoNew)
        else:
            self.scale(1.0 / cn, RhoNew)
        bottomH = self.temp("H")
        self.msum(0.0, bottomH, 1.0, RhoNew)
        energy = self.ptrace(bottomH, self.H)
        if abs(c2) < 1.0e-6:
            c = -0.01
        return energy, c

    def mcw_min(self, n_L_iterations):
        oldE = 1.0e30
        oldL = self.copy(self.L)
        RhoNew = self.temp("L")
        deltaE = self.delta_e
        n_it = n_L_iterations + 1
        for n in range(1, n_L_iterations + 1):
            omega1, cn = self.mcw_mm_nonds(RhoNew)
            if omega1 > oldE or abs(omega1 - oldE) < 1.0e-8 or cn > 1.0 or cn < 0.0:
                n_it = n
                break
            deltaE = 0.0
            deltaE += self.spin_factor * (omega1 - oldE)
            self.msum(0.0, self.L, 1.0, RhoNew)
            oldE = omega1
            self.symmetrise_L()
        if n_it < 3:
            self.msum(0.0, self.L, 1.0, oldL)
        self.log.append(("McWMin", n_it, oldE))
        return deltaE

    # ---- DMMin (DMMinModule.f90) --------------------------------------------
    @staticmethod
    def solve_cubic(a, b, c, guess):
        Q = (a * a - 3.0 * b) / 9.0
        R = (2.0 * a * a * a - 9.0 * a * b + 27.0 * c) / 54.0
        if R * R < Q * Q * Q:
            theta = math.acos(R / (math.sqrt(Q * Q * Q)))
            T = -2.0 * math.sqrt(Q)
            twopi = 2.0 * math.pi
            z1 = T * math.cos(theta / 3.0) - (a / 3.0)
            z2 = T * math.cos((theta + twopi) / 3.0) - (a / 3.0)
            z3 = T * math.cos((theta - twopi) / 3.0) - (a / 3.0)
            if abs(z1) <= abs(z2) and abs(z1) <= abs(z3):
                return z1
            elif abs(z2) <= abs(z3):
                return z2
            return z3
        Q = -Q
        R = -R
        S = R + math.sqrt(Q * Q * Q + R * R)
        T = R - math.sqrt(Q * Q * Q + R * R)
        S = S ** (1.0 / 3.0) if S >= 0.0 else -abs(S) ** (1.0 / 3.0)
        T = T ** (1.0 / 3.0) if T >= 0.0 else -abs(T) ** (1.0 / 3.0)
        x = S + T - a / 3.0
        if abs(x) > 10.0 * abs(guess):
            x = guess
        return x

    def correct_electron_number(self):
        self.transpose(self.T, self.Ttran)
        TL = self.temp("TL"); phi2 = self.temp("L"); Sphi = self.temp("L"); Sphi2 = self.temp("L")
        ne0 = self.ne
        done = False
        it = 0
        while not done and it < 20:
            electrons, _ = self.lnv(dophi=True, phi=self.phi)
            self.TMT(self.phi, Sphi, TL, self.Ttran)
            g0 = self.ptrace(Sphi, self.phi)
            step1 = (ne0 - electrons) / g0
            step = 0.1
            if abs(ne0 - electrons) < 1.0e-9:
                self.msum(1.0, self.L, step1, Sphi)
                done = True
            else:
                step = step1
                self.msum(1.0, self.L, step1, Sphi)
                electrons2, _ = self.lnv(dophi=True, phi=phi2)
                self.TMT(phi2, Sphi2, TL, self.Ttran)
                g1 = self.ptrace(self.phi, Sphi2)
                D = electrons - ne0
                C = g0
                B = 3.0 * (electrons2 - electrons) / (step * step) - (g1 + 2.0 * g0) / step
                recA = (step * step * step) / (2.0 * (electrons - electrons2) + (g0 + g1) * step)
                B = B * recA
                C = C * recA
                D = D * recA
                truestep = self.solve_cubic(B, C, D, step)
                self.msum(1.0, self.L, truestep - step, Sphi)
                if truestep == step:
                    electrons2, _ = self.lnv(dophi=True, phi=self.phi)
                    dne = abs(electrons2 - ne0)
                    if dne < 1e-4:
                        done = True
                    it += 1
                else:
                    done = True
                    self.lnv(dophi=True, phi=self.phi)

    def line_min_L(self, M3, D, mat_temp, SM3, energy_in):
        sf = self.spin_factor
        M3old = self.copy(M3)
        g0 = sf * self.ptrace(D, M3)
        ig0 = sf * self.ptrace(D, M3)
        energy_0 = energy_in
        step = self.delta_e / g0
        if abs(step) < 1.0e-2:
            step = 0.01
        if abs(step) > 0.1:
            step = 0.1
        self.msum(1.0, self.L, step, D)
        _, e1 = self.lnv(doK=True, doM3=True, doE=True, M3=M3)
        energy_1 = sf * e1
        g1 = sf * self.ptrace(D, M3)
        igcross = sf * self.ptrace(SM3, M3)
        self.TMT(M3, SM3, mat_temp, self.T)
        ig1 = sf * self.ptrace(SM3, M3)
        ig1_step = ig1
        Dq = energy_0
        C = g0
        B = 3.0 * (energy_1 - Dq) / (step * step) - (g1 - 2.0 * C) / step
        A = (g1 - 2.0 * B * step - C) / (3.0 * step * step)
        SQ = 4.0 * B * B - 12.0 * A * C
        if SQ < 0:
            return True, energy_in, 0.0
        if abs(A) > RD_ERR:
            truestep = (-2.0 * B + math.sqrt(SQ)) / (6.0 * A)
        else:
            truestep = -C / (2.0 * B)
        if truestep < 1.0e-04:
            truestep = 1.0e-04
        self.msum(1.0, self.L, truestep - step, D)
        self.symmetrise_L()
        _, e2 = self.lnv(doK=True, doM3=True, doE=True, M3=M3)
        energy_out = sf * e2
        self.delta_e = energy_out - energy_in
        if truestep < step:
            lamG = truestep / step
            interpG = ig0 * (1 - lamG) * (1 - lamG) + ig1 * lamG * lamG + 2.0 * igcross * lamG * (1 - lamG)
            zeta = (interpG - ig1) / (ig0 - ig1)
        else:
            self.TMT(M3, SM3, mat_temp, self.T)
            ig1 = sf * self.ptrace(SM3, M3)
            igcross = sf * self.ptrace(SM3, M3old)
            lamG = step / truestep
            interpG = ig0 * (1 - lamG) * (1 - lamG) + ig1 * lamG * lamG + 2.0 * igcross * lamG * (1 - lamG)
            zeta = (interpG - ig1_step) / (ig0 - ig1_step)
        return False, energy_out, zeta

    def _project_search(self, mat_search, SM3, Sphi, mat_temp):
        """earlyDM electron-number projection of the search direction (DMMinModule.f90:456-512)."""
        self.TMT(self.phi, Sphi, mat_temp, self.T)
        e_dot_n = self.ptrace(SM3, self.phi)
        n_dot_n = self.ptrace(Sphi, self.phi)
        if abs(n_dot_n) > RD_ERR:
            self.msum(1.0, mat_search, e_dot_n / n_dot_n, Sphi)

    def early_dm(self, ndone):
        p = self.p
        sf = self.spin_factor
        M3 = self.temp("L"); SM3 = self.temp("L"); Sphi = self.temp("L")
        mat_temp = self.temp("TL"); mat_search = self.temp("L")
        if p.vary_mu:
            self.correct_electron_number()
        electrons, e0 = self.lnv(doM3=True, dophi=True, doE=True, M3=M3, phi=self.phi)
        energy0 = sf * e0
        self.TMT(M3, SM3, mat_temp, self.T)
        self.msum(0.0, mat_search, -1.0, SM3)
        if p.vary_mu:
            self._project_search(mat_search, SM3, Sphi, mat_temp)
        self.delta_e = 0.0
        for n_iter in range(1, p.n_L_iterations + 1):
            g0 = self.gsum_norm(M3, SM3)
            inflex, energy1, interpG = self.line_min_L(M3, mat_search, mat_temp, SM3, energy0)
            if inflex:
                self.log.append(("earlyDM-inflex", n_iter))
                return n_iter, False, True
            self.TMT(M3, SM3, mat_temp, self.T)
            zeta = interpG
            if p.vary_mu:
                self.correct_electron_number()
            electrons, e1 = self.lnv(doM3=True, dophi=True, doE=True, M3=M3, phi=self.phi)
            energy1 = sf * e1
            self.TMT(M3, SM3, mat_temp, self.T)
            energy0 = energy1
            self.msum(0.0, mat_search, -1.0, SM3)
            if p.vary_mu:
                self._project_search(mat_search, SM3, Sphi, mat_temp)
            g0 = self.gsum_norm(M3, SM3)
            self.log.append(("earlyDM", n_iter, energy0, g0, zeta))
            if abs(zeta) < p.lintol:
                return n_iter, False, False
        return ndone, False, False   # loop exhausted: ndone is left unchanged (DMMinModule.f90:712-722)

    def _late_project(self, M3, SM3, Sphi, mat_temp):
        self.TMT(self.phi, Sphi, mat_temp, self.T)
        e_dot_n = self.ptrace(SM3, self.phi)
        n_dot_n = self.ptrace(Sphi, self.phi)
        e_tot = self.spin_factor * e_dot_n
        n_tot = self.spin_factor * n_dot_n
        if abs(n_tot) > RD_ERR:
            f = e_tot / n_tot
            self.msum(1.0, SM3, -f, Sphi)
            self.msum(1.0, M3, -f, self.phi)

    def late_dm(self, ndone, deltaE):
        p = self.p
        sf = self.spin_factor
        npul = p.maxpulay
        Lst = [self.temp("L") for _ in range(npul)]
        Gst = [self.temp("L") for _ in range(npul)]
        SGst = [self.temp("L") for _ in range(npul)]
        M3 = self.temp("L"); SM3 = self.temp("L"); Sphi = self.temp("L"); mat_temp = self.temp("TL")
        iter_stuck = 0
        if self.h_rebuild is not None:
            self.rebuild_H()
        electrons, e0 = self.lnv(doM3=True, dophi=True, doE=True, M3=M3, phi=self.phi)
        energy0 = sf * e0
        self.TMT(M3, SM3, mat_temp, self.T)
        if p.vary_mu:
            # preliminaries use the per-spin ratio (nspin == 1 branch, DMMinModule.f90:949-966)
            self.TMT(self.phi, Sphi, mat_temp, self.T)
            e_dot_n = self.ptrace(SM3, self.phi)
            n_dot_n = self.ptrace(Sphi, self.phi)
            if abs(n_dot_n) > RD_ERR:
                f = e_dot_n / n_dot_n
                self.msum(1.0, SM3, -f, Sphi)
                self.msum(1.0, M3, -f, self.phi)
        self.msum(0.0, SGst[0], -1.0, SM3)
        self.msum(0.0, Gst[0], -1.0, M3)
        self.msum(0.0, Lst[0], 1.0, self.L)
        g0 = self.gsum_norm(M3, SM3)
        done = p.n_L_iterations == 0
        for n_iter in range(1, p.n_L_iterations + 1):
            npmod = (n_iter % npul) + 1
            pul_mx = min(n_iter + 1, npul)
            if p.global_tolerance:
                step = deltaE / (g0 + RD_ERR)
            else:
                step = deltaE / (float(self.ni_in_cell) * g0 + RD_ERR)
            step = abs(step)
            if abs(step) < p.minpulaystep:
                step = p.minpulaystep
            if abs(step) > p.maxpulaystep:
                step = p.maxpulaystep
            src = npmod - 1 if npmod > 1 else pul_mx
            self.msum(0.0, self.L, 1.0, Lst[src - 1])
            self.msum(1.0, self.L, step, SGst[src - 1])
            if p.vary_mu:
                self.correct_electron_number()
            electrons, e1 = self.lnv(doM3=True, dophi=True, doE=True, M3=M3, phi=self.phi)
            energy1 = sf * e1
            self.TMT(M3, SM3, mat_temp, self.T)
            if p.vary_mu:
                self._late_project(M3, SM3, Sphi, mat_temp)
            self.msum(0.0, SGst[npmod - 1], -1.0, SM3)
            self.msum(0.0, Gst[npmod - 1], -1.0, M3)
            self.msum(0.0, Lst[npmod - 1], 1.0, self.L)
            Aij = np.zeros((npul, npul))
            for i in range(pul_mx):
                for j in range(pul_mx):
                    Aij[j, i] = sf * self.ptrace(Gst[j], SGst[i])
            alph = self.do_pulay(npmod, Aij, pul_mx, npul)
            self.scale(0.0, self.L)
            for i in range(pul_mx):
                self.msum(1.0, self.L, alph[i], Lst[i])
            if p.vary_mu:
                self.correct_electron_number()
            if self.h_rebuild is not None:
                self.rebuild_H()
            electrons, e1 = self.lnv(doM3=True, dophi=True, doE=True, M3=M3, phi=self.phi)
            energy1 = sf * e1
            self.TMT(M3, SM3, mat_temp, self.T)
            if p.vary_mu:
                self._late_project(M3, SM3, Sphi, mat_temp)
            deltaE = energy1 - energy0
            g1 = self.gsum_norm(M3, SM3)
            self.log.append(("lateDM", n_iter, energy1, g1))
            if g1 < p.tolerance:
                return n_iter, True, deltaE
            elif self.h_rebuild is None and g1 > 2.0 * g0:     # off with the H coupling (1261)
                return n_iter, False, deltaE
            elif g1 > 0.99 * g0:
                iter_stuck += 1
                if iter_stuck > 5:
                    return n_iter, False, deltaE
            self.msum(0.0, SGst[npmod - 1], -1.0, SM3)
            self.msum(0.0, Gst[npmod - 1], -1.0, M3)
            self.msum(0.0, Lst[npmod - 1], 1.0, self.L)
            g0 = g1
            energy0 = energy1
        return p.n_L_iterations, done, deltaE

    def rebuild_H(self):
        """Mixed-L self-consistency step (DMMinModule.f90:894-907, 1138-1149): K and E of the
        current L (LNV_matrix_multiply with doK, doE), then H from the density of K."""
        self.lnv(doK=True, doE=True)
        self.h_rebuilds += 1
        self.H.v[:] = np.asarray(self.h_rebuild(self.K.v.copy()), dtype=np.float64)

    @staticmethod
    def do_pulay(iPulay, Aij_in, n, max_n, use_lapack=False):
        """DoPulay2D_nospin (Pulay.f90:188-262): alphas from the inverse of the residual overlap.

        The inverse follows LAPACK's unblocked Bunch-Kaufman path (dsytrf falls back to dsytf2 for
        n <= 5, then dsytri, upper triangle) written out below; use_lapack=True calls scipy's LAPACK.
        """
        invertible = True
        if n == 1:
            A = np.array([[1.0 / Aij_in[0, 0]]])
        elif use_lapack:
            A = np.array(Aij_in[:n, :n], dtype=np.float64, order="F")
            lu, ipiv, info = lapack.dsytrf(A, lower=0)
            inv, info2 = lapack.dsytri(lu, ipiv, lower=0)
            if info2 != 0:
                invertible = False
            else:
                A = np.triu(inv) + np.triu(inv, 1).T
        else:
            A = bk_inverse([[float(Aij_in[i, j]) for j in range(n)] for i in range(n)])
            if A is None:
                invertible = False
            else:
                A = np.array(A)
        al = np.zeros(max_n)
        if invertible:
            s = 0.0
            for i in range(n):
                for j in range(n):
                    al[i] += A[j, i]
                    s += A[j, i]
            al[:n] /= s
        else:
            al[iPulay - 1] = 1.0
        return al

    def find_min_dm(self, resetL=True, max_outer=40):
        """FindMinDM (DMMinModule.f90:172-312); returns (band energy, electrons) of the final L.

        The reference loops until done; after max_outer passes the loop stops and self.converged
        stays False (a residual stalled above the tolerance), as the library's solver does."""
        p = self.p
        problem = inflex = done = False
        early = True
        self.transpose(self.T, self.Ttran)
        ndone = 0
        niter = 0
        outer = 0
        while not done:
            outer += 1
            if outer > max_outer:
                break
            if resetL or inflex:
                self.init_mcw()
                self.delta_e = self.mcw_min(p.n_L_iterations)
                early = True
                resetL = False
            if early or problem:
                inflex = False
                ndone, done, inflex = self.early_dm(ndone)
            if not done and not inflex:
                ndone, done, self.delta_e = self.late_dm(ndone, self.delta_e)
            niter += 1
            if problem:
                resetL = True
            if niter > 10:
                problem = True
                niter = 0
        self.converged = done
        electrons, energy = self.lnv(doK=True, dophi=True, doE=True, phi=self.phi)
        return self.spin_factor * energy, self.spin_factor * electrons
