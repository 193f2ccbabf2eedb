"""2D SBP-SAT operators assembled as sparse matrices (oracle; test infrastructure only).

Restates the matrix construction of source/sbpOps_m_constGrid.cpp and
source/sbpOps_m_varGrid.cpp (constructors, computeMatrices, constructA,
constructD2, constructDyymu/Dzzmu, constructRymu/Rzmu including the
flattened-index ``mu3`` averages, constructBC_Dirichlet/Neumann and
constructBCMats).  Body vectors use the reference layout: flattened index
``Ii = iy*Nz + iz`` (source/domain.cpp:380-381), z fastest.
"""
import numpy as np
import scipy.sparse as sp

from .sbp1d import sbp_spmat, sbp_spmat2, sbp_spmat4


def _csr(a):
    return sp.csr_matrix(a)


def _diag(v):
    return sp.diags(np.asarray(v, dtype=np.float64), 0, format="csr")


def mu3_y(vec):
    """Averaged coefficient used by the order-4 Rymu term.

    sbpOps_m_constGrid.cpp:1238-1257 / sbpOps_m_varGrid.cpp:1410-1431: the
    average is taken in the *flattened* index, so for y it mixes the z
    neighbour (and at iz = Nz-1 the next y-column).
    """
    v = np.asarray(vec, dtype=np.float64)
    n = v.size
    m = v.copy()
    m[n - 1] += v[n - 2]
    m[0:n - 1] += v[1:n]
    return 0.5 * m


def mu3_z(vec):
    """Averaged coefficient used by the order-4 Rzmu term.

    sbpOps_m_constGrid.cpp:1087-1112 / sbpOps_m_varGrid.cpp:1262-1286.
    """
    v = np.asarray(vec, dtype=np.float64)
    n = v.size
    m = v.copy()
    m[0] += v[1]
    m[n - 1] += v[n - 2]
    m[0:n - 2] += v[1:n - 1]
    return 0.5 * m


class SbpOps:
    """Assembled SBP-SAT operator for one body grid.

    Parameters mirror the reference constructors
    ``SbpOps_m_constGrid(order, Ny, Nz, Ly, Lz, mu)`` and
    ``SbpOps_m_varGrid(order, Ny, Nz, Ly, Lz, mu)`` + ``setGrid(y, z)``,
    ``setCompatibilityType``, ``setBCTypes``, ``setMultiplyByH``.
    The Laplace type is always "yz" (the only one LinearElastic uses,
    linearElastic.cpp:445).
    """

    def __init__(self, order, Ny, Nz, Ly, Lz, mu, grid="constantGridSpacing",
                 y=None, z=None, compat="fullyCompatible",
                 bcs=("Dirichlet", "Neumann", "Dirichlet", "Neumann"), multByH=1, laplace="yz"):
        assert order in (2, 4)
        self.order, self.Ny, self.Nz = order, Ny, Nz
        self.N = Ny * Nz
        self.Ly, self.Lz = Ly, Lz
        self.grid = grid
        self.compat = compat
        self.multByH = multByH
        # setLaplaceType (constGrid.cpp:159-164): "yz", "y" or "z" selects the
        # parts of D2, the SAT terms in A and the sides setRhs uses (:621-690, :886-905)
        assert laplace in ("yz", "y", "z")
        self.laplace = laplace
        self.mu_vec = np.asarray(mu, dtype=np.float64).copy()
        assert self.mu_vec.size == self.N
        if grid == "constantGridSpacing":
            # sbpOps_m_constGrid.cpp:9-50
            self.dy = Ly / (Ny - 1.0) if Ny > 1 else Ly
            self.dz = Lz / (Nz - 1.0) if Nz > 1 else Lz
        else:
            # sbpOps_m_varGrid.cpp:5-45 (logical spacing)
            self.dy = 1.0 / (Ny - 1.0) if Ny > 1 else 1.0
            self.dz = 1.0 / (Nz - 1.0) if Nz > 1 else 1.0
        if order == 2:
            self.alphaDy = -4.0 / self.dy
            self.alphaDz = -4.0 / self.dz
        else:
            self.alphaDy = 2.0 * -48.0 / 17.0 / self.dy
            self.alphaDz = 2.0 * -48.0 / 17.0 / self.dz
        self.alphaT = -1.0
        self._y = None if y is None else np.asarray(y, dtype=np.float64)
        self._z = None if z is None else np.asarray(z, dtype=np.float64)
        self.bcR, self.bcT, self.bcL, self.bcB = bcs
        self._build()

    # ------------------------------------------------------------------
    def _build(self):
        Ny, Nz = self.Ny, self.Nz
        o1y = sbp_spmat(self.order, Ny, 1.0 / self.dy, self.compat)
        o1z = sbp_spmat(self.order, Nz, 1.0 / self.dz, self.compat)
        self.o1y, self.o1z = o1y, o1z
        Iy = sp.identity(Ny, format="csr"); Iz = sp.identity(Nz, format="csr")
        kr = lambda a, b: sp.kron(_csr(a) if not sp.issparse(a) else a,
                                  _csr(b) if not sp.issparse(b) else b, format="csr")
        self.Hy_Iz = kr(o1y["H"], Iz); self.Iy_Hz = kr(Iy, o1z["H"])
        self.H = (self.Hy_Iz @ self.Iy_Hz).tocsr()
        self.Hyinv_Iz = kr(o1y["Hinv"], Iz); self.Iy_Hzinv = kr(Iy, o1z["Hinv"])
        self.Hinv = (self.Hyinv_Iz @ self.Iy_Hzinv).tocsr()
        E0y = np.zeros((Ny, Ny)); ENy = np.zeros((Ny, Ny))
        E0z = np.zeros((Nz, Nz)); ENz = np.zeros((Nz, Nz))
        e0y = np.zeros((Ny, 1)); eNy = np.zeros((Ny, 1)); e0z = np.zeros((Nz, 1)); eNz = np.zeros((Nz, 1))
        if Ny > 1:
            E0y[0, 0] = 1; ENy[Ny - 1, Ny - 1] = 1; e0y[0, 0] = 1; eNy[Ny - 1, 0] = 1
        if Nz > 1:
            E0z[0, 0] = 1; ENz[Nz - 1, Nz - 1] = 1; e0z[0, 0] = 1; eNz[Nz - 1, 0] = 1
        self.E0y_Iz = kr(E0y, Iz); self.ENy_Iz = kr(ENy, Iz)
        self.Iy_E0z = kr(Iy, E0z); self.Iy_ENz = kr(Iy, ENz)
        self.e0y_Iz = kr(e0y, Iz); self.eNy_Iz = kr(eNy, Iz)
        self.Iy_e0z = kr(Iy, e0z); self.Iy_eNz = kr(Iy, eNz)
        self.mu = _diag(self.mu_vec)
        N = self.N
        if self.grid == "constantGridSpacing":
            # sbpOps_m_constGrid.cpp:261-286, 1402-1419
            self.Dy_Iz = kr(o1y["D1"], Iz)
            self.Iy_Dz = kr(Iy, o1z["D1"])
            self.yq = _diag(np.ones(N)); self.zr = _diag(np.ones(N))
            self.qy = _diag(np.ones(N)); self.rz = _diag(np.ones(N))
            self.muqy = self.mu; self.murz = self.mu
            self.Dq_Iz = self.Dy_Iz; self.Iy_Dr = self.Iy_Dz
            Ly_fac = None
        else:
            # sbpOps_m_varGrid.cpp:333-436
            self.Dq_Iz = kr(o1y["D1"], Iz)
            self.Iy_Dr = kr(Iy, o1z["D1"])
            yq = np.ones(N) if (self._y is None or Ny == 1) else self.Dq_Iz @ self._y
            zr = np.ones(N) if (self._z is None or Nz == 1) else self.Iy_Dr @ self._z
            self.yq_vec, self.zr_vec = yq, zr
            self.yq = _diag(yq); self.qy = _diag(1.0 / yq)
            self.zr = _diag(zr); self.rz = _diag(1.0 / zr)
            self.muqy = (self.mu @ self.qy).tocsr()
            self.murz = (self.mu @ self.rz).tocsr()
            self.Dy_Iz = (self.qy @ self.Dq_Iz).tocsr()
            self.Iy_Dz = (self.rz @ self.Iy_Dr).tocsr()
        BSy_Iz = kr(o1y["BS"], Iz); Iy_BSz = kr(Iy, o1z["BS"])
        self.muxBySy_IzT = (BSy_Iz.T @ self.muqy).tocsr()
        self.Iy_muxBzSzT = (Iy_BSz.T @ self.murz).tocsr()
        if self.laplace == "yz":
            self.D2 = (self._dyymu() + self._dzzmu()).tocsr()
        elif self.laplace == "y":
            self.D2 = self._dyymu().tocsr()
        else:
            self.D2 = self._dzzmu().tocsr()
        self._build_bc()

    # ------------------------------------------------------------------
    def _rmu(self, direction):
        """Rymu / Rzmu (constGrid.cpp:1023-1315, varGrid.cpp:1209-1504)."""
        Ny, Nz = self.Ny, self.Nz
        var = self.grid != "constantGridSpacing"
        if direction == "y":
            n, h = Ny, self.dy
            coef_mat = self.muqy
            coef_vec = self.muqy.diagonal()
            kr = lambda a: sp.kron(_csr(a), sp.identity(Nz, format="csr"), format="csr")
            mu3f = mu3_y
        else:
            n, h = Nz, self.dz
            coef_mat = self.murz
            coef_vec = self.murz.diagonal()
            kr = lambda a: sp.kron(sp.identity(Ny, format="csr"), _csr(a), format="csr")
            mu3f = mu3_z
        if n == 1:
            return sp.csr_matrix((self.N, self.N))
        if self.order == 2:
            D2, C2 = sbp_spmat2(n, 1.0 / h)
            D2k = kr(D2); C2k = kr(C2)
            R = (D2k.T @ C2k @ coef_mat @ D2k) * (0.25 * h ** 3)
            return R.tocsr()
        D3, D4, C3, C4 = sbp_spmat4(n, 1.0 / h)
        mu3 = _diag(mu3f(coef_vec))
        D3k = kr(D3); C3k = kr(C3); D4k = kr(D4); C4k = kr(C4)
        t2 = (D3k.T @ C3k) @ mu3 @ D3k * (1.0 / h / 18.0)
        R = (D4k.T @ C4k) @ coef_mat @ D4k * (1.0 / h / 144.0)
        return (R + t2).tocsr()

    def _dyymu(self):
        Rymu = self._rmu("y")
        if self.grid == "constantGridSpacing":
            # constGrid.cpp:963-991
            D = self.Dy_Iz @ self.mu @ self.Dy_Iz - self.Hyinv_Iz @ Rymu
            if self.multByH:
                D = self.H @ D
            return D
        # varGrid.cpp:1133-1171
        D = self.Dq_Iz @ self.muqy @ self.Dq_Iz - self.Hyinv_Iz @ Rymu
        D = (self.H @ self.zr @ D) if self.multByH else (self.zr @ D)
        return D

    def _dzzmu(self):
        Rzmu = self._rmu("z")
        if self.grid == "constantGridSpacing":
            D = self.Iy_Dz @ self.mu @ self.Iy_Dz - self.Iy_Hzinv @ Rzmu
            if self.multByH:
                D = self.H @ D
            return D
        D = self.Iy_Dr @ self.murz @ self.Iy_Dr - self.Iy_Hzinv @ Rzmu
        D = (self.H @ self.yq @ D) if self.multByH else (self.yq @ D)
        return D

    # ------------------------------------------------------------------
    def _bc_dirichlet(self, alphaD, L, mu, Hinv, BD1T, E):
        # constGrid.cpp:504-535 (L = I) / varGrid.cpp:667-695
        LHHinv = (self.H @ L @ Hinv) if self.multByH else (L @ Hinv)
        return (LHHinv @ BD1T @ E + alphaD * (LHHinv @ mu @ E)).tocsr()

    def _bc_neumann_A(self, L, Hinv, Bfact, E, mu, D1):
        # constGrid.cpp:438-471 / varGrid.cpp:607-633
        M = L @ Hinv @ E @ mu
        out = (self.H @ M @ D1) if self.multByH else (M @ D1)
        return (Bfact * self.alphaT * out).tocsr()

    def _bc_neumann_rhs(self, L, Hinv, Bfact, e):
        # constGrid.cpp:475-497 / varGrid.cpp:638-662
        out = (self.H @ L @ Hinv @ e) if self.multByH else (L @ Hinv @ e)
        return (Bfact * self.alphaT * out).tocsr()

    def _build_bc(self):
        """constructBCMats (constGrid.cpp:537-603, varGrid.cpp:700-772)."""
        var = self.grid != "constantGridSpacing"
        Ly_ = self.zr if var else _diag(np.ones(self.N))
        Lz_ = self.yq if var else _diag(np.ones(self.N))
        mu_y = self.muqy if var else self.mu
        mu_z = self.murz if var else self.mu
        sides = {
            "R": (self.bcR, self.alphaDy, Ly_, mu_y, self.Hyinv_Iz, self.muxBySy_IzT, self.ENy_Iz, self.eNy_Iz, 1.0, self.Dy_Iz),
            "T": (self.bcT, self.alphaDz, Lz_, mu_z, self.Iy_Hzinv, self.Iy_muxBzSzT, self.Iy_E0z, self.Iy_e0z, -1.0, self.Iy_Dz),
            "L": (self.bcL, self.alphaDy, Ly_, mu_y, self.Hyinv_Iz, self.muxBySy_IzT, self.E0y_Iz, self.e0y_Iz, -1.0, self.Dy_Iz),
            "B": (self.bcB, self.alphaDz, Lz_, mu_z, self.Iy_Hzinv, self.Iy_muxBzSzT, self.Iy_ENz, self.Iy_eNz, 1.0, self.Iy_Dz),
        }
        self.A_side = {}; self.rhs_side = {}
        for s, (typ, alphaD, L, mu_d, Hinv, BD1T, E, e, Bfact, D1) in sides.items():
            if typ == "Dirichlet":
                self.A_side[s] = self._bc_dirichlet(alphaD, L, mu_d, Hinv, BD1T, E)
                self.rhs_side[s] = self._bc_dirichlet(alphaD, L, mu_d, Hinv, BD1T, e)
            elif typ == "Neumann":
                # the Neumann SAT uses plain mu and Dy = qy*Dq (varGrid.cpp:735-741)
                self.A_side[s] = self._bc_neumann_A(L, Hinv, Bfact, E, self.mu, D1)
                self.rhs_side[s] = self._bc_neumann_rhs(L, Hinv, Bfact, e)
            else:
                raise ValueError(typ)
        used = {"yz": "LRTB", "y": "LR", "z": "TB"}[self.laplace]
        self.A = self.D2.copy()
        for side in used:
            self.A = self.A + self.A_side[side]
        self.A = self.A.tocsr()

    # ------------------------------------------------------------------
    def change_bc_types(self, bcR, bcT, bcL, bcB):
        """changeBCTypes (constGrid.cpp:163-195)."""
        self.bcR, self.bcT, self.bcL, self.bcB = bcR, bcT, bcL, bcB
        self._build_bc()

    def set_rhs(self, bcL, bcR, bcT, bcB):
        """setRhs (constGrid.cpp:877-914)."""
        out = np.zeros(self.N)
        used = {"yz": "LRTB", "y": "LR", "z": "TB"}[self.laplace]
        for side, v in (("L", bcL), ("R", bcR), ("T", bcT), ("B", bcB)):
            if side in used:
                out = out + self.rhs_side[side] @ v
        return out

    def Dy(self, u):
        return self.Dy_Iz @ u

    def Dz(self, u):
        return self.Iy_Dz @ u

    def muxDy(self, u):
        """mu * Dy * u (constGrid.cpp:1466-1478)."""
        return self.mu_vec * (self.Dy_Iz @ u)

    def muxDz(self, u):
        return self.mu_vec * (self.Iy_Dz @ u)

    def Hx(self, u):
        return self.H @ u

    def Hinvx(self, u):
        return self.Hinv @ u
