"""Rate-and-state fault: root find and state laws (oracle; test infrastructure only).

Restates source/fault.cpp (Fault_qd::computeVel :812-857, Fault_qd::d_dt
:861-918, ComputeVel_qd :954-1059, agingLaw_psi :1984-1994, slipLaw_psi
:2072-2088, strength_psi :2247-2251) and BracketedNewton::findRoot
(source/rootFinder.cpp:168-266), and the fully dynamic fault (Fault_fd
:1065-1575, ComputeVel_fd :1588-1685, ComputeAging_fd / ComputeSlipLaw_fd
:1690-1879).  The per-node Newton iteration is vectorised across nodes with
masks; each node follows exactly the scalar control flow of the reference.
"""
import numpy as np


def strength_psi(sN, psi, V, a, v0):
    """fault.cpp:2247-2251."""
    return a * sN * np.arcsinh((0.5 * V / v0) * np.exp(psi / a))


def resid_qd(V, tauQS, eta, sN, psi, a, v0):
    """ComputeVel_qd::getResid with Jacobian (fault.cpp:1037-1059).

    The returned derivative reproduces the reference's expression
    ``a*sN*V/sqrt(B^2 V^2 + 1) + eta`` (B = exp(psi/a)/(2 v0)); the exact
    derivative would have B in place of V in the numerator.  It only steers
    the Newton/bisection choice, not the converged root.
    """
    strength = strength_psi(sN, psi, V, a, v0)
    f = strength - (tauQS - eta * V)
    A = a * sN
    B = np.exp(psi / a) / (2.0 * v0)
    J = A * V / np.sqrt(B * B * V * V + 1.0) + eta
    return f, J


def known_answer_resid(val):
    """TestRoots::getResid (rootFinder.cpp:12-24), the reference's known-answer residual."""
    tauQS = 0.75 * (3.000075e+01 - 9.999920e-06)
    return 0.015 * 50 * np.arcsinh((val / 2.0 / 1e-6) * np.exp(0.6 / 0.015)) + 0.5 * 12 * val - tauQS


def bracketed_newton(resid, left, right, x0, atol, max_its):
    """Vectorised BracketedNewton::findRoot (rootFinder.cpp:174-257).

    ``resid(x, idx)`` returns (f, f') at the nodes ``idx``.  The reference's
    first residual check reads an uninitialised member (rootFinder.cpp:182);
    the restatement evaluates it at x0, which returns the same root.
    Returns (x, its, converged).
    """
    left = np.array(left, dtype=np.float64, copy=True)
    right = np.array(right, dtype=np.float64, copy=True)
    x = np.array(x0, dtype=np.float64, copy=True)
    n = x.size
    idx_all = np.arange(n)
    out = x.copy()
    its = np.zeros(n, dtype=np.int64)
    done = np.zeros(n, dtype=bool)
    f0, _ = resid(x, idx_all)
    done |= np.abs(f0) <= atol
    fl, _ = resid(left, idx_all)
    fr, _ = resid(right, idx_all)
    m = (~done) & (np.sqrt(fl * fl) <= atol)
    out[m] = left[m]; done |= m
    m = (~done) & (np.sqrt(fr * fr) <= atol)
    out[m] = right[m]; done |= m
    swap = (~done) & (fl > 0)
    left[swap], right[swap] = right[swap].copy(), left[swap].copy()
    dxold = np.abs(right - left)
    dx = dxold.copy()
    f, fp = resid(x, idx_all)
    active = (~done) & (np.abs(f) >= atol)
    while True:
        active &= (its <= max_its) & (np.abs(f) >= atol)
        if not active.any():
            break
        i = np.nonzero(active)[0]
        xi, fi, fpi = x[i], f[i], fp[i]
        li, ri = left[i], right[i]
        bis = (((xi - ri) * fpi - fi) * ((xi - li) * fpi - fi) > 0.0) | (np.abs(2.0 * fi) > np.abs(dxold[i] * fpi))
        newdx = np.where(bis, 0.5 * (ri - li), fi / fpi)
        dxold[i] = dx[i]
        dx[i] = newdx
        x[i] = np.where(bis, li + newdx, xi - newdx)
        fn, fpn = resid(x[i], i)
        f[i] = fn; fp[i] = fpn
        neg = fn < 0.0
        left[i] = np.where(neg, x[i], li)
        right[i] = np.where(neg, ri, x[i])
        its[i] += 1
    conv = np.abs(f) <= atol
    out[~done] = x[~done]
    converged = done | conv
    return out, its, converged


def compute_vel_qd(Vprev, tauQS, eta, sN, psi, a, locked, v0, vL, root_tol=1e-12, max_its=10000):
    """ComputeVel_qd::computeVel (fault.cpp:961-1015).  Returns (V, total root iterations, all converged)."""
    V = np.array(Vprev, dtype=np.float64, copy=True)
    locked = np.asarray(locked, dtype=np.float64)
    lk = locked > 0.5
    ck = locked < -0.5
    V[lk] = 0.0
    V[ck] = vL
    free = np.nonzero(~(lk | ck))[0]
    if free.size == 0:
        return V, 0, True
    right = tauQS[free] / eta[free]
    left = np.zeros_like(right)
    if np.isnan(right).any():
        raise FloatingPointError("NaN root bound")
    out = V[free].copy()
    deg = np.abs(left - right) < 1e-14
    out[deg] = left[deg]
    nd = np.nonzero(~deg)[0]
    conv = True
    its_total = 0
    if nd.size:
        sel = free[nd]

        def resid(x, idx):
            j = sel[idx]
            return resid_qd(x, tauQS[j], eta[j], sN[j], psi[j], a[j], v0)

        x, its, c = bracketed_newton(resid, left[nd], right[nd], V[sel], root_tol, max_its)
        out[nd] = x
        conv = bool(c.all())
        its_total = int(its.sum())
    V[free] = out
    return V, its_total, conv


def aging_law_psi(psi, V, b, f0, v0, Dc):
    """fault.cpp:1984-1994 (zero when b <= 1e-3 or the exponential overflows)."""
    with np.errstate(over="ignore"):
        A = np.exp((f0 - psi) / b)
    ok = (~np.isinf(A)) & (b > 1e-3)
    return np.where(ok, (b * v0 / Dc) * (A - V / v0), 0.0)


def slip_law_psi(psi, V, a, b, f0, v0, Dc):
    """fault.cpp:2072-2088 (zero where V == 0)."""
    absV = np.abs(V)
    with np.errstate(divide="ignore", invalid="ignore"):
        fss = f0 + (a - b) * np.log(absV / v0)
        f = a * np.arcsinh((absV / 2.0 / v0) * np.exp(psi / a))
        d = -absV / Dc * (f - fss)
    return np.where(V == 0, 0.0, d)


def flash_heating_vw(T, rho, c, k, D, Tw, tau_c):
    """flashHeating_Vw (fault.cpp:2162-2168): weakening velocity."""
    rc = rho * c
    ath = k / rc
    return (np.pi * ath / D) * np.power(rc * (Tw - T) / tau_c, 2.0)


def flash_heating_psi(psi, V, Vw, fw, Dc, a, b, f0, v0):
    """flashHeating_psi (fault.cpp:2171-2196): the regularised steady-state
    friction fLV, weakened to fw + (fLV - fw) Vw / |V| above Vw."""
    absV = np.abs(V)
    fLV = (a - b) * np.arcsinh(absV / v0 / 2.0 * np.exp(f0 / (a - b)))
    with np.errstate(divide="ignore", invalid="ignore"):
        fss = np.where(absV > Vw, fw + (fLV - fw) * (Vw / absV), fLV)
    f = a * np.arcsinh((absV / 2.0 / v0) * np.exp(psi / a))
    return -absV / Dc * (f - fss)


class FaultQD:
    """Fault_qd state (fault.hpp:138-160) with the fields d_dt touches."""

    def __init__(self, z, a, b, sN, Dc, psi, mu, rho, locked=None, prestress=None,
                 f0=0.6, v0=1e-6, vL=1e-9, state_law="agingLaw", fault_type_scale=2.0,
                 root_tol=1e-12, max_its=10000):
        n = len(z)
        self.z = np.asarray(z, float)
        self.a = np.asarray(a, float); self.b = np.asarray(b, float)
        self.sN = np.asarray(sN, float); self.Dc = np.asarray(Dc, float)
        self.psi = np.asarray(psi, float).copy()
        self.slip = np.zeros(n)
        self.slipVel = np.zeros(n)
        self.locked = np.zeros(n) if locked is None else np.asarray(locked, float)
        self.prestress = np.zeros(n) if prestress is None else np.asarray(prestress, float)
        self.tauQSP = np.zeros(n); self.tauP = np.zeros(n); self.strength = np.zeros(n)
        self.f0, self.v0, self.vL = f0, v0, vL
        self.state_law = state_law
        # eta_rad = sqrt(mu*rho)/faultTypeScale (fault.cpp:732-737)
        self.eta = np.sqrt(np.abs(np.asarray(mu, float) * np.asarray(rho, float))) / fault_type_scale
        self.root_tol, self.max_its = root_tol, max_its
        self.root_its = 0

    def update_fields(self, var):
        """Fault_qd::updateFields (fault.cpp:791-807)."""
        self.psi = var["psi"].copy()
        self.slip = var["slip"].copy()

    def d_dt(self, tauQS_from_body):
        """Fault_qd::d_dt (fault.cpp:861-918).  Returns (dslip, dpsi)."""
        self.tauQSP = tauQS_from_body + self.prestress
        V, its, conv = compute_vel_qd(self.slipVel, self.tauQSP, self.eta, self.sN, self.psi, self.a,
                                      self.locked, self.v0, self.vL, self.root_tol, self.max_its)
        if not conv:
            raise FloatingPointError("rootFinder BracketedNewton did not converge")
        self.root_its += its
        self.slipVel = V
        if self.state_law == "agingLaw":
            dpsi = aging_law_psi(self.psi, V, self.b, self.f0, self.v0, self.Dc)
        elif self.state_law == "slipLaw":
            dpsi = slip_law_psi(self.psi, V, self.a, self.b, self.f0, self.v0, self.Dc)
        elif self.state_law == "constantState":
            dpsi = np.zeros_like(V)
        elif self.state_law == "flashHeating":
            # flashHeating_psi_Vec (fault.cpp:2199-2243) with the fault's
            # temperature, density and the heat equation's c, k
            fh = self.flash
            self.Vw = flash_heating_vw(fh["T"], fh["rho"], fh["c"], fh["k"], fh["D"], fh["Tw"], fh["tau_c"])
            dpsi = flash_heating_psi(self.psi, V, self.Vw, fh["fw"], self.Dc, self.a, self.b, self.f0, self.v0)
        else:
            raise ValueError(self.state_law)
        self.tauP = self.tauQSP - self.eta * V
        self.strength = strength_psi(self.sN, self.psi, V, self.a, self.v0)
        return V.copy(), dpsi


# ---------------------------------------------------------------------------
# Fully dynamic fault (Fault_fd, fault.cpp:1065-1575; ComputeVel_fd
# :1588-1685; ComputeAging_fd / ComputeSlipLaw_fd :1690-1879)

def resid_vel_fd(V, Phi, fricPen, sN, psi, a, v0):
    """ComputeVel_fd::getResid with Jacobian (fault.cpp:1649-1685):
    fricPen*strength(V) - (|Phi| - V) and its exact derivative."""
    constraints = fricPen * strength_psi(sN, psi, V, a, v0)
    stress = np.abs(Phi) - V
    f = constraints - stress
    A = a * sN
    B = np.exp(psi / a) / (2.0 * v0)
    J = 1 + fricPen * A * B / np.sqrt(1. + B * B * V * V)
    return f, J


def compute_vel_fd(Vprev, Phi, fricPen, sN, psi, a, locked, v0, vL, root_tol=1e-12, max_its=10000):
    """ComputeVel_fd::computeVel (fault.cpp:1594-1644): |V| from a bracketed
    Newton on [0, |Phi|] started at |V_prev|; locked nodes are held at 0 or vL."""
    V = np.abs(np.array(Vprev, dtype=np.float64, copy=True))
    locked = np.asarray(locked, dtype=np.float64)
    lk = locked > 0.5
    ck = locked < -0.5
    out = V.copy()
    out[lk] = 0.0
    out[ck] = vL
    free = np.nonzero(~(lk | ck))[0]
    its_total, conv = 0, True
    if free.size == 0:
        return out, its_total, conv
    left = np.zeros(free.size)
    right = np.abs(Phi[free])
    deg = np.abs(left - right) < 1e-14
    out[free[deg]] = left[deg]
    nd = np.nonzero(~deg)[0]
    if nd.size:
        sel = free[nd]

        def resid(x, idx):
            j = sel[idx]
            return resid_vel_fd(x, Phi[j], fricPen[j], sN[j], psi[j], a[j], v0)

        x, its, c = bracketed_newton(resid, left[nd], right[nd], V[sel], root_tol, max_its)
        out[sel] = x
        its_total = int(its.sum())
        conv = bool(c.all())
    return out, its_total, conv


def resid_state_fd(law, state, psiPrev, V, a, b, f0, v0, Dc, dt):
    """ComputeAging_fd / ComputeSlipLaw_fd ::getResid with Jacobian
    (fault.cpp:1750-1763, :1851-1865): implicit midpoint about psiPrev,
    -2 dt G((psiPrev + state)/2, V) + (state - psiPrev)."""
    mid = (psiPrev + state) / 2.0
    temp = state - psiPrev
    if law == "agingLaw":
        G = aging_law_psi(mid, V, b, f0, v0, Dc)
        J = 1 + dt * v0 / Dc * np.exp((f0 - (psiPrev + state) / 2.) / b)
    elif law == "slipLaw":
        G = slip_law_psi(mid, V, a, b, f0, v0, Dc)
        A = np.abs(V) / 2. / v0 * np.exp((psiPrev + state) / 2.0 / a)
        J = 1 + dt * np.abs(V) / Dc * A / np.sqrt(1 + A * A)
    else:
        raise ValueError(law)
    return -2 * dt * G + temp, J


def compute_state_fd(law, psi, psiPrev, V, a, b, f0, v0, Dc, dt, root_tol=1e-12, max_its=10000):
    """ComputeAging_fd / ComputeSlipLaw_fd ::computeLaw (fault.cpp:1702-1745,
    :1802-1846): root on [-2, 2] started at psi."""
    n = psi.size
    left = np.full(n, -2.0)
    right = np.full(n, 2.0)

    def resid(x, idx):
        return resid_state_fd(law, x, psiPrev[idx], V[idx], a[idx], b[idx], f0, v0, Dc[idx], dt)

    x, its, c = bracketed_newton(resid, left, right, psi, root_tol, max_its)
    return x, int(its.sum()), bool(c.all())


class FaultFD:
    """Fault_fd::d_dt and setPhi (fault.cpp:1436-1575) on the fields the
    cycle driver keeps.  ``fq`` is the quasi-dynamic fault whose friction
    parameters and eta_rad the fully dynamic fault shares."""

    def __init__(self, fq, rho, alphay, fault_type_scale):
        self.fq = fq
        n = fq.a.size
        self.rho = np.asarray(rho, float)
        self.alphay = np.asarray(alphay, float)
        self.fts = fault_type_scale
        self.psi = fq.psi.copy(); self.slip = np.zeros(n); self.slip0 = np.zeros(n)
        self.slipVel = np.zeros(n); self.tau0 = np.zeros(n)
        self.tauQSP = np.zeros(n); self.tauP = np.zeros(n); self.strength = np.zeros(n)
        self.u = np.zeros(n); self.uPrev = np.zeros(n); self.d2u = np.zeros(n)
        self.an = np.zeros(n); self.Phi = np.zeros(n); self.fricPen = np.zeros(n)
        self.root_its = 0

    def set_phi(self, dt):
        """fault.cpp:1527-1575."""
        self.an = self.d2u + self.tau0 / self.alphay
        self.Phi = 2.0 / dt * (self.u - self.uPrev) + dt * self.an / self.rho
        self.fricPen = dt / self.alphay / self.rho

    def d_dt(self, dt, var, varPrev):
        """fault.cpp:1436-1523.  Returns (psiNext, slipNext); self.u holds the
        fault displacement at the next step."""
        fq = self.fq
        self.psi = var["psi"].copy()
        self.slip = var["slip"].copy()
        self.uPrev = (varPrev["slip"] - self.slip0) * (1.0 / self.fts)
        self.u = (var["slip"] - self.slip0) * (1.0 / self.fts)
        self.set_phi(dt)
        V, its, conv = compute_vel_fd(self.slipVel, self.Phi, self.fricPen, fq.sN, self.psi, fq.a, fq.locked,
                                      fq.v0, fq.vL, fq.root_tol, fq.max_its)
        if not conv:
            raise FloatingPointError("rootFinder BracketedNewton did not converge")
        self.root_its += its
        mv = ~(V < 1e-14)
        fric = strength_psi(fq.sN, self.psi, V, fq.a, fq.v0)
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha = 1.0 / (self.rho * self.alphay) * fric / V
        A = 1.0 + alpha * dt
        Vn = np.where(mv, self.Phi / (1. + dt * alpha), V)
        un = np.where(mv, (2. * self.u + (self.an * dt * dt / self.rho) + (dt * alpha - 1.) * self.uPrev) / A,
                      self.u)
        self.slipVel = Vn
        self.u = un
        psiNext, its, conv = compute_state_fd(fq.state_law, var["psi"], varPrev["psi"], self.slipVel, fq.a, fq.b,
                                              fq.f0, fq.v0, fq.Dc, dt, fq.root_tol, fq.max_its)
        if not conv:
            raise FloatingPointError("rootFinder BracketedNewton did not converge (state)")
        self.psi = psiNext.copy()
        self.slip = self.fts * self.u + self.slip0
        self.strength = strength_psi(fq.sN, self.psi, self.slipVel, fq.a, fq.v0)
        return psiNext, self.slip.copy()
