"""CPU restatement (numpy, FP64) of FlurryPP's explicit FR residual and RK update.

TEST INFRASTRUCTURE ONLY: this module is the checker for the CUDA path.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import it; the product library never calls it.

It restates, array-wise and in the reference's own formulation (dense
operator GEMMs on [point][element][field] arrays), these reference functions:

  solver::update               src/solver.cpp:319-363
  solver::calcResidual         src/solver.cpp:366-445
  solver::extrapolateU         src/solver.cpp:556-572
  solver::calcInviscidFlux_spts src/solver.cpp:707-736, inviscidFlux src/flux.cpp:37-76
  face::calcInviscidFlux       src/face.cpp:163-208 (+ intFace.cpp:114-154)
  face::rusanovFlux            src/face.cpp:314-374
  face::roeFlux                src/face.cpp:376-495
  boundFace::applyBCs          src/boundFace.cpp:65-314
  solver::extrapolateNormalFlux src/solver.cpp:956-1034 (static mesh branch)
  solver::calcDivF_spts        src/solver.cpp:925-954
  solver::correctDivFlux       src/solver.cpp:1036-1058
  solver::timeStepA/B          src/solver.cpp:470-536
  solver::calcDt               src/solver.cpp:447-468, ele::calcDt ele.cpp:1127-1146,
  ele::calcWaveSpFpts          src/ele.cpp:1076-1125
  ele::getNormResidual         src/ele.cpp:1922-1944

Its inputs are the setup arrays (operators, metrics, face table) of a case,
either from a golden fixture (the reference's own dump) or from the
product's host setup; it is pinned against the reference's outputs by
``tests/test_oracle.py``.
"""
from __future__ import annotations

import numpy as np

BC_PERIODIC, BC_CHAR, BC_SUP_IN, BC_SUP_OUT, BC_SUB_IN, BC_SUB_OUT = 0, 1, 2, 3, 4, 5
BC_SLIP_WALL, BC_ISO_NOSLIP, BC_ADI_NOSLIP, BC_SYMMETRY, BC_ISO_MOVING = 8, 9, 10, 12, 13

CFL_LIMIT = [1.393, 0.464, 0.235, 0.1453, 0.100, 0.0736]  # src/global.cpp:81-105

RK_TABLES = {  # src/input.cpp:469-505
    0: (1, [0.0], [1.0]),
    2: (2, [0.0, 1.0], [0.5, 0.5]),
    4: (4, [0.0, 0.5, 0.5, 1.0], [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]),
    5: (4, [0.0, 1.0 / 4.0, 1.0 / 3.0, 1.0 / 2.0, 1.0], [0.0]),
}


def rk_table(time_type: int, order: int):
    if time_type == 6:
        a = [0.0, 0.153, 0.442, 0.931, 1.0] if order <= 2 else [0.0, 0.158, 0.477, 1.0, 1.0]
        return 4, a, [0.0]
    return RK_TABLES[time_type]


def gauss_weights(order: int) -> np.ndarray:
    x, w = np.polynomial.legendre.leggauss(order + 1)
    return w


def spt_weights(nd: int, order: int) -> np.ndarray:
    w = gauss_weights(order)
    if nd == 2:
        return np.einsum("i,j->ij", w, w).ravel()
    return np.einsum("i,j,k->ijk", w, w, w).ravel()


def inviscid_flux(U: np.ndarray, gam: float) -> np.ndarray:
    """F[d, ..., k] for U[..., k]  (src/flux.cpp:37-76)."""
    nf = U.shape[-1]
    nd = nf - 2
    rho = U[..., 0]
    u = U[..., 1] / rho
    v = U[..., 2] / rho
    F = np.zeros((nd,) + U.shape)
    if nd == 2:
        E = U[..., 3]
        p = (gam - 1.0) * (E - 0.5 * rho * (u * u + v * v))
        F[0, ..., 0] = rho * u; F[1, ..., 0] = rho * v
        F[0, ..., 1] = rho * u * u + p; F[1, ..., 1] = rho * u * v
        F[0, ..., 2] = rho * v * u; F[1, ..., 2] = rho * v * v + p
        F[0, ..., 3] = (E + p) * u; F[1, ..., 3] = (E + p) * v
    else:
        w = U[..., 3] / rho
        E = U[..., 4]
        p = (gam - 1.0) * (E - 0.5 * rho * (u * u + v * v + w * w))
        F[0, ..., 0] = rho * u; F[1, ..., 0] = rho * v; F[2, ..., 0] = rho * w
        F[0, ..., 1] = rho * u * u + p; F[1, ..., 1] = rho * u * v; F[2, ..., 1] = rho * u * w
        F[0, ..., 2] = rho * v * u; F[1, ..., 2] = rho * v * v + p; F[2, ..., 2] = rho * v * w
        F[0, ..., 3] = rho * w * u; F[1, ..., 3] = rho * w * v; F[2, ..., 3] = rho * w * w + p
        F[0, ..., 4] = (E + p) * u; F[1, ..., 4] = (E + p) * v; F[2, ..., 4] = (E + p) * w
    return F


def rusanov(UL, UR, n, gam):
    """Common flux and stored wave speed (src/face.cpp:314-374)."""
    nd = n.shape[-1]
    FL = inviscid_flux(UL, gam)
    FR = inviscid_flux(UR, gam)
    rhoL, rhoR = UL[:, 0], UR[:, 0]
    uL, uR = UL[:, 1] / rhoL, UR[:, 1] / rhoR
    vL, vR = UL[:, 2] / rhoL, UR[:, 2] / rhoR
    if nd == 2:
        pL = (gam - 1.0) * (UL[:, 3] - 0.5 * rhoL * (uL * uL + vL * vL))
        pR = (gam - 1.0) * (UR[:, 3] - 0.5 * rhoR * (uR * uR + vR * vR))
    else:
        wL, wR = UL[:, 3] / rhoL, UR[:, 3] / rhoR
        pL = (gam - 1.0) * (UL[:, 4] - 0.5 * rhoL * (uL * uL + vL * vL + wL * wL))
        pR = (gam - 1.0) * (UR[:, 4] - 0.5 * rhoR * (uR * uR + vR * vR + wR * wR))
    vnL = np.zeros_like(rhoL)
    vnR = np.zeros_like(rhoR)
    tL = np.zeros_like(UL)
    tR = np.zeros_like(UR)
    for d in range(nd):
        vnL = vnL + n[:, d] * UL[:, d + 1] / rhoL
        vnR = vnR + n[:, d] * UR[:, d + 1] / rhoR
        tL = tL + n[:, d:d + 1] * FL[d]
        tR = tR + n[:, d:d + 1] * FR[d]
    csqL = np.maximum(gam * pL / rhoL, 0.0)
    csqR = np.maximum(gam * pR / rhoR, 0.0)
    eigL = np.abs(vnL) + np.sqrt(csqL)
    eigR = np.abs(vnR) + np.sqrt(csqR)
    eig = np.maximum(eigL, eigR)
    Fn = 0.5 * (tL + tR - eig[:, None] * (UR - UL))
    return Fn, np.maximum(eigL, eigR)


def roe2d(UL, UR, n, gamma):
    """Roe flux with entropy fix, 2-D (src/face.cpp:376-495)."""
    vL = UL[:, 1:3] / UL[:, :1]
    vR = UR[:, 1:3] / UR[:, :1]
    pL = (gamma - 1.0) * (UL[:, 3] - (0.5 * UL[:, 0] * (vL[:, 0] ** 2 + vL[:, 1] ** 2)))
    pR = (gamma - 1.0) * (UR[:, 3] - (0.5 * UR[:, 0] * (vR[:, 0] ** 2 + vR[:, 1] ** 2)))
    hL = (UL[:, 3] + pL) / UL[:, 0]
    hR = (UR[:, 3] + pR) / UR[:, 0]
    sq_rho = np.sqrt(UR[:, 0] / UL[:, 0])
    rrho = 1.0 / (sq_rho + 1.0)
    um = rrho[:, None] * (vL + sq_rho[:, None] * vR)
    usq = 0.5 * um[:, 0] * um[:, 0] + 0.5 * um[:, 1] * um[:, 1]
    unm = um[:, 0] * n[:, 0] + um[:, 1] * n[:, 1]
    hm = rrho * (hL + sq_rho * hR)
    am_sq = (gamma - 1.0) * (hm - usq)
    am = np.sqrt(am_sq)
    rhoUnL = UL[:, 1] * n[:, 0] + UL[:, 2] * n[:, 1]
    rhoUnR = UR[:, 1] * n[:, 0] + UR[:, 2] * n[:, 1]
    Fn = np.empty_like(UL)
    Fn[:, 0] = rhoUnL + rhoUnR
    Fn[:, 1] = rhoUnL * vL[:, 0] + rhoUnR * vR[:, 0] + (pL + pR) * n[:, 0]
    Fn[:, 2] = rhoUnL * vL[:, 1] + rhoUnR * vR[:, 1] + (pL + pR) * n[:, 1]
    Fn[:, 3] = rhoUnL * hL + rhoUnR * hR
    du = UR - UL
    lam0 = np.abs(unm)
    lamP = np.abs(unm + am)
    lamM = np.abs(unm - am)
    eps = 0.5 * (np.abs(rhoUnL / UL[:, 0] - rhoUnR / UR[:, 0])
                 + np.abs(np.sqrt(gamma * pL / UL[:, 0]) - np.sqrt(gamma * pR / UR[:, 0])))
    with np.errstate(divide="ignore", invalid="ignore"):
        lam0 = np.where(lam0 < 2.0 * eps, 0.25 * lam0 * lam0 / eps + eps, lam0)
        lamP = np.where(lamP < 2.0 * eps, 0.25 * lamP * lamP / eps + eps, lamP)
        lamM = np.where(lamM < 2.0 * eps, 0.25 * lamM * lamM / eps + eps, lamM)
    a2 = 0.5 * (lamP + lamM) - lam0
    a3 = 0.5 * (lamP - lamM) / am
    a1 = a2 * (gamma - 1.0) / am_sq
    a4 = a3 * (gamma - 1.0)
    a5 = usq * du[:, 0] - um[:, 0] * du[:, 1] - um[:, 1] * du[:, 2] + du[:, 3]
    a6 = unm * du[:, 0] - n[:, 0] * du[:, 1] - n[:, 1] * du[:, 2]
    aL1 = a1 * a5 - a3 * a6
    bL1 = a4 * a5 - a2 * a6
    Fn[:, 0] -= lam0 * du[:, 0] + aL1
    Fn[:, 1] -= lam0 * du[:, 1] + aL1 * um[:, 0] + bL1 * n[:, 0]
    Fn[:, 2] -= lam0 * du[:, 2] + aL1 * um[:, 1] + bL1 * n[:, 1]
    Fn[:, 3] -= lam0 * du[:, 3] + aL1 * hm + bL1 * unm
    return 0.5 * Fn


def boundary_state(bc, UL, n, ph):
    """Ghost states (src/boundFace.cpp:65-314), static mesh."""
    nd = n.shape[-1]
    gam = ph["gamma"]
    gmo = gam - 1.0
    vB = np.array([ph["uBound"], ph["vBound"], ph["wBound"]])[:nd]
    rhoL = UL[:, 0]
    eL = UL[:, nd + 1]
    vL = UL[:, 1:nd + 1] / rhoL[:, None]
    pL = gmo * (eL - 0.5 * rhoL * np.sum(vL * vL, axis=1))
    rhoR = np.empty_like(rhoL)
    vR = np.zeros_like(vL)
    ER = np.empty_like(rhoL)

    def energy(p, rho, v):
        return p / gmo + 0.5 * rho * np.sum(v * v, axis=1)

    for code in np.unique(bc):
        m = bc == code
        if code == BC_SUB_IN:
            rhoR[m] = ph["rhoBound"]; vR[m] = vB; ER[m] = energy(pL[m], rhoR[m], vR[m])
        elif code == BC_SUB_OUT:
            rhoR[m] = rhoL[m]; vR[m] = vL[m]
            ER[m] = energy(np.full(m.sum(), ph["pBound"]), rhoR[m], vR[m])
        elif code == BC_SUP_IN:
            rhoR[m] = ph["rhoBound"]; vR[m] = vB
            ER[m] = energy(np.full(m.sum(), ph["pBound"]), rhoR[m], vR[m])
        elif code == BC_SUP_OUT:
            rhoR[m] = rhoL[m]; vR[m] = vL[m]; ER[m] = eL[m]
        elif code in (BC_SLIP_WALL, BC_SYMMETRY):
            rhoR[m] = rhoL[m]
            vnL = np.sum(vL[m] * n[m], axis=1)
            vR[m] = vL[m] - 2.0 * vnL[:, None] * n[m]
            ER[m] = eL[m]
        elif code == BC_ADI_NOSLIP:
            rhoR[m] = rhoL[m]; vR[m] = 0.0; ER[m] = energy(pL[m], rhoR[m], vR[m])
        elif code in (BC_ISO_NOSLIP, BC_ISO_MOVING):
            rhoR[m] = pL[m] / (ph["RGas"] * ph["TWall"])
            vR[m] = 0.0 if code == BC_ISO_NOSLIP else np.array([ph["uWall"], ph["vWall"], ph["wWall"]])[:nd]
            ER[m] = energy(pL[m], rhoR[m], vR[m])
        elif code == BC_CHAR:
            vnL = np.sum(vL[m] * n[m], axis=1)
            vnB = np.sum(vB[None, :] * n[m], axis=1)
            cL = np.sqrt(gam * pL[m] / rhoL[m])
            cB = np.sqrt(gam * ph["pBound"] / ph["rhoBound"])
            sup = np.abs(vnB) >= cB
            R_L = np.where(sup & (vnL >= 0), vnB + 2.0 / gmo * cB, vnL + 2.0 / gmo * cL)
            R_B = np.where(sup & (vnL < 0), vnL - 2.0 / gmo * cL, vnB - 2.0 / gmo * cB)
            rhoFac = 0.25 * gmo * (R_L - R_B)
            rhoBG = rhoFac * rhoFac / gam
            rhoBG = np.where(vnL < 0, rhoBG * ph["rhoBound"] ** gam / ph["pBound"],
                             rhoBG * rhoL[m] ** gam / pL[m])
            rr = rhoBG ** (1.0 / gmo)
            pR = rhoFac * rhoFac * rr / gam
            VB = 0.5 * (R_L + R_B)
            vR[m] = np.where((vnL < 0)[:, None], vB[None, :] + (VB - vnB)[:, None] * n[m],
                             vL[m] + (VB - vnL)[:, None] * n[m])
            rhoR[m] = rr
            ER[m] = pR / gmo + 0.5 * rr * np.sum(vR[m] * vR[m], axis=1)
        else:
            raise ValueError(f"boundary condition {code} not on the path")
    UR = np.empty_like(UL)
    UR[:, 0] = rhoR
    UR[:, 1:nd + 1] = rhoR[:, None] * vR
    UR[:, nd + 1] = ER
    return UR


def viscous_flux(U, gU, ph, quirk=True):
    """Navier-Stokes viscous flux Fv[d, ..., k] (src/flux.cpp:79-210).

    U[..., k], gU[d, ..., k] physical gradient.  With quirk, the reference's
    3-D tauxz/tauyz and the z-momentum entries of the x/y fluxes are kept."""
    nd = gU.shape[0]
    rho = U[..., 0]
    u = U[..., 1] / rho
    v = U[..., 2] / rho
    e = U[..., nd + 1] / rho - 0.5 * (u * u + v * v)
    if nd == 3:
        w = U[..., 3] / rho
        e = e - 0.5 * (w * w)
    else:
        w = np.zeros_like(rho)
    g = lambda d, k: gU[d][..., k]
    dRho_dx, dRhoU_dx, dRhoV_dx, dE_dx = g(0, 0), g(0, 1), g(0, 2), g(0, nd + 1)
    dRho_dy, dRhoU_dy, dRhoV_dy, dE_dy = g(1, 0), g(1, 1), g(1, 2), g(1, nd + 1)
    z = np.zeros_like(rho)
    dRho_dz = dRhoU_dz = dRhoV_dz = dRhoW_dx = dRhoW_dy = dRhoW_dz = dE_dz = z
    if nd == 3:
        dRho_dz, dRhoU_dz, dRhoV_dz = g(2, 0), g(2, 1), g(2, 2)
        dRhoW_dx, dRhoW_dy, dRhoW_dz, dE_dz = g(0, 3), g(1, 3), g(2, 3), g(2, 4)
    mu = np.full_like(rho, ph["mu_inf"])
    if not ph.get("fixVis", 0):
        rt = (ph["gamma"] - 1.0) * e / ph["rt_inf"]
        mu = mu * (rt ** 1.5 * (1. + ph["c_sth"]) / (rt + ph["c_sth"]))
    du_dx = (dRhoU_dx - dRho_dx * u) / rho
    du_dy = (dRhoU_dy - dRho_dy * u) / rho
    dv_dx = (dRhoV_dx - dRho_dx * v) / rho
    dv_dy = (dRhoV_dy - dRho_dy * v) / rho
    du_dz = dv_dz = dw_dx = dw_dy = dw_dz = z
    if nd == 3:
        du_dz = (dRhoU_dz - dRho_dz * u) / rho
        dv_dz = (dRhoV_dz - dRho_dz * v) / rho
        dw_dx = (dRhoW_dx - dRho_dx * w) / rho
        dw_dy = (dRhoW_dy - dRho_dy * w) / rho
        dw_dz = (dRhoW_dz - dRho_dz * w) / rho
    if nd == 2:
        dK_dx = 0.5 * (u * u + v * v) * dRho_dx + rho * (u * du_dx + v * dv_dx)
        dK_dy = 0.5 * (u * u + v * v) * dRho_dy + rho * (u * du_dy + v * dv_dy)
        dK_dz = z
    else:
        q = u * u + v * v + w * w
        dK_dx = 0.5 * q * dRho_dx + rho * (u * du_dx + v * dv_dx + w * dw_dx)
        dK_dy = 0.5 * q * dRho_dy + rho * (u * du_dy + v * dv_dy + w * dw_dy)
        dK_dz = 0.5 * q * dRho_dz + rho * (u * du_dz + v * dv_dz + w * dw_dz)
    de_dx = (dE_dx - dK_dx - dRho_dx * e) / rho
    de_dy = (dE_dy - dK_dy - dRho_dy * e) / rho
    de_dz = (dE_dz - dK_dz - dRho_dz * e) / rho if nd == 3 else z
    diag = (du_dx + dv_dy + dw_dz) / 3.0
    tauxx = 2.0 * mu * (du_dx - diag)
    tauyy = 2.0 * mu * (dv_dy - diag)
    tauxy = mu * (du_dy + dv_dx)
    tauxz = tauyz = tauzz = z
    if nd == 3:
        if quirk:
            tauxz = mu * (du_dz + dv_dx)
            tauyz = mu * (du_dz + dv_dy)
        else:
            tauxz = mu * (du_dz + dw_dx)
            tauyz = mu * (dv_dz + dw_dy)
        tauzz = 2.0 * mu * (dw_dz - diag)
    kq = (mu / ph["prandtl"]) * ph["gamma"]
    F = np.zeros((nd,) + U.shape)
    F[0, ..., 1] = -tauxx
    F[0, ..., 2] = -tauxy
    F[0, ..., nd + 1] = -(u * tauxx + v * tauxy + w * tauxz + kq * de_dx)
    F[1, ..., 1] = -tauxy
    F[1, ..., 2] = -tauyy
    F[1, ..., nd + 1] = -(u * tauxy + v * tauyy + w * tauyz + kq * de_dy)
    if nd == 3:
        F[0, ..., 3] = -tauzz if quirk else -tauxz
        F[1, ..., 3] = -tauyz
        F[2, ..., 1] = -tauxz
        F[2, ..., 2] = -tauyz
        F[2, ..., 3] = -tauzz
        F[2, ..., 4] = -(u * tauxz + v * tauyz + w * tauzz + kq * de_dz)
    return F


def ldg_pen(n, penFact):
    """Penalty direction switch (src/face.cpp:596-604)."""
    nd = n.shape[-1]
    s = n[:, 0] + n[:, 1] if nd == 2 else n[:, 0] + n[:, 1] + np.sqrt(2.) * n[:, 2]
    return np.where(s < 0, -penFact, penFact)


def adiabatic_gradient(UL, UR, gL, gamma):
    """Right gradient at an adiabatic wall (src/boundFace.cpp:316-350)."""
    nd = gL.shape[0]
    g = gL.copy()
    rhovSq = np.sum(UL[:, 1:nd + 1] ** 2, axis=1)
    pL = (gamma - 1.) * (UL[:, nd + 1] - 0.5 * rhovSq / UL[:, 0])
    e = pL / ((gamma - 1.) * UR[:, 0])
    gradVel = np.empty((nd, nd, UL.shape[0]))
    for d1 in range(nd):
        for d2 in range(nd):
            gradVel[d1, d2] = (gL[d1][:, d2 + 1] - gL[d1][:, 0] * UR[:, d2 + 1] / UR[:, 0]) / UR[:, 0]
    vSq = np.sum(UR[:, 1:nd + 1] ** 2 / (UR[:, :1] ** 2), axis=1)
    for d1 in range(nd):
        v = (e + 0.5 * vSq) * gL[d1][:, 0]
        for d2 in range(nd):
            v = v + UR[:, d2 + 1] * gradVel[d2, d1]
        g[d1][:, nd + 1] = v
    return g


class OracleCase:
    """A case described by its setup arrays (reference layout)."""

    def __init__(self, arrays: dict, params: dict):
        self.p = params
        self.nd = nd = int(params["nDims"])
        self.order = int(params["order"])
        self.ext = arrays["opp_spts_to_fpts"]
        self.nFp, self.nS = self.ext.shape
        self.grad = [arrays[f"opp_grad_spts_{d}"] for d in range(nd)]
        self.extFn = [arrays[f"opp_extrapolateFn_{d}"] for d in range(nd)]
        self.corr = arrays["opp_correction"]
        self.viscous = int(params.get("viscous", 0))
        if self.viscous:
            self.corrU = [arrays[f"opp_correctU_{d}"] for d in range(nd)]
        self.detJ = arrays["detJac_spts"]
        self.JGinv = arrays["JGinv_spts"]
        self.norm = arrays["norm_fpts"]
        self.dA = arrays["dA_fpts"]
        self.E = self.detJ.shape[1]
        self.nF = nd + 2
        self.nPF = self.nFp // (2 * nd)
        eL, locL = arrays["face_eL"], arrays["face_locL"]
        eR, fptR, bc = arrays["face_eR"], arrays["face_fptR"].reshape(len(eL), -1), arrays["face_bc"]
        j = np.arange(self.nPF)
        fL = locL[:, None] * self.nPF + j[None, :]
        self.slotL = (fL * self.E + eL[:, None]).ravel()
        interior = np.repeat(eR >= 0, self.nPF)
        self.slotR = np.where(interior, (fptR * self.E + np.maximum(eR, 0)[:, None]).ravel(), -1)
        self.fbc = np.repeat(bc, self.nPF)
        self.interior = interior
        self.wSpt = spt_weights(nd, self.order)
        self.wSurf = spt_weights(nd - 1, self.order) if nd == 3 else gauss_weights(self.order)
        self.waveSp = np.zeros(self.nFp * self.E)
        self.nRK, self.RKa, self.RKb = rk_table(int(params.get("timeType", 4)), self.order)
        self.quirk = bool(params.get("visc_flux_quirk", 1))
        self.iter = 0
        self.dt = float(params.get("dt", 0.0))
        self.eleDt = np.zeros(self.E)

    # --- residual pieces -----------------------------------------------------
    def extrapolate(self, U):
        return np.einsum("fs,sek->fek", self.ext, U)  # solver.cpp:556-572

    def flux_spts(self, U):
        Fp = inviscid_flux(U, self.p["gamma"])  # [d][s][e][k]
        F = np.zeros_like(Fp)
        for d1 in range(self.nd):  # solver.cpp:722-731
            for d2 in range(self.nd):
                F[d1] = F[d1] + self.JGinv[d1, :, :, d2][..., None] * Fp[d2]
        return F

    def faces(self, Uf):
        nF = self.nF
        Ufl = Uf.reshape(-1, nF)
        n = self.norm.reshape(-1, self.nd)[self.slotL]
        UL = Ufl[self.slotL]
        Fn = np.zeros_like(Ufl)
        dA = self.dA.ravel()
        m = self.interior
        ph = self.p
        # interior faces
        UR = Ufl[self.slotR[m]]
        if self.nd == 2 and int(ph.get("riemannType", 0)) == 1:
            F = roe2d(UL[m], UR, n[m], ph["gamma"])
        else:
            F, ws = rusanov(UL[m], UR, n[m], ph["gamma"])
            self.waveSp[self.slotL[m]] = ws
        Fn[self.slotL[m]] = F * dA[self.slotL[m]][:, None]
        Fn[self.slotR[m]] = -F * dA[self.slotR[m]][:, None]
        # boundary faces: always Rusanov (face.cpp:174-176)
        b = ~m
        if b.any():
            URb = boundary_state(self.fbc[b], UL[b], n[b], ph)
            Fb, wsb = rusanov(UL[b], URb, n[b], ph["gamma"])
            self.waveSp[self.slotL[b]] = wsb
            Fn[self.slotL[b]] = Fb * dA[self.slotL[b]][:, None]
        return Fn.reshape(Uf.shape)

    def faces_viscous(self, U, Uf):
        """Viscous calcResidual up to Fn and F_spts (solver.cpp:366-445 with
        viscous = 1): LDG solution, corrected gradient, viscous fluxes."""
        nd, nF = self.nd, self.nF
        ph = self.p
        gam = ph["gamma"]
        Ufl = Uf.reshape(-1, nF)
        n = self.norm.reshape(-1, nd)[self.slotL]
        dA = self.dA.ravel()
        m = self.interior
        b = ~m
        UL = Ufl[self.slotL]
        # 1. gradient in reference space (solver.cpp:1060-1078)
        dUr = [np.einsum("ts,sek->tek", self.grad[d], U) for d in range(nd)]
        # 2. inviscid common flux (kept per face point, before *dA) and LDG solution
        Fn_raw = np.zeros_like(UL)
        URall = np.empty_like(UL)
        URall[m] = Ufl[self.slotR[m]]
        if b.any():
            URall[b] = boundary_state(self.fbc[b], UL[b], n[b], ph)
        if nd == 2 and int(ph.get("riemannType", 0)) == 1:
            Fn_raw[m] = roe2d(UL[m], URall[m], n[m], gam)
        else:
            Fn_raw[m], ws = rusanov(UL[m], URall[m], n[m], gam)
            self.waveSp[self.slotL[m]] = ws
        if b.any():
            Fn_raw[b], wsb = rusanov(UL[b], URall[b], n[b], gam)
            self.waveSp[self.slotL[b]] = wsb
        dUc = np.zeros_like(Ufl)
        pen = ldg_pen(n[m], ph["penFact"])[:, None]
        UC = 0.5 * (UL[m] + URall[m]) - pen * (UL[m] - URall[m])
        dUc[self.slotL[m]] = UC - UL[m]
        dUc[self.slotR[m]] = UC - URall[m]
        if b.any():
            dUc[self.slotL[b]] = 0.5 * (UL[b] + URall[b]) - UL[b]
        dUc = dUc.reshape(Uf.shape)
        # 3. correction and physical transform (solver.cpp:1080-1137)
        for d in range(nd):
            dUr[d] = dUr[d] + np.einsum("sf,fek->sek", self.corrU[d], dUc)
        invDet = (1. / self.detJ)[..., None]
        dU = []
        for d2 in range(nd):
            v = dUr[0] * self.JGinv[0, :, :, d2][..., None] + dUr[1] * self.JGinv[1, :, :, d2][..., None]
            if nd == 3:
                v = v + dUr[2] * self.JGinv[2, :, :, d2][..., None]
            dU.append(invDet * v)
        dU = np.array(dU)
        dUf = np.array([self.extrapolate(dU[d]) for d in range(nd)])  # solver.cpp:1139-1158
        # 4. flux at the solution points (solver.cpp:777-811)
        Fv = viscous_flux(U, dU, ph, self.quirk) + inviscid_flux(U, gam)
        F = np.zeros_like(Fv)
        for d1 in range(nd):
            for d2 in range(nd):
                F[d1] = F[d1] + self.JGinv[d1, :, :, d2][..., None] * Fv[d2]
        # 5. viscous common flux (face.cpp:210-311)
        gflat = dUf.reshape(nd, -1, nF)
        gL = gflat[:, self.slotL]
        Fn_tot = Fn_raw.copy()
        if m.any():
            gR = gflat[:, self.slotR[m]]
            FL = viscous_flux(UL[m], gL[:, m], ph, self.quirk)
            FR = viscous_flux(URall[m], gR, ph, self.quirk)
            nn = n[m]
            pen = ldg_pen(nn, ph["penFact"])[:, None]
            dUj = UL[m] - URall[m]
            dF = [FL[0] - FR[0], FL[1] - FR[1]]
            if nd == 3:
                dF.append(FL[1] - FR[2] if self.quirk else FL[2] - FR[2])
            sdot = sum(nn[:, d:d + 1] * dF[d] for d in range(nd)) if nd == 3 else \
                nn[:, 0:1] * dF[0] + nn[:, 1:2] * dF[1]
            for d in range(nd):
                Fc = 0.5 * (FL[d] + FR[d]) + pen * nn[:, d:d + 1] * sdot + ph["tau"] * nn[:, d:d + 1] * dUj
                Fn_tot[m] = Fn_tot[m] + Fc * nn[:, d:d + 1]
        if b.any():
            adi = self.fbc[b] == BC_ADI_NOSLIP
            Fv_b = viscous_flux(UL[b], gL[:, b], ph, self.quirk)
            if adi.any():
                bi = np.nonzero(b)[0][adi]
                gA = adiabatic_gradient(UL[bi], URall[bi], gflat[:, self.slotL[bi]], gam)
                Fv_b[:, adi] = viscous_flux(URall[bi], gA, ph, self.quirk)
            nb = n[b]
            for d in range(nd):
                Fc = Fv_b[d] + ph["tau"] * nb[:, d:d + 1] * (UL[b] - URall[b])
                Fn_tot[b] = Fn_tot[b] + Fc * nb[:, d:d + 1]
        Fn = np.zeros_like(Ufl)
        Fn[self.slotL] = Fn_tot * dA[self.slotL][:, None]
        Fn[self.slotR[m]] = -Fn_tot[m] * dA[self.slotR[m]][:, None]
        self.last_visc = {"dU_spts": dU, "dU_fpts": dUf, "dUc_fpts": dUc}
        return F, Fn.reshape(Uf.shape)

    def residual(self, U, keep: dict | None = None):
        """divF of solver::calcResidual (solver.cpp:366-445)."""
        Uf = self.extrapolate(U)
        if self.viscous:
            F, Fn = self.faces_viscous(U, Uf)
        else:
            F = self.flux_spts(U)
            Fn = self.faces(Uf)
        disFn = np.einsum("fs,sek->fek", self.extFn[0], F[0])
        for d in range(1, self.nd):
            disFn = disFn + np.einsum("fs,sek->fek", self.extFn[d], F[d])
        divF = np.einsum("ts,sek->tek", self.grad[0], F[0])
        for d in range(1, self.nd):
            divF = divF + np.einsum("ts,sek->tek", self.grad[d], F[d])
        Q = Fn - disFn
        divF = divF + np.einsum("sf,fek->sek", self.corr, Q)
        if keep is not None:
            keep.update(U_fpts=Uf, F_spts=F, Fn_fpts=Fn, disFn_fpts=Q, divF=divF)
        return divF

    # --- time step ------------------------------------------------------------
    def wave_speed_init(self, Uf):
        """ele::calcWaveSpFpts (ele.cpp:1076-1125) on every element."""
        gam = self.p["gamma"]
        rho = Uf[..., 0]
        u = Uf[..., 1] / rho
        v = Uf[..., 2] / rho
        w = Uf[..., 3] / rho if self.nd == 3 else 0.0
        p = (gam - 1) * (Uf[..., self.nd + 1] - 0.5 * rho * (u * u + v * v + w * w))
        vN = u * self.norm[..., 0] + v * self.norm[..., 1]
        if self.nd == 3:
            vN = vN + w * self.norm[..., 2]
        self.waveSp = (np.abs(vN) + np.sqrt(np.maximum(gam * p / rho, 0.0))).ravel()

    def calc_dt(self, U):
        """solver::calcDt (solver.cpp:447-468)."""
        if self.iter == 1:
            self.wave_speed_init(self.extrapolate(U))
        vol = np.einsum("se,s->e", self.detJ, self.wSpt)
        ws = self.waveSp.reshape(self.nFp, self.E)
        wsurf = np.tile(self.wSurf, 2 * self.nd)
        intWave = np.einsum("fe,f,fe->e", ws, wsurf, self.dA)
        self.eleDt = self.p["CFL"] * CFL_LIMIT[self.order] * 2 * vol / intWave
        self.dt = float(np.min(self.eleDt))

    def _dt_field(self):
        if int(self.p.get("dtType", 0)) == 2:
            return self.eleDt[None, :, None]
        return self.dt

    def update(self, U):
        """One solver::update (solver.cpp:319-363); returns the new state."""
        self.iter += 1
        dtType = int(self.p.get("dtType", 0))
        timeType = int(self.p.get("timeType", 4))
        U = U.copy()
        U0 = U.copy()
        divs = []
        for step in range(self.nRK - 1):
            if step == 0 and dtType != 0:
                self.calc_dt(U)
            if step == 0:
                U0 = U.copy()
            d = self.residual(U)
            divs.append(d)
            dt = self._dt_field()
            U = U0 - self.RKa[step + 1] * d / self.detJ[..., None] * dt  # timeStepA
        d = self.residual(U)
        divs.append(d)
        if timeType < 5:
            if self.nRK > 1:
                U = U0.copy()
            elif dtType != 0:
                self.calc_dt(U)
            dt = self._dt_field()
            for step in range(self.nRK):  # timeStepB
                U = U - self.RKb[step] * divs[step] / self.detJ[..., None] * dt
        else:
            dt = self._dt_field()
            U = U0 - self.RKa[self.nRK] * d / self.detJ[..., None] * dt
        self.last_div0 = divs[0]
        return U

    def residual_norm(self, divF, res_type: int = 2):
        """writeResidual's per-field norm (output.cpp:1011-1090, ele.cpp:1922-1944)."""
        w = self.wSpt[:, None, None]
        if res_type == 1:
            return np.sum(np.abs(divF) * w, axis=(0, 1))
        if res_type == 2:
            return np.sqrt(np.sum(divF * divF / self.detJ[..., None] * w, axis=(0, 1)))
        return np.max(np.abs(divF) / self.detJ[..., None], axis=(0, 1))


def params_from_deck(path: str) -> dict:
    """Options the oracle needs, from a reference deck (first key wins)."""
    vals: dict = {}
    for line in open(path):
        t = line.split()
        if t and t[0] not in vals and len(t) > 1:
            vals[t[0]] = t[1]
    f = lambda k, d: float(vals.get(k, d))
    i = lambda k, d: int(float(vals.get(k, d)))
    nd = i("nDims", 2)
    p = {
        "nDims": nd, "order": i("order", 3), "gamma": f("gamma", 1.4),
        "rhoBound": f("rhoBound", 1.0), "uBound": f("uBound", 0.2), "vBound": f("vBound", 0.0),
        "wBound": f("wBound", 0.0) if nd == 3 else 0.0, "pBound": f("pBound", 0.7142857143),
        "riemannType": i("riemannType", 0), "timeType": i("timeType", 4), "dtType": i("dtType", 0),
        "CFL": f("CFL", 0.0), "dt": f("dt", 0.0), "RGas": f("RGas", 286.9), "TWall": f("TWall", 300.0),
        "uWall": 0.0, "vWall": 0.0, "wWall": 0.0, "viscous": i("viscous", 0),
    }
    if p["viscous"]:
        # input::nonDimensionalize (src/input.cpp:526-596)
        g = p["gamma"]
        Re, Lref, muGas = f("Re", 0.0), f("Lref", 1.0), f("muGas", 1.827e-5)
        SGas, TGas, RGas = f("SGas", 120.0), f("TGas", 291.15), f("RGas", 286.9)
        TBound, TWall, M = f("TBound", 300.0), f("TWall", 300.0), f("MachBound", 0.0)
        nxB, nyB, nzB = f("nxBound", 1.0), f("nyBound", 0.0), f("nzBound", 0.0) if nd == 3 else 0.0
        nm = np.sqrt(nxB * nxB + nyB * nyB + nzB * nzB)
        nxB, nyB, nzB = nxB / nm, nyB / nm, nzB / nm
        UB = M * np.sqrt(g * RGas * TBound)
        muB = muGas * (TBound / TGas) ** 1.5 * ((TGas + SGas) / (TBound + SGas))
        rhoB = muB * Re / (UB * Lref)
        pB = rhoB * RGas * TBound
        rhoRef = rhoB
        pRef = rhoRef * UB * UB
        muRef = rhoRef * UB * Lref
        # the moving wall's velocity (src/input.cpp:551-554, 583-585)
        UW = f("MachWall", 0.0) * np.sqrt(g * RGas * TWall)
        nxW, nyW, nzW = f("nxWall", 1.0), f("nyWall", 0.0), f("nzWall", 0.0)
        p.update(uWall=UW * nxW / UB, vWall=UW * nyW / UB, wWall=UW * nzW / UB)
        p.update(c_sth=SGas / TGas, mu_inf=muGas / muRef, rt_inf=TGas * RGas / (UB * UB),
                 RGas=RGas * TBound / (UB * UB), rhoBound=1.0, uBound=UB * nxB / UB, vBound=UB * nyB / UB,
                 wBound=UB * nzB / UB, pBound=pB / pRef, TWall=TWall / TBound,
                 prandtl=f("prandtl", 0.72), fixVis=i("fixVis", 0), penFact=f("LDG_penFact", 0.0),
                 tau=f("LDG_tau", 1.0))
    return p
