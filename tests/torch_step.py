"""Plain FP64 PyTorch transcription of one vertical step (Rusanov solver) in
the GITM-array form: coefficient producers, gather, set_vertical_bcs, the
four RK4 stages of advance_vertical_1d_rusanov, scatter and the optional
heating line.  TEST INFRASTRUCTURE: the autograd reference the adjoint
kernel is checked against (and itself pinned to the oracle).

It follows the statements of the CUDA kernel (vert_kernel.cuh), which follow
the reference:
  advance_vertical.f90:45-219 (gather / scatter), calc_pressure.f90:56-83,
  calc_rates.Earth.f90:34-50, calc_timestep.f90:114-118 (producers),
  vertical_solver_rusanov.f90:10-779 (RK4, stage, sweeps, face values),
  calc_neutral_friction.f90:47-106, set_vertical_bcs.Earth.f90:8-652,
  add_sources.f90:53-66 (heating).
Every function is differentiable by torch autograd; branches (limiter, clamp,
boundary switches) take the side the values select, so autograd
differentiates the branch the forward took.

Scope: the Rusanov solver with improved or log ion advection, friction,
Coriolis, damping, MSIS lower boundary and producers on or off.  The upper
ion boundary's negative-density repair (set_vertical_bcs.Earth.f90:608-649)
is not transcribed: inputs that reach it are rejected.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from gitm_b200 import synthetic as S

KB = S.KB
MASS = [float(m) for m in S.MASS]
NS = 6
NI = 9
NADV = 2
PHOTO = (3, 4)  # N(4S), NO
F1 = 0.6250000
F2 = 0.0416667
# friction constants (ModEarth.f90:237-262): Diff0 and the DiffExp table
_D0 = [[0.000, 0.969, 0.969, 0.969, 0.715, 3.440], [0.969, 0.000, 0.715, 0.969, 0.715, 3.208],
       [0.969, 0.715, 0.000, 0.969, 0.527, 2.939], [0.969, 0.969, 0.969, 0.000, 0.969, 2.939],
       [0.715, 0.715, 0.527, 0.969, 0.000, 2.939], [3.440, 3.208, 2.939, 2.939, 2.939, 0.000]]
_EXPS = [0.774, 0.750, 0.749, 0.710, 0.718, 0.810]
_EIDX = [[0, 0, 0, 0, 1, 2], [0, 0, 1, 0, 1, 3], [0, 1, 0, 0, 5, 4],
         [0, 0, 0, 0, 0, 4], [1, 1, 5, 0, 0, 4], [2, 3, 4, 4, 4, 0]]
INV_VIB2 = [1.0 / (v - 2) for v in S.VIBRATION]


def _kc(i, j):
    return 1.0e-2 * KB / (MASS[i] * (1.0e17 * _D0[i][j]))


class Grid:
    """Grid coefficients of one altitude grid (host arithmetic of gitm_vert.cu)."""

    def __init__(self, alt, grav, dalt_c, inv_r, device, dtype=torch.float64):
        alt = np.asarray(alt, dtype=np.float64)
        G = alt.shape[0]
        nA = G - 4
        self.nA, self.G = nA, G
        dAF = np.zeros(G)
        for i in range(0, nA + 3):
            dAF[i + 1] = alt[i + 1] - alt[i]
        dAF[0] = dAF[1]
        IDF = 1.0 / dAF
        F = lambda i: dAF[i + 1]  # noqa: E731
        mc = np.zeros((5, G))
        for i in range(1, nA + 1):
            h1, h2, h3, h4 = F(i - 1), F(i), F(i + 1), F(i + 2)
            H2, H3, H4 = h2 + h1, h3 + h2 + h1, h4 + h3 + h2 + h1
            mc[0, i + 1] = (h2 * h3 * (h3 + h4)) / (h1 * H2 * H3 * H4)
            mc[1, i + 1] = -1.0 * (H2 * h3 * (h3 + h4)) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4))
            mc[2, i + 1] = ((h2 * h3 * (h3 + h4) + H2 * h3 * (h3 + h4) - H2 * h2 * (h3 + h4) - H2 * h2 * h3) /
                            (H2 * h2 * h3 * (h3 + h4)))
            mc[3, i + 1] = H2 * h2 * (h4 + h3) / (H3 * (h2 + h3) * h3 * h4)
            mc[4, i + 1] = -1.0 * H2 * h2 * h3 / (H4 * (h2 + h3 + h4) * (h3 + h4) * h4)
        bl = np.zeros((2, 5))
        for k in range(2):
            iA = -k
            h1, h2, h3, h4 = F(iA + 2), F(iA + 3), F(iA + 4), F(iA + 5)
            M1, M2, M3, M4 = h1, h1 + h2, h1 + h2 + h3, h1 + h2 + h3 + h4
            bl[k] = [-1.0 * (M2 * M3 * M4 + M1 * M3 * M4 + M1 * M2 * M4 + M1 * M2 * M3) / (M1 * M2 * M3 * M4),
                     1.0 * (M2 * M3 * M4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4)),
                     -1.0 * (M1 * M3 * M4) / (M2 * h2 * h3 * (h3 + h4)),
                     1.0 * (M1 * M2 * M4) / (M3 * (h3 + h2) * h3 * h4),
                     -1.0 * (M1 * M2 * M3) / (M4 * (h2 + h3 + h4) * (h3 + h4) * h4)]
        bu = np.zeros((2, 5))
        for k in range(2):
            iA = nA + 1 + k
            h1, h2, h3, h4 = F(iA - 1), F(iA - 2), F(iA - 3), F(iA - 4)
            M1, M2, M3, M4 = h1, h1 + h2, h1 + h2 + h3, h1 + h2 + h3 + h4
            bu[k] = [1.0 * (M2 * M3 * M4 + M1 * M3 * M4 + M1 * M2 * M4 + M1 * M2 * M3) / (M1 * M2 * M3 * M4),
                     -1.0 * (M2 * M3 * M4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4)),
                     1.0 * (M1 * M3 * M4) / (M2 * h2 * h3 * (h3 + h4)),
                     -1.0 * (M1 * M2 * M4) / (M3 * (h3 + h2) * h3 * h4),
                     1.0 * (M1 * M2 * M3) / (M4 * (h2 + h3 + h4) * (h3 + h4) * h4)]
        t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=device, dtype=dtype)  # noqa: E731
        self.dAF_np, self.bl, self.bu = dAF, bl, bu
        self.dAF = t(dAF)[:, None]
        self.IDF = t(IDF)[:, None]
        self.H2 = t(IDF * 2.0)[:, None]
        self.IDC = t(1.0 / np.asarray(dalt_c, dtype=np.float64))[:, None]
        self.grav = t(grav)[:, None]
        self.invr = t(inv_r)[:, None]
        self.R = t(1.0 / np.asarray(inv_r, dtype=np.float64))[:, None]
        self.alt = t(alt)[:, None]
        self.mc = t(mc)[:, :, None]


# Branch recording: while a list is installed, every branch point appends
# the decisions it took, so that finite-difference checks can keep only the
# directions that cross no kink.
_BRANCHES = None


def _record(*conds):
    if _BRANCHES is not None:
        for c in conds:
            _BRANCHES.append(c.detach().clone() if torch.is_tensor(c) else torch.tensor(bool(c)))


def branch_signature(fn, *args, **kw):
    """Runs fn and returns the list of its branch decisions."""
    global _BRANCHES
    _BRANCHES = []
    try:
        with torch.no_grad():
            fn(*args, **kw)
        return _BRANCHES
    finally:
        _BRANCHES = None


def same_branches(a, b) -> bool:
    return len(a) == len(b) and all(torch.equal(x, y) for x, y in zip(a, b))


def limiter_mc(u, d, beta):
    """ModLimiter.f90:16-36, elementwise."""
    bu, bd, av = beta * u, beta * d, (u + d) * 0.5
    if _BRANCHES is not None:
        # which formula the limiter returned: 0, beta*u, beta*d or the mean
        lo = torch.where(bu <= bd, 1, 2)
        lo = torch.where(torch.minimum(bu, bd) <= av, lo, 3)
        hi = torch.where(bu >= bd, 1, 2)
        hi = torch.where(torch.maximum(bu, bd) >= av, hi, 3)
        code = torch.where(u > 0.0, torch.where(d > 0.0, lo, 0), torch.where(d < 0.0, hi, 0))
        _record(code)
    pos = torch.where(d > 0.0, torch.minimum(torch.minimum(bu, bd), av), torch.zeros_like(u))
    neg = torch.where(d < 0.0, torch.maximum(torch.maximum(bu, bd), av), torch.zeros_like(u))
    return torch.where(u > 0.0, pos, neg)


def _lsum(vals):
    s = torch.zeros_like(vals[0])
    for v in vals:
        s = s + v
    return s


# --------------------------------------------------------------- boundaries
def set_vertical_bcs(X, gr: Grid, cs, prm, pre):
    """set_vertical_bcs (Earth) on every column.  X: dict of row lists
    (index g = cell + 1); pre: the rows of X before the call (the values of
    cells the boundary reads before it overwrites them).  cs: per-column
    scalars (EG at the boundary cells, MMM at -1/0, plasma switch, lbc)."""
    nA = gr.nA
    g = lambda i: i + 1  # noqa: E731
    dAF = lambda i: float(gr.dAF_np[i + 1])  # noqa: E731
    L, W, I = X["lns"], X["w"], X["ion"]
    T, VE, VN, VU, LR = X["t"], X["ve"], X["vn"], X["vu"], X["lrho"]
    msis = bool(prm.use_msis_bcs) and cs["lbc"] is not None
    zero = torch.zeros_like(T[0])
    # ---- lower boundary
    l0 = [L[s][g(0)] for s in range(NS)]
    if msis:
        t = cs["lbc"]
        for s in range(NS):
            L[s][g(-1)] = t[0, s]
            L[s][g(0)] = t[1, s]
        T[g(-1)], T[g(0)] = t[0, 6], t[1, 6]
        LR[g(-1)], LR[g(0)] = t[0, 7], t[1, 7]
        VE[g(-1)], VE[g(0)] = t[0, 8], t[1, 8]
        VN[g(-1)], VN[g(0)] = t[0, 9], t[1, 9]
    else:
        VE[g(-1)] = VE[g(0)] = zero
        VN[g(-1)] = VN[g(0)] = zero
    VU[g(-1)] = VU[g(0)] = zero
    for s in range(NS):
        W[s][g(-1)] = W[s][g(0)] = zero
    T[g(-1)] = T[g(0)]
    VE[g(-1)] = VE[g(0)]
    VN[g(-1)] = VN[g(0)]
    VU[g(-1)] = VU[g(0)]
    bl = gr.bl
    for s in range(NS):
        if s not in PHOTO:
            mg = -0.5 * (cs["eg"][0] + cs["eg"][1])
            mt = 0.5 * (T[g(0)] + T[g(-1)])
            mm = 0.5 * (cs["mmm0"] + cs["mmm_m1"])
            ish = mg * mm / (mt * KB)
            L[s][g(-1)] = L[s][g(0)] if s == 0 else l0[s] + ish * dAF(-1)
        else:
            for k in range(2):
                i = -k
                C = bl[k]
                d = (L[s][g(i + 1)] * C[0] + L[s][g(i + 2)] * C[1] + L[s][g(i + 3)] * C[2] +
                     L[s][g(i + 4)] * C[3] + L[s][g(i + 5)] * C[4])
                up = L[s][g(i + 1)]
                v = up - dAF(i + 1) * d
                _record(d <= 0.0)
                v = torch.where(d <= 0.0, up, v)
                if s == 4:
                    _record(v < up - 0.333)
                    v = torch.where(v < up - 0.333, up - 0.333, v)
                L[s][g(i)] = v
        for k in range(2):
            i = -k
            C = bl[k]
            d = (W[s][g(i + 1)] * C[0] + W[s][g(i + 2)] * C[1] + W[s][g(i + 3)] * C[2] +
                 W[s][g(i + 4)] * C[3] + W[s][g(i + 5)] * C[4])
            W[s][g(i)] = W[s][g(i + 1)] - dAF(i + 1) * d
    for s in range(NI):
        v = I[s][g(1)]
        I[s][g(0)] = v
        I[s][g(-1)] = v
    for c in (0, -1):
        ms = [MASS[s] * torch.exp(L[s][g(c)]) for s in range(NS)]
        r = _lsum(ms)
        mw = _lsum([ms[s] * W[s][g(c)] for s in range(NS)])
        LR[g(c)] = torch.log(r)
        VU[g(c)] = mw / r
    if msis:
        C = bl[1]
        for F in (VE, VN):
            d = F[g(0)] * C[0] + F[g(1)] * C[1] + F[g(2)] * C[2] + F[g(3)] * C[3] + F[g(4)] * C[4]
            F[g(-1)] = F[g(0)] - dAF(0) * d
    for s in PHOTO:
        flip = W[s][g(1)] > 0.0
        _record(flip)
        W[s][g(0)] = torch.where(flip, -1.0 * W[s][g(1)], W[s][g(0)])
        W[s][g(-1)] = torch.where(flip, -1.0 * W[s][g(1)], W[s][g(-1)])
    # ---- upper boundary
    for F in (VE, VN):
        F[g(nA + 1)] = F[g(nA)]
        F[g(nA + 2)] = F[g(nA)]
    for s in range(NS):
        wn = W[s][g(nA)]
        w1, w2 = wn, wn
        if s in PHOTO:
            neg = wn < 0.0
            _record(neg)
            w1 = torch.where(neg, -wn, wn)
            w2 = torch.where(neg, -W[s][g(nA - 1)], wn)
        W[s][g(nA + 1)] = w1
        W[s][g(nA + 2)] = w2
        Tn = T[g(nA)]
        ish1 = (-0.5 * (cs["eg"][3] + cs["eg"][2])) * MASS[s] / (0.5 * (Tn + Tn) * KB)
        ish2 = (-0.5 * (cs["eg"][4] + cs["eg"][3])) * MASS[s] / (0.5 * (Tn + Tn) * KB)
        l1 = L[s][g(nA)] - ish1 * dAF(nA + 1)
        L[s][g(nA + 1)] = l1
        L[s][g(nA + 2)] = l1 - ish2 * dAF(nA + 2)
    _record(VU[g(nA)] < 0.0)
    a = torch.abs(VU[g(nA)])
    VU[g(nA + 1)] = a
    VU[g(nA + 2)] = a
    T[g(nA + 1)] = T[g(nA)]
    T[g(nA + 2)] = T[g(nA)]
    improved = bool(prm.use_improved_ion_advection)
    tp = _lsum([float(gr.dAF_np[i + 1]) * (I[0][g(i)] if improved else torch.exp(I[0][g(i)]))
                for i in range(1, nA + 1)])
    hold = (tp / 1e16 < prm.min_tec) & (cs["plasma"] > 0.5)
    _record(hold)
    bu = gr.bu
    for s in range(NI):
        if improved:
            for q in range(nA - 5, nA + 3):
                if bool((I[s][g(q)] < 0.0).any()):
                    raise ValueError("negative ion density at the upper boundary: not transcribed")
            n = [torch.log(pre["ion"][s][g(nA + 1)])] + [torch.log(I[s][g(nA + 1 - j)]) for j in range(1, 6)]
            C = bu[0]
            dn = C[0] * n[1] + C[1] * n[2] + C[2] * n[3] + C[3] * n[4] + C[4] * n[5]
            lim = -(0.001 * n[0] / dAF(nA))
            _record(dn > lim)
            dn = torch.where(dn > lim, lim, dn)
            v1 = torch.exp(n[1] + dn * dAF(nA + 1))
            g0 = torch.log(pre["ion"][s][g(nA + 2)])
            n1 = torch.log(v1)
            D = bu[1]
            dn2 = D[0] * n1 + D[1] * n[1] + D[2] * n[2] + D[3] * n[3] + D[4] * n[4]
            lim2 = -(0.001 * g0 / dAF(nA))
            _record(dn2 > lim2)
            dn2 = torch.where(dn2 > lim2, lim2, dn2)
            v2 = torch.exp(n1 + dn2 * dAF(nA + 2))
            I[s][g(nA + 1)] = torch.where(hold, I[s][g(nA + 1)], v1)
            I[s][g(nA + 2)] = torch.where(hold, I[s][g(nA + 2)], v2)
        else:
            for k in range(2):
                iA = nA + 1 + k
                C = bu[k]
                dn = (C[0] * I[s][g(iA - 1)] + C[1] * I[s][g(iA - 2)] + C[2] * I[s][g(iA - 3)] +
                      C[3] * I[s][g(iA - 4)] + C[4] * I[s][g(iA - 5)])
                lim = -(0.001 * pre["ion"][s][g(iA)] / dAF(nA))
                _record(dn > lim)
                dn = torch.where(dn > lim, lim, dn)
                v = I[s][g(iA - 1)] + dn * dAF(nA + 1 + k)
                I[s][g(iA)] = torch.where(hold, I[s][g(iA)], v)
    for c in (nA + 1, nA + 2):
        LR[g(c)] = torch.log(_lsum([MASS[s] * torch.exp(L[s][g(c)]) for s in range(NS)]))


# --------------------------------------------------------------- the stage
def _to_rows(x):
    return list(x.unbind(0))


def _pack(X):
    return {k: ([torch.stack(r) for r in v] if isinstance(v[0], list) else torch.stack(v)) for k, v in X.items()}


def _unpack(P):
    return {k: ([_to_rows(r) for r in v] if isinstance(v, list) else _to_rows(v)) for k, v in P.items()}


def _copy_rows(X):
    return {k: ([list(r) for r in v] if isinstance(v[0], list) else list(v)) for k, v in X.items()}


def _slopes(v, gr: Grid, beta):
    """Limited slopes on cells 0..nAlts+1 (index c = cell), [nA+2, C]."""
    nA = gr.nA
    g = lambda i: i + 1  # noqa: E731
    sl = slice(g(1), g(nA) + 1)
    vi = lambda o: v[g(1) + o:g(nA) + 1 + o]  # noqa: E731
    up = gr.H2[g(2):g(nA + 1) + 1] * (F1 * (vi(1) - vi(0)) - F2 * (vi(2) - vi(-1)))
    dn = gr.H2[sl] * (F1 * (vi(0) - vi(-1)) - F2 * (vi(1) - vi(-2)))
    mid = limiter_mc(up, dn, beta)
    e0 = limiter_mc((v[g(1)] - v[g(0)]) * gr.IDF[g(1)], (v[g(0)] - v[g(-1)]) * gr.IDF[g(0)], beta)
    e1 = limiter_mc((v[g(nA + 2)] - v[g(nA + 1)]) * gr.IDF[g(nA + 2)],
                    (v[g(nA + 1)] - v[g(nA)]) * gr.IDF[g(nA + 1)], beta)
    return torch.cat([e0[None], mid, e1[None]])


def _sweep(v, d, gr: Grid, fc0, fc1):
    """Gradient and Rusanov dissipation at cells 1..nAlts, [nA, C]."""
    nA = gr.nA
    dF0 = gr.dAF[2:nA + 2]
    dF1 = gr.dAF[3:nA + 3]
    idc = gr.IDC[2:nA + 2]
    vm, v0, vp = v[1:nA + 1], v[2:nA + 2], v[3:nA + 3]
    dm, d0, dp = d[0:nA], d[1:nA + 1], d[2:nA + 2]
    L0 = vm + 0.5 * dm * dF0
    R0 = v0 - 0.5 * d0 * dF0
    L1 = v0 + 0.5 * d0 * dF1
    R1 = vp - 0.5 * dp * dF1
    grad = 0.5 * (L1 + R1 - L0 - R0) * idc
    diff = (fc1 * (R1 - L1) - fc0 * (R0 - L0)) * idc
    return grad, diff


def stage_k(P, gr: Grid, cs, co, prm, dt):
    """K = New - state at cells 1..nAlts for every field (advance_vertical_1stage)."""
    nA = gr.nA
    it = slice(2, nA + 2)
    beta = prm.beta_limiter
    cm = co["cmax"]
    _record(cm[1:nA + 1] < cm[2:nA + 2], cm[2:nA + 2] < cm[3:nA + 3])
    fc0 = 0.5 * torch.maximum(cm[1:nA + 1], cm[2:nA + 2])
    fc1 = 0.5 * torch.maximum(cm[2:nA + 2], cm[3:nA + 3])

    def sw(v):
        return _sweep(v, _slopes(v, gr, beta), gr, fc0, fc1)

    T, VE, VN, VU, LR = P["t"][it], P["ve"][it], P["vn"][it], P["vu"][it], P["lrho"][it]
    invr, rr, grav = gr.invr[it], gr.R[it], gr.grav[it]
    gT, dT = sw(P["t"])
    gE, dE = sw(P["ve"])
    gN, dN = sw(P["vn"])
    gU, _ = sw(P["vu"])
    K = {}
    K["ve"] = (VE - dt * VU * gE + dt * dE) - VE
    K["vn"] = (VN - dt * VU * gN + dt * dN) - VN
    divv = gU + 2 * VU * invr
    K["t"] = (T - dt * (VU * gT + (co["gamma"][it] - 1.0) * (T * divv)) + dt * dT) - T
    K["ion"] = []
    for s in range(NADV):
        gI, dI = sw(P["ion"][s])
        Iv = P["ion"][s][it]
        K["ion"].append((Iv - dt * (co["ivup"][it] * gI) + dt * dI) - Iv)
    if prm.use_damping:
        itau = 1.0 / (15 - (1 - torch.exp(-1.0 * gr.alt[it] / 1000.0 / 40.0)) * 5.0)
    else:
        itau = 1.0 / prm.vert_tau
    hz = (VN * VN + VE * VE) * invr
    cor = dt * (cs["cent"] * rr + cs["cori"] * VE) if prm.use_coriolis else 0.0
    wv, nl = [], []
    for s in range(NS):
        gL, dL = sw(P["lns"][s])
        gW, dW = sw(P["w"][s])
        Ls, Ws = P["lns"][s][it], P["w"][s][it]
        divw = gW + 2 * Ws * invr
        n_l = Ls - dt * (divw + Ws * gL) + dt * dL
        nl.append(n_l)
        km = KB / MASS[s]
        w = Ws - dt * (Ws * gW - hz + T * gL * km + gT * km - grav) + dt * dW - Ws * itau
        w = w + cor
        w = w - dt * (prm.thermal_diff_coef[s] * km) * gT
        wv.append(w)
    K["lns"] = [nl[s] - P["lns"][s][it] for s in range(NS)]
    sumrho = _lsum([MASS[s] * torch.exp(nl[s]) for s in range(NS)])
    K["lrho"] = torch.log(sumrho) - LR
    ns = [torch.exp(P["lns"][s][it]) for s in range(NS)]
    ir = torch.exp(-LR)
    if prm.use_neutral_friction:
        lr5 = [P["lrho"][q:nA + q] for q in range(5)]
        mc = gr.mc[:, it]
        glc = []
        for s in range(NS):
            acc = torch.zeros_like(T)
            for q in range(5):
                acc = acc + mc[q] * (math.log(MASS[s]) + P["lns"][s][q:nA + q] - lr5[q])
            glc.append(acc)
        lt = torch.log(T)
        pw = [torch.exp((1.0 - e) * lt) for e in _EXPS]
        rows = []
        for r in range(NS):
            cij = [None] * NS
            rs = torch.zeros_like(T)
            for q in range(NS):
                if q == r:
                    continue
                cij[q] = _kc(r, q) * ns[q] * pw[_EIDX[r][q]]
                rs = rs + cij[q]
            rows.append([(1.0 + dt * rs) if q == r else (-dt * cij[q]) for q in range(NS)])
        A = torch.stack([torch.stack(rw, -1) for rw in rows], -2)  # [nA, C, 6, 6]
        b = torch.stack(wv, -1)
        sol = torch.linalg.solve(A, b)
        wv = [sol[..., s] + (-co["eddy"][it] * glc[s]) for s in range(NS)]
    vu = torch.zeros_like(T)
    K["w"] = []
    for s in range(NS):
        _record(wv[s] < -prm.max_vertical_velocity, wv[s] > prm.max_vertical_velocity)
        w = torch.clamp(wv[s], min=-prm.max_vertical_velocity)
        w = torch.clamp(w, max=prm.max_vertical_velocity)
        K["w"].append(w - P["w"][s][it])
        vu = vu + w * (MASS[s] * ns[s] * ir)
    K["vu"] = vu - VU
    return K


def _combine(O, K, c):
    """Interior cells O + c K, ghosts O (passive ions: O)."""
    out = {}
    for k, v in O.items():
        if isinstance(v, list):
            lst = []
            for s, x in enumerate(v):
                if k == "ion" and s >= NADV:
                    lst.append(x)
                    continue
                kk = K[k][s]
                lst.append(torch.cat([x[:2], x[2:-2] + c(kk), x[-2:]]))
            out[k] = lst
        else:
            out[k] = torch.cat([v[:2], v[2:-2] + c(K[k]), v[-2:]])
    return out


def _bc(P, gr, cs, prm, pre_P):
    X = _unpack(P)
    pre = _unpack(pre_P)
    set_vertical_bcs(X, gr, cs, prm, pre)
    return _pack(X)


def step(state: dict, inp: dict, prm, dt: float) -> dict:
    """One vertical step of every column.  state: nd [6,G,C], ion [10,G,C],
    rho, temp (normalised Temperature), [G,C]; vel [3,G,C]; ww [6,G,C].
    inp: ivel_up, eddy [G,C]; cos_lat, sza, mlat [C]; lbc [2,10,C] or None;
    grid (Grid); heating [G,C] or None; heating_scale [C] or None.
    Returns the new state plus log_ns and ndensity."""
    gr = inp["grid"]
    nA = gr.nA
    nd, ww, temp = state["nd"], state["ww"], state["temp"]
    # producers
    N = _lsum([nd[s] for s in range(NS)])
    gg = _lsum([nd[s] * INV_VIB2[s] for s in range(NS)])
    gamma = gg * 2.0 / N + 1
    rn = 1.0 / (N + 1.0)
    mmm = _lsum([MASS[s] * nd[s] * rn for s in range(NS)])
    tu = mmm * (1.0 / KB)
    mx = torch.abs(ww[0])
    _record(ww < 0.0)
    for s in range(1, NS):
        _record(mx < torch.abs(ww[s]))
        mx = torch.maximum(mx, torch.abs(ww[s]))
    cmx = mx + torch.sqrt(gamma * temp)
    cmask = torch.zeros_like(temp)
    cmask[1:nA + 3] = 1.0
    cmx = cmx * cmask
    co = {"gamma": gamma, "cmax": cmx, "ivup": inp["ivel_up"], "eddy": inp["eddy"]}
    cl = inp["cos_lat"]
    om = prm.omega_body
    cent = (cl * om) * (cl * om)
    cori = 2 * cl * om
    plasma = torch.zeros_like(cl)
    if prm.use_nighttime_ion_bcs:
        sza, mlat = inp["sza"], inp["mlat"]
        m1 = (sza > math.pi / 2) & (((mlat > 30.0) & (mlat < 70.0)) | ((mlat > -60.0) & (mlat < -30.0)))
        plasma = m1.to(cl.dtype)
    eg = [gr.grav[c + 1, 0] + cent * gr.R[c + 1, 0] for c in (-1, 0, nA, nA + 1, nA + 2)]
    lbc = inp.get("lbc")
    cs = {"cent": cent, "cori": cori, "plasma": plasma, "eg": eg, "mmm_m1": mmm[0], "mmm0": mmm[1],
          "lbc": None if lbc is None else lbc}
    improved = bool(prm.use_improved_ion_advection)
    # gather
    P = {"lns": [torch.log(nd[s]) for s in range(NS)], "w": [ww[s] for s in range(NS)],
         "t": temp * tu, "ve": state["vel"][0], "vn": state["vel"][1], "vu": state["vel"][2],
         "lrho": torch.log(state["rho"]),
         "ion": [state["ion"][s] if improved else torch.log(state["ion"][s]) for s in range(NI)]}
    P = _bc(P, gr, cs, prm, P)
    O = P
    w = [1.0, 2.0, 2.0, 1.0]
    c = [0.5, 0.5, 1.0]
    Ks = []
    for k in range(4):
        K = stage_k(P, gr, cs, co, prm, dt)
        Ks.append(K)
        if k < 3:
            Pn = _combine(O, K, lambda kk, cc=c[k]: cc * kk)
        else:
            acc = {}
            for key in K:
                if isinstance(K[key], list):
                    acc[key] = [Ks[0][key][s] + 2.0 * Ks[1][key][s] + 2.0 * Ks[2][key][s] + Ks[3][key][s]
                                for s in range(len(K[key]))]
                else:
                    acc[key] = Ks[0][key] + 2.0 * Ks[1][key] + 2.0 * Ks[2][key] + Ks[3][key]
            Pn = _combine(O, acc, lambda a: (1.0 / 6.0) * a)
        P = _bc(Pn, gr, cs, prm, Pn)
    # scatter
    out = {}
    out["rho"] = torch.exp(P["lrho"])
    t_new = P["t"] / tu
    if inp.get("heating") is not None:
        hs = inp["heating_scale"] if inp.get("heating_scale") is not None else torch.ones_like(cl)
        add = dt * (hs * inp["heating"])
        add = torch.cat([torch.zeros_like(add[:2]), add[2:-2], torch.zeros_like(add[-2:])])
        t_new = t_new + add
    out["temp"] = t_new
    out["vel"] = torch.stack([P["ve"], P["vn"], P["vu"]])
    out["ww"] = torch.stack(P["w"])
    out["log_ns"] = torch.stack(P["lns"])
    nd_new = torch.stack([torch.exp(x) for x in P["lns"]])
    out["nd"] = nd_new
    out["ndensity"] = _lsum([nd_new[s] for s in range(NS)])
    ions = []
    for s in range(NI):
        v = P["ion"][s] if improved else torch.exp(P["ion"][s])
        if improved:
            floor = torch.zeros_like(v, dtype=torch.bool)
            floor[2:-2] = True
            _record(floor & (v < 1))
            v = torch.where(floor & (v < 1), torch.ones_like(v), v)
        ions.append(v)
    if prm.use_ion_advection:
        e = _lsum(ions)
        out["ion"] = torch.stack(ions + [e])
    else:
        out["ion"] = state["ion"]
    return out


# --------------------------------------------------------------- helpers
def from_member(m, device="cpu", requires_grad=False):
    """(state, inputs) tensors of a synthetic.Member with one shared grid."""
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=device, dtype=torch.float64)  # noqa: E731
    state = {"nd": t(m.ndensity_s), "ion": t(m.idensity_s), "rho": t(m.rho[0]), "temp": t(m.temperature[0]),
             "vel": t(m.velocity), "ww": t(m.vert_vel)}
    if requires_grad:
        for v in state.values():
            v.requires_grad_(True)
    inp = {"ivel_up": t(m.ivel_up[0]), "eddy": t(m.eddy[0]), "cos_lat": t(m.cos_lat), "sza": t(m.sza),
           "mlat": t(m.mlat), "lbc": None if m.lbc is None else t(m.lbc),
           "grid": Grid(m.altitude, m.gravity, m.dalt_c, m.inv_r, device),
           "heating": None if m.heating is None else t(m.heating[0]),
           "heating_scale": None if m.heating_scale is None else t(m.heating_scale)}
    return state, inp


def to_member_arrays(out: dict) -> dict:
    """Step outputs as numpy arrays named like synthetic.Member fields."""
    n = lambda x: x.detach().cpu().numpy()  # noqa: E731
    return {"ndensity_s": n(out["nd"]), "idensity_s": n(out["ion"]), "rho": n(out["rho"])[None],
            "temperature": n(out["temp"])[None], "velocity": n(out["vel"]), "vert_vel": n(out["ww"]),
            "log_ns": n(out["log_ns"]), "ndensity": n(out["ndensity"])[None]}
