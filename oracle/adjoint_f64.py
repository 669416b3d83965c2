"""Binary64 torch restatements of the operators the adjoint kernels
differentiate - TEST INFRASTRUCTURE ONLY.

Vectorised torch (float64) versions of the forward operators, so that
autograd gives the binary64 gradient the hand-written adjoint kernels are
checked against, and central finite differences can be taken in binary64:

  scalar_advection5     cpu_scalar_advection5_inplace with the whole-domain
                        lateral edits (src/cm1core/cuda_advection5.py:440-579,
                        :669), restated from oracle/advection_oracle.c
  open_fill_scalar      bcs on open sides (src/cm1core/cuda_sound3_open_boundary.py:249-335)
  pack                  the compact scalar into the padded interior
  tridiagonal_solve     a(k) x(k-1) + b(k) x(k) + c(k) x(k+1) = d(k) per column
  kessler_collection    autoconversion + accretion with the qc limiter
                        (cpu_gm1_kessler_local_inplace, src/cm1core/cuda_gm1_kessler_local.py:251)
  satadj1               the equation-set-1 saturation adjustment of the
                        Kessler driver (_cpu_satadj, src/cm1core/cuda_gm1_kessler_driver.py:337-428)
  warm_rain_transport   the reduced differentiable model the adjoint serves:
                        RK3 WENO5 transport of theta', qv, qc, qr under frozen
                        mass fluxes (the scalar RK of cuda_scalar_moist_rk.py),
                        then qc, qr clipped at zero, collection and satadj1,
                        repeated per large step

The arithmetic is the same formulas in binary64 (not binary32 one operation
at a time), which is what a gradient check wants.
"""

from __future__ import annotations

import torch

NG = 3
F5 = (2.0 / 60.0, -13.0 / 60.0, 47.0 / 60.0, 27.0 / 60.0, -3.0 / 60.0)
F3 = (-1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0)


def flx5(s1, s2, s3, s4, s5):
    return F5[0] * s1 + F5[1] * s2 + F5[2] * s3 + F5[3] * s4 + F5[4] * s5


def flx3(s1, s2, s3):
    return F3[0] * s1 + F3[1] * s2 + F3[2] * s3


def weno5(s1, s2, s3, s4, s5, eps):
    d1, e1 = s1 - 2 * s2 + s3, s1 - 4 * s2 + 3 * s3
    d2, e2 = s2 - 2 * s3 + s4, s2 - s4
    d3, e3 = s3 - 2 * s4 + s5, 3 * s3 - 4 * s4 + s5
    c = 13.0 / 12.0
    b1 = c * d1 * d1 + 0.25 * e1 * e1
    b2 = c * d2 * d2 + 0.25 * e2 * e2
    b3 = c * d3 * d3 + 0.25 * e3 * e3
    tau = torch.abs(b1 - b3)
    cap = torch.tensor(1.0e30, dtype=s1.dtype, device=s1.device)
    q1 = torch.minimum(tau / (b1 + eps), cap)
    q2 = torch.minimum(tau / (b2 + eps), cap)
    q3 = torch.minimum(tau / (b3 + eps), cap)
    g1, g2, g3 = float(torch.tensor(0.1, dtype=torch.float32)), float(torch.tensor(0.6, dtype=torch.float32)), \
        float(torch.tensor(0.3, dtype=torch.float32))
    w1, w2, w3 = g1 * (1 + q1 * q1), g2 * (1 + q2 * q2), g3 * (1 + q3 * q3)
    p1 = (1.0 / 3.0) * s1 - (7.0 / 6.0) * s2 + (11.0 / 6.0) * s3
    p2 = -(1.0 / 6.0) * s2 + (5.0 / 6.0) * s3 + (1.0 / 3.0) * s4
    p3 = (1.0 / 3.0) * s3 + (5.0 / 6.0) * s4 - (1.0 / 6.0) * s5
    return (w1 * p1 + w2 * p2 + w3 * p3) / (w1 + w2 + w3)


def upstrpd(s1, s2, s3, weps):
    dd = s2 - s1
    se = torch.where(dd >= 0, torch.full_like(dd, abs(weps)), torch.full_like(dd, -abs(weps)))
    rr = (s3 - s2) / (se + dd)
    cand = 1.0 / 6.0 + (1.0 / 3.0) * rr
    one = torch.ones_like(rr)
    phi = torch.clamp(torch.minimum(rr, torch.minimum(cand, one)), min=0.0)
    return s2 + phi * dd


def _recon(st, weno, eps):
    return weno5(*st, eps) if weno else flx5(*st)


def scalar_advection5(s, rru, rrv, rrw, c1, c2, rr0, gz, divx, *, nrk, dx, dy, dz, weps, obc, wflag=True):
    """Tendency (nk, nj, ni) of the padded scalar s (nk+2, nj+6, ni+6) under
    the fixed mass fluxes, all float64 tensors."""
    nk, nj, ni = divx.shape
    weno = bool(wflag and nrk == 3)
    ks, js, is_ = slice(1, nk + 1), slice(NG, NG + nj), slice(NG, NG + ni)
    # x faces F = NG .. NG+ni on interior rows and levels
    m = rru[ks, js, NG:NG + ni + 1]
    up = [s[ks, js, NG - 3 + q:NG - 3 + q + ni + 1] for q in range(5)]
    dn = [s[ks, js, NG + 2 - q:NG + 2 - q + ni + 1] for q in range(5)]
    fx = m * torch.where(m >= 0, _recon(up, weno, weps), _recon(dn, weno, weps))
    m = rrv[ks, NG:NG + nj + 1, is_]
    up = [s[ks, NG - 3 + q:NG - 3 + q + nj + 1, is_] for q in range(5)]
    dn = [s[ks, NG + 2 - q:NG + 2 - q + nj + 1, is_] for q in range(5)]
    fy = m * torch.where(m >= 0, _recon(up, weno, weps), _recon(dn, weno, weps))
    col = s[:, js, is_]
    faces = [torch.zeros_like(col[0])] * 2  # fz at padded levels 0 (unused) and 1
    wf = float(torch.tensor(weps, dtype=torch.float32))
    for k in range(2, nk + 1):
        m = rrw[k, js, is_]
        a1, a2 = c1[k - 1], c2[k - 1]

        def S(kk):
            return col[kk]

        def three(k1, k2, k3):
            return upstrpd(S(k1), S(k2), S(k3), wf) if weno else flx3(S(k1), S(k2), S(k3))

        def five(k1, st):
            return _recon([S(k1 + st * q) for q in range(5)], weno, weps)

        lin = a1 * S(k - 1) + a2 * S(k)
        if k == 2:
            r = torch.where(m >= 0, lin, three(k + 1, k, k - 1))
        elif k == nk:
            upw = (m > 0) if weno else (m >= 0)
            r = torch.where(upw, three(k - 2, k - 1, k), lin)
        elif k == 3:
            r = torch.where(m >= 0, three(k - 2, k - 1, k), five(k + 2, -1))
        elif k == nk - 1:
            r = torch.where(m >= 0, five(k - 3, 1), three(k + 1, k, k - 1))
        else:
            r = torch.where(m >= 0, five(k - 3, 1), five(k + 2, -1))
        faces.append(m * r)
    faces.append(torch.zeros_like(col[0]))  # level nk+1
    fz = torch.stack(faces)  # (nk+2, nj, ni)
    fw, fe = fx[:, :, :-1], fx[:, :, 1:]
    fs, fn = fy[:, :-1, :], fy[:, 1:, :]
    sv = s[ks, js, is_]
    uw, ue = rru[ks, js, NG:NG + ni], rru[ks, js, NG + 1:NG + ni + 1]
    vs, vn = rrv[ks, NG:NG + nj, is_], rrv[ks, NG + 1:NG + nj + 1, is_]
    ii = torch.arange(ni, device=s.device).view(1, 1, ni)
    jj = torch.arange(nj, device=s.device).view(1, nj, 1)
    iw = (ii == 0) & (((obc >> 0) & 15) == 2) & (uw >= 0)
    ie = (ii == ni - 1) & (((obc >> 4) & 15) == 2) & (ue <= 0)
    js_ = (jj == 0) & (((obc >> 8) & 15) == 2) & (vs >= 0)
    jn = (jj == nj - 1) & (((obc >> 12) & 15) == 2) & (vn <= 0)
    fw2 = torch.where(iw, fe, fw)
    fe2 = torch.where(ie, fw2, fe)
    fs2 = torch.where(js_, fn, fs)
    fn2 = torch.where(jn, fs2, fn)
    ax = (fw2 - fe2) / dx
    ay = (fs2 - fn2) / dy
    ax = torch.where(iw | ie, ax - sv * (ue - uw) / dx, ax)
    ay = torch.where(js_ | jn, ay - sv * (vn - vs) / dy, ay)
    az = (fz[1:nk + 1] - fz[2:nk + 2]) / dz
    total = ax + ay + az + sv * divx
    return total * rr0 * gz.unsqueeze(0)


def pack(q, ni, nj, nk):
    """The compact (nk, nj, ni) scalar into a zero padded array (nk+2, nj+6, ni+6)."""
    p = torch.zeros((nk + 2, nj + 2 * NG, ni + 2 * NG), dtype=q.dtype, device=q.device)
    return p.index_put((torch.arange(1, nk + 1, device=q.device).view(nk, 1, 1),
                        torch.arange(NG, NG + nj, device=q.device).view(1, nj, 1),
                        torch.arange(NG, NG + ni, device=q.device).view(1, 1, ni)), q)


def open_fill_scalar(p, ni, nj, nk):
    """bcs on all-open sides: west/east halo columns of rows y0-1..yl+1 from
    the edge columns, then south/north halo rows of columns x0-1..xl+1 from
    the edge rows (functional: returns a new tensor)."""
    x0, xl, y0, yl = NG, NG + ni - 1, NG, NG + nj - 1
    rows = slice(y0 - 1, yl + 2)
    lev = slice(1, nk + 1)
    dev = p.device

    def ar(lo, hi, axis):
        shape = [1, 1, 1]
        shape[axis] = -1
        return torch.arange(lo, hi, device=dev).view(*shape)

    q = p.clone()
    left = q[lev, rows, x0:x0 + 1].expand(-1, -1, NG)
    right = q[lev, rows, xl:xl + 1].expand(-1, -1, NG)
    q = q.index_put((ar(1, nk + 1, 0), ar(y0 - 1, yl + 2, 1), ar(x0 - NG, x0, 2)), left)
    q = q.index_put((ar(1, nk + 1, 0), ar(y0 - 1, yl + 2, 1), ar(xl + 1, xl + 1 + NG, 2)), right)
    cols = slice(x0 - 1, xl + 2)
    south = q[lev, y0:y0 + 1, cols].expand(-1, NG, -1)
    north = q[lev, yl:yl + 1, cols].expand(-1, NG, -1)
    q = q.index_put((ar(1, nk + 1, 0), ar(y0 - NG, y0, 1), ar(x0 - 1, xl + 2, 2)), south)
    q = q.index_put((ar(1, nk + 1, 0), ar(yl + 1, yl + 1 + NG, 1), ar(x0 - 1, xl + 2, 2)), north)
    return q


def tridiagonal_solve(a, b, c, d):
    """a, b, c, d of shape (n, columns); returns x (Thomas, float64)."""
    n = b.shape[0]
    cp, dp = [], []
    cprev = torch.zeros_like(b[0])
    dprev = torch.zeros_like(b[0])
    for k in range(n):
        lo = a[k] if k > 0 else torch.zeros_like(b[0])
        up = c[k] if k < n - 1 else torch.zeros_like(b[0])
        piv = b[k] - lo * cprev
        cprev = up / piv
        dprev = (d[k] - lo * dprev) / piv
        cp.append(cprev)
        dp.append(dprev)
    x = [None] * n
    x[n - 1] = dp[n - 1]
    for k in range(n - 2, -1, -1):
        x[k] = dp[k] - cp[k] * x[k + 1]
    return torch.stack(x)


def kessler_collection(qc, qr, dt):
    """(qc', qr') after autoconversion and accretion with the qc limiter."""
    zero = torch.zeros_like(qc)
    ar = torch.where(qc > 0, torch.clamp(0.001 * (qc - 0.001), min=0.0) * dt, zero)
    rp = torch.where(qr > 0, torch.clamp(qr, min=1e-300) ** 0.875, zero)
    cr = torch.where((qc > 0) & (qr > 0), 2.2 * qc * rp * dt, zero)
    t = ar + cr
    t = torch.where(t > qc, qc, t)
    return qc - t, qr + t


RD, CP, CPV, RV, XLV, CPL = 287.04, 1005.7, 1870.0, 461.5, 2501000.0, 4190.0


def _f32(x: float) -> float:
    return float(torch.tensor(x, dtype=torch.float32))


def sat_constants():
    """The binary32 constants of the Kessler operator, as binary64 numbers."""
    f = lambda v: torch.tensor(v, dtype=torch.float32)  # noqa: E731
    eps = f(RD) / f(RV)
    lv2 = f(CPL) - f(CPV)
    lv1 = f(XLV) + lv2 * f(273.15)
    return float(f(CP)), float(eps), float(lv1), float(lv2)


def satadj1(th0, pi0, pp3d, prs, th3d, qv, qc):
    """(th3d', qv', qc') after one equation-set-1 adjustment at the frozen
    pressure (the same branch order as the binary32 operator)."""
    cp, eps, lv1, lv2 = sat_constants()
    pisum = pi0 + pp3d
    tnew = (th0 + th3d) * pisum
    esl = torch.minimum(611.2 * torch.exp(17.67 * (tnew - 273.15) / (tnew - 29.65)), 0.5 * prs)
    qvs = eps * esl / (prs - esl)
    lhv = lv1 - lv2 * tnew
    square = (tnew - 29.65) ** 2
    dqv = (qvs - qv) / (1.0 + lhv * qvs * 17.67 * 243.5 / (cp * square))
    dqv = torch.where(qv + dqv < 1.0e-20, 1.0e-20 - qv, dqv)
    dqv = torch.minimum(dqv, torch.clamp(qc, min=0.0))
    return th3d - dqv * (lhv / (cp * pisum)), qv + dqv, qc - dqv


RK3_FRACTIONS = (1.0 / 3.0, 0.5, 1.0)


def warm_rain_transport(state, frozen, *, ni, nj, nk, dt, dx, dy, dz, weps, steps=1, obc=0x2222):
    """state: dict th3d, qv, qc, qr (nk, nj, ni) float64; frozen: rru, rrv,
    rrw (padded), c1, c2, rr0 (cells), gz (nj, ni), divx, th0, pi0, pp3d,
    prs (cells); weps one number or a dict per field.  Per large step: each
    scalar takes the three RK stages
    s_n = s_0 + (dt * f_n) T_n(s_{n-1}) with nrk = n (WENO5 at the third),
    its padded carrier open-filled before every tendency; then qc and qr
    clipped at zero (the transport's undershoots; the Kessler operators take
    non-negative water), collection and satadj1.  Returns the new state."""
    names = ("th3d", "qv", "qc", "qr")
    eps_of = weps if isinstance(weps, dict) else {n: weps for n in names}
    s = dict(state)
    for _ in range(steps):
        new = {}
        for n in names:
            cur = s[n]
            for nrk, frac in enumerate(RK3_FRACTIONS, start=1):
                padded = open_fill_scalar(pack(cur, ni, nj, nk), ni, nj, nk)
                ten = scalar_advection5(padded, frozen["rru"], frozen["rrv"], frozen["rrw"], frozen["c1"],
                                        frozen["c2"], frozen["rr0"], frozen["gz"], frozen["divx"], nrk=nrk, dx=dx,
                                        dy=dy, dz=dz, weps=eps_of[n], obc=obc)
                cur = s[n] + (dt * frac) * ten
            new[n] = cur
        qc, qr = kessler_collection(torch.clamp(new["qc"], min=0.0), torch.clamp(new["qr"], min=0.0), dt)
        th, qv, qc = satadj1(frozen["th0"], frozen["pi0"], frozen["pp3d"], frozen["prs"], new["th3d"], new["qv"], qc)
        s = {"th3d": th, "qv": qv, "qc": qc, "qr": qr}
    return s
