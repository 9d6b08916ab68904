"""CPU oracle for the fourth-order GL eta44 graph (no Stokes corrections).

TEST INFRASTRUCTURE ONLY (same rules as ``oracle/gl_oracle.py``).  A plain FP64
NumPy restatement of the reference's C++ executor
``paper/order4/cpp/gl_eta44_fftw.cpp`` (itself checked against the MATLAB
authority ``src/internal/finite_depth_directional_green_laplace_eta44_three_kernels.m``
to 1.79e-10 on the paper field).  The C++ cannot be built here (FFTW3 is not
in the image), so this restatement is pinned instead against the paper's
published GL-vs-WIT metrics on the 382-mode field
(``paper/order4/data/eta44_no_stokes_rank_metrics.csv``: raw relative L2
9.1656674905729 % / 4.20839343830129 % / 2.03486173251526 % at GL6/8/10).

Layout: arrays are ``[iy, ix]`` like the rest of the oracle (the C++ stores
x-major; the transforms are the same up to the order of the 1-D passes).
"""

from __future__ import annotations

import numpy as np

EPS = float(np.finfo(float).eps)
DMIN = float(np.finfo(float).tiny)


def _ifft(x):
    return np.fft.ifft2(x)


def _fft(x):
    return np.fft.fft2(x)


class Grid:
    """Per-bin tables, supports, shifts and scales (``gl_eta44_fftw.cpp:76-155``)."""

    def __init__(self, spectrum, dk, depth, peak, nodes, weights):
        n = spectrum.shape[0]
        self.n = n
        axis = np.where(np.arange(n) < n // 2, np.arange(n), np.arange(n) - n).astype(float)
        ax_x, ax_y = np.meshgrid(axis, axis)
        self.qx = depth * dk * ax_x
        self.qy = depth * dk * ax_y
        self.q = np.hypot(self.qx, self.qy)
        self.nu = np.sqrt(self.q * np.tanh(self.q))
        self.A = self.q * np.tanh(self.q)
        self.sqrtA = np.sqrt(self.A)
        self.safe = np.maximum(self.nu, DMIN)
        thr = 1e-13 * max(1.0, float(np.max(np.abs(spectrum))))
        self.support = np.abs(spectrum) > thr
        if np.any(self.qx[self.support] <= 0) or np.any(self.q[self.support] <= 0):
            raise ValueError("support")
        self.m2, self.m3, self.m4 = (self._power_mask(p) for p in (2, 3, 4))
        mn = float(np.min(self.nu[self.support]))
        self.shift2 = 0.5 * (mn + float(np.max(self.sqrtA[self.m2])) / 2)
        self.shift3 = 0.5 * (mn + float(np.max(self.sqrtA[self.m3])) / 3)
        self.shift4 = 0.5 * (mn + float(np.max(self.sqrtA[self.m4])) / 4)
        pn = np.sqrt(peak * np.tanh(peak))
        self.l2 = 2 * pn - np.sqrt(2 * peak * np.tanh(2 * peak))
        self.l3 = 3 * pn - np.sqrt(3 * peak * np.tanh(3 * peak))
        self.l4 = 4 * pn - np.sqrt(4 * peak * np.tanh(4 * peak))
        self.nodes = np.asarray(nodes, dtype=float)
        self.weights = np.asarray(weights, dtype=float)

    def _power_mask(self, p):
        f = _fft(self.support.astype(float)) ** p
        return np.real(_ifft(f)) > 0.5

    def sh_ch(self, t):
        sh = np.full_like(self.sqrtA, t)
        nz = self.sqrtA > 0
        sh[nz] = np.sinh(self.sqrtA[nz] * t) / self.sqrtA[nz]
        return sh, np.cosh(self.sqrtA * t)


def zero_suppress(x, mask):
    """Mask and roundoff floor (``gl_eta44_fftw.cpp:157-171``)."""
    x = np.where(mask, x, 0.0)
    s = float(np.max(np.abs(x[mask]))) if np.any(mask) else 0.0
    f = 16 * EPS * max(1.0, np.log2(x.size))
    if s:
        x = np.where(mask & (np.abs(x) < f * s), 0.0, x)
    return x


def first(g: Grid, s, order4=False):
    """First-order banks (``gl_eta44_fftw.cpp:188-290``)."""
    q2 = g.q * g.q
    f = {
        "eta": _ifft(s),
        "ex": _ifft(s * (1j * g.qx)), "ey": _ifft(s * (1j * g.qy)),
        "px": _ifft(s * (g.qx / g.safe)), "py": _ifft(s * (g.qy / g.safe)),
        "pz": _ifft(s * (-1j * g.nu)),
        "pxz": _ifft(s * (g.nu * g.qx)), "pyz": _ifft(s * (g.nu * g.qy)),
        "pzz": _ifft(s * (-1j * (q2 / g.safe))), "pzzz": _ifft(s * (-1j * (q2 * g.nu))),
        "ptz": _ifft(s * (-g.A)), "ptzz": _ifft(s * (-q2)),
        "pxz_t": _ifft(s * (-1j * (g.nu * g.nu * g.qx))),
        "pyz_t": _ifft(s * (-1j * (g.nu * g.nu * g.qy))),
        "pzzz_t": _ifft(s * (-(q2 * g.A))), "ptz_t": _ifft(s * (1j * (g.A * g.nu))),
    }
    if order4:
        phi = np.zeros_like(s)
        nz = g.nu > 0
        phi[nz] = -1j * s[nz] / g.nu[nz]
        f["pxzz"] = _ifft(phi * (1j * (g.qx * q2)))
        f["pyzz"] = _ifft(phi * (1j * (g.qy * q2)))
        f["pzzzz"] = _ifft(phi * (q2 * q2))
    return f


def pair(g: Grid, s, order4=False):
    """Inner GL loop and pair banks (``gl_eta44_fftw.cpp:299-529``)."""
    q2 = g.q * g.q
    nu = g.nu
    es = np.zeros_like(s)
    ets = np.zeros_like(s)
    ps = np.zeros_like(s)
    pts = np.zeros_like(s)
    ptts = np.zeros_like(s)
    mult = {
        "v": 1.0, "vn": nu, "vn2": nu * nu, "vn3": nu * nu * nu, "vn4": nu * nu * nu * nu,
        "hx": g.qx / g.safe, "hy": g.qy / g.safe, "jx": g.qx, "jy": g.qy, "ro": q2 / g.safe,
        "q2": q2, "q2n": q2 * nu, "njx": nu * g.qx, "njy": nu * g.qy,
        "n2jx": nu * nu * g.qx, "n2jy": nu * nu * g.qy,
    }
    for x, w in zip(g.nodes, g.weights):
        t = x / g.l2
        damp = s * np.exp(-t * (nu - g.shift2))
        b = {k: _ifft(damp * m) for k, m in mult.items()}
        v, vn, vn2, vn3, vn4 = b["v"], b["vn"], b["vn2"], b["vn3"], b["vn4"]
        hx, hy, jx, jy, ro = b["hx"], b["hy"], b["jx"], b["jy"], b["ro"]
        qq, q2n, njx, njy, n2jx, n2jy = b["q2"], b["q2n"], b["njx"], b["njy"], b["n2jx"], b["n2jy"]
        sd = 2 * v * vn2 + vn * vn - hx * hx - hy * hy
        sk = 2 * v * ro + 2 * (hx * jx + hy * jy)
        sds = 2 * v * vn3 + 4 * vn * vn2 - 2 * hx * jx - 2 * hy * jy
        sks = 2 * (vn * ro + v * qq) + 2 * (jx * jx + hx * njx + jy * jy + hy * njy)
        sdss = (2 * v * vn4 + 6 * vn * vn3 + 4 * vn2 * vn2
                - 2 * (jx * jx + hx * njx + jy * jy + hy * njy))
        skss = (2 * (vn2 * ro + 2 * vn * qq + v * q2n) + 6 * (jx * njx + jy * njy)
                + 2 * (hx * n2jx + hy * n2jy))
        sd, sk, sds, sks, sdss, skss = (zero_suppress(_fft(a), g.m2)
                                        for a in (sd, sk, sds, sks, sdss, skss))
        co = w * np.exp(x) / g.l2 * np.exp(-2 * g.shift2 * t) / 4
        sh, ch = g.sh_ch(t)
        es = es + co * (-g.A * sh * sd + ch * sk)
        ets = ets - 1j * co * (-g.A * sh * sds + ch * sks)
        ps = ps + 1j * co * (ch * sd - sh * sk)
        pts = pts + co * (ch * sds - sh * sks)
        ptts = ptts - 1j * co * (ch * sdss - sh * skss)
    es, ets, ps, pts, ptts = (zero_suppress(a, g.m2) for a in (es, ets, ps, pts, ptts))
    p = {
        "eta": _ifft(es), "ex": _ifft(es * (1j * g.qx)), "ey": _ifft(es * (1j * g.qy)),
        "eta_t": _ifft(ets), "ex_t": _ifft(ets * (1j * g.qx)), "ey_t": _ifft(ets * (1j * g.qy)),
        "px": _ifft(ps * (1j * g.qx)), "py": _ifft(ps * (1j * g.qy)), "pz": _ifft(ps * g.A),
        "pzz": _ifft(ps * q2), "ptz": _ifft(pts * g.A),
        "px_t": _ifft(pts * (1j * g.qx)), "py_t": _ifft(pts * (1j * g.qy)),
        "pzz_t": _ifft(pts * q2), "ptz_t": _ifft(ptts * g.A),
    }
    if order4:
        p["pxz"] = _ifft(ps * (1j * (g.qx * g.A)))
        p["pyz"] = _ifft(ps * (1j * (g.qy * g.A)))
        p["pzzz"] = _ifft(ps * (q2 * g.A))
    return p


def third_forcing(f, p):
    """Cubic forcing and its time derivative (``gl_eta44_fftw.cpp:548-566``)."""
    kp = (f["px"] * p["ex"] + f["py"] * p["ey"] + p["px"] * f["ex"] + p["py"] * f["ey"]
          - f["eta"] * p["pzz"] - p["eta"] * f["pzz"])
    kd = f["eta"] * (f["pxz"] * f["ex"] + f["pyz"] * f["ey"]) - 0.5 * f["eta"] * f["eta"] * f["pzzz"]
    dp = (f["eta"] * p["ptz"] + p["eta"] * f["ptz"] + f["px"] * p["px"] + f["py"] * p["py"]
          + f["pz"] * p["pz"])
    dd = (0.5 * f["eta"] * f["eta"] * f["ptzz"]
          + f["eta"] * (f["px"] * f["pxz"] + f["py"] * f["pyz"] + f["pz"] * f["pzz"]))
    kpt = (-f["ex"] * p["ex"] + f["px"] * p["ex_t"] - f["ey"] * p["ey"] + f["py"] * p["ey_t"]
           + p["px_t"] * f["ex"] + p["px"] * f["pxz"] + p["py_t"] * f["ey"] + p["py"] * f["pyz"]
           - f["pz"] * p["pzz"] - f["eta"] * p["pzz_t"] - p["eta_t"] * f["pzz"]
           - p["eta"] * f["ptzz"])
    kdt = (f["pz"] * (f["pxz"] * f["ex"] + f["pyz"] * f["ey"])
           + f["eta"] * (f["pxz_t"] * f["ex"] + f["pxz"] * f["pxz"] + f["pyz_t"] * f["ey"]
                         + f["pyz"] * f["pyz"])
           - f["eta"] * f["pz"] * f["pzzz"] - 0.5 * f["eta"] * f["eta"] * f["pzzz_t"])
    dpt = (f["pz"] * p["ptz"] + f["eta"] * p["ptz_t"] + p["eta_t"] * f["ptz"]
           + p["eta"] * f["ptz_t"] - f["ex"] * p["px"] + f["px"] * p["px_t"]
           - f["ey"] * p["py"] + f["py"] * p["py_t"] + f["ptz"] * p["pz"] + f["pz"] * p["ptz"])
    ddt = (f["eta"] * f["pz"] * f["ptzz"] - 0.5 * f["eta"] * f["eta"] * f["pzzz"]
           + f["pz"] * (f["px"] * f["pxz"] + f["py"] * f["pyz"] + f["pz"] * f["pzz"])
           + f["eta"] * (-f["ex"] * f["pxz"] + f["px"] * f["pxz_t"] - f["ey"] * f["pyz"]
                         + f["py"] * f["pyz_t"] + f["ptz"] * f["pzz"] + f["pz"] * f["ptzz"]))
    return kd / 4 + kp / 2, dd / 4 + dp / 2, kdt / 4 + kpt / 2, ddt / 4 + dpt / 2


def third(g: Grid, s, only=None, eta_t=False):
    """Nested order-3 state (``gl_eta44_fftw.cpp:537-637``).  With ``eta_t``
    also the third-order eta_t field of the MATLAB graph
    (``finite_depth_directional_nested_green_laplace_eta33.m:127-131, 165-166``),
    accumulated from the time-derivative forcings and floored like its
    siblings."""
    es = np.zeros_like(s)
    ps = np.zeros_like(s)
    pts = np.zeros_like(s)
    ets = np.zeros_like(s)
    for oi, (x, w) in enumerate(zip(g.nodes, g.weights)):
        if only is not None and oi != only:
            continue
        t = x / g.l3
        damp = s * np.exp(-t * (g.nu - g.shift3))
        f = first(g, damp)
        p = pair(g, damp)
        fk, fd, fkt, fdt = (zero_suppress(_fft(a), g.m3) for a in third_forcing(f, p))
        co = w * np.exp(x) / g.l3 * np.exp(-3 * g.shift3 * t)
        sh, ch = g.sh_ch(t)
        es = es + co * (g.A * sh * fd - 1j * ch * fk)
        ps = ps + co * (-1j * ch * fd - sh * fk)
        pts = pts + co * (-1j * ch * fdt - sh * fkt)
        if eta_t:
            ets = ets + co * (g.A * sh * fdt - 1j * ch * fkt)
    es, ps, pts = (zero_suppress(a, g.m3) for a in (es, ps, pts))
    q2 = g.q * g.q
    out = {
        "eta": _ifft(es), "ex": _ifft(es * (1j * g.qx)), "ey": _ifft(es * (1j * g.qy)),
        "px": _ifft(ps * (1j * g.qx)), "py": _ifft(ps * (1j * g.qy)), "pz": _ifft(ps * g.A),
        "pzz": _ifft(ps * q2), "pzt": _ifft(pts * g.A),
    }
    if eta_t:
        out["eta_t"] = _ifft(zero_suppress(ets, g.m3))
    return out


def order4_forcing(f, p, t):
    """Partitions 31, 22, 211, 1111 of the quartic forcing (``gl_eta44_fftw.cpp:712-735``)."""
    k31, d31 = order4_forcing_31(f, t)
    kb, db = order4_forcing_base(f, p)
    return k31 / 2 + kb, d31 / 2 + db


def order4_forcing_31(f, t):
    """Partition 31 of the quartic forcing (``gl_eta44_fftw.cpp:716-717``)."""
    k31 = (f["px"] * t["ex"] + f["py"] * t["ey"] + t["px"] * f["ex"] + t["py"] * f["ey"]
           - f["eta"] * t["pzz"] - t["eta"] * f["pzz"])
    d31 = (f["eta"] * t["pzt"] + t["eta"] * f["ptz"] + f["px"] * t["px"] + f["py"] * t["py"]
           + f["pz"] * t["pz"])
    return k31, d31


def order4_forcing_base(f, p):
    """Partitions 22, 211 and 1111 of the quartic forcing, weighted
    (``gl_eta44_fftw.cpp:721-731``)."""
    k22 = p["px"] * p["ex"] + p["py"] * p["ey"] - p["eta"] * p["pzz"]
    d22 = p["eta"] * p["ptz"] + 0.5 * (p["px"] * p["px"] + p["py"] * p["py"] + p["pz"] * p["pz"])
    fe = f["eta"]
    k211 = (fe * (f["pxz"] * p["ex"] + f["pyz"] * p["ey"])
            + (fe * p["pxz"] + p["eta"] * f["pxz"]) * f["ex"]
            + (fe * p["pyz"] + p["eta"] * f["pyz"]) * f["ey"]
            - 0.5 * fe * fe * p["pzzz"] - fe * p["eta"] * f["pzzz"])
    d211 = (0.5 * fe * fe * p["pzz_t"] + fe * p["eta"] * f["ptzz"]
            + f["px"] * (fe * p["pxz"] + p["eta"] * f["pxz"])
            + f["py"] * (fe * p["pyz"] + p["eta"] * f["pyz"])
            + f["pz"] * (fe * p["pzz"] + p["eta"] * f["pzz"])
            + p["px"] * (fe * f["pxz"]) + p["py"] * (fe * f["pyz"]) + p["pz"] * (fe * f["pzz"]))
    k1111 = (0.5 * fe * fe * (f["pxzz"] * f["ex"] + f["pyzz"] * f["ey"])
             - fe * fe * fe * f["pzzzz"] / 6)
    d1111 = (fe * fe * fe * f["pzzz_t"] / 6
             + 0.5 * fe * fe * (f["px"] * f["pxzz"] + f["py"] * f["pyzz"] + f["pz"] * f["pzzz"])
             + 0.5 * fe * fe * (f["pxz"] * f["pxz"] + f["pyz"] * f["pyz"] + f["pzz"] * f["pzz"]))
    return k1111 / 8 + k211 / 4 + k22 / 2, d1111 / 8 + d211 / 4 + d22 / 2


def order4_contact(f, p, t):
    """Surface Taylor contact of psi44 and its time derivative
    (``src/internal/finite_depth_directional_green_laplace_eta44_three_kernels.m:221-241``).
    First-order aliases: eta_t = phiz (pz), phiz_t = phitz (ptz),
    phizz_t = phitzz (ptzz); pair phiz_t = phitz (ptz)."""
    fe, fet = f["eta"], f["pz"]
    contact = (0.5 * fe * t["pz"] + 0.5 * p["eta"] * p["pz"] + 0.5 * t["eta"] * f["pz"]
               + 0.125 * fe * fe * p["pzz"] + 0.25 * fe * p["eta"] * f["pzz"]
               + (1.0 / 48.0) * fe * fe * fe * f["pzzz"])
    contact_t = (0.5 * (fet * t["pz"] + fe * t["pzt"])
                 + 0.5 * (p["eta_t"] * p["pz"] + p["eta"] * p["ptz"])
                 + 0.5 * (t["eta_t"] * f["pz"] + t["eta"] * f["ptz"])
                 + 0.125 * (2 * fe * fet * p["pzz"] + fe * fe * p["pzz_t"])
                 + 0.25 * (fet * p["eta"] * f["pzz"] + fe * p["eta_t"] * f["pzz"]
                           + fe * p["eta"] * f["ptzz"])
                 + (1.0 / 48.0) * (3 * fe * fe * fet * f["pzzz"] + fe * fe * fe * f["pzzz_t"]))
    return contact, contact_t


def eta44_psi44(spectrum, dk, depth, peak, nodes, weights):
    """Dimensionless analytic eta44 and surface psi44 fields
    (``src/gl_pure_sum_order4.m:1-15`` ->
    ``finite_depth_directional_green_laplace_eta44_three_kernels.m:52-178``):
    per outer node the eta44 forcing of ``eta44`` plus the contact spectra
    (masked, floored), the surface forcings fk + A c, fd - c_t and
    psi += coef (-i cosh fd_s - sinh/sqrt(A) fk_s); psi44 is masked to the
    quartic support (no final floor, as in the MATLAB graph)."""
    g = Grid(spectrum, dk, depth, peak, nodes, weights)
    out = np.zeros_like(spectrum)
    psi = np.zeros_like(spectrum)
    for x, w in zip(g.nodes, g.weights):
        tm = x / g.l4
        damp = spectrum * np.exp(-tm * (g.nu - g.shift4))
        t = third(g, damp, eta_t=True)
        f = first(g, damp, True)
        p = pair(g, damp, True)
        fk, fd = (zero_suppress(_fft(a), g.m4) for a in order4_forcing(f, p, t))
        c, ct = (zero_suppress(_fft(a), g.m4) for a in order4_contact(f, p, t))
        co = w * np.exp(x) / g.l4 * np.exp(-4 * g.shift4 * tm)
        sh, ch = g.sh_ch(tm)
        out = out + co * (g.A * sh * fd - 1j * ch * fk)
        psi = psi + co * (-1j * ch * (fd - ct) - sh * (fk + g.A * c))
    out = zero_suppress(out, g.m4)
    psi = np.where(g.m4, psi, 0.0)
    return _ifft(out), _ifft(psi)


def eta44(spectrum, dk, depth, peak, nodes, weights, outer_subset=None):
    """Dimensionless analytic eta44 field (``gl_eta44_fftw.cpp:639-749``).

    ``spectrum`` is the N^2-scaled analytic first-order spectrum ``[iy, ix]``.
    """
    g = Grid(spectrum, dk, depth, peak, nodes, weights)
    out = np.zeros_like(spectrum)
    for oi, (x, w) in enumerate(zip(g.nodes, g.weights)):
        if outer_subset is not None and oi not in outer_subset:
            continue
        tm = x / g.l4
        damp = spectrum * np.exp(-tm * (g.nu - g.shift4))
        t = third(g, damp)
        f = first(g, damp, True)
        p = pair(g, damp, True)
        fk, fd = (zero_suppress(_fft(a), g.m4) for a in order4_forcing(f, p, t))
        co = w * np.exp(x) / g.l4 * np.exp(-4 * g.shift4 * tm)
        sh, ch = g.sh_ch(tm)
        out = out + co * (g.A * sh * fd - 1j * ch * fk)
    out = zero_suppress(out, g.m4)
    return _ifft(out)


def eta44_partial(spectrum, dk, depth, peak, nodes, weights, outer_subset):
    """Order-4 spectrum accumulated over ``outer_subset`` only, before the final
    floor (the quantity one GPU contributes when outer nodes are sharded)."""
    g = Grid(spectrum, dk, depth, peak, nodes, weights)
    out = np.zeros_like(spectrum)
    for oi, (x, w) in enumerate(zip(g.nodes, g.weights)):
        if oi not in outer_subset:
            continue
        tm = x / g.l4
        damp = spectrum * np.exp(-tm * (g.nu - g.shift4))
        t = third(g, damp)
        f = first(g, damp, True)
        p = pair(g, damp, True)
        fk, fd = (zero_suppress(_fft(a), g.m4) for a in order4_forcing(f, p, t))
        co = w * np.exp(x) / g.l4 * np.exp(-4 * g.shift4 * tm)
        sh, ch = g.sh_ch(tm)
        out = out + co * (g.A * sh * fd - 1j * ch * fk)
    return out, g.m4


def eta44_split_part(spectrum, dk, depth, peak, nodes, weights, outer, part):
    """One part of the reference's split mode (``gl_eta44_fftw.cpp:639-749``
    with OUTER4_INDEX = ``outer``, PART_INDEX = ``part``): outer node
    ``outer`` alone; ``part`` -2 every partition, -1 the base partitions 22,
    211, 1111 (no third state), t >= 0 partition 31 with the third state of
    third-level node t alone.  The part's spectrum gets its own final floor
    and transform; the reference's merger sums the parts' fields."""
    g = Grid(spectrum, dk, depth, peak, nodes, weights)
    x, w = g.nodes[outer], g.weights[outer]
    tm = x / g.l4
    damp = spectrum * np.exp(-tm * (g.nu - g.shift4))
    include31 = part == -2 or part >= 0
    include_base = part in (-2, -1)
    f = first(g, damp, True)
    k = d = 0.0
    if include31:
        t = third(g, damp, only=part if part >= 0 else None)
        k31, d31 = order4_forcing_31(f, t)
        k, d = k + k31 / 2, d + d31 / 2
    if include_base:
        p = pair(g, damp, True)
        kb, db = order4_forcing_base(f, p)
        k, d = k + kb, d + db
    fk, fd = (zero_suppress(_fft(a), g.m4) for a in (k, d))
    co = w * np.exp(x) / g.l4 * np.exp(-4 * g.shift4 * tm)
    sh, ch = g.sh_ch(tm)
    out = co * (g.A * sh * fd - 1j * ch * fk)
    return _ifft(zero_suppress(out, g.m4))


def eta44_finalize(out_sum, quartic_mask):
    """Final floor and inverse transform of a summed order-4 spectrum."""
    return _ifft(zero_suppress(out_sum, quartic_mask))


def spectrum_from_wit_input(modes, amplitude, n, depth):
    """Deposit s = n^2 c / h at (my, mx) (``paper/order4/prepare_order4_inputs.m:12-16``)."""
    s = np.zeros((n, n), dtype=complex)
    for (mx, my), c in zip(modes, amplitude):
        s[my % n, mx % n] = n * n * c / depth
    return s
