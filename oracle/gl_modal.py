"""CPU oracle for the single-direction time path (modal GL resolvent).

TEST INFRASTRUCTURE ONLY (same rules as ``oracle/gl_oracle.py``).  A plain FP64
NumPy restatement of the reference's ``python/src/green_laplace/modal_time.py``
(``reconstruct_unidirectional_modal_timeseries``, lines 26-399) and
``_eta20.py`` (``unidirectional_eta20``, lines 13-186).  Pinned against the
reference's MATLAB fixtures (``python/tests/fixtures/unidirectional_*.json``)
and outputs of the reference Python function on seeded records
(``tests/golden/modal_time.npz``, written by
``tests/golden/make_modal_golden.py``).

The record is a real time series eta1(t_n) of ``count`` uniform samples.  Its
positive-frequency DFT bins 1..B carry the first-order amplitudes; each bin's
frequency gives a dimensionless wavenumber q by the finite-depth dispersion
relation.  The amplitudes are spread onto a one-dimensional modal q-axis
(linear interpolation) in a joint (q, frequency-bin) array; the GL products
are evaluated in the joint (x, t) space by FFTs along both axes, and every
output frequency bin sums the GL node responses over the q-axis.
"""

from __future__ import annotations

import numpy as np

from . import gl_oracle as O

TINY = float(np.finfo(float).tiny)


def select_bins(values, times, order, energy_fraction, omega_max):
    """Record checks, DFT amplitudes and the retained band (``modal_time.py:46-99``)."""
    count = values.size
    dt = float(np.mean(np.diff(times)))
    period = count * dt
    pos = (count - 1) // 2
    cand = np.arange(1, pos + 1)
    coeffs = np.fft.fft(values) / count
    energy = np.abs(coeffs[cand]) ** 2
    total = float(np.sum(energy))
    if total == 0:
        raise ValueError("eta1 has no positive-frequency content")
    cum = np.cumsum(energy) / total
    top = int(cand[min(int(np.searchsorted(cum, energy_fraction)), cand.size - 1)])
    top = min(top, pos // order)
    if omega_max is not None:
        top = min(top, int(np.floor(omega_max * period / (2 * np.pi))))
    if top < 1:
        raise ValueError("the selected eta1 frequency band is empty")
    bins = np.arange(1, top + 1)
    omega = 2 * np.pi * bins / period
    amps = 2 * np.conj(coeffs[bins])
    base = np.zeros(count, dtype=complex)
    base[bins] = amps
    eta11 = np.real(np.fft.fft(base))
    return dict(count=count, dt=dt, period=period, bins=bins, omega=omega, amps=amps,
                eta11=eta11, energy=energy, total=total, top=top)


def modal_axis(points, parent, order, limit=None):
    """Symmetric q-axis of ``points`` nodes (``modal_time.py:363-372``)."""
    if limit is None:
        limit = (order + 0.05) * float(np.max(np.abs(parent))) / (1 - 2 / points)
    elif limit <= order * float(np.max(np.abs(parent))):
        raise ValueError("modal_limit must exceed the requested nonlinear output support")
    step = 2 * limit / points
    return np.arange(-points / 2, points / 2) * step, step


def deposit(amps, work_bins, q, axis, step, width):
    """Linear interpolation of each amplitude onto its two q-axis neighbours
    (``modal_time.py:375-386``); returns the joint array and the rms relative
    projection error."""
    pos = (q - axis[0]) / step
    lo = np.clip(np.floor(pos).astype(int), 0, axis.size - 2)
    hi = lo + 1
    w_hi = np.clip(pos - lo, 0.0, 1.0)
    w_lo = 1.0 - w_hi
    joint = np.zeros((axis.size, width), dtype=complex)
    np.add.at(joint, (lo, work_bins), amps * w_lo)
    np.add.at(joint, (hi, work_bins), amps * w_hi)
    mass = np.abs(amps) ** 2
    err = np.concatenate((np.abs(axis[lo] - q) / q, np.abs(axis[hi] - q) / q))
    wts = np.concatenate((mass * w_lo, mass * w_hi))
    rms = float(np.sqrt(np.sum(wts * err**2) / max(np.sum(wts), TINY)))
    return joint, rms


def to_field(spec, points):
    """(q, bin) spectrum -> (x, t) field (``modal_time.py:389-390``)."""
    return np.fft.fft(np.fft.ifft(spec, axis=0) * points, axis=1)


def to_spectrum(field, points):
    """(x, t) field -> (q, bin) spectrum (``modal_time.py:397-398``)."""
    return np.fft.fft(np.fft.ifft(field, axis=1), axis=0) / points


def node_sums(s, a, valid, scale, nodes, weights):
    """GL sums S = sum w/scale e^x (e^{-(s-a)tau} - e^{-(s+a)tau})/(2a),
    C = the same with + (tau = x/scale), and their a = 0 limits
    (``modal_time.py:401-416``)."""
    S = np.zeros_like(a)
    C = np.zeros_like(a)
    nz = valid & (a > 0)
    z = valid & (a == 0)
    av = a[nz]
    for x, w in zip(nodes, weights):
        tau = x / scale
        plus = w / scale * np.exp(x - (s - av) * tau)
        minus = w / scale * np.exp(x - (s + av) * tau)
        S[nz] += (plus - minus) / (2 * av)
        C[nz] += (plus + minus) / 2
        if np.any(z):
            b = w / scale * np.exp(x - s * tau)
            S[z] += b * tau
            C[z] += b
    return S, C


def modal_level(amps, bins, q, *, count, dt, depth, gravity, peak_q, rank, order, points, limit):
    """eta22 (and eta33) on one modal grid (``modal_time.py:217-360``).
    Returns (eta22, eta33 or None, projection rms)."""
    b0 = int(np.min(bins))
    wb = bins - b0
    wmax = int(np.max(wb))
    width = order * wmax + 1
    if width > count:
        raise ValueError("the nonlinear output band does not fit in the time record")
    axis, step = modal_axis(points, q, order, limit)
    joint_c, rms = deposit(amps, wb, q, axis, step, width)
    joint = np.fft.ifftshift(joint_c, axes=0)
    qs = np.fft.ifftshift(axis)
    qabs = np.abs(qs)
    sq = qs[:, None]
    sq2 = sq**2
    fstep = 2 * np.pi / (count * dt) * np.sqrt(depth / gravity)
    nu = ((b0 + np.arange(width)) * fstep)[None, :]
    snu = np.maximum(nu, TINY)

    def bank(mult):
        return to_field(joint * mult, points)

    v = bank(1.0)
    vn = bank(nu)
    vn2 = bank(nu**2)
    hx = bank(sq / snu)
    jx = bank(sq)
    rad = bank(sq2 / snu)
    sd_h = to_spectrum(2 * v * vn2 + vn**2 - hx**2, points)
    sk_h = to_spectrum(2 * v * rad + 2 * hx * jx, points)

    nodes, weights = O.gauss_laguerre(rank)
    pnu = np.sqrt(peak_q * np.tanh(peak_q))
    scale22 = np.sqrt(4 * peak_q * np.tanh(peak_q) - 2 * peak_q * np.tanh(2 * peak_q))
    ra = np.sqrt(qabs * np.tanh(qabs))
    aq = qabs * np.tanh(qabs)
    c22 = np.zeros(count, dtype=complex)
    for w2 in range(2 * wmax + 1):
        s = (2 * b0 + w2) * fstep
        valid = s > ra
        S, C = node_sums(s, ra, valid, scale22, nodes, weights)
        resp = np.zeros(points, dtype=complex)
        resp[valid] = (-aq[valid] * S[valid] * sd_h[valid, w2] + C[valid] * sk_h[valid, w2]) / (4 * depth)
        c22[2 * b0 + w2] = np.sum(resp)
    eta22 = np.fft.fft(c22)
    if order < 3:
        return eta22, None, rms

    lam2 = 2 * pnu - np.sqrt(2 * peak_q * np.tanh(2 * peak_q))
    lam3 = 3 * pnu - np.sqrt(3 * peak_q * np.tanh(3 * peak_q))
    inner_nu = (2 * b0 + np.arange(width)) * fstep
    e2 = np.zeros((points, width), dtype=complex)
    p2 = np.zeros_like(e2)
    for w2 in range(2 * wmax + 1):
        s = inner_nu[w2]
        valid = s > ra
        S, C = node_sums(s, ra, valid, lam2, nodes, weights)
        sd = sd_h[:, w2]
        sk = sk_h[:, w2]
        e2[valid, w2] = (-aq[valid] * S[valid] * sd[valid] + C[valid] * sk[valid]) / 4
        p2[valid, w2] = 1j * (C[valid] * sd[valid] - S[valid] * sk[valid]) / 4
    f = {"eta": v, "etax": bank(1j * sq), "phix": hx, "phiz": bank(-1j * nu),
         "phixz": bank(nu * sq), "phizz": bank(-1j * sq2 / snu), "phizzz": bank(-1j * sq2 * nu),
         "phitz": bank(-nu**2), "phitzz": bank(-sq2)}
    aq2 = aq[:, None]
    p = {"eta": to_field(e2, points), "etax": to_field(e2 * (1j * sq), points),
         "phix": to_field(p2 * (1j * sq), points), "phiz": to_field(p2 * aq2, points),
         "phizz": to_field(p2 * sq2, points),
         "phitz": to_field(p2 * (-1j * inner_nu[None, :]) * aq2, points)}
    k_pair = f["phix"] * p["etax"] + p["phix"] * f["etax"] - f["eta"] * p["phizz"] - p["eta"] * f["phizz"]
    k_dir = f["eta"] * f["phixz"] * f["etax"] - 0.5 * f["eta"] ** 2 * f["phizzz"]
    d_pair = f["eta"] * p["phitz"] + p["eta"] * f["phitz"] + f["phix"] * p["phix"] + f["phiz"] * p["phiz"]
    d_dir = 0.5 * f["eta"] ** 2 * f["phitzz"] + f["eta"] * (f["phix"] * f["phixz"] + f["phiz"] * f["phizz"])
    fk_h = to_spectrum(k_dir / 4 + k_pair / 2, points)
    fd_h = to_spectrum(d_dir / 4 + d_pair / 2, points)
    c33 = np.zeros(count, dtype=complex)
    for w3 in range(3 * wmax + 1):
        s = (3 * b0 + w3) * fstep
        valid = s > ra
        S, C = node_sums(s, ra, valid, lam3, nodes, weights)
        resp = np.zeros(points, dtype=complex)
        resp[valid] = (aq[valid] * S[valid] * fd_h[valid, w3] - 1j * C[valid] * fk_h[valid, w3]) / depth**2
        c33[3 * b0 + w3] = np.sum(resp)
    return eta22, np.fft.fft(c33), rms


def eta20(amps, omega, q, times, *, depth, gravity, rank=16, nx=128, ny=16):
    """Difference-frequency eta20 on a 2-D modal grid (``_eta20.py:13-151``)."""
    count = times.size
    dt = float(np.mean(np.diff(times)))
    bins = np.rint(omega * count * dt / (2 * np.pi)).astype(int)
    b0 = int(np.min(bins))
    wb = bins - b0
    span = int(np.max(wb))
    width = 2 * span + 1
    qx = q
    qy = np.zeros_like(q)
    ax_x, dx = _axis20(nx, qx, 2)
    ax_y, dy = _axis20(ny, qy, 2, (2.05 * float(np.max(q))) / (1.0 - 2.0 / ny))
    ix0, ix1, wx0, wx1 = _bracket(qx, ax_x, dx)
    iy0, iy1, wy0, wy1 = _bracket(qy, ax_y, dy)
    joint = np.zeros((ny, nx, width), dtype=complex)
    for ix, wx in ((ix0, wx0), (ix1, wx1)):
        for iy, wy in ((iy0, wy0), (iy1, wy1)):
            np.add.at(joint, (iy, ix, wb), amps * wx * wy)
    joint = np.fft.ifftshift(np.fft.ifftshift(joint, axes=0), axes=1)
    oqx, oqy = np.meshgrid(np.fft.ifftshift(ax_x), np.fft.ifftshift(ax_y))
    oq = np.hypot(oqx, oqy)
    ra = np.sqrt(oq * np.tanh(oq))
    qx3 = oqx[:, :, None]
    qy3 = oqy[:, :, None]
    q23 = qx3**2 + qy3**2
    fstep = 2 * np.pi / (count * dt) * np.sqrt(depth / gravity)
    nu3 = ((b0 + np.arange(width)) * fstep)[None, None, :]
    snu = np.maximum(nu3, TINY)

    def field(mult):
        return np.fft.fft(np.fft.ifft(np.fft.ifft(joint * mult, axis=0), axis=1) * (nx * ny), axis=2)

    one, dno, nuf = field(1.0), field(nu3**2), field(nu3)
    bx, by = field(qx3 / snu), field(qy3 / snu)
    qxf, qyf, rad = field(qx3), field(qy3), field(q23 / snu)
    fd = -dno * np.conj(one) - one * np.conj(dno) + nuf * np.conj(nuf) + bx * np.conj(bx) + by * np.conj(by)
    fk = (1j * rad * np.conj(one) - 1j * bx * np.conj(qxf) - 1j * by * np.conj(qyf)
          + 1j * qxf * np.conj(bx) + 1j * qyf * np.conj(by) - 1j * one * np.conj(rad))
    fd_h = np.fft.fft2(np.fft.ifft(fd, axis=2), axes=(0, 1)) / (nx * ny)
    fk_h = np.fft.fft2(np.fft.ifft(fk, axis=2), axes=(0, 1)) / (nx * ny)
    energy = np.abs(amps) ** 2
    esum = float(np.sum(energy))
    mean_q = float(np.sum(q * energy) / esum)
    dq = float(np.sqrt(2.0 * np.sum((q - mean_q) ** 2 * energy) / esum))
    if dq <= 64.0 * np.finfo(float).eps * max(1.0, float(np.max(q))):
        return np.zeros(count), dq
    nodes, weights = O.gauss_laguerre(rank)
    signed = np.concatenate((np.arange(0, span + 1), np.arange(-span, 0)))
    coeffs = np.zeros(count, dtype=complex)
    for k, sb in enumerate(signed):
        sig = sb * fstep
        valid = (oq > 0) & (ra > abs(sig))
        md = np.zeros_like(oq)
        mk = np.zeros(oq.shape, dtype=complex)
        av = ra[valid]
        for x, w in zip(nodes, weights):
            tau = x / dq
            plus = w / dq * np.exp(x - (av - sig) * tau)
            minus = w / dq * np.exp(x - (av + sig) * tau)
            md[valid] -= av * (plus + minus) / 4.0
            mk[valid] += 1j * (plus - minus) / 4.0
        resp = np.zeros(oq.shape, dtype=complex)
        resp[valid] = (md[valid] * fd_h[:, :, k][valid] + mk[valid] * fk_h[:, :, k][valid]) / (2.0 * depth)
        coeffs[sb % count] = np.sum(resp)
    coeffs = _hermitian(coeffs)
    return np.real(np.fft.fft(coeffs)), dq


def _axis20(count, parent, order, limit=0.0):
    if limit == 0.0:
        pm = float(np.max(np.abs(parent)))
        limit = (order + 0.05) * pm / (1.0 - 2.0 / count)
    step = 2.0 * limit / count
    return np.arange(-count / 2, count / 2) * step, step


def _bracket(value, axis, step):
    pos = (value - axis[0]) / step
    lo = np.clip(np.floor(pos).astype(int), 0, axis.size - 2)
    w_hi = np.clip(pos - lo, 0.0, 1.0)
    return lo, lo + 1, 1.0 - w_hi, w_hi


def _hermitian(c):
    out = c.copy()
    n = out.size
    for k in range(1, (n - 1) // 2 + 1):
        m = (out[k] + np.conj(out[-k])) / 2.0
        out[k] = m
        out[-k] = np.conj(m)
    out[0] = np.real(out[0])
    if n % 2 == 0:
        out[n // 2] = np.real(out[n // 2])
    return out


def modal_timeseries(eta1, time, *, depth, gravity=9.81, omega_max=None, energy_fraction=0.999,
                     quadrature_rank=8, order=3, modal_points=(2048, 4096, 8192, 16384, 32768, 65536),
                     modal_limit=None, relative_tolerance=1.0e-3, include_eta20=True, eta20_rank=16,
                     eta20_grid=(128, 16)):
    """``reconstruct_unidirectional_modal_timeseries`` (``modal_time.py:26-214``):
    returns (eta, components dict, audit dict)."""
    values = np.asarray(eta1, dtype=float).reshape(-1)
    times = np.asarray(time, dtype=float).reshape(-1)
    ladder = (modal_points,) if isinstance(modal_points, int) else tuple(int(v) for v in modal_points)
    sel = select_bins(values, times, order, energy_fraction, omega_max)
    q = O.dispersion_q(sel["omega"], depth, gravity)
    peak_q = float(q[int(np.argmax(np.abs(sel["amps"])))])
    prev = None
    converged = False
    levels = []
    e22 = e33 = None
    for pts in ladder:
        e22, e33, rms = modal_level(sel["amps"], sel["bins"], q, count=sel["count"], dt=sel["dt"],
                                    depth=depth, gravity=gravity, peak_q=peak_q,
                                    rank=quadrature_rank, order=order, points=pts, limit=modal_limit)
        cur = (e22,) if e33 is None else (e22, e33)
        if prev is not None:
            ch = tuple(float(np.linalg.norm(a - b) / np.linalg.norm(a)) for a, b in zip(cur, prev))
            converged = max(ch) <= relative_tolerance
        levels.append(pts)
        prev = cur
        if converged:
            break
    comps = {"eta11": sel["eta11"], "eta22": np.real(e22), "eta22_analytic": e22}
    eta = sel["eta11"] + np.real(e22)
    if e33 is not None:
        comps["eta33"] = np.real(e33)
        comps["eta33_analytic"] = e33
        eta = eta + np.real(e33)
    if include_eta20:
        e20, _ = eta20(sel["amps"], sel["omega"], q, times, depth=depth, gravity=gravity,
                       rank=eta20_rank, nx=eta20_grid[0], ny=eta20_grid[1])
        comps["eta20"] = e20
        eta = eta + e20
    audit = {"modal_points": levels[-1], "levels": levels, "converged": converged}
    return eta, comps, audit
