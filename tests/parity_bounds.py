"""Per-case parity bounds for FP64 engine-vs-oracle tests.

The reference's FFT graph zeroes spectral bins below a roundoff floor,
16 eps log2(Nx Ny) times the spectrum's peak
(``python/src/green_laplace/_spectral.py:52-64``), and multiplies node
spectra by cosh(sqrt(A) tau) responses that amplify whatever survives it.
Whether a bin within roundoff of that floor is kept is decided by roundoff,
so two correct FP64 implementations of the graph differ by more than FFT
roundoff.  The oracle measures that spread on each case by re-running the
same inputs with only roundoff-level changes:

* every 2-D FFT taken in the other axis order;
* the input spectrum scaled by 1 + 2^-52 and by 1 - 2^-52;
* the floor threshold moved by one ulp of the peak, i.e. scaled by
  1 + 1/(16 log2(Nx Ny)) and 1 - 1/(16 log2(Nx Ny)): a bin whose modulus lies
  within one ulp of the peak from the threshold has no roundoff-free
  decision, and any FFT decides it by its own roundoff (on deep-water states
  at high GL rank one such bin moves eta33 by 1e-5).

The spread is the largest relative L2 change over these runs.  The engine
must agree with the oracle within ``SPREAD_FACTOR`` times the spread, and
never worse than the FP64 bar of 1e-12 where the spread is smaller.
"""

from __future__ import annotations

import contextlib

import numpy as np
import numpy.fft as F

FP64_BAR = 1e-12
SPREAD_FACTOR = 4.0


def rel(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def max_rel(a, b) -> float:
    """max |a - b| / max |b| (the per-field max error next to the L2 one)."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@contextlib.contextmanager
def swapped_fft_axes():
    f2, i2 = F.fft2, F.ifft2
    F.fft2 = lambda a: F.fft(F.fft(a, axis=-2), axis=-1)
    F.ifft2 = lambda a: F.ifft(F.ifft(a, axis=-2), axis=-1)
    try:
        yield
    finally:
        F.fft2, F.ifft2 = f2, i2


@contextlib.contextmanager
def floor_threshold_scaled(factor: float):
    """The oracle's roundoff floor with its threshold times ``factor``."""
    from oracle import gl_oracle as O

    orig = O.zero_below_roundoff_floor

    def floor(spectrum, support):
        out = spectrum.copy()
        mags = np.abs(out[support])
        if mags.size == 0:
            return out
        peak = float(np.max(mags))
        if peak == 0.0:
            return out
        thr = 16.0 * O.EPS * max(1.0, np.log2(out.size)) * factor
        out[support & (np.abs(out) < thr * peak)] = 0.0
        return out

    O.zero_below_roundoff_floor = floor
    try:
        yield
    finally:
        O.zero_below_roundoff_floor = orig


@contextlib.contextmanager
def eta44_floor_threshold_scaled(factor: float):
    """The order-4 oracle's roundoff floor (``oracle/gl_eta44.py``) with its
    threshold times ``factor``."""
    from oracle import gl_eta44 as OE

    orig = OE.zero_suppress

    def zero_suppress(x, mask):
        x = np.where(mask, x, 0.0)
        peak = float(np.max(np.abs(x[mask]))) if np.any(mask) else 0.0
        thr = 16 * OE.EPS * max(1.0, np.log2(x.size)) * factor
        if peak:
            x = np.where(mask & (np.abs(x) < thr * peak), 0.0, x)
        return x

    OE.zero_suppress = zero_suppress
    try:
        yield
    finally:
        OE.zero_suppress = orig


PERTURBATIONS = ("axes", "scale+", "scale-", "floor+", "floor-")


def perturbed(run, kind: str, grid_points: int, floor_scaled=floor_threshold_scaled):
    """One roundoff-level re-run of ``run(scale)`` (see the module docstring);
    ``floor_scaled`` is the oracle's floor-threshold context."""
    eps = 2.0 ** -52
    ulp = 1.0 / (16.0 * np.log2(grid_points))
    if kind == "axes":
        with swapped_fft_axes():
            return run()
    if kind in ("scale+", "scale-"):
        return run(1.0 + eps if kind == "scale+" else 1.0 - eps)
    with floor_scaled(1.0 + ulp if kind == "floor+" else 1.0 - ulp):
        return run()


def oracle_with_spread(run, grid_points: int, floor_scaled=floor_threshold_scaled):
    """``run(scale)`` -> {name: field} for the input spectrum times ``scale``
    (``run()`` uses 1) on a grid of ``grid_points`` = Nx Ny bins.  Returns the
    oracle's fields and, per field, the largest relative L2 change over the
    roundoff-level perturbations."""
    base = run()
    alts = [perturbed(run, k, grid_points, floor_scaled) for k in PERTURBATIONS]
    return base, {k: max(rel(a[k], base[k]) for a in alts) for k in base}


def eta44_oracle_with_spread(call, spectrum):
    """``call(spectrum)`` -> field of the order-4 oracle.  Returns its field
    and its roundoff spread (same perturbations, the order-4 floor)."""
    def run(scale=1.0):
        return {"f": call(spectrum * scale) / scale}

    base, spread = oracle_with_spread(run, spectrum.size, eta44_floor_threshold_scaled)
    return base["f"], spread["f"]


def bound(spread: float) -> float:
    return max(FP64_BAR, SPREAD_FACTOR * spread)


def check_fields(got: dict, ref: dict, spread: dict, label: str = "") -> None:
    """Assert every field of ``ref`` within its per-case bound; print L2 and max."""
    for name in ref:
        e2, em = rel(got[name], ref[name]), max_rel(got[name], ref[name])
        b = bound(spread[name])
        print(f"{label} {name}: rel L2 {e2:.3e} max {em:.3e}; oracle spread {spread[name]:.3e};"
              f" bound {b:.3e}")
        assert e2 <= b, f"{label} {name}: {e2:.3e} > {b:.3e}"


def oracle_surface_with_spread(args: dict):
    """Oracle fields of one snapshot and their roundoff spread; ``args`` holds
    order, gravity, depth, a, b, kx, ky, eta22_rank, inner, outer, lx, ly, n,
    t and the component names to return.  A plain function of picklable
    arguments, so a spawned process pool can run cases side by side."""
    from oracle import gl_oracle as O

    def run(scale=1.0):
        oc = O.spectral_coefficients(args["order"], args["gravity"], args["depth"], args["a"],
                                     args["b"], args["kx"], args["ky"],
                                     options={"eta22_rank": args["eta22_rank"]})
        n = args["n"]
        h = args["depth"]
        kxg, kyg = O.fft_wavenumber_grid(args["lx"], args["ly"], n, n)
        s = scale * O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], h,
                                    args["lx"], args["ly"], n, n, args["t"])
        if args["order"] == 3:
            e, p, _ = O.order3(s, h * kxg, h * kyg, inner_rank=args["inner"],
                               outer_rank=args["outer"])
            ps = h * np.sqrt(args["gravity"] * h)
            full = {"eta33": h * e, "psi33": ps * p}
        else:
            r = O.evaluate_spectrum(s, h * kxg, h * kyg, depth=h, gravity=args["gravity"],
                                    order=args["order"], eta22_rank=args["eta22_rank"])
            full = {k[:-5]: r[k] for k in r if k.endswith("_plus")}
        # the perturbed runs are compared at the unperturbed scale
        return {k: full[k] / scale for k in args["names"]}

    if "perturbation" in args:  # one run of a spread, for a process pool
        kind = args["perturbation"]
        return run() if kind == "base" else perturbed(run, kind, args["n"] * args["n"])
    return oracle_with_spread(run, args["n"] * args["n"])


def oracle_fields_with_spread(order, gravity, depth, a, b, kx, ky, lx, ly, nx, ny, t,
                              eta22_rank=6):
    """All component fields of the two-stage oracle (complex ``*_plus`` and
    real parts) with their roundoff spreads."""
    from oracle import gl_oracle as O

    def run(scale=1.0):
        oc = O.spectral_coefficients(order, gravity, depth, a, b, kx, ky,
                                     options={"eta22_rank": eta22_rank})
        kxg, kyg = O.fft_wavenumber_grid(lx, ly, nx, ny)
        s = scale * O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], depth, lx,
                                    ly, nx, ny, t, oc["options"]["grid_tolerance"])
        r = O.evaluate_spectrum(s, depth * kxg, depth * kyg, depth=depth, gravity=gravity,
                                order=order, eta22_rank=eta22_rank)
        return {k: v / scale for k, v in r.items() if isinstance(v, np.ndarray)}

    return oracle_with_spread(run, nx * ny)
