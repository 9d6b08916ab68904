"""Per-case parity bounds for FP64 engine-vs-oracle tests.

The reference's FFT graph zeroes spectral bins below a roundoff floor
(``python/src/green_laplace/_spectral.py:52-64``).  Which bins fall below it
depends on FFT roundoff, so two correct FP64 implementations of the graph
differ by more than FFT roundoff wherever bins sit near the floor.  The
oracle measures that spread on each case: it runs the same inputs a second
time with every 2-D FFT taken in the other axis order (same mathematics,
different roundoff) and compares the two answers.  The engine must then
agree with the oracle within ``SPREAD_FACTOR`` times that spread, and never
worse than the FP64 bar of 1e-12 where the spread is smaller.
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


def oracle_with_spread(run):
    """``run()`` -> {name: field}.  Returns the oracle's fields and, per field,
    the relative L2 change when only the oracle's FFT roundoff changes."""
    base = run()
    with swapped_fft_axes():
        alt = run()
    return base, {k: rel(alt[k], base[k]) for k in base}


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

    def run():
        oc = O.spectral_coefficients(args["order"], args["gravity"], args["depth"], args["a"],
                                     args["b"], args["kx"], args["ky"],
                                     options={"eta22_rank": args["eta22_rank"]})
        n = args["n"]
        if args["order"] == 3:
            kxg, kyg = O.fft_wavenumber_grid(args["lx"], args["ly"], n, n)
            s = O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], args["depth"],
                                args["lx"], args["ly"], n, n, args["t"])
            h = args["depth"]
            e, p, _ = O.order3(s, h * kxg, h * kyg, inner_rank=args["inner"],
                               outer_rank=args["outer"])
            ps = h * np.sqrt(args["gravity"] * h)
            full = {"eta33": h * e, "psi33": ps * p}
        else:
            r = O.spectral_surface(oc, args["lx"], args["ly"], n, n, args["t"])
            full = {k[:-5]: r[k] for k in r if k.endswith("_plus")}
        return {k: full[k] for k in args["names"]}

    return oracle_with_spread(run)


def oracle_fields_with_spread(order, gravity, depth, a, b, kx, ky, lx, ly, nx, ny, t,
                              eta22_rank=6):
    """All component fields of the two-stage oracle (complex ``*_plus`` and
    real parts) with their roundoff spreads."""
    from oracle import gl_oracle as O

    def run():
        oc = O.spectral_coefficients(order, gravity, depth, a, b, kx, ky,
                                     options={"eta22_rank": eta22_rank})
        r = O.spectral_surface(oc, lx, ly, nx, ny, t)
        return {k: v for k, v in r.items() if isinstance(v, np.ndarray)}

    return oracle_with_spread(run)
