"""Generate tests/golden/order3_rank_pairs.npz (run in a container that has the reference).

The reference's ``green_laplace_order3(spectrum, qx, qy, inner_rank, outer_rank)``
(``python/src/green_laplace/_order3.py:18-26``) takes the inner and outer GL
ranks as arguments; its unified API fixes GL4/GL4.  This script evaluates it
at rank pairs with unequal inner and outer counts on one seeded 64 x 64
JONSWAP state (t = 0.3 s) and stores its dimensionless eta33 / psi33 fields
next to the state's mode list, so the oracle's ``order3`` and the engine can be
checked against the reference itself at those ranks.  The equal pairs (6, 6)
and (8, 8) are the ones the uneven batch workload runs.  The analytic spectrum fed to
the reference comes from the oracle's deposit restatement, which
``test_oracle_golden.py`` pins separately.

Usage: ``python tests/golden/make_rank_pairs.py /path/to/reference`` (or set
``GL_REFERENCE`` to the reference checkout).
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

RANK_PAIRS = [(6, 3), (8, 6), (4, 10), (12, 4), (6, 6), (8, 8), (10, 10)]
T = 0.3


def main(reference: Path) -> None:
    sys.path.insert(0, str(reference / "python" / "src"))
    sys.path.insert(0, str(ROOT / "green-laplace-wave-reconstruction_b200"))
    sys.path.insert(0, str(ROOT))
    from green_laplace import _order3 as ref_order3  # noqa: E402
    from gl_engine import seastate  # noqa: E402
    from oracle import gl_oracle  # noqa: E402  (deposit restatement only)

    st = seastate.jonswap_sea_state(n=64, length=160.0, depth=25.0, hs=2.0, tp=8.0, modes=20,
                                    seed=0, order=3)
    oc = gl_oracle.spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    s = gl_oracle.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], st.depth,
                                st.lx, st.ly, st.nx, st.ny, T)
    kxg, kyg = gl_oracle.fft_wavenumber_grid(st.lx, st.ly, st.nx, st.ny)
    out = {
        "meta": np.array([st.gravity, st.depth, st.lx, st.ly, st.nx, st.ny, T]),
        "modes": np.array([st.a, st.b, st.kx, st.ky]),
    }
    for inner, outer in RANK_PAIRS:
        e33, p33, audit = ref_order3.green_laplace_order3(s, st.depth * kxg, st.depth * kyg,
                                                          inner_rank=inner, outer_rank=outer)
        assert audit["inner_quadrature_rank"] == inner
        assert audit["outer_quadrature_rank"] == outer
        out[f"gl{inner}_{outer}/eta33"] = e33
        out[f"gl{inner}_{outer}/psi33"] = p33
    np.savez_compressed(HERE / "order3_rank_pairs.npz", **out)


if __name__ == "__main__":
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GL_REFERENCE")
    if not where:
        sys.exit("usage: make_rank_pairs.py REFERENCE_CHECKOUT (or set GL_REFERENCE)")
    main(Path(where))
