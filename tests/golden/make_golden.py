"""Generate the golden vectors under tests/golden/ (run in a container that has the reference).

Two files are written:

* ``matlab_fixtures.npz`` -- the reference's own MATLAB-generated spatial
  fixtures (``python/tests/fixtures/directional_spatial_{eta22,order3,
  nonzero_time}.json``, MATLAB rev eaca157) re-packed as arrays;
* ``reference_python.npz`` -- outputs of the reference Python package
  (``python/src/green_laplace``) on seeded inputs: the fixture mode lists
  through the two-stage deposit (t=0 and t=0.7) and small JONSWAP sea states.

Usage: ``python tests/golden/make_golden.py /path/to/reference``
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def main(reference: Path) -> None:
    sys.path.insert(0, str(reference / "python" / "src"))
    sys.path.insert(0, str(ROOT / "green-laplace-wave-reconstruction_b200"))
    sys.path.insert(0, str(ROOT))
    from green_laplace import spatial as ref_spatial  # noqa: E402
    from green_laplace import _order3 as ref_order3  # noqa: E402
    from gl_engine import seastate  # noqa: E402
    from oracle import gl_oracle  # noqa: E402  (deposit restatement only)

    fixtures = {}
    for tag, name in (("eta22", "directional_spatial_eta22.json"),
                      ("order3", "directional_spatial_order3.json"),
                      ("time", "directional_spatial_nonzero_time.json")):
        data = json.loads((reference / "python" / "tests" / "fixtures" / name).read_text())
        for key, value in data.items():
            if key in ("x", "y", "matlab_source_revision"):
                continue
            fixtures[f"{tag}/{key}"] = np.asarray(value, dtype=float)
    np.savez_compressed(HERE / "matlab_fixtures.npz", **fixtures)

    cases = {}

    def run_reference(tag, s, qx, qy, depth, gravity, order, rank):
        pscale = depth * np.sqrt(gravity * depth)
        q = np.hypot(qx, qy)
        nu = np.sqrt(q * np.tanh(q))
        cases[f"{tag}/eta11"] = np.real(depth * np.fft.ifft2(s))
        psi_hat = np.zeros_like(s)
        psi_hat[nu > 0] = -1j * s[nu > 0] / nu[nu > 0]
        cases[f"{tag}/psi11"] = np.real(pscale * np.fft.ifft2(psi_hat))
        if order >= 2:
            e22, _ = ref_spatial._green_laplace_eta22(s, qx, qy, rank)
            p22, _ = ref_spatial._green_laplace_psi22(s, qx, qy,
                                                      allow_below_model_parent_domain=False)
            cases[f"{tag}/eta22"] = np.real(depth * e22)
            cases[f"{tag}/psi22"] = np.real(pscale * p22)
        if order >= 3:
            e33, p33, _ = ref_order3.green_laplace_order3(s, qx, qy)
            cases[f"{tag}/eta33"] = np.real(depth * e33)
            cases[f"{tag}/psi33"] = np.real(pscale * p33)
            cases[f"{tag}/eta33_plus"] = depth * e33
            cases[f"{tag}/psi33_plus"] = pscale * p33

    def two_stage(tag, order, g, h, a, b, kx, ky, lx, ly, nx, ny, t, rank):
        coeffs = gl_oracle.spectral_coefficients(order, g, h, a, b, kx, ky,
                                                 options={"eta22_rank": rank})
        s = gl_oracle.deposit_modes(coeffs["a"], coeffs["b"], coeffs["kx"], coeffs["ky"],
                                    coeffs["omega"], h, lx, ly, nx, ny, t)
        kxg, kyg = gl_oracle.fft_wavenumber_grid(lx, ly, nx, ny)
        meta = np.array([order, g, h, lx, ly, nx, ny, t, rank], dtype=float)
        cases[f"{tag}/meta"] = meta
        cases[f"{tag}/modes"] = np.stack([coeffs["a"], coeffs["b"], coeffs["kx"], coeffs["ky"]])
        run_reference(tag, s, h * kxg, h * kyg, h, g, order, rank)

    two_pi = 2.0 * np.pi
    # the fixture mode lists (python/tools/generate_matlab_fixtures.m:11-35)
    two_stage("fixture_t0", 3, 9.81, 1.0, [.01, .006], [0, -.002], [2, 3], [0, 1],
              two_pi, two_pi, 64, 64, 0.0, 6)
    two_stage("fixture_t07", 3, 9.81, 1.0, [.009, .005, .0035], [.001, -.0015, .0008],
              [2, 3, 4], [0, 1, -1], two_pi, two_pi, 64, 64, 0.7, 8)
    # seeded JONSWAP states
    st = seastate.small_order3(seed=3, n=64, modes=24)
    two_stage("jonswap64_o3", 3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
              st.lx, st.ly, st.nx, st.ny, 1.3, 4)
    st = seastate.jonswap_sea_state(n=64, length=256.0, depth=15.0, hs=1.5, tp=7.0, modes=40,
                                    seed=5, order=2)
    two_stage("jonswap64_o2", 2, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
              st.lx, st.ly, st.nx, st.ny, 0.0, 6)
    st = seastate.small_order3(seed=11, n=128, modes=96, depth=20.0, length=300.0)
    two_stage("jonswap128_o3", 3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
              st.lx, st.ly, st.nx, st.ny, 4.0, 4)
    for key in [k for k in cases if k.startswith("jonswap128_o3/") and
                k.split("/")[1] in ("eta11", "psi11", "eta22", "psi22", "eta33_plus",
                                    "psi33_plus")]:
        del cases[key]
    np.savez_compressed(HERE / "reference_python.npz", **cases)
    print("wrote", sorted(cases)[:5], "...", len(cases), "arrays")


if __name__ == "__main__":
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GL_REFERENCE")
    if not where:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set GL_REFERENCE)" % Path(__file__).name)
    main(Path(where))
