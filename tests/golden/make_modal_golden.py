"""Golden vectors of the reference's single-direction time path
(``python/src/green_laplace/modal_time.py``, ``_eta20.py``, ``temporal.py``).

Writes ``tests/golden/modal_time.npz`` with
* the reference's MATLAB fixtures ``python/tests/fixtures/
  unidirectional_modal_order3.json`` and ``unidirectional_time_eta20.json``;
* outputs of the reference Python function
  ``reconstruct_unidirectional_modal_timeseries`` on seeded records: an
  off-grid order-3 record through a modal ladder, an order-2 record with the
  eta20 difference-frequency term, and the on-grid two-mode case of the
  reference's own test (``python/tests/test_modal_time.py:9-69``).

Usage: ``python tests/golden/make_modal_golden.py /path/to/reference``
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _nu(q):
    return np.sqrt(q * np.tanh(q))


def main(reference: Path) -> None:
    sys.path.insert(0, str(reference / "python" / "src"))
    from green_laplace import reconstruct_unidirectional_modal_timeseries as run  # noqa: E402

    out = {}
    fx = reference / "python" / "tests" / "fixtures"
    for tag, name in (("m3", "unidirectional_modal_order3.json"),
                      ("e20", "unidirectional_time_eta20.json")):
        data = json.loads((fx / name).read_text())
        for key, value in data.items():
            if key == "matlab_source_revision":
                continue
            out[f"{tag}/{key}"] = np.asarray(value, dtype=float)

    def case(tag, eta1, time, **kw):
        res = run(eta1, time, **kw)
        out[f"{tag}/eta1"] = np.asarray(eta1, dtype=float)
        out[f"{tag}/time"] = np.asarray(time, dtype=float)
        out[f"{tag}/kw"] = np.array(json.dumps({k: (list(v) if isinstance(v, tuple) else v)
                                                for k, v in kw.items()}))
        for name, value in res.components.items():
            out[f"{tag}/{name}"] = np.asarray(value)
        out[f"{tag}/eta"] = res.eta
        out[f"{tag}/modal_points"] = np.array(res.audit["modal_points"])
        out[f"{tag}/converged"] = np.array(bool(res.audit["converged"]))
        out[f"{tag}/levels"] = np.array([lv["modal_points"] for lv in res.audit["levels"]])

    # off-grid order-3 record through a ladder (reference test shape)
    n, dt = 512, 0.2
    t = np.arange(n) * dt
    bins = np.array([20, 22, 24])
    amps = np.array([0.01, 0.006, 0.004])
    ph = np.array([0.2, -0.7, 1.1])
    eta1 = sum(a * np.cos(2 * np.pi * b * np.arange(n) / n + p) for a, b, p in zip(amps, bins, ph))
    case("ladder3", eta1, t, depth=1.0, omega_max=2 * np.pi * 24 / (n * dt) + 1e-12,
         energy_fraction=1.0, quadrature_rank=4, order=3, modal_points=(256, 512, 1024, 2048),
         relative_tolerance=1e-2, include_eta20=False)
    # seeded broadband order-3 record, default ladder start, GL rank 8
    rng = np.random.default_rng(11)
    n, dt = 256, 0.25
    t = np.arange(n) * dt
    kb = np.arange(8, 20)
    eta1 = sum(0.01 * rng.standard_normal() * np.cos(2 * np.pi * b * np.arange(n) / n + rng.uniform(0, 6))
               for b in kb)
    case("broad3", eta1, t, depth=4.0, energy_fraction=1.0, quadrature_rank=8, order=3,
         modal_points=(512, 1024), relative_tolerance=1e-12, include_eta20=True, eta20_rank=12,
         eta20_grid=(64, 16))
    # order 2 with eta20 on its default grid
    case("o2e20", eta1, t, depth=4.0, energy_fraction=0.999, quadrature_rank=6, order=2,
         modal_points=512, include_eta20=True)
    np.savez_compressed(HERE / "modal_time.npz", **out)
    print(sorted(out))


if __name__ == "__main__":
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GL_REFERENCE")
    if not where:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set GL_REFERENCE)" % Path(__file__).name)
    main(Path(where))
