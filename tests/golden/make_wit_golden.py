"""Golden vectors for the sector-44 WIT quartet sum (run where the reference exists).

* seeded small inputs run through the reference's own C++ binary
  (oracle/_ref/wit_eta44, built by `make -C oracle` from
  paper/order4/cpp/directional_eta4_openmp.cpp + its streaming patch); the
  non-zero bins of all five output fields are stored sparsely;
* the archived 256^2 field of the 382-mode paper input
  (paper/order4/inputs/field_n0382, paper/order4/data/wit_field_n0382.bin):
  the input file itself, per-field L2 norms and the 256 largest |eta| bins.

Usage: python tests/golden/make_wit_golden.py /path/to/reference
"""

from __future__ import annotations

import shutil
import subprocess
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "green-laplace-wave-reconstruction_b200"))
from gl_engine import wit  # noqa: E402


def small_case(seed: int, m: int, n: int, cases: int) -> wit.WitInput:
    rng = np.random.default_rng(seed)
    cells = [(x, y) for x in range(1, 6) for y in range(-4, 5)]
    pick = rng.choice(len(cells), size=m, replace=False)
    modes = np.array([cells[i] for i in sorted(pick)], dtype=np.int32)
    amps = (rng.standard_normal((cases, m)) + 1j * rng.standard_normal((cases, m))) * 0.01
    return wit.WitInput(modes=modes, amplitudes=amps, nx=n, ny=n, gravity=1.0, depth=1.0,
                        dkx=0.2, dky=0.2, threshold=1e-6)


def main(reference: Path) -> None:
    binary = ROOT / "oracle" / "_ref" / "wit_eta44"
    if not binary.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), f"REF={reference}"], check=True)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        cases_ = {"small10": (1, 10, 32, 2, 44), "small24": (2, 24, 64, 1, 44),
                  "s40_small12": (3, 12, 32, 2, 40), "s42_small12": (4, 12, 32, 2, 42)}
        for tag, (seed, m, n, cases, sector) in cases_.items():
            inp = small_case(seed, m, n, cases)
            fin, fout = Path(tmp) / f"{tag}.bin", Path(tmp) / f"{tag}.out"
            wit.write_dir4in(fin, inp)
            subprocess.run([str(binary), str(fin), str(fout), "--sector", str(sector)],
                           check=True, capture_output=True)
            out[f"{tag}/sector"] = np.array(sector)
            res = wit.read_dir4out(fout)
            out[f"{tag}/modes"] = inp.modes
            out[f"{tag}/amplitudes"] = inp.amplitudes
            out[f"{tag}/grid"] = np.array([inp.nx, inp.ny])
            nz = np.zeros(res.fields["eta"].shape, dtype=bool)
            for f in wit.FIELDS:
                nz |= res.fields[f] != 0
            idx = np.flatnonzero(nz)
            out[f"{tag}/bins"] = idx
            for f in wit.FIELDS:
                out[f"{tag}/{f}"] = res.fields[f].ravel()[idx]
            out[f"{tag}/counts"] = np.array([res.stats[k] for k in (
                "candidates", "kept", "near", "strict_zero_output", "strict_zero_intermediate")])
    # archived paper field
    order4 = reference / "paper" / "order4"
    shutil.copyfile(order4 / "inputs" / "field_n0382" / "directional_eta44_input.bin",
                    HERE / "wit_field_n0382_input.bin")
    arch = wit.read_dir4out(order4 / "data" / "wit_field_n0382.bin")
    for f in wit.FIELDS:
        out[f"n0382/norm_{f}"] = np.array(np.linalg.norm(arch.fields[f]))
    eta = arch.fields["eta"].ravel()
    top = np.argsort(np.abs(eta))[::-1][:256]
    out["n0382/top_bins"] = top
    out["n0382/top_eta"] = eta[top]
    out["n0382/top_psi"] = arch.fields["psi"].ravel()[top]
    out["n0382/counts"] = np.array([arch.stats[k] for k in (
        "candidates", "kept", "near", "strict_zero_output", "strict_zero_intermediate")])
    np.savez_compressed(HERE / "wit_reference.npz", **out)
    print({k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items() if "counts" in k})


if __name__ == "__main__":
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GL_REFERENCE")
    if not where:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set GL_REFERENCE)" % Path(__file__).name)
    main(Path(where))
