"""Per-node FP32 error table of the order-3 graph (measurement on the oracle).

Test and measurement infrastructure, not part of the engine: it runs the
oracle's FP64 restatement of ``green_laplace_order3``
(``python/src/green_laplace/_order3.py:18-148``) on the 1024^2 order-3
workload (h = 30 m, L = 1024 m, 4096 JONSWAP modes, Hs = 3 m, seed 0, t = 0)
once in FP64 and then once per GL node with only that node's 2-D transforms
in complex64 (inputs rounded to complex64, FP32 FFT, result widened back).
Everything else keeps FP64, including the reference's roundoff floor
(``_spectral.py:52-64``: max-reduce and threshold in FP64).  A node is

* an inner node (j, i): the 12 multiplier-bank inverse transforms and the 4
  product forward transforms of outer node j's inner GL node i
  (``_order3.py:196-252``), or
* an outer node j: its 12 first-order and 9 pair-field inverse transforms and
  its 4 forcing forward transforms (``_order3.py:54-134``).

For each node the table lists the output amplification the node's spectra
meet -- max over the output support of cosh(sqrt(A) tau) e^{-n c tau}, with
tau = x / lambda and c the balance shift (n = 2 for inner, 3 for outer
nodes), times the node's coefficient e^{x} w / lambda -- and the relative L2
and max error of eta33 and psi33 against the all-FP64 oracle.  A row below
the bar admits that node to FP32 by itself; summed rows bound a set.

Usage: ``python oracle/node_precision.py [--workers 8] [--out FILE.md]``.
"""

from __future__ import annotations

import argparse
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "green-laplace-wave-reconstruction_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def _ffts32():
    def ifft2(x):
        return np.fft.ifft2(np.asarray(x, dtype=np.complex64)).astype(np.complex128)

    def fft2(x):
        return np.fft.fft2(np.asarray(x, dtype=np.complex64)).astype(np.complex128)

    return ifft2, fft2


def _case():
    from gl_engine import seastate
    from oracle import gl_oracle as O

    st = seastate.config2(0)
    oc = O.spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    s = O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], st.depth, st.lx,
                        st.ly, st.nx, st.ny, 0.0)
    kxg, kyg = O.fft_wavenumber_grid(st.lx, st.ly, st.nx, st.ny)
    return s, st.depth * kxg, st.depth * kyg


def _run(node):
    """node None: all FP64; ("inner", j, i) or ("outer", j): that node in FP32."""
    from oracle import gl_oracle as O

    s, qx, qy = _case()

    def ffts_for(j, i):
        if node is not None:
            if node[0] == "inner" and node[1] == j and node[2] == i:
                return _ffts32()
            if node[0] == "outer" and node[1] == j and i is None:
                return _ffts32()
        return np.fft.ifft2, np.fft.fft2

    e, p, audit = O.order3(s, qx, qy, ffts_for=ffts_for)
    return node, e, p, audit


def _amplification(audit, node, qx, qy, s):
    from oracle import gl_oracle as O

    g = O.Geometry(qx, qy)
    support = O.support_of(s)
    hat = np.fft.fft2(support.astype(float))
    s2 = np.real(np.fft.ifft2(hat**2)) > 0.5
    s3 = np.real(np.fft.ifft2(hat**3)) > 0.5
    if node[0] == "inner":
        x, w = O.gauss_laguerre(4)[0][node[2]], O.gauss_laguerre(4)[1][node[2]]
        lam, c, n, sup = audit["inner_scale"], audit["inner_balance_shift"], 2, s2
    else:
        x, w = O.gauss_laguerre(4)[0][node[1]], O.gauss_laguerre(4)[1][node[1]]
        lam, c, n, sup = audit["outer_scale"], audit["outer_balance_shift"], 3, s3
    tau = x / lam
    amp = np.cosh(g.sqrt_a[sup] * tau) * np.exp(-n * c * tau)
    return float(tau), float(amp.max()), float(amp.max() * np.exp(x) * w / lam)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def max_rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--out", type=Path, default=None)
    args = ap.parse_args(argv)
    nodes = [("inner", j, i) for j in range(4) for i in range(4)] + [("outer", j) for j in range(4)]
    t0 = time.time()
    with mp.get_context("spawn").Pool(args.workers) as pool:
        results = pool.map(_run, [None] + nodes)
    base = results[0]
    _, e0, p0, audit = base
    s, qx, qy = _case()
    lines = [
        "| node | tau | max cosh(sqrt(A) tau) e^(-n c tau) | x coef | eta33 rel L2 | eta33 max | "
        "psi33 rel L2 | psi33 max |",
        "|---|---|---|---|---|---|---|---|",
    ]
    rows = []
    for node, e, p, _ in results[1:]:
        tau, amp, ampc = _amplification(audit, node, qx, qy, s)
        name = f"inner (j={node[1]}, i={node[2]})" if node[0] == "inner" else f"outer j={node[1]}"
        row = (name, tau, amp, ampc, rel(e, e0), max_rel(e, e0), rel(p, p0), max_rel(p, p0))
        rows.append(row)
        lines.append("| %s | %.3f | %.3e | %.3e | %.2e | %.2e | %.2e | %.2e |" % row)
    text = "\n".join(lines)
    print(text)
    print(f"({time.time() - t0:.0f} s, {args.workers} workers)")
    if args.out:
        args.out.write_text(text + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
