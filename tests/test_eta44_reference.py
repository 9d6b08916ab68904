"""Field-level pin of the order-4 eta44 against the reference's own executor.

``oracle/Makefile`` builds ``paper/order4/cpp/gl_eta44_fftw.cpp`` unchanged
into ``oracle/_ref/gl_eta44_fftw`` against ``oracle/fftw_shim`` (this
project's implementation of the FFTW3 calls it makes).  Its transforms differ
from FFTW's by roundoff, so it is compared with the CPU restatement
(``oracle/gl_eta44.py``) and with the engine within the restatement's own
roundoff spread (``parity_bounds``): whole runs at GL ranks 3..10 and the
split mode's parts (``OUTER4_INDEX [PART_INDEX]``).
"""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from gl_engine import eta44 as E44
from oracle import gl_eta44 as OE
from oracle import gl_oracle as O
from parity_bounds import bound, eta44_oracle_with_spread

REF_BIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "gl_eta44_fftw"

needs_ref = pytest.mark.skipif(not REF_BIN.exists(),
                               reason="oracle/_ref/gl_eta44_fftw not built (needs a reference "
                                      "checkout: python __graft_entry__.py build)")


def _state(n, seed, count, dk):
    rng = np.random.default_rng(seed)
    cells = [(x, y) for x in range(1, 7) for y in range(-4, 5)]
    pick = rng.choice(len(cells), size=count, replace=False)
    modes = np.array([cells[i] for i in pick])
    c = 0.02 * (rng.standard_normal(count) + 1j * rng.standard_normal(count))
    return E44.spectrum_from_modes(modes, c, n, 1.0), dk


def _reference(tmp_path, s, dk, peak, rank, *split):
    nodes, weights = O.gauss_laguerre(rank)
    inp, out = tmp_path / "in.bin", tmp_path / f"out_{rank}_{'_'.join(map(str, split))}.bin"
    E44.write_glrti(inp, E44.GlInput(n=s.shape[0], dk=dk, depth=1.0, peak_depth=peak,
                                     rules={rank: (nodes, weights)}, spectrum=s))
    r = subprocess.run([str(REF_BIN), str(inp), str(out), str(rank), "4", *map(str, split)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "CPP_GL_ETA44_DONE" in r.stderr
    got = E44.read_gle44(out)
    assert got["n"] == s.shape[0] and got["rank"] == rank
    return got["field"], nodes, weights


@needs_ref
@pytest.mark.parametrize("n,seed,count,dk,peak,rank", [
    (32, 6, 4, 0.25, 1.0, 3),
    (32, 6, 4, 0.25, 1.0, 4),
    (32, 7, 8, 0.25, 1.1, 6),
    (32, 8, 8, 0.3, 1.0, 10),
])
def test_restatement_matches_reference_executor(tmp_path, n, seed, count, dk, peak, rank):
    s, dk = _state(n, seed, count, dk)
    ref, nodes, weights = _reference(tmp_path, s, dk, peak, rank)
    want, spread = eta44_oracle_with_spread(
        lambda x: OE.eta44(x, dk, 1.0, peak, nodes, weights), s)
    err = np.linalg.norm(ref - want) / np.linalg.norm(want)
    print(f"rank {rank}: reference executor vs restatement {err:.3e}; spread {spread:.3e}")
    assert err <= bound(spread)


@needs_ref
@pytest.mark.parametrize("outer,part", [(0, -1), (1, 0), (2, 2)])
def test_split_parts_match_reference_executor(tmp_path, outer, part):
    s, dk = _state(32, 6, 4, 0.25)
    rank = 3
    ref, nodes, weights = _reference(tmp_path, s, dk, 1.0, rank, outer, part)
    want, spread = eta44_oracle_with_spread(
        lambda x: OE.eta44_split_part(x, dk, 1.0, 1.0, nodes, weights, outer, part), s)
    err = np.linalg.norm(ref - want) / np.linalg.norm(want)
    assert err <= bound(spread), (err, spread)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("n,seed,count,dk,peak,rank", [
    # (the engine refuses grids on which the quartic support reaches Nyquist,
    # where the executor aliases silently, so these grids leave it room)
    (64, 8, 8, 0.3, 1.0, 10),
    (64, 9, 10, 0.2, 1.2, 6),
    (64, 9, 10, 0.2, 1.2, 8),
])
def test_engine_matches_reference_executor(tmp_path, n, seed, count, dk, peak, rank):
    """The engine's eta44 against the reference executor's field; the bound
    is the restatement's roundoff spread on the same case."""
    s, dk = _state(n, seed, count, dk)
    ref, nodes, weights = _reference(tmp_path, s, dk, peak, rank)
    got = E44.eta44(s, dk=dk, depth=1.0, peak_depth=peak, rank=rank, nodes=nodes,
                    weights=weights)
    _, spread = eta44_oracle_with_spread(lambda x: OE.eta44(x, dk, 1.0, peak, nodes, weights), s)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    emax = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    print(f"n {n} rank {rank}: engine vs reference executor L2 {err:.3e} max {emax:.3e}; "
          f"restatement spread {spread:.3e}")
    # both sides carry their own roundoff: twice the bound
    assert err <= 2 * bound(spread)
