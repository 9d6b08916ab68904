"""The order-4 command-line drop-ins (``bin/gl_eta44``, ``bin/wit_eta44``):
the reference's executable argument conventions and files
(paper/order4/run_cpp.py:18-35), served by the GPU engine."""

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from gl_engine import eta44 as E44
from gl_engine import wit
from oracle import gl_oracle as O

BIN = Path(__file__).resolve().parents[1] / "green-laplace-wave-reconstruction_b200" / "bin"


def _run(name, *args):
    return subprocess.run([sys.executable, str(BIN / name), *map(str, args)], capture_output=True,
                          text=True)


def test_wit_cli_usage_and_sector_errors(tmp_path):
    r = _run("wit_eta44", "only-one-arg")
    assert r.returncode == 2 and "--sector" in r.stderr
    r = _run("wit_eta44", tmp_path / "in.bin", tmp_path / "out.bin", "--sector", "41")
    assert r.returncode == 1 and "DIRECTIONAL_CPP_ERROR sector must be 40, 42, or 44" in r.stderr


def test_gl_eta44_cli_usage_errors(tmp_path):
    r = _run("gl_eta44", "a", "b")
    assert r.returncode == 1 and r.stderr.startswith("CPP_GL_ETA44_ERROR usage")
    # the split mode's argument checks, in the reference's order (before the input is read)
    r = _run("gl_eta44", "a", "b", "6", "1", "6")
    assert r.returncode == 1 and r.stderr.strip() == "CPP_GL_ETA44_ERROR outer index"
    r = _run("gl_eta44", "a", "b", "6", "1", "2", "6")
    assert r.returncode == 1 and r.stderr.strip() == "CPP_GL_ETA44_ERROR part index"
    r = _run("gl_eta44", "a", "b", "6", "1", "-1", "0")
    assert r.returncode == 1 and "split mode requires one outer4 index" in r.stderr
    r = _run("merge_eta44_outer", "out.bin", "only-one.bin")
    assert r.returncode == 1 and r.stderr.startswith("CPP_GL_ETA44_MERGE_ERROR usage")


@pytest.mark.gpu
def test_wit_cli_matches_library_call(tmp_path):
    rng = np.random.default_rng(3)
    cells = [(x, y) for x in range(1, 6) for y in range(-4, 5)]
    pick = sorted(rng.choice(len(cells), size=12, replace=False))
    inp = wit.WitInput(modes=np.array([cells[i] for i in pick], dtype=np.int32),
                       amplitudes=0.02 * (rng.standard_normal((2, 12)) + 1j * rng.standard_normal((2, 12))),
                       nx=32, ny=32, gravity=9.81, depth=3.0, dkx=0.2, dky=0.2, threshold=1e-6)
    wit.write_dir4in(tmp_path / "in.bin", inp)
    r = _run("wit_eta44", tmp_path / "in.bin", tmp_path / "out.bin", "--sector", "44")
    assert r.returncode == 0, r.stderr
    assert "DIRECTIONAL_CPP_DONE sector=44" in r.stderr
    got = wit.read_dir4out(tmp_path / "out.bin")
    want = wit.wit_sector(inp, 44)
    # the direct sum accumulates with FP64 atomics: two runs agree to roundoff
    for f in wit.FIELDS:
        w = want.fields[f]
        if np.linalg.norm(w) == 0:
            assert np.linalg.norm(got.fields[f]) == 0, f
        else:
            assert np.linalg.norm(got.fields[f] - w) / np.linalg.norm(w) < 1e-12, f
    assert got.stats["kept"] == want.stats["kept"]


@pytest.mark.gpu
def test_gl_eta44_cli_matches_library_call(tmp_path):
    rng = np.random.default_rng(4)
    modes = np.array([(1, 0), (2, 1), (3, -1)])
    c = 0.02 * (rng.standard_normal(3) + 1j * rng.standard_normal(3))
    s = E44.spectrum_from_modes(modes, c, 32, 1.0)
    nodes, weights = O.gauss_laguerre(4)
    E44.write_glrti(tmp_path / "in.bin", E44.GlInput(n=32, dk=0.25, depth=1.0, peak_depth=1.0,
                                                     rules={4: (nodes, weights)}, spectrum=s))
    r = _run("gl_eta44", tmp_path / "in.bin", tmp_path / "out.bin", 4, 1)
    assert r.returncode == 0, r.stderr
    got = E44.read_gle44(tmp_path / "out.bin")
    want = E44.eta44(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=4, nodes=nodes, weights=weights)
    assert got["n"] == 32 and got["rank"] == 4
    assert np.array_equal(got["field"], want / 1.0)


@pytest.mark.gpu
def test_gl_eta44_split_mode_and_merge_follow_the_reference(tmp_path):
    """The reference's split launcher (paper/order4/run_gl_split.sh:29-38): one
    process per outer node for the base partitions (PART -1) and one per
    (outer node, third-level node) for partition 31, then merge_eta44_outer.
    Each part equals the CPU restatement of that part within the
    restatement's roundoff spread (parity_bounds); the merged field equals the
    restatement's merge and, here, the one-call field."""
    from oracle import gl_eta44 as OE
    from parity_bounds import bound, eta44_oracle_with_spread

    rng = np.random.default_rng(6)
    modes = np.array([(1, 0), (2, 1), (3, -1), (2, -2)])
    c = 0.02 * (rng.standard_normal(4) + 1j * rng.standard_normal(4))
    s = E44.spectrum_from_modes(modes, c, 32, 1.0)
    rank = 3
    nodes, weights = O.gauss_laguerre(rank)
    E44.write_glrti(tmp_path / "in.bin", E44.GlInput(n=32, dk=0.25, depth=1.0, peak_depth=1.0,
                                                     rules={rank: (nodes, weights)}, spectrum=s))
    parts, want, budget = [], 0, 0.0
    for outer in range(rank):
        for part in [-1] + list(range(rank)):
            out = tmp_path / f"p_{outer}_{part}.bin"
            r = _run("gl_eta44", tmp_path / "in.bin", out, rank, 1, outer, part)
            assert r.returncode == 0, r.stderr
            assert f"outer={outer} part={part}" in r.stderr
            ref, spread = eta44_oracle_with_spread(
                lambda x, o=outer, q=part: OE.eta44_split_part(x, 0.25, 1.0, 1.0, nodes, weights,
                                                              o, q), s)
            got = E44.read_gle44(out)["field"]
            assert np.linalg.norm(got - ref) <= bound(spread) * np.linalg.norm(ref), (outer, part)
            parts.append(out)
            want = want + ref
            budget += bound(spread) * np.linalg.norm(ref)
    r = _run("merge_eta44_outer", tmp_path / "merged.bin", *parts)
    assert r.returncode == 0, r.stderr
    assert f"partials={len(parts)}" in r.stderr
    merged = E44.read_gle44(tmp_path / "merged.bin")
    assert merged["rank"] == rank and merged["threads"] == len(parts)
    # the merge adds the parts' deviations at most
    assert np.linalg.norm(merged["field"] - want) <= budget + 1e-12 * np.linalg.norm(want)
    mono = OE.eta44(s, 0.25, 1.0, 1.0, nodes, weights)
    assert np.linalg.norm(want - mono) <= 1e-12 * np.linalg.norm(mono)

