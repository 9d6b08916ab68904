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
    r = _run("gl_eta44", "a", "b", "6", "1", "0")
    assert r.returncode == 1 and "split mode" in r.stderr


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
