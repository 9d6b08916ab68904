"""Fourth-order GL eta44: file formats (CPU), GPU parity with the CPU
restatement of paper/order4/cpp/gl_eta44_fftw.cpp, and the paper's GL-vs-WIT
metrics on the 382-mode field (paper/order4/data/eta44_no_stokes_rank_metrics.csv)."""

from pathlib import Path

import numpy as np
import pytest
import torch

from gl_engine import _lib
from gl_engine import eta44 as E44
from gl_engine import wit
from oracle import gl_eta44 as OE
from oracle import gl_oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
# raw relative L2 of GL vs WIT eta44, percent (eta44_no_stokes_rank_metrics.csv:2-4)
PAPER_L2_PCT = {6: 9.1656674905729, 8: 4.20839343830129, 10: 2.03486173251526}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_glrti_and_gle44_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    spec = rng.standard_normal((16, 16)) + 1j * rng.standard_normal((16, 16))
    nodes, weights = O.gauss_laguerre(6)
    inp = E44.GlInput(n=16, dk=0.2, depth=1.0, peak_depth=1.0, rules={6: (nodes, weights)},
                      spectrum=spec)
    E44.write_glrti(tmp_path / "in.bin", inp)
    back = E44.read_glrti(tmp_path / "in.bin")
    assert np.array_equal(back.spectrum, spec) and back.rules[6][0].tolist() == nodes.tolist()
    raw = (tmp_path / "in.bin").read_bytes()
    # x-major storage: flat index ix*n + iy
    off = 8 + 32 + 8 + 8 + 2 * 6 * 8
    first = np.frombuffer(raw, "<f8", 4, off)
    assert first[0] == spec[0, 0].real and first[2] == spec[1, 0].real
    E44.write_gle44(tmp_path / "out.bin", 16, 6, spec)
    assert np.array_equal(E44.read_gle44(tmp_path / "out.bin")["field"], spec)


def _small(seed, n=32, m=4):
    rng = np.random.default_rng(seed)
    cells = [(x, y) for x in range(1, 4) for y in range(-2, 3)]
    pick = rng.choice(len(cells), size=m, replace=False)
    modes = np.array([cells[i] for i in pick])
    c = 0.02 * (rng.standard_normal(m) + 1j * rng.standard_normal(m))
    return E44.spectrum_from_modes(modes, c, n, 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("seed,rank", [(0, 2), (1, 3), (2, 4)])
def test_eta44_matches_cpu_restatement(seed, rank):
    s = _small(seed)
    nodes, weights = O.gauss_laguerre(rank)
    ref = OE.eta44(s, 0.25, 1.0, 1.0, nodes, weights)
    got = E44.eta44(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=rank)
    err = rel(got, ref)
    print(f"seed {seed} GL{rank}: rel L2 {err:.3e}")
    assert err < 1e-9


def _tall(seed, h, n=128, w=8, m=12):
    """Modes filling a parent box w columns (mx = 1..w) by h rows."""
    rng = np.random.default_rng(seed)
    lo = -((h - 1) // 2)
    cells = {(1, lo), (w, lo + h - 1)}
    while len(cells) < m:
        cells.add((int(rng.integers(1, w + 1)), int(rng.integers(lo, lo + h))))
    modes = np.array(sorted(cells))
    c = 0.01 * (rng.standard_normal(len(modes)) + 1j * rng.standard_normal(len(modes)))
    return E44.spectrum_from_modes(modes, c, n, 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("h,pair_cols,third_cols", [(20, 48, 64), (25, 64, 80)])
def test_eta44_stage_grids_match_cpu_restatement(h, pair_cols, third_cols):
    """The pair and third stages on their own grids (columns of the mixed
    lengths 48 = 3 x 16 and 80 = 5 x 16 here; the order-4 stage on 128)
    reproduce the CPU restatement on the 128^2 grid."""
    s = _tall(h, h)
    box = E44._box(np.abs(s))
    desc = _lib.Eta44Desc(n=128, dk=0.25, depth=1.0, peak_depth=1.0, rank=2, nodes=None,
                          weights=None, box_x0=box[0], box_y0=box[1], box_w=box[2], box_h=box[3],
                          max_units=1, output=_lib.OUT_COMPLEX, components=_lib.COMP_ETA44,
                          gravity=1.0)
    info = E44.Eta44Plan(desc, torch.device("cuda")).info
    assert (info.ncy_pair, info.ncy_triple, info.ncy) == (pair_cols, third_cols, 128)
    nodes, weights = O.gauss_laguerre(2)
    ref = OE.eta44(s, 0.25, 1.0, 1.0, nodes, weights)
    # the oracle's own answer under a 1-ulp change of its input: where the
    # roundoff floor sits near some bins (h = 20 here) FP64 implementations
    # that differ only in FFT roundoff spread by ~1e-9, the grid used or not
    spread = rel(OE.eta44(s * (1 + 2.2e-16), 0.25, 1.0, 1.0, nodes, weights), ref)
    got = E44.eta44(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=2)
    err = rel(got, ref)
    print(f"h {h} (pair cols {pair_cols}, third cols {third_cols}): rel L2 {err:.3e}, "
          f"oracle 1-ulp spread {spread:.3e}")
    assert err < max(1e-9, 8 * spread)


@pytest.mark.gpu
@pytest.mark.parametrize("rank", [6, 8, 10])
def test_eta44_reproduces_paper_gl_vs_wit_metric(rank):
    """GL eta44 against the WIT field (which the WIT kernel reproduces to
    1e-14, test_wit.py) gives the paper's raw relative L2 at each rank."""
    inp = wit.read_dir4in(GOLD / "wit_field_n0382_input.bin")
    n = inp.nx
    w = wit.wit_eta44(inp)
    ref = np.real(np.fft.ifft2(w.fields["eta"][0] * n * n))
    s = E44.spectrum_from_modes(inp.modes, inp.amplitudes[0], n, inp.depth)
    gl = np.real(E44.eta44(s, dk=inp.dkx, depth=inp.depth, peak_depth=1.0, rank=rank))
    pct = 100 * rel(gl, ref)
    print(f"GL{rank} vs WIT raw rel L2 {pct:.13f} % (paper {PAPER_L2_PCT[rank]})")
    assert abs(pct / PAPER_L2_PCT[rank] - 1) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("seed,rank", [(0, 2), (1, 3), (2, 4)])
def test_psi44_matches_cpu_restatement(seed, rank):
    """psi44 (src/gl_pure_sum_order4.m; the C++ has none) against the CPU
    restatement of the MATLAB graph; eta44 is unchanged by asking for psi44."""
    s = _small(seed)
    nodes, weights = O.gauss_laguerre(rank)
    e_ref, p_ref = OE.eta44_psi44(s, 0.25, 1.0, 1.0, nodes, weights)
    e, p = E44.eta44(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=rank, psi44=True, gravity=1.0)
    e_only = E44.eta44(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=rank)
    print(f"seed {seed} GL{rank}: eta44 {rel(e, e_ref):.3e}, psi44 {rel(p, p_ref):.3e}")
    assert np.array_equal(e, e_only)
    assert rel(e, e_ref) < 1e-9 and rel(p, p_ref) < 1e-9


@pytest.mark.gpu
def test_gl_pure_sum_order4_dimensionless_api():
    s = _small(3)
    n = s.shape[0]
    line = 0.25 * np.rint(np.fft.fftfreq(n) * n)
    qx, qy = np.meshgrid(line, line)
    eta, psi, audit = E44.gl_pure_sum_order4(s, qx, qy, 1.0, 4)
    nodes, weights = O.gauss_laguerre(4)
    e_ref, p_ref = OE.eta44_psi44(s, 0.25, 1.0, 1.0, nodes, weights)
    assert rel(eta, e_ref) < 1e-9 and rel(psi, p_ref) < 1e-9
    assert audit["quadrature_rank"] == 4 and not audit["order4_stokes_correction_used"]
    with pytest.raises(ValueError):
        E44.gl_pure_sum_order4(s, qx, qy, 1.0, 5)


@pytest.mark.gpu
def test_psi44_approaches_wit_with_rank():
    """No psi44 numbers are published; as a physics check the GL surface
    potential approaches the WIT direct sum's surface potential on the paper
    field as the rank grows, as eta44 does (9.2 / 4.2 / 2.0 %)."""
    inp = wit.read_dir4in(GOLD / "wit_field_n0382_input.bin")
    n = inp.nx
    w = wit.wit_eta44(inp)
    ref = np.real(np.fft.ifft2(w.fields["psi"][0] * n * n))
    s = E44.spectrum_from_modes(inp.modes, inp.amplitudes[0], n, inp.depth)
    errs = []
    for rank in (6, 8, 10):
        _, p = E44.eta44(s, dk=inp.dkx, depth=inp.depth, peak_depth=1.0, rank=rank, psi44=True,
                         gravity=inp.gravity)
        errs.append(100 * rel(np.real(p), ref))
        print(f"GL{rank} psi44 vs WIT psi: raw rel L2 {errs[-1]:.4f} %")
    assert errs[0] > errs[1] > errs[2]


@pytest.mark.gpu
@pytest.mark.parametrize("seed,rank,outer,part", [(0, 2, 1, -2), (1, 3, 0, -1), (1, 3, 2, 1),
                                                  (2, 4, 3, 0), (2, 4, 1, 3)])
def test_split_parts_match_cpu_restatement(seed, rank, outer, part):
    """One part of the reference's split mode (outer node, base or partition
    31 with one third-level node) against its CPU restatement."""
    from parity_bounds import bound, eta44_oracle_with_spread

    s = _small(seed)
    nodes, weights = O.gauss_laguerre(rank)
    ref, spread = eta44_oracle_with_spread(
        lambda x: OE.eta44_split_part(x, 0.25, 1.0, 1.0, nodes, weights, outer, part), s)
    got = E44.eta44_part(s, dk=0.25, depth=1.0, peak_depth=1.0, rank=rank, outer=outer, part=part)
    err = rel(got, ref)
    print(f"seed {seed} GL{rank} outer {outer} part {part}: rel L2 {err:.3e}, "
          f"oracle spread {spread:.3e}")
    assert err <= bound(spread)
