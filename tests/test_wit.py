"""Sector-44 WIT quartet sum: file formats (CPU) and GPU parity with the
reference's own C++ (golden vectors from oracle/_ref/wit_eta44 and the
archived 382-mode paper field)."""

import subprocess
import time
from pathlib import Path

import numpy as np
import pytest

from gl_engine import wit

GOLD = Path(__file__).resolve().parent / "golden"
REF_BIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "wit_eta44"


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_dir4in_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    inp = wit.WitInput(modes=np.array([[1, 0], [2, -1], [3, 2]], dtype=np.int32),
                       amplitudes=rng.standard_normal((2, 3)) + 1j * rng.standard_normal((2, 3)),
                       nx=32, ny=16, gravity=1.0, depth=2.0, dkx=0.2, dky=0.3, threshold=1e-6)
    wit.write_dir4in(tmp_path / "x.bin", inp)
    back = wit.read_dir4in(tmp_path / "x.bin")
    assert np.array_equal(back.modes, inp.modes)
    assert np.array_equal(back.amplitudes, inp.amplitudes)
    assert (back.nx, back.ny, back.gravity, back.depth, back.dkx, back.dky, back.threshold) == \
        (32, 16, 1.0, 2.0, 0.2, 0.3, 1e-6)


def test_reads_the_reference_paper_input():
    inp = wit.read_dir4in(GOLD / "wit_field_n0382_input.bin")
    assert inp.modes.shape == (382, 2)
    assert (inp.nx, inp.ny) == (256, 256)
    assert inp.amplitudes.shape == (1, 382)


def _golden_case(gold, tag):
    n = int(gold[f"{tag}/grid"][0])
    return wit.WitInput(modes=gold[f"{tag}/modes"], amplitudes=gold[f"{tag}/amplitudes"], nx=n,
                        ny=n, gravity=1.0, depth=1.0, dkx=0.2, dky=0.2, threshold=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["small10", "small24", "s40_small12", "s42_small12"])
def test_wit_matches_reference_cpp_golden(tag):
    gold = dict(np.load(GOLD / "wit_reference.npz"))
    res = wit.wit_sector(_golden_case(gold, tag), int(gold[f"{tag}/sector"]))
    bins = gold[f"{tag}/bins"]
    for f in wit.FIELDS:
        got = res.fields[f].ravel()
        assert np.all(np.delete(got, bins) == 0), f
        want = gold[f"{tag}/{f}"]
        if np.linalg.norm(want) == 0:
            assert np.all(got[bins] == 0), f
            continue
        err = rel(got[bins], want)
        print(f"{tag} {f}: rel L2 {err:.3e}")
        assert err < 1e-11, f
    cand, kept, near, szo, szi = gold[f"{tag}/counts"]
    assert res.stats["candidates"] == cand and res.stats["kept"] == kept
    assert res.stats["near"] == near and res.stats["strict_zero_output"] == szo


@pytest.mark.gpu
@pytest.mark.parametrize("sector", [44, 40, 42])
def test_wit_matches_live_reference_binary(tmp_path, sector):
    if not REF_BIN.exists():
        pytest.skip("reference WIT binary not built (make -C oracle)")
    rng = np.random.default_rng(7)
    cells = [(x, y) for x in range(1, 7) for y in range(-5, 6)]
    pick = sorted(rng.choice(len(cells), size=16, replace=False))
    inp = wit.WitInput(modes=np.array([cells[i] for i in pick], dtype=np.int32),
                       amplitudes=0.02 * (rng.standard_normal((3, 16)) + 1j * rng.standard_normal((3, 16))),
                       nx=64, ny=64, gravity=9.81, depth=3.0, dkx=0.15, dky=0.15, threshold=1e-6)
    wit.write_dir4in(tmp_path / "in.bin", inp)
    subprocess.run([str(REF_BIN), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "--sector",
                    str(sector)], check=True, capture_output=True)
    ref = wit.read_dir4out(tmp_path / "out.bin")
    res = wit.wit_sector(inp, sector)
    for f in wit.FIELDS:
        if np.linalg.norm(ref.fields[f]) == 0:
            assert np.linalg.norm(res.fields[f]) == 0, f
            continue
        err = rel(res.fields[f], ref.fields[f])
        print(f"live sector {sector} {f}: {err:.3e}")
        assert err < 1e-11, f
    for k in ("candidates", "kept", "near", "strict_zero_output"):
        assert res.stats[k] == ref.stats[k], k


@pytest.mark.gpu
def test_wit_reproduces_archived_paper_field():
    """382 modes, 256^2, 901,244,960 quartets: the archived reference field."""
    gold = dict(np.load(GOLD / "wit_reference.npz"))
    inp = wit.read_dir4in(GOLD / "wit_field_n0382_input.bin")
    t0 = time.perf_counter()
    res = wit.wit_eta44(inp)
    dt = time.perf_counter() - t0
    top = gold["n0382/top_bins"]
    e_top = rel(res.fields["eta"].ravel()[top], gold["n0382/top_eta"])
    p_top = rel(res.fields["psi"].ravel()[top], gold["n0382/top_psi"])
    e_norm = abs(np.linalg.norm(res.fields["eta"]) / float(gold["n0382/norm_eta"]) - 1)
    print(f"n0382: {dt:.2f} s, {res.stats['kept']} quartets; top-256 rel {e_top:.3e} / {p_top:.3e}; "
          f"norm rel {e_norm:.3e}")
    assert res.stats["kept"] == int(gold["n0382/counts"][1])
    assert e_top < 1e-11 and p_top < 1e-11 and e_norm < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["small24", "s40_small12", "s42_small12"])
def test_wit_quartet_ranges_sum_to_the_whole_sector(tag):
    """Sequential stand-in for the multi-GPU split: three contiguous shares of
    the candidate quartets (one of them empty), summed, give the one-call
    fields, and their statistics combine to the one-call statistics."""
    from gl_engine import parallel

    gold = dict(np.load(GOLD / "wit_reference.npz"))
    inp = _golden_case(gold, tag)
    sector = int(gold[f"{tag}/sector"])
    whole = wit.wit_sector(inp, sector)
    count = wit.candidates(sector, inp.modes.shape[0])
    assert count == whole.stats["candidates"]
    cuts = [0, count // 3, count // 3, count]
    parts = [wit.wit_sector(inp, sector, q_range=(cuts[i], cuts[i + 1])) for i in range(3)]
    for f in wit.FIELDS:
        total = sum(p.fields[f] for p in parts)
        scale = max(np.abs(whole.fields[f]).max(), 1e-300)
        assert np.abs(total - whole.fields[f]).max() <= 1e-13 * scale, f
    merged = parallel.combine_wit_stats([p.stats for p in parts])
    for k in parallel.STAT_SUMS:
        assert merged[k] == whole.stats[k], k
    assert merged["min_detuning"] == whole.stats["min_detuning"]
    assert merged["max_residual"] == whole.stats["max_residual"]
