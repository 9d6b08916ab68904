"""CUDA engine parity against the CPU oracle and the reference's golden
vectors.  Every call goes through the C ABI (libgl_b200.so) on cuda:0.

Tolerances (raw relative L2, the reference's metric, test_spatial.py:68-71):
* the MATLAB fixtures: the reference's own bars (2e-13 .. 8e-11);
* reference-Python goldens and seeded sea states: per case and per field,
  max(1e-12, 4 x the oracle's own roundoff spread on that case), where the
  spread is how far the FP64 oracle moves when only its FFT roundoff changes
  (parity_bounds: the roundoff floor then zeroes different bins); the L2 and
  max errors are printed per field;
* the 1024^2 order-3 workload: <= 1e-6 (the metric's bar) and within 3x the
  oracle's spread there.
"""

from pathlib import Path

import numpy as np
import pytest
import torch

import gl_engine
from gl_engine import api, seastate
from oracle import gl_oracle as O
from parity_bounds import check_fields, oracle_fields_with_spread

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
COMPS = ("eta11", "psi11", "eta22", "psi22", "eta33", "psi33")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def matlab():
    return dict(np.load(GOLD / "matlab_fixtures.npz"))


@pytest.fixture(scope="module")
def refpy():
    return dict(np.load(GOLD / "reference_python.npz"))


def test_fft2_matches_numpy():
    rng = np.random.default_rng(0)
    for ny, nx in ((16, 16), (64, 32), (128, 256), (1024, 1024), (8, 2048)):
        x = rng.standard_normal((2, ny, nx)) + 1j * rng.standard_normal((2, ny, nx))
        t = torch.from_numpy(x).cuda()
        f = api.fft2_device(t).cpu().numpy()
        i = api.fft2_device(t, inverse=True).cpu().numpy()
        assert rel(f, np.fft.fft2(x)) < 1e-14
        assert rel(i, np.fft.ifft2(x)) < 1e-14


def _fixture(m, tag, order, grid="compact"):
    rank = int(m[f"{tag}/rank"]) if f"{tag}/rank" in m else 6
    time = float(m[f"{tag}/time"]) if f"{tag}/time" in m else 0.0
    return gl_engine.reconstruct_directional_field(
        m[f"{tag}/eta1"], lx=float(m[f"{tag}/lx"]), ly=float(m[f"{tag}/ly"]),
        depth=float(m[f"{tag}/depth"]), gravity=float(m[f"{tag}/gravity"]), time=time,
        order=order, eta22_rank=rank, grid=grid)


@pytest.mark.parametrize("grid", ["compact", "reference"])
def test_matlab_eta22_fixture(matlab, grid):
    r = _fixture(matlab, "eta22", 2, grid).components
    assert rel(r["eta11"], matlab["eta22/eta1"]) < 2e-13
    assert rel(r["eta22"], matlab["eta22/eta22"]) < 2e-12
    assert rel(r["psi11"], matlab["eta22/psi11"]) < 2e-13
    assert rel(r["psi22"], matlab["eta22/psi22"]) < 3e-12


@pytest.mark.parametrize("grid", ["compact", "reference"])
def test_matlab_order3_fixture(matlab, grid):
    r = _fixture(matlab, "order3", 3, grid).components
    assert rel(r["eta33"], matlab["order3/eta33"]) < 5e-11
    assert rel(r["psi33"], matlab["order3/psi33"]) < 5e-11


def test_matlab_nonzero_time_fixture(matlab):
    r = _fixture(matlab, "time", 3).components
    for c in COMPS:
        assert rel(r[c], matlab[f"time/{c}"]) < 8e-11, c


@pytest.mark.parametrize("tag", ["fixture_t0", "fixture_t07", "jonswap64_o3", "jonswap64_o2",
                                 "jonswap128_o3"])
def test_two_stage_matches_reference_python(refpy, tag):
    order, g, h, lx, ly, nx, ny, t, rank = refpy[f"{tag}/meta"]
    a, b, kx, ky = refpy[f"{tag}/modes"]
    c = gl_engine.gl_spectral_coefficients(int(order), g, h, a, b, kx, ky, 0.0, 0.0,
                                           {"eta22_rank": int(rank)})
    _, _, _, _, comps, audit = gl_engine.gl_spectral_surface(c, lx, ly, int(nx), int(ny), t)
    _, spread = oracle_fields_with_spread(int(order), g, h, a, b, kx, ky, lx, ly, int(nx),
                                          int(ny), t, eta22_rank=int(rank))
    ref = {}
    for key in refpy:
        if not key.startswith(tag + "/"):
            continue
        name = key.split("/")[1]
        if name in ("meta", "modes"):
            continue
        ref[name] = refpy[key]
    assert len(ref) >= 2
    check_fields(comps, ref, spread, tag)
    assert audit["engine"]["precision"] == "fp64"


def _oracle_surface(st, order, t, rank=6):
    oc = O.spectral_coefficients(order, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                 options={"eta22_rank": rank})
    return O.spectral_surface(oc, st.lx, st.ly, st.nx, st.ny, t)


@pytest.mark.parametrize("seed,n,modes,order", [(0, 64, 20, 3), (1, 128, 60, 3), (2, 128, 80, 2),
                                                (3, 64, 1, 3), (4, 64, 2, 2)])
def test_seeded_states_match_oracle(seed, n, modes, order):
    st = seastate.jonswap_sea_state(n=n, length=2.5 * n, depth=25.0, hs=2.0, tp=8.0,
                                    modes=modes, seed=seed, order=order)
    t = 0.37 * seed
    c = gl_engine.gl_spectral_coefficients(order, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                           0, 0, {"eta22_rank": 6})
    _, _, _, _, comps, _ = gl_engine.gl_spectral_surface(c, st.lx, st.ly, n, n, t)
    ref, spread = oracle_fields_with_spread(order, st.gravity, st.depth, st.a, st.b, st.kx,
                                            st.ky, st.lx, st.ly, n, n, t)
    plus = {k: v for k, v in ref.items() if k.endswith("_plus")}
    check_fields(comps, plus, spread, f"seed {seed}")


def _box_state(order, h, n, seed, w=4, depth=30.0):
    """Modes on the lattice of an n x n, 256 m domain whose parent box is w
    columns (mx = 2 .. w+1) by h rows (my spans h consecutive values centred
    on 0), so the pair and triple boxes have heights 2h-1 and 3h-2."""
    rng = np.random.default_rng(seed)
    lx = 256.0
    lo = -((h - 1) // 2)
    cells = {(2, lo), (w + 1, lo + h - 1)}          # the box corners
    while len(cells) < 12:
        cells.add((int(rng.integers(2, w + 2)), int(rng.integers(lo, lo + h))))
    m = np.array(sorted(cells), dtype=float)
    dk = 2 * np.pi / lx
    amp = 0.04 / np.sqrt(len(m))
    return dict(order=order, gravity=9.81, depth=depth, a=amp * rng.standard_normal(len(m)),
                b=amp * rng.standard_normal(len(m)), kx=dk * m[:, 0], ky=dk * m[:, 1], lx=lx,
                ly=lx, n=n)


# (order, parent box height, grid, expected pair / triple column lengths):
# every mixed length 16 m the column kernels run, as a pair grid and as a
# triple grid, next to the power-of-two lengths they replace.
MIXED_CASES = [
    (2, 20, 64, 48, None), (2, 36, 128, 80, None), (2, 44, 128, 96, None),
    (2, 69, 256, 144, None), (2, 76, 256, 160, None), (2, 90, 256, 192, None),
    (2, 110, 256, 240, None),
    (3, 14, 128, 32, 48), (3, 25, 256, 64, 80), (3, 30, 256, 64, 96),
    (3, 46, 256, 96, 144), (3, 52, 512, 128, 160), (3, 60, 512, 128, 192),
    (3, 69, 256, 144, 240),
]


@pytest.mark.parametrize("order,h,n,pair,triple", MIXED_CASES)
def test_mixed_column_grids_match_oracle(order, h, n, pair, triple):
    """Pair/triple stages on column grids of length 16 m (m = 3, 5, 6, 9,
    10, 12, 15) reproduce the oracle on the reference grid like the
    power-of-two grids do (alias-free products have the same coefficients on
    any period covering the box)."""
    st = _box_state(order, h, n, seed=h)
    t = 0.3
    c = gl_engine.gl_spectral_coefficients(order, st["gravity"], st["depth"], st["a"], st["b"],
                                           st["kx"], st["ky"], 0, 0, {"eta22_rank": 4})
    _, _, _, _, comps, audit = gl_engine.gl_spectral_surface(c, st["lx"], st["ly"], n, n, t)
    grids = audit["engine"]["column_grids"]
    assert grids["pair"] == pair
    if triple is not None:
        assert grids["triple"] == triple
    ref, spread = oracle_fields_with_spread(order, st["gravity"], st["depth"], st["a"], st["b"],
                                            st["kx"], st["ky"], st["lx"], st["ly"], n, n, t,
                                            eta22_rank=4)
    names = [c + "_plus" for c in COMPS[2: 2 * order]]
    check_fields(comps, {k: ref[k] for k in names}, spread, f"order {order} h {h} ({pair}/{triple})")


# (order, parent box width, grid, expected pair row length): the mixed row
# lengths of the pair-stage row kernels (144, 160, 192, 240), reached through
# wide parent boxes (the pair box is 2w - 1 wide).
MIXED_ROW_CASES = [
    (2, 70, 512, 144), (2, 76, 512, 160), (2, 90, 512, 192), (2, 110, 512, 240),
    (3, 70, 512, 144), (3, 76, 512, 160),
]


@pytest.mark.parametrize("order,w,n,pair_row", MIXED_ROW_CASES)
def test_mixed_row_grids_match_oracle(order, w, n, pair_row):
    """Pair-stage rows on the mixed lengths 16 m reproduce the oracle on the
    reference grid."""
    st = _box_state(order, 5, n, seed=w, w=w)
    t = 0.3
    c = gl_engine.gl_spectral_coefficients(order, st["gravity"], st["depth"], st["a"], st["b"],
                                           st["kx"], st["ky"], 0, 0, {"eta22_rank": 4})
    _, _, _, _, comps, audit = gl_engine.gl_spectral_surface(c, st["lx"], st["ly"], n, n, t)
    assert audit["engine"]["pair_row_length"] == pair_row
    ref, spread = oracle_fields_with_spread(order, st["gravity"], st["depth"], st["a"], st["b"],
                                            st["kx"], st["ky"], st["lx"], st["ly"], n, n, t,
                                            eta22_rank=4)
    names = [c + "_plus" for c in COMPS[2: 2 * order]]
    check_fields(comps, {k: ref[k] for k in names}, spread, f"order {order} w {w} (rows {pair_row})")


def test_compact_and_reference_grids_agree():
    st = seastate.small_order3(seed=7, n=64, modes=12)
    c = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                           0, 0, {"eta22_rank": 4})
    a = api.surface_batch_device(c, st.lx, st.ly, 64, 64, [0.0, 1.0], grid="compact")
    b = api.surface_batch_device(c, st.lx, st.ly, 64, 64, [0.0, 1.0], grid="reference")
    assert a.plan.info.ncx < 64
    assert b.plan.info.ncx == 64
    fa, fb = a.fields.cpu().numpy(), b.fields.cpu().numpy()
    # both grids against the oracle's spread at each snapshot
    for i, t in enumerate((0.0, 1.0)):
        ref, spread = oracle_fields_with_spread(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                                st.lx, st.ly, 64, 64, t, eta22_rank=4)
        names = [api.COMP_NAMES[c] for c in a.plan.component_ids]
        check_fields({nm + "_plus": fa[i, k] for k, nm in enumerate(names)},
                     {nm + "_plus": fb[i, k] for k, nm in enumerate(names)},
                     {nm + "_plus": spread[nm + "_plus"] for nm in names}, f"grids t={t}")


def test_batched_times_equal_single_calls():
    st = seastate.small_order3(seed=5, n=64, modes=16)
    c = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                           0, 0, {"eta22_rank": 4})
    times = [0.0, 0.5, 3.0]
    batch = api.surface_batch_device(c, st.lx, st.ly, 64, 64, times, max_units=2)
    for i, t in enumerate(times):
        one = api.surface_batch_device(c, st.lx, st.ly, 64, 64, [t], max_units=1)
        assert torch.equal(batch.fields[i], one.fields[0])


def test_real_output_mode_matches_complex():
    st = seastate.small_order3(seed=6, n=64, modes=10)
    c = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    a = api.surface_batch_device(c, st.lx, st.ly, 64, 64, [0.2], output="complex",
                                 components=["eta33", "psi33"])
    b = api.surface_batch_device(c, st.lx, st.ly, 64, 64, [0.2], output="real",
                                 components=["eta33", "psi33"])
    assert a.names == ["eta33", "psi33"]
    assert torch.equal(a.fields.real, b.fields)


def test_device_status_reports_order3_domain():
    # a parent with kh <= 0.5 in the real-grid entry is caught on the device
    n = 64
    x = np.arange(n) * (2 * np.pi / n)
    X, Y = np.meshgrid(x, x)
    eta1 = 0.01 * np.cos(1 * X) + 0.005 * np.cos(3 * X + 2 * Y)
    with pytest.raises(ValueError, match="kh > 0.5"):
        gl_engine.reconstruct_directional_field(eta1, lx=2 * np.pi, ly=2 * np.pi, depth=0.3,
                                                order=3)


def test_config1_order2_matches_oracle():
    st = seastate.config1(0)
    c = gl_engine.gl_spectral_coefficients(2, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                           0, 0, {"eta22_rank": 4})
    _, _, _, _, comps, _ = gl_engine.gl_spectral_surface(c, st.lx, st.ly, st.nx, st.ny, 0.0)
    ref, spread = oracle_fields_with_spread(2, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                            st.lx, st.ly, st.nx, st.ny, 0.0, eta22_rank=4)
    names = [c + "_plus" for c in ("eta11", "psi11", "eta22", "psi22")]
    check_fields(comps, {k: ref[k] for k in names}, spread, "config1")


def test_config2_order3_matches_oracle():
    st = seastate.config2(0)
    c = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    res = api.surface_batch_device(c, st.lx, st.ly, st.nx, st.ny, [0.0],
                                   components=["eta33", "psi33"])
    got = res.fields[0].cpu().numpy()
    kxg, kyg = O.fft_wavenumber_grid(st.lx, st.ly, st.nx, st.ny)
    oc = O.spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    s = O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], st.depth, st.lx,
                        st.ly, st.nx, st.ny, 0.0)
    e33, p33, _ = O.order3(s, st.depth * kxg, st.depth * kyg)
    pscale = st.depth * np.sqrt(st.gravity * st.depth)
    ee = rel(got[0], st.depth * e33)
    pe = rel(got[1], pscale * p33)
    emax = float(np.max(np.abs(got[0] - st.depth * e33)) / np.max(np.abs(st.depth * e33)))
    print(f"config2 eta33 rel L2 {ee:.3e} max {emax:.3e}; psi33 rel L2 {pe:.3e}")
    assert ee < 1e-6 and pe < 1e-6


def test_config2_deviation_is_within_oracle_roundoff_sensitivity():
    """The FP64 oracle itself moves when only its FFT roundoff changes (the
    roundoff floor of _spectral.py:52-64 then zeroes different bins).  The
    engine's deviation from the oracle must stay within 3x of that spread,
    measured here by re-running the oracle with its 2-D FFTs taken in the
    other axis order."""
    import numpy.fft as F

    st = seastate.config2(0)
    kxg, kyg = O.fft_wavenumber_grid(st.lx, st.ly, st.nx, st.ny)
    oc = O.spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    s = O.deposit_modes(oc["a"], oc["b"], oc["kx"], oc["ky"], oc["omega"], st.depth, st.lx,
                        st.ly, st.nx, st.ny, 0.0)
    qx, qy = st.depth * kxg, st.depth * kyg
    e0, p0, _ = O.order3(s, qx, qy)
    f2, i2 = F.fft2, F.ifft2
    try:
        F.fft2 = lambda a: F.fft(F.fft(a, axis=0), axis=1)
        F.ifft2 = lambda a: F.ifft(F.ifft(a, axis=0), axis=1)
        e1, p1, _ = O.order3(s, qx, qy)
    finally:
        F.fft2, F.ifft2 = f2, i2
    c = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    got = api.surface_batch_device(c, st.lx, st.ly, st.nx, st.ny, [0.0],
                                   components=["eta33", "psi33"]).fields[0].cpu().numpy()
    pscale = st.depth * np.sqrt(st.gravity * st.depth)
    spread_e, spread_p = rel(e1, e0), rel(p1, p0)
    dev_e, dev_p = rel(got[0], st.depth * e0), rel(got[1], pscale * p0)
    print(f"oracle self-spread eta33 {spread_e:.3e} psi33 {spread_p:.3e}; "
          f"engine deviation eta33 {dev_e:.3e} psi33 {dev_p:.3e}")
    assert dev_e < 3 * spread_e and dev_p < 3 * spread_p


def test_units_with_different_supports_in_one_launch():
    """One launch over units whose supports differ (all modes, half of them,
    all again): each unit equals its own single-unit launch, so support
    sums shared between equal-support units never leak across units."""
    st = seastate.small_order3(seed=11, n=64, modes=20)
    c = gl_engine.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                           0, 0, {"eta22_rank": 4})
    dep = api.prepare_deposit(c, st.lx, st.ly, 64, 64)
    plan = api.get_plan(nx=64, ny=64, lx=st.lx, ly=st.ly, depth=c.h, gravity=c.g, order=3,
                        components=api._components_for(3, None), eta22_rank=4,
                        allow_below=False, box=dep.box, grid=api.GRID_COMPACT, max_units=3,
                        output=api.OUT_COMPLEX, device=torch.device("cuda"), inner_rank=4,
                        outer_rank=4)
    pairs = dep.ab.reshape(-1, 2)  # (a, b) per mode
    keep = np.ones((pairs.shape[0], 1))
    keep[1::2] = 0.0
    abs_ = [dep.ab, (pairs * keep).ravel(), dep.ab]
    dev = torch.device("cuda")
    w, h = dep.box[2], dep.box[3]

    def box_spectra(ab_list, times):
        out = []
        for ab, t in zip(ab_list, times):
            spec = torch.empty((1, h, w, 2), dtype=torch.float64, device=dev)
            plan.deposit(1, torch.as_tensor(dep.seg_offsets, dtype=torch.int32, device=dev),
                         torch.as_tensor(dep.seg_bins, dtype=torch.int32, device=dev),
                         torch.as_tensor(ab, dtype=torch.float64, device=dev),
                         torch.as_tensor(dep.omega, dtype=torch.float64, device=dev),
                         torch.as_tensor([t], dtype=torch.float64, device=dev), spec,
                         torch.cuda.current_stream().cuda_stream)
            out.append(spec)
        return torch.cat(out)

    times = [0.3, 0.3, 1.7]
    spec = box_spectra(abs_, times)
    ncomp = plan.info.n_components
    both = torch.empty((3, ncomp, 64, 64), dtype=torch.complex128, device=dev)
    status = torch.zeros(3, dtype=torch.int32, device=dev)
    plan.execute(3, spec, api.SPECTRA_BOX, both, status, torch.cuda.current_stream().cuda_stream)
    assert int(status.abs().sum()) == 0
    for u in range(3):
        one = torch.empty((1, ncomp, 64, 64), dtype=torch.complex128, device=dev)
        st1 = torch.zeros(1, dtype=torch.int32, device=dev)
        plan.execute(1, spec[u:u + 1].contiguous(), api.SPECTRA_BOX, one, st1,
                     torch.cuda.current_stream().cuda_stream)
        assert torch.equal(both[u], one[0]), u
    assert not torch.equal(both[0], both[1])
