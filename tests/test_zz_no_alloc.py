"""gl_box_synthesize_noalloc: box spectra -> physical field with no device allocation.

Callers that cannot allocate device memory while they run -- a real-time
loop on a fixed memory budget, where cudaMalloc may synchronise the device, or
a host runtime whose GPU binding only hands over buffers it already owns -- use
this entry point.  It keeps its scratch in a static device array instead of a
caller workspace.

These tests call it through the C ABI twice in a row (different sea states,
boxes and unit counts, so stale scratch from the first call cannot leak into
the second) and compare each result with the eta11 plane that the workspace-
based gl_execute computes from the same box spectra: the same transform with
scale = depth.  One more case uses a scale other than the depth and checks the
result against numpy.fft.ifft2 of the box embedded on the full grid.
Tolerance: relative L2 < 1e-14, the FFT bar of the other GPU tests.  The file
is collected last so a failure here cannot hide other tests.
"""

import ctypes as C

import numpy as np
import pytest
import torch

import gl_engine
from gl_engine import _lib, api, seastate

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _workspace_reference(seed, n, times):
    st = seastate.small_order3(seed=seed, n=n, modes=12)
    coeffs = gl_engine.gl_spectral_coefficients(1, st.gravity, st.depth, st.a, st.b, st.kx, st.ky)
    dep = api.prepare_deposit(coeffs, st.lx, st.ly, n, n)
    dev = torch.device("cuda", 0)
    plan = api.get_plan(nx=n, ny=n, lx=st.lx, ly=st.ly, depth=st.depth, gravity=st.gravity,
                        order=1, components=_lib.COMP_ETA11, eta22_rank=6, allow_below=False,
                        box=dep.box, grid=_lib.GRID_COMPACT, max_units=len(times),
                        output=_lib.OUT_COMPLEX, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    spectra = torch.empty((len(times), dep.box[3], dep.box[2], 2), dtype=torch.float64,
                          device=dev)
    plan.deposit(len(times), t(dep.seg_offsets, torch.int32), t(dep.seg_bins, torch.int32),
                 t(dep.ab, torch.float64), t(dep.omega, torch.float64),
                 t(np.asarray(times, dtype=float), torch.float64), spectra, stream)
    out = torch.empty((len(times), 1, n, n), dtype=torch.complex128, device=dev)
    status = torch.zeros(len(times), dtype=torch.int32, device=dev)
    plan.execute(len(times), spectra, _lib.SPECTRA_BOX, out, status, stream)
    torch.cuda.synchronize()
    assert int(status.abs().sum()) == 0
    return st, dep.box, spectra, out[:, 0].cpu().numpy()


def _noalloc(n, box, spectra, scale, units, real_only=False):
    lib = _lib.load()
    dev = spectra.device
    dtype = torch.float64 if real_only else torch.complex128
    out = torch.full((units, n, n), float("nan"), dtype=dtype, device=dev)
    st = lib.gl_box_synthesize_noalloc(units, n, n, box[0], box[1], box[2], box[3],
                                       C.c_void_p(spectra.data_ptr()), float(scale),
                                       C.c_void_p(out.data_ptr()), int(real_only),
                                       C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    _lib.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_workspace_entry_on_two_calls_in_a_row():
    st1, box1, spec1, ref1 = _workspace_reference(seed=3, n=64, times=[0.0, 0.8, 2.5])
    got1 = _noalloc(64, box1, spec1, st1.depth, 3)
    st2, box2, spec2, ref2 = _workspace_reference(seed=9, n=128, times=[1.1])
    got2 = _noalloc(128, box2, spec2, st2.depth, 1)
    assert box1 != box2
    for got, ref in ((got1, ref1), (got2, ref2)):
        assert np.all(np.isfinite(got))
        assert rel(got, ref) < 1e-14


def test_noalloc_real_output_and_repeat():
    st, box, spec, ref = _workspace_reference(seed=4, n=64, times=[0.3, 0.6])
    first = _noalloc(64, box, spec, st.depth, 2, real_only=True)
    second = _noalloc(64, box, spec, st.depth, 2, real_only=True)
    assert rel(first, ref.real) < 1e-14
    assert np.array_equal(first, second)


def test_noalloc_matches_numpy_ifft2_of_the_embedded_box():
    st, box, spec, _ = _workspace_reference(seed=5, n=64, times=[0.4, 1.9])
    scale = 2.75
    got = _noalloc(64, box, spec, scale, 2)
    again = _noalloc(64, box, spec, scale, 2)
    x0, y0, w, h = box
    s = spec.cpu().numpy()
    s = s[..., 0] + 1j * s[..., 1]
    for u in range(2):
        full = np.zeros((64, 64), dtype=complex)
        for iy in range(h):
            for ix in range(w):
                full[(y0 + iy) % 64, (x0 + ix) % 64] = s[u, iy, ix]
        ref = scale * np.fft.ifft2(full)
        assert rel(got[u], ref) < 1e-14
        assert rel(again[u], ref) < 1e-14


def test_noalloc_rejects_requests_beyond_its_static_scratch():
    lib = _lib.load()
    dummy = torch.zeros(2, dtype=torch.float64, device="cuda")
    # 64 units x 200 columns x 1024 rows x 16 B = 210 MB > 16 MiB
    st = lib.gl_box_synthesize_noalloc(64, 1024, 1024, 1, -50, 200, 101,
                                       C.c_void_p(dummy.data_ptr()), 1.0,
                                       C.c_void_p(dummy.data_ptr()), 0, None)
    assert st == 20  # GL_ERR_WORKSPACE
    assert "static array" in _lib.last_error()
