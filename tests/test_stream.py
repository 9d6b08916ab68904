"""SurfaceStream: batches streamed to pinned host memory with the copy of one
batch overlapping the next batch's evaluation.  Each result equals the
device-resident evaluation of the same snapshots."""

import numpy as np
import pytest
import torch

from gl_engine import api, seastate

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graphs", [True, False])
def test_stream_results_equal_device_batches(graphs):
    """Replayed graphs (inputs copied from pinned staging each batch) and
    eager launches both give the device-resident evaluation bit for bit,
    also when the batch size changes mid-stream."""
    st = seastate.small_order3(seed=9, n=64, modes=16)
    c = api.gl_spectral_coefficients(3, st.gravity, st.depth, st.a, st.b, st.kx, st.ky,
                                     0, 0, {"eta22_rank": 4})
    batches = [[0.0, 0.4], [1.1, 2.5], [3.0, 0.2], [7.5, 9.0, 4.0], [0.0, 0.4], [2.2, 3.3]]
    ss = api.SurfaceStream(c, st.lx, st.ly, 64, 64, components=["eta33", "psi33"], output="real",
                           graphs=graphs)
    tickets, got = [], []
    for times in batches:
        tickets.append(ss.submit(times))
        if len(tickets) >= 2:  # read the previous batch while this one runs
            got.append(ss.result(tickets[-2]).fields.clone())
    got.append(ss.result(tickets[-1]).fields.clone())
    assert not got[0].is_cuda
    for times, host in zip(batches, got):
        ref = api.surface_batch_device(c, st.lx, st.ly, 64, 64, times,
                                       components=["eta33", "psi33"], output="real")
        assert torch.equal(host, ref.fields.cpu())
    with pytest.raises(ValueError):
        ss.result(tickets[0])
