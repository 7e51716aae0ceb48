"""The allocation-free FP64 direct sum (nbx_direct_fp64_noalloc).

For callers that cannot allocate device memory -- their memory belongs to
another allocator or was budgeted at start-up, or they must not pay
cudaMalloc's device-wide synchronisation inside their loop -- the library
offers this entry point: the caller passes device buffers for every input
and output, and the partial sums live in a fixed array inside the library.
Here the buffers come from PyTorch (the test may allocate; the entry point
must not), and two calls in a row, with different targets so that the
second reuses the shared array, must agree with nbx_direct_fp64.

The file is named to be collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_direct_fp64_twice(nbx):
    import torch
    n = 20000
    sim = nbx.Simulation(nbx.uniform_disc(n))
    sim.step(3)
    s = sim.download()  # current order, the order the targets index
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(np.ascontiguousarray(s["px"])).to(dev)
    y = torch.from_numpy(np.ascontiguousarray(s["py"])).to(dev)
    m = torch.from_numpy(np.ascontiguousarray(s["mass"])).to(dev)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(21)
    for call in range(2):
        k = 4096 if call == 0 else 1500
        tg = np.sort(rng.choice(n, k, replace=False)).astype(np.uint32)
        ref_x, ref_y = sim.direct_fp64(tg)
        t = torch.from_numpy(tg.astype(np.int32)).to(dev)
        ax = torch.full((k,), float("nan"), dtype=torch.float64, device=dev)
        ay = torch.full((k,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        rc = nbx.lib().nbx_direct_fp64_noalloc(
            x.data_ptr(), y.data_ptr(), m.data_ptr(), n, t.data_ptr(), k, 1.0,
            ax.data_ptr(), ay.data_ptr(), stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize(dev)
        gx, gy = ax.cpu().numpy(), ay.cpu().numpy()
        rel = np.hypot(gx - ref_x, gy - ref_y) / np.maximum(np.hypot(ref_x, ref_y), 1e-30)
        assert np.isfinite(rel).all() and rel.max() < 1e-12, (call, rel.max())
    # targets outside 0..n-1 (they live in device memory, so only the kernel
    # can tell): not read through, NaN outputs; the in-range ones unchanged
    tg = np.array([5, n, 17, 0xFFFFFFFF, n - 1], np.uint32)
    ref_x, ref_y = sim.direct_fp64(tg[[0, 2, 4]])
    t = torch.from_numpy(tg.view(np.int32)).to(dev)
    ax = torch.zeros(5, dtype=torch.float64, device=dev)
    ay = torch.zeros(5, dtype=torch.float64, device=dev)
    rc = nbx.lib().nbx_direct_fp64_noalloc(
        x.data_ptr(), y.data_ptr(), m.data_ptr(), n, t.data_ptr(), 5, 1.0,
        ax.data_ptr(), ay.data_ptr(), stream.cuda_stream)
    assert rc == 0
    torch.cuda.synchronize(dev)
    gx, gy = ax.cpu().numpy(), ay.cpu().numpy()
    assert np.isnan(gx[[1, 3]]).all() and np.isnan(gy[[1, 3]]).all()
    rel = np.hypot(gx[[0, 2, 4]] - ref_x, gy[[0, 2, 4]] - ref_y) / np.hypot(ref_x, ref_y)
    assert rel.max() < 1e-12
    # more targets than the fixed array holds: rejected before any launch
    big = torch.zeros(4097, dtype=torch.int32, device=dev)
    out = torch.zeros(4097, dtype=torch.float64, device=dev)
    rc = nbx.lib().nbx_direct_fp64_noalloc(
        x.data_ptr(), y.data_ptr(), m.data_ptr(), n, big.data_ptr(), 4097, 1.0,
        out.data_ptr(), out.data_ptr(), stream.cuda_stream)
    assert rc == 3  # NBX_ERR_CAPACITY
    sim.close()
