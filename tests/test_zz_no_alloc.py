"""The allocation-free estimate entry point, for callers that cannot call
cudaMalloc (a memory pool or arena owns every device allocation, or the
allocator is locked after start-up).  It must give the same estimate as the
allocating entry point pfk_estimate, call after call, while its scratch lives
in a static device array shared by all calls.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(seed, m, nsub, log_weights):
    rng = np.random.default_rng(seed)
    T = m * nsub
    st = np.stack([rng.normal(0, 2, T), rng.normal(1, 3, T), rng.uniform(-np.pi, np.pi, T)]).astype(np.float32)
    keys = (rng.normal(-40, 15, T) if log_weights else rng.exponential(1, T)).astype(np.float32)
    return keys, st


def _noalloc(E, torch, keys, st, m, mask, lw):
    dk = torch.from_numpy(keys).cuda()
    ds = torch.from_numpy(np.ascontiguousarray(st)).cuda()
    dout = torch.zeros(E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    E.estimate_noalloc(dk.data_ptr(), ds.data_ptr(), st.shape[0], len(keys), m, dout.data_ptr(), mask, lw)
    torch.cuda.synchronize()
    return dout.cpu().numpy().view(E.ESTIMATE_DTYPE)[0]


@pytest.mark.parametrize("lw", [1, 0])
def test_noalloc_matches_allocating_entry_point(gpu, lw):
    import torch
    E = gpu
    # two calls in a row with different shapes: the second must not see the first's scratch
    for seed, m, nsub in ((3, 512, 64), (4, 256, 4096)):
        keys, st = _inputs(seed + 10 * lw, m, nsub, lw)
        ref = E.estimate(keys, st, m, angle_mask=0b100, log_weights=lw)
        got = _noalloc(E, torch, keys, st, m, 0b100, lw)
        assert np.allclose(got["mean"][:3], ref["mean"][:3], rtol=1e-12, atol=1e-12)
        assert abs(got["log_norm"] - ref["log_norm"]) <= 1e-12 * abs(ref["log_norm"]) + 1e-12
        assert got["best_subfilter"] == ref["best_subfilter"] and got["best_key"] == ref["best_key"]
        assert np.array_equal(got["best"][:3], ref["best"][:3]) and got["flags"] == ref["flags"] == 0


def test_noalloc_allocates_no_device_memory(gpu):
    """The one promise of the entry point: after a first call (which loads the
    module and looks up its scratch address), further calls leave the device's
    free memory unchanged."""
    import torch
    E = gpu
    keys, st = _inputs(7, 512, 2048, 1)
    dk = torch.from_numpy(keys).cuda()
    ds = torch.from_numpy(np.ascontiguousarray(st)).cuda()
    dout = torch.zeros(E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    E.estimate_noalloc(dk.data_ptr(), ds.data_ptr(), 3, len(keys), 512, dout.data_ptr(), 0b100, 1)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(20):
        E.estimate_noalloc(dk.data_ptr(), ds.data_ptr(), 3, len(keys), 512, dout.data_ptr(), 0b100, 1)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_more_than_its_scratch(gpu):
    import torch
    E = gpu
    keys = torch.zeros(64 * 4097, device="cuda")
    st = torch.zeros(3 * 64 * 4097, device="cuda")
    out = torch.zeros(E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    with pytest.raises(E.PFError) as ei:
        E.estimate_noalloc(keys.data_ptr(), st.data_ptr(), 3, 64 * 4097, 64, out.data_ptr())
    assert ei.value.status == E.PF_ERR_INVALID and "4096" in str(ei.value)
