"""GPU test of the allocation-free product bcr_mv_noalloc (its own file, named
to be collected last).

bcr_mv_noalloc serves callers that cannot allocate device memory where they
need A*x -- a fixed memory budget owned by the host application, or a loop
that must not call into the CUDA allocator.  They own every buffer; the
library's only scratch is a fixed device array.  The test calls it through the
C ABI twice in a row on caller-owned buffers and compares each result with the
existing handle-based entry point bcr_mv_device on the same data."""
import numpy as np
import pytest

from alglin_b200 import bcr as B
from alglin_b200 import synth

pytestmark = pytest.mark.gpu


def _device_arrays(s, torch):
    return [torch.from_numpy(np.ascontiguousarray(getattr(s, k))).cuda()
            for k in ("D", "E", "B", "C", "Cq", "F", "H")]


@pytest.mark.parametrize("dims", [(3001, 8, 2, 2, 3, 3), (257, 16, 2, 2, 4, 4), (5, 3, 0, 1, 2, 0)])
def test_mv_noalloc_matches_handle_mv_twice(dims):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    s = synth.collocation(*dims, seed=11)
    h = B.BorderedCR()
    h.load_system(s)
    h.upload()
    arrs = _device_arrays(s, torch)
    ptrs = [a.data_ptr() if a.numel() else 0 for a in arrs]
    rng = np.random.default_rng(3)
    for call in range(2):
        x = torch.from_numpy(rng.standard_normal(s.ncols)).cuda()
        res0 = torch.from_numpy(rng.standard_normal(s.nrows)).cuda()
        alpha, beta = (1.0, 0.0) if call == 0 else (-0.5, 2.0)
        ref = res0.clone()
        h.mv_device(alpha, x.data_ptr(), beta, ref.data_ptr())
        h.synchronize()
        out = res0.clone()
        rc, msg = B.mv_noalloc(s.dims(), *ptrs, alpha, x.data_ptr(), beta, out.data_ptr())
        assert rc == B.BCR_OK, msg
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        assert np.abs(o - r).max() <= 1e-12 * max(np.abs(r).max(), 1.0), (call, np.abs(o - r).max())


def test_mv_noalloc_rejects_too_many_border_rows():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    s = synth.collocation(9, 2, 0, 0, 65, 1, seed=1)
    arrs = _device_arrays(s, torch)
    ptrs = [a.data_ptr() if a.numel() else 0 for a in arrs]
    x = torch.zeros(s.ncols, dtype=torch.float64, device="cuda")
    out = torch.zeros(s.nrows, dtype=torch.float64, device="cuda")
    rc, msg = B.mv_noalloc(s.dims(), *ptrs, 1.0, x.data_ptr(), 0.0, out.data_ptr())
    assert rc == B.BCR_BAD_ARGUMENT
    assert "maximum of 64" in msg
