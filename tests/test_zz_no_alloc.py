"""GPU test of the allocation-free product bcr_mv_noalloc (its own file, named
to be collected last).

bcr_mv_noalloc serves callers that cannot allocate device memory where they
need A*x -- a fixed memory budget owned by the host application, or a loop
that must not call into the CUDA allocator.  They own every buffer; the
library's only scratch is a fixed device array.  The test calls it through the
C ABI twice in a row on caller-owned buffers and compares each result with the
CPU oracle's Mv (the restatement of the reference's Mv) and with the existing
handle-based entry point bcr_mv_device on the same data; it also checks that
the calls leave the device's free memory unchanged."""
import numpy as np
import pytest

from alglin_b200 import bcr as B
from alglin_b200 import synth
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _device_arrays(s, torch):
    return [torch.from_numpy(np.ascontiguousarray(getattr(s, k))).cuda()
            for k in ("D", "E", "B", "C", "Cq", "F", "H")]


# (nblock, n, qr, qx, nr, nx): borders of every width, no border rows (the
# scratch array is then never read), and the largest border the array allows
@pytest.mark.parametrize("dims", [(3001, 8, 2, 2, 3, 3), (257, 16, 2, 2, 4, 4), (5, 3, 0, 1, 2, 0),
                                  (100, 4, 1, 1, 0, 2), (40, 2, 0, 0, 64, 1)])
def test_mv_noalloc_matches_oracle_and_handle_mv_twice(dims):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    s = synth.collocation(*dims, seed=11)
    h = B.BorderedCR()
    h.load_system(s)
    h.upload()
    o = po.Oracle(s, "LU", "LU")
    arrs = _device_arrays(s, torch)
    ptrs = [a.data_ptr() if a.numel() else 0 for a in arrs]
    rng = np.random.default_rng(3)
    xs = [rng.standard_normal(s.ncols) for _ in range(2)]
    r0s = [rng.standard_normal(s.nrows) for _ in range(2)]
    xd = [torch.from_numpy(v).cuda() for v in xs]
    outs = [torch.from_numpy(v).cuda() for v in r0s]
    refs = [torch.from_numpy(v).cuda() for v in r0s]
    coef = [(1.0, 0.0), (-0.5, 2.0)]
    # a first call performs the once-per-device set-up; the two calls checked
    # below must then leave the device's free memory as it was
    warm = torch.zeros(s.nrows, dtype=torch.float64, device="cuda")
    rc, msg = B.mv_noalloc(s.dims(), *ptrs, 1.0, xd[0].data_ptr(), 0.0, warm.data_ptr())
    assert rc == B.BCR_OK, msg
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for call in range(2):
        alpha, beta = coef[call]
        rc, msg = B.mv_noalloc(s.dims(), *ptrs, alpha, xd[call].data_ptr(), beta, outs[call].data_ptr())
        assert rc == B.BCR_OK, msg
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for call in range(2):
        alpha, beta = coef[call]
        h.mv_device(alpha, xd[call].data_ptr(), beta, refs[call].data_ptr())
        h.synchronize()
        out, dev = outs[call].cpu().numpy(), refs[call].cpu().numpy()
        orc = alpha * o.mv(xs[call]) + beta * r0s[call]
        scale = max(np.abs(orc).max(), 1.0)
        assert np.abs(out - orc).max() <= 1e-12 * scale, (call, np.abs(out - orc).max())
        assert np.abs(out - dev).max() <= 1e-12 * scale, (call, np.abs(out - dev).max())


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
