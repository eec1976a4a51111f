"""The allocation-free line-search reduction, pt_ls_frames_noalloc.

Some callers cannot allocate device memory at the moment they call in: an
application whose memory pool owns all of the device memory, or a loop that
must not call cudaMalloc (it can synchronise the device) once it is running.
For them the library keeps this reduction's scratch in a static device array
of its own, so the call needs neither an allocation nor a workspace argument.

Checked through the C ABI against pt_ls_frames, which takes a caller-allocated
workspace, on two calls in a row.  The second call uses fewer step lengths and
the other likelihood, so partial sums left in the shared scratch by the first
call would show up in its result.  Both entry points run the same reduction in
the same order, so the FP64 sums must agree to rounding (rtol 1e-12).  The
file is named to be collected last; it also passes when run on its own, where
its first call performs the per-device set-up.
"""
import numpy as np
import pytest

from ptychotomo_b200 import _lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _inputs(n, seed):
    g = torch.Generator().manual_seed(seed)
    f = torch.randn(n, dtype=torch.complex64, generator=g)
    d = 0.1 * torch.randn(n, dtype=torch.complex64, generator=g)
    data = torch.floor(50 * torch.rand(n, generator=g))
    return f.cuda(), d.cuda(), data.cuda()


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    lib = _lib.lib()
    n = 3 * 9 * 32 * 32
    f, d, data = _inputs(n, 5)
    work = torch.empty(lib.pt_reduce_workspace_bytes() // 8, dtype=torch.float64, device="cuda")
    for J, model in ((16, 0), (5, 1)):
        gam = torch.tensor([2.0 * 0.5 ** j for j in range(J)], dtype=torch.float64, device="cuda")
        ref = torch.full((J,), float("nan"), dtype=torch.float64, device="cuda")
        out = torch.full((J,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.pt_ls_frames(f.data_ptr(), d.data_ptr(), data.data_ptr(), 0.01, n, model, gam.data_ptr(), J,
                              work.data_ptr(), ref.data_ptr(), None)
        assert rc == 0, _lib.last_error()
        rc = lib.pt_ls_frames_noalloc(f.data_ptr(), d.data_ptr(), data.data_ptr(), 0.01, n, model,
                                      gam.data_ptr(), J, out.data_ptr(), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        assert np.all(np.isfinite(r)) and np.any(r != 0)
        np.testing.assert_allclose(o, r, rtol=1e-12, atol=0)


def test_noalloc_call_allocates_no_device_memory():
    """After a first call (which loads the module and looks up the scratch),
    a further call leaves the device's free memory unchanged."""
    lib = _lib.lib()
    n = 4096
    f, d, data = _inputs(n, 7)
    gam = torch.tensor([1.0, 0.5, 0.25], dtype=torch.float64, device="cuda")
    out = torch.empty(3, dtype=torch.float64, device="cuda")

    def call():
        rc = lib.pt_ls_frames_noalloc(f.data_ptr(), d.data_ptr(), data.data_ptr(), 1.0, n, 0, gam.data_ptr(), 3,
                                      out.data_ptr(), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()

    call()
    free0, _ = torch.cuda.mem_get_info()
    call()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_more_step_lengths_than_its_scratch_holds():
    lib = _lib.lib()
    n = 1024
    f, d, data = _inputs(n, 6)
    gam = torch.ones(17, dtype=torch.float64, device="cuda")
    out = torch.empty(17, dtype=torch.float64, device="cuda")
    rc = lib.pt_ls_frames_noalloc(f.data_ptr(), d.data_ptr(), data.data_ptr(), 1.0, n, 0, gam.data_ptr(), 17,
                                  out.data_ptr(), None)
    assert rc == _lib.PT_ERR_ARG
    assert "exceeds the static scratch" in _lib.last_error()
