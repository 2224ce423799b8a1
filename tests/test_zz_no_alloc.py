"""twos_estimate_noalloc: the estimator for callers that cannot allocate
device memory (a framework owns the memory pool, or the service has a fixed
device-memory budget).  Its per-call scratch lives in the library's static
device array, so this test checks, through the C ABI, that two calls in a row
give exactly the rows of twos_estimate_device (same kernels, same samples:
tolerance zero, as the other bit-exact GPU tests), that the largest request
the array holds is served and one site more is refused with a usage error,
and that it works in a fresh process as well as after the other tests (the
file is collected last)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TWOS_SCRATCH_BYTES = 16 * 1024 * 1024  # TWOS_NOALLOC_SCRATCH_BYTES


def _call(L, fn, mesh, req, d_sites, n, d_out):
    from twos_b200 import _abi
    summ = _abi.Summary()
    rc = fn(mesh._h, ctypes.byref(req), ctypes.c_void_p(d_sites.data_ptr()), n, None, 0,
            ctypes.c_void_p(d_out.data_ptr()), ctypes.byref(summ))
    return rc, summ


def test_noalloc_matches_device_entry_point_twice(lib_built, bunny1000, eval_points):
    import torch
    import twos_b200 as tb
    from twos_b200 import _abi
    L = _abi.load()
    with tb.Mesh(*bunny1000) as mesh:
        sites = eval_points[:96]
        d_sites = torch.tensor(sites, dtype=torch.float64, device="cuda")
        for precision, mode, walks in [("mixed", "compliance", 512), ("fp64", "paired", 256)]:
            cfg = tb.Config(walks=walks, mode=mode, precision=precision, seed=41, epsilon=5e-4, green=mode != "compliance",
                            source=tb.sources.affine(0.65), adjoint=tb.sources.sensor(1) if mode != "compliance" else [])
            req = cfg.to_request()
            ref = torch.zeros((len(sites), 7), dtype=torch.float64, device="cuda")
            rc, ref_summ = _call(L, L.twos_estimate_device, mesh, req, d_sites, len(sites), ref)
            assert rc == 0, L.twos_last_error()
            ref_rows = ref.cpu().numpy().copy()
            for call in range(2):
                out = torch.full((len(sites), 7), float("nan"), dtype=torch.float64, device="cuda")
                rc, summ = _call(L, L.twos_estimate_noalloc, mesh, req, d_sites, len(sites), out)
                assert rc == 0, L.twos_last_error()
                np.testing.assert_array_equal(out.cpu().numpy(), ref_rows, err_msg=f"{precision} call {call}")
                assert summ.steps == ref_summ.steps and summ.paths == ref_summ.paths and summ.caps == 0


def test_noalloc_rejects_requests_beyond_its_scratch(lib_built, bunny1000, eval_points):
    import torch
    import twos_b200 as tb
    from twos_b200 import _abi
    L = _abi.load()
    with tb.Mesh(*bunny1000) as mesh:
        sites = np.repeat(eval_points[:8], 1000, axis=0)  # 8,000 sites x 1,024 walks > 16 MiB of samples
        d_sites = torch.tensor(sites, dtype=torch.float64, device="cuda")
        out = torch.zeros((len(sites), 7), dtype=torch.float64, device="cuda")
        req = tb.Config(walks=1024, precision="mixed").to_request()
        rc, _ = _call(L, L.twos_estimate_noalloc, mesh, req, d_sites, len(sites), out)
        assert rc == _abi.ERR_USAGE
        msg = L.twos_last_error().decode()
        assert "bytes of scratch" in msg and str(16 * 1024 * 1024) in msg


def test_noalloc_boundary_of_its_scratch(lib_built, bunny1000, eval_points):
    """The largest mixed compliance request that fits the 16 MiB scratch is
    accepted and equals twos_estimate_device bit for bit (twice in a row); one
    more site is refused.  The boundary is found by bisection over the call's
    own size check, so the test follows the scratch layout without restating
    it, and it checks the documented capacity (about 2.0 M walks at 8 bytes
    per walk in this mode)."""
    import torch
    import twos_b200 as tb
    from twos_b200 import _abi
    L = _abi.load()
    walks = 256
    with tb.Mesh(*bunny1000) as mesh:
        sites = np.repeat(eval_points[:64], 160, axis=0)  # 10,240 sites: above the limit at 256 walks
        d_sites = torch.tensor(sites, dtype=torch.float64, device="cuda")
        out = torch.zeros((len(sites), 7), dtype=torch.float64, device="cuda")
        req = tb.Config(walks=walks, precision="mixed", seed=43, epsilon=5e-4,
                        source=tb.sources.affine(0.65)).to_request()
        lo, hi = 1, len(sites)
        assert _call(L, L.twos_estimate_noalloc, mesh, req, d_sites, hi, out)[0] == _abi.ERR_USAGE
        while hi - lo > 1:
            mid = (lo + hi) // 2
            rc, _ = _call(L, L.twos_estimate_noalloc, mesh, req, d_sites, mid, out)
            assert rc in (_abi.OK, _abi.ERR_USAGE), L.twos_last_error()
            if rc == _abi.OK:
                lo = mid
            else:
                hi = mid
        n_max = lo
        assert 1.95e6 <= n_max * walks <= TWOS_SCRATCH_BYTES // 8
        ref = torch.zeros((n_max, 7), dtype=torch.float64, device="cuda")
        rc, ref_summ = _call(L, L.twos_estimate_device, mesh, req, d_sites, n_max, ref)
        assert rc == 0, L.twos_last_error()
        ref_rows = ref.cpu().numpy().copy()
        for call in range(2):
            got = torch.full((n_max, 7), float("nan"), dtype=torch.float64, device="cuda")
            rc, summ = _call(L, L.twos_estimate_noalloc, mesh, req, d_sites, n_max, got)
            assert rc == 0, L.twos_last_error()
            np.testing.assert_array_equal(got.cpu().numpy(), ref_rows, err_msg=f"boundary call {call}")
            assert summ.steps == ref_summ.steps and summ.error_flags == 0
        rc, _ = _call(L, L.twos_estimate_noalloc, mesh, req, d_sites, n_max + 1, out)
        assert rc == _abi.ERR_USAGE and "bytes of scratch" in L.twos_last_error().decode()

