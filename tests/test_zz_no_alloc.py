"""The no-allocation update_xrz entry point (xplus_update_xrz_noalloc), for callers that cannot
call cudaMalloc.  It must give the same x, r, z and {r.z, r.r} as update_xrz_kernel, the entry
point it is a variant of, on two calls in a row (the second call reuses the shared scratch
array the first one left behind).  Collected last on purpose: a failure here leaves every other
test already run."""
import ctypes as C

import numpy as np
import pytest

from project_xplus_b200 import _lib
from project_xplus_b200 import kernels as K

pytestmark = pytest.mark.gpu


def test_noalloc_update_xrz_matches_update_xrz_twice(gpu):
    import torch
    rng = np.random.default_rng(7)
    n = 300_001
    dev = torch.device("cuda", 0)
    p, ap = rng.standard_normal(n), rng.standard_normal(n)
    m_inv = rng.uniform(0.5, 2.0, n)
    x0, r0 = rng.standard_normal(n), rng.standard_normal(n)
    # reference: the existing entry point, run twice with host arrays
    x_ref, r_ref, z_ref, met_ref = x0.copy(), r0.copy(), np.empty(n), np.empty(2)
    ref = []
    for alpha in (0.37, -1.25):
        K.update_xrz_kernel(x_ref, p, r_ref, ap, m_inv, z_ref, met_ref, alpha, n)
        ref.append((x_ref.copy(), r_ref.copy(), z_ref.copy(), met_ref.copy()))
    # the no-allocation entry point, twice in a row on device buffers
    t = {k: torch.from_numpy(v).to(dev) for k, v in
         dict(x=x0, r=r0, p=p, ap=ap, m_inv=m_inv).items()}
    z = torch.empty(n, dtype=torch.float64, device=dev)
    met = torch.full((2,), np.nan, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for k, alpha in enumerate((0.37, -1.25)):
        rc = _lib.lib.xplus_update_xrz_noalloc(t["x"].data_ptr(), t["p"].data_ptr(), t["r"].data_ptr(),
                                               t["ap"].data_ptr(), t["m_inv"].data_ptr(), z.data_ptr(),
                                               met.data_ptr(), alpha, n, C.c_void_p(stream))
        assert rc == _lib.XPLUS_OK, _lib.last_error()
        torch.cuda.synchronize()
        xr, rr, zr, mr = ref[k]
        assert np.array_equal(t["x"].cpu().numpy(), xr)
        assert np.array_equal(t["r"].cpu().numpy(), rr)
        assert np.array_equal(z.cpu().numpy(), zr)
        np.testing.assert_allclose(met.cpu().numpy(), mr, rtol=1e-14)


def test_noalloc_update_xrz_matches_the_oracle(gpu, oracle):
    """Against the oracle's restatement of the reference's update_xrz_kernel
    (archived/kernels/cg_kernels.cpp:118-147): x, r and z bit for bit (every product and sum
    is rounded on its own on both sides), {r.z, r.r} to the reduction-order rounding."""
    import torch
    rng = np.random.default_rng(11)
    n = 65_537
    dev = torch.device("cuda", 0)
    p, ap = rng.standard_normal(n), rng.standard_normal(n)
    m_inv = rng.uniform(0.5, 2.0, n)
    x, r, z, met = rng.standard_normal(n), rng.standard_normal(n), np.empty(n), np.empty(2)
    t = {k: torch.from_numpy(v.copy()).to(dev) for k, v in dict(x=x, r=r, p=p, ap=ap, m_inv=m_inv).items()}
    zd = torch.empty(n, dtype=torch.float64, device=dev)
    md = torch.empty(2, dtype=torch.float64, device=dev)
    c = oracle.clib()
    for alpha in (0.61, -0.07):
        c.or_update_xrz(n, oracle._p(x), oracle._p(p), oracle._p(r), oracle._p(ap), oracle._p(m_inv),
                        oracle._p(z), oracle._p(met), C.c_double(alpha))
        rc = _lib.lib.xplus_update_xrz_noalloc(t["x"].data_ptr(), t["p"].data_ptr(), t["r"].data_ptr(),
                                               t["ap"].data_ptr(), t["m_inv"].data_ptr(), zd.data_ptr(),
                                               md.data_ptr(), alpha, n, None)
        assert rc == _lib.XPLUS_OK, _lib.last_error()
        torch.cuda.synchronize()
        assert np.array_equal(t["x"].cpu().numpy(), x)
        assert np.array_equal(t["r"].cpu().numpy(), r)
        assert np.array_equal(zd.cpu().numpy(), z)
        np.testing.assert_allclose(md.cpu().numpy(), met, rtol=1e-12)


def test_noalloc_rejects_host_arrays(gpu):
    """Host arrays (which update_xrz_kernel stages) are an argument error here, returned
    before any launch, so passing them cannot fault the GPU."""
    import torch
    n = 1000
    host = [np.zeros(n) for _ in range(6)]
    met_h = np.zeros(2)
    rc = _lib.lib.xplus_update_xrz_noalloc(*[h.ctypes.data for h in host], met_h.ctypes.data, 0.5, n, None)
    assert rc == _lib.XPLUS_ERR_ARG
    assert "host memory" in _lib.last_error()
    # one host array among device ones is caught too
    dev = [torch.zeros(n, dtype=torch.float64, device="cuda:0") for _ in range(6)]
    met_d = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    ptrs = [d.data_ptr() for d in dev]
    ptrs[3] = host[3].ctypes.data
    rc = _lib.lib.xplus_update_xrz_noalloc(*ptrs, met_d.data_ptr(), 0.5, n, None)
    assert rc == _lib.XPLUS_ERR_ARG and "ap: host memory" in _lib.last_error()
    torch.cuda.synchronize()


def test_noalloc_rejects_sizes_beyond_its_limit(gpu):
    rc = _lib.lib.xplus_update_xrz_noalloc(None, None, None, None, None, None, None, 1.0,
                                           _lib.XPLUS_NOALLOC_MAX_N + 1, None)
    assert rc == _lib.XPLUS_ERR_ARG
    assert "no-allocation limit" in _lib.last_error()
