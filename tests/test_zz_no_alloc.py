"""The allocation-free covariance entry point (mra_eval_covariance_static).

It exists for callers that cannot let the library allocate device memory --
programs that route all device memory through their own pool, and loops that
cannot pay for the synchronisation of cudaMalloc/cudaFree on each call.  The
test gives it device buffers owned by the test (allocated here with torch, not
by the library), calls it through the C ABI twice in a row, and checks each
result against the allocating entry point mra_eval_covariance within the
tolerance of the other covariance tests (1e-12 relative).  Kept in its own file
so that it runs last; it also passes alone in a fresh process.
"""
import ctypes as C
import os

import numpy as np
import pytest

from nonstationary_mra_b200 import api, capi, refio

pytestmark = pytest.mark.gpu

CASE = os.path.join(os.path.dirname(__file__), "golden", "example")


def _device(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _call_static(md, th, p1, p2, self_block, out):
    lib = capi.load()
    m, keep = api._model_struct(md)
    t = api._theta_struct(th)
    n1 = p1.shape[1]
    n2 = 0 if self_block else p2.shape[1]
    status = lib.mra_eval_covariance_static(C.byref(m), C.byref(t), C.c_void_p(p1.data_ptr()), n1,
                                            None if self_block else C.c_void_p(p2.data_ptr()), n2,
                                            1 if self_block else 0, C.c_void_p(out.data_ptr()), None)
    capi.check(status, "mra_eval_covariance_static")
    del keep


def test_static_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    api.set_device(0)
    torch.cuda.set_device(0)
    st, md, _ = refio.load_case(CASE, mode="likelihood")
    th = dict(sill_scale=md.sill_scale, range_scale=md.range_scale, nugget_scale=md.nugget_scale)
    p1 = st.obs[:, :300]
    p2 = st.knots[:, :40]
    # first call: cross block
    d1, d2 = _device(p1, torch), _device(p2, torch)
    out = torch.full((300, 40), float("nan"), dtype=torch.float64, device="cuda")
    _call_static(md, th, d1, d2, False, out)
    torch.cuda.synchronize()
    ref = api.eval_covariance(md, th, p1, p2)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=0)
    # second call right after: self block of other points, reusing the shared scratch
    p3 = st.obs[:, 500:620]
    d3 = _device(p3, torch)
    out2 = torch.full((120, 120), float("nan"), dtype=torch.float64, device="cuda")
    _call_static(md, th, d3, None, True, out2)
    torch.cuda.synchronize()
    ref2 = api.eval_covariance(md, th, p3)
    np.testing.assert_allclose(out2.cpu().numpy(), ref2, rtol=1e-12, atol=0)


def test_static_rejects_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    api.set_device(0)
    st, md, _ = refio.load_case(CASE, mode="likelihood")
    big = torch.zeros((3, 40000), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.MRAError) as e:
        _call_static(md, dict(), big, None, True, out)
    assert e.value.status == capi.MRA_ERR_ARG
    assert "MRA_STATIC_MAX_POINTS" in str(e.value)


def test_static_rejects_a_model_the_allocating_entry_point_rejects():
    # the same model check as mra_eval_covariance: a zero basis length would
    # otherwise give inf/NaN covariances without an error
    torch = pytest.importorskip("torch")
    api.set_device(0)
    st, md, _ = refio.load_case(CASE, mode="likelihood")
    assert md.nonstationary
    md.basis_len = 0.0
    pts = _device(st.obs[:, :8], torch)
    out = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(capi.MRAError) as e:
        _call_static(md, dict(), pts, None, True, out)
    assert e.value.status == capi.MRA_ERR_ARG
    assert "basis length" in str(e.value)
