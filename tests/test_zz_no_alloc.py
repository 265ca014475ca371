"""The allocation-free entry point cf_ldu_spmv_dot_noalloc, for callers that
cannot allocate device memory (inside another component's graph capture, on
threads that must not take the allocator's locks, or in frameworks that hand
out only their own buffers).  Its output must equal the context entry point
cf_spmv32 on the same FP32 operator: y bit for bit (same per-row order) and
the dot within 1e-12 relative, on two calls in a row (the shared scratch and
its completion counter are reused).  Without w the dot is 0; without dot
only y is written.  The test allocates its own buffers with torch; the entry
point allocates none.  Collected last on purpose."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["symmetric", "asymmetric"])
def test_noalloc_matches_context_spmv(require_gpu, kind):
    import torch

    from metal4foam_b200 import _lib, mesh
    if kind == "symmetric":
        s = mesh.varcoeff3d((23, 19, 17), seed=31, permute=True)
    else:
        s = mesh.upwind3d((21, 20, 13), seed=32)
    a = s.addr
    ctx = _lib.Context(0)
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(s.n).astype(np.float32)
    w = rng.standard_normal(s.n).astype(np.float32)
    y_ref, dot_ref = ctx.spmv32(x, w)
    ctx.close()

    dev = torch.device("cuda", 0)
    f32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(dev)  # noqa: E731
    i32 = lambda v: torch.from_numpy(np.ascontiguousarray(v, np.int32)).to(dev)  # noqa: E731
    d_diag, d_upper = f32(s.diag), f32(s.upper)
    d_lower = None if s.lower is None else f32(s.lower)
    addr = [i32(v) for v in a.arrays()]
    d_x, d_w = f32(x), f32(w)
    d_y = torch.empty(s.n, dtype=torch.float32, device=dev)
    d_dot = torch.empty(1, dtype=torch.float64, device=dev)
    L = _lib.load()
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        d_y.fill_(float("nan"))
        d_dot.fill_(float("nan"))
        rc = L.cf_ldu_spmv_dot_noalloc(
            s.n, _lib.ptr(d_diag), _lib.ptr(d_upper), _lib.ptr(d_lower),
            *(_lib.ptr(t) for t in addr), _lib.ptr(d_x), _lib.ptr(d_w), _lib.ptr(d_y),
            _lib.ptr(d_dot), _lib.vp(stream.cuda_stream))
        torch.cuda.synchronize()
        assert rc == 0, L.cf_last_error()
        assert np.array_equal(d_y.cpu().numpy(), y_ref), f"call {call}"
        assert d_dot.item() == pytest.approx(dot_ref, rel=1e-12, abs=1e-12), f"call {call}"

    # w = NULL: y as before, the dot of nothing is exactly 0
    d_y.fill_(float("nan"))
    d_dot.fill_(float("nan"))
    rc = L.cf_ldu_spmv_dot_noalloc(
        s.n, _lib.ptr(d_diag), _lib.ptr(d_upper), _lib.ptr(d_lower),
        *(_lib.ptr(t) for t in addr), _lib.ptr(d_x), None, _lib.ptr(d_y),
        _lib.ptr(d_dot), _lib.vp(stream.cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0, L.cf_last_error()
    assert np.array_equal(d_y.cpu().numpy(), y_ref)
    assert d_dot.item() == 0.0

    # dot = NULL: y only; the dot buffer is left untouched
    d_y.fill_(float("nan"))
    d_dot.fill_(7.0)
    rc = L.cf_ldu_spmv_dot_noalloc(
        s.n, _lib.ptr(d_diag), _lib.ptr(d_upper), _lib.ptr(d_lower),
        *(_lib.ptr(t) for t in addr), _lib.ptr(d_x), _lib.ptr(d_w), _lib.ptr(d_y),
        None, _lib.vp(stream.cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0, L.cf_last_error()
    assert np.array_equal(d_y.cpu().numpy(), y_ref)
    assert d_dot.item() == 7.0

    # and a full call again after both: the shared counter is still sound
    rc = L.cf_ldu_spmv_dot_noalloc(
        s.n, _lib.ptr(d_diag), _lib.ptr(d_upper), _lib.ptr(d_lower),
        *(_lib.ptr(t) for t in addr), _lib.ptr(d_x), _lib.ptr(d_w), _lib.ptr(d_y),
        _lib.ptr(d_dot), _lib.vp(stream.cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0, L.cf_last_error()
    assert d_dot.item() == pytest.approx(dot_ref, rel=1e-12, abs=1e-12)


def test_noalloc_rejects_sizes_beyond_scratch(require_gpu):
    import torch

    from metal4foam_b200 import _lib
    L = _lib.load()
    buf = torch.zeros(8, dtype=torch.float32, device="cuda")
    ibuf = torch.zeros(8, dtype=torch.int32, device="cuda")
    p, ip = _lib.ptr(buf), _lib.ptr(ibuf)
    rc = L.cf_ldu_spmv_dot_noalloc(16_777_216 + 1, p, p, None, ip, ip, ip, ip, ip, p, p, p, None,
                                   None)
    assert rc == 9 and b"exceeds" in L.cf_last_error()
