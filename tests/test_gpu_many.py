"""Many independent systems solved concurrently (cf_solve_many_device: host
threads with their own CUDA streams, one context per system): every system
gets exactly what cf_solve_device on it alone returns -- psi bit for bit,
the same iterations and residuals -- with either preconditioner and any
number of streams."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

FIELDS = ("initialResidual", "finalResidual", "nIterations", "nRestarts", "converged",
          "singular", "normFactor", "residualL2")


def systems():
    return [mesh.varcoeff3d((24, 20, 18), seed=1, permute=True), mesh.poisson2d(60, 50, seed=2),
            mesh.varcoeff3d((12, 11, 10), seed=3, permute=False),
            mesh.varcoeff3d((30, 16), seed=4, permute=False),
            mesh.varcoeff3d((16, 16, 16), seed=5, permute=True), mesh.poisson2d(20, 20, seed=6),
            mesh.varcoeff3d((40, 30, 8), seed=7, permute=True)]


def contexts(ss):
    out = []
    for s in ss:
        c = _lib.Context(0)
        a = s.addr
        c.set_topology(a.n, a.nf, *a.arrays())
        out.append(c)
    return out


@pytest.mark.parametrize("precond,streams", [("Chebyshev", 3), ("GAMG", 4), ("Chebyshev", 1),
                                             ("GAMG", 16)])
def test_many_equals_single(require_gpu, precond, streams):
    import torch
    ss = systems()
    opts = _lib.default_options(tolerance=1e-8, preconditioner=precond)
    dev = torch.device("cuda", 0)
    dd = [torch.from_numpy(s.diag).to(dev) for s in ss]
    du = [torch.from_numpy(s.upper).to(dev) for s in ss]
    db = [torch.from_numpy(s.source).to(dev) for s in ss]
    # one at a time
    ref = []
    for s, c, d, u, b in zip(ss, contexts(ss), dd, du, db):
        x = torch.zeros(s.n, dtype=torch.float64, device=dev)
        c.set_coeffs_device(d, u, None)
        p = c.solve_device(_lib.CF_SOLVER_PCG, x, b, opts)
        torch.cuda.synchronize()
        ref.append((x.cpu().numpy(), p))
        c.close()
    # concurrently, coefficients staged by the call
    cs = contexts(ss)
    xs = [torch.zeros(s.n, dtype=torch.float64, device=dev) for s in ss]
    perfs = _lib.solve_many_device(cs, _lib.CF_SOLVER_PCG, xs, db, opts, streams=streams,
                                   diags=dd, uppers=du)
    for k, (x, p) in enumerate(zip(xs, perfs)):
        xr, pr = ref[k]
        assert np.array_equal(x.cpu().numpy(), xr), k
        for f in FIELDS:
            assert getattr(p, f) == getattr(pr, f), (k, f)
        assert p.converged
    # a second call reuses the staged coefficients (diags omitted)
    xs2 = [torch.zeros(s.n, dtype=torch.float64, device=dev) for s in ss]
    perfs2 = _lib.solve_many_device(cs, _lib.CF_SOLVER_PCG, xs2, db, opts, streams=streams)
    for k in range(len(ss)):
        assert np.array_equal(xs2[k].cpu().numpy(), ref[k][0]), k
        assert perfs2[k].nIterations == perfs[k].nIterations
    for c in cs:
        c.close()


def test_many_rejects(require_gpu):
    import torch
    s = mesh.poisson2d(10, 10, seed=8)
    cs = contexts([s])
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    b = torch.from_numpy(s.source).cuda()
    opts = _lib.default_options()
    for streams in (0, 65):
        with pytest.raises(_lib.CudaFoamError) as ei:
            _lib.solve_many_device(cs, _lib.CF_SOLVER_PCG, [x], [b], opts, streams=streams)
        assert ei.value.code == 1
    with pytest.raises(_lib.CudaFoamError) as ei:
        _lib.solve_many_device(cs + cs, _lib.CF_SOLVER_PCG, [x, x], [b, b], opts)
    assert ei.value.code == 1
    # coefficients never staged: the solve reports it
    with pytest.raises(_lib.CudaFoamError) as ei:
        _lib.solve_many_device(cs, _lib.CF_SOLVER_PCG, [x], [b], opts)
    assert ei.value.code == 4
    assert _lib.solve_many_device([], _lib.CF_SOLVER_PCG, [], [], opts) == []
    cs[0].close()
