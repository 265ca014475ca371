"""Adjoint of the solve (the design's differentiation row): the transpose
solve reuses the forward kernels on A^T (upper/lower exchanged) and a
face-parallel kernel forms the gradients.  Checked against an FP64 CPU
adjoint on all coefficients (1e-4 relative) and central FP64 finite
differences (h = 1e-6) on 64 seeded coefficients, through the thin
torch.autograd.Function of tests/ldu_autograd.py."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

TIGHT = dict(tolerance=1e-10, relTol=0.0, maxRestarts=12, maxIter=5000)
# the adjoint source x - x* is not consistent: after the source transfer the
# FP32-inner refinement reaches a few 1e-10 on the 64^3 pinned Poisson
# matrix; 1e-9 is five orders tighter than the 1e-4 gradient check needs
ADJ = dict(tolerance=1e-9, relTol=0.0, maxRestarts=12, maxIter=5000)


def cpu_adjoint(oracle, s, xstar):
    """FP64 reference: x and lambda from FP64 Krylov solves (x to 1e-13 L2;
    lambda to 1e-10, about the attainable floor for an adjoint source with a
    large mean, which the single pinned cell turns into a point sink), the
    gradients from the oracle's face pass.  tests/test_oracle_adjoint.py
    checks this reference against sparse direct solves."""
    x, _ = oracle.cg64(s, tol=1e-13)
    lam, _ = oracle.cg64(s, b=x - xstar, tol=1e-10, transpose=True)
    dU, dL, dD = oracle.face_gradients(s, lam, x)
    return x, lam, dU, dL, dD


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_face_gradients_bit_exact(require_gpu, oracle):
    s = mesh.upwind3d((11, 9, 7), seed=41)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    rng = np.random.default_rng(1)
    lam, x = rng.standard_normal(s.n), rng.standard_normal(s.n)
    got = ctx.face_gradients(lam, x, s.nf)
    ref = oracle.face_gradients(s, lam, x)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
    ctx.close()


def test_transpose_operator(require_gpu, oracle):
    s = mesh.upwind3d((10, 9, 8), seed=42)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    x = np.random.default_rng(2).standard_normal(s.n)
    ctx.set_transpose(True)
    assert np.array_equal(ctx.amul(x), oracle.amul(s, x, transpose=True))
    ctx.set_transpose(False)
    assert np.array_equal(ctx.amul(x), oracle.amul(s, x))
    ctx.close()


@pytest.mark.parametrize("kind", ["symmetric", "asymmetric", "symmetric_gamg"])
def test_adjoint_vs_fp64_cpu_adjoint(require_gpu, oracle, kind):
    """symmetric_gamg: forward and adjoint solves preconditioned by the
    opt-in multigrid V-cycle, checked against the same FP64 reference."""
    extra = dict(preconditioner="GAMG") if kind == "symmetric_gamg" else {}
    if kind.startswith("symmetric"):
        s, xstar = mesh.adjoint_system((20, 20, 20), seed=43)
        solver = _lib.CF_SOLVER_PCG
    else:
        s = mesh.upwind3d((16, 16, 16), seed=44)
        xstar = np.random.default_rng(3).standard_normal(s.n)
        solver = _lib.CF_SOLVER_PBICGSTAB
    x_ref, lam_ref, dU_ref, dL_ref, dD_ref = cpu_adjoint(oracle, s, xstar)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    opts = _lib.default_options(**TIGHT, **extra)
    x = np.zeros(s.n)
    p = ctx.solve(solver, x, s.source, opts)
    assert p.converged and p.finalResidual < 1e-10
    lam, dU, dL, dD, pa = ctx.solve_adjoint(solver, x, x - xstar, s.nf,
                                            _lib.default_options(**ADJ, **extra))
    assert pa.converged and pa.finalResidual < 1e-9
    assert rel_err(x, x_ref) < 1e-6
    assert rel_err(lam, lam_ref) < 1e-4
    assert rel_err(dU, dU_ref) < 1e-4
    assert rel_err(dL, dL_ref) < 1e-4
    assert rel_err(dD, dD_ref) < 1e-4
    # after the adjoint the forward operator is staged again
    xx = np.random.default_rng(4).standard_normal(s.n)
    assert np.array_equal(ctx.amul(xx), oracle.amul(s, xx))
    ctx.close()


def test_autograd_vs_central_fd(require_gpu):
    """Gradients of L = 0.5 ||x - x*||^2 wrt b, diag, upper and lower through
    the torch.autograd.Function, against central FP64 finite differences
    (h = 1e-6, direct sparse solves) on 64 seeded coefficients."""
    import scipy.sparse.linalg as spla
    import torch

    from ldu_autograd import solve

    s0, xstar = mesh.adjoint_system((10, 9, 8), seed=45)
    # independent lower so dL/dlower is a genuine partial derivative
    s = mesh.LduSystem(s0.name, s0.addr, s0.diag, s0.upper, s0.upper.copy(), s0.source,
                       s0.psi)
    diag = torch.tensor(s.diag, requires_grad=True)
    upper = torch.tensor(s.upper, requires_grad=True)
    lower = torch.tensor(s.lower, requires_grad=True)
    b = torch.tensor(s.source, requires_grad=True)
    ctx = _lib.Context(0)
    opts = _lib.default_options(**TIGHT)
    x = solve(diag, upper, lower, b, ctx, s.addr, opts, _lib.CF_SOLVER_PBICGSTAB)
    loss = 0.5 * torch.sum((x - torch.from_numpy(xstar)) ** 2)
    loss.backward()
    grads = {"diag": diag.grad.numpy(), "upper": upper.grad.numpy(),
             "lower": lower.grad.numpy(), "b": b.grad.numpy()}

    def L_of(arrs):
        t = mesh.LduSystem("fd", s.addr, arrs["diag"], arrs["upper"], arrs["lower"],
                           arrs["b"], s.psi)
        xs = spla.spsolve(mesh.to_csr(t).tocsc(), arrs["b"])
        return 0.5 * float(np.sum((xs - xstar) ** 2))

    base = {"diag": s.diag.copy(), "upper": s.upper.copy(), "lower": s.lower.copy(),
            "b": s.source.copy()}
    rng = np.random.default_rng(46)
    h = 1e-6
    scale = max(np.max(np.abs(g)) for g in grads.values())
    checked = 0
    for name in ("diag", "upper", "lower", "b"):
        for idx in rng.choice(base[name].shape[0], 16, replace=False):
            p = {k: v.copy() for k, v in base.items()}
            m = {k: v.copy() for k, v in base.items()}
            p[name][idx] += h
            m[name][idx] -= h
            fd = (L_of(p) - L_of(m)) / (2 * h)
            an = grads[name][idx]
            assert abs(fd - an) <= 1e-4 * abs(an) + 1e-6 * scale, (name, idx, fd, an)
            checked += 1
    assert checked == 64
    ctx.close()


def test_c5_full_size_adjoint(require_gpu, oracle):
    """The 64^3 adjoint configuration: gradients wrt b, diag, upper, lower vs
    the FP64 CPU adjoint on all coefficients, 1e-4 relative."""
    s, xstar = mesh.adjoint_system((64, 64, 64), seed=5)
    x_ref, lam_ref, dU_ref, dL_ref, dD_ref = cpu_adjoint(oracle, s, xstar)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    opts = _lib.default_options(**TIGHT)
    x = np.zeros(s.n)
    p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, opts)
    assert p.converged and p.finalResidual < 1e-10
    lam, dU, dL, dD, pa = ctx.solve_adjoint(_lib.CF_SOLVER_PCG, x, x - xstar, s.nf,
                                            _lib.default_options(**ADJ))
    assert pa.converged and pa.finalResidual < 1e-9
    for got, ref in ((lam, lam_ref), (dU, dU_ref), (dL, dL_ref), (dD, dD_ref)):
        assert rel_err(got, ref) < 1e-4
    ctx.close()
