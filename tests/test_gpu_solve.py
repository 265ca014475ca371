"""Solver-level parity on the GPU through the C ABI and the plugin surface.

The inner FP32 solves are compared with the oracle's emulation of the
reference backend (metalFoamBackend.C:568-959): both converge and their
iteration counts agree within 10%.  Full solves (metalFoamSolver.C:77-437)
match the oracle driver's decisions (deflation, restarts) and reach the FP64
tolerance; the solution is checked against an FP64 CG oracle converged to
1e-12.  Edge cases: maxIter 0, already converged, zero source, breakdown.
"""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh
from metal4foam_b200.solver import backend_cache_clear, cudaPBiCGStab, cudaPCG, lduMatrix

pytestmark = pytest.mark.gpu


def close_iters(a, b, rel=0.10, slack=2):
    return abs(a - b) <= max(slack, rel * max(a, b))


def reference_envelope(s, run, relabels=3):
    """Iteration counts of the reference algorithm (oracle emulation) on the
    system and on relabelled copies: the spread the reference's own FP32
    rounding produces when only the reduction order changes."""
    out = [run(s)]
    for k in range(1, relabels + 1):
        out.append(run(mesh.relabel(s, 100 + k)))
    return out


def within_envelope(it, env, rel=0.10):
    return min(env) * (1 - rel) - 2 <= it <= max(env) * (1 + rel) + 2


def make_ctx(s, reorder="auto"):
    ctx = _lib.Context(0, reorder=reorder)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    return ctx


def l1_residual(s, psi, oracle, psi0=None):
    """sum|b - A psi| / normFactor, the factor taken at the initial psi0 as
    the driver does (metalFoamSolver.C:120,363-364)."""
    psi0 = np.zeros(s.n) if psi0 is None else psi0
    r = s.source - oracle.amul(s, psi)
    nf = oracle.normfactor(psi0, s.source, oracle.amul(s, psi0), oracle.sumA(s))
    return np.sum(np.abs(r)) / nf


@pytest.mark.parametrize("order", [1, 4, 8])
def test_inner_pcg_vs_reference_backend(require_gpu, oracle, order):
    # diagonally shifted so FP32 CG converges without deflation (the
    # quasi-singular pressure matrix stalls plain FP32 CG in the reference too)
    s = mesh.varcoeff3d((24, 24, 24), seed=11, permute=True, reference_cell=True)
    s.diag = s.diag * 1.02
    ctx = make_ctx(s)
    ctx.set_coeffs(s.diag, s.upper, None)
    r = s.source.copy()
    target = 1e-5 * np.sum(np.abs(r))
    bk = oracle.Backend(s)
    bk.set_coeffs(s.diag, s.upper, None)
    st_o = bk.pcg(r, target, 2000, 1, order, 3.0, 30.0)

    def ref_run(t):
        b2 = oracle.Backend(t)
        b2.set_coeffs(t.diag, t.upper, None)
        st = b2.pcg(t.source, target, 2000, 1, order, 3.0, 30.0)
        assert st.converged
        return st.nIterations

    env = reference_envelope(s, ref_run, relabels=2)
    st_g = ctx.pcg(r, target, 2000, 1, order, 3.0, 30.0)
    assert st_o.converged and st_g.converged
    assert within_envelope(st_g.nIterations, env), (st_g.nIterations, env)
    d_g = ctx.delta(s.n).astype(np.float64)
    d_o = bk.delta().astype(np.float64)
    # both corrections reduce the L1 residual to the target (FP64 check)
    for d in (d_g, d_o):
        assert np.sum(np.abs(r - oracle.amul(s, d))) <= 3 * target
    ctx.close()


def test_inner_bicgstab_vs_reference_backend(require_gpu, oracle):
    s = mesh.upwind3d((20, 20, 20), seed=12)
    ctx = make_ctx(s)
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    r = s.source.copy()
    target = 1e-5 * np.sum(np.abs(r))

    def ref_run(t):
        bk = oracle.Backend(t)
        bk.set_coeffs(t.diag, t.upper, t.lower)
        st = bk.bicgstab(t.source, target, 2000)
        assert st.converged
        return st.nIterations

    env = reference_envelope(s, ref_run)
    st_g = ctx.bicgstab(r, target, 2000)
    assert st_g.converged
    assert within_envelope(st_g.nIterations, env), (st_g.nIterations, env)
    d_g = ctx.delta(s.n).astype(np.float64)
    assert np.sum(np.abs(r - oracle.amul(s, d_g))) <= 3 * target
    ctx.close()


def test_inner_iterations_per_sync(require_gpu, oracle):
    s = mesh.poisson2d(40, 40, seed=13)
    ctx = make_ctx(s)
    ctx.set_coeffs(s.diag, s.upper, None)
    r = s.source.copy()
    target = 1e-4 * np.sum(np.abs(r))
    st1 = ctx.pcg(r, target, 5000, 1, 1)
    st7 = ctx.pcg(r, target, 5000, 7, 1)
    # convergence is only tested every 7 iterations: ceil to the batch
    assert st7.nIterations % 7 == 0
    assert st1.nIterations <= st7.nIterations < st1.nIterations + 7


def c1_controls(**kw):
    c = {"solver": "cudaPCG", "tolerance": 1e-6, "relTol": 0.0,
         "cuda": {"chebyshevOrder": 4, "deflate": "auto", "maxRestarts": 4}}
    c["cuda"].update(kw)
    return c


def test_c1_poisson_cudapcg_vs_reference_driver(require_gpu, oracle):
    s = mesh.poisson2d(128, 128, seed=0)
    m = lduMatrix(s.addr, s.diag, s.upper)
    psi = np.zeros(s.n)
    perf = lduMatrix.solver.New("p", m, c1_controls()).solve(psi, s.source)
    ref = oracle.metal_solve(s, chebyshevOrder=4, maxRestarts=4)
    assert perf.converged and ref.converged
    assert perf.finalResidual < 1e-6
    assert perf.deflated == ref.deflated
    assert close_iters(perf.nIterations, ref.nIterations), (perf.nIterations, ref.nIterations)
    assert perf.initialResidual == pytest.approx(ref.initialResidual, rel=1e-12)
    # independent FP64 residual of the returned psi
    assert l1_residual(s, psi, oracle) == pytest.approx(perf.finalResidual, rel=1e-6)
    x, _ = oracle.cg64(s)
    assert np.max(np.abs(psi - x)) < 1e-3 * np.max(np.abs(x))
    backend_cache_clear()


def test_residual_fields(require_gpu, oracle):
    s = mesh.varcoeff3d((18, 17, 16), seed=17, permute=True)
    ctx = make_ctx(s)
    ctx.set_coeffs(s.diag, s.upper, None)
    psi0 = np.random.default_rng(3).standard_normal(s.n)
    psi = psi0.copy()
    ctx.solve(_lib.CF_SOLVER_PCG, psi, s.source, _lib.default_options())
    r0 = ctx.residual(s.n, "initial")
    r1 = ctx.residual(s.n, "final")
    assert np.array_equal(r0, s.source - oracle.amul(s, psi0))
    ref = s.source - oracle.amul(s, psi)
    assert np.max(np.abs(r1 - ref)) <= 1e-12 * np.max(np.abs(s.source))
    ctx.close()


def test_graph_and_host_sync_agree_bitwise(require_gpu):
    s = mesh.varcoeff3d((20, 20, 20), seed=14, permute=True)
    m = lduMatrix(s.addr, s.diag, s.upper)
    p1 = np.zeros(s.n)
    p2 = np.zeros(s.n)
    a = lduMatrix.solver.New("p", m, c1_controls(graph=True)).solve(p1, s.source)
    b = lduMatrix.solver.New("q", m, c1_controls(graph=False)).solve(p2, s.source)
    assert a.nIterations == b.nIterations
    assert np.array_equal(p1, p2)
    backend_cache_clear()


@pytest.mark.parametrize("deflate", ["auto", "on", "off"])
def test_deflation_options_match_reference(require_gpu, oracle, deflate):
    s = mesh.varcoeff3d((16, 16, 16), seed=15, permute=False)
    m = lduMatrix(s.addr, s.diag, s.upper)
    psi = np.zeros(s.n)
    perf = cudaPCG("p", m, c1_controls(deflate=deflate, chebyshevOrder=8)).solve(psi, s.source)
    ref = oracle.metal_solve(s, deflate=deflate, chebyshevOrder=8, maxRestarts=4)
    assert perf.deflated == ref.deflated
    assert perf.chebBeta == ref.chebBeta          # Gershgorin bound bit-exact
    assert perf.converged == ref.converged
    assert perf.finalResidual < 1e-6
    backend_cache_clear()


def test_bicgstab_upwind_tolerance(require_gpu, oracle):
    s = mesh.upwind3d((32, 32, 32), seed=16)
    m = lduMatrix(s.addr, s.diag, s.upper, s.lower)
    psi = np.zeros(s.n)
    perf = cudaPBiCGStab("U", m, {"solver": "cudaPBiCGStab", "tolerance": 1e-8}).solve(
        psi, s.source)
    env = reference_envelope(
        s, lambda t: oracle.metal_solve(t, bicgstab=True, tolerance=1e-8).nIterations)
    assert perf.converged
    assert perf.finalResidual < 1e-8
    assert within_envelope(perf.nIterations, env), (perf.nIterations, env)
    assert l1_residual(s, psi, oracle) < 1.01e-8
    backend_cache_clear()


def test_edge_max_iter_zero(require_gpu, oracle):
    s = mesh.poisson2d(16, 16, seed=1)
    m = lduMatrix(s.addr, s.diag, s.upper)
    psi = np.zeros(s.n)
    perf = cudaPCG("p", m, {"solver": "cudaPCG", "maxIter": 0}).solve(psi, s.source)
    ref = oracle.metal_solve(s, maxIter=0)
    assert perf.nIterations == 0 == ref.nIterations
    assert not perf.converged and not ref.converged
    # one outer pass still runs: with deflation the constant-mode shift
    # (metalFoamSolver.C:344-361) moves psi by c = (u.r)/(u.u), as the reference
    assert perf.deflated and ref.deflated
    assert np.allclose(psi, ref.psi, rtol=0, atol=1e-12)
    assert perf.finalResidual == pytest.approx(ref.finalResidual, rel=1e-10)
    psi_off = np.zeros(s.n)
    cudaPCG("p", m, {"solver": "cudaPCG", "maxIter": 0, "cuda": {"deflate": "off"}}).solve(
        psi_off, s.source)
    assert np.all(psi_off == 0.0)
    backend_cache_clear()


def test_edge_already_converged_and_zero_source(require_gpu, oracle):
    s = mesh.poisson2d(16, 16, seed=2)
    x, _ = oracle.cg64(s, tol=1e-14)
    m = lduMatrix(s.addr, s.diag, s.upper)
    psi = x.copy()
    perf = cudaPCG("p", m, {"solver": "cudaPCG"}).solve(psi, s.source)
    assert perf.nIterations == 0 and perf.converged
    assert np.array_equal(psi, x)
    psi0 = np.zeros(s.n)
    perf0 = cudaPCG("p", m, {"solver": "cudaPCG"}).solve(psi0, np.zeros(s.n))
    assert perf0.initialResidual == 0.0 and perf0.nIterations == 0
    backend_cache_clear()


def test_edge_breakdown_reports_singular(require_gpu):
    s = mesh.poisson2d(16, 16, seed=3)
    diag = s.diag.copy()
    diag[7] = np.nan
    m = lduMatrix(s.addr, diag, s.upper)
    psi = np.zeros(s.n)
    perf = cudaPCG("p", m, {"solver": "cudaPCG", "cuda": {"deflate": "off"}}).solve(
        psi, s.source)
    assert perf.singular
    assert not perf.converged
    backend_cache_clear()


def test_bicgstab_where_fp32_reductions_break_down(require_gpu, oracle):
    """Upwind 64^3 to 1e-8: the reference's algorithm, whose dot products
    are folded in FP32, loses rA0.rA to cancellation (it falls from ~1e5 to
    rounding noise and then to exactly 0) and stops with a breakdown after
    55 iterations; the same iteration with FP64-accumulated reductions
    converges and states its FP64 residual."""
    s = mesh.upwind3d((64, 64, 64), seed=2)
    ref = oracle.metal_solve(s, bicgstab=True, tolerance=1e-8, maxIter=5000)
    assert ref.singular and not ref.converged
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    x = np.zeros(s.n)
    p = ctx.solve(_lib.CF_SOLVER_PBICGSTAB, x, s.source,
                  _lib.default_options(tolerance=1e-8, maxIter=5000))
    assert p.converged and not p.singular and p.finalResidual < 1e-8
    r = s.source - mesh.amul_numpy(s, x)
    assert np.sum(np.abs(r)) / p.normFactor == pytest.approx(p.finalResidual, rel=1e-9)
    ctx.close()


def _edge_system(n, low, upp, diag, upper, src):
    a = mesh.ldu_addressing(n, np.array(low, np.int32), np.array(upp, np.int32))
    return mesh.LduSystem("edge", a, np.asarray(diag, float), np.asarray(upper, float), None,
                          np.asarray(src, float), np.zeros(n))


@pytest.mark.parametrize("case", ["one_cell", "disconnected", "diagonal_only"])
@pytest.mark.parametrize("solver", [_lib.CF_SOLVER_PCG, _lib.CF_SOLVER_PBICGSTAB])
def test_edge_degenerate_meshes(require_gpu, oracle, case, solver):
    """A single cell (no faces), cells without neighbours next to a coupled
    chain, and a diagonal-only matrix: same iterations, flags and result as
    the reference algorithm."""
    if case == "one_cell":
        s = _edge_system(1, [], [], [2.0], [], [4.0])
    elif case == "disconnected":
        s = _edge_system(5, [0, 1], [1, 2], [2.0, 3.0, 2.0, 5.0, 1.0], [-1.0, -1.0],
                         [1.0, 2.0, 3.0, 4.0, 5.0])
    else:
        s = _edge_system(1000, [], [], np.linspace(1, 3, 1000), [], np.sin(np.arange(1000.0)))
    ref = oracle.metal_solve(s, bicgstab=solver == _lib.CF_SOLVER_PBICGSTAB)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    x = np.zeros(s.n)
    p = ctx.solve(solver, x, s.source, _lib.default_options())
    assert p.converged == ref.converged and p.deflated == ref.deflated
    assert p.nIterations == ref.nIterations and p.nRestarts == ref.nRestarts
    xd = np.linalg.solve(mesh.to_csr(s).toarray(), s.source)
    assert np.max(np.abs(x - xd)) <= 2 * max(np.max(np.abs(ref.psi - xd)), 1e-7) * np.max(np.abs(xd))
    ctx.close()
