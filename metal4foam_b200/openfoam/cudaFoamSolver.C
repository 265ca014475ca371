/*---------------------------------------------------------------------------*\
    cudaFoam: B200 (sm_100a) Krylov solvers for OpenFOAM lduMatrix systems

    Driver of cudaPCG / cudaPBiCGStab over libcudafoam.so.  Same controls,
    same residual definitions and the same fatal errors as metal4Foam's
    metalFoamSolver (src/metal4Foam/solvers/metalFoamSolver.C:32-437); the
    FP64 steps that file runs on the CPU run inside cf_solve on the device.
\*---------------------------------------------------------------------------*/

#include "cudaFoamSolver.H"
#include "PrecisionAdaptor.H"
#include "Pstream.H"
#include "processorLduInterface.H"
#include "cudafoam.h"

#include <fenv.h>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

static_assert
(
    sizeof(Foam::solveScalar) == 8,
    "cudaFoam requires a double-precision (WM_PRECISION_OPTION=DP) build"
);
static_assert
(
    sizeof(Foam::label) == 4,
    "cudaFoam requires a 32-bit label (WM_LABEL_SIZE=32) build"
);

namespace
{

// OpenFOAM traps SIGFPE; driver and runtime code may raise FP exceptions
// legitimately.  Run every library call with the default FP environment and
// restore the caller's afterwards (per thread).
struct FpTrapGuard
{
    fenv_t saved;
    FpTrapGuard() { fegetenv(&saved); fesetenv(FE_DFL_ENV); }
    ~FpTrapGuard() { fesetenv(&saved); }
};

struct ContextDeleter
{
    void operator()(cf_context* c) const { cf_context_destroy(c); }
};

struct SubdomainDeleter
{
    void operator()(cf_subdomain* d) const { cf_subdomain_destroy(d); }
};

// The subdomain solve's communication over Pstream (MPI): global sums and
// maxima by reduce, halo values by non-blocking raw transfers with each
// neighbouring processor.  The library stages device data through host
// buffers (hostBuffers = 1), so MPI needs no CUDA awareness.
struct PstreamComm
{
    Foam::label comm;
    int tag;

    static int allreduce(void* user, double* values, int32_t count, int32_t op, void*)
    {
        const PstreamComm& c = *static_cast<const PstreamComm*>(user);
        for (int32_t i = 0; i < count; ++i)
        {
            if (op == 1)
                Foam::reduce(values[i], Foam::maxOp<double>(), c.tag, c.comm);
            else
                Foam::reduce(values[i], Foam::sumOp<double>(), c.tag, c.comm);
        }
        return 0;
    }

    static int exchange(void* user, int32_t nInterfaces, const int32_t* neighbour,
                        const int32_t* nFaces, int32_t elemBytes, const void* const* send,
                        void* const* recv, void*)
    {
        const PstreamComm& c = *static_cast<const PstreamComm*>(user);
        const Foam::label start = Foam::UPstream::nRequests();
        for (int32_t p = 0; p < nInterfaces; ++p)
        {
            Foam::UIPstream::read
            (
                Foam::UPstream::commsTypes::nonBlocking, neighbour[p],
                static_cast<char*>(recv[p]), std::streamsize(nFaces[p])*elemBytes, c.tag,
                c.comm
            );
        }
        for (int32_t p = 0; p < nInterfaces; ++p)
        {
            Foam::UOPstream::write
            (
                Foam::UPstream::commsTypes::nonBlocking, neighbour[p],
                static_cast<const char*>(send[p]), std::streamsize(nFaces[p])*elemBytes,
                c.tag, c.comm
            );
        }
        Foam::UPstream::waitRequests(start);
        return 0;
    }
};

int deflateMode(const Foam::word& w)
{
    if (w == "on") return CF_DEFLATE_ON;
    if (w == "off") return CF_DEFLATE_OFF;
    if (w == "auto") return CF_DEFLATE_AUTO;
    FatalErrorInFunction
        << "deflate must be on, off or auto, not " << w << Foam::exit(Foam::FatalError);
    return CF_DEFLATE_AUTO;
}

int preconditionerKind(const Foam::word& w)
{
    if (w == "Chebyshev") return CF_PRECOND_CHEBYSHEV;
    if (w == "GAMG") return CF_PRECOND_GAMG;
    FatalErrorInFunction
        << "preconditioner must be Chebyshev or GAMG, not " << w
        << Foam::exit(Foam::FatalError);
    return CF_PRECOND_CHEBYSHEV;
}

} // anonymous namespace


Foam::cudaFoamSolver::cudaFoamSolver
(
    const word& fieldName,
    const lduMatrix& matrix,
    const FieldField<Field, scalar>& interfaceBouCoeffs,
    const FieldField<Field, scalar>& interfaceIntCoeffs,
    const lduInterfaceFieldPtrsList& interfaces,
    const dictionary& solverControls
)
:
    lduMatrix::solver
    (
        fieldName,
        matrix,
        interfaceBouCoeffs,
        interfaceIntCoeffs,
        interfaces,
        solverControls
    ),
    cudaDict_
    (
        solverControls.found("cuda")
      ? solverControls.subDict("cuda")
      : solverControls.subOrEmptyDict("metal")
    )
{}


cf_context* Foam::cudaFoamSolver::backend() const
{
    // The solver object is rebuilt on every fvMatrix::solve: keep one device
    // context per (field, mesh) for the run, as the reference does.
    static std::map<std::string, std::unique_ptr<cf_context, ContextDeleter>> cache;

    std::ostringstream key;
    key << fieldName_ << '@' << static_cast<const void*>(&matrix_.mesh());
    auto& slot = cache[key.str()];
    if (!slot)
    {
        FpTrapGuard fpe;
        cf_context* c = nullptr;
        if (cf_context_create(&c, 0) != CF_OK)
        {
            FatalErrorInFunction
                << "CUDA backend unavailable: " << cf_last_error()
                << exit(FatalError);
        }
        slot.reset(c);
        Info<< "    " << cf_context_description(c) << nl;
    }
    return slot.get();
}


Foam::solverPerformance Foam::cudaFoamSolver::solveImpl
(
    const word& solverName,
    const bool useBiCGStab,
    solveScalarField& psi,
    const solveScalarField& source,
    const direction cmpt
) const
{
    // Processor interfaces of a decomposed case: the subdomain solve
    // (halo exchange and global sums over Pstream).  Other coupled
    // interfaces (cyclic/AMI) cannot be applied inside the device-resident
    // iteration, as in the reference (metalFoamSolver.C:89-99).
    bool decomposed = false;
    forAll(interfaces_, patchi)
    {
        if (interfaces_.set(patchi))
        {
            if
            (
                !UPstream::parRun()
             || !isA<processorLduInterface>(interfaces_[patchi].interface())
            )
            {
                FatalErrorInFunction
                    << solverName << " supports processor interfaces only "
                    << "(no cyclic/AMI coupled boundaries)."
                    << exit(FatalError);
            }
            decomposed = true;
        }
    }
    if (decomposed)
    {
        return solveDecomposed(solverName, useBiCGStab, psi, source);
    }

    (void)cmpt;   // every component of a segregated solve is a scalar system here
    solverPerformance solverPerf(solverName, fieldName_);
    cf_context* ctx = backend();
    FpTrapGuard fpe;

    const lduAddressing& addr = matrix_.mesh().lduAddr();
    const label nCells = addr.size();
    const label nFaces = addr.upperAddr().size();

    auto check = [&](int rc, const char* what)
    {
        if (rc != CF_OK)
        {
            FatalErrorInFunction
                << solverName << ": " << what << " failed: " << cf_last_error()
                << exit(FatalError);
        }
    };

    check
    (
        cf_set_topology
        (
            ctx, nCells, nFaces,
            addr.lowerAddr().cdata(),
            addr.upperAddr().cdata(),
            addr.ownerStartAddr().cdata(),
            addr.losortAddr().cdata(),
            addr.losortStartAddr().cdata()
        ),
        "cf_set_topology"
    );
    double tConvert = 0;
    check
    (
        cf_set_coeffs
        (
            ctx,
            matrix_.diag().cdata(),
            matrix_.upper().cdata(),
            matrix_.hasLower() ? matrix_.lower().cdata() : nullptr,
            &tConvert
        ),
        "cf_set_coeffs"
    );

    cf_options opts = cudaOptions();
    // autotune yes: time the SpMV launch shapes once per context (the mesh
    // of a context does not change during a run) and keep the fastest
    if (cudaDict_.getOrDefault<bool>("autotune", false))
    {
        static std::set<const cf_context*> tuned;
        if (tuned.insert(ctx).second)
        {
            cf_spmv_config best;
            check(cf_autotune(ctx, 20, 1, &best, nullptr, 0, nullptr), "cf_autotune");
            if (opts.verbose)
            {
                Info<< "    " << solverName << " SpMV shape: layout " << best.layout
                    << " rowsPerWarp " << best.rowsPerWarp << " blockSize "
                    << best.blockSize << " rhsTile " << best.rhsTile << nl;
            }
        }
    }

    cf_performance perf;
    check
    (
        cf_solve
        (
            ctx,
            useBiCGStab ? CF_SOLVER_PBICGSTAB : CF_SOLVER_PCG,
            psi.data(),
            source.cdata(),
            &opts,
            &perf
        ),
        "cf_solve"
    );

    solverPerf.initialResidual() = perf.initialResidual;
    solverPerf.finalResidual() = perf.finalResidual;
    solverPerf.nIterations() = perf.nIterations;
    solverPerf.checkConvergence(tolerance_, relTol_, log_);
    if (perf.singular)
    {
        solverPerf.checkSingularity(0);
    }

    // residual fields at entry and exit, as metalFoamSolver.C:112-117,429-434
    solveScalarField rA(nCells);
    check(cf_residual(ctx, 0, rA.data()), "cf_residual");
    matrix().setResidualField
    (
        ConstPrecisionAdaptor<scalar, solveScalar>(rA)(), fieldName_, true
    );
    check(cf_residual(ctx, 1, rA.data()), "cf_residual");
    matrix().setResidualField
    (
        ConstPrecisionAdaptor<scalar, solveScalar>(rA)(), fieldName_, false
    );

    if (opts.profile)
    {
        Info<< "    " << solverName << " profile: tConvert=" << 1000*tConvert
            << "ms" << nl;
    }
    return solverPerf;
}

cf_options Foam::cudaFoamSolver::cudaOptions() const
{
    cf_options opts;
    cf_options_default(&opts);
    opts.tolerance = tolerance_;
    opts.relTol = relTol_;
    opts.maxIter = maxIter_;
    opts.minIter = minIter_;
    opts.maxRestarts = cudaDict_.getOrDefault<label>("maxRestarts", 8);
    opts.iterationsPerSync = cudaDict_.getOrDefault<label>("iterationsPerSync", 1);
    opts.deflate = deflateMode(cudaDict_.getOrDefault<word>("deflate", "auto"));
    opts.chebyshevOrder = cudaDict_.getOrDefault<label>("chebyshevOrder", 8);
    opts.chebyshevRatio = cudaDict_.getOrDefault<scalar>("chebyshevRatio", 30.0);
    opts.profile = cudaDict_.getOrDefault<bool>("profile", false);
    opts.verbose = cudaDict_.getOrDefault<bool>("verbose", false);
    opts.graph = cudaDict_.getOrDefault<bool>("graph", true);
    opts.stagnationLimit = cudaDict_.getOrDefault<label>("stagnationLimit", 0);
    opts.persistentMaxCells = cudaDict_.getOrDefault<label>("persistentMaxCells", 0);
    opts.clusterMaxCells = cudaDict_.getOrDefault<label>("clusterMaxCells", 0);
    opts.preconditioner =
        preconditionerKind(cudaDict_.getOrDefault<word>("preconditioner", "Chebyshev"));
    opts.nSweeps = cudaDict_.getOrDefault<label>("nSweeps", 3);
    opts.nCellsInCoarsestLevel = cudaDict_.getOrDefault<label>("nCellsInCoarsestLevel", 128);
    opts.scaleCorrection = cudaDict_.getOrDefault<scalar>("scaleCorrection", 1.8);
    opts.smootherRatio = cudaDict_.getOrDefault<scalar>("smootherRatio", 8.0);

    return opts;
}


Foam::solverPerformance Foam::cudaFoamSolver::solveDecomposed
(
    const word& solverName,
    const bool useBiCGStab,
    solveScalarField& psi,
    const solveScalarField& source
) const
{
    FpTrapGuard fpe;
    auto check = [&](int rc, const char* what)
    {
        if (rc != CF_OK)
        {
            FatalErrorInFunction
                << solverName << ": " << what << " failed: " << cf_last_error()
                << exit(FatalError);
        }
    };

    // processor patches in patch order: neighbour, faceCells, coefficients
    std::vector<int32_t> neighbour, nIfFaces, faceCells;
    std::vector<double> ifCoeffs;
    label comm = UPstream::worldComm;
    int tag = UPstream::msgType();
    forAll(interfaces_, patchi)
    {
        if (!interfaces_.set(patchi)) continue;
        const lduInterface& iface = interfaces_[patchi].interface();
        const processorLduInterface& proc = refCast<processorLduInterface>(iface);
        const labelUList& fc = iface.faceCells();
        const Field<scalar>& coeffs = interfaceBouCoeffs_[patchi];
        neighbour.push_back(proc.neighbProcNo());
        nIfFaces.push_back(fc.size());
        for (label k = 0; k < fc.size(); ++k)
        {
            faceCells.push_back(fc.cdata()[k]);
            ifCoeffs.push_back(coeffs.cdata()[k]);
        }
        comm = proc.comm();
        tag = proc.tag();
    }

    // one subdomain per (field, mesh) for the run; topology set once
    static std::map<std::string, std::unique_ptr<cf_subdomain, SubdomainDeleter>> cache;
    std::ostringstream key;
    key << fieldName_ << '@' << static_cast<const void*>(&matrix_.mesh());
    auto& slot = cache[key.str()];
    const lduAddressing& addr = matrix_.mesh().lduAddr();
    if (!slot)
    {
        cf_subdomain* d = nullptr;
        check(cf_subdomain_create(&d, 0), "cf_subdomain_create");
        slot.reset(d);
        check
        (
            cf_subdomain_set_topology
            (
                d, addr.size(), addr.upperAddr().size(),
                addr.lowerAddr().cdata(), addr.upperAddr().cdata(),
                addr.ownerStartAddr().cdata(), addr.losortAddr().cdata(),
                addr.losortStartAddr().cdata(),
                int32_t(neighbour.size()), neighbour.data(), nIfFaces.data(),
                faceCells.data(), CF_REORDER_AUTO
            ),
            "cf_subdomain_set_topology"
        );
    }
    check
    (
        cf_subdomain_set_coeffs
        (
            slot.get(), matrix_.diag().cdata(), matrix_.upper().cdata(),
            matrix_.hasLower() ? matrix_.lower().cdata() : nullptr, ifCoeffs.data()
        ),
        "cf_subdomain_set_coeffs"
    );

    PstreamComm pc{comm, tag};
    cf_comm cc;
    cc.user = &pc;
    cc.allreduce = &PstreamComm::allreduce;
    cc.exchange = &PstreamComm::exchange;
    cc.abort = nullptr;
    cc.hostBuffers = 1;

    const cf_options opts = cudaOptions();
    cf_performance perf;
    check
    (
        cf_subdomain_solve
        (
            slot.get(), useBiCGStab ? CF_SOLVER_PBICGSTAB : CF_SOLVER_PCG, psi.data(),
            source.cdata(), &opts, &cc, &perf
        ),
        "cf_subdomain_solve"
    );

    solverPerformance solverPerf(solverName, fieldName_);
    solverPerf.initialResidual() = perf.initialResidual;
    solverPerf.finalResidual() = perf.finalResidual;
    solverPerf.nIterations() = perf.nIterations;
    solverPerf.checkConvergence(tolerance_, relTol_, log_);
    if (perf.singular)
    {
        solverPerf.checkSingularity(0);
    }
    return solverPerf;
}
