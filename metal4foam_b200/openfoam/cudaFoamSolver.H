/*---------------------------------------------------------------------------*\
    cudaFoam: B200 (sm_100a) Krylov solvers for OpenFOAM lduMatrix systems

Class
    Foam::cudaFoamSolver

Description
    Common driver of the cudaPCG / cudaPBiCGStab run-time selectable
    lduMatrix solvers: a drop-in for metalPCG / metalPBiCGStab
    (src/metal4Foam/solvers/metalFoamSolver.H:60-108 of metal4Foam).

    Everything below the solver call runs on the GPU through the C ABI of
    libcudafoam.so (include/cudafoam.h): the FP64 residual, normFactor and
    convergence tests, the row sums and constant-mode deflation, the FP32
    Krylov iterations, psi += delta and the restarts.  This class only hands
    over psi, source, the coefficients and the addressing.

    Controls (all optional), in the solver dictionary of fvSolution; the
    sub-dictionary may be called "cuda" or, for existing cases, "metal":

    \verbatim
    p
    {
        solver          cudaPCG;
        tolerance       1e-06;
        relTol          0.05;

        cuda
        {
            maxRestarts        8;     // FP64 refinement restarts
            iterationsPerSync  1;     // convergence-test granularity
            deflate            auto;  // on | off | auto (PCG)
            chebyshevOrder     8;     // 1 = Jacobi
            chebyshevRatio     30;
            graph              true;  // device-side iteration loop
            profile            false;
            verbose            false;
        }
    }
    \endverbatim

SourceFiles
    cudaFoamSolver.C

\*---------------------------------------------------------------------------*/

#ifndef Foam_cudaFoamSolver_H
#define Foam_cudaFoamSolver_H

#include "lduMatrix.H"

struct cf_context;
#include "cudafoam.h"

namespace Foam
{

class cudaFoamSolver
:
    public lduMatrix::solver
{
protected:

        //- The "cuda" (or "metal") sub-dictionary
        dictionary cudaDict_;

        //- The device context of this (field, mesh); created on first use
        cf_context* backend() const;

        //- The solver controls as the C ABI takes them
        cf_options cudaOptions() const;

        //- Decomposed case: this processor's subdomain, processor
        //  interfaces coupled over Pstream (cf_subdomain_solve)
        solverPerformance solveDecomposed
        (
            const word& solverName,
            const bool useBiCGStab,
            solveScalarField& psi,
            const solveScalarField& source
        ) const;

        //- The FP64 driver + GPU solve
        solverPerformance solveImpl
        (
            const word& solverName,
            const bool useBiCGStab,
            solveScalarField& psi,
            const solveScalarField& source,
            const direction cmpt
        ) const;

        cudaFoamSolver(const cudaFoamSolver&) = delete;
        void operator=(const cudaFoamSolver&) = delete;

public:

        cudaFoamSolver
        (
            const word& fieldName,
            const lduMatrix& matrix,
            const FieldField<Field, scalar>& interfaceBouCoeffs,
            const FieldField<Field, scalar>& interfaceIntCoeffs,
            const lduInterfaceFieldPtrsList& interfaces,
            const dictionary& solverControls
        );

        virtual ~cudaFoamSolver() = default;
};

} // End namespace Foam

#endif
