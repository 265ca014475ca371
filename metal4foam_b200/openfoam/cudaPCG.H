/*---------------------------------------------------------------------------*\
    cudaFoam: B200 (sm_100a) Krylov solvers for OpenFOAM lduMatrix systems

    Provenance: the lduMatrix::solver boilerplate of this file (run-time
    selection registration, constructor, solve forwarding) mirrors
    metal4Foam's metalPCG.H, Copyright (C) 2026 metal4Foam authors,
    SPDX-License-Identifier: GPL-3.0-or-later; this file is distributed
    under the same licence.

Class
    Foam::cudaPCG

Description
    Chebyshev-Jacobi PCG for symmetric lduMatrices: FP32 Krylov iterations, FP64 refinement and constant-mode deflation, all on the GPU.
    Drop-in for metal4Foam's metalPCG (metalPCG.C:16-19, metalPCG.H:47-92); selected
    in fvSolution with "solver cudaPCG;".

SourceFiles
    cudaPCG.C

\*---------------------------------------------------------------------------*/

#ifndef Foam_cudaPCG_H
#define Foam_cudaPCG_H

#include "cudaFoamSolver.H"

namespace Foam
{

class cudaPCG
:
    public cudaFoamSolver
{
public:

    TypeName("cudaPCG");

    cudaPCG
    (
        const word& fieldName,
        const lduMatrix& matrix,
        const FieldField<Field, scalar>& interfaceBouCoeffs,
        const FieldField<Field, scalar>& interfaceIntCoeffs,
        const lduInterfaceFieldPtrsList& interfaces,
        const dictionary& solverControls
    );

    virtual ~cudaPCG() = default;

    //- Solve in solveScalar precision
    virtual solverPerformance scalarSolve
    (
        solveScalarField& psi,
        const solveScalarField& source,
        const direction cmpt = 0
    ) const;

    //- Solve the matrix with this solver
    virtual solverPerformance solve
    (
        scalarField& psi,
        const scalarField& source,
        const direction cmpt = 0
    ) const;
};

} // End namespace Foam

#endif
