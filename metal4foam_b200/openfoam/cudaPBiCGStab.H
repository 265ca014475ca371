/*---------------------------------------------------------------------------*\
    cudaFoam: B200 (sm_100a) Krylov solvers for OpenFOAM lduMatrix systems

    Provenance: the lduMatrix::solver boilerplate of this file (run-time
    selection registration, constructor, solve forwarding) mirrors
    metal4Foam's metalPBiCGStab.H, Copyright (C) 2026 metal4Foam authors,
    SPDX-License-Identifier: GPL-3.0-or-later; this file is distributed
    under the same licence.

Class
    Foam::cudaPBiCGStab

Description
    Jacobi BiCGStab for symmetric and asymmetric lduMatrices: FP32 Krylov iterations and FP64 refinement on the GPU.
    Drop-in for metal4Foam's metalPBiCGStab (metalPBiCGStab.C:16-22); selected
    in fvSolution with "solver cudaPBiCGStab;".

SourceFiles
    cudaPBiCGStab.C

\*---------------------------------------------------------------------------*/

#ifndef Foam_cudaPBiCGStab_H
#define Foam_cudaPBiCGStab_H

#include "cudaFoamSolver.H"

namespace Foam
{

class cudaPBiCGStab
:
    public cudaFoamSolver
{
public:

    TypeName("cudaPBiCGStab");

    cudaPBiCGStab
    (
        const word& fieldName,
        const lduMatrix& matrix,
        const FieldField<Field, scalar>& interfaceBouCoeffs,
        const FieldField<Field, scalar>& interfaceIntCoeffs,
        const lduInterfaceFieldPtrsList& interfaces,
        const dictionary& solverControls
    );

    virtual ~cudaPBiCGStab() = default;

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
