/*---------------------------------------------------------------------------*\
    cudaFoam: B200 (sm_100a) Krylov solvers for OpenFOAM lduMatrix systems

    Provenance: the lduMatrix::solver boilerplate of this file (run-time
    selection registration, constructor, solve forwarding) mirrors
    metal4Foam's metalPCG.C, Copyright (C) 2026 metal4Foam authors,
    SPDX-License-Identifier: GPL-3.0-or-later; this file is distributed
    under the same licence.
\*---------------------------------------------------------------------------*/

#include "cudaPCG.H"
#include "PrecisionAdaptor.H"

namespace Foam
{
    defineTypeNameAndDebug(cudaPCG, 0);

    lduMatrix::solver::addsymMatrixConstructorToTable<cudaPCG>
        addcudaPCGSymMatrixConstructorToTable_;
}


Foam::cudaPCG::cudaPCG
(
    const word& fieldName,
    const lduMatrix& matrix,
    const FieldField<Field, scalar>& interfaceBouCoeffs,
    const FieldField<Field, scalar>& interfaceIntCoeffs,
    const lduInterfaceFieldPtrsList& interfaces,
    const dictionary& solverControls
)
:
    cudaFoamSolver
    (
        fieldName,
        matrix,
        interfaceBouCoeffs,
        interfaceIntCoeffs,
        interfaces,
        solverControls
    )
{}


Foam::solverPerformance Foam::cudaPCG::scalarSolve
(
    solveScalarField& psi,
    const solveScalarField& source,
    const direction cmpt
) const
{
    return solveImpl(typeName, false, psi, source, cmpt);
}


Foam::solverPerformance Foam::cudaPCG::solve
(
    scalarField& psi_s,
    const scalarField& source,
    const direction cmpt
) const
{
    PrecisionAdaptor<solveScalar, scalar> tpsi(psi_s);
    return scalarSolve
    (
        tpsi.ref(),
        ConstPrecisionAdaptor<solveScalar, scalar>(source)(),
        cmpt
    );
}
