/*---------------------------------------------------------------------------*\
    cudaFoam: B200 (sm_100a) Krylov solvers for OpenFOAM lduMatrix systems

    Provenance: the lduMatrix::solver boilerplate of this file (run-time
    selection registration, constructor, solve forwarding) mirrors
    metal4Foam's metalPBiCGStab.C, Copyright (C) 2026 metal4Foam authors,
    SPDX-License-Identifier: GPL-3.0-or-later; this file is distributed
    under the same licence.
\*---------------------------------------------------------------------------*/

#include "cudaPBiCGStab.H"
#include "PrecisionAdaptor.H"

namespace Foam
{
    defineTypeNameAndDebug(cudaPBiCGStab, 0);

    lduMatrix::solver::addsymMatrixConstructorToTable<cudaPBiCGStab>
        addcudaPBiCGStabSymMatrixConstructorToTable_;

    lduMatrix::solver::addasymMatrixConstructorToTable<cudaPBiCGStab>
        addcudaPBiCGStabAsymMatrixConstructorToTable_;
}


Foam::cudaPBiCGStab::cudaPBiCGStab
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


Foam::solverPerformance Foam::cudaPBiCGStab::scalarSolve
(
    solveScalarField& psi,
    const solveScalarField& source,
    const direction cmpt
) const
{
    return solveImpl(typeName, true, psi, source, cmpt);
}


Foam::solverPerformance Foam::cudaPBiCGStab::solve
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
