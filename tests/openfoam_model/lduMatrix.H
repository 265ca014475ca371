// A minimal model of the OpenFOAM v2506 interfaces the cudaFoam adapter
// uses (lduMatrix::solver, lduAddressing, dictionary, solverPerformance,
// Field, the run-time selection and message macros), written for one
// purpose: compiling metal4foam_b200/openfoam/*.C with -fsyntax-only where
// OpenFOAM is not installed, so that the adapter's use of the C ABI
// (include/cudafoam.h) is type-checked.  It is not OpenFOAM and implements
// nothing.
#pragma once

#include <cstdint>
#include <ostream>
#include <string>
#include <vector>

namespace Foam
{

typedef int32_t label;
typedef double scalar;
typedef double solveScalar;
typedef unsigned char direction;

class word : public std::string
{
public:
    word() = default;
    word(const char* s) : std::string(s) {}
    word(const std::string& s) : std::string(s) {}
};

template <class T>
class UList
{
public:
    label size() const;
    const T* cdata() const;
    T* data();
};

typedef UList<label> labelUList;

template <class T>
class Field : public UList<T>
{
public:
    Field() = default;
    explicit Field(label n);
};

typedef Field<scalar> scalarField;
typedef Field<solveScalar> solveScalarField;

template <template <class> class F, class T>
class FieldField
{
public:
    const F<T>& operator[](label i) const;
};

class lduInterface
{
public:
    virtual ~lduInterface() = default;
    virtual const labelUList& faceCells() const = 0;
};

class lduInterfaceField
{
public:
    virtual ~lduInterfaceField() = default;
    const lduInterface& interface() const;
};

class lduInterfaceFieldPtrsList
{
public:
    label size() const;
    bool set(label i) const;
    const lduInterfaceField& operator[](label i) const;
};

template <class Type, class U>
inline bool isA(const U& t)
{
    return dynamic_cast<const Type*>(&t) != nullptr;
}

template <class Type, class U>
inline const Type& refCast(const U& t)
{
    return dynamic_cast<const Type&>(t);
}

class dictionary
{
public:
    dictionary() = default;
    bool found(const word& key) const;
    const dictionary& subDict(const word& key) const;
    dictionary subOrEmptyDict(const word& key) const;
    template <class T>
    T getOrDefault(const word& key, const T& deflt) const;
};

class lduAddressing
{
public:
    label size() const;
    const labelUList& lowerAddr() const;
    const labelUList& upperAddr() const;
    const labelUList& ownerStartAddr() const;
    const labelUList& losortAddr() const;
    const labelUList& losortStartAddr() const;
};

class lduMesh
{
public:
    const lduAddressing& lduAddr() const;
};

class SolverPerformance
{
public:
    SolverPerformance(const word& solverName, const word& fieldName);
    scalar& initialResidual();
    scalar& finalResidual();
    label& nIterations();
    bool checkConvergence(scalar tolerance, scalar relTolerance, int log = 0);
    bool checkSingularity(scalar residual);
};

typedef SolverPerformance solverPerformance;

class lduMatrix
{
public:
    const lduMesh& mesh() const;
    const scalarField& diag() const;
    const scalarField& upper() const;
    const scalarField& lower() const;
    bool hasLower() const;
    void setResidualField(const scalarField& residual, const word& fieldName,
                          bool initial) const;

    class solver
    {
    protected:
        word fieldName_;
        const lduMatrix& matrix_;
        const FieldField<Field, scalar>& interfaceBouCoeffs_;
        const FieldField<Field, scalar>& interfaceIntCoeffs_;
        lduInterfaceFieldPtrsList interfaces_;
        dictionary controlDict_;
        int log_;
        label minIter_;
        label maxIter_;
        scalar tolerance_;
        scalar relTol_;

    public:
        solver(const word& fieldName, const lduMatrix& matrix,
               const FieldField<Field, scalar>& interfaceBouCoeffs,
               const FieldField<Field, scalar>& interfaceIntCoeffs,
               const lduInterfaceFieldPtrsList& interfaces, const dictionary& solverControls);
        virtual ~solver() = default;
        const lduMatrix& matrix() const { return matrix_; }
        virtual solverPerformance solve(scalarField& psi, const scalarField& source,
                                        const direction cmpt = 0) const = 0;
        virtual solverPerformance scalarSolve(solveScalarField& psi,
                                              const solveScalarField& source,
                                              const direction cmpt = 0) const;

        template <class Type>
        struct addsymMatrixConstructorToTable
        {
            addsymMatrixConstructorToTable();
        };
        template <class Type>
        struct addasymMatrixConstructorToTable
        {
            addasymMatrixConstructorToTable();
        };
    };
};

struct errorExit
{
};
extern errorExit FatalError;

struct messageStream
{
};
extern std::ostream Info;
extern const char nl;

struct errorManip
{
};
errorManip exit(errorExit&, int errNo = 1);
std::ostream& operator<<(std::ostream& os, errorManip);
std::ostream& fatalErrorStream(const char* function);

}  // namespace Foam

#define FatalErrorInFunction ::Foam::fatalErrorStream(__func__)
#define forAll(list, i) for (::Foam::label i = 0; i < (list).size(); ++i)
#define TypeName(name) static const char* typeName
#define defineTypeNameAndDebug(Type, debug) const char* Type::typeName = #Type
