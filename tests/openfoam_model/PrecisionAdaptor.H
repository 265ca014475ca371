// Minimal model of OpenFOAM's PrecisionAdaptor.H (see lduMatrix.H here).
#pragma once

#include "lduMatrix.H"

namespace Foam
{

template <class To, class From>
class PrecisionAdaptor
{
public:
    explicit PrecisionAdaptor(Field<From>& f);
    Field<To>& ref();
};

template <class To, class From>
class ConstPrecisionAdaptor
{
public:
    explicit ConstPrecisionAdaptor(const Field<From>& f);
    const Field<To>& operator()() const;
};

}  // namespace Foam
