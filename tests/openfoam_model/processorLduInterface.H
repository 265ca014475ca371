// Minimal model of OpenFOAM's processorLduInterface.H (see lduMatrix.H here).
#pragma once

#include "lduMatrix.H"

namespace Foam
{

class processorLduInterface
{
public:
    virtual ~processorLduInterface() = default;
    virtual label comm() const = 0;
    virtual int myProcNo() const = 0;
    virtual int neighbProcNo() const = 0;
    virtual int tag() const = 0;
};

}  // namespace Foam
