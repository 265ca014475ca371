// Minimal model of OpenFOAM's Pstream.H: UPstream, UIPstream/UOPstream raw
// transfers and reduce (see lduMatrix.H here).
#pragma once

#include <ios>

#include "lduMatrix.H"

namespace Foam
{

class UPstream
{
public:
    enum class commsTypes : char { buffered, scheduled, nonBlocking };
    static label worldComm;
    static bool parRun();
    static int myProcNo(const label communicator = worldComm);
    static int msgType();
    static label nRequests();
    static void waitRequests(const label pos = 0);
};

class UIPstream
{
public:
    static std::streamsize read(const UPstream::commsTypes commsType, const int fromProcNo,
                                char* buf, const std::streamsize bufSize,
                                const int tag = UPstream::msgType(),
                                const label communicator = UPstream::worldComm);
};

class UOPstream
{
public:
    static bool write(const UPstream::commsTypes commsType, const int toProcNo,
                      const char* buf, const std::streamsize bufSize,
                      const int tag = UPstream::msgType(),
                      const label communicator = UPstream::worldComm);
};

template <class T>
struct sumOp
{
    T operator()(const T& a, const T& b) const { return a + b; }
};

template <class T>
struct maxOp
{
    T operator()(const T& a, const T& b) const { return a > b ? a : b; }
};

template <class T, class BinaryOp>
void reduce(T& value, const BinaryOp& bop, const int tag = UPstream::msgType(),
            const label comm = UPstream::worldComm);

}  // namespace Foam
