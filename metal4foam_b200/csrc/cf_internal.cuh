// cf_internal.cuh -- device layout and state shared by the host driver and
// the kernels of the sm_100a Krylov path.
//
// Device layout of one LDU matrix (built once per mesh by cf_set_topology):
//
//   rows are cells in an internal order perm[] (identity or reverse
//   Cuthill-McKee), stored as SELL-32: 32 consecutive rows form a slice
//   (one warp), each slice is padded to its longest row, entries are
//   column-major inside a slice so lane l of a warp reads row l's k-th
//   entry at sliceOff[s] + 32*k + l (one 128-byte line per k).
//
//   Row i's off-diagonal entries keep the reference's order: first the
//   faces i owns (upper[f], ascending f = the ownerStart range), then the
//   faces whose neighbour is i (lower[f], losort order).  col[e] holds the
//   internal column, with bit 31 set on the neighbour-side entries; padding
//   is -1.  eface[e] is the face index of the entry (-1 on padding); it is
//   used once per cf_set_coeffs to gather upper/lower into val32/val64.
//
//   FP32 SpMV (the Krylov bulk) sums diag*x, then the entries in stored
//   order -- the order of the reference's ldu_spmv kernels.  FP64 SpMV (the
//   refinement residual) sums diag*x, then the neighbour-side entries, then
//   the owner-side entries -- the per-row order of lduMatrix::Amul's face
//   loop.  Both use separately rounded multiplies and adds, so each row is
//   bit-identical to the CPU oracle.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cf {

constexpr int NT = 256;            // threads per block (8 warps = 8 slices)
constexpr int SLICE = 32;          // SELL slice height = warp size
constexpr int MAXW_UNROLL = 8;     // unrolled slice width (3-D hex: 6)
constexpr int NPART = 4;           // reduction slots per kernel
constexpr int STAG_LIMIT = 50;     // metalFoamBackend.C:606
constexpr double VSMALL = 1.0e-300;

// Column offsets of the compact index stream: entry e of row r holds
// col - r in 16 bits (padding COL16_PAD).  Built when every column of the
// reordered matrix lies within 32767 rows of its row (RCM keeps a 3-D mesh's
// bandwidth near one plane of cells); it halves the index bytes of the FP32
// SpMVs and names the same columns, so every sum is unchanged.
constexpr short COL16_PAD = -32768;

// Paired order of a uniform-width (W) SELL slice starting at sliceBase:
// lane l's entries 2g and 2g+1 sit side by side (one 4-byte column pair, one
// 8-byte value pair per lane, 256 contiguous bytes of values per warp and
// pair), the last entry of an odd width alone.  Same entries as the
// column-major order, read with half the load instructions.
// The paired copy is kept for the slice widths of hexahedral (6), prismatic
// (5) and tetrahedral / 2-D quadrilateral (4) meshes, each with kernels
// compiled for that width.
constexpr int PAIR_MIN_W = 4;
constexpr int PAIR_MAX_W = 6;

__host__ __device__ inline long long pair_index(long long sliceBase, int W, int k, int lane)
{
    const int even = W & ~1;
    return k < even ? sliceBase + 64LL * (k >> 1) + 2 * lane + (k & 1)
                    : sliceBase + 32LL * even + lane;
}

struct DevSell
{
    int n;                          // rows
    int nslices;
    const int* sliceOff;            // [nslices + 1]
    const int* col;                 // [nnz_padded]
    const float* val;               // [nnz_padded]
    const double* val64;            // [nnz_padded]
    const short* col16 = nullptr;   // [nnz_padded] row-relative columns, or null
    int ellW = 0;                   // > 0: every slice has this width and slice s
                                    // starts at 32 s ellW (no sliceOff load)
    const short* pcol16 = nullptr;  // col16 in the paired order (uniform width only),
    const float* pval = nullptr;    // val in the paired order: the FP32 row reads these
};

// State of one inner solve (metalFoamBackend::Stats plus the device scalars
// of metalFoamKernels.metal:20-32, kept in FP64).
struct InnerState
{
    double wArA, wArAold, wApA, alpha, beta, res;
    double rA0rA, rA0rAold, rA0AyA, omega, tAtA, tAsA, resS;
    double bestRes, target, finalResSum;
    int it, maxIter, ips, lastSync, noProgress, stagLimit;
    int cur, best, nxt;             // correction buffer indices (0..2)
    int converged, singular, stagnated, done, early;
    int sel;                        // buffer holding the returned correction
    unsigned int ticket;
};

// FP64 driver quantities (metalFoamSolver.C:101-415).
struct DriverState
{
    double xbar, normFactor, initRes, finalRes;
    double rmean, dmean, ur, uu, l2r, l2b;
    double chebBeta;
    long long nPinned;
    int signflip;
    unsigned int ticket;
};

}  // namespace cf
