// cf_host.hpp -- the context object behind the opaque cf_context handle.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "cf_internal.cuh"
#include "cf_kernels.cuh"

constexpr int CF_MAX_CHEB = 64;

struct cf_context
{
    // device / runtime (metalFoamBackend::Impl::init, metalFoamBackend.C:192-282)
    int device = 0;
    int numSMs = 1;
    int maxBlocksPerSM = 8;
    int l2Bytes = 0;
    bool good = false;
    std::string description = "cudaFoam: no device";
    cudaStream_t ownStream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
    std::map<const void*, int> occ;        // kernel -> resident blocks per SM
    long long launches = 0;                // kernels launched (graph bodies counted per pass)

    // topology (metalFoamBackend::setTopology, .C:454-519)
    bool hasTopo = false;
    int reorderMode = 2;                   // CF_REORDER_AUTO
    int topoReorderMode = -1;
    int n = 0, nf = 0, nslices = 0, maxRowLen = 0;
    int ellW = 0;                          // uniform slice width, 0 if the widths differ
    long long nnzp = 0;
    const int32_t* lastLow = nullptr;
    const int32_t* lastUpp = nullptr;
    std::vector<int32_t> perm;             // internal row -> caller's cell
    bool identityPerm = true;
    std::vector<void*> topoAllocs;
    int* d_sliceOff = nullptr;
    int* d_col = nullptr;
    short* d_col16 = nullptr;              // row-relative columns, when they fit in 16 bits
    short* d_pcol16 = nullptr;             // d_col16 in the paired order (uniform width)
    float* d_pval32 = nullptr;             // d_val32 in the paired order
    int* d_eface = nullptr;
    int* d_perm = nullptr;
    int* d_low = nullptr;
    int* d_upp = nullptr;

    // coefficients (metalFoamBackend::setCoeffs, .C:522-565)
    bool hasCoeffs = false;
    bool hasLower = false;
    int val32Sym = 1;
    double* d_diagIn = nullptr;            // caller's order
    double* d_upper = nullptr;             // face order
    double* d_lower = nullptr;
    double* d_diag64 = nullptr;            // internal order
    double* d_u = nullptr;                 // row sums A 1
    float* d_val32 = nullptr;
    double* d_val64 = nullptr;
    double* d_valT64 = nullptr;
    float* d_diag32 = nullptr;
    float* d_rD32 = nullptr;

    // vectors (internal order)
    double* d_psi = nullptr;
    double* d_b = nullptr;
    double* d_r64 = nullptr;
    double* d_io64 = nullptr;              // staging for caller-order FP64 data
    double* d_io64b = nullptr;
    double* d_r0 = nullptr;                // residual at the entry of the last solve
    bool hasResidual = false;
    bool transposed = false;               // operator staged as A^T (adjoint solves)
    double* d_gU = nullptr;                // face gradients (face order)
    double* d_gL = nullptr;
    double* d_gD = nullptr;                // diagonal gradient (caller order)
    float* d_rA = nullptr;
    float* d_W0 = nullptr;
    float* d_W1 = nullptr;
    float* d_Z0 = nullptr;
    float* d_Z1 = nullptr;
    float* d_P = nullptr;                  // 2n
    float* d_Q = nullptr;                  // 2n (BiCGStab's A yA ping-pong)
    float* d_T = nullptr;
    float* d_D = nullptr;                  // 3n
    float* d_io32 = nullptr;
    float* d_io32b = nullptr;
    float* d_io32c = nullptr;

    // scalars
    double* d_part = nullptr;
    cf::InnerState* d_st = nullptr;
    cf::DriverState* d_drv = nullptr;
    float* d_chebC = nullptr;
    double* d_scratch64 = nullptr;
    cf::InnerState* h_st = nullptr;        // pinned mirrors
    cf::DriverState* h_drv = nullptr;
    int lastInnerKind = -1;                // 0 pcg, 1 bicgstab (for cf_delta)
    int pendingBodyKernels = 0;            // kernels per graph-body pass of the last inner solve

    // instantiated inner-loop graphs keyed by (kind, chebyshev order)
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    std::map<std::pair<int, int>, int> graphKernels;   // kernels in each graph's loop body

    // several right-hand sides on this matrix (cf_multi.cu), built on first use
    void* multi = nullptr;
    std::vector<cf_context*> clones;       // contexts solving on this matrix (multi-RHS streams)

    // SpMV launch shape of the FP32 Krylov kernels (cf_tune.cu): layout
    // (CF_LAYOUT_*), rows per warp, block size, multi-RHS tile
    int maxCtasPerSM = 32;
    bool coopLaunch = false;               // device supports cooperative launches
    void* amg = nullptr;                   // GAMG hierarchy of the topology (cf_amg.cu)
    bool amgActive = false;                // inner PCG iterations use the V-cycle
    int clusterShift = 10;                 // log2(rows per CTA) of the cluster PCG for this mesh
    double clusterRemote = 1.0;            // fraction of entries whose column lies in another CTA
    unsigned int* d_bar = nullptr;         // grid barrier of persistent inner solves: count, generation, error
    long long waitPolls = 1LL << 24;       // polls of a bounded device-side wait before it gives up
    int cfgLayout = 0;
    int cfgRowsPerWarp = 32;
    int cfgBlockSize = 256;
    int cfgRhsTile = 0;         // 0: multi-RHS components as concurrent single solves
    int cfgIndexBits = 16;      // SELL-32 column stream: 16 (when built) or 32
    // the reference's addressing read directly (CF_LAYOUT_LDU), built on
    // first use; topology-lifetime allocations
    bool lduReady = false;
    int* d_own = nullptr;       // ownerStartAddr [n+1], caller's numbering
    int* d_losS = nullptr;      // losortStartAddr [n+1]
    int* d_los = nullptr;       // losortAddr [nf]
    int* d_uppI = nullptr;      // internal row of upperAddr[f]
    int* d_lowI = nullptr;      // internal row of lowerAddr[f]
    float* d_face32 = nullptr;  // [2 nf]: FP32 upper, then FP32 lower (face order)
};

// Frees the multi-RHS buffers and graphs (with the topology they point into).
void cf_multi_release(cf_context* c);

namespace cf {
// A context that solves on src's matrix: src's topology and coefficient
// arrays (read only, shared), every vector, state, graph and the FP32
// diagonal its own.  Freed with src's topology.
int context_clone_matrix(cf_context* src, cf_context** out);
// Refreshes a clone's own copies (FP32 diagonal, staging flags, launch
// shape) from src before a solve on src's current coefficients.
int context_clone_sync(cf_context* src, cf_context* clone);
}  // namespace cf

namespace cf {

// Host-side SELL-32 layout of one mesh (see cf_internal.cuh).
struct HostLayout
{
    std::vector<int32_t> perm;      // internal row -> caller's cell
    std::vector<int32_t> sliceOff;  // nslices + 1
    std::vector<int32_t> col;       // internal columns, bit 31 = neighbour side, -1 padding
    std::vector<int32_t> eface;     // face of each entry, -1 padding
    int32_t nslices = 0;
    long long nnzp = 0;
    int32_t maxw = 0;
    int32_t uniformW = 0;           // every slice this wide (0: widths differ)
};

int check_addressing(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
                     const int32_t* own, const int32_t* los, const int32_t* losS);
// xStart/xCol/xFace (optional, CSR over the caller's cells): extra entries
// appended to a row after its losort faces, with internal columns xCol and
// face indices xFace (processor-interface faces of a subdomain)
int build_layout(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
                 const int32_t* own, const int32_t* los, const int32_t* losS, bool rcm,
                 HostLayout& L, const int32_t* xStart = nullptr, const int32_t* xCol = nullptr,
                 const int32_t* xFace = nullptr);

int fail(int code, const std::string& msg);
double wall_now();
int grid_for(cf_context* c, const void* fn, long long work);
// One thread per row: the grid of row kernels without a grid-wide sum (their
// results do not depend on the grid; blocks that retire early are replaced,
// which keeps more loads in flight than a grid-stride loop per thread).
inline int rows_grid(long long n) { return (int)std::max(1LL, (n + NT - 1) / NT); }
DevSell sell_of(const cf_context* c);
PcgBufs pcg_bufs(const cf_context* c);
BicgBufs bicg_bufs(const cf_context* c);
int stage_vals(cf_context* c, int sym32);
int stage_diag32(cf_context* c, int deflate);
int stage_rowsums(cf_context* c);

// Launch-shape variants of the SpMV-carrying FP32 kernels (cf_tune.cu).
// spmv_default(c): the context runs the SELL-32 row-per-thread kernels of
// cf_kernels.cuh with 256-thread blocks; otherwise the launches below run
// the variant the configuration names.  Every variant forms each row of
// A x with the same operations in the same order, so A x is bit-identical;
// only the order in which the dot products are folded differs.
bool spmv_default(const cf_context* c);
int stage_face32(cf_context* c, const double* up, const double* lo, int sym32);
int launch_cheb_step_v(cf_context* c, bool last, const PcgBufs& B, const float* zin,
                       const float* win, float* wout, float* zout, int j);
int launch_pcg_p_spmv_v(cf_context* c, const PcgBufs& B, const float* wA);
int launch_bicg_ab_v(cf_context* c, const BicgBufs& B);
int launch_bicg_cd_v(cf_context* c, const BicgBufs& B, cudaGraphConditionalHandle h, int useCond);
int launch_spmv32_v(cf_context* c, const float* diag, const float* x, const float* w, float* y,
                    double* out);

// Inner solve as one cooperative kernel (cf_persist.cu) when the mesh has
// at most maxCells cells (<= 0: never) and the launch fits;
// *ran tells whether it was launched.  persistent_status reads the grid
// barrier's error word after the stream has completed.
int persistent_inner(cf_context* c, int kind, int order, int maxCells, bool* ran);
// Inner PCG inside one thread-block cluster (cf_cluster.cu) for meshes of
// at most min(maxCells, 16384) cells whose columns lie mostly in their own
// CTA; *ran tells whether it was launched.
int cluster_inner(cf_context* c, int order, int maxCells, bool* ran);
// log2(rows per CTA) of the cluster PCG for an n-row mesh: the smallest
// power of two >= 32 that needs at most 16 CTAs.
int cluster_shift(int n);
int persistent_status(cf_context* c);

// Aggregation multigrid preconditioner of the inner PCG (cf_amg.cu):
// hierarchy of the topology down to at most coarsestCap (<= 128) cells,
// coefficients of every level from the staged operator (deflated or not),
// and one inner iteration with the V-cycle as z = M r.
int amg_prepare(cf_context* c, int coarsestCap, bool profile = false);
int amg_stage(cf_context* c, int deflate, float scaleCorrection);
int launch_amg_body(cf_context* c, int degree, cudaGraphConditionalHandle h, int useCond,
                    int* kernels);
int amg_levels(const cf_context* c);
int amg_level_cells(const cf_context* c, int level);
void amg_release(cf_context* c);

}  // namespace cf
