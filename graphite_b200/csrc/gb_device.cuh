// Device data layout and kernel launchers of libgraphite_b200.so.
//
// Layout in HBM (all indices uint32, new = renumbered order):
//   cell_geo  float4[N+G]   centroid xyz, volume            (interior, then ghosts)
//   face_geo  float4[2F]    (unit normal xyz, area), (face centre xyz, 0)
//   lsq       float4[2N]    inverse LSQ matrix, symmetric: (a00 a01 a02 a11), (a12 a22 - -)
//   ghost     uint2[G]      (interior cell, face) of each ghost
//   nfc       uint8[N]      faces of each interior cell (at most kSlots = 6)
// Per-face entries are slot-major: entry (slot t, cell i) at t * N + i, slot
// t = the cell's t-th face in the reference's element-local face order, so a
// warp's threads (consecutive cells) touch consecutive entries.  S = 6 N.
//   nb        uint2[S]      (face, neighbour cell)
//   twin      uint32[S]     the entry of the same face among the neighbour's
//                           entries, or S + g for a ghost neighbour N + g
//   cf_geo    float4[S]     face normal oriented away from the cell, area /
//                           cell volume
//   nbc       uint32[S]     neighbour cell
//   dn        float4[S]     neighbour centroid - cell centroid, 1 / |.|^2
//   df        float4[S]     face centre - cell centroid, |.|^3
// Fields (double-buffered values so that the update is a Jacobi sweep):
//   scalar    float [N+G] x2
//   vector    float4[N+G] x2 (xyz, pad)
//   gradient  scalar: float4[N] (gradient xyz, limiter)
//             vector: float4[3N], entry 3i+a = (gradient of component a, its limiter)
//   face rec  float[S+G] (rho) and float4[S+G] (rho u, rho E), owned by the
//             rho and rhou fields: the limited reconstruction of the cell's
//             state at each of its faces (per entry), then of each ghost's
//             state at its face (S + g)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "graphite_b200.h"

namespace gb {

struct DevMesh {
    int64_t N = 0, G = 0, F = 0, S = 0;   // S = kSlots * N per-face entries
    int max_faces = 0;                    // most faces of any interior cell (4 tet .. 6 hex)
    float4* cell_geo = nullptr;
    float4* face_geo = nullptr;
    uint8_t* nfc = nullptr;
    uint2* nb = nullptr;
    float4* lsq = nullptr;
    uint2* ghost = nullptr;
    uint32_t* twin = nullptr;
    float4* cf_geo = nullptr;
    uint32_t* nbc = nullptr;
    float4* dn = nullptr;
    float4* df = nullptr;
    // reduction scratch owned by the mesh
    double* red = nullptr;        // n_red_max partials + 1 result
    int n_red_max = 0;
    // nonzero *halt: the iteration kernels return at once (set by
    // k_reduce_final of a replayed loop once it has stopped); null in the
    // mesh's own copy, set only in the copy a replayed loop is captured with
    const int* halt = nullptr;
};

// Device control word of a replayed loop (gbEulerRun, gbNSIRun), updated by
// k_reduce_final after each iteration's residual: that residual goes to
// history[it_chunk] (below the history's capacity), the first of the run is
// kept as res0, and halt becomes 1 once a residual is below tolerance x res0
// or 2 once one is not finite; from then on the iterations left in the chunk
// do nothing.
struct RunCtl {
    unsigned long long it_chunk;   // iterations run in the current chunk
    unsigned long long it_run;     // iterations run since the loop started
    double res0;
    int halt;
    int pad;
};

// Pointers of the three conserved fields as one kernel argument.
struct EulerState {
    const float* rho;
    const float4* rhou;
    const float* rhoe;
};

// Outputs of the gradient / limiter pass: the gradients (may be null, then
// they are not stored) and the reconstructed face states the flux reads.
struct EulerGrad {
    float4* rho;       // N
    float4* rhou;      // 3N
    float4* rhoe;      // N
    float* rec_rho;    // S + G: reconstructed rho
    float4* rec_rhou;  // S + G: reconstructed (rho u, rho E)
};

struct FaceRecs {
    const float* rho;
    const float4* rhou;   // (rho u, rho E)
};

constexpr int kBlock = 256;
constexpr int kSlots = 6;   // faces per cell: tet 4, prism / pyramid 5, hex 6

int reduce_blocks(int64_t n);

// ---- metrics (float64, reference order), metrics.cu ----
void launch_face_metrics64(int64_t F, const double* nodes, const uint32_t* fns, const uint32_t* fn, double* area,
                           double* normal, double* centre, cudaStream_t s);
void launch_cell_metrics64(int64_t N, const uint32_t* cfs, const uint32_t* cf, const double* area,
                           const double* normal, const double* fcentre, double* ccentre, double* volume,
                           cudaStream_t s);
void launch_ghost_metrics64(int64_t G, int64_t N, const uint32_t* cfs, const uint32_t* cf, const uint32_t* cc,
                            const double* area, const double* normal, const double* fcentre, double* ccentre,
                            double* volume, cudaStream_t s);
void launch_lsq64(int64_t N, const uint32_t* cfs, const uint32_t* cc, const double* ccentre, double* minv,
                  cudaStream_t s);
void launch_layout(const DevMesh& m, const uint32_t* cell_old, const uint32_t* face_old, const double* area,
                   const double* normal, const double* fcentre, const double* ccentre, const double* volume,
                   const double* minv, cudaStream_t s);

// ---- Euler path, euler.cu ----
void launch_init(int64_t n, float* rho, float4* rhou, float* rhoe, float r, float3 ru, float e, cudaStream_t s);
void launch_bc_slip(const DevMesh& m, uint32_t g0, uint32_t g1, float* rho[2], float4* rhou[2], float* rhoe[2],
                    int cur, cudaStream_t s);
void launch_bc_farfield(const DevMesh& m, uint32_t g0, uint32_t g1, float* rho[2], float4* rhou[2],
                        float* rhoe[2], int cur, float3 mach, float p, float t, cudaStream_t s);
void launch_entry_geo(const DevMesh& m, cudaStream_t s);
// Boundary conditions the Euler gradient pass applies itself, by ghost
// region: ghosts [start[r], start[r+1]) (absolute cell indices) get type[r]:
// -1 none (their stored state), 0 slip, 1 far field with mach[r], p[r],
// temp[r]; with store set the computed ghost states are also stored into
// both value buffers (the replayed loop leaves them out and applies the
// table once after its last iteration instead, k_bc_table on the buffer the
// last gradient pass read).
constexpr int kMaxBcRegions = 16;
struct GhostBcTable {
    int n;
    int store;
    uint32_t start[kMaxBcRegions + 1];
    int type[kMaxBcRegions];
    float3 mach[kMaxBcRegions];
    float p[kMaxBcRegions], temp[kMaxBcRegions];
    float* rho[2];
    float4* rhou[2];
    float* rhoe[2];
};

void launch_grad_lim(const DevMesh& m, EulerState q, EulerGrad g, bool transposed, cudaStream_t s,
                     const GhostBcTable* ghosts = nullptr);
// every region's condition of the table in one ghost kernel (reads buffer cur)
void launch_bc_table(const DevMesh& m, const GhostBcTable& t, int cur, cudaStream_t s);

// Boundary conditions of the incompressible path applied by its gradient
// kernel, by ghost region: ghosts [start[r], start[r+1]) (absolute cell
// indices) get type[r]: -1 none (their stored state), 0 slip, 1 inlet/outlet
// with vinf[r], pinf[r], 2 no-slip wall; the computed ghost states are stored
// into both value buffers p[], u[].
constexpr int kMaxNsiRegions = 16;
struct NsiGhostTable {
    int n;
    uint32_t start[kMaxNsiRegions + 1];
    int type[kMaxNsiRegions];
    float3 vinf[kMaxNsiRegions];
    float pinf[kMaxNsiRegions];
    float* p[2];
    float4* u[2];
};
// partials_rho (may be null): also the per-block sums of the density part
// F_rho^2 V of the residual
void launch_flux(const DevMesh& m, EulerState q, FaceRecs r, float* rho_n, float4* rhou_n, float* rhoe_n,
                 float* err, double* partials, float cfl, cudaStream_t s, double* partials_rho = nullptr);
// the sum of the partials into history[ctl->it_chunk], before the iteration's
// k_reduce_final (which advances it_chunk)
void launch_reduce_history(int n_partials, const double* partials, const RunCtl* ctl, double* history,
                           unsigned long long history_cap, cudaStream_t s);
void launch_reduce_partials(int64_t n, const float* v, double* partials, cudaStream_t s);
// stage 1 with a caller-chosen number of blocks (one partial per block)
void launch_reduce_partials_blocks(int64_t n, const float* v, double* partials, int blocks, cudaStream_t s);
// Sum of the partials into out[0]; with ctl (a replayed loop) also the
// RunCtl bookkeeping above (history may be null).
void launch_reduce_final(int n_partials, const double* partials, double* out, cudaStream_t s,
                         RunCtl* ctl = nullptr, double* history = nullptr, unsigned long long history_cap = 0,
                         double tolerance = 0.0);

// One term coef x operator of gbFvmApplyTerms, on device arrays (fvmops.cu).
constexpr int kFvmMaxTerms = 8;
struct FvmTermDev {
    int op;
    float coef;
    const float* s;       // scalar input values (N + G) or null
    const float4* v;      // vector input values (N + G) or null
    const float4* g;      // the scalar input's gradients + limiters (N) or null
    const float4* phi;    // velocity field (N + G) or null
    float3 phi_c;         // constant velocity
};
// out_comps 1: out_s[i] = the sum at interior cell i; 3: out_v[i]
void launch_fvm_terms(const DevMesh& m, int out_comps, int n_terms, const FvmTermDev* terms, float* out_s,
                      float4* out_v, cudaStream_t st);

// permute helpers for host transfers (new <-> reference order)
void launch_gather_scalar(int64_t n, const float* src, const uint32_t* idx, float* dst, cudaStream_t s);
void launch_gather_vector(int64_t n, const float4* src, const uint32_t* idx, float* dst3, cudaStream_t s);
void launch_scatter_scalar(int64_t n, const float* src, const uint32_t* idx, float* dst, cudaStream_t s);
void launch_scatter_vector(int64_t n, const float* src3, const uint32_t* idx, float4* dst, cudaStream_t s);

void count_launch(int n = 1);

struct Topology;
struct Numbering;

// Device view of a loaded mesh, for other translation units of the library.
struct MeshAccess {
    const DevMesh* dev;
    const uint32_t* d_cell_new;            // reference order -> device order, N + G
    const uint32_t* region_start;          // device ghost ranges per region (host array)
    int n_regions;
    int64_t N, G;
    const Topology* topo;                  // host topology (reference numbering)
    const Numbering* num;                  // reference <-> device numbering
};
bool mesh_access(::cuMesh* mesh, MeshAccess* out);
bool reference_momentum();

// Device buffers of a field (device cell order; val[cur] is the current value).
struct FieldAccess {
    void* val[2];
    int cur;
    int comps;                             // 1 scalar (float), 3 vector (float4)
    size_t size;
    const float4* grad;                    // last stored gradients + limiters, or null
};
// Binds the field to `mesh` (its device order becomes the mesh's) and checks
// its size and number of components.
bool field_access(::FvmField* f, ::cuMesh* mesh, int comps, FieldAccess* out);

// State buffers of one instance of a batch (device cell order of its mesh).
struct BatchInstanceAccess {
    float* rho[2];
    float4* rhou[2];
    float* rhoe[2];
    int cur;
    ::cuMesh* mesh;
};
bool batch_instance(::gbBatch* b, int inst, BatchInstanceAccess* out);

}  // namespace gb
