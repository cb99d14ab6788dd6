// The Euler iteration on sm_100a: boundary ghosts, fused least-squares
// gradient + limiter of all five conserved variables, and the fused
// reconstruction / central flux / scalar dissipation / local-time-step
// update / squared-residual kernel with a deterministic float64 block
// reduction of the residual.
//
// Both hot kernels are cell-gathers over the renumbered (reverse
// Cuthill-McKee) mesh: one thread per interior cell walks its faces in the
// reference's element-local order, so every sum is taken in the reference's
// order and no atomics are used -- runs are bitwise reproducible.  Per-face
// data is stored slot-major (face slot t of cell i at t * N + i), so a warp
// reads and writes it coalesced.  The gradient pass streams the static face
// geometry, gathers the neighbours' states and writes, per face entry, the
// cell's limited reconstruction at that face; the flux pass streams its own
// entries (twin index, oriented normal with area / volume, reconstructed
// state) and gathers only the neighbour's 20-byte reconstructed state through
// the twin index.
#include "euler_ops.cuh"

namespace gb {
namespace {

// Resident blocks per SM the two hot kernels are compiled for (register
// budget 65536 / (kBlock * blocks)).
#ifndef GB_FLUX_BLOCKS
#define GB_FLUX_BLOCKS 6
#endif
#ifndef GB_GRAD_STAGED
#define GB_GRAD_STAGED 1
#endif
#ifndef GB_GRAD_BLOCKS
#define GB_GRAD_BLOCKS 5
#endif
constexpr int kFluxBlocksPerSM = GB_FLUX_BLOCKS;
constexpr int kGradBlocksPerSM = GB_GRAD_BLOCKS;

__global__ void k_init(int64_t n, float* rho, float4* rhou, float* rhoe, float r, float3 ru, float e) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rho[i] = r;
    rhou[i] = make_float4(ru.x, ru.y, ru.z, 0.f);
    rhoe[i] = e;
}

struct GhostBuf {
    float* rho[2];
    float4* rhou[2];
    float* rhoe[2];
    const int* halt;
};

// euler_slip_bc, src/models/euler.cu:412-442, on the ghosts [g0, g1); written
// to both value buffers so that the ghost values are current whichever buffer
// the next sweep reads.
__global__ void k_bc_slip(uint32_t g0, uint32_t g1, uint32_t N, const float4* __restrict__ cell_geo,
                          const float4* __restrict__ face_geo, const uint2* __restrict__ ghost, GhostBuf b, int cur) {
    const uint32_t t = g0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g1 || halted(b.halt)) return;
    float r, e;
    float4 ru;
    slip_ghost(cell_geo, face_geo, ghost[t - N], b.rho[cur], b.rhou[cur], b.rhoe[cur], r, ru, e);
    for (int k = 0; k < 2; ++k) {
        b.rho[k][t] = r;
        b.rhou[k][t] = ru;
        b.rhoe[k][t] = e;
    }
}

// euler_inletoutlet_bc, src/models/euler.cu:446-520, on the ghosts [g0, g1).
__global__ void k_bc_farfield(uint32_t g0, uint32_t g1, uint32_t N, const float4* __restrict__ cell_geo,
                              const float4* __restrict__ face_geo, const uint2* __restrict__ ghost, GhostBuf b,
                              int cur, float3 imach, float ip, float it) {
    const uint32_t t = g0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g1 || halted(b.halt)) return;
    float r, e;
    float4 ru;
    farfield_ghost(cell_geo, face_geo, ghost[t - N], b.rho[cur], b.rhou[cur], b.rhoe[cur], imach, ip, it, r, ru, e);
    for (int k = 0; k < 2; ++k) {
        b.rho[k][t] = r;
        b.rhou[k][t] = ru;
        b.rhoe[k][t] = e;
    }
}

// All regions' boundary conditions in one launch, from a GhostBcTable: ghost
// t takes its region's condition (the same slip_ghost / farfield_ghost as the
// per-region kernels; regions of type -1 are left as they are).
__global__ void k_bc_table(uint32_t N, uint32_t G, const float4* __restrict__ cell_geo,
                           const float4* __restrict__ face_geo, const uint2* __restrict__ ghost, GhostBcTable tb,
                           int cur, const int* halt) {
    const uint32_t t = N + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N + G || halted(halt)) return;
    int k = 0;
    while (k < tb.n - 1 && t >= tb.start[k + 1]) ++k;
    if (tb.type[k] < 0) return;
    float r, e;
    float4 ru;
    if (tb.type[k] == 0)
        slip_ghost(cell_geo, face_geo, ghost[t - N], tb.rho[cur], tb.rhou[cur], tb.rhoe[cur], r, ru, e);
    else
        farfield_ghost(cell_geo, face_geo, ghost[t - N], tb.rho[cur], tb.rhou[cur], tb.rhoe[cur], tb.mach[k], tb.p[k],
                       tb.temp[k], r, ru, e);
    for (int b = 0; b < 2; ++b) {
        tb.rho[b][t] = r;
        tb.rhou[b][t] = ru;
        tb.rhoe[b][t] = e;
    }
}

// Fused FvmEulerStepPrepare over the interior cells of one mesh: gradients,
// limiters and the reconstructed face states.
template <bool TRANSPOSED>
__global__ void __launch_bounds__(kBlock, kGradBlocksPerSM) k_grad_lim(MeshDev m, EulerState q, EulerGrad g) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (halted(m.halt)) return;
    if (i < m.N) grad_lim_cell<TRANSPOSED>(m, q, g, i);
}

// k_grad_lim with each cell's per-face entries (neighbour, LSQ offset, face
// offset: 36 B per face) staged in shared memory by cp.async as the first thing the
// thread does: all of a cell's entry streams are in flight together while the
// cell's own state loads, instead of one face per memory round trip.
#ifndef GB_GRAD_STAGE_THREADS
#define GB_GRAD_STAGE_THREADS 64
#endif
// 1: the face offsets are staged too; 0: read where used (less shared memory)
#ifndef GB_GRAD_STAGE_DF
#define GB_GRAD_STAGE_DF 1
#endif
// resident blocks per SM the registers are budgeted for, by the mesh's most
// faces per cell (shared-memory slots per thread)
#ifndef GB_STAGE_BLOCKS_F4
#define GB_STAGE_BLOCKS_F4 18
#endif
#ifndef GB_STAGE_BLOCKS_F5
#define GB_STAGE_BLOCKS_F5 16
#endif
#ifndef GB_STAGE_BLOCKS_F6
#define GB_STAGE_BLOCKS_F6 15
#endif
constexpr int kStageThreads = GB_GRAD_STAGE_THREADS;
constexpr bool kStageDf = GB_GRAD_STAGE_DF != 0;
template <int MAXF>
constexpr int stage_blocks() {
    return MAXF <= 4 ? GB_STAGE_BLOCKS_F4 : (MAXF == 5 ? GB_STAGE_BLOCKS_F5 : GB_STAGE_BLOCKS_F6);
}

// MAXF: shared-memory slots per thread, at least the mesh's most faces per cell
template <bool TRANSPOSED, typename Ghosts, int MAXF>
__global__ void __launch_bounds__(kStageThreads, stage_blocks<MAXF>())
    k_grad_lim_staged(MeshDev m, EulerState q, EulerGrad g, Ghosts gh) {
    constexpr int B = kStageThreads;
    __shared__ float4 s_dn[MAXF * B], s_df[kStageDf ? MAXF * B : 1];
    __shared__ uint32_t s_nbc[MAXF * B];
    const uint32_t tid = threadIdx.x;
    const uint32_t i = blockIdx.x * B + tid;
    if (i >= m.N || halted(m.halt)) return;
    const uint32_t nf = __ldg(&m.nfc[i]);
    for (uint32_t t = 0; t < nf; ++t) {
        const uint32_t k = i + t * m.N;
        cp_async4(&s_nbc[t * B + tid], &m.nbc[k]);
        cp_async16(&s_dn[t * B + tid], &m.dn[k]);
        if (kStageDf) cp_async16(&s_df[t * B + tid], &m.df[k]);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if constexpr (kStageDf)
        grad_lim_cell<TRANSPOSED>(m, q, g, i, nf, EntriesStaged<B>{s_nbc + tid, s_dn + tid, s_df + tid}, gh);
    else
        grad_lim_cell<TRANSPOSED>(m, q, g, i, nf, EntriesStagedDn<B>{s_nbc + tid, s_dn + tid, m.df + i, m.N}, gh);
}

template <bool TRANSPOSED, typename Ghosts>
void launch_staged(const DevMesh& d, const MeshDev& md, EulerState q, EulerGrad g, Ghosts gh, cudaStream_t s) {
    const unsigned gs = (unsigned)((d.N + kStageThreads - 1) / kStageThreads);
    if (d.max_faces <= 4) k_grad_lim_staged<TRANSPOSED, Ghosts, 4><<<gs, kStageThreads, 0, s>>>(md, q, g, gh);
    else if (d.max_faces == 5) k_grad_lim_staged<TRANSPOSED, Ghosts, 5><<<gs, kStageThreads, 0, s>>>(md, q, g, gh);
    else k_grad_lim_staged<TRANSPOSED, Ghosts, kSlots><<<gs, kStageThreads, 0, s>>>(md, q, g, gh);
}

// Fused flux / local-time-step update / squared residual over the interior
// cells of one mesh, with the residual summed per block in float64.
// RHO: also the density part of each cell's residual, F_rho^2 V, summed per
// block into partials_rho.
template <bool RHO>
__global__ void __launch_bounds__(kBlock, kFluxBlocksPerSM)
    k_flux(MeshDev m, EulerState q, FaceRecs r, float* __restrict__ rho_n, float4* __restrict__ rhou_n,
           float* __restrict__ rhoe_n, float* __restrict__ err, double* __restrict__ partials, float cfl,
           double* __restrict__ partials_rho) {
    if (halted(m.halt)) return;              // uniform over the grid
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double res = 0.0;
    float rsq = 0.f;
    if (i < m.N) res = (double)flux_cell(m, q, r, rho_n, rhou_n, rhoe_n, err, cfl, i, RHO ? &rsq : nullptr);
    const double bs = block_sum(res);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
    if (RHO) {
        __syncthreads();                     // block_sum's scratch is reused
        const double br = block_sum((double)rsq);
        if (threadIdx.x == 0) partials_rho[blockIdx.x] = br;
    }
}

// one-off setup of the static per-entry geometry
__global__ void k_entry_geo(MeshDev m, float4* cf_geo, uint32_t* nbc, float4* dn, float4* df) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.N) entry_geo_cell(m, cf_geo, nbc, dn, df, i);
}

__global__ void k_reduce_partials(int64_t n, const float* __restrict__ v, double* partials) {
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += (double)v[i];
    const double bs = block_sum(s);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

// The sum of the partials into history[ctl->it_chunk] (the iteration the
// next k_reduce_final records), k_reduce_final's order; nothing once halted.
__global__ void k_reduce_history(int n, const double* __restrict__ partials, const RunCtl* ctl, double* history,
                                 unsigned long long history_cap) {
    if (*(const volatile int*)&ctl->halt) return;   // uniform over the block
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
    const double bs = block_sum(s);
    if (threadIdx.x == 0) {
        const unsigned long long it = ctl->it_chunk;
        if (it < history_cap) history[it] = bs;
    }
}

__global__ void k_reduce_final(int n, const double* __restrict__ partials, double* out, RunCtl* ctl, double* history,
                               unsigned long long history_cap, double tol) {
    if (ctl && *(volatile int*)&ctl->halt) return;   // uniform over the block
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
    const double bs = block_sum(s);
    if (threadIdx.x == 0) {
        out[0] = bs;
        if (ctl) {
            const unsigned long long it = ctl->it_chunk;
            if (history && it < history_cap) history[it] = bs;
            ctl->it_chunk = it + 1;
            if (ctl->it_run == 0) ctl->res0 = bs;
            ctl->it_run += 1;
            if (!(bs == bs) || bs > 1e300) ctl->halt = 2;
            else if (tol > 0.0 && ctl->res0 > 0.0 && bs / ctl->res0 < tol) ctl->halt = 1;
        }
    }
}

__global__ void k_gather_scalar(int64_t n, const float* __restrict__ src, const uint32_t* __restrict__ idx, float* dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
__global__ void k_gather_vector(int64_t n, const float4* __restrict__ src, const uint32_t* __restrict__ idx, float* dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = src[idx[i]];
    dst[3 * i] = v.x; dst[3 * i + 1] = v.y; dst[3 * i + 2] = v.z;
}
__global__ void k_scatter_scalar(int64_t n, const float* __restrict__ src, const uint32_t* __restrict__ idx, float* dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[idx[i]] = src[i];
}
__global__ void k_scatter_vector(int64_t n, const float* __restrict__ src, const uint32_t* __restrict__ idx, float4* dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[idx[i]] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.f);
}

inline unsigned grid(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

int reduce_blocks(int64_t n) {
    int64_t b = (n + kBlock * 8 - 1) / (kBlock * 8);
    if (b < 1) b = 1;
    if (b > 1184) b = 1184;   // 8 x 148 SMs
    return (int)b;
}

void launch_init(int64_t n, float* rho, float4* rhou, float* rhoe, float r, float3 ru, float e, cudaStream_t s) {
    if (n == 0) return;
    k_init<<<grid(n), kBlock, 0, s>>>(n, rho, rhou, rhoe, r, ru, e);
    count_launch();
}

void launch_bc_slip(const DevMesh& m, uint32_t g0, uint32_t g1, float* rho[2], float4* rhou[2], float* rhoe[2],
                    int cur, cudaStream_t s) {
    if (g1 <= g0) return;
    GhostBuf b = {{rho[0], rho[1]}, {rhou[0], rhou[1]}, {rhoe[0], rhoe[1]}, m.halt};
    k_bc_slip<<<grid(g1 - g0), kBlock, 0, s>>>(g0, g1, (uint32_t)m.N, m.cell_geo, m.face_geo, m.ghost, b, cur);
    count_launch();
}

void launch_bc_farfield(const DevMesh& m, uint32_t g0, uint32_t g1, float* rho[2], float4* rhou[2],
                        float* rhoe[2], int cur, float3 mach, float p, float t, cudaStream_t s) {
    if (g1 <= g0) return;
    GhostBuf b = {{rho[0], rho[1]}, {rhou[0], rhou[1]}, {rhoe[0], rhoe[1]}, m.halt};
    k_bc_farfield<<<grid(g1 - g0), kBlock, 0, s>>>(g0, g1, (uint32_t)m.N, m.cell_geo, m.face_geo, m.ghost, b, cur,
                                                   mach, p, t);
    count_launch();
}

void launch_bc_table(const DevMesh& m, const GhostBcTable& t, int cur, cudaStream_t s) {
    if (m.G == 0) return;
    k_bc_table<<<grid(m.G), kBlock, 0, s>>>((uint32_t)m.N, (uint32_t)m.G, m.cell_geo, m.face_geo, m.ghost, t, cur,
                                            m.halt);
    count_launch();
}

MeshDev mesh_dev(const DevMesh& m) {
    return MeshDev{m.cell_geo, m.face_geo, m.nfc, m.nb, m.lsq, m.twin, m.cf_geo, m.nbc, m.dn, m.df,
                   (uint32_t)m.N, (uint32_t)m.S, m.halt};
}

void launch_entry_geo(const DevMesh& m, cudaStream_t s) {
    if (m.N == 0) return;
    k_entry_geo<<<grid(m.N), kBlock, 0, s>>>(mesh_dev(m), m.cf_geo, m.nbc, m.dn, m.df);
    count_launch();
}

void launch_grad_lim(const DevMesh& m, EulerState q, EulerGrad g, bool transposed, cudaStream_t s,
                     const GhostBcTable* ghosts) {
    if (m.N == 0) return;
#if GB_GRAD_STAGED
    const MeshDev md = mesh_dev(m);
    if (ghosts) {
        if (transposed) launch_staged<true>(m, md, q, g, GhostBcs{*ghosts}, s);
        else launch_staged<false>(m, md, q, g, GhostBcs{*ghosts}, s);
    } else {
        if (transposed) launch_staged<true>(m, md, q, g, NoGhostBcs{}, s);
        else launch_staged<false>(m, md, q, g, NoGhostBcs{}, s);
    }
#else
    if (transposed) k_grad_lim<true><<<grid(m.N), kBlock, 0, s>>>(mesh_dev(m), q, g);
    else k_grad_lim<false><<<grid(m.N), kBlock, 0, s>>>(mesh_dev(m), q, g);
#endif
    count_launch();
}

void launch_flux(const DevMesh& m, EulerState q, FaceRecs r, float* rho_n, float4* rhou_n, float* rhoe_n,
                 float* err, double* partials, float cfl, cudaStream_t s, double* partials_rho) {
    if (m.N == 0) return;
    if (partials_rho)
        k_flux<true><<<grid(m.N), kBlock, 0, s>>>(mesh_dev(m), q, r, rho_n, rhou_n, rhoe_n, err, partials, cfl,
                                                  partials_rho);
    else
        k_flux<false><<<grid(m.N), kBlock, 0, s>>>(mesh_dev(m), q, r, rho_n, rhou_n, rhoe_n, err, partials, cfl,
                                                   nullptr);
    count_launch();
}

void launch_reduce_history(int n_partials, const double* partials, const RunCtl* ctl, double* history,
                           unsigned long long history_cap, cudaStream_t s) {
    k_reduce_history<<<1, kBlock, 0, s>>>(n_partials, partials, ctl, history, history_cap);
    count_launch();
}

void launch_reduce_partials(int64_t n, const float* v, double* partials, cudaStream_t s) {
    k_reduce_partials<<<reduce_blocks(n), kBlock, 0, s>>>(n, v, partials);
    count_launch();
}

void launch_reduce_partials_blocks(int64_t n, const float* v, double* partials, int blocks, cudaStream_t s) {
    k_reduce_partials<<<blocks, kBlock, 0, s>>>(n, v, partials);
    count_launch();
}

void launch_reduce_final(int n_partials, const double* partials, double* out, cudaStream_t s, RunCtl* ctl,
                         double* history, unsigned long long history_cap, double tolerance) {
    k_reduce_final<<<1, kBlock, 0, s>>>(n_partials, partials, out, ctl, history, history_cap, tolerance);
    count_launch();
}

void launch_gather_scalar(int64_t n, const float* src, const uint32_t* idx, float* dst, cudaStream_t s) {
    if (n == 0) return;
    k_gather_scalar<<<grid(n), kBlock, 0, s>>>(n, src, idx, dst);
    count_launch();
}
void launch_gather_vector(int64_t n, const float4* src, const uint32_t* idx, float* dst3, cudaStream_t s) {
    if (n == 0) return;
    k_gather_vector<<<grid(n), kBlock, 0, s>>>(n, src, idx, dst3);
    count_launch();
}
void launch_scatter_scalar(int64_t n, const float* src, const uint32_t* idx, float* dst, cudaStream_t s) {
    if (n == 0) return;
    k_scatter_scalar<<<grid(n), kBlock, 0, s>>>(n, src, idx, dst);
    count_launch();
}
void launch_scatter_vector(int64_t n, const float* src3, const uint32_t* idx, float4* dst, cudaStream_t s) {
    if (n == 0) return;
    k_scatter_vector<<<grid(n), kBlock, 0, s>>>(n, src3, idx, dst);
    count_launch();
}

}  // namespace gb
