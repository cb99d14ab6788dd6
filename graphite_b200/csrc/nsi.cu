// Steady incompressible Navier-Stokes (config 2) by artificial compressibility
// (Chorin): the pressure p (kinematic, p / rho) and velocity u march in
// pseudo-time to the steady state of
//     dp/dt + beta^2 div u = 0,
//     du/dt + div(u u + p I) - nu lap u = 0,
// with the Euler path's machinery: least-squares gradients and the
// reference's limiter on the same per-entry geometry, second-order
// reconstruction of (p, u) at each face, a Rusanov flux with the
// artificial-compressibility wave speed |u.n| + sqrt((u.n)^2 + beta^2), a
// viscous flux from the face gradient of u, and a local pseudo-time step
// cfl / sum((lambda + 2 nu / |d|) A / V).
//
// The reference has no incompressible solver: src/models/nsi.cu is a
// skeleton that calls FvmNSIInit / FvmNSISlipBc / FvmNSIInletOutletBc /
// FvmNSIStepPrepare / FvmNSIStep, which it never defines.  This file gives
// those calls their meaning.  The face gradient of the viscous term is the
// average of the two cells' gradients, as the reference's generic operator
// fvmLaplacianC takes it (include/fvmops.cuh:96-102), plus (mode 1, the
// default) the compact correction ((u_j - u_i) - G.d) d / |d|^2 along the
// centroid offset d, which couples neighbouring cells directly and removes
// the odd-even decoupling of the plain average.
#include "euler_ops.cuh"

namespace gb {
namespace {

constexpr int kNsiBlocks = 4;

__global__ void k_nsi_init(int64_t n, float* p, float4* u, float p0, float3 u0) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p[i] = p0;
    u[i] = make_float4(u0.x, u0.y, u0.z, 0.f);
}

// Ghosts [g0, g1) of one region; type 0 slip (normal velocity mirrored),
// 1 inlet / outlet (inflow where u_inf . n < 0: free-stream velocity with the
// interior pressure; outflow: interior velocity with the free-stream
// pressure), 2 no-slip wall (velocity mirrored through zero).  The pressure
// is extrapolated from the interior except at outflow.  Both value buffers
// are written.
// The ghost state of one boundary face from its interior state (pi, ui) and
// outward normal n.
__device__ __forceinline__ void nsi_ghost_state(int type, float3 n, float pi, float3 ui, float3 vinf, float pinf,
                                                float& pg, float3& ug) {
    // explicitly rounded (xdot): the ghost kernel and the gradient kernel both
    // form these states and must agree bitwise
    if (type == 0) {
        const float s = __fmul_rn(2.f, xdot(n, ui));
        ug = make_float3(__fmaf_rn(-n.x, s, ui.x), __fmaf_rn(-n.y, s, ui.y), __fmaf_rn(-n.z, s, ui.z));
        pg = pi;
    } else if (type == 2) {
        ug = make_float3(-ui.x, -ui.y, -ui.z);
        pg = pi;
    } else if (xdot(vinf, n) < 0.f) {
        ug = vinf;
        pg = pi;
    } else {
        ug = ui;
        pg = pinf;
    }
}

__global__ void k_nsi_bc(uint32_t g0, uint32_t g1, uint32_t N, const float4* __restrict__ cell_geo,
                         const float4* __restrict__ face_geo, const uint2* __restrict__ ghost, float* pa, float* pb,
                         float4* ua, float4* ub, int cur, int type, float3 vinf, float pinf, const int* halt) {
    const uint32_t t = g0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g1 || halted(halt)) return;
    const uint2 gl = ghost[t - N];
    const uint32_t c1 = gl.x;
    const float3 n = outer_normal(f3(face_geo[2 * gl.y]), f3(face_geo[2 * gl.y + 1]) - f3(cell_geo[c1]));
    const float* p = cur ? pb : pa;
    const float4* u = cur ? ub : ua;
    float pg;
    float3 ug;
    nsi_ghost_state(type, n, p[c1], f3(u[c1]), vinf, pinf, pg, ug);
    const float4 u4 = make_float4(ug.x, ug.y, ug.z, 0.f);
    pa[t] = pg;
    pb[t] = pg;
    ua[t] = u4;
    ub[t] = u4;
}

// Least-squares gradients of p, u_x, u_y, u_z (src/fvmops.cu:51-111 on the
// per-entry geometry) and, when `limited`, the reference's limiters
// (src/fvmops.cu:175-266); otherwise the limiter is 1 (unlimited second order).
// With GHOSTS the boundary conditions of gh are applied here: the thread of a
// ghost's interior cell computes the ghost's state (nsi_ghost_state with the
// entry's outward normal, bitwise the normal k_nsi_bc computes), uses it and
// stores it into both value buffers, for the flux pass and the caller.
template <bool GHOSTS>
__global__ void __launch_bounds__(kBlock, kNsiBlocks)
    k_nsi_grad(MeshDev m, const float* __restrict__ p, const float4* __restrict__ u, float4* gp, float4* gu,
               int limited, NsiGhostTable gh) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N || halted(m.halt)) return;
    float v[4];
    {
        const float4 ui = __ldg(&u[i]);
        v[0] = __ldg(&p[i]); v[1] = ui.x; v[2] = ui.y; v[3] = ui.z;
    }
    float3 gs[4];
    float vmin[4], vmax[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) { gs[c] = make_float3(0.f, 0.f, 0.f); vmin[c] = v[c]; vmax[c] = v[c]; }
    const uint32_t nf = __ldg(&m.nfc[i]);
    const uint32_t kend = i + nf * m.N;
    for (uint32_t k = i; k < kend; k += m.N) {
        const uint32_t j = __ldg(&m.nbc[k]);
        const float4 dw = __ldg(&m.dn[k]);
        const float3 d = f3(dw);
        float vj[4];
        bool computed = false;
        if (GHOSTS && j >= m.N) {
            int r = 0;
            while (r < gh.n - 1 && j >= gh.start[r + 1]) ++r;
            if (gh.type[r] >= 0) {
                float pg;
                float3 ug;
                nsi_ghost_state(gh.type[r], f3(__ldg(&m.cf_geo[k])), v[0], make_float3(v[1], v[2], v[3]),
                                gh.vinf[r], gh.pinf[r], pg, ug);
                const float4 u4 = make_float4(ug.x, ug.y, ug.z, 0.f);
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    gh.p[b][j] = pg;
                    gh.u[b][j] = u4;
                }
                vj[0] = pg; vj[1] = ug.x; vj[2] = ug.y; vj[3] = ug.z;
                computed = true;
            }
        }
        if (!computed) {
            const float4 uj = __ldg(&u[j]);
            vj[0] = __ldg(&p[j]); vj[1] = uj.x; vj[2] = uj.y; vj[3] = uj.z;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            gs[c] = gs[c] + (d * (vj[c] - v[c])) * dw.w;
            vmin[c] = fminf(vmin[c], vj[c]);
            vmax[c] = fmaxf(vmax[c], vj[c]);
        }
    }
    const float4 l0 = __ldg(&m.lsq[2 * i]), l1 = __ldg(&m.lsq[2 * i + 1]);
#pragma unroll
    for (int c = 0; c < 4; ++c) gs[c] = sym_mul(l0, l1, gs[c]);
    float lim[4] = {1.f, 1.f, 1.f, 1.f};
    if (limited) {
        lim[0] = lim[1] = lim[2] = lim[3] = 2.f;
        for (uint32_t k = i; k < kend; k += m.N) {
            const float4 dk = __ldg(&m.df[k]);
#pragma unroll
            for (int c = 0; c < 4; ++c) lim[c] = fminf(lim[c], limiter(v[c], gs[c], vmin[c], vmax[c], f3(dk), dk.w));
        }
    }
    gp[i] = make_float4(gs[0].x, gs[0].y, gs[0].z, lim[0]);
#pragma unroll
    for (int a = 0; a < 3; ++a) gu[3 * i + a] = make_float4(gs[a + 1].x, gs[a + 1].y, gs[a + 1].z, lim[a + 1]);
}

struct NsiParams {
    float cfl, nu, beta2;
    int corrected;            // 1: compact correction of the face gradient
};

__global__ void __launch_bounds__(kBlock, kNsiBlocks)
    k_nsi_flux(MeshDev m, const float* __restrict__ p, const float4* __restrict__ u, const float4* __restrict__ gp,
               const float4* __restrict__ gu, float* __restrict__ p_n, float4* __restrict__ u_n,
               float* __restrict__ err, double* __restrict__ partials, NsiParams P) {
    if (halted(m.halt)) return;              // uniform over the grid
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double res = 0.0;
    if (i < m.N) {
        const float vol = __ldg(&m.cell_geo[i]).w;
        const float pi = __ldg(&p[i]);
        const float3 ui = f3(__ldg(&u[i]));
        const float4 gpi = __ldg(&gp[i]);
        const float4 gui[3] = {__ldg(&gu[3 * i]), __ldg(&gu[3 * i + 1]), __ldg(&gu[3 * i + 2])};
        float rp = 0.f, sr = 0.f;
        float3 ru = make_float3(0.f, 0.f, 0.f);
        const uint32_t nf = __ldg(&m.nfc[i]);
        for (uint32_t k = i; k < i + nf * m.N; k += m.N) {
            const uint32_t t = __ldg(&m.twin[k]);
            const uint32_t j = __ldg(&m.nbc[k]);
            const float4 gk = __ldg(&m.cf_geo[k]);
            const float3 n = f3(gk);
            const float ds = gk.w;
            const float3 d0 = f3(__ldg(&m.df[k]));
            const float4 dw = __ldg(&m.dn[k]);      // centroid offset, 1 / |d|^2
            const float pj = __ldg(&p[j]);
            const float3 uj = f3(__ldg(&u[j]));
            float3 d1;
            float4 gpj, guj[3];
            if (t < m.S) {
                d1 = f3(__ldg(&m.df[t]));
                gpj = __ldg(&gp[j]);
                guj[0] = __ldg(&gu[3 * j]);
                guj[1] = __ldg(&gu[3 * j + 1]);
                guj[2] = __ldg(&gu[3 * j + 2]);
            } else {
                // a ghost carries its interior cell's gradient and limiter
                d1 = f3(__ldg(&m.face_geo[2 * __ldg(&m.nb[k]).x + 1])) - f3(__ldg(&m.cell_geo[j]));
                gpj = gpi;
                guj[0] = gui[0]; guj[1] = gui[1]; guj[2] = gui[2];
            }
            const float pL = pi + dot(f3(gpi), d0) * gpi.w;
            const float pR = pj + dot(f3(gpj), d1) * gpj.w;
            const float3 uL = make_float3(ui.x + dot(f3(gui[0]), d0) * gui[0].w, ui.y + dot(f3(gui[1]), d0) * gui[1].w,
                                          ui.z + dot(f3(gui[2]), d0) * gui[2].w);
            const float3 uR = make_float3(uj.x + dot(f3(guj[0]), d1) * guj[0].w, uj.y + dot(f3(guj[1]), d1) * guj[1].w,
                                          uj.z + dot(f3(guj[2]), d1) * guj[2].w);
            const float unL = dot(uL, n), unR = dot(uR, n);
            const float lam = fmaxf(fabsf(unL) + sqrtf(unL * unL + P.beta2), fabsf(unR) + sqrtf(unR * unR + P.beta2));
            const float h = 0.5f * ds;
            rp += P.beta2 * (unL + unR) * h - lam * h * (pR - pL);
            ru = ru + (uL * unL + n * pL + uR * unR + n * pR) * h - (uR - uL) * (lam * h);
            // viscous flux: face gradient of u dotted with n
            const float3 d = f3(dw);
            float3 vis;
            {
                float g[3];
                const float du[3] = {uj.x - ui.x, uj.y - ui.y, uj.z - ui.z};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float3 ga = (f3(gui[a]) + f3(guj[a])) * 0.5f;
                    float gn = dot(ga, n);
                    if (P.corrected) gn += (du[a] - dot(ga, d)) * dw.w * dot(d, n);
                    g[a] = gn;
                }
                vis = make_float3(g[0], g[1], g[2]);
            }
            ru = ru - vis * (P.nu * ds);
            sr += (lam + 2.f * P.nu * sqrtf(dw.w)) * ds;
        }
        const float dt = P.cfl / sr;
        p_n[i] = pi - rp * dt;
        u_n[i] = make_float4(ui.x - ru.x * dt, ui.y - ru.y * dt, ui.z - ru.z * dt, 0.f);
        const float e = (rp * rp + dot(ru, ru)) * vol;
        if (err) err[i] = e;
        res = (double)e;
    }
    const double bs = block_sum(res);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

// Force on the wall faces [g0, g1): sum of A (p n - nu G_f . n), n out of the
// fluid, G_f the face gradient of u as the flux takes it, float64 partials.
__global__ void k_nsi_force_partials(uint32_t g0, uint32_t g1, uint32_t N, const float4* __restrict__ cell_geo,
                                     const float4* __restrict__ face_geo, const uint2* __restrict__ ghost,
                                     const float* __restrict__ p, const float4* __restrict__ u,
                                     const float4* __restrict__ gu, float nu, int corrected, double* partials) {
    __shared__ double red[3][kBlock];
    const uint32_t t = g0 + blockIdx.x * kBlock + threadIdx.x;
    double f[3] = {0.0, 0.0, 0.0};
    if (t < g1) {
        const uint2 gl = ghost[t - N];
        const uint32_t i = gl.x;
        const float4 na = face_geo[2 * gl.y];
        const float3 ci = f3(cell_geo[i]);
        const float3 n = outer_normal(f3(na), f3(face_geo[2 * gl.y + 1]) - ci);
        const float3 d = f3(cell_geo[t]) - ci;
        const float w2 = 1.f / dot(d, d);
        const float3 ui = f3(u[i]), ug = f3(u[t]);
        const float du[3] = {ug.x - ui.x, ug.y - ui.y, ug.z - ui.z};
        const double pf = 0.5 * ((double)p[i] + (double)p[t]);
        for (int a = 0; a < 3; ++a) {
            const float3 ga = f3(gu[3 * i + a]);     // the ghost carries the interior gradient
            float gn = dot(ga, n);
            if (corrected) gn += (du[a] - dot(ga, d)) * w2 * dot(d, n);
            const double nc = a == 0 ? n.x : (a == 1 ? n.y : n.z);
            f[a] = (double)na.w * (pf * nc - (double)nu * gn);
        }
    }
    for (int a = 0; a < 3; ++a) red[a][threadIdx.x] = f[a];
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int a = 0; a < 3; ++a) red[a][threadIdx.x] += red[a][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 3) partials[3 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_nsi_force_final(const double* __restrict__ partials, int n, double scale, double* out) {
    if (threadIdx.x >= 3) return;
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += partials[3 * b + threadIdx.x];
    out[threadIdx.x] = s * scale;
}

inline unsigned grid_of(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

MeshDev mesh_dev(const DevMesh& m);

void launch_nsi_init(int64_t n, float* p, float4* u, float p0, float3 u0, cudaStream_t s) {
    if (n == 0) return;
    k_nsi_init<<<grid_of(n), kBlock, 0, s>>>(n, p, u, p0, u0);
    count_launch();
}

void launch_nsi_bc(const DevMesh& m, uint32_t g0, uint32_t g1, int type, float* p[2], float4* u[2], int cur,
                   float3 vinf, float pinf, cudaStream_t s) {
    if (g1 <= g0) return;
    k_nsi_bc<<<grid_of(g1 - g0), kBlock, 0, s>>>(g0, g1, (uint32_t)m.N, m.cell_geo, m.face_geo, m.ghost, p[0], p[1],
                                                 u[0], u[1], cur, type, vinf, pinf, m.halt);
    count_launch();
}

void launch_nsi_grad(const DevMesh& m, const float* p, const float4* u, float4* gp, float4* gu, int limited,
                     cudaStream_t s, const NsiGhostTable* ghosts) {
    if (m.N == 0) return;
    if (ghosts) k_nsi_grad<true><<<grid_of(m.N), kBlock, 0, s>>>(mesh_dev(m), p, u, gp, gu, limited, *ghosts);
    else k_nsi_grad<false><<<grid_of(m.N), kBlock, 0, s>>>(mesh_dev(m), p, u, gp, gu, limited, NsiGhostTable{});
    count_launch();
}

void launch_nsi_flux(const DevMesh& m, const float* p, const float4* u, const float4* gp, const float4* gu, float* p_n,
                     float4* u_n, float* err, double* partials, float cfl, float nu, float beta2, int corrected,
                     cudaStream_t s) {
    if (m.N == 0) return;
    k_nsi_flux<<<grid_of(m.N), kBlock, 0, s>>>(mesh_dev(m), p, u, gp, gu, p_n, u_n, err, partials,
                                               NsiParams{cfl, nu, beta2, corrected});
    count_launch();
}

int launch_nsi_force(const DevMesh& m, uint32_t g0, uint32_t g1, const float* p, const float4* u, const float4* gu,
                     float nu, int corrected, double density, double* partials, double* out, cudaStream_t s) {
    const int blocks = (int)grid_of(g1 - g0);
    if (blocks == 0) return 0;
    k_nsi_force_partials<<<blocks, kBlock, 0, s>>>(g0, g1, (uint32_t)m.N, m.cell_geo, m.face_geo, m.ghost, p, u, gu,
                                                   nu, corrected, partials);
    k_nsi_force_final<<<1, 32, 0, s>>>(partials, blocks, density, out);
    count_launch(2);
    return blocks;
}

}  // namespace gb
