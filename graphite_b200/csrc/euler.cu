// The Euler iteration on sm_100a: boundary ghosts, fused least-squares
// gradient + limiter of all five conserved variables, and the fused
// reconstruction / central flux / scalar dissipation / local-time-step
// update / squared-residual kernel with a deterministic float64 block
// reduction of the residual.
//
// Both hot kernels are cell-gathers over the renumbered (reverse
// Cuthill-McKee) mesh: one thread per interior cell walks its faces in the
// reference's element-local order, so every sum is taken in the reference's
// order and no atomics are used -- runs are bitwise reproducible.  They are
// HBM-bandwidth bound: per cell and iteration they stream the cell's own
// record once and gather neighbour records that the renumbering keeps
// resident in L2.
#include "gb_device.cuh"

namespace gb {
namespace {

// Resident blocks per SM the two hot kernels are compiled for (register
// budget 65536 / (kBlock * blocks)).
#ifndef GB_FLUX_BLOCKS
#define GB_FLUX_BLOCKS 3
#endif
#ifndef GB_GRAD_BLOCKS
#define GB_GRAD_BLOCKS 4
#endif
constexpr int kFluxBlocksPerSM = GB_FLUX_BLOCKS;
constexpr int kGradBlocksPerSM = GB_GRAD_BLOCKS;

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float norm(float3 a) { return sqrtf(dot(a, a)); }
// include/datatypes.cuh:144-150: n * sign(n . d) with sign(0) = +1
__device__ __forceinline__ float3 outer_normal(float3 n, float3 d) {
    return dot(n, d) >= 0.f ? n : make_float3(-n.x, -n.y, -n.z);
}
// include/datatypes.cuh:375-377
__device__ __forceinline__ float lsqrt(float x) { return sqrtf(fmaxf(1e-12f, fminf(1e30f, x))); }

// A^-1 g with the symmetric inverse (a00 a01 a02 a11) (a12 a22).
__device__ __forceinline__ float3 sym_mul(float4 l0, float4 l1, float3 g) {
    return make_float3(l0.x * g.x + l0.y * g.y + l0.z * g.z,
                       l0.y * g.x + l0.w * g.y + l1.x * g.z,
                       l0.z * g.x + l1.x * g.y + l1.y * g.z);
}

// limiter(), src/fvmops.cu:118-169: smoothed switch on (max-min)^2 against
// (K |d|)^3 with K = 1, Michalak function y - y^2/4 (y < 2), scaled by 0.8.
// k3 = |d|^3 is shared by the five variables of a face.
__device__ __forceinline__ float limiter(float u, float3 g, float umin, float umax, float3 d, float k3) {
    const float delta = dot(g, d);
    const float du = umax - u, dd = umin - u;
    const float dmm2 = (du - dd) * (du - dd);
    float sig;
    if (dmm2 <= k3) {
        sig = 1.f;
    } else if (dmm2 <= 2.f * k3) {
        const float y = dmm2 / k3 - 1.f;
        sig = 2.f * y * y * y - 3.f * y * y + 1.f;
    } else {
        sig = 0.f;
    }
    float lim = 1.f;
    if (delta > 1e-6f) {
        const float y = du / delta;
        lim = y < 2.f ? y - 0.25f * y * y : 1.f;
    } else if (delta < -1e-6f) {
        const float y = dd / delta;
        lim = y < 2.f ? y - 0.25f * y * y : 1.f;
    }
    lim *= 0.8f;
    return sig + (1.f - sig) * lim;
}

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
};

// euler_slip_bc, src/models/euler.cu:412-442: ghost = interior with the
// normal momentum mirrored.  Written to both value buffers so that the ghost
// values are current whichever buffer the next sweep reads.
__global__ void k_bc_slip(uint32_t g0, uint32_t g1, uint32_t N, const float4* __restrict__ cell_geo,
                          const float4* __restrict__ face_geo, const uint2* __restrict__ ghost, GhostBuf b, int cur) {
    const uint32_t t = g0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g1) return;
    const uint2 gl = ghost[t - N];
    const uint32_t c1 = gl.x;
    const float3 n = outer_normal(f3(face_geo[2 * gl.y]), f3(face_geo[2 * gl.y + 1]) - f3(cell_geo[c1]));
    const float r = b.rho[cur][c1];
    const float3 u = f3(b.rhou[cur][c1]);
    const float e = b.rhoe[cur][c1];
    const float3 ug = u - n * (2.f * dot(n, u));
    const float4 ug4 = make_float4(ug.x, ug.y, ug.z, 0.f);
    for (int k = 0; k < 2; ++k) {
        b.rho[k][t] = r;
        b.rhou[k][t] = ug4;
        b.rhoe[k][t] = e;
    }
}

// euler_inletoutlet_bc, src/models/euler.cu:446-520 (gamma = 1.4, R = 1):
// inflow (u.n < 0) supersonic -> free stream, subsonic -> interior pressure
// with free-stream temperature and Mach; outflow supersonic -> interior,
// subsonic -> free-stream pressure with interior temperature and velocity.
__global__ void k_bc_farfield(uint32_t g0, uint32_t g1, uint32_t N, const float4* __restrict__ cell_geo,
                              const float4* __restrict__ face_geo, const uint2* __restrict__ ghost, GhostBuf b,
                              int cur, float3 imach, float ip, float it) {
    const uint32_t t = g0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g1) return;
    const uint2 gl = ghost[t - N];
    const uint32_t c1 = gl.x;
    const float3 n = outer_normal(f3(face_geo[2 * gl.y]), f3(face_geo[2 * gl.y + 1]) - f3(cell_geo[c1]));
    const float r1 = b.rho[cur][c1];
    const float3 ru1 = f3(b.rhou[cur][c1]);
    const float e1 = b.rhoe[cur][c1];
    const float3 u = ru1 * (1.f / r1);
    const float p = 0.4f * (e1 - 0.5f / r1 * dot(ru1, ru1));
    const float tt = p / r1;
    const float mach = sqrtf(dot(u, u) / (1.4f * p / r1));
    const float idens = ip / it;
    float r, e;
    float3 ru;
    if (dot(u, n) < 0.f) {
        if (mach > 1.f) {
            const float ic = sqrtf(1.4f * ip / idens);
            const float3 iv = imach * ic;
            r = idens;
            ru = imach * ic * idens;
            e = ip / 0.4f + 0.5f * idens * dot(iv, iv);
        } else {
            r = p / it;
            const float ic = sqrtf(1.4f * p / r);
            const float3 v = imach * ic;
            ru = v * r;
            e = p / 0.4f + 0.5f * r * dot(v, v);
        }
    } else {
        if (mach > 1.f) {
            r = r1; ru = ru1; e = e1;
        } else {
            r = ip / tt;
            ru = u * r;
            e = ip / 0.4f + 0.5f * r * dot(u, u);
        }
    }
    const float4 ru4 = make_float4(ru.x, ru.y, ru.z, 0.f);
    for (int k = 0; k < 2; ++k) {
        b.rho[k][t] = r;
        b.rhou[k][t] = ru4;
        b.rhoe[k][t] = e;
    }
}

// Fused FvmEulerStepPrepare (src/models/euler.cu:597-647): least-squares
// gradients (src/fvmops.cu:51-111) and limiters (src/fvmops.cu:175-266) of
// rho, rhou (3 components) and rhoE in one pass over each cell's faces.
__global__ void __launch_bounds__(kBlock, kGradBlocksPerSM) k_grad_lim(uint32_t N, const float4* __restrict__ cell_geo,
                                                    const float4* __restrict__ face_geo,
                                                    const uint32_t* __restrict__ start, const uint2* __restrict__ nb,
                                                    const float4* __restrict__ lsq, EulerState q, EulerGrad g) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float3 ci = f3(__ldg(&cell_geo[i]));
    float v[5];
    {
        const float4 u = __ldg(&q.rhou[i]);
        v[0] = __ldg(&q.rho[i]); v[1] = u.x; v[2] = u.y; v[3] = u.z; v[4] = __ldg(&q.rhoe[i]);
    }
    float3 gs[5];
    float vmin[5], vmax[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) { gs[c] = make_float3(0.f, 0.f, 0.f); vmin[c] = v[c]; vmax[c] = v[c]; }
    const uint32_t s0 = __ldg(&start[i]), s1 = __ldg(&start[i + 1]);
    for (uint32_t k = s0; k < s1; ++k) {
        const uint32_t j = __ldg(&nb[k]).y;
        const float3 d = f3(__ldg(&cell_geo[j])) - ci;
        const float w2 = 1.f / dot(d, d);
        const float4 uj = __ldg(&q.rhou[j]);
        const float vj[5] = {__ldg(&q.rho[j]), uj.x, uj.y, uj.z, __ldg(&q.rhoe[j])};
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            gs[c] = gs[c] + (d * (vj[c] - v[c])) * w2;
            vmin[c] = fminf(vmin[c], vj[c]);
            vmax[c] = fmaxf(vmax[c], vj[c]);
        }
    }
    const float4 l0 = __ldg(&lsq[2 * i]), l1 = __ldg(&lsq[2 * i + 1]);
#pragma unroll
    for (int c = 0; c < 5; ++c) gs[c] = sym_mul(l0, l1, gs[c]);
    float lim[5] = {2.f, 2.f, 2.f, 2.f, 2.f};
    for (uint32_t k = s0; k < s1; ++k) {
        const uint32_t f = __ldg(&nb[k]).x;
        const float3 d = f3(__ldg(&face_geo[2 * f + 1])) - ci;
        const float dn = norm(d);
        const float k3 = dn * dn * dn;
#pragma unroll
        for (int c = 0; c < 5; ++c) lim[c] = fminf(lim[c], limiter(v[c], gs[c], vmin[c], vmax[c], d, k3));
    }
    g.rho[i] = make_float4(gs[0].x, gs[0].y, gs[0].z, lim[0]);
    g.rhou[3 * i] = make_float4(gs[1].x, gs[1].y, gs[1].z, lim[1]);
    g.rhou[3 * i + 1] = make_float4(gs[2].x, gs[2].y, gs[2].z, lim[2]);
    g.rhou[3 * i + 2] = make_float4(gs[3].x, gs[3].y, gs[3].z, lim[3]);
    g.rhoe[i] = make_float4(gs[4].x, gs[4].y, gs[4].z, lim[4]);
}

// Deterministic block sum of one double per thread (fixed shuffle tree).
__device__ __forceinline__ double block_sum(double x) {
    __shared__ double warp_sums[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_sums[w] = x;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < kBlock / 32 ? warp_sums[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    return t;   // valid in thread 0
}

// Reconstructed state on one side of a face: q + (grad q . d) * limiter, with
// the momentum delta either as the reference computes it (the transposed
// gradient, src/models/euler.cu:252-253 with include/datatypes.cuh:296-302)
// or as the consistent gradient.
template <bool TRANSPOSED>
__device__ __forceinline__ void reconstruct(float r, float4 u, float e, float4 gr, const float4 gu[3], float4 ge,
                                            float3 d, float& rr, float3& ru, float& re) {
    rr = r + dot(f3(gr), d) * gr.w;
    re = e + dot(f3(ge), d) * ge.w;
    float3 du;
    if (TRANSPOSED) {
        du = make_float3(gu[0].x * d.x + gu[1].x * d.y + gu[2].x * d.z,
                         gu[0].y * d.x + gu[1].y * d.y + gu[2].y * d.z,
                         gu[0].z * d.x + gu[1].z * d.y + gu[2].z * d.z);
    } else {
        du = make_float3(dot(f3(gu[0]), d), dot(f3(gu[1]), d), dot(f3(gu[2]), d));
    }
    ru = make_float3(u.x + du.x * gu[0].w, u.y + du.y * gu[1].w, u.z + du.z * gu[2].w);
}

// Fused fvmEulerSteadyOp + euler_steady_step (src/models/euler.cu:236-381):
// per face, reconstruct both sides, central flux 0.5 (F0 + F1) . n A / V
// minus scalar dissipation 0.5 eig (q1 - q0) A / V with
// eig = max(|u| + c) over both sides, accumulate eig A / V; then
// dt = cfl / sum, q_new = q - F dt (into the other buffer), and the squared
// residual (F_rho^2 + |F_rhou|^2 + F_rhoE^2) V, summed per block in float64.
template <bool TRANSPOSED>
__global__ void __launch_bounds__(kBlock, kFluxBlocksPerSM) k_flux(uint32_t N, const float4* __restrict__ cell_geo,
                                                const float4* __restrict__ face_geo,
                                                const uint32_t* __restrict__ start, const uint2* __restrict__ nb,
                                                EulerState q, const float4* __restrict__ g_rho,
                                                const float4* __restrict__ g_rhou, const float4* __restrict__ g_rhoe,
                                                float* __restrict__ rho_n, float4* __restrict__ rhou_n,
                                                float* __restrict__ rhoe_n, float* __restrict__ err,
                                                double* __restrict__ partials, float cfl) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double res = 0.0;
    if (i < N) {
        const float4 c0 = __ldg(&cell_geo[i]);
        const float3 ci = f3(c0);
        const float inv_v = 1.f / c0.w;
        const float r0 = __ldg(&q.rho[i]);
        const float4 u0 = __ldg(&q.rhou[i]);
        const float e0 = __ldg(&q.rhoe[i]);
        const float4 gr0 = __ldg(&g_rho[i]), ge0 = __ldg(&g_rhoe[i]);
        const float4 gu0[3] = {__ldg(&g_rhou[3 * i]), __ldg(&g_rhou[3 * i + 1]), __ldg(&g_rhou[3 * i + 2])};
        float fr = 0.f, fe = 0.f, dts = 0.f;
        float3 fu = make_float3(0.f, 0.f, 0.f);
        const uint32_t s0 = __ldg(&start[i]), s1 = __ldg(&start[i + 1]);
        for (uint32_t k = s0; k < s1; ++k) {
            const uint2 fj = __ldg(&nb[k]);
            const uint32_t f = fj.x, j = fj.y;
            const float4 na = __ldg(&face_geo[2 * f]);
            const float3 fc = f3(__ldg(&face_geo[2 * f + 1]));
            const float3 d0 = fc - ci;
            const float3 d1 = fc - f3(__ldg(&cell_geo[j]));
            const float3 n = outer_normal(f3(na), d0);
            const float ds = na.w * inv_v;
            const float r1 = __ldg(&q.rho[j]);
            const float4 u1 = __ldg(&q.rhou[j]);
            const float e1 = __ldg(&q.rhoe[j]);
            float4 gr1, ge1, gu1[3];
            if (j < N) {
                gr1 = __ldg(&g_rho[j]);
                ge1 = __ldg(&g_rhoe[j]);
                gu1[0] = __ldg(&g_rhou[3 * j]);
                gu1[1] = __ldg(&g_rhou[3 * j + 1]);
                gu1[2] = __ldg(&g_rhou[3 * j + 2]);
            } else {
                // a ghost carries its interior cell's gradient and limiter
                // (fvmScalGradLimBc / fvmVecGradLimBc, src/fvmops.cu:272-304)
                gr1 = gr0; ge1 = ge0; gu1[0] = gu0[0]; gu1[1] = gu0[1]; gu1[2] = gu0[2];
            }
            float ra, rb, ea, eb;
            float3 ua, ub;
            reconstruct<TRANSPOSED>(r0, u0, e0, gr0, gu0, ge0, d0, ra, ua, ea);
            reconstruct<TRANSPOSED>(r1, u1, e1, gr1, gu1, ge1, d1, rb, ub, eb);
            // one reciprocal of the density per side, reused by every quotient
            const float ia = 1.f / ra, ib = 1.f / rb;
            const float qa = dot(ua, ua), qb = dot(ub, ub);
            const float pa = 0.4f * (ea - 0.5f * ia * qa);
            const float pb = 0.4f * (eb - 0.5f * ib * qb);
            const float va = dot(ua, n) * ia;
            const float vb = dot(ub, n) * ib;
            const float h = ds * 0.5f;
            fr += (va * ra + vb * rb) * h;
            fu = fu + ((ua * va + n * pa) + (ub * vb + n * pb)) * h;
            fe += (va * (ea + pa) + vb * (eb + pb)) * h;
            const float eig = fmaxf(sqrtf(qa) * ia + lsqrt(1.4f * pa * ia),
                                    sqrtf(qb) * ib + lsqrt(1.4f * pb * ib));
            const float eh = eig * h;
            fr -= eh * (rb - ra);
            fu = fu - (ub - ua) * eh;
            fe -= eh * (eb - ea);
            dts += eig * ds;
        }
        const float dt = cfl / dts;
        rho_n[i] = r0 - fr * dt;
        rhou_n[i] = make_float4(u0.x - fu.x * dt, u0.y - fu.y * dt, u0.z - fu.z * dt, 0.f);
        rhoe_n[i] = e0 - fe * dt;
        const float e = (fr * fr + dot(fu, fu) + fe * fe) * c0.w;
        err[i] = e;
        res = (double)e;
    }
    const double bs = block_sum(res);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

__global__ void k_reduce_partials(int64_t n, const float* __restrict__ v, double* partials) {
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += (double)v[i];
    const double bs = block_sum(s);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

__global__ void k_reduce_final(int n, const double* __restrict__ partials, double* out, double* history,
                               unsigned long long* counter) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
    const double bs = block_sum(s);
    if (threadIdx.x == 0) {
        out[0] = bs;
        if (history) {
            const unsigned long long it = *counter;
            history[it] = bs;
            *counter = it + 1;
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
    GhostBuf b = {{rho[0], rho[1]}, {rhou[0], rhou[1]}, {rhoe[0], rhoe[1]}};
    k_bc_slip<<<grid(g1 - g0), kBlock, 0, s>>>(g0, g1, (uint32_t)m.N, m.cell_geo, m.face_geo, m.ghost, b, cur);
    count_launch();
}

void launch_bc_farfield(const DevMesh& m, uint32_t g0, uint32_t g1, float* rho[2], float4* rhou[2],
                        float* rhoe[2], int cur, float3 mach, float p, float t, cudaStream_t s) {
    if (g1 <= g0) return;
    GhostBuf b = {{rho[0], rho[1]}, {rhou[0], rhou[1]}, {rhoe[0], rhoe[1]}};
    k_bc_farfield<<<grid(g1 - g0), kBlock, 0, s>>>(g0, g1, (uint32_t)m.N, m.cell_geo, m.face_geo, m.ghost, b, cur,
                                                   mach, p, t);
    count_launch();
}

void launch_grad_lim(const DevMesh& m, EulerState q, EulerGrad g, cudaStream_t s) {
    if (m.N == 0) return;
    k_grad_lim<<<grid(m.N), kBlock, 0, s>>>((uint32_t)m.N, m.cell_geo, m.face_geo, m.start, m.nb, m.lsq, q, g);
    count_launch();
}

void launch_flux(const DevMesh& m, EulerState q, EulerGrad g, float* rho_n, float4* rhou_n, float* rhoe_n,
                 float* err, double* partials, float cfl, bool transposed, cudaStream_t s) {
    if (m.N == 0) return;
    if (transposed)
        k_flux<true><<<grid(m.N), kBlock, 0, s>>>((uint32_t)m.N, m.cell_geo, m.face_geo, m.start, m.nb, q, g.rho,
                                                  g.rhou, g.rhoe, rho_n, rhou_n, rhoe_n, err, partials, cfl);
    else
        k_flux<false><<<grid(m.N), kBlock, 0, s>>>((uint32_t)m.N, m.cell_geo, m.face_geo, m.start, m.nb, q, g.rho,
                                                   g.rhou, g.rhoe, rho_n, rhou_n, rhoe_n, err, partials, cfl);
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

void launch_reduce_final(int n_partials, const double* partials, double* out, double* history,
                         unsigned long long* counter, cudaStream_t s) {
    k_reduce_final<<<1, kBlock, 0, s>>>(n_partials, partials, out, history, counter);
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
