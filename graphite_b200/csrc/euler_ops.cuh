// Per-cell device math of the Euler iteration, shared by the single-mesh
// kernels (euler.cu) and the batched multi-instance kernels (batch.cu).
#pragma once

#include "gb_device.cuh"

namespace gb {

// Read-only view of a mesh's renumbered device layout.
struct MeshDev {
    const float4* cell_geo;
    const float4* face_geo;
    const uint8_t* nfc;
    const uint2* nb;
    const float4* lsq;
    const uint32_t* twin;
    const float4* cf_geo;
    const uint32_t* nbc;
    const float4* dn;
    const float4* df;
    uint32_t N;
    uint32_t S;
    const int* halt;      // nonzero *halt: a stopped replayed loop's kernels return (may be null)
};

__device__ __forceinline__ bool halted(const int* halt) { return halt && *(const volatile int*)halt; }

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float norm(float3 a) { return sqrtf(dot(a, a)); }
// Explicitly rounded dot product (its multiply-adds fused in a fixed order):
// the boundary states below are formed by several kernels (the ghost kernels
// and the gradient kernels that apply the conditions themselves) and must come
// out bitwise the same in each, whatever the compiler would fuse in context.
__device__ __forceinline__ float xdot(float3 a, float3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
// include/datatypes.cuh:144-150: n * sign(n . d) with sign(0) = +1
__device__ __forceinline__ float3 outer_normal(float3 n, float3 d) {
    return xdot(n, d) >= 0.f ? n : make_float3(-n.x, -n.y, -n.z);
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
// Where sig = 1 the blend sig + (1 - sig) lim is exactly 1 for the finite
// lim this function forms, so that case returns before lim is computed.
__device__ __forceinline__ float limiter(float u, float3 g, float umin, float umax, float3 d, float k3) {
    const float du = umax - u, dd = umin - u;
    const float dmm2 = (du - dd) * (du - dd);
    if (dmm2 <= k3) return 1.f;
    const float delta = dot(g, d);
    float sig;
    if (dmm2 <= 2.f * k3) {
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

// euler_slip_bc, src/models/euler.cu:412-442: the ghost of a boundary face is
// the interior state (r1, u, e1) with the normal momentum mirrored (n outward
// from the interior cell).
__device__ __forceinline__ void slip_state(float3 n, float r1, float3 u, float e1, float& r, float4& ru, float& e) {
    r = r1;
    e = e1;
    const float s = __fmul_rn(2.f, xdot(n, u));
    ru = make_float4(__fmaf_rn(-n.x, s, u.x), __fmaf_rn(-n.y, s, u.y), __fmaf_rn(-n.z, s, u.z), 0.f);
}

// The outward normal of boundary face gl = (interior cell, face); the same
// arithmetic as the per-entry normals of entry_geo_cell.
__device__ __forceinline__ float3 ghost_normal(const float4* __restrict__ cell_geo,
                                               const float4* __restrict__ face_geo, uint2 gl) {
    return outer_normal(f3(face_geo[2 * gl.y]), f3(face_geo[2 * gl.y + 1]) - f3(cell_geo[gl.x]));
}

__device__ __forceinline__ void slip_ghost(const float4* __restrict__ cell_geo, const float4* __restrict__ face_geo,
                                           uint2 gl, const float* rho, const float4* rhou, const float* rhoe,
                                           float& r, float4& ru, float& e) {
    const uint32_t c1 = gl.x;
    slip_state(ghost_normal(cell_geo, face_geo, gl), rho[c1], f3(rhou[c1]), rhoe[c1], r, ru, e);
}

// euler_inletoutlet_bc, src/models/euler.cu:446-520 (gamma = 1.4, R = 1):
// inflow (u.n < 0) supersonic -> free stream, subsonic -> interior pressure
// with free-stream temperature and Mach; outflow supersonic -> interior,
// subsonic -> free-stream pressure with interior temperature and velocity.
// (r1, ru1, e1) is the interior state, n the outward normal.
__device__ __forceinline__ void farfield_state(float3 n, float r1, float3 ru1, float e1, float3 imach, float ip,
                                               float it, float& r, float4& ru4, float& e) {
    // every multiply-add explicitly rounded (see xdot)
    auto scale = [](float3 a, float k) { return make_float3(__fmul_rn(a.x, k), __fmul_rn(a.y, k), __fmul_rn(a.z, k)); };
    const float3 u = scale(ru1, 1.f / r1);
    const float p = __fmul_rn(0.4f, __fmaf_rn(-(0.5f / r1), xdot(ru1, ru1), e1));
    const float tt = p / r1;
    const float mach = sqrtf(xdot(u, u) / (__fmul_rn(1.4f, p) / r1));
    const float idens = ip / it;
    float3 ru;
    if (xdot(u, n) < 0.f) {
        if (mach > 1.f) {
            const float ic = sqrtf(__fmul_rn(1.4f, ip) / idens);
            const float3 iv = scale(imach, ic);
            r = idens;
            ru = scale(iv, idens);
            e = __fmaf_rn(__fmul_rn(0.5f, idens), xdot(iv, iv), ip / 0.4f);
        } else {
            r = p / it;
            const float ic = sqrtf(__fmul_rn(1.4f, p) / r);
            const float3 v = scale(imach, ic);
            ru = scale(v, r);
            e = __fmaf_rn(__fmul_rn(0.5f, r), xdot(v, v), p / 0.4f);
        }
    } else {
        if (mach > 1.f) {
            r = r1; ru = ru1; e = e1;
        } else {
            r = ip / tt;
            ru = scale(u, r);
            e = __fmaf_rn(__fmul_rn(0.5f, r), xdot(u, u), ip / 0.4f);
        }
    }
    ru4 = make_float4(ru.x, ru.y, ru.z, 0.f);
}

__device__ __forceinline__ void farfield_ghost(const float4* __restrict__ cell_geo,
                                               const float4* __restrict__ face_geo, uint2 gl, const float* rho,
                                               const float4* rhou, const float* rhoe, float3 imach, float ip,
                                               float it, float& r, float4& ru4, float& e) {
    const uint32_t c1 = gl.x;
    farfield_state(ghost_normal(cell_geo, face_geo, gl), rho[c1], f3(rhou[c1]), rhoe[c1], imach, ip, it, r, ru4, e);
}

// A Ghosts policy of grad_lim_cell applies boundary conditions inside the
// gradient pass instead of by a separate ghost kernel: with kActive,
// state(j, n, interior state) gives the state of ghost j when a condition
// covers it (slip_state / farfield_state with the entry's outward normal,
// which is bitwise the normal the ghost kernels compute) and store() writes
// it into both value buffers.  NoGhostBcs leaves every ghost to its stored
// state.
struct NoGhostBcs {
    static constexpr bool kActive = false;
    __device__ __forceinline__ bool state(uint32_t, float3, float, float3, float, float&, float4&, float&) const {
        return false;
    }
    __device__ __forceinline__ void store(uint32_t, float, float4, float) const {}
};

// GhostBcTable (gb_device.cuh) as a Ghosts policy.
struct GhostBcs {
    static constexpr bool kActive = true;
    GhostBcTable t;
    // j: the ghost's cell index
    __device__ __forceinline__ bool state(uint32_t j, float3 nrm, float r1, float3 u1, float e1, float& r, float4& ru,
                                          float& e) const {
        int k = 0;
        while (k < t.n - 1 && j >= t.start[k + 1]) ++k;
        if (t.type[k] < 0) return false;
        if (t.type[k] == 0) slip_state(nrm, r1, u1, e1, r, ru, e);
        else farfield_state(nrm, r1, u1, e1, t.mach[k], t.p[k], t.temp[k], r, ru, e);
        return true;
    }
    __device__ __forceinline__ void store(uint32_t j, float r, float4 ru, float e) const {
        if (!t.store) return;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            t.rho[b][j] = r;
            t.rhou[b][j] = ru;
            t.rhoe[b][j] = e;
        }
    }
};

// How the per-cell functions read data that an iteration writes (states,
// face states): through the read-only cache (LdNc, for kernels that never
// write what they read in the same launch) or from L2 (LdCg, for a kernel
// that writes those arrays itself and reads them again after a grid-wide
// barrier, where the non-coherent read-only path could return stale lines).
struct LdNc {
    template <typename T>
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};
struct LdCg {
    template <typename T>
    __device__ __forceinline__ static T ld(const T* p) { return __ldcg(p); }
};

// Per-face entry data of cell i (slot t = 0..nf-1), read straight from the
// slot-major arrays at entry i + t N.
struct EntriesGlobal {
    const MeshDev& m;
    uint32_t i;
    __device__ __forceinline__ uint32_t nbc(uint32_t t) const { return __ldg(&m.nbc[i + t * m.N]); }
    __device__ __forceinline__ float4 dn(uint32_t t) const { return __ldg(&m.dn[i + t * m.N]); }
    __device__ __forceinline__ float4 df(uint32_t t) const { return __ldg(&m.df[i + t * m.N]); }
    __device__ __forceinline__ void ready() const {}
};

// The same entries copied by this thread into its own shared-memory slots
// (slot t at t * B past the thread's base) with cp.async: every face's
// stream is in flight at once instead of one face at a time.
template <int B>
struct EntriesStaged {
    const uint32_t* s_nbc;
    const float4* s_dn;
    const float4* s_df;
    __device__ __forceinline__ uint32_t nbc(uint32_t t) const { return s_nbc[t * B]; }
    __device__ __forceinline__ float4 dn(uint32_t t) const { return s_dn[t * B]; }
    __device__ __forceinline__ float4 df(uint32_t t) const { return s_df[t * B]; }
    __device__ __forceinline__ void ready() const { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
};

// Neighbour index and neighbour offset staged like EntriesStaged, the face
// offset read from its slot-major array when it is used (a smaller
// shared-memory footprint per thread).
template <int B>
struct EntriesStagedDn {
    const uint32_t* s_nbc;
    const float4* s_dn;
    const float4* df_cell;    // &m.df[i]; slot t at t * N
    uint32_t N;
    __device__ __forceinline__ uint32_t nbc(uint32_t t) const { return s_nbc[t * B]; }
    __device__ __forceinline__ float4 dn(uint32_t t) const { return s_dn[t * B]; }
    __device__ __forceinline__ float4 df(uint32_t t) const { return __ldg(df_cell + t * N); }
    __device__ __forceinline__ void ready() const { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(gmem) : "memory");
}

// Faces per step of grad_lim_cell's gathering loop: two faces' neighbour
// gathers in flight together (1.6 % faster per call on the swept wing than
// one, with the same results; three or five were slower).
#ifndef GB_GRAD_UNROLL
#define GB_GRAD_UNROLL 2
#endif
constexpr int kGradUnroll = GB_GRAD_UNROLL;
// Fused FvmEulerStepPrepare for one interior cell i (src/models/euler.cu:597-647):
// least-squares gradients (src/fvmops.cu:51-111) and limiters
// (src/fvmops.cu:175-266) of rho, rhou (3 components) and rhoE, then the
// limited reconstruction q + lim (grad q . d) of the cell at each of its faces
// (the face states of fvmEulerSteadyOp, src/models/euler.cu:250-255) and of
// each ghost neighbour, which carries this cell's gradient and limiter
// (fvmScalGradLimBc / fvmVecGradLimBc, src/fvmops.cu:272-304).  nf is the
// cell's face count; e supplies its entries.
template <bool TRANSPOSED, typename Entries, typename Ghosts = NoGhostBcs, typename Ld = LdNc>
__device__ __forceinline__ void grad_lim_cell(const MeshDev& m, EulerState q, EulerGrad g, uint32_t i, uint32_t nf,
                                              const Entries& e, const Ghosts& gh = Ghosts()) {
    float v[5];
    float4 u0;
    {
        u0 = Ld::ld(&q.rhou[i]);
        v[0] = Ld::ld(&q.rho[i]); v[1] = u0.x; v[2] = u0.y; v[3] = u0.z; v[4] = Ld::ld(&q.rhoe[i]);
    }
    e.ready();
    float3 gs[5];
    float vmin[5], vmax[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) { gs[c] = make_float3(0.f, 0.f, 0.f); vmin[c] = v[c]; vmax[c] = v[c]; }
#pragma unroll kGradUnroll
    for (uint32_t t = 0; t < nf; ++t) {
        const uint32_t j = e.nbc(t);
        const float4 dw = e.dn(t);                   // (c_j - c_i, 1 / |c_j - c_i|^2)
        const float3 d = f3(dw);
        float rj, ej;
        float4 uj;
        if (!(Ghosts::kActive && j >= m.N &&
              gh.state(j, f3(__ldg(&m.cf_geo[i + t * m.N])), v[0], f3(u0), v[4], rj, uj, ej))) {
            uj = Ld::ld(&q.rhou[j]);
            rj = Ld::ld(&q.rho[j]);
            ej = Ld::ld(&q.rhoe[j]);
        }
        const float vj[5] = {rj, uj.x, uj.y, uj.z, ej};
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            gs[c] = gs[c] + (d * (vj[c] - v[c])) * dw.w;
            vmin[c] = fminf(vmin[c], vj[c]);
            vmax[c] = fmaxf(vmax[c], vj[c]);
        }
    }
    const float4 l0 = __ldg(&m.lsq[2 * i]), l1 = __ldg(&m.lsq[2 * i + 1]);
#pragma unroll
    for (int c = 0; c < 5; ++c) gs[c] = sym_mul(l0, l1, gs[c]);
    float lim[5] = {2.f, 2.f, 2.f, 2.f, 2.f};
    for (uint32_t t = 0; t < nf; ++t) {
        const float4 dk = e.df(t);                   // (f_c - c_i, |f_c - c_i|^3)
#pragma unroll
        for (int c = 0; c < 5; ++c) lim[c] = fminf(lim[c], limiter(v[c], gs[c], vmin[c], vmax[c], f3(dk), dk.w));
    }
    const float4 gr = make_float4(gs[0].x, gs[0].y, gs[0].z, lim[0]);
    const float4 gu[3] = {make_float4(gs[1].x, gs[1].y, gs[1].z, lim[1]),
                          make_float4(gs[2].x, gs[2].y, gs[2].z, lim[2]),
                          make_float4(gs[3].x, gs[3].y, gs[3].z, lim[3])};
    const float4 ge = make_float4(gs[4].x, gs[4].y, gs[4].z, lim[4]);
    if (g.rho) {
        g.rho[i] = gr;
        g.rhou[3 * i] = gu[0];
        g.rhou[3 * i + 1] = gu[1];
        g.rhou[3 * i + 2] = gu[2];
        g.rhoe[i] = ge;
    }
    for (uint32_t t = 0; t < nf; ++t) {
        const uint32_t k = i + t * m.N;
        float rr, re;
        float3 ru;
        reconstruct<TRANSPOSED>(v[0], u0, v[4], gr, gu, ge, f3(e.df(t)), rr, ru, re);
        g.rec_rho[k] = rr;
        g.rec_rhou[k] = make_float4(ru.x, ru.y, ru.z, re);
        const uint32_t j = e.nbc(t);
        if (j >= m.N) {
            // ghost neighbour N + g: its state with this cell's gradient and
            // limiter, stored at the ghost's face-state slot S + g
            const uint32_t tw = m.S + (j - m.N);
            const float3 fc = f3(__ldg(&m.face_geo[2 * __ldg(&m.nb[k]).x + 1]));
            float rj, ej;
            float4 uj;
            if (Ghosts::kActive && gh.state(j, f3(__ldg(&m.cf_geo[k])), v[0], f3(u0), v[4], rj, uj, ej)) {
                gh.store(j, rj, uj, ej);
            } else {
                uj = Ld::ld(&q.rhou[j]);
                rj = Ld::ld(&q.rho[j]);
                ej = Ld::ld(&q.rhoe[j]);
            }
            reconstruct<TRANSPOSED>(rj, uj, ej, gr, gu, ge, fc - f3(__ldg(&m.cell_geo[j])), rr, ru, re);
            g.rec_rho[tw] = rr;
            g.rec_rhou[tw] = make_float4(ru.x, ru.y, ru.z, re);
        }
    }
}

template <bool TRANSPOSED>
__device__ __forceinline__ void grad_lim_cell(const MeshDev& m, EulerState q, EulerGrad g, uint32_t i) {
    grad_lim_cell<TRANSPOSED>(m, q, g, i, __ldg(&m.nfc[i]), EntriesGlobal{m, i});
}

// Fused fvmEulerSteadyOp + euler_steady_step for one interior cell i
// (src/models/euler.cu:236-381): per face, from the two reconstructed face
// states (this cell's, and the neighbour's through the twin entry), central
// flux 0.5 (F0 + F1) . n A / V minus scalar dissipation 0.5 eig (q1 - q0) A / V
// with eig = max(|u| + c) over both sides, accumulate eig A / V; then
// dt = cfl / sum, q_new = q - F dt (into the other buffer).  Returns the
// squared residual (F_rho^2 + |F_rhou|^2 + F_rhoE^2) V, also stored in err[i]
// when err is not null; with rho_sq, also the density part F_rho^2 V.
template <typename Ld = LdNc>
__device__ __forceinline__ float flux_cell(const MeshDev& m, EulerState q, FaceRecs rec, float* __restrict__ rho_n,
                                           float4* __restrict__ rhou_n, float* __restrict__ rhoe_n,
                                           float* __restrict__ err, float cfl, uint32_t i, float* rho_sq = nullptr) {
    const float vol = __ldg(&m.cell_geo[i]).w;
    float fr = 0.f, fe = 0.f, dts = 0.f;
    float3 fu = make_float3(0.f, 0.f, 0.f);
    const uint32_t nf = __ldg(&m.nfc[i]);
    for (uint32_t k = i; k < i + nf * m.N; k += m.N) {
        const uint32_t t = __ldg(&m.twin[k]);
        const float4 gk = __ldg(&m.cf_geo[k]);
        const float3 n = f3(gk);
        const float ds = gk.w;
        const float ra = Ld::ld(&rec.rho[k]), rb = Ld::ld(&rec.rho[t]);
        const float4 uea = Ld::ld(&rec.rhou[k]), ueb = Ld::ld(&rec.rhou[t]);   // (rho u, rho E)
        const float3 ua = f3(uea), ub = f3(ueb);
        const float ea = uea.w, eb = ueb.w;
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
        const float eig = fmaxf(sqrtf(qa) * ia + lsqrt(1.4f * pa * ia), sqrtf(qb) * ib + lsqrt(1.4f * pb * ib));
        const float eh = eig * h;
        fr -= eh * (rb - ra);
        fu = fu - (ub - ua) * eh;
        fe -= eh * (eb - ea);
        dts += eig * ds;
    }
    const float r0 = Ld::ld(&q.rho[i]);
    const float4 u0 = Ld::ld(&q.rhou[i]);
    const float e0 = Ld::ld(&q.rhoe[i]);
    const float dt = cfl / dts;
    rho_n[i] = r0 - fr * dt;
    rhou_n[i] = make_float4(u0.x - fu.x * dt, u0.y - fu.y * dt, u0.z - fu.z * dt, 0.f);
    rhoe_n[i] = e0 - fe * dt;
    const float e = (fr * fr + dot(fu, fu) + fe * fe) * vol;
    if (err) err[i] = e;
    // explicitly rounded, so that the residual e above compiles as it does
    // without this output
    if (rho_sq) *rho_sq = __fmul_rn(__fmul_rn(fr, fr), vol);
    return e;
}

// The static per-entry geometry of cell i, computed with the arithmetic the
// iteration would otherwise repeat every step: for the flux the face normal
// oriented away from the cell (outer_normal) and the face area over the cell
// volume; for the gradient the neighbour offset with its LSQ weight
// 1 / |d|^2 and the face offset with the limiter's |d|^3.
__device__ __forceinline__ void entry_geo_cell(const MeshDev& m, float4* cf_geo, uint32_t* nbc, float4* dn,
                                               float4* df, uint32_t i) {
    const float4 c0 = __ldg(&m.cell_geo[i]);
    const float3 ci = f3(c0);
    const float inv_v = 1.f / c0.w;
    const uint32_t nf = __ldg(&m.nfc[i]);
    for (uint32_t k = i; k < i + nf * m.N; k += m.N) {
        const uint2 fj = __ldg(&m.nb[k]);
        const float4 na = __ldg(&m.face_geo[2 * fj.x]);
        const float3 fd = f3(__ldg(&m.face_geo[2 * fj.x + 1])) - ci;
        const float3 n = outer_normal(f3(na), fd);
        cf_geo[k] = make_float4(n.x, n.y, n.z, na.w * inv_v);
        const float3 d = f3(__ldg(&m.cell_geo[fj.y])) - ci;
        const float w2 = 1.f / dot(d, d);
        dn[k] = make_float4(d.x, d.y, d.z, w2);
        const float dl = norm(fd);
        df[k] = make_float4(fd.x, fd.y, fd.z, dl * dl * dl);
        nbc[k] = fj.y;
    }
}

}  // namespace gb
