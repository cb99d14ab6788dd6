// The reference's generic finite-volume operators (include/fvmops.cuh:96-219)
// on the renumbered layout, and the least-squares gradient + limiter of any
// scalar or vector field (ScalarVarComputeGradient / VectorVarComputeGradient
// and the limiter pass, src/fvmops.cu:51-266).
//
// Every operator is a per-cell sum over the cell's faces (fvmOpSetup,
// include/fvmops.cuh:33-48): with c1 the neighbour across the face,
// d0 = face centre - c0, d1 = face centre - c1, n the face normal oriented
// away from c0 and ds = face area / volume of c0.  A ghost neighbour carries
// its interior cell's gradient and limiter (fvmScalGradLimBc,
// src/fvmops.cu:272-304).  Tensors are stored as the reference's
// tensor{u, v, w}: outer(a, b) = (a b.x, a b.y, a b.z).
#include "euler_ops.cuh"

namespace gb {
namespace {

struct OpIn {
    const float* s;        // scalar values (N+G) or null
    const float4* v;       // vector values (N+G) or null
    const float4* g;       // gradients + limiters: N (scalar) or 3N (vector)
    const float4* phi;     // per-cell vector field (convection ops) or null
    float3 phi_c;          // constant vector (convection ops)
};

__device__ __forceinline__ float3 gvec(const float4* g, uint32_t c, int a, int comps) {
    return f3(__ldg(&g[comps * c + a]));
}

template <int COMPS>
__global__ void k_fvm_grad(MeshDev m, const float* __restrict__ s, const float4* __restrict__ v, float4* grad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.N) return;
    float u[COMPS];
    if (COMPS == 1) u[0] = __ldg(&s[i]);
    else { const float4 x = __ldg(&v[i]); u[0] = x.x; u[COMPS > 1 ? 1 : 0] = x.y; u[COMPS > 2 ? 2 : 0] = x.z; }
    float3 gs[COMPS];
    float lo[COMPS], hi[COMPS];
#pragma unroll
    for (int c = 0; c < COMPS; ++c) { gs[c] = make_float3(0.f, 0.f, 0.f); lo[c] = hi[c] = u[c]; }
    const uint32_t nf = __ldg(&m.nfc[i]);
    for (uint32_t k = i; k < i + nf * m.N; k += m.N) {
        const uint32_t j = __ldg(&m.nbc[k]);
        const float4 dw = __ldg(&m.dn[k]);
        float uj[COMPS];
        if (COMPS == 1) uj[0] = __ldg(&s[j]);
        else { const float4 x = __ldg(&v[j]); uj[0] = x.x; uj[COMPS > 1 ? 1 : 0] = x.y; uj[COMPS > 2 ? 2 : 0] = x.z; }
#pragma unroll
        for (int c = 0; c < COMPS; ++c) {
            gs[c] = gs[c] + (f3(dw) * (uj[c] - u[c])) * dw.w;
            lo[c] = fminf(lo[c], uj[c]);
            hi[c] = fmaxf(hi[c], uj[c]);
        }
    }
    const float4 l0 = __ldg(&m.lsq[2 * i]), l1 = __ldg(&m.lsq[2 * i + 1]);
    float lim[COMPS];
#pragma unroll
    for (int c = 0; c < COMPS; ++c) { gs[c] = sym_mul(l0, l1, gs[c]); lim[c] = 2.f; }
    for (uint32_t k = i; k < i + nf * m.N; k += m.N) {
        const float4 dk = __ldg(&m.df[k]);
#pragma unroll
        for (int c = 0; c < COMPS; ++c) lim[c] = fminf(lim[c], limiter(u[c], gs[c], lo[c], hi[c], f3(dk), dk.w));
    }
#pragma unroll
    for (int c = 0; c < COMPS; ++c) grad[COMPS * i + c] = make_float4(gs[c].x, gs[c].y, gs[c].z, lim[c]);
}

// out: planar, out[q * N + i] for component q of cell i
__global__ void k_fvm_apply(MeshDev m, int op, OpIn in, float* __restrict__ out) {
    const uint32_t c0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c0 >= m.N) return;
    float x[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) x[q] = 0.f;
    const int comps = in.v ? 3 : 1;
    const uint32_t nf = __ldg(&m.nfc[c0]);
    for (uint32_t k = c0; k < c0 + nf * m.N; k += m.N) {
        const uint32_t c1 = __ldg(&m.nbc[k]);
        const uint32_t t = __ldg(&m.twin[k]);
        const bool ghost = t >= m.S;
        const uint32_t g1 = ghost ? c0 : c1;            // gradient owner of the neighbour
        const float4 gk = __ldg(&m.cf_geo[k]);
        const float3 n = f3(gk);
        const float ds = gk.w;
        const float3 d0 = f3(__ldg(&m.df[k]));
        const float3 fc = f3(__ldg(&m.face_geo[2 * __ldg(&m.nb[k]).x + 1]));
        const float3 d1 = ghost ? fc - f3(__ldg(&m.cell_geo[c1])) : f3(__ldg(&m.df[t]));
        if (comps == 1) {
            const float u0 = __ldg(&in.s[c0]), u1 = __ldg(&in.s[c1]);
            switch (op) {
                case 0: {   // fvmLaplacianC: dot(grad c1 + grad c0, n) / 2 ds
                    x[0] += dot(gvec(in.g, g1, 0, 1) + gvec(in.g, c0, 0, 1), n) * 0.5f * ds;
                    break;
                }
                case 1: {   // fvmScalGradC
                    const float phi = norm(d0) / norm(d0 - d1);
                    const float3 r = n * ((u1 * phi + u0 * (1.f - phi)) * ds);
                    x[0] += r.x; x[1] += r.y; x[2] += r.z;
                    break;
                }
                case 2: {   // fvmScalGradCCorrect (face centre taken as is, as the reference does)
                    const float phi = norm(d0) / norm(d0 - d1);
                    const float3 d_err = fc - (d0 - d1) * phi;
                    const float3 r = n * (dot(gvec(in.g, c0, 0, 1), d_err) * ds);
                    x[0] += r.x; x[1] += r.y; x[2] += r.z;
                    break;
                }
                case 4: {   // fvmBoundScalGradC
                    const float3 r = n * ((u1 - u0) * ds);
                    x[0] += r.x; x[1] += r.y; x[2] += r.z;
                    break;
                }
                case 7: case 8: {   // fvmConvConstScalU / fvmConvConstScalU2
                    float a = u0, b = u1;
                    if (op == 8) {
                        const float4 ga = __ldg(&in.g[c0]), gb = __ldg(&in.g[g1]);
                        a = u0 + dot(f3(ga), d0) * ga.w;
                        b = u1 + dot(f3(gb), d1) * gb.w;
                    }
                    const float an = dot(n, in.phi_c);
                    x[0] += ((an * a + an * b) - fmaxf(fabsf(an), fabsf(an)) * (b - a)) * 0.5f * ds;
                    break;
                }
                case 9: {   // fvmConvScalU
                    const float a0 = dot(n, f3(__ldg(&in.phi[c0]))), a1 = dot(n, f3(__ldg(&in.phi[c1])));
                    x[0] += ((a0 * u0 + a1 * u1) - fmaxf(fabsf(a0), fabsf(a1)) * (u1 - u0)) * 0.5f * ds;
                    break;
                }
                default: break;
            }
        } else {
            const float3 u0 = f3(__ldg(&in.v[c0])), u1 = f3(__ldg(&in.v[c1]));
            switch (op) {
                case 3: {   // fvmVecGradC: outer(n, u1 phi + u0 (1 - phi)) ds
                    const float l0 = norm(d0), l1 = norm(d1);
                    const float phi = l0 / (l0 + l1);
                    const float3 w = (u1 * phi + u0 * (1.f - phi)) * ds;
                    const float wc[3] = {w.x, w.y, w.z};
#pragma unroll
                    for (int b = 0; b < 3; ++b) { x[3 * b] += n.x * wc[b]; x[3 * b + 1] += n.y * wc[b]; x[3 * b + 2] += n.z * wc[b]; }
                    break;
                }
                case 5: {   // fvmBoundVecGradC: outer(u1 - u0, n) ds
                    const float3 du = (u1 - u0) * ds;
                    const float nc[3] = {n.x, n.y, n.z};
#pragma unroll
                    for (int b = 0; b < 3; ++b) { x[3 * b] += du.x * nc[b]; x[3 * b + 1] += du.y * nc[b]; x[3 * b + 2] += du.z * nc[b]; }
                    break;
                }
                case 6: {   // fvmDivC
                    x[0] += dot(u0 + u1, n) * 0.5f * ds;
                    break;
                }
                case 10: {  // fvmConvVecU (the dissipation takes max(a0, a1), not of |a|, as the reference does)
                    const float a0 = dot(n, f3(__ldg(&in.phi[c0]))), a1 = dot(n, f3(__ldg(&in.phi[c1])));
                    const float3 r = ((u0 * a0 + u1 * a1) - (u1 - u0) * fmaxf(a0, a1)) * (0.5f * ds);
                    x[0] += r.x; x[1] += r.y; x[2] += r.z;
                    break;
                }
                default: break;
            }
        }
    }
    const int oc = (op == 3 || op == 5) ? 9 : ((op == 1 || op == 2 || op == 4 || op == 10) ? 3 : 1);
    for (int q = 0; q < oc; ++q) out[(size_t)q * m.N + c0] = x[q];
}

inline unsigned grid_n(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

MeshDev mesh_dev(const DevMesh& m);

void launch_fvm_grad(const DevMesh& m, int comps, const float* s, const float4* v, float4* grad, cudaStream_t st) {
    if (m.N == 0) return;
    if (comps == 1) k_fvm_grad<1><<<grid_n(m.N), kBlock, 0, st>>>(mesh_dev(m), s, v, grad);
    else k_fvm_grad<3><<<grid_n(m.N), kBlock, 0, st>>>(mesh_dev(m), s, v, grad);
    count_launch();
}

void launch_fvm_apply(const DevMesh& m, int op, const float* s, const float4* v, const float4* g, const float4* phi,
                      float3 phi_c, float* out, cudaStream_t st) {
    if (m.N == 0) return;
    k_fvm_apply<<<grid_n(m.N), kBlock, 0, st>>>(mesh_dev(m), op, OpIn{s, v, g, phi, phi_c}, out);
    count_launch();
}

}  // namespace gb
