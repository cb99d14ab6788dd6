// Launches of the reference's generic finite-volume operators
// (include/fvmops.cuh:96-219; the operators themselves are the device
// functors of fvm_ops.cuh): one operator over every interior cell, or a
// linear combination of operators in one pass over each cell's faces; and the
// least-squares gradient + limiter of any scalar or vector field
// (ScalarVarComputeGradient / VectorVarComputeGradient and the limiter pass,
// src/fvmops.cu:51-266).
#include <algorithm>

#include "fvm_ops.cuh"

namespace gb {
namespace {

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
__device__ __forceinline__ void store_planar(float* out, uint32_t N, uint32_t i, float x) { out[i] = x; }
__device__ __forceinline__ void store_planar(float* out, uint32_t N, uint32_t i, float3 x) {
    out[i] = x.x; out[N + i] = x.y; out[2 * N + i] = x.z;
}
__device__ __forceinline__ void store_planar(float* out, uint32_t N, uint32_t i, const fvm::Tens3& x) {
#pragma unroll
    for (int b = 0; b < 3; ++b) store_planar(out + 3 * b * (size_t)N, N, i, x.r[b]);
}

template <class Op>
__global__ void k_fvm_op(MeshDev m, Op op, float* __restrict__ out) {
    const uint32_t c0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c0 < m.N) store_planar(out, m.N, c0, fvm::cell_sum(m, c0, op));
}

// One term of a linear combination of operators (gbFvmApplyTerms).
struct TermDev {
    int op;
    float coef;
    const float* s;
    const float4* v;
    const float4* g;
    const float4* phi;
    float3 phi_c;
};
struct TermList {
    int n;
    TermDev t[kFvmMaxTerms];
};

// the face contribution of term t (operators of the output type of OUT)
template <int OUT>
__device__ __forceinline__ void term_contrib(const TermDev& t, const fvm::OpFace& f, float& x1, float3& x3) {
    using namespace fvm;
    if (OUT == 1) {
        switch (t.op) {
            case 0: x1 = x1 + LaplacianC{t.g}.contrib(f) * t.coef; break;
            case 6: x1 = x1 + DivC{t.v}.contrib(f) * t.coef; break;
            case 7: x1 = x1 + ConvConstScal<false>{t.s, t.g, t.phi_c}.contrib(f) * t.coef; break;
            case 8: x1 = x1 + ConvConstScal<true>{t.s, t.g, t.phi_c}.contrib(f) * t.coef; break;
            case 9: x1 = x1 + ConvScalU{t.s, t.phi}.contrib(f) * t.coef; break;
            default: break;
        }
    } else {
        switch (t.op) {
            case 1: x3 = x3 + ScalGradC{t.s}.contrib(f) * t.coef; break;
            case 2: x3 = x3 + ScalGradCCorrect{t.g}.contrib(f) * t.coef; break;
            case 4: x3 = x3 + BoundScalGradC{t.s}.contrib(f) * t.coef; break;
            case 10: x3 = x3 + ConvVecU{t.v, t.phi}.contrib(f) * t.coef; break;
            default: break;
        }
    }
}

// sum of coef x operator over the terms, one pass over each cell's faces,
// into the interior cells of a scalar (OUT = 1) or vector (OUT = 3) field
template <int OUT>
__global__ void k_fvm_terms(MeshDev m, TermList terms, float* __restrict__ out_s, float4* __restrict__ out_v) {
    const uint32_t c0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c0 >= m.N) return;
    float x1 = 0.f;
    float3 x3 = make_float3(0.f, 0.f, 0.f);
    fvm::for_each_face(m, c0, [&](const fvm::OpFace& f) {
        for (int q = 0; q < terms.n; ++q) term_contrib<OUT>(terms.t[q], f, x1, x3);
    });
    if (OUT == 1) out_s[c0] = x1;
    else out_v[c0] = make_float4(x3.x, x3.y, x3.z, 0.f);
}

// ScalarVarInit / VectorVarInit (src/fvmops.cu:8-44): every value, cells and
// ghosts, in both buffers; gradients zero with limiter 1 where the field has
// them.
__global__ void k_field_init(int64_t n, float* s0, float* s1, float4* v0, float4* v1, float4 value, int64_t n_grad,
                             float4* grad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        if (s0) { s0[i] = value.x; s1[i] = value.x; }
        else { v0[i] = value; v1[i] = value; }
    }
    if (i < n_grad) grad[i] = make_float4(0.f, 0.f, 0.f, 1.f);
}

// fvmScalarBcFixed (src/fvmops.cu:308-323) and fvmScalarBcZeroGrad /
// fvmVectorBcZeroGrad (src/fvmops.cu:326-366) on the ghosts [g0, g1) of one
// region: the given value, or the interior cell's current value, into both
// buffers.
__global__ void k_field_bc(uint32_t g0, uint32_t g1, uint32_t N, const uint2* __restrict__ ghost, int zero_grad,
                           int cur, float* s0, float* s1, float4* v0, float4* v1, float4 value) {
    const uint32_t t = g0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g1) return;
    if (s0) {
        const float x = zero_grad ? (cur ? s1 : s0)[ghost[t - N].x] : value.x;
        s0[t] = x;
        s1[t] = x;
    } else {
        const float4 x = zero_grad ? (cur ? v1 : v0)[ghost[t - N].x] : value;
        v0[t] = x;
        v1[t] = x;
    }
}

// y += a x over the interior cells (scalar: s, vector: v arrays)
__global__ void k_field_axpy(uint32_t N, float a, const float* __restrict__ xs, float* ys, const float4* __restrict__ xv,
                             float4* yv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (ys) {
        ys[i] = ys[i] + a * xs[i];
    } else {
        const float4 x = xv[i], y = yv[i];
        yv[i] = make_float4(y.x + a * x.x, y.y + a * x.y, y.z + a * x.z, y.w);
    }
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
    using namespace fvm;
    const MeshDev md = mesh_dev(m);
    const unsigned gn = grid_n(m.N);
    switch (op) {
        case 0: k_fvm_op<<<gn, kBlock, 0, st>>>(md, LaplacianC{g}, out); break;
        case 1: k_fvm_op<<<gn, kBlock, 0, st>>>(md, ScalGradC{s}, out); break;
        case 2: k_fvm_op<<<gn, kBlock, 0, st>>>(md, ScalGradCCorrect{g}, out); break;
        case 3: k_fvm_op<<<gn, kBlock, 0, st>>>(md, VecGradC{v}, out); break;
        case 4: k_fvm_op<<<gn, kBlock, 0, st>>>(md, BoundScalGradC{s}, out); break;
        case 5: k_fvm_op<<<gn, kBlock, 0, st>>>(md, BoundVecGradC{v}, out); break;
        case 6: k_fvm_op<<<gn, kBlock, 0, st>>>(md, DivC{v}, out); break;
        case 7: k_fvm_op<<<gn, kBlock, 0, st>>>(md, ConvConstScal<false>{s, g, phi_c}, out); break;
        case 8: k_fvm_op<<<gn, kBlock, 0, st>>>(md, ConvConstScal<true>{s, g, phi_c}, out); break;
        case 9: k_fvm_op<<<gn, kBlock, 0, st>>>(md, ConvScalU{s, phi}, out); break;
        case 10: k_fvm_op<<<gn, kBlock, 0, st>>>(md, ConvVecU{v, phi}, out); break;
        default: return;
    }
    count_launch();
}

void launch_field_init(int64_t n, int comps, void* val0, void* val1, float4 value, int64_t n_grad, float4* grad,
                       cudaStream_t st) {
    const int64_t m = std::max(n, n_grad);
    if (m == 0) return;
    if (comps == 1)
        k_field_init<<<grid_n(m), kBlock, 0, st>>>(n, (float*)val0, (float*)val1, nullptr, nullptr, value, n_grad, grad);
    else
        k_field_init<<<grid_n(m), kBlock, 0, st>>>(n, nullptr, nullptr, (float4*)val0, (float4*)val1, value, n_grad, grad);
    count_launch();
}

void launch_field_bc(const DevMesh& m, uint32_t g0, uint32_t g1, int comps, int zero_grad, int cur, void* val0,
                     void* val1, float4 value, cudaStream_t st) {
    if (g1 <= g0) return;
    if (comps == 1)
        k_field_bc<<<grid_n(g1 - g0), kBlock, 0, st>>>(g0, g1, (uint32_t)m.N, m.ghost, zero_grad, cur, (float*)val0,
                                                       (float*)val1, nullptr, nullptr, value);
    else
        k_field_bc<<<grid_n(g1 - g0), kBlock, 0, st>>>(g0, g1, (uint32_t)m.N, m.ghost, zero_grad, cur, nullptr, nullptr,
                                                       (float4*)val0, (float4*)val1, value);
    count_launch();
}

void launch_field_axpy(const DevMesh& m, int comps, float a, const void* x, void* y, cudaStream_t st) {
    if (m.N == 0) return;
    if (comps == 1)
        k_field_axpy<<<grid_n(m.N), kBlock, 0, st>>>((uint32_t)m.N, a, (const float*)x, (float*)y, nullptr, nullptr);
    else
        k_field_axpy<<<grid_n(m.N), kBlock, 0, st>>>((uint32_t)m.N, a, nullptr, nullptr, (const float4*)x, (float4*)y);
    count_launch();
}

void launch_fvm_terms(const DevMesh& m, int out_comps, int n_terms, const FvmTermDev* terms, float* out_s,
                      float4* out_v, cudaStream_t st) {
    if (m.N == 0) return;
    TermList tl{};
    tl.n = n_terms;
    for (int q = 0; q < n_terms; ++q)
        tl.t[q] = TermDev{terms[q].op, terms[q].coef, terms[q].s, terms[q].v, terms[q].g, terms[q].phi, terms[q].phi_c};
    if (out_comps == 1) k_fvm_terms<1><<<grid_n(m.N), kBlock, 0, st>>>(mesh_dev(m), tl, out_s, nullptr);
    else k_fvm_terms<3><<<grid_n(m.N), kBlock, 0, st>>>(mesh_dev(m), tl, nullptr, out_v);
    count_launch();
}

}  // namespace gb
