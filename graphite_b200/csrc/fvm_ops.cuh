// The reference's generic finite-volume operators (include/fvmops.cuh:96-219)
// as composable device functors over the renumbered layout.
//
// Each operator is a per-cell sum over the cell's faces (fvmOpSetup,
// include/fvmops.cuh:33-48).  OpFace is one face of cell c0 as every
// operator sees it: c1 the neighbour across the face, d0 = face centre - c0,
// d1 = face centre - c1, n the face normal oriented away from c0 and
// ds = face area / volume of c0.  A ghost neighbour carries its interior
// cell's gradient and limiter (fvmScalGradLimBc, src/fvmops.cu:272-304), so
// g1 (the owner of the neighbour's gradient) is c0 there.
//
// An operator functor holds its inputs and gives its contribution of one
// face, `contrib(face)`, of type Out: float (scalar), float3 (vector) or Tens3
// (the reference's tensor{u, v, w}, outer(a, b) = (a b.x, a b.y, a b.z)).
// cell_sum(m, c0, op) is the operator at cell c0; a kernel composes several
// operators by adding their contributions inside one for_each_face pass (as
// k_fvm_terms does for a linear combination).
#pragma once

#include "euler_ops.cuh"

namespace gb {
namespace fvm {

// the float3 arithmetic of euler_ops.cuh (the Tens3 operators below would
// otherwise hide it here)
using gb::operator+;
using gb::operator-;
using gb::operator*;

struct Tens3 {
    float3 r[3];
};
__device__ __forceinline__ Tens3 operator+(const Tens3& a, const Tens3& b) {
    return Tens3{{a.r[0] + b.r[0], a.r[1] + b.r[1], a.r[2] + b.r[2]}};
}
__device__ __forceinline__ Tens3 operator*(const Tens3& a, float c) { return Tens3{{a.r[0] * c, a.r[1] * c, a.r[2] * c}}; }
// outer(a, b) = (a b.x, a b.y, a b.z)
__device__ __forceinline__ Tens3 outer(float3 a, float3 b) { return Tens3{{a * b.x, a * b.y, a * b.z}}; }

template <class T>
__device__ __forceinline__ T zero();
template <>
__device__ __forceinline__ float zero<float>() { return 0.f; }
template <>
__device__ __forceinline__ float3 zero<float3>() { return make_float3(0.f, 0.f, 0.f); }
template <>
__device__ __forceinline__ Tens3 zero<Tens3>() { return Tens3{{zero<float3>(), zero<float3>(), zero<float3>()}}; }

struct OpFace {
    uint32_t c0, c1, g1;
    float3 n;
    float ds;
    float3 d0, d1, fc;
};

// face slot k (entry c0 + t N) of cell c0
__device__ __forceinline__ OpFace op_face(const MeshDev& m, uint32_t c0, uint32_t k) {
    OpFace f;
    f.c0 = c0;
    f.c1 = __ldg(&m.nbc[k]);
    const uint32_t t = __ldg(&m.twin[k]);
    const bool ghost = t >= m.S;
    f.g1 = ghost ? c0 : f.c1;
    const float4 gk = __ldg(&m.cf_geo[k]);
    f.n = f3(gk);
    f.ds = gk.w;
    f.d0 = f3(__ldg(&m.df[k]));
    f.fc = f3(__ldg(&m.face_geo[2 * __ldg(&m.nb[k]).x + 1]));
    f.d1 = ghost ? f.fc - f3(__ldg(&m.cell_geo[f.c1])) : f3(__ldg(&m.df[t]));
    return f;
}

template <class F>
__device__ __forceinline__ void for_each_face(const MeshDev& m, uint32_t c0, F&& fn) {
    const uint32_t nf = __ldg(&m.nfc[c0]);
    for (uint32_t k = c0; k < c0 + nf * m.N; k += m.N) fn(op_face(m, c0, k));
}

__device__ __forceinline__ float3 grad_of(const float4* g, uint32_t c) { return f3(__ldg(&g[c])); }

// fvmLaplacianC: dot(grad c1 + grad c0, n) / 2 ds (needs the gradient)
struct LaplacianC {
    using Out = float;
    const float4* g;
    __device__ __forceinline__ float contrib(const OpFace& f) const {
        return dot(grad_of(g, f.g1) + grad_of(g, f.c0), f.n) * 0.5f * f.ds;
    }
};

// fvmScalGradC: n (u1 phi + u0 (1 - phi)) ds, phi = |d0| / |d0 - d1|
struct ScalGradC {
    using Out = float3;
    const float* s;
    __device__ __forceinline__ float3 contrib(const OpFace& f) const {
        const float phi = norm(f.d0) / norm(f.d0 - f.d1);
        return f.n * ((__ldg(&s[f.c1]) * phi + __ldg(&s[f.c0]) * (1.f - phi)) * f.ds);
    }
};

// fvmScalGradCCorrect: n (grad c0 . (fc - (d0 - d1) phi)) ds, the face centre
// taken as is, as the reference does (needs the gradient)
struct ScalGradCCorrect {
    using Out = float3;
    const float4* g;
    __device__ __forceinline__ float3 contrib(const OpFace& f) const {
        const float phi = norm(f.d0) / norm(f.d0 - f.d1);
        const float3 d_err = f.fc - (f.d0 - f.d1) * phi;
        return f.n * (dot(grad_of(g, f.c0), d_err) * f.ds);
    }
};

// fvmVecGradC: outer(n, u1 phi + u0 (1 - phi)) ds, phi = |d0| / (|d0| + |d1|)
struct VecGradC {
    using Out = Tens3;
    const float4* v;
    __device__ __forceinline__ Tens3 contrib(const OpFace& f) const {
        const float l0 = norm(f.d0), l1 = norm(f.d1);
        const float phi = l0 / (l0 + l1);
        const float3 w = (f3(__ldg(&v[f.c1])) * phi + f3(__ldg(&v[f.c0])) * (1.f - phi)) * f.ds;
        return outer(f.n, w);
    }
};

// fvmBoundScalGradC: n (u1 - u0) ds
struct BoundScalGradC {
    using Out = float3;
    const float* s;
    __device__ __forceinline__ float3 contrib(const OpFace& f) const {
        return f.n * ((__ldg(&s[f.c1]) - __ldg(&s[f.c0])) * f.ds);
    }
};

// fvmBoundVecGradC: outer(u1 - u0, n) ds
struct BoundVecGradC {
    using Out = Tens3;
    const float4* v;
    __device__ __forceinline__ Tens3 contrib(const OpFace& f) const {
        return outer((f3(__ldg(&v[f.c1])) - f3(__ldg(&v[f.c0]))) * f.ds, f.n);
    }
};

// fvmDivC: (u0 + u1) . n / 2 ds
struct DivC {
    using Out = float;
    const float4* v;
    __device__ __forceinline__ float contrib(const OpFace& f) const {
        return dot(f3(__ldg(&v[f.c0])) + f3(__ldg(&v[f.c1])), f.n) * 0.5f * f.ds;
    }
};

// fvmConvConstScalU (SECOND = false) and fvmConvConstScalU2 (SECOND: the
// face values reconstructed with each side's gradient and limiter): upwinded
// flux of u by the constant velocity phi
template <bool SECOND>
struct ConvConstScal {
    using Out = float;
    const float* s;
    const float4* g;   // SECOND only
    float3 phi;
    __device__ __forceinline__ float contrib(const OpFace& f) const {
        float a = __ldg(&s[f.c0]), b = __ldg(&s[f.c1]);
        if (SECOND) {
            const float4 ga = __ldg(&g[f.c0]), gb = __ldg(&g[f.g1]);
            a = a + dot(f3(ga), f.d0) * ga.w;
            b = b + dot(f3(gb), f.d1) * gb.w;
        }
        const float an = dot(f.n, phi);
        return ((an * a + an * b) - fmaxf(fabsf(an), fabsf(an)) * (b - a)) * 0.5f * f.ds;
    }
};

// fvmConvScalU: upwinded flux of u by the velocity field phi
struct ConvScalU {
    using Out = float;
    const float* s;
    const float4* phi;
    __device__ __forceinline__ float contrib(const OpFace& f) const {
        const float u0 = __ldg(&s[f.c0]), u1 = __ldg(&s[f.c1]);
        const float a0 = dot(f.n, f3(__ldg(&phi[f.c0]))), a1 = dot(f.n, f3(__ldg(&phi[f.c1])));
        return ((a0 * u0 + a1 * u1) - fmaxf(fabsf(a0), fabsf(a1)) * (u1 - u0)) * 0.5f * f.ds;
    }
};

// fvmConvVecU: the same for a vector u; the dissipation takes max(a0, a1),
// not of |a|, as the reference does
struct ConvVecU {
    using Out = float3;
    const float4* v;
    const float4* phi;
    __device__ __forceinline__ float3 contrib(const OpFace& f) const {
        const float3 u0 = f3(__ldg(&v[f.c0])), u1 = f3(__ldg(&v[f.c1]));
        const float a0 = dot(f.n, f3(__ldg(&phi[f.c0]))), a1 = dot(f.n, f3(__ldg(&phi[f.c1])));
        return ((u0 * a0 + u1 * a1) - (u1 - u0) * fmaxf(a0, a1)) * (0.5f * f.ds);
    }
};

// The operator at cell c0.
template <class Op>
__device__ __forceinline__ typename Op::Out cell_sum(const MeshDev& m, uint32_t c0, const Op& op) {
    typename Op::Out x = zero<typename Op::Out>();
    for_each_face(m, c0, [&](const OpFace& f) { x = x + op.contrib(f); });
    return x;
}

}  // namespace fvm
}  // namespace gb
