// Mesh metrics in float64, computed once per mesh load (setup, not the
// iteration).  Same formulas as the reference's metric kernels
// (src/mesh.cu:44-219), evaluated in double instead of float; the results
// are then laid out in the renumbered float32 arrays the iteration reads.
#include "gb_device.cuh"

namespace gb {
namespace {

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 ld3(const double* p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void st3(double* p, int64_t i, d3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator*(d3 a, double b) { return {a.x * b, a.y * b, a.z * b}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double nrm(d3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// outer_normal, include/datatypes.cuh:144-150: n * sign(n.d), sign(0) = +1
__device__ __forceinline__ d3 outer_normal(d3 n, d3 d) { return dot(n, d) >= 0.0 ? n : d3{-n.x, -n.y, -n.z}; }

// Fan triangulation from the node average: area, unit normal, area-weighted
// triangle centroid.  src/mesh.cu:44-97.
__global__ void k_face_metrics(int64_t F, const double* __restrict__ nodes, const uint32_t* __restrict__ fns,
                               const uint32_t* __restrict__ fn, double* area, double* normal, double* centre) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F) return;
    const uint32_t s = fns[i], e = fns[i + 1];
    d3 c = {0, 0, 0};
    for (uint32_t k = s; k < e; ++k) c = c + ld3(nodes, fn[k]);
    c = c * (1.0 / (double)(e - s));
    d3 nc = {0, 0, 0}, nsum = {0, 0, 0};
    double a = 0;
    for (uint32_t k = s; k < e; ++k) {
        const d3 p0 = ld3(nodes, fn[k]);
        const d3 p1 = ld3(nodes, fn[k + 1 < e ? k + 1 : s]);
        const d3 x = cross(c - p0, c - p1);
        const double h = nrm(x) * 0.5;
        a += h;
        nsum = nsum + x;
        nc = nc + (p0 + p1 + c) * (h / 3.0);
    }
    area[i] = a;
    st3(normal, i, nsum * (1.0 / nrm(nsum)));
    st3(centre, i, nc * (1.0 / a));
}

// Approximate centroid (area-weighted face centres, then the 0.75 pyramid
// correction weighted by |d| * A) and divergence-theorem volume.
// src/mesh.cu:102-143.
__global__ void k_cell_metrics(int64_t N, const uint32_t* __restrict__ cfs, const uint32_t* __restrict__ cf,
                               const double* __restrict__ area, const double* __restrict__ normal,
                               const double* __restrict__ fcentre, double* ccentre, double* volume) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const uint32_t s = cfs[i], e = cfs[i + 1];
    d3 c0 = {0, 0, 0};
    double w = 0;
    for (uint32_t k = s; k < e; ++k) {
        const uint32_t f = cf[k];
        c0 = c0 + ld3(fcentre, f) * area[f];
        w += area[f];
    }
    c0 = c0 * (1.0 / w);
    d3 c1 = {0, 0, 0};
    w = 0;
    for (uint32_t k = s; k < e; ++k) {
        const uint32_t f = cf[k];
        const d3 d = ld3(fcentre, f) - c0;
        const double wf = nrm(d) * area[f];
        c1 = c1 + (c0 + d * 0.75) * wf;
        w += wf;
    }
    c1 = c1 * (1.0 / w);
    st3(ccentre, i, c1);
    double v = 0;
    for (uint32_t k = s; k < e; ++k) {
        const uint32_t f = cf[k];
        const d3 d = ld3(fcentre, f) - c1;
        v += dot(d, outer_normal(ld3(normal, f), d)) * area[f];
    }
    volume[i] = v / 3.0;
}

// Ghost centroid mirrored through the face along the outward normal, volume
// 2 * A * distance.  src/mesh.cu:148-173.
__global__ void k_ghost_metrics(int64_t G, int64_t N, const uint32_t* __restrict__ cfs, const uint32_t* __restrict__ cf,
                                const uint32_t* __restrict__ cc, const double* __restrict__ area,
                                const double* __restrict__ normal, const double* __restrict__ fcentre,
                                double* ccentre, double* volume) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= G) return;
    const int64_t i = N + t;
    const uint32_t other = cc[cfs[i]];
    const uint32_t f = cf[cfs[i]];
    const d3 fc = ld3(fcentre, f);
    const d3 d = fc - ld3(ccentre, other);
    const double dx = nrm(d);
    st3(ccentre, i, fc + outer_normal(ld3(normal, f), d) * dx);
    volume[i] = area[f] * 2.0 * dx;
}

// Inverse of sum_j d d^T / |d|^2 over all neighbours (ghosts included), by
// adjugate over determinant, stored as 3 columns.  src/mesh.cu:178-219.
__global__ void k_lsq(int64_t N, const uint32_t* __restrict__ cfs, const uint32_t* __restrict__ cc,
                      const double* __restrict__ ccentre, double* minv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const d3 ci = ld3(ccentre, i);
    for (uint32_t k = cfs[i]; k < cfs[i + 1]; ++k) {
        const d3 d = ld3(ccentre, cc[k]) - ci;
        const double w2 = 1.0 / dot(d, d);
        const double v[3] = {d.x, d.y, d.z};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) a[r][c] += v[r] * v[c] * w2;
    }
    double m[3][3];
    m[0][0] = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    m[0][1] = a[0][2] * a[2][1] - a[0][1] * a[2][2];
    m[0][2] = a[0][1] * a[1][2] - a[0][2] * a[1][1];
    m[1][0] = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    m[1][1] = a[0][0] * a[2][2] - a[0][2] * a[2][0];
    m[1][2] = a[0][2] * a[1][0] - a[0][0] * a[1][2];
    m[2][0] = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    m[2][1] = a[0][1] * a[2][0] - a[0][0] * a[2][1];
    m[2][2] = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    const double det = a[0][0] * m[0][0] + a[0][1] * m[1][0] + a[0][2] * m[2][0];
    const double inv = 1.0 / det;
    // column-major like the reference's tensor (u, v, w columns)
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) minv[9 * i + 3 * c + r] = m[r][c] * inv;
}

__global__ void k_layout_cells(int64_t NG, const uint32_t* __restrict__ cell_old, const double* __restrict__ ccentre,
                               const double* __restrict__ volume, float4* cell_geo) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NG) return;
    const uint32_t o = cell_old[i];
    cell_geo[i] = make_float4((float)ccentre[3 * o], (float)ccentre[3 * o + 1], (float)ccentre[3 * o + 2],
                              (float)volume[o]);
}

__global__ void k_layout_faces(int64_t F, const uint32_t* __restrict__ face_old, const double* __restrict__ area,
                               const double* __restrict__ normal, const double* __restrict__ fcentre,
                               float4* face_geo) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F) return;
    const uint32_t o = face_old[i];
    face_geo[2 * i] = make_float4((float)normal[3 * o], (float)normal[3 * o + 1], (float)normal[3 * o + 2],
                                  (float)area[o]);
    face_geo[2 * i + 1] = make_float4((float)fcentre[3 * o], (float)fcentre[3 * o + 1], (float)fcentre[3 * o + 2], 0.f);
}

__global__ void k_layout_lsq(int64_t N, const uint32_t* __restrict__ cell_old, const double* __restrict__ minv,
                             float4* lsq) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double* m = minv + 9 * (int64_t)cell_old[i];
    // column-major: element (r, c) = m[3c + r]; symmetric, so the upper
    // triangle (averaged with the lower one) is kept.
    const double a00 = m[0], a11 = m[4], a22 = m[8];
    const double a01 = 0.5 * (m[3] + m[1]), a02 = 0.5 * (m[6] + m[2]), a12 = 0.5 * (m[7] + m[5]);
    lsq[2 * i] = make_float4((float)a00, (float)a01, (float)a02, (float)a11);
    lsq[2 * i + 1] = make_float4((float)a12, (float)a22, 0.f, 0.f);
}

inline unsigned grid(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

void launch_face_metrics64(int64_t F, const double* nodes, const uint32_t* fns, const uint32_t* fn, double* area,
                           double* normal, double* centre, cudaStream_t s) {
    if (F == 0) return;
    k_face_metrics<<<grid(F), kBlock, 0, s>>>(F, nodes, fns, fn, area, normal, centre);
    count_launch();
}

void launch_cell_metrics64(int64_t N, const uint32_t* cfs, const uint32_t* cf, const double* area,
                           const double* normal, const double* fcentre, double* ccentre, double* volume,
                           cudaStream_t s) {
    if (N == 0) return;
    k_cell_metrics<<<grid(N), kBlock, 0, s>>>(N, cfs, cf, area, normal, fcentre, ccentre, volume);
    count_launch();
}

void launch_ghost_metrics64(int64_t G, int64_t N, const uint32_t* cfs, const uint32_t* cf, const uint32_t* cc,
                            const double* area, const double* normal, const double* fcentre, double* ccentre,
                            double* volume, cudaStream_t s) {
    if (G == 0) return;
    k_ghost_metrics<<<grid(G), kBlock, 0, s>>>(G, N, cfs, cf, cc, area, normal, fcentre, ccentre, volume);
    count_launch();
}

void launch_lsq64(int64_t N, const uint32_t* cfs, const uint32_t* cc, const double* ccentre, double* minv,
                  cudaStream_t s) {
    if (N == 0) return;
    k_lsq<<<grid(N), kBlock, 0, s>>>(N, cfs, cc, ccentre, minv);
    count_launch();
}

void launch_layout(const DevMesh& m, const uint32_t* cell_old, const uint32_t* face_old, const double* area,
                   const double* normal, const double* fcentre, const double* ccentre, const double* volume,
                   const double* minv, cudaStream_t s) {
    const int64_t NG = m.N + m.G;
    if (NG) { k_layout_cells<<<grid(NG), kBlock, 0, s>>>(NG, cell_old, ccentre, volume, m.cell_geo); count_launch(); }
    if (m.F) { k_layout_faces<<<grid(m.F), kBlock, 0, s>>>(m.F, face_old, area, normal, fcentre, m.face_geo); count_launch(); }
    if (m.N) { k_layout_lsq<<<grid(m.N), kBlock, 0, s>>>(m.N, cell_old, minv, m.lsq); count_launch(); }
}

}  // namespace gb
