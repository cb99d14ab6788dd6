// Headless colour map of a scalar field on a boundary region: the data the
// reference's renderer puts in its OpenGL vertex buffer (RenderMesh built
// from a region, src/render/window.cu:560-627, coloured by
// KernelRenderScalarField, :682-756), written to a caller's buffer instead
// of a GL buffer.  Each face of the region is fanned into triangles (nodes
// 0, j+1, j+2); each triangle carries its ghost and interior cell; each
// vertex gets the value u + (grad u . (vertex - triangle centre)) lim, with
// u, grad u and lim averaged over the two cells (the ghost carries its
// interior cell's gradient and limiter), normalised to [u_min, u_max] and
// mapped blue -> cyan -> green/yellow -> red by the reference's five-segment
// map.  Output: 18 floats per triangle, (x, y, z, r, g, b) per vertex.
#include <vector>

#include "gb_device.cuh"
#include "gb_internal.h"

namespace gb {
namespace {

__device__ __forceinline__ float3 colour(float t) {
    if (t <= 0.2f) return make_float3(0.f, 0.f, 0.5f + t * 0.5f / 0.2f);
    if (t <= 0.4f) return make_float3(0.f, (t - 0.2f) / 0.2f, 1.f);
    if (t <= 0.6f) return make_float3((t - 0.4f) / 0.2f, 1.f, 1.f - (t - 0.4f) / 0.2f);
    if (t <= 0.8f) return make_float3(1.f, 1.f - (t - 0.6f) / 0.2f, 0.f);
    return make_float3(1.f - (t - 0.8f) * 0.5f / 0.2f, 0.f, 0.f);
}

// tri[9 t ..] vertex coordinates, cells[2 t ..] (ghost, interior)
__global__ void k_colour_triangles(int64_t n, const float* __restrict__ tri, const uint32_t* __restrict__ cells,
                                   const float* __restrict__ value, const float4* __restrict__ grad, float u_min,
                                   float u_max, float* out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t g = cells[2 * t], i = cells[2 * t + 1];
    const float u = 0.5f * (value[g] + value[i]);
    const float4 gl = grad ? grad[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    float c[3] = {0.f, 0.f, 0.f};
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) c[k] += tri[9 * t + 3 * v + k] / 3.0f;
    for (int v = 0; v < 3; ++v) {
        const float* p = tri + 9 * t + 3 * v;
        const float d = gl.x * (p[0] - c[0]) + gl.y * (p[1] - c[1]) + gl.z * (p[2] - c[2]);
        float uf = (u + d * gl.w - u_min) / (u_max - u_min);
        uf = fmaxf(0.f, fminf(1.f, uf));
        const float3 col = colour(uf);
        float* o = out + 18 * t + 6 * v;
        o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
        o[3] = col.x; o[4] = col.y; o[5] = col.z;
    }
}

bool ok_(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int64_t gbRenderRegionScalar(cuMesh* mesh, unsigned region_id, FvmField* field, gb_scalar u_min, gb_scalar u_max,
                             float* out, int64_t capacity_triangles) {
    clear_error();
    MeshAccess A;
    FieldAccess F;
    if (!mesh_access(mesh, &A) || !field_access(field, mesh, 1, &F)) return -1;
    if ((int)region_id >= A.n_regions) { set_error("gbRenderRegionScalar: unknown region"); return -1; }
    if (!(u_max > u_min)) { set_error("gbRenderRegionScalar: u_max must exceed u_min"); return -1; }
    const Topology& T = *A.topo;
    const Numbering& U = *A.num;
    std::vector<float> tri;
    std::vector<uint32_t> cells;
    for (uint32_t g = U.region_start[region_id]; g < U.region_start[region_id + 1]; ++g) {
        const uint32_t f = U.face_old[U.ghost_face[g - A.N]];
        const uint32_t b = T.fns[f], e = T.fns[f + 1];
        for (uint32_t j = b + 1; j + 1 < e; ++j) {
            for (uint32_t n : {b, j, j + 1})
                for (int k = 0; k < 3; ++k) tri.push_back((float)T.nodes[3 * (size_t)T.fn[n] + k]);
            cells.push_back(g);
            cells.push_back(U.ghost_cell[g - A.N]);
        }
    }
    const int64_t n = (int64_t)cells.size() / 2;
    if (!out) return n;
    if (capacity_triangles < n) { set_error("gbRenderRegionScalar: output holds fewer triangles than the region has"); return -1; }
    if (n == 0) return 0;
    cudaStream_t s = (cudaStream_t)gbGetStream();
    float *d_tri = nullptr, *d_out = nullptr;
    uint32_t* d_cells = nullptr;
    bool ok = ok_(cudaMalloc((void**)&d_tri, tri.size() * sizeof(float)), "gbRenderRegionScalar") &&
              ok_(cudaMalloc((void**)&d_cells, cells.size() * sizeof(uint32_t)), "gbRenderRegionScalar") &&
              ok_(cudaMalloc((void**)&d_out, (size_t)n * 18 * sizeof(float)), "gbRenderRegionScalar") &&
              ok_(cudaMemcpyAsync(d_tri, tri.data(), tri.size() * sizeof(float), cudaMemcpyHostToDevice, s),
                  "gbRenderRegionScalar") &&
              ok_(cudaMemcpyAsync(d_cells, cells.data(), cells.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
                  "gbRenderRegionScalar");
    if (ok) {
        k_colour_triangles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, d_tri, d_cells, (const float*)F.val[F.cur],
                                                                        F.grad, u_min, u_max, d_out);
        count_launch();
        ok = ok_(cudaGetLastError(), "gbRenderRegionScalar") &&
             ok_(cudaMemcpyAsync(out, d_out, (size_t)n * 18 * sizeof(float), cudaMemcpyDefault, s),
                 "gbRenderRegionScalar") &&
             ok_(cudaStreamSynchronize(s), "gbRenderRegionScalar");
    }
    for (void* p : {(void*)d_tri, (void*)d_out, (void*)d_cells})
        if (p) cudaFree(p);
    return ok ? n : -1;
}

}  // extern "C"
