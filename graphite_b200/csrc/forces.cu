// Pressure force on a boundary region (lift / drag): F = sum over the
// region's faces of p * A * n, with n the face normal pointing out of the
// fluid (from the interior cell towards its ghost) and p the pressure
// 0.4 (rho E - |rho u|^2 / (2 rho)) of the interior cell -- the slip
// condition mirrors the interior pressure into the ghost, so this is also
// the face pressure of the scheme.  Accumulated in float64 in a fixed order
// (block partials, then one block over the partials), so the result is
// deterministic.  No counterpart in the reference (its Euler model reports
// residuals only).
#include <vector>

#include "gb_device.cuh"
#include "gb_internal.h"

namespace gb {
namespace {

constexpr int kForceBlock = 256;

__global__ void k_force_partials(const uint2* __restrict__ ghost, uint32_t g0, uint32_t g1,
                                 const float4* __restrict__ cell_geo, const float4* __restrict__ face_geo, const float* __restrict__ rho,
                                 const float4* __restrict__ rhou, const float* __restrict__ rhoe, double* partials) {
    __shared__ double red[3][kForceBlock];
    const uint32_t g = g0 + blockIdx.x * kForceBlock + threadIdx.x;
    double f[3] = {0.0, 0.0, 0.0};
    if (g < g1) {
        const uint2 gi = ghost[g];                 // (interior cell, face)
        const uint32_t i = gi.x;
        const float4 nA = face_geo[2 * (size_t)gi.y];
        const float4 fc = face_geo[2 * (size_t)gi.y + 1];
        const float4 cc = cell_geo[i];
        // the stored normal's sign is arbitrary: orient it away from the cell
        const float dn = nA.x * (fc.x - cc.x) + nA.y * (fc.y - cc.y) + nA.z * (fc.z - cc.z);
        const double sA = dn >= 0.f ? (double)nA.w : -(double)nA.w;
        const double r = rho[i];
        const float4 ru = rhou[i];
        const double ke = 0.5 * ((double)ru.x * ru.x + (double)ru.y * ru.y + (double)ru.z * ru.z) / r;
        const double p = 0.4 * ((double)rhoe[i] - ke);
        f[0] = p * sA * nA.x;
        f[1] = p * sA * nA.y;
        f[2] = p * sA * nA.z;
    }
    for (int k = 0; k < 3; ++k) red[k][threadIdx.x] = f[k];
    __syncthreads();
    for (int s = kForceBlock / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 3) partials[3 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_force_final(const double* __restrict__ partials, int n, double* out) {
    if (threadIdx.x >= 3) return;
    double s = 0.0;
    for (int b = 0; b < n; ++b) s += partials[3 * b + threadIdx.x];
    out[threadIdx.x] = s;
}

bool ok_(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

}  // namespace

// force on region `region` of a mesh from a state in device order
bool wall_force(const MeshAccess& A, unsigned region, const float* rho, const float4* rhou, const float* rhoe,
                double* force, const char* what) {
    if ((int)region >= A.n_regions) { set_error(std::string(what) + ": unknown region"); return false; }
    const uint32_t g0 = A.region_start[region] - (uint32_t)A.N;
    const uint32_t g1 = A.region_start[region + 1] - (uint32_t)A.N;
    const int blocks = (int)((g1 - g0 + kForceBlock - 1) / kForceBlock);
    cudaStream_t s = (cudaStream_t)gbGetStream();
    if (blocks == 0) {
        force[0] = force[1] = force[2] = 0.0;
        return true;
    }
    double* d = nullptr;
    if (!ok_(cudaMalloc((void**)&d, (3 * (size_t)blocks + 3) * sizeof(double)), what)) return false;
    k_force_partials<<<blocks, kForceBlock, 0, s>>>(A.dev->ghost, g0, g1, A.dev->cell_geo, A.dev->face_geo, rho, rhou, rhoe, d);
    k_force_final<<<1, 32, 0, s>>>(d, blocks, d + 3 * blocks);
    count_launch(2);
    const bool ok = ok_(cudaGetLastError(), what) &&
                    ok_(cudaMemcpyAsync(force, d + 3 * blocks, 3 * sizeof(double), cudaMemcpyDeviceToHost, s), what) &&
                    ok_(cudaStreamSynchronize(s), what);
    cudaFree(d);
    return ok;
}

}  // namespace gb

using namespace gb;

extern "C" {

int gbWallForce(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, unsigned region_id, double* force) {
    clear_error();
    MeshAccess A;
    FieldAccess a, b, c;
    if (!force) { set_error("gbWallForce: null output"); return 1; }
    if (!mesh_access(mesh, &A) || !field_access(rho, mesh, 1, &a) || !field_access(rhou, mesh, 3, &b) ||
        !field_access(rhoe, mesh, 1, &c))
        return 1;
    return wall_force(A, region_id, (const float*)a.val[a.cur], (const float4*)b.val[b.cur],
                      (const float*)c.val[c.cur], force, "gbWallForce")
               ? 0
               : 1;
}

int gbBatchWallForce(gbBatch* batch, int instance, unsigned region_id, double* force) {
    clear_error();
    BatchInstanceAccess bi;
    MeshAccess A;
    if (!force) { set_error("gbBatchWallForce: null output"); return 1; }
    if (!batch_instance(batch, instance, &bi) || !mesh_access(bi.mesh, &A)) return 1;
    return wall_force(A, region_id, bi.rho[bi.cur], bi.rhou[bi.cur], bi.rhoe[bi.cur], force, "gbBatchWallForce") ? 0
                                                                                                               : 1;
}

}  // extern "C"
