// Headless harness for the reference's generic finite-volume operators
// (test infrastructure only).
//
// Built by oracle/Makefile.ref against the reference's own sources and run
// on a GPU box to produce tests/golden/*_fvmops.npz.  It reads a mesh with
// the reference's cuMeshFromSu2 / cuMeshFromFile, makes three fields with
// FvmFieldNew (a scalar s and a vector v with gradients, a vector phi),
// computes the gradients and limiters of s and v with the reference's own
// kernels in FvmEulerStepPrepare's order (ScalarVarComputeGradient,
// ScalarVarComputeLimiters, fvmScalGradLimBc; the Vector* ones for v;
// src/models/euler.cu:597-647), and evaluates every operator of
// include/fvmops.cuh:96-219 -- the reference's inline device functions
// themselves -- at every interior cell.
//
// usage: ref_fvmops <mesh.su2> <fields.bin> <out.bin> <phi_x> <phi_y> <phi_z>
//   fields.bin: raw float32 s[n], v[3n], phi[3n] in the reference's cell
//   order, n = cells + ghosts
// Output: records as oracle/ref_driver.cu writes them: "ops" (float32,
// 35 per interior cell: LaplacianC 1, ScalGradC 3, ScalGradCCorrect 3,
// VecGradC 9 (tensor columns u, v, w), BoundScalGradC 3, BoundVecGradC 9,
// DivC 1, ConvConstScalU 1, ConvConstScalU2 1, ConvScalU 1, ConvVecU 3),
// then s and v's gradient and limiter.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fvmfields.cuh"
#include "fvmops.cuh"
#include "meshio.cuh"

namespace {

constexpr int kOut = 35;

__device__ void put(scalar* o, const scalar& x) { o[0] = x; }
__device__ void put(scalar* o, const vector& x) { o[0] = x.x; o[1] = x.y; o[2] = x.z; }
__device__ void put(scalar* o, const tensor& x) { put(o, x.u); put(o + 3, x.v); put(o + 6, x.w); }

__global__ void k_ops(cuMeshBase* mesh, FvmFieldBase* s, FvmFieldBase* v, FvmFieldBase* phi, vector phi_c,
                      scalar* out) {
    const int c0 = cudaGlobalId;
    if (c0 >= (int)mesh->n_cells) return;
    scalar* o = out + (size_t)c0 * kOut;
    vector* ph = (vector*)phi->value;
    put(o + 0, fvmLaplacianC(mesh, c0, s));
    put(o + 1, fvmScalGradC(mesh, c0, s));
    put(o + 4, fvmScalGradCCorrect(mesh, c0, s));
    put(o + 7, fvmVecGradC(mesh, c0, v));
    put(o + 16, fvmBoundScalGradC(mesh, c0, s));
    put(o + 19, fvmBoundVecGradC(mesh, c0, v));
    put(o + 28, fvmDivC(mesh, c0, v));
    put(o + 29, fvmConvConstScalU(mesh, c0, s, phi_c));
    put(o + 30, fvmConvConstScalU2(mesh, c0, s, phi_c));
    put(o + 31, fvmConvScalU(mesh, c0, s, ph));
    put(o + 32, fvmConvVecU(mesh, c0, v, ph));
}

void record(FILE* f, const char* name, const void* data, uint64_t count) {
    char nm[64] = {0};
    strncpy(nm, name, 63);
    const uint32_t dtype = sizeof(scalar) == 8 ? 2 : 0;
    fwrite(nm, 1, 64, f);
    fwrite(&dtype, 4, 1, f);
    fwrite(&count, 8, 1, f);
    if (count) fwrite(data, sizeof(scalar), count, f);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 7) {
        fprintf(stderr, "usage: ref_fvmops <mesh.su2> <fields.bin> <out.bin> <phi_x> <phi_y> <phi_z>\n");
        return 2;
    }
    std::string su2(argv[1]);
    std::string fvm = su2.substr(0, su2.size() - 3) + "fvm";
    if (cuMeshFromSu2(su2.c_str(), fvm.c_str())) { fprintf(stderr, "cuMeshFromSu2 failed\n"); return 1; }
    cuMesh* mesh = cuMeshFromFile(fvm.c_str());
    const size_t N = mesh->_cpu->n_cells, G = mesh->_cpu->n_ghosts, n = N + G;
    std::vector<float> buf(7 * n);
    FILE* ff = fopen(argv[2], "rb");
    if (!ff || fread(buf.data(), 4, buf.size(), ff) != buf.size()) { fprintf(stderr, "bad fields file\n"); return 2; }
    fclose(ff);
    std::vector<scalar> sv(buf.begin(), buf.end());
    FvmField* s = FvmFieldNew(sizeof(scalar), n, "s", 1);
    FvmField* v = FvmFieldNew(sizeof(vector), n, "v", 1);
    FvmField* phi = FvmFieldNew(sizeof(vector), n, "phi", 0);
    cudaExec(cudaMemcpy(s->_hgpu->value, sv.data(), n * sizeof(scalar), cudaMemcpyHostToDevice));
    cudaExec(cudaMemcpy(v->_hgpu->value, sv.data() + n, 3 * n * sizeof(scalar), cudaMemcpyHostToDevice));
    cudaExec(cudaMemcpy(phi->_hgpu->value, sv.data() + 4 * n, 3 * n * sizeof(scalar), cudaMemcpyHostToDevice));
    const int n_c = cuda_size(N, CKW), n_g = cuda_size(G, CKW);
    ScalarVarComputeGradient<<<n_c, CKW>>>(kernelInput(mesh), kernelInput(s));
    ScalarVarComputeLimiters<<<n_c, CKW>>>(kernelInput(mesh), kernelInput(s));
    fvmScalGradLimBc<<<n_g, CKW>>>(kernelInput(mesh), kernelInput(s));
    VectorVarComputeGradient<<<n_c, CKW>>>(kernelInput(mesh), kernelInput(v));
    VectorVarComputeLimiters<<<n_c, CKW>>>(kernelInput(mesh), kernelInput(v));
    fvmVecGradLimBc<<<n_g, CKW>>>(kernelInput(mesh), kernelInput(v));
    scalar* d_out = nullptr;
    cudaExec(cudaMalloc(&d_out, N * kOut * sizeof(scalar)));
    const vector phi_c = make_vector((scalar)atof(argv[4]), (scalar)atof(argv[5]), (scalar)atof(argv[6]));
    k_ops<<<n_c, CKW>>>(kernelInput(mesh), kernelInput(s), kernelInput(v), kernelInput(phi), phi_c, d_out);
    cudaExec(cudaDeviceSynchronize());
    std::vector<scalar> out(N * kOut);
    cudaExec(cudaMemcpy(out.data(), d_out, out.size() * sizeof(scalar), cudaMemcpyDeviceToHost));
    VarAllGpuToCpu(s);
    VarAllGpuToCpu(v);
    FILE* f = fopen(argv[3], "wb");
    if (!f) { fprintf(stderr, "cannot open output\n"); return 2; }
    record(f, "ops", out.data(), out.size());
    record(f, "s.gradient", s->_cpu->gradient, 3 * n);
    record(f, "s.limiter", s->_cpu->limiter, n);
    record(f, "v.gradient", v->_cpu->gradient, 9 * n);
    record(f, "v.limiter", v->_cpu->limiter, 3 * n);
    fclose(f);
    printf("ref_fvmops: %zu cells, %zu ghosts\n", N, G);
    return 0;
}
