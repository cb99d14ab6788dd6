// Headless driver for the reference solver (test infrastructure only).
//
// Built by oracle/Makefile.ref against the reference's own sources
// (src/mesh.cu, src/meshio.cu, src/flexarray.cu, src/fvmfields.cu,
// src/fvmfieldsio.cu, src/fvmops.cu, src/models/euler.cu) and run on a GPU
// box to produce the golden fixtures under tests/golden/.  It drives the
// reference only through its public entry points, in the order
// PhysicsEuler::setup/step use them (src/models/euler.cu:59-175):
//   cuMeshFromSu2 -> cuMeshFromFile -> FvmFieldNew x4 -> FvmEulerInit
//   per iteration: Fvm*Bc per region -> FvmEulerStepPrepare -> FvmEulerStep
//                  -> FvmFieldReduceSum (normalised by the iteration-0 value)
//
// The same source builds against the reference's float32 headers (as
// shipped, include/datatypes.cuh:32 defines FLOAT_PREC) and against a copy
// with that define removed (scalar = double); records of scalar arrays carry
// the matching dtype.
//
// usage: ref_driver <case.txt> <mesh.su2> <out.bin> <mode>
//   mode = metrics | prepare | solve
// case.txt lines (processed in file order):
//   init mx my mz p T
//   slip <region>
//   farfield <region> mx my mz p T
//   cfl <c>      iters <n>      tol <t>
//   state <file> (prepare mode: raw float32 rho[n], rhou[3n], rhoe[n], n = N+G)
// Output: a sequence of records {char name[64]; uint32 dtype(0=f32,1=u32,2=f64,3=u64);
// uint64 count; data}.
#include <chrono>
#include <string>
#include <vector>

#include "fvmops.cuh"
#include "fvmfields.cuh"
#include "meshio.cuh"
#include "models/euler.cuh"

namespace {

struct BcSpec {
    std::string type, region;
    vector mach;
    scalar p, T;
};

struct Case {
    vector mach = make_vector((scalar)0.5, (scalar)0, (scalar)0);
    scalar p = 1.f, T = 1.f / 1.4f, cfl = 0.8f, tol = 0.f;
    int iters = 100;
    std::string state;
    std::vector<BcSpec> bcs;
};

// reads n numbers into scalars whatever scalar is
bool read_scalars(FILE* f, int n, scalar** out) {
    for (int i = 0; i < n; ++i) {
        double v;
        if (fscanf(f, "%lf", &v) != 1) return false;
        *out[i] = (scalar)v;
    }
    return true;
}

constexpr uint32_t kScalarType = sizeof(scalar) == 8 ? 2 : 0;

Case read_case(const char* path) {
    Case c;
    FILE* f = fopen(path, "r");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    char key[128];
    while (fscanf(f, "%127s", key) == 1) {
        std::string k(key);
        if (k == "init") {
            scalar* v[5] = {&c.mach.x, &c.mach.y, &c.mach.z, &c.p, &c.T};
            if (!read_scalars(f, 5, v)) exit(2);
        } else if (k == "slip") {
            char r[128];
            if (fscanf(f, "%127s", r) != 1) exit(2);
            BcSpec b; b.type = "slip"; b.region = r; b.mach = make_vector((scalar)0, (scalar)0, (scalar)0); b.p = b.T = 0;
            c.bcs.push_back(b);
        } else if (k == "farfield") {
            char r[128];
            BcSpec b; b.type = "farfield";
            scalar* v[5] = {&b.mach.x, &b.mach.y, &b.mach.z, &b.p, &b.T};
            if (fscanf(f, "%127s", r) != 1 || !read_scalars(f, 5, v)) exit(2);
            b.region = r;
            c.bcs.push_back(b);
        } else if (k == "cfl") {
            scalar* v[1] = {&c.cfl};
            if (!read_scalars(f, 1, v)) exit(2);
        } else if (k == "iters") {
            if (fscanf(f, "%d", &c.iters) != 1) exit(2);
        } else if (k == "tol") {
            scalar* v[1] = {&c.tol};
            if (!read_scalars(f, 1, v)) exit(2);
        } else if (k == "state") {
            char s[512];
            if (fscanf(f, "%511s", s) != 1) exit(2);
            c.state = s;
        } else {
            fprintf(stderr, "unknown key %s\n", key);
            exit(2);
        }
    }
    fclose(f);
    return c;
}

void put(FILE* f, const char* name, uint32_t dtype, const void* data, uint64_t count) {
    char nm[64] = {0};
    strncpy(nm, name, 63);
    fwrite(nm, 1, 64, f);
    fwrite(&dtype, 4, 1, f);
    fwrite(&count, 8, 1, f);
    size_t es = dtype >= 2 ? 8 : 4;
    if (count) fwrite(data, es, count, f);
}

void apply_bcs(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, const Case& c) {
    for (const BcSpec& b : c.bcs) {
        if (b.type == "slip") {
            FvmEulerSlipBc(mesh, rho, rhou, rhoe, b.region.c_str());
        } else {
            FvmEulerInletOutletBc(mesh, rho, rhou, rhoe, b.mach, b.p, b.T, b.region.c_str());
        }
    }
}

void dump_field(FILE* out, FvmField* v, const char* name, size_t n, int comps) {
    VarAllGpuToCpu(v);
    std::string nm(name);
    put(out, (nm + ".value").c_str(), kScalarType, v->_cpu->value, (uint64_t)n * comps);
    put(out, (nm + ".gradient").c_str(), kScalarType, v->_cpu->gradient, (uint64_t)n * comps * 3);
    put(out, (nm + ".limiter").c_str(), kScalarType, v->_cpu->limiter, (uint64_t)n * comps);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: ref_driver <case.txt> <mesh.su2> <out.bin> <metrics|prepare|solve>\n");
        return 2;
    }
    Case c = read_case(argv[1]);
    std::string su2(argv[2]);
    std::string fvm = su2.substr(0, su2.size() - 3) + "fvm";
    std::string mode(argv[4]);

    auto t0 = std::chrono::steady_clock::now();
    if (cuMeshFromSu2(su2.c_str(), fvm.c_str())) {
        fprintf(stderr, "cuMeshFromSu2 failed\n");
        return 1;
    }
    cuMesh* mesh = cuMeshFromFile(fvm.c_str());
    cudaExec(cudaDeviceSynchronize());
    auto t1 = std::chrono::steady_clock::now();

    cuMeshBase* m = mesh->_cpu;
    const size_t N = m->n_cells, G = m->n_ghosts, NG = N + G, F = m->n_faces;
    FILE* out = fopen(argv[3], "wb");
    if (!out) { fprintf(stderr, "cannot open output\n"); return 2; }
    uint64_t sizes[5] = {N, G, F, m->n_nodes, m->n_regions};
    put(out, "sizes", 3, sizes, 5);
    double setup_s = std::chrono::duration<double>(t1 - t0).count();
    put(out, "setup_seconds", 2, &setup_s, 1);

    if (mode == "metrics") {
        put(out, "cell_faces_starts", 1, m->cell_faces_starts, NG + 1);
        put(out, "cell_faces", 1, m->cell_faces, m->cell_faces_starts[NG]);
        put(out, "cell_connects", 1, m->cell_connects, m->cell_faces_starts[NG]);
        put(out, "face_nodes_starts", 1, m->face_nodes_starts, F + 1);
        put(out, "face_nodes", 1, m->face_nodes, m->face_nodes_starts[F]);
        put(out, "ghost_cell_ids", 1, m->ghost_cell_ids, G);
        put(out, "ghost_cell_starts", 1, m->ghost_cell_starts, m->n_regions + 1);
        put(out, "nodes", kScalarType, m->nodes, m->n_nodes * 3);
        put(out, "face_areas", kScalarType, m->face_areas, F);
        put(out, "face_normals", kScalarType, m->face_normals, F * 3);
        put(out, "face_centers", kScalarType, m->face_centers, F * 3);
        put(out, "cell_volumes", kScalarType, m->cell_volumes, NG);
        put(out, "cell_centers", kScalarType, m->cell_centers, NG * 3);
        put(out, "cell_matrices", kScalarType, m->cell_matrices, N * 9);
        fclose(out);
        return 0;
    }

    FvmField* rho = FvmFieldNew(sizeof(scalar), NG, "rho", 1);
    FvmField* rhou = FvmFieldNew(sizeof(vector), NG, "rhou", 1);
    FvmField* rhoe = FvmFieldNew(sizeof(scalar), NG, "rhoe", 1);
    FvmField* error = FvmFieldNew(sizeof(scalar), NG, "error", 1);
    FvmEulerInit(mesh, rho, rhou, rhoe, c.mach, c.p, c.T);

    if (mode == "prepare") {
        if (!c.state.empty()) {
            std::vector<float> buf(NG * 5);
            FILE* sf = fopen(c.state.c_str(), "rb");
            if (!sf || fread(buf.data(), 4, NG * 5, sf) != NG * 5) { fprintf(stderr, "bad state file\n"); return 2; }
            fclose(sf);
            std::vector<scalar> sv(buf.begin(), buf.end());
            cudaExec(cudaMemcpy(rho->_hgpu->value, sv.data(), NG * sizeof(scalar), cudaMemcpyHostToDevice));
            cudaExec(cudaMemcpy(rhou->_hgpu->value, sv.data() + NG, NG * 3 * sizeof(scalar), cudaMemcpyHostToDevice));
            cudaExec(cudaMemcpy(rhoe->_hgpu->value, sv.data() + NG * 4, NG * sizeof(scalar), cudaMemcpyHostToDevice));
        }
        apply_bcs(mesh, rho, rhou, rhoe, c);
        FvmEulerStepPrepare(mesh, rho, rhou, rhoe);
        cudaExec(cudaDeviceSynchronize());
        dump_field(out, rho, "rho", NG, 1);
        dump_field(out, rhou, "rhou", NG, 3);
        dump_field(out, rhoe, "rhoe", NG, 1);
        fclose(out);
        return 0;
    }

    // solve: the PhysicsEuler::step loop with a steady residual.
    std::vector<double> hist;
    hist.reserve(c.iters);
    scalar err0 = 1.f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaExec(cudaDeviceSynchronize());
    auto w0 = std::chrono::steady_clock::now();
    cudaEventRecord(e0);
    int it = 0;
    for (; it < c.iters; ++it) {
        apply_bcs(mesh, rho, rhou, rhoe, c);
        FvmEulerStepPrepare(mesh, rho, rhou, rhoe);
        FvmEulerStep(mesh, rho, rhou, rhoe, c.cfl, "steady", NULL, error);
        scalar err = FvmFieldReduceSum(mesh, error);
        if (it == 0) err0 = err;
        hist.push_back((double)err);
        if (c.tol > 0 && err / err0 < c.tol) { ++it; break; }
    }
    cudaEventRecord(e1);
    cudaExec(cudaDeviceSynchronize());
    auto w1 = std::chrono::steady_clock::now();
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    double wall = std::chrono::duration<double>(w1 - w0).count();
    double iters_done = it;
    put(out, "iterations", 2, &iters_done, 1);
    put(out, "wall_seconds", 2, &wall, 1);
    double evs = ms * 1e-3;
    put(out, "event_seconds", 2, &evs, 1);
    put(out, "residual_history", 2, hist.data(), hist.size());
    dump_field(out, rho, "rho", NG, 1);
    dump_field(out, rhou, "rhou", NG, 3);
    dump_field(out, rhoe, "rhoe", NG, 1);
    VarGpuToCpu(error);
    put(out, "error.value", kScalarType, error->_cpu->value, NG);
    fclose(out);
    printf("ref_driver: %d iterations, %.3f s wall, %.3e cell-updates/s\n", it, wall,
           (double)N * it / wall);
    return 0;
}
