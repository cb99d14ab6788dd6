/*
 * A C caller of libgraphite_b200.so, compiled against include/graphite_b200.h
 * by tests/test_abi.py.
 *
 *   physics_euler layout
 *       prints "struct.field offset size" for every field of the header's
 *       structs and "struct sizeof N" for each struct (no GPU needed);
 *   physics_euler run <mesh.su2> <mesh.fvm> <iterations>
 *       runs the PhysicsEuler loop (src/models/euler.cu:12-175) on the
 *       channel-with-bump boundary regions through the reference's entry
 *       points, exactly as a reference caller would: cuMeshFromSu2,
 *       cuMeshFromFile, FvmFieldNew x4, FvmEulerInit, then per iteration the
 *       boundary conditions in PhysicsEuler's sorted-key order,
 *       FvmEulerStepPrepare, FvmEulerStep and FvmFieldReduceSum; prints
 *       "residual <i> <value>" per iteration and, after VarGpuToCpu, the
 *       interior density as "rho <i> <value>" lines; before the loop, the
 *       host mirror's faces, cells (faces:neighbours) and region ghost counts
 *       through the header's CSR helpers ("face", "cell", "region" lines).
 */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "graphite_b200.h"

#define FIELD(s, f) printf(#s "." #f " %zu %zu\n", offsetof(s, f), sizeof(((s*)0)->f))

static int layout(void) {
    FIELD(gb_vector, x); FIELD(gb_vector, y); FIELD(gb_vector, z);
    FIELD(gb_tensor, u); FIELD(gb_tensor, v); FIELD(gb_tensor, w);
    FIELD(cuMeshBase, type); FIELD(cuMeshBase, allocated); FIELD(cuMeshBase, n_cells);
    FIELD(cuMeshBase, n_faces); FIELD(cuMeshBase, n_nodes); FIELD(cuMeshBase, n_ghosts);
    FIELD(cuMeshBase, n_regions); FIELD(cuMeshBase, cell_faces); FIELD(cuMeshBase, cell_connects);
    FIELD(cuMeshBase, cell_faces_starts); FIELD(cuMeshBase, cell_volumes); FIELD(cuMeshBase, cell_centers);
    FIELD(cuMeshBase, cell_matrices); FIELD(cuMeshBase, face_nodes); FIELD(cuMeshBase, face_nodes_starts);
    FIELD(cuMeshBase, face_areas); FIELD(cuMeshBase, face_centers); FIELD(cuMeshBase, face_normals);
    FIELD(cuMeshBase, nodes); FIELD(cuMeshBase, ghost_cell_ids); FIELD(cuMeshBase, ghost_cell_starts);
    FIELD(cuMesh, _cpu); FIELD(cuMesh, _hgpu); FIELD(cuMesh, _gpu); FIELD(cuMesh, region_names);
    FIELD(cuMesh, region_names_alloc); FIELD(cuMesh, region_names_size); FIELD(cuMesh, impl);
    FIELD(FvmFieldBase, elem_size); FIELD(FvmFieldBase, size); FIELD(FvmFieldBase, value);
    FIELD(FvmFieldBase, gradient); FIELD(FvmFieldBase, limiter);
    FIELD(FvmField, _cpu); FIELD(FvmField, _hgpu); FIELD(FvmField, _gpu); FIELD(FvmField, name);
    FIELD(FvmField, impl);
    FIELD(gbBc, type); FIELD(gbBc, region_id); FIELD(gbBc, mach); FIELD(gbBc, pressure);
    FIELD(gbBc, temperature);
    FIELD(gbBatchInstance, mesh); FIELD(gbBatchInstance, n_bc); FIELD(gbBatchInstance, bcs);
    FIELD(gbFvmTerm, op); FIELD(gbFvmTerm, coef); FIELD(gbFvmTerm, u); FIELD(gbFvmTerm, phi);
    FIELD(gbFvmTerm, phi_const);
    printf("gb_vector sizeof %zu\n", sizeof(gb_vector));
    printf("gb_tensor sizeof %zu\n", sizeof(gb_tensor));
    printf("cuMeshBase sizeof %zu\n", sizeof(cuMeshBase));
    printf("cuMesh sizeof %zu\n", sizeof(cuMesh));
    printf("FvmFieldBase sizeof %zu\n", sizeof(FvmFieldBase));
    printf("FvmField sizeof %zu\n", sizeof(FvmField));
    printf("gbBc sizeof %zu\n", sizeof(gbBc));
    printf("gbBatchInstance sizeof %zu\n", sizeof(gbBatchInstance));
    printf("gbFvmTerm sizeof %zu\n", sizeof(gbFvmTerm));
    return 0;
}

#define CHECK(call)                                                            \
    do {                                                                       \
        if ((call) != 0) {                                                     \
            fprintf(stderr, "%s failed: %s\n", #call, gbGetLastError());       \
            return 1;                                                          \
        }                                                                      \
    } while (0)

static int run(const char* su2, const char* fvm, int iterations) {
    const gb_scalar p = 1.f, t = 1.f / 1.4f;
    const gb_vector mach = {0.5f, 0.f, 0.f};
    CHECK(cuMeshFromSu2(su2, fvm));
    cuMesh* mesh = cuMeshFromFile(fvm);
    if (!mesh) { fprintf(stderr, "cuMeshFromFile: %s\n", gbGetLastError()); return 1; }
    const size_t n = cuMeshGetVarSize(mesh);
    /* the host mirror through the header's CSR helpers */
    cuMeshBase* hb = mesh->_cpu;
    for (int i = 0; i < (int)hb->n_faces; ++i) {
        printf("face %d %u", i, cuMeshGetFaceSize(hb, i));
        for (const unsigned int* q = cuMeshGetFaceStart(hb, i); q != cuMeshGetFaceEnd(hb, i); ++q) printf(" %u", *q);
        printf("\n");
    }
    for (int i = 0; i < (int)n; ++i) {
        printf("cell %d %u", i, cuMeshGetCellSize(hb, i));
        const unsigned int* c = cuMeshGetCellConnect(hb, i);
        for (const unsigned int* q = cuMeshGetCellStart(hb, i); q != cuMeshGetCellEnd(hb, i); ++q, ++c)
            printf(" %u:%u", *q, *c);
        if (i >= (int)hb->n_cells) printf(" ghostface %u", cuMeshGetGhostCellFace(hb, i));
        printf("\n");
    }
    for (unsigned int r = 0; r < (unsigned int)hb->n_regions; ++r) printf("region %u %u\n", r, cuMeshGetRegionSize(hb, r));
    FvmField* rho = FvmFieldNew(sizeof(gb_scalar), n, "rho", 1);
    FvmField* rhou = FvmFieldNew(sizeof(gb_vector), n, "rhou", 1);
    FvmField* rhoe = FvmFieldNew(sizeof(gb_scalar), n, "rhoe", 1);
    FvmField* error = FvmFieldNew(sizeof(gb_scalar), n, "error", 1);
    if (!rho || !rhou || !rhoe || !error) { fprintf(stderr, "FvmFieldNew: %s\n", gbGetLastError()); return 1; }
    CHECK(FvmEulerInit(mesh, rho, rhou, rhoe, mach, p, t));
    for (int it = 0; it < iterations; ++it) {
        /* the "bcs" object of a channel case, in PhysicsEuler's key order */
        CHECK(FvmEulerInletOutletBc(mesh, rho, rhou, rhoe, mach, p, t, "inlet"));
        CHECK(FvmEulerSlipBc(mesh, rho, rhou, rhoe, "lower"));
        CHECK(FvmEulerInletOutletBc(mesh, rho, rhou, rhoe, mach, p, t, "outlet"));
        CHECK(FvmEulerSlipBc(mesh, rho, rhou, rhoe, "sides"));
        CHECK(FvmEulerSlipBc(mesh, rho, rhou, rhoe, "upper"));
        CHECK(FvmEulerStepPrepare(mesh, rho, rhou, rhoe));
        CHECK(FvmEulerStep(mesh, rho, rhou, rhoe, 0.8f, "steady", NULL, error));
        const gb_scalar r = FvmFieldReduceSum(mesh, error);
        if (r != r) { fprintf(stderr, "FvmFieldReduceSum: %s\n", gbGetLastError()); return 1; }
        printf("residual %d %.9g\n", it, (double)r);
    }
    VarAllGpuToCpu(rho);
    if (gbGetLastError()[0]) { fprintf(stderr, "VarAllGpuToCpu: %s\n", gbGetLastError()); return 1; }
    const float* v = (const float*)rho->_cpu->value;
    for (size_t i = 0; i < mesh->_cpu->n_cells; ++i) printf("rho %zu %.9g\n", i, (double)v[i]);
    FvmFieldFree(rho); FvmFieldFree(rhou); FvmFieldFree(rhoe); FvmFieldFree(error);
    cuMeshFree(mesh);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 2 && strcmp(argv[1], "layout") == 0) return layout();
    if (argc >= 5 && strcmp(argv[1], "run") == 0) return run(argv[2], argv[3], atoi(argv[4]));
    fprintf(stderr, "usage: %s layout | run <mesh.su2> <mesh.fvm> <iterations>\n", argv[0]);
    return 2;
}
