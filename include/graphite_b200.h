/*
 * graphite_b200.h -- C ABI of libgraphite_b200.so, a B200 (sm_100a)
 * implementation of the explicit second-order unstructured finite-volume
 * Euler iteration of Alexsimulation/graphite.
 *
 * The entry points keep the names, argument meaning and call order of the
 * reference's mesh, field and FvmEuler* functions (the surface apps/main.cu
 * drives through PhysicsEuler), with C linkage so that any FFI can bind them:
 *
 *   cuMeshFromSu2 -> cuMeshFromFile -> FvmFieldNew x4 -> FvmEulerInit
 *   per iteration: FvmEulerSlipBc / FvmEulerInletOutletBc per region
 *                  -> FvmEulerStepPrepare -> FvmEulerStep -> FvmFieldReduceSum
 *   at the end:    VarAllGpuToCpu, FieldsWriteVtu
 *
 * Differences a caller can see, all deliberate:
 *   - errors are returned (nonzero int, NULL pointer or NaN) with a message in
 *     gbGetLastError(), where the reference prints and exit()s;
 *   - C has no references, so `const vector&` / `const scalar&` arguments are
 *     passed by value (gb_vector is layout-compatible with CUDA's float3);
 *   - the device layout is private: cuMesh._hgpu/_gpu and FvmField._hgpu/_gpu
 *     are NULL.  The host mirrors (_cpu) keep the reference's layout and the
 *     reference's cell order, so code that reads mesh->_cpu or field->_cpu
 *     after VarGpuToCpu sees what the reference would show;
 *   - FvmEulerStep updates the state as a Jacobi sweep (every cell reads the
 *     old state); the reference updates in place while neighbours read, a
 *     race with the same fixed point.
 *   - everything runs on the stream set with gbSetStream (default: the
 *     legacy default stream, as in the reference).
 *
 * Additions that have no reference counterpart carry the gb prefix.
 */
#ifndef GRAPHITE_B200_H
#define GRAPHITE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/datatypes.cuh:36-47 (FLOAT_PREC build): scalar = float,
 * vector = float3, tensor = three float3 columns (include/datatypes.cuh:52-54). */
typedef float gb_scalar;
typedef struct gb_vector { float x, y, z; } gb_vector;
typedef struct gb_tensor { gb_vector u, v, w; } gb_tensor;

/* include/mesh.cuh:12-16 */
typedef enum CUMESH_t { _CPU, _HGPU, _GPU } CUMESH_t;

/* Host mirror of a mesh, field for field as include/mesh.cuh:18-52, in the
 * reference's cell order (elements in file order, then one ghost cell per
 * boundary face, grouped by region).  Metrics are the float32 rounding of
 * float64 values computed on the device. */
typedef struct cuMeshBase {
    CUMESH_t type;
    int allocated;
    size_t n_cells, n_faces, n_nodes, n_ghosts, n_regions;
    unsigned int* cell_faces;
    unsigned int* cell_connects;
    unsigned int* cell_faces_starts;
    gb_scalar* cell_volumes;
    gb_vector* cell_centers;
    gb_tensor* cell_matrices;
    unsigned int* face_nodes;
    unsigned int* face_nodes_starts;
    gb_scalar* face_areas;
    gb_vector* face_centers;
    gb_vector* face_normals;
    gb_vector* nodes;
    unsigned int* ghost_cell_ids;
    unsigned int* ghost_cell_starts;
} cuMeshBase;

/* include/mesh.cuh:55-63, plus a private pointer to the device mesh. */
typedef struct cuMesh {
    cuMeshBase* _cpu;
    cuMeshBase* _hgpu; /* NULL: the device layout is private */
    cuMeshBase* _gpu;  /* NULL */
    char** region_names;
    size_t region_names_alloc;
    size_t region_names_size;
    void* impl;
} cuMesh;

/* include/fvmfields.cuh:8-13 */
typedef enum FvmFieldType { SCALAR, VECTOR, TENSOR, FIELD_UNKNOWN } FvmFieldType;

/* include/fvmfields.cuh:16-22: value[size], gradient[3*size] and
 * limiter[size] in element units (vector fields: gradient is a tensor whose
 * columns are the gradients of x, y and z). */
typedef struct FvmFieldBase {
    size_t elem_size;
    size_t size;
    void* value;
    void* gradient;
    void* limiter;
} FvmFieldBase;

/* include/fvmfields.cuh:25-30, plus a private pointer to the device field. */
typedef struct FvmField {
    FvmFieldBase* _cpu;
    FvmFieldBase* _hgpu; /* NULL: the device layout is private */
    FvmFieldBase* _gpu;  /* NULL */
    char* name;
    void* impl;
} FvmField;

/* ---------------------------------------------------------------- mesh --- */

/* Converts an SU2 text mesh (3-D; element kinds 10 tet, 12 hex, 13 prism,
 * 14 pyramid; boundary kinds 5 triangle, 9 quad) to the binary .fvm format.
 * Replaces cuMeshFromSu2, src/meshio.cu:817-1250 (same file layout; same
 * cell, ghost and per-cell face order; faces are numbered in order of first
 * appearance instead of hash-bucket order).  Returns 0 on success. */
int cuMeshFromSu2(const char* su2_filename, const char* out_filename);

/* Reads a .fvm mesh, renumbers cells (reverse Cuthill-McKee) and faces for
 * locality, computes the metrics in float64 on the device and fills the host
 * mirror.  Replaces cuMeshFromFile, src/meshio.cu:166-292 (and the metric
 * kernels src/mesh.cu:44-219 it launches).  NULL on error. */
cuMesh* cuMeshFromFile(const char* filename);

/* Frees host and device memory.  Replaces cuMeshFree, src/mesh.cu:401-411. */
void cuMeshFree(cuMesh* mesh);

/* Size queries, src/mesh.cu:5-31. */
size_t cuMeshGetVarSize(cuMesh* mesh);          /* cells + ghosts */
size_t cuMeshGetnCells(cuMesh* mesh);
size_t cuMeshGetnGhosts(cuMesh* mesh);
size_t cuMeshGetnCellsAndGhosts(cuMesh* mesh);
size_t cuMeshGetnRegionCells(cuMesh* mesh, unsigned int region_id);

/* Region index by name, src/mesh.cu:17-23.  The reference prints and returns
 * 0 for an unknown name; this returns UINT32_MAX and sets the last error. */
unsigned int cuMeshGetRegionId(cuMesh* mesh, const char* name);

/* Prints the mesh sizes, src/meshio.cu:8-21. */
void cuMeshPrintInfo(cuMesh* mesh);

/* CSR views of a host mirror (mesh->_cpu, reference order), the reference's
 * inline helpers include/mesh.cuh:83-141: the nodes of face i; the faces of
 * cell i and, in the same pattern, the cells across them (a ghost cell has
 * one face, its boundary face); the ghost count of region r. */
static inline unsigned int* cuMeshGetFaceStart(cuMeshBase* m, int i) { return m->face_nodes + m->face_nodes_starts[i]; }
static inline unsigned int* cuMeshGetFaceEnd(cuMeshBase* m, int i) { return m->face_nodes + m->face_nodes_starts[i + 1]; }
static inline unsigned int cuMeshGetFaceSize(cuMeshBase* m, int i) {
    return m->face_nodes_starts[i + 1] - m->face_nodes_starts[i];
}
static inline unsigned int* cuMeshGetCellStart(cuMeshBase* m, int i) { return m->cell_faces + m->cell_faces_starts[i]; }
static inline unsigned int* cuMeshGetCellEnd(cuMeshBase* m, int i) { return m->cell_faces + m->cell_faces_starts[i + 1]; }
static inline unsigned int cuMeshGetCellSize(cuMeshBase* m, int i) {
    return m->cell_faces_starts[i + 1] - m->cell_faces_starts[i];
}
static inline unsigned int* cuMeshGetCellConnect(cuMeshBase* m, int i) {
    return m->cell_connects + m->cell_faces_starts[i];
}
static inline unsigned int cuMeshGetGhostCellFace(cuMeshBase* m, int i) { return m->cell_faces[m->cell_faces_starts[i]]; }
static inline unsigned int cuMeshGetRegionSize(cuMeshBase* m, unsigned int r) {
    return m->ghost_cell_starts[r + 1] - m->ghost_cell_starts[r];
}

/* -------------------------------------------------------------- fields --- */

/* A field of `size` elements of `elem_size` bytes (sizeof(gb_scalar) or
 * sizeof(gb_vector)), with gradient and limiter storage when alloc_grads is
 * nonzero.  Replaces FvmFieldNew, src/fvmfields.cu:7-46.  The device storage
 * takes the mesh's cell order the first time the field is used with a mesh.
 * NULL on error. */
FvmField* FvmFieldNew(size_t elem_size, size_t size, const char* name, int alloc_grads);

/* src/fvmfields.cu:49-64 */
void FvmFieldFree(FvmField* v);

/* src/fvmfields.cu:67-83 */
FvmFieldType FvmFieldGetType(const FvmField* v);
void* FvmFieldValueIndex(FvmField* v, size_t i);

/* Copies the values (VarGpuToCpu) or values, gradients and limiters
 * (VarAllGpuToCpu) to field->_cpu in the reference's layout and cell order.
 * Ghost gradients/limiters are those of the ghost's interior cell, as the
 * reference's fvmScalGradLimBc/fvmVecGradLimBc leave them.  Synchronises the
 * stream.  src/fvmfields.cu:85-101. */
void VarGpuToCpu(FvmField* var);
void VarAllGpuToCpu(FvmField* var);

/* ----------------------------------------------------------- euler ops --- */

/* Uniform state from Mach vector, pressure and temperature in cells and
 * ghosts (gamma = 1.4, R = 1).  src/models/euler.cu:385-409, 529-549. */
int FvmEulerInit(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                 gb_scalar pressure, gb_scalar temperature);

/* Slip wall on a region's ghosts: mirrored momentum, copied density and
 * energy.  src/models/euler.cu:412-442, 552-568.  Recorded and applied with
 * the other conditions by the next call that uses the fields on the device
 * (see gbApplyBoundaryConditions); an unknown region is an error at once. */
int FvmEulerSlipBc(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, const char* region);

/* Far-field ghosts (sub/supersonic inflow/outflow from the interior Mach
 * number and the sign of u.n).  src/models/euler.cu:446-520, 571-593.
 * Recorded like FvmEulerSlipBc. */
int FvmEulerInletOutletBc(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                          gb_scalar pressure, gb_scalar temperature, const char* region);

/* Least-squares gradients and limiters of rho, rhou, rhoe (one fused kernel).
 * src/models/euler.cu:597-647 (9 kernels there). */
int FvmEulerStepPrepare(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe);

/* One local-time-step explicit update: reconstruction, central flux with
 * scalar dissipation, dt = cfl / sum(eig * A / V), and the squared residual
 * (F_rho^2 + |F_rhou|^2 + F_rhoE^2) * V into `error` (one fused kernel).
 * time_scheme must be "steady"; dt is unused (NULL), as in the reference.
 * src/models/euler.cu:236-381, 649-673. */
int FvmEulerStep(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_scalar cfl,
                 const char* time_scheme, FvmField* dt, FvmField* error);

/* Sum of a scalar field over the interior cells, accumulated in float64 on
 * the device in a fixed order (the result is deterministic) and returned
 * rounded to float.  Replaces FvmFieldReduceSum, src/fvmops.cu:369-383, which
 * copies the field to the host and sums it serially in float.  NaN on error. */
gb_scalar FvmFieldReduceSum(cuMesh* mesh, FvmField* var);

/* ----------------------------------------------------------- additions --- */

/* Message of the last error on this thread ("" if none). */
const char* gbGetLastError(void);

/* Stream for all subsequent work of this library on this thread (a
 * cudaStream_t; NULL = legacy default stream). */
int gbSetStream(void* stream);
void* gbGetStream(void);

/* Copies field->_cpu->value (reference layout and order) to the device; the
 * reverse of VarGpuToCpu, which the reference does not have.  Needs a field
 * already bound to `mesh`'s cell order (used with the mesh once) or binds
 * it now. */
int gbVarCpuToGpu(cuMesh* mesh, FvmField* var);

/* Momentum reconstruction: 1 (default) reproduces the reference, which
 * reconstructs rhou with the transposed gradient (dot(tensor, d) is a column
 * combination, include/datatypes.cuh:296-302, used at
 * src/models/euler.cu:252-253); 0 uses the consistent gradient. */
int gbSetReferenceMomentumReconstruction(int enabled);

/* Cell renumbering applied by cuMeshFromFile / gbMeshFromSu2: 1 (default)
 * reverse Cuthill-McKee, 0 keeps the file order. */
int gbSetRenumbering(int enabled);

/* Loads an SU2 mesh directly (no .fvm round trip; node coordinates stay
 * float64).  NULL on error. */
cuMesh* gbMeshFromSu2(const char* su2_filename);

/* Boundary condition for gbEulerRun: type 0 slip, 1 far field (mach,
 * pressure, temperature used). */
typedef struct gbBc {
    int type;
    unsigned int region_id;
    gb_vector mach;
    gb_scalar pressure;
    gb_scalar temperature;
} gbBc;

/* FvmEulerSlipBc and FvmEulerInletOutletBc record their condition and return;
 * all recorded conditions are applied together, in one kernel, by the next
 * call that reads or writes the fields on the device (FvmEulerStepPrepare in
 * the reference's loop, VarGpuToCpu, gbVarCpuToGpu, ...), with the results
 * of applying each at once (each ghost's state depends only on its interior
 * cell's; a later condition on a region replaces an earlier one).  This
 * applies them now.  Returns 0, or nonzero on error. */
int gbApplyBoundaryConditions(cuMesh* mesh);

/* Runs n_iter iterations of the PhysicsEuler::step loop (boundary conditions
 * in the given order, prepare, step, residual sum) as a replayed CUDA graph,
 * writing the residual sum of each iteration to residual_history (host
 * array of n_iter doubles, may be NULL).  With tolerance > 0 it stops after
 * the first iteration in which residual/residual[0] < tolerance: the device
 * stops iterating there, although the host looks only every check_every
 * iterations (the iterations left in that chunk do nothing).  A residual
 * that is not finite stops it too, and the call returns -1 with "not finite"
 * in gbGetLastError().  Returns the number of iterations run, or -1 on
 * error.
 * The results, ghost values included, are bitwise those of the per-call
 * loop (FvmEuler*Bc, FvmEulerStepPrepare, FvmEulerStep, FvmFieldReduceSum);
 * where a region appears twice in bcs the later condition holds, and the
 * gradients and limiters of the fields are not stored (the per-call
 * FvmEulerStepPrepare stores them).  Inside, all conditions are applied by
 * one ghost kernel, or, when the ghosts number at least a quarter of the
 * cells, by the gradient kernel itself. */
int64_t gbEulerRun(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, FvmField* error,
                   gb_scalar cfl, int64_t n_iter, const gbBc* bcs, int n_bc, double tolerance,
                   int check_every, double* residual_history);

/* gbEulerRun that also writes, per iteration, the density part of the
 * residual, sum over cells of F_rho^2 V (float64, fixed order), to
 * density_history (host array of n_iter doubles; its square root relative
 * to the first is the density residual's L2 drop).  The iterates, the
 * residual history and the stop test are gbEulerRun's. */
int64_t gbEulerRunDensityResidual(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, FvmField* error,
                                  gb_scalar cfl, int64_t n_iter, const gbBc* bcs, int n_bc, double tolerance,
                                  int check_every, double* residual_history, double* density_history);

/* Launches of this library's kernels since load (for accounting). */
uint64_t gbKernelLaunchCount(void);

/* ------------------------------------------------ batched instances --- */

/* Many instances (mesh, boundary conditions) advanced together: each
 * iteration is four persistent kernels over all active instances (ghosts,
 * gradients + limiters, flux + update, per-instance residual and
 * convergence), replayed as a CUDA graph.  An instance stops updating (is
 * frozen) when its residual ratio drops below the tolerance.  Each instance
 * computes exactly what a plain solve of it computes.  No counterpart in the
 * reference. */
typedef struct gbBatchImpl gbBatch;

typedef struct gbBatchInstance {
    int mesh;            /* index into the meshes passed to gbBatchCreate */
    int n_bc;
    const gbBc* bcs;     /* as for gbEulerRun (region ids of that mesh) */
} gbBatchInstance;

gbBatch* gbBatchCreate(int n_meshes, cuMesh* const* meshes, int n_instances, const gbBatchInstance* instances);
void gbBatchFree(gbBatch* batch);

/* Uniform free-stream state (euler_init) for one instance. */
int gbBatchInitUniform(gbBatch* batch, int instance, gb_vector mach, gb_scalar pressure, gb_scalar temperature);

/* Instance state from / to host arrays in the reference's layout and cell
 * order: rho[n], rhou[3n], rhoe[n] with n = cells + ghosts of its mesh. */
int gbBatchSetState(gbBatch* batch, int instance, const float* rho, const float* rhou, const float* rhoe);
int gbBatchGetState(gbBatch* batch, int instance, float* rho, float* rhou, float* rhoe);

/* Work decomposition: cells per work item (multiple of 256) and schedule =
 * order + 2 * kernel variant (schedule 0..9); order 0 runs instance by
 * instance, 1 tile by tile across the instances of a mesh; variant 0 / 1
 * compiles the gradient and flux kernels for 4 / 5 resident 256-thread blocks
 * per SM, variant 2 runs the gradient pass in 64-thread blocks that stage
 * each cell's face entries in shared memory (flux as variant 1), variants 3
 * and 4 are one persistent cooperative kernel per check_every iterations
 * (the three phases of an iteration separated by grid-wide barriers), with 4
 * or 3 resident 256-thread blocks per SM; a barrier wait that gives up,
 * after a few seconds, fails the run with an error. */
int gbBatchSetTuning(gbBatch* batch, int tile_cells, int schedule);
int gbBatchGetTuning(gbBatch* batch, int* tile_cells, int* schedule);

/* Test hook for failure detection: the next persistent launch of this batch
 * (schedule variants 3 and 4) starts with its grid barrier in a state no block
 * can complete, and with a short wait bound, so every block's wait gives up
 * and the run returns an error instead of hanging; the launch after it runs
 * normally. */
int gbBatchInjectBarrierFault(gbBatch* batch);

/* Times trial_iters iterations of every (tile, schedule) candidate from the
 * current states (restored afterwards), then the 4 fastest again over
 * 4 x trial_iters, and keeps the fastest of those; results are cached per
 * (mesh sizes, instances per mesh) for the process. */
int gbBatchAutotune(gbBatch* batch, gb_scalar cfl, int trial_iters, int* tile_cells, int* schedule);

/* Runs until every instance has converged (residual / first residual <
 * tolerance), hit max_iter, or produced a non-finite residual; polls every
 * check_every iterations.  Per-instance outputs (arrays of n_instances, may
 * be NULL): iterations, final residual ratio, status (1 converged, 2
 * iteration cap, 3 not finite); history (n_instances x max_iter doubles, may
 * be NULL) receives the residual sums.  Returns the iterations of the loop,
 * or -1 on error. */
int64_t gbBatchRun(gbBatch* batch, gb_scalar cfl, int64_t max_iter, double tolerance, int check_every,
                   int64_t* iterations, double* ratios, int* status, double* history);

/* Divide instance `instance`'s residuals by res0 instead of by its first
 * residual (0 restores the default).  A warm-started instance given the first
 * residual of its cold start converges to the same absolute level as the cold
 * start does.  No counterpart in the reference. */
int gbBatchSetResidualScale(gbBatch* batch, int instance, double res0);

/* ---- Learned warm start (no counterpart in the reference) ----
 * A per-cell MLP (inputs: centroid x, y, z, wall distance, Mach, sin AoA,
 * cos AoA, 1; three SiLU layers of 128; outputs rho, rho u, rho v, rho w,
 * rho E) trained on converged fields of one mesh and used to predict the
 * initial state of new cases.  The angle of attack is taken in the x-z plane
 * (mach = M (cos a, 0, sin a)).  Weights are 36864 floats in the order
 * W1[128][16] (inputs 8..15 are zero padding), W2[128][128], W3[128][128],
 * W4[16][128] (outputs 5..15 are padding); layer k computes
 * z = W_k a_{k-1}. */
typedef struct gbWarmStartImpl gbWarmStart;

/* mesh may be NULL (then only gbWarmStartGradient / gbWarmStartForward and
 * the weight calls work); wall_region = cuMeshGetRegionId of the wall. */
gbWarmStart* gbWarmStartCreate(cuMesh* mesh, unsigned wall_region, uint64_t seed);
void gbWarmStartFree(gbWarmStart* ws);
int64_t gbWarmStartParamCount(void);
int gbWarmStartGetWeights(gbWarmStart* ws, float* weights);
int gbWarmStartSetWeights(gbWarmStart* ws, const float* weights);
/* geometry[4] = wall centre xyz and extent L of the input map
 * u -> u / sqrt(1 + u^2), u = offset / L; target[5] = output scales s
 * (prediction = free stream + s * output). */
int gbWarmStartGetScales(gbWarmStart* ws, float* geometry, float* target);
int gbWarmStartSetScales(gbWarmStart* ws, const float* target);
/* Mapped geometry inputs (x', y', z', wall distance') per interior cell,
 * reference cell order: geo[4 n]. */
int gbWarmStartGetFeatures(gbWarmStart* ws, float* geo);
/* Adds a converged field as training data: the current state of a batch
 * instance on the same mesh, or three fields. */
int gbWarmStartAddBatchField(gbWarmStart* ws, gbBatch* batch, int instance, gb_vector mach, gb_scalar pressure,
                             gb_scalar temperature);
int gbWarmStartAddField(gbWarmStart* ws, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                        gb_scalar pressure, gb_scalar temperature);
int64_t gbWarmStartFieldCount(gbWarmStart* ws);
/* Adam (beta 0.9 / 0.999, eps 1e-8) on the mean squared error of the scaled
 * outputs; each step takes tiles_per_cta tiles of 128 cells per SM, tiles
 * shuffled per epoch.  loss_history (may be NULL) receives up to history_len
 * per-step losses.  Returns the number of steps, or -1. */
int64_t gbWarmStartTrain(gbWarmStart* ws, int epochs, int tiles_per_cta, float lr, double* loss_history,
                         int64_t history_len);
/* Writes the predicted state into a batch instance / three fields (both
 * value buffers of interior cells; ghosts are set by the next iteration's
 * boundary conditions). */
int gbWarmStartPredictBatch(gbWarmStart* ws, gbBatch* batch, int instance, gb_vector mach, gb_scalar pressure,
                            gb_scalar temperature);
int gbWarmStartPredict(gbWarmStart* ws, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                       gb_scalar pressure, gb_scalar temperature);
/* Explicit samples, for checking the kernels: x[n][8] inputs, t[n][5] scaled
 * targets.  Gradient: grad[36864] of the loss mean((y - t)^2) and the loss;
 * forward: y[n][5]. */
int gbWarmStartGradient(gbWarmStart* ws, int64_t n, const float* x, const float* t, float* grad, double* loss);
int gbWarmStartForward(gbWarmStart* ws, int64_t n, const float* x, float* y);
/* Bound, in SM clock cycles, on each wait of the MLP kernels for their
 * tensor-core work (cycles <= 0: the default, about 2 s).  A wait that gives
 * up makes the call return an error naming the stage; the kernel first lets
 * the work in flight finish (bounded by the default) and frees its tensor
 * memory, so later calls run normally.  Tests set a tiny bound to exercise
 * that path without a fault. */
int gbWarmStartSetWaitLimit(gbWarmStart* ws, long long cycles);

/* Pressure force on boundary region region_id (sum of p A n over its faces,
 * n pointing out of the fluid, p of the adjacent interior cell), float64,
 * deterministic; force[3].  Lift and drag are its components normal and
 * parallel to the free stream.  No counterpart in the reference. */
int gbWallForce(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, unsigned region_id, double* force);
int gbBatchWallForce(gbBatch* batch, int instance, unsigned region_id, double* force);

/* Writes the mesh (VTK polyhedra, type 42) and the fields' host values (one
 * per interior cell; call VarGpuToCpu first) as an ASCII VTU file, as the
 * reference's FieldsWriteVtu (src/fvmfieldsio.cu:5-287; include/
 * fvmfieldsio.cuh:12-17) does.  gbFieldsWriteVtuBinary writes the same file
 * with raw appended binary arrays.  0 on success. */
int FieldsWriteVtu(const char* filename, cuMesh* mesh, const FvmField** vars, const size_t nvars);
int gbFieldsWriteVtuBinary(const char* filename, cuMesh* mesh, const FvmField** vars, const size_t nvars);

/* Headless colour map of a scalar field on a boundary region: what the
 * reference's renderer writes into its OpenGL buffer (RenderMesh from a
 * region, src/render/window.cu:560-627; KernelRenderScalarField, :682-756),
 * written to `out` (host or device memory): 18 floats per triangle,
 * (x, y, z, r, g, b) for each of its 3 vertices.  Colours use the field's
 * last stored gradients and limiters (FvmEulerStepPrepare; zero before the
 * first).  out = NULL returns the number of triangles; otherwise returns
 * the number written, or -1 (also if capacity_triangles is too small). */
int64_t gbRenderRegionScalar(cuMesh* mesh, unsigned region_id, FvmField* field, gb_scalar u_min, gb_scalar u_max,
                             float* out, int64_t capacity_triangles);

/* ---- Generic finite-volume operators (include/fvmops.cuh:96-219) ----
 * gbFvmGradient: least-squares gradient and limiter of any scalar or vector
 * field (ScalarVarComputeGradient / VectorVarComputeGradient and the limiter
 * pass, src/fvmops.cu:51-266), stored in the field (VarAllGpuToCpu shows
 * them); a ghost carries its interior cell's.
 * gbFvmApply: one operator over every interior cell, out[n_cells x k] in the
 * reference's cell order, k = 1 (scalar), 3 (vector) or 9 (tensor
 * {u, v, w}, outer(a, b) = (a b.x, a b.y, a b.z)). */
enum {
    GB_FVM_LAPLACIAN = 0,          /* fvmLaplacianC       scalar -> scalar, needs gradient */
    GB_FVM_SCAL_GRAD = 1,          /* fvmScalGradC        scalar -> vector */
    GB_FVM_SCAL_GRAD_CORRECT = 2,  /* fvmScalGradCCorrect scalar -> vector, needs gradient */
    GB_FVM_VEC_GRAD = 3,           /* fvmVecGradC         vector -> tensor */
    GB_FVM_BOUND_SCAL_GRAD = 4,    /* fvmBoundScalGradC   scalar -> vector */
    GB_FVM_BOUND_VEC_GRAD = 5,     /* fvmBoundVecGradC    vector -> tensor */
    GB_FVM_DIV = 6,                /* fvmDivC             vector -> scalar */
    GB_FVM_CONV_CONST_SCAL = 7,    /* fvmConvConstScalU   scalar, constant phi -> scalar */
    GB_FVM_CONV_CONST_SCAL2 = 8,   /* fvmConvConstScalU2  scalar, constant phi -> scalar, needs gradient */
    GB_FVM_CONV_SCAL = 9,          /* fvmConvScalU        scalar, vector field phi -> scalar */
    GB_FVM_CONV_VEC = 10           /* fvmConvVecU         vector, vector field phi -> vector */
};
int gbFvmGradient(cuMesh* mesh, FvmField* u);
int gbFvmApply(cuMesh* mesh, int op, FvmField* u, FvmField* phi, gb_vector phi_const, float* out);

/* Generic field setup and boundary conditions on the device, for models
 * built from the operators (a scalar field takes value.x):
 * gbFieldInit: every value, cells and ghosts, = value; gradients 0 and
 *   limiters 1 where the field has them (ScalarVarInit / VectorVarInit,
 *   src/fvmops.cu:8-44);
 * gbFieldBcFixed: the ghosts of region_id = value (fvmScalarBcFixed,
 *   src/fvmops.cu:308-323, for vector fields too);
 * gbFieldBcZeroGrad: each ghost of region_id = its interior cell's value
 *   (fvmScalarBcZeroGrad / fvmVectorBcZeroGrad, src/fvmops.cu:326-366).
 * Returns 0, or 1 with gbGetLastError() set (unknown region included). */
int gbFieldInit(cuMesh* mesh, FvmField* u, gb_vector value);
int gbFieldBcFixed(cuMesh* mesh, FvmField* u, gb_vector value, unsigned int region_id);
int gbFieldBcZeroGrad(cuMesh* mesh, FvmField* u, unsigned int region_id);
/* y += a x over the interior cells (an explicit update with a residual from
 * gbFvmApplyTerms); x and y of the same kind, distinct. */
int gbFieldAxpy(cuMesh* mesh, FvmField* y, gb_scalar a, FvmField* x);

/* gbFvmApplyTerms: sum over terms of coef x operator at every interior cell,
 * the operators composed in one pass over each cell's faces (as a model
 * kernel composes the reference's inline operators), into the interior
 * values of `out` on the device: a scalar field when the operators give
 * scalars, a vector field when they give vectors (tensor-valued operators
 * have no field form).  Ghost values of `out` are left as they are; `out`
 * must not be an input of any term.  1 to 8 terms, all of one output kind;
 * an operator that needs a gradient reads its input's (gbFvmGradient).
 * Returns 0, or 1 with gbGetLastError() set. */
typedef struct gbFvmTerm {
    int op;                /* GB_FVM_* */
    gb_scalar coef;        /* multiplies the operator */
    FvmField* u;           /* input field */
    FvmField* phi;         /* velocity field of GB_FVM_CONV_SCAL / GB_FVM_CONV_VEC, else NULL */
    gb_vector phi_const;   /* constant velocity of GB_FVM_CONV_CONST_SCAL / _SCAL2 */
} gbFvmTerm;
int gbFvmApplyTerms(cuMesh* mesh, int n_terms, const gbFvmTerm* terms, FvmField* out);

/* ---- Incompressible Navier-Stokes (artificial compressibility) ----
 * The reference's NSI model (src/models/nsi.cu:71,114,137,144) calls
 * FvmNSIInit, FvmNSISlipBc, FvmNSIInletOutletBc, FvmNSIStepPrepare and
 * FvmNSIStep on a "velocity" (vector) and a "pressure" (scalar, p / rho)
 * field but never defines them; these are those calls.  Steady solutions of
 * div u = 0, div(u u + p I) = nu lap u are reached in pseudo-time
 * (dp/dt + beta^2 div u = 0) with second-order LSQ reconstruction, the
 * reference's limiter, a Rusanov flux with the artificial-compressibility
 * wave speed, and local time steps.  Constants (per thread, like the stream):
 * density (scales forces), kinematic viscosity nu, artificial sound speed
 * beta, and the face gradient of the viscous term: the two cells' average as
 * fvmLaplacianC (include/fvmops.cuh:96-102) takes it (0), or that average
 * with the compact correction along the centroid offset (1, default), and
 * whether the reconstruction uses the reference's limiter (1) or none (0,
 * default: smooth incompressible flow needs none, and the limiter's first-
 * order switching adds dissipation that shortens a laminar wake). */
int gbNSISetConstants(gb_scalar density, gb_scalar viscosity, gb_scalar beta, int corrected_laplacian, int limited);
int FvmNSIInit(cuMesh* mesh, FvmField* velocity, FvmField* pressure, gb_vector init_velocity, gb_scalar init_pressure);
/* symmetry: normal velocity mirrored, pressure extrapolated */
int FvmNSISlipBc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, const char* region);
/* no-slip wall: velocity mirrored through zero, pressure extrapolated (new) */
int FvmNSIWallBc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, const char* region);
/* inflow (inlet_velocity . n < 0): that velocity, interior pressure;
 * outflow: interior velocity, outlet_pressure */
int FvmNSIInletOutletBc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, gb_vector inlet_velocity,
                        gb_scalar outlet_pressure, const char* region);
int FvmNSIStepPrepare(cuMesh* mesh, FvmField* velocity, FvmField* pressure);
/* error[i] = (R_p^2 + |R_u|^2) V, summed by FvmFieldReduceSum */
int FvmNSIStep(cuMesh* mesh, FvmField* velocity, FvmField* pressure, gb_scalar cfl, const char* time_scheme,
               FvmField* dt, FvmField* error);
/* The whole loop as replayed graphs (as gbEulerRun).  Boundary conditions:
 * type 0 slip, 1 inlet / outlet (mach = inlet velocity, pressure = outlet
 * pressure), 2 no-slip wall.  The results, ghost values included, are
 * bitwise those of the per-call loop; when the ghosts number at least a
 * quarter of the cells the gradient kernel applies the conditions itself.
 * Stops on the device at the tolerance as gbEulerRun does. */
int64_t gbNSIRun(cuMesh* mesh, FvmField* velocity, FvmField* pressure, FvmField* error, gb_scalar cfl,
                 int64_t n_iter, const gbBc* bcs, int n_bc, double tolerance, int check_every,
                 double* residual_history);
/* Force on a wall region: density * sum of A (p n - nu (grad u)_f . n), n out
 * of the fluid; float64, deterministic. */
int gbNSIWallForce(cuMesh* mesh, FvmField* velocity, FvmField* pressure, unsigned region_id, double* force);

/* Sum of n float values in device memory into *result (one double in device
 * memory), accumulated in float64 in a fixed order: the reduction behind
 * FvmFieldReduceSum, for callers that cannot allocate device memory -- hosts
 * that hand out all device memory from their own pool, plugins whose device
 * footprint must not grow after setup.  It allocates nothing: its scratch is
 * a static array of 4096 partial sums (32 KiB per GPU, held by every GPU that
 * loads the library until exit), so n is limited to 4096 * 2048 = 8,388,608;
 * larger n is rejected with an error.  values and result must be device (or
 * managed) memory; other pointers are rejected.  The first call on each
 * device looks the array's address up (cudaGetSymbolAddress) and keeps it;
 * that address does not survive a cudaDeviceReset of that device.  All
 * calls share the array: calls that
 * overlap on the GPU (other streams, other threads) race and must be ordered
 * by the caller.  Asynchronous on `stream` (a cudaStream_t; NULL = legacy
 * default stream).  Returns 0, or nonzero with gbGetLastError set.  No
 * counterpart in the reference. */
int gbReduceSumNoAlloc(const float* values, uint64_t n, double* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRAPHITE_B200_H */
