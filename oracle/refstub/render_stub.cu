// No-op definitions for the headless reference build (test infrastructure).
// See oracle/refstub/render/window.cuh.
#include "render/window.cuh"

RenderControls RGC = {1};

RenderMesh* RenderMesh_from_region(cuMesh*, const char*) { return NULL; }
void RenderMesh_map(RenderMesh*) {}
void RenderMesh_unmap(RenderMesh*) {}
void RenderScalarField(RenderMesh*, FvmField*, scalar, scalar) {}

// src/models/euler.cu prints the mesh read time through this helper, which
// the reference defines in src/models/model.cu (not built headless).
void print_time(double t) { printf("%.3f s", t); }
