// Headless stand-in for the reference's OpenGL renderer header.
//
// Test infrastructure only: this header lets the reference's own solver
// sources (mesh, meshio, fvmfields, fvmops, models/euler) compile without
// GLFW/GLEW/OpenGL so that they can be run as the parity reference.  It is
// found before the reference's include/render/window.cuh because the build
// recipe (oracle/Makefile.ref) puts oracle/refstub first on the include path.
// The declarations mirror only what include/models/model.cuh and
// src/models/euler.cu name; every function is a no-op defined in
// oracle/refstub/render_stub.cu.
#pragma once

#include <stdio.h>
#include <stdlib.h>

#include "datatypes.cuh"
#include "mesh.cuh"
#include "fvmfields.cuh"

typedef unsigned int GLuint;
typedef struct GLFWwindow GLFWwindow;

typedef struct {
    int compute;
} RenderControls;

extern RenderControls RGC;

typedef struct {
    int unused;
} RenderMesh;

RenderMesh* RenderMesh_from_region(cuMesh* mesh, const char* region);
void RenderMesh_map(RenderMesh* mesh);
void RenderMesh_unmap(RenderMesh* mesh);
void RenderScalarField(RenderMesh* mesh, FvmField* field, scalar u_min, scalar u_max);
