// extern "C" entry points of libgraphite_b200.so (see include/graphite_b200.h).
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "gb_device.cuh"
#include "gb_internal.h"

namespace gb {

namespace {
thread_local std::string t_error;
thread_local cudaStream_t t_stream = nullptr;
std::atomic<uint64_t> g_launches{0};
std::atomic<int> g_transposed{1};
std::atomic<int> g_renumber{1};
thread_local bool t_counting = true;
}  // namespace

void set_error(const std::string& msg) { t_error = msg; }
void clear_error() { t_error.clear(); }
void count_launch(int n) {
    if (t_counting) g_launches += (uint64_t)n;
}

namespace {

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

bool launch_ok(const char* what) { return cuda_ok(cudaGetLastError(), what); }

template <typename T>
bool dalloc(T*& p, size_t n, const char* what) {
    p = nullptr;
    if (n == 0) return true;
    return cuda_ok(cudaMalloc((void**)&p, n * sizeof(T)), what);
}

template <typename T>
bool upload(T*& p, const std::vector<T>& v, const char* what) {
    if (!dalloc(p, v.size(), what)) return false;
    if (v.empty()) return true;
    return cuda_ok(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, t_stream), what);
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// The instantiated graphs of a replayed loop (gbEulerRun / gbNSIRun), kept
// on the mesh between calls.  `key` holds everything the captured launches
// bake in (field identities and device buffers, CFL, tolerance, boundary
// conditions, modes); a call whose key matches replays the graphs without
// capturing again.  The residual history of one chunk of iterations goes to
// `hist` (capacity `cap`); the RunCtl word stops the iterations on the
// device once the tolerance is met (or the residual is not finite), so a
// run ends exactly there although the host checks only every chunk.
struct RunGraphs {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    double* hist = nullptr;
    RunCtl* ctl = nullptr;            // device control word (counters, first residual, halt)
    RunCtl* h_ctl = nullptr;          // pinned host copy
    int64_t cap = 0;
    int per_iter = 0;
    int n_hist = 1;                   // histories of `cap` entries each in `hist`
    void release() {
        for (int k = 0; k < 2; ++k)
            if (exec[k]) cudaGraphExecDestroy(exec[k]);
        exec[0] = exec[1] = nullptr;
        if (hist) cudaFree(hist);
        if (ctl) cudaFree(ctl);
        if (h_ctl) cudaFreeHost(h_ctl);
        hist = nullptr;
        ctl = nullptr;
        h_ctl = nullptr;
        cap = 0;
        key.clear();
    }
};

struct FieldImpl;

// Boundary conditions that FvmEulerSlipBc / FvmEulerInletOutletBc have been
// asked for and that have not been applied yet.  They are applied together,
// by one k_bc_table launch, before anything reads or writes the fields'
// device values (the next FvmEulerStepPrepare in the reference's loop); each
// ghost's state depends only on its interior cell's, so this is bitwise what
// applying each call at once gives, a later condition on a region replacing
// an earlier one as it overwrote it.
struct PendingBcs {
    FvmField* f[3] = {nullptr, nullptr, nullptr};   // rho, rhou, rhoe
    GhostBcTable t{};
    bool any = false;
};

struct MeshImpl {
    Topology topo;
    Numbering num;
    DevMesh dev;
    uint32_t* d_cell_new = nullptr;   // old -> new, N+G
    PendingBcs pending;
    RunGraphs euler_run, nsi_run;
    cudaStream_t capture = nullptr;   // stream the loops are captured on
    double* h_result = nullptr;       // pinned: FvmFieldReduceSum's value on the host
};

std::atomic<uint64_t> g_field_ids{0};

struct FieldImpl {
    uint64_t id = ++g_field_ids;      // never reused: cached graphs refer to a field by it
    int comps = 1;                    // 1 scalar, 3 vector
    size_t size = 0;
    int alloc_grads = 0;
    void* val[2] = {nullptr, nullptr};   // float* or float4*
    int cur = 0;
    float4* grad = nullptr;           // N (scalar) or 3N (vector), bound mesh order
    void* rec = nullptr;              // S + G reconstructed face states: rho (float), rhou (float4 with rho E)
    const cuMesh* bound = nullptr;
    double* partials = nullptr;
    int n_partials = 0;
    bool partials_valid = false;
    float* staging = nullptr;         // size * comps floats
};

MeshImpl* impl(cuMesh* m) { return m ? static_cast<MeshImpl*>(m->impl) : nullptr; }
FieldImpl* impl(const FvmField* f) { return f ? static_cast<FieldImpl*>(f->impl) : nullptr; }

template <typename T>
T* hmalloc(size_t n) {
    return static_cast<T*>(calloc(n ? n : 1, sizeof(T)));
}

void free_host_mesh(cuMeshBase* b) {
    if (!b) return;
    free(b->cell_faces); free(b->cell_connects); free(b->cell_faces_starts);
    free(b->cell_volumes); free(b->cell_centers); free(b->cell_matrices);
    free(b->face_nodes); free(b->face_nodes_starts); free(b->face_areas);
    free(b->face_centers); free(b->face_normals); free(b->nodes);
    free(b->ghost_cell_ids); free(b->ghost_cell_starts);
    free(b);
}

void free_mesh(cuMesh* m) {
    if (!m) return;
    MeshImpl* mi = impl(m);
    if (mi) {
        DevMesh& d = mi->dev;
        dfree(d.cell_geo); dfree(d.face_geo); dfree(d.nfc); dfree(d.nb); dfree(d.lsq); dfree(d.ghost); dfree(d.red);
        dfree(d.twin); dfree(d.cf_geo); dfree(d.nbc); dfree(d.dn); dfree(d.df);
        dfree(mi->d_cell_new);
        mi->euler_run.release();
        mi->nsi_run.release();
        if (mi->capture) cudaStreamDestroy(mi->capture);
        if (mi->h_result) cudaFreeHost(mi->h_result);
        delete mi;
    }
    free_host_mesh(m->_cpu);
    for (size_t i = 0; i < m->region_names_size; ++i) free(m->region_names[i]);
    free(m->region_names);
    free(m);
}

// Topology -> device mesh + host mirror.
cuMesh* create_mesh(Topology&& topo) {
    cudaStream_t s = t_stream;
    // every device index is 32-bit: cells with ghosts, faces, and the
    // per-face entries with the ghosts' face-state slots after them (S + G)
    if ((uint64_t)kSlots * (uint64_t)topo.N + (uint64_t)topo.G >= (1ull << 32) || (uint64_t)topo.F >= (1ull << 32)) {
        set_error("mesh too large for 32-bit device indices: " + std::to_string(topo.N) + " cells, " +
                  std::to_string(topo.G) + " ghosts, " + std::to_string(topo.F) + " faces");
        return nullptr;
    }
    cuMesh* m = hmalloc<cuMesh>(1);
    MeshImpl* mi = new MeshImpl();
    m->impl = mi;
    mi->topo = std::move(topo);
    const Topology& t = mi->topo;
    const int64_t N = t.N, G = t.G, NG = N + G, F = t.F;
    number_cells(t, g_renumber.load() != 0, mi->num);
    const Numbering& num = mi->num;
    DevMesh& d = mi->dev;
    d.N = N; d.G = G; d.F = F; d.S = kSlots * N;

    // float64 metrics in the reference's order
    double *d_nodes = nullptr, *area = nullptr, *normal = nullptr, *fcen = nullptr, *ccen = nullptr, *vol = nullptr,
           *minv = nullptr;
    uint32_t *d_fns = nullptr, *d_fn = nullptr, *d_cfs = nullptr, *d_cf = nullptr, *d_cc = nullptr,
             *d_cell_old = nullptr, *d_face_old = nullptr;
    bool ok = upload(d_nodes, t.nodes, "upload nodes") && upload(d_fns, t.fns, "upload face nodes") &&
              upload(d_fn, t.fn, "upload face nodes") && upload(d_cfs, t.cfs, "upload cells") &&
              upload(d_cf, t.cf, "upload cells") && upload(d_cc, t.cc, "upload cells") &&
              dalloc(area, F, "alloc metrics") && dalloc(normal, 3 * F, "alloc metrics") &&
              dalloc(fcen, 3 * F, "alloc metrics") && dalloc(ccen, 3 * NG, "alloc metrics") &&
              dalloc(vol, NG, "alloc metrics") && dalloc(minv, 9 * N, "alloc metrics");
    if (ok) {
        launch_face_metrics64(F, d_nodes, d_fns, d_fn, area, normal, fcen, s);
        launch_cell_metrics64(N, d_cfs, d_cf, area, normal, fcen, ccen, vol, s);
        launch_ghost_metrics64(G, N, d_cfs, d_cf, d_cc, area, normal, fcen, ccen, vol, s);
        launch_lsq64(N, d_cfs, d_cc, ccen, minv, s);
        ok = launch_ok("metric kernels");
    }
    // renumbered float32 layout
    // slot-major per-face entries: (slot t, cell i) at t * N + i
    std::vector<uint2> nb((size_t)d.S, make_uint2(0, 0)), gl(G);
    std::vector<uint8_t> nfc((size_t)N);
    std::vector<uint32_t> twin((size_t)d.S, 0);
    auto entry = [&](uint32_t cell, uint32_t slot) { return (uint32_t)(slot * N + cell); };
    for (int64_t i = 0; i < N && ok; ++i) {
        const uint32_t nf = num.start[i + 1] - num.start[i];
        if (nf > (uint32_t)kSlots) {
            set_error("mesh: a cell has more than 6 faces");
            ok = false;
            break;
        }
        nfc[i] = (uint8_t)nf;
        d.max_faces = std::max<int>(d.max_faces, (int)nf);
        for (uint32_t t = 0; t < nf; ++t) {
            const uint32_t k = num.start[i] + t;
            nb[entry((uint32_t)i, t)] = make_uint2(num.nb_face[k], num.nb_cell[k]);
        }
    }
    for (int64_t g = 0; g < G; ++g) gl[g] = make_uint2(num.ghost_cell[g], num.ghost_face[g]);
    // twin of each entry: the same face among the neighbour's entries, or the
    // ghost's slot S + g
    for (int64_t i = 0; i < N && ok; ++i)
        for (uint32_t t = 0; t < nfc[i] && ok; ++t) {
            const uint32_t j = num.nb_cell[num.start[i] + t], f = num.nb_face[num.start[i] + t];
            uint32_t& tw = twin[entry((uint32_t)i, t)];
            if (j >= (uint32_t)N) { tw = (uint32_t)(d.S + (j - N)); continue; }
            tw = UINT32_MAX;
            for (uint32_t t2 = 0; t2 < num.start[j + 1] - num.start[j]; ++t2)
                if (num.nb_face[num.start[j] + t2] == f) { tw = entry(j, t2); break; }
            if (tw == UINT32_MAX) {
                set_error("mesh: face " + std::to_string(f) + " missing from a neighbour's face list");
                ok = false;
            }
        }
    ok = ok && upload(d_cell_old, num.cell_old, "upload numbering") && upload(d_face_old, num.face_old, "upload numbering") &&
         upload(mi->d_cell_new, num.cell_new, "upload numbering") && dalloc(d.cell_geo, NG, "alloc mesh") &&
         dalloc(d.face_geo, 2 * F, "alloc mesh") && upload(d.nfc, nfc, "upload csr") &&
         upload(d.nb, nb, "upload csr") && dalloc(d.lsq, 2 * N, "alloc mesh") && upload(d.ghost, gl, "upload ghosts") &&
         upload(d.twin, twin, "upload csr") && dalloc(d.cf_geo, (size_t)d.S, "alloc mesh") &&
         dalloc(d.nbc, (size_t)d.S, "alloc mesh") && dalloc(d.dn, (size_t)d.S, "alloc mesh") &&
         dalloc(d.df, (size_t)d.S, "alloc mesh");
    d.n_red_max = std::max<int>(reduce_blocks(NG), (int)((N + kBlock - 1) / kBlock));
    ok = ok && dalloc(d.red, (size_t)d.n_red_max + 1, "alloc reduction") &&
         cuda_ok(cudaMallocHost((void**)&mi->h_result, sizeof(double)), "alloc reduction");
    if (ok) {
        launch_layout(d, d_cell_old, d_face_old, area, normal, fcen, ccen, vol, minv, s);
        launch_entry_geo(d, s);
        ok = launch_ok("layout kernels");
    }
    // host mirror in the reference's layout and order
    cuMeshBase* b = hmalloc<cuMeshBase>(1);
    m->_cpu = b;
    b->type = _CPU;
    b->allocated = 1;
    b->n_cells = N; b->n_faces = F; b->n_nodes = t.nodes.size() / 3; b->n_ghosts = G; b->n_regions = t.regions.size();
    if (ok) {
        std::vector<double> h_area(F), h_normal(3 * F), h_fcen(3 * F), h_ccen(3 * NG), h_vol(NG), h_minv(9 * N);
        ok = cuda_ok(cudaMemcpyAsync(h_area.data(), area, F * 8, cudaMemcpyDeviceToHost, s), "download metrics") &&
             cuda_ok(cudaMemcpyAsync(h_normal.data(), normal, 3 * F * 8, cudaMemcpyDeviceToHost, s), "download metrics") &&
             cuda_ok(cudaMemcpyAsync(h_fcen.data(), fcen, 3 * F * 8, cudaMemcpyDeviceToHost, s), "download metrics") &&
             cuda_ok(cudaMemcpyAsync(h_ccen.data(), ccen, 3 * NG * 8, cudaMemcpyDeviceToHost, s), "download metrics") &&
             cuda_ok(cudaMemcpyAsync(h_vol.data(), vol, NG * 8, cudaMemcpyDeviceToHost, s), "download metrics") &&
             cuda_ok(cudaMemcpyAsync(h_minv.data(), minv, 9 * N * 8, cudaMemcpyDeviceToHost, s), "download metrics") &&
             cuda_ok(cudaStreamSynchronize(s), "mesh setup");
        if (ok) {
            auto cpy_u32 = [](const std::vector<uint32_t>& v) {
                unsigned* p = hmalloc<unsigned>(v.size());
                if (!v.empty()) memcpy(p, v.data(), v.size() * 4);
                return p;
            };
            b->cell_faces = cpy_u32(t.cf); b->cell_connects = cpy_u32(t.cc); b->cell_faces_starts = cpy_u32(t.cfs);
            b->face_nodes = cpy_u32(t.fn); b->face_nodes_starts = cpy_u32(t.fns);
            b->ghost_cell_ids = cpy_u32(t.ghost_ids); b->ghost_cell_starts = cpy_u32(t.ghost_starts);
            b->cell_volumes = hmalloc<float>(NG);
            b->cell_centers = hmalloc<gb_vector>(NG);
            b->cell_matrices = hmalloc<gb_tensor>(N);
            b->face_areas = hmalloc<float>(F);
            b->face_centers = hmalloc<gb_vector>(F);
            b->face_normals = hmalloc<gb_vector>(F);
            b->nodes = hmalloc<gb_vector>(b->n_nodes);
            for (int64_t i = 0; i < NG; ++i) {
                b->cell_volumes[i] = (float)h_vol[i];
                b->cell_centers[i] = {(float)h_ccen[3 * i], (float)h_ccen[3 * i + 1], (float)h_ccen[3 * i + 2]};
            }
            for (int64_t i = 0; i < N; ++i) {
                float* p = &b->cell_matrices[i].u.x;
                for (int k = 0; k < 9; ++k) p[k] = (float)h_minv[9 * i + k];
            }
            for (int64_t f = 0; f < F; ++f) {
                b->face_areas[f] = (float)h_area[f];
                b->face_centers[f] = {(float)h_fcen[3 * f], (float)h_fcen[3 * f + 1], (float)h_fcen[3 * f + 2]};
                b->face_normals[f] = {(float)h_normal[3 * f], (float)h_normal[3 * f + 1], (float)h_normal[3 * f + 2]};
            }
            for (size_t i = 0; i < b->n_nodes; ++i)
                b->nodes[i] = {(float)t.nodes[3 * i], (float)t.nodes[3 * i + 1], (float)t.nodes[3 * i + 2]};
        }
    }
    dfree(d_nodes); dfree(area); dfree(normal); dfree(fcen); dfree(ccen); dfree(vol); dfree(minv);
    dfree(d_fns); dfree(d_fn); dfree(d_cfs); dfree(d_cf); dfree(d_cc); dfree(d_cell_old); dfree(d_face_old);
    m->region_names_alloc = m->region_names_size = t.regions.size();
    m->region_names = hmalloc<char*>(t.regions.size());
    for (size_t r = 0; r < t.regions.size(); ++r) m->region_names[r] = strdup(t.regions[r].c_str());
    if (!ok) {
        free_mesh(m);
        return nullptr;
    }
    return m;
}

bool check_mesh(cuMesh* m) {
    if (!m || !impl(m)) { set_error("null mesh"); return false; }
    return true;
}

// Binds a field's device storage to a mesh's cell order (first use).
bool bind(cuMesh* mesh, FvmField* f, int comps, const char* what) {
    FieldImpl* fi = impl(f);
    if (!fi) { set_error(std::string(what) + ": null field"); return false; }
    if (fi->comps != comps) {
        set_error(std::string(what) + ": field '" + f->name + (comps == 1 ? "' must be a scalar field" : "' must be a vector field"));
        return false;
    }
    const MeshImpl* mi = impl(mesh);
    if ((int64_t)fi->size != mi->topo.N + mi->topo.G) {
        set_error(std::string(what) + ": field '" + f->name + "' has " + std::to_string(fi->size) +
                  " elements, the mesh has " + std::to_string(mi->topo.N + mi->topo.G) + " cells and ghosts");
        return false;
    }
    if (fi->bound && fi->bound != mesh) {
        set_error(std::string(what) + ": field '" + f->name + "' is already used with another mesh");
        return false;
    }
    fi->bound = mesh;
    return true;
}

bool ensure_grad(cuMesh* mesh, FvmField* f) {
    FieldImpl* fi = impl(f);
    if (fi->grad && fi->rec) return true;
    const DevMesh& d = impl(mesh)->dev;
    if (!fi->grad && (!dalloc(fi->grad, (size_t)d.N * fi->comps, "alloc gradient") ||
                      !cuda_ok(cudaMemsetAsync(fi->grad, 0, (size_t)d.N * fi->comps * sizeof(float4), t_stream),
                               "zero gradient")))
        return false;
    uint8_t* r = nullptr;
    const size_t bytes = (size_t)(d.S + d.G) * (fi->comps == 1 ? sizeof(float) : sizeof(float4));
    if (!dalloc(r, bytes, "alloc face states")) return false;
    fi->rec = r;
    return true;
}

bool ensure_partials(FieldImpl* fi, int n) {
    if (fi->n_partials >= n) return true;
    dfree(fi->partials);
    fi->n_partials = 0;
    if (!dalloc(fi->partials, (size_t)n, "alloc partials")) return false;
    fi->n_partials = n;
    return true;
}

bool ensure_staging(FieldImpl* fi) {
    if (fi->staging) return true;
    return dalloc(fi->staging, fi->size * fi->comps, "alloc staging");
}

bool euler_fields(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, const char* what) {
    if (!check_mesh(mesh)) return false;
    if (!bind(mesh, rho, 1, what) || !bind(mesh, rhou, 3, what) || !bind(mesh, rhoe, 1, what)) return false;
    FieldImpl *a = impl(rho), *b = impl(rhou), *c = impl(rhoe);
    if (a->cur != b->cur || a->cur != c->cur) {
        set_error(std::string(what) + ": rho, rhou and rhoe were not updated together");
        return false;
    }
    return true;
}

EulerState state_of(FvmField* rho, FvmField* rhou, FvmField* rhoe, int buf) {
    return EulerState{(const float*)impl(rho)->val[buf], (const float4*)impl(rhou)->val[buf],
                      (const float*)impl(rhoe)->val[buf]};
}

int region_lookup(cuMesh* mesh, const char* region) {
    const Topology& t = impl(mesh)->topo;
    if (!region) { set_error("null region name"); return -1; }
    for (size_t r = 0; r < t.regions.size(); ++r)
        if (t.regions[r] == region) return (int)r;
    set_error(std::string("region with name ") + region + " not found in mesh");
    return -1;
}

void enqueue_slip(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, int r, int cur, cudaStream_t s,
                  const DevMesh* dm = nullptr) {
    MeshImpl* mi = impl(mesh);
    float* pr[2] = {(float*)impl(rho)->val[0], (float*)impl(rho)->val[1]};
    float4* pu[2] = {(float4*)impl(rhou)->val[0], (float4*)impl(rhou)->val[1]};
    float* pe[2] = {(float*)impl(rhoe)->val[0], (float*)impl(rhoe)->val[1]};
    launch_bc_slip(dm ? *dm : mi->dev, mi->num.region_start[r], mi->num.region_start[r + 1], pr, pu, pe, cur, s);
}

void enqueue_farfield(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, int r, int cur, gb_vector mach,
                      float p, float t, cudaStream_t s, const DevMesh* dm = nullptr) {
    MeshImpl* mi = impl(mesh);
    float* pr[2] = {(float*)impl(rho)->val[0], (float*)impl(rho)->val[1]};
    float4* pu[2] = {(float4*)impl(rhou)->val[0], (float4*)impl(rhou)->val[1]};
    float* pe[2] = {(float*)impl(rhoe)->val[0], (float*)impl(rhoe)->val[1]};
    launch_bc_farfield(dm ? *dm : mi->dev, mi->num.region_start[r], mi->num.region_start[r + 1], pr, pu, pe, cur,
                       make_float3(mach.x, mach.y, mach.z), p, t, s);
}

// Applies the deferred boundary conditions of the mesh, if any.
bool flush_bcs(cuMesh* mesh) {
    MeshImpl* mi = impl(mesh);
    if (!mi || !mi->pending.any) return true;
    PendingBcs& pb = mi->pending;
    for (int k = 0; k < 2; ++k) {
        pb.t.rho[k] = (float*)impl(pb.f[0])->val[k];
        pb.t.rhou[k] = (float4*)impl(pb.f[1])->val[k];
        pb.t.rhoe[k] = (float*)impl(pb.f[2])->val[k];
    }
    pb.any = false;
    launch_bc_table(mi->dev, pb.t, impl(pb.f[0])->cur, t_stream);
    return launch_ok("boundary conditions");
}

// Applies them when f is one of the fields they are for.
bool flush_for(const FvmField* f) {
    FieldImpl* fi = impl(f);
    if (!fi || !fi->bound) return true;
    cuMesh* mesh = const_cast<cuMesh*>(fi->bound);
    const PendingBcs& pb = impl(mesh)->pending;
    if (pb.any && (pb.f[0] == f || pb.f[1] == f || pb.f[2] == f)) return flush_bcs(mesh);
    return true;
}

// Records a boundary condition of region r (type 0 slip, 1 far field);
// false when the mesh has more regions than the table holds (the caller
// then applies it at once).
bool defer_bc(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, int r, int type, gb_vector mach, float p,
              float temp, bool* ok) {
    MeshImpl* mi = impl(mesh);
    const int n_regions = (int)mi->topo.regions.size();
    *ok = true;
    if (n_regions > kMaxBcRegions) return false;
    PendingBcs& pb = mi->pending;
    if (pb.any && (pb.f[0] != rho || pb.f[1] != rhou || pb.f[2] != rhoe)) *ok = flush_bcs(mesh);
    if (!pb.any) {
        pb.f[0] = rho;
        pb.f[1] = rhou;
        pb.f[2] = rhoe;
        pb.t = GhostBcTable{};
        pb.t.n = n_regions;
        pb.t.store = 1;
        for (int k = 0; k <= n_regions; ++k) pb.t.start[k] = mi->num.region_start[k];
        for (int k = 0; k < n_regions; ++k) pb.t.type[k] = -1;
        pb.any = true;
    }
    pb.t.type[r] = type;
    pb.t.mach[r] = make_float3(mach.x, mach.y, mach.z);
    pb.t.p[r] = p;
    pb.t.temp[r] = temp;
    return true;
}

// store_gradients = false: only the face states the flux needs are written
EulerGrad grad_of(FvmField* rho, FvmField* rhou, FvmField* rhoe, bool store_gradients) {
    return EulerGrad{store_gradients ? impl(rho)->grad : nullptr, store_gradients ? impl(rhou)->grad : nullptr,
                     store_gradients ? impl(rhoe)->grad : nullptr, (float*)impl(rho)->rec, (float4*)impl(rhou)->rec};
}

FaceRecs recs_of(FvmField* rho, FvmField* rhou) {
    return FaceRecs{(const float*)impl(rho)->rec, (const float4*)impl(rhou)->rec};
}

void enqueue_flux(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, FvmField* error, float cfl, int cur,
                  cudaStream_t s, const DevMesh* dm = nullptr, double* partials_rho = nullptr) {
    MeshImpl* mi = impl(mesh);
    const int nxt = 1 - cur;
    FieldImpl* ei = impl(error);
    launch_flux(dm ? *dm : mi->dev, state_of(rho, rhou, rhoe, cur), recs_of(rho, rhou), (float*)impl(rho)->val[nxt],
                (float4*)impl(rhou)->val[nxt], (float*)impl(rhoe)->val[nxt], (float*)ei->val[ei->cur], ei->partials,
                cfl, s, partials_rho);
}

// Reference-order host copy of the current values.
bool download_values(FvmField* f) {
    FieldImpl* fi = impl(f);
    cudaStream_t s = t_stream;
    const size_t bytes = fi->size * fi->comps * sizeof(float);
    if (fi->size == 0) return true;
    if (!fi->bound) {
        // never used with a mesh: the device order is the caller's order
        if (fi->comps == 1)
            return cuda_ok(cudaMemcpyAsync(f->_cpu->value, fi->val[fi->cur], bytes, cudaMemcpyDeviceToHost, s), "copy field") &&
                   cuda_ok(cudaStreamSynchronize(s), "copy field");
        if (!ensure_staging(fi)) return false;
        std::vector<float4> tmp(fi->size);
        if (!cuda_ok(cudaMemcpyAsync(tmp.data(), fi->val[fi->cur], fi->size * 16, cudaMemcpyDeviceToHost, s), "copy field") ||
            !cuda_ok(cudaStreamSynchronize(s), "copy field"))
            return false;
        float* h = (float*)f->_cpu->value;
        for (size_t i = 0; i < fi->size; ++i) { h[3 * i] = tmp[i].x; h[3 * i + 1] = tmp[i].y; h[3 * i + 2] = tmp[i].z; }
        return true;
    }
    if (!ensure_staging(fi)) return false;
    const uint32_t* idx = impl(const_cast<cuMesh*>(fi->bound))->d_cell_new;
    if (fi->comps == 1) launch_gather_scalar((int64_t)fi->size, (const float*)fi->val[fi->cur], idx, fi->staging, s);
    else launch_gather_vector((int64_t)fi->size, (const float4*)fi->val[fi->cur], idx, fi->staging, s);
    return launch_ok("gather field") &&
           cuda_ok(cudaMemcpyAsync(f->_cpu->value, fi->staging, bytes, cudaMemcpyDeviceToHost, s), "copy field") &&
           cuda_ok(cudaStreamSynchronize(s), "copy field");
}

bool download_gradients(FvmField* f) {
    FieldImpl* fi = impl(f);
    if (!fi->alloc_grads || !f->_cpu->gradient) return true;
    const size_t n = fi->size;
    float* hg = (float*)f->_cpu->gradient;   // 3 (scalar) or 9 (vector) floats per element
    float* hl = (float*)f->_cpu->limiter;    // 1 or 3 floats per element
    if (!fi->grad || !fi->bound) {
        memset(hg, 0, n * fi->comps * 3 * sizeof(float));
        for (size_t i = 0; i < n * fi->comps; ++i) hl[i] = 1.f;
        return true;
    }
    const MeshImpl* mi = impl(const_cast<cuMesh*>(fi->bound));
    const Topology& t = mi->topo;
    const int64_t N = t.N;
    std::vector<float4> g((size_t)N * fi->comps);
    if (!cuda_ok(cudaMemcpyAsync(g.data(), fi->grad, g.size() * 16, cudaMemcpyDeviceToHost, t_stream), "copy gradient") ||
        !cuda_ok(cudaStreamSynchronize(t_stream), "copy gradient"))
        return false;
    for (size_t o = 0; o < n; ++o) {
        // ghosts carry their interior cell's gradient and limiter
        const uint32_t src = (int64_t)o < N ? (uint32_t)o : t.cc[t.cfs[o]];
        const uint32_t i = mi->num.cell_new[src];
        for (int a = 0; a < fi->comps; ++a) {
            const float4 v = g[(size_t)i * fi->comps + a];
            hg[(o * fi->comps + a) * 3 + 0] = v.x;
            hg[(o * fi->comps + a) * 3 + 1] = v.y;
            hg[(o * fi->comps + a) * 3 + 2] = v.z;
            hl[o * fi->comps + a] = v.w;
        }
    }
    return true;
}

// ---- replayed loops (gbEulerRun, gbNSIRun) ----

void key_field(std::vector<uint64_t>& k, const FvmField* f) {
    const FieldImpl* fi = impl(f);
    for (uint64_t w : {fi->id, (uint64_t)(uintptr_t)fi->val[0], (uint64_t)(uintptr_t)fi->val[1],
                       (uint64_t)(uintptr_t)fi->rec, (uint64_t)(uintptr_t)fi->grad,
                       (uint64_t)(uintptr_t)fi->partials, (uint64_t)fi->n_partials})
        k.push_back(w);
}

void key_bytes(std::vector<uint64_t>& k, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i += 8) {
        uint64_t w = 0;
        memcpy(&w, c + i, std::min<size_t>(8, n - i));
        k.push_back(w);
    }
}

// Makes `rg` hold graphs for `key` with a history of at least `need` entries
// per chunk, capturing them (enqueue(k, stream, device mesh with the halt
// word, ctl, hist, cap) for value buffer parity k) only when the key or the
// capacity changed.
template <class Enqueue>
bool ensure_run_graphs(MeshImpl* mi, RunGraphs& rg, std::vector<uint64_t>& key, int64_t need, int per_iter,
                       Enqueue&& enqueue, const char* what, int n_hist = 1) {
    if (rg.exec[0] && rg.exec[1] && rg.key == key && rg.cap >= need && rg.n_hist == n_hist) return true;
    const int64_t cap = std::max<int64_t>(need, std::max<int64_t>(256, rg.cap));
    rg.release();
    if (!mi->capture && !cuda_ok(cudaStreamCreateWithFlags(&mi->capture, cudaStreamNonBlocking), what)) return false;
    if (!dalloc(rg.hist, (size_t)(cap * n_hist), what) || !dalloc(rg.ctl, 1, what) ||
        !cuda_ok(cudaMallocHost((void**)&rg.h_ctl, sizeof(RunCtl)), what)) {
        rg.release();
        return false;
    }
    rg.cap = cap;
    rg.n_hist = n_hist;
    DevMesh dh = mi->dev;          // the iteration kernels of this loop stop on the halt word
    dh.halt = &rg.ctl->halt;
    bool ok = true;
    t_counting = false;
    for (int k = 0; k < 2 && ok; ++k) {
        cudaGraph_t g = nullptr;
        ok = cuda_ok(cudaStreamBeginCapture(mi->capture, cudaStreamCaptureModeThreadLocal), "graph capture");
        if (!ok) break;
        enqueue(k, mi->capture, dh, rg.ctl, rg.hist, (unsigned long long)cap);
        ok = cuda_ok(cudaStreamEndCapture(mi->capture, &g), "graph capture") &&
             cuda_ok(cudaGraphInstantiate(&rg.exec[k], g, 0), "graph instantiate");
        if (g) cudaGraphDestroy(g);
    }
    t_counting = true;
    if (!ok) { rg.release(); return false; }
    rg.key = key;
    rg.per_iter = per_iter;
    return true;
}

// Replays the graphs from value buffer `cur` for up to n_iter iterations,
// check_every at a time.  The device stops iterating once a residual is
// below tolerance x the run's first one (tolerance > 0) or is not finite;
// after each chunk the iterations it actually ran come back to `hist`.
// Returns the iterations run (the last one the first below tolerance, when
// the tolerance is met), or -1 when a residual was not finite (an error);
// `cur` becomes the buffer holding the last state.
int64_t replay_run_graphs(RunGraphs& rg, int& cur, int64_t n_iter, int64_t check_every, std::vector<double>& hist,
                          cudaStream_t s, const char* what, std::vector<double>* hist2 = nullptr) {
    const int cur0 = cur;
    int64_t done = 0;
    bool ok = cuda_ok(cudaMemsetAsync(rg.ctl, 0, sizeof(RunCtl), s), what);
    while (ok && done < n_iter) {
        const int64_t chunk = std::min<int64_t>(check_every, n_iter - done);
        ok = cuda_ok(cudaMemsetAsync(&rg.ctl->it_chunk, 0, sizeof(unsigned long long), s), what);
        int k = (int)((cur0 + done) & 1);
        for (int64_t i = 0; i < chunk && ok; ++i) {
            ok = cuda_ok(cudaGraphLaunch(rg.exec[k], s), "graph launch");
            count_launch(rg.per_iter);
            k = 1 - k;
        }
        if (!ok) break;
        ok = cuda_ok(cudaMemcpyAsync(hist.data() + done, rg.hist, (size_t)chunk * sizeof(double),
                                     cudaMemcpyDeviceToHost, s), what) &&
             (!hist2 || rg.n_hist < 2 ||
              cuda_ok(cudaMemcpyAsync(hist2->data() + done, rg.hist + rg.cap, (size_t)chunk * sizeof(double),
                                      cudaMemcpyDeviceToHost, s), what)) &&
             cuda_ok(cudaMemcpyAsync(rg.h_ctl, rg.ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, s), what) &&
             cuda_ok(cudaStreamSynchronize(s), what);
        if (!ok) break;
        const int64_t ran = (int64_t)std::min<unsigned long long>(rg.h_ctl->it_chunk, (unsigned long long)chunk);
        done += ran;
        if (rg.h_ctl->halt == 2) {
            set_error(std::string(what) + ": residual is not finite (diverged)");
            ok = false;
            break;
        }
        if (rg.h_ctl->halt != 0 || ran < chunk) break;
    }
    cur = (int)((cur0 + done) & 1);
    return ok ? done : -1;
}
}  // namespace

bool mesh_access(cuMesh* mesh, MeshAccess* out) {
    MeshImpl* mi = impl(mesh);
    if (!mi) { set_error("null mesh"); return false; }
    out->dev = &mi->dev;
    out->d_cell_new = mi->d_cell_new;
    out->region_start = mi->num.region_start.data();
    out->n_regions = (int)mi->topo.regions.size();
    out->N = mi->topo.N;
    out->G = mi->topo.G;
    out->topo = &mi->topo;
    out->num = &mi->num;
    return true;
}

bool field_access(FvmField* f, cuMesh* mesh, int comps, FieldAccess* out) {
    FieldImpl* fi = impl(f);
    if (!fi || !fi->val[0]) { set_error("null or unallocated field"); return false; }
    if (!flush_for(f)) return false;
    if (mesh ? !bind(mesh, f, comps, "field") : fi->comps != comps) {
        if (!mesh) set_error("field has the wrong number of components");
        return false;
    }
    out->val[0] = fi->val[0];
    out->val[1] = fi->val[1];
    out->cur = fi->cur;
    out->comps = fi->comps;
    out->size = fi->size;
    out->grad = fi->grad;
    return true;
}

bool reference_momentum() { return g_transposed.load() != 0; }

}  // namespace gb

using namespace gb;

extern "C" {

const char* gbGetLastError(void) { return t_error.c_str(); }

int gbSetStream(void* stream) {
    t_stream = (cudaStream_t)stream;
    return 0;
}

void* gbGetStream(void) { return (void*)t_stream; }

uint64_t gbKernelLaunchCount(void) { return g_launches.load(); }

int gbSetReferenceMomentumReconstruction(int enabled) {
    g_transposed = enabled ? 1 : 0;
    return 0;
}

int gbSetRenumbering(int enabled) {
    g_renumber = enabled ? 1 : 0;
    return 0;
}

int cuMeshFromSu2(const char* su2_filename, const char* out_filename) {
    clear_error();
    ElementSet es;
    Topology t;
    if (!su2_filename || !out_filename) { set_error("null file name"); return 1; }
    if (!parse_su2(su2_filename, es) || !build_topology(es, t) || !write_fvm(out_filename, t)) return 1;
    return 0;
}

cuMesh* cuMeshFromFile(const char* filename) {
    clear_error();
    Topology t;
    if (!filename) { set_error("null file name"); return nullptr; }
    if (!read_fvm(filename, t)) return nullptr;
    return create_mesh(std::move(t));
}

cuMesh* gbMeshFromSu2(const char* su2_filename) {
    clear_error();
    ElementSet es;
    Topology t;
    if (!su2_filename) { set_error("null file name"); return nullptr; }
    if (!parse_su2(su2_filename, es) || !build_topology(es, t)) return nullptr;
    return create_mesh(std::move(t));
}

void cuMeshFree(cuMesh* mesh) { free_mesh(mesh); }

size_t cuMeshGetVarSize(cuMesh* m) { return m ? m->_cpu->n_cells + m->_cpu->n_ghosts : 0; }
size_t cuMeshGetnCells(cuMesh* m) { return m ? m->_cpu->n_cells : 0; }
size_t cuMeshGetnGhosts(cuMesh* m) { return m ? m->_cpu->n_ghosts : 0; }
size_t cuMeshGetnCellsAndGhosts(cuMesh* m) { return cuMeshGetVarSize(m); }

size_t cuMeshGetnRegionCells(cuMesh* m, unsigned int r) {
    if (!m || r >= m->_cpu->n_regions) return 0;
    return m->_cpu->ghost_cell_starts[r + 1] - m->_cpu->ghost_cell_starts[r];
}

unsigned int cuMeshGetRegionId(cuMesh* m, const char* name) {
    clear_error();
    if (!check_mesh(m)) return UINT32_MAX;
    const int r = region_lookup(m, name);
    return r < 0 ? UINT32_MAX : (unsigned)r;
}

void cuMeshPrintInfo(cuMesh* m) {
    if (!m) return;
    const cuMeshBase* b = m->_cpu;
    printf("Printing info on cuMesh object\n");
    printf("- n_cells = %zu\n", b->n_cells);
    printf("- n_faces = %zu\n", b->n_faces);
    printf("- n_nodes = %zu\n", b->n_nodes);
    printf("- n_ghosts = %zu\n", b->n_ghosts);
    printf("- n_regions = %zu\n", b->n_regions);
    printf("- n_cells_faces = %u\n", b->cell_faces_starts[b->n_cells + b->n_ghosts]);
    printf("- n_face_nodes = %u\n", b->face_nodes_starts[b->n_faces]);
    printf("- renumbering bandwidth = %lld\n", (long long)impl(m)->num.bandwidth);
}

FvmField* FvmFieldNew(size_t elem_size, size_t size, const char* name, int alloc_grads) {
    clear_error();
    int comps;
    if (elem_size == sizeof(gb_scalar)) comps = 1;
    else if (elem_size == sizeof(gb_vector)) comps = 3;
    else { set_error("FvmFieldNew: elem_size must be sizeof(scalar) or sizeof(vector)"); return nullptr; }
    FvmField* f = hmalloc<FvmField>(1);
    FieldImpl* fi = new FieldImpl();
    f->impl = fi;
    f->name = strdup(name ? name : "");
    fi->comps = comps;
    fi->size = size;
    fi->alloc_grads = alloc_grads;
    f->_cpu = hmalloc<FvmFieldBase>(1);
    f->_cpu->elem_size = elem_size;
    f->_cpu->size = size;
    // the value mirror is pinned so that VarGpuToCpu / gbVarCpuToGpu run at
    // full PCIe/C2C bandwidth
    bool ok = cuda_ok(cudaMallocHost(&f->_cpu->value, (size ? size : 1) * elem_size), "FvmFieldNew");
    if (ok) memset(f->_cpu->value, 0, (size ? size : 1) * elem_size);
    if (alloc_grads) {
        f->_cpu->gradient = calloc(size ? size : 1, elem_size * 3);
        f->_cpu->limiter = calloc(size ? size : 1, elem_size);
    }
    const size_t vb = comps == 1 ? sizeof(float) : sizeof(float4);
    for (int k = 0; k < 2 && ok; ++k) {
        ok = cuda_ok(cudaMalloc(&fi->val[k], (size ? size : 1) * vb), "FvmFieldNew") &&
             cuda_ok(cudaMemsetAsync(fi->val[k], 0, (size ? size : 1) * vb, t_stream), "FvmFieldNew");
    }
    if (!ok) {
        FvmFieldFree(f);
        return nullptr;
    }
    return f;
}

void FvmFieldFree(FvmField* f) {
    if (!f) return;
    FieldImpl* fi = impl(f);
    if (fi) {
        flush_for(f);
        dfree(fi->val[0]); dfree(fi->val[1]); dfree(fi->grad); dfree(fi->partials); dfree(fi->staging);
        if (fi->rec) cudaFree(fi->rec);
        delete fi;
    }
    if (f->_cpu) {
        if (f->_cpu->value) cudaFreeHost(f->_cpu->value);
        free(f->_cpu->gradient); free(f->_cpu->limiter);
        free(f->_cpu);
    }
    free(f->name);
    free(f);
}

FvmFieldType FvmFieldGetType(const FvmField* v) {
    if (!v) return FIELD_UNKNOWN;
    if (v->_cpu->elem_size == sizeof(gb_scalar)) return SCALAR;
    if (v->_cpu->elem_size == sizeof(gb_vector)) return VECTOR;
    if (v->_cpu->elem_size == sizeof(gb_tensor)) return TENSOR;
    return FIELD_UNKNOWN;
}

void* FvmFieldValueIndex(FvmField* v, size_t i) {
    return v ? (void*)((char*)v->_cpu->value + v->_cpu->elem_size * i) : nullptr;
}

void VarGpuToCpu(FvmField* var) {
    clear_error();
    if (var && impl(var) && flush_for(var)) download_values(var);
}

void VarAllGpuToCpu(FvmField* var) {
    clear_error();
    if (var && impl(var) && flush_for(var) && download_values(var)) download_gradients(var);
}

int gbVarCpuToGpu(cuMesh* mesh, FvmField* var) {
    clear_error();
    if (!check_mesh(mesh)) return 1;
    FieldImpl* fi = impl(var);
    if (!fi || !bind(mesh, var, fi->comps, "gbVarCpuToGpu") || !flush_for(var) || !ensure_staging(fi)) return 1;
    cudaStream_t s = t_stream;
    const uint32_t* idx = impl(mesh)->d_cell_new;
    if (!cuda_ok(cudaMemcpyAsync(fi->staging, var->_cpu->value, fi->size * fi->comps * 4, cudaMemcpyHostToDevice, s),
                 "gbVarCpuToGpu"))
        return 1;
    for (int k = 0; k < 2; ++k) {
        if (fi->comps == 1) launch_scatter_scalar((int64_t)fi->size, fi->staging, idx, (float*)fi->val[k], s);
        else launch_scatter_vector((int64_t)fi->size, fi->staging, idx, (float4*)fi->val[k], s);
    }
    fi->partials_valid = false;
    return launch_ok("gbVarCpuToGpu") ? 0 : 1;
}

int FvmEulerInit(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach, gb_scalar pressure,
                 gb_scalar temperature) {
    clear_error();
    if (!check_mesh(mesh) || !bind(mesh, rho, 1, "FvmEulerInit") || !bind(mesh, rhou, 3, "FvmEulerInit") ||
        !bind(mesh, rhoe, 1, "FvmEulerInit") || !flush_bcs(mesh))
        return 1;
    // euler_init, src/models/euler.cu:401-404
    const float r = pressure / temperature;
    const float c = sqrtf(1.4f * pressure / r);
    const float3 vel = make_float3(mach.x * c, mach.y * c, mach.z * c);
    const float3 ru = make_float3(vel.x * r, vel.y * r, vel.z * r);
    const float e = pressure / 0.4f + 0.5f * r * (vel.x * vel.x + vel.y * vel.y + vel.z * vel.z);
    const int64_t n = (int64_t)impl(rho)->size;
    for (int k = 0; k < 2; ++k)
        launch_init(n, (float*)impl(rho)->val[k], (float4*)impl(rhou)->val[k], (float*)impl(rhoe)->val[k], r, ru, e,
                    t_stream);
    impl(rho)->cur = impl(rhou)->cur = impl(rhoe)->cur = 0;
    return launch_ok("FvmEulerInit") ? 0 : 1;
}

int FvmEulerSlipBc(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, const char* region) {
    clear_error();
    if (!euler_fields(mesh, rho, rhou, rhoe, "FvmEulerSlipBc")) return 1;
    const int r = region_lookup(mesh, region);
    if (r < 0) return 1;
    bool ok = true;
    if (defer_bc(mesh, rho, rhou, rhoe, r, 0, gb_vector{0.f, 0.f, 0.f}, 0.f, 0.f, &ok)) return ok ? 0 : 1;
    enqueue_slip(mesh, rho, rhou, rhoe, r, impl(rho)->cur, t_stream);
    return launch_ok("FvmEulerSlipBc") ? 0 : 1;
}

int FvmEulerInletOutletBc(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                          gb_scalar pressure, gb_scalar temperature, const char* region) {
    clear_error();
    if (!euler_fields(mesh, rho, rhou, rhoe, "FvmEulerInletOutletBc")) return 1;
    const int r = region_lookup(mesh, region);
    if (r < 0) return 1;
    bool ok = true;
    if (defer_bc(mesh, rho, rhou, rhoe, r, 1, mach, pressure, temperature, &ok)) return ok ? 0 : 1;
    enqueue_farfield(mesh, rho, rhou, rhoe, r, impl(rho)->cur, mach, pressure, temperature, t_stream);
    return launch_ok("FvmEulerInletOutletBc") ? 0 : 1;
}

int gbApplyBoundaryConditions(cuMesh* mesh) {
    clear_error();
    if (!check_mesh(mesh)) return 1;
    return flush_bcs(mesh) ? 0 : 1;
}

int FvmEulerStepPrepare(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe) {
    clear_error();
    if (!euler_fields(mesh, rho, rhou, rhoe, "FvmEulerStepPrepare") || !flush_bcs(mesh)) return 1;
    if (!ensure_grad(mesh, rho) || !ensure_grad(mesh, rhou) || !ensure_grad(mesh, rhoe)) return 1;
    launch_grad_lim(impl(mesh)->dev, state_of(rho, rhou, rhoe, impl(rho)->cur), grad_of(rho, rhou, rhoe, true),
                    g_transposed.load() != 0, t_stream);
    return launch_ok("FvmEulerStepPrepare") ? 0 : 1;
}

int FvmEulerStep(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_scalar cfl, const char* time_scheme,
                 FvmField* dt, FvmField* error) {
    (void)dt;
    clear_error();
    if (!time_scheme || strcmp(time_scheme, "steady") != 0) {
        set_error("FvmEulerStep: only the \"steady\" scheme exists");
        return 1;
    }
    if (!euler_fields(mesh, rho, rhou, rhoe, "FvmEulerStep") || !bind(mesh, error, 1, "FvmEulerStep") ||
        !flush_bcs(mesh))
        return 1;
    if (!impl(rho)->rec || !impl(rhou)->rec) {
        set_error("FvmEulerStep: call FvmEulerStepPrepare first");
        return 1;
    }
    FieldImpl* ei = impl(error);
    const int nb = (int)((impl(mesh)->dev.N + kBlock - 1) / kBlock);
    if (!ensure_partials(ei, std::max(nb, 1))) return 1;
    const int cur = impl(rho)->cur;
    enqueue_flux(mesh, rho, rhou, rhoe, error, cfl, cur, t_stream);
    if (!launch_ok("FvmEulerStep")) return 1;
    impl(rho)->cur = impl(rhou)->cur = impl(rhoe)->cur = 1 - cur;
    ei->partials_valid = true;
    return 0;
}

gb_scalar FvmFieldReduceSum(cuMesh* mesh, FvmField* var) {
    clear_error();
    const float nan = std::numeric_limits<float>::quiet_NaN();
    if (!check_mesh(mesh) || !bind(mesh, var, 1, "FvmFieldReduceSum") || !flush_for(var)) return nan;
    FieldImpl* fi = impl(var);
    MeshImpl* mi = impl(mesh);
    cudaStream_t s = t_stream;
    double* out = mi->dev.red + mi->dev.n_red_max;
    if (fi->partials_valid) {
        launch_reduce_final((int)((mi->dev.N + kBlock - 1) / kBlock), fi->partials, out, s);
    } else {
        const int nb = reduce_blocks(mi->dev.N);
        launch_reduce_partials(mi->dev.N, (const float*)fi->val[fi->cur], mi->dev.red, s);
        launch_reduce_final(nb, mi->dev.red, out, s);
    }
    // read back through a pinned word: a copy into pageable memory would be
    // staged by the driver
    double* h = mi->h_result;
    if (!launch_ok("FvmFieldReduceSum") ||
        !cuda_ok(cudaMemcpyAsync(h, out, sizeof(double), cudaMemcpyDeviceToHost, s), "FvmFieldReduceSum") ||
        !cuda_ok(cudaStreamSynchronize(s), "FvmFieldReduceSum"))
        return nan;
    return (gb_scalar)*h;
}

static int64_t euler_run(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, FvmField* error, gb_scalar cfl,
                         int64_t n_iter, const gbBc* bcs, int n_bc, double tolerance, int check_every,
                         double* residual_history, double* density_history) {
    clear_error();
    if (n_iter < 0 || n_bc < 0 || (n_bc > 0 && !bcs)) { set_error("gbEulerRun: bad arguments"); return -1; }
    if (!euler_fields(mesh, rho, rhou, rhoe, "gbEulerRun") || !bind(mesh, error, 1, "gbEulerRun") ||
        !flush_bcs(mesh))
        return -1;
    MeshImpl* mi = impl(mesh);
    for (int b = 0; b < n_bc; ++b) {
        if (bcs[b].region_id >= mi->topo.regions.size() || (bcs[b].type != 0 && bcs[b].type != 1)) {
            set_error("gbEulerRun: bad boundary condition " + std::to_string(b));
            return -1;
        }
    }
    if (n_iter == 0) return 0;
    if (!ensure_grad(mesh, rho) || !ensure_grad(mesh, rhou) || !ensure_grad(mesh, rhoe)) return -1;
    FieldImpl* ei = impl(error);
    const int nb = (int)((mi->dev.N + kBlock - 1) / kBlock);
    const bool density = density_history != nullptr;   // the density residual's partials follow the residual's
    if (!ensure_partials(ei, std::max(nb, 1) * (density ? 2 : 1))) return -1;
    if (check_every <= 0) check_every = 100;
    cudaStream_t s = t_stream;
    double* out = mi->dev.red + mi->dev.n_red_max;
    // The boundary conditions as a table by ghost region.  On ghost-heavy
    // meshes (one-layer extrusions carry two span ghosts per cell) the
    // gradient kernel applies them itself; on the others one ghost kernel
    // applies all regions' conditions (it costs less than the extra work in
    // the gradient pass).  Meshes with more regions than the table holds use
    // one ghost kernel per condition.
    const int n_regions = (int)mi->topo.regions.size();
    const bool table_bcs = n_regions > 0 && n_regions <= kMaxBcRegions;
    const bool inline_bcs = table_bcs && 4 * mi->dev.G >= mi->dev.N;
    GhostBcTable gbt{};
    if (table_bcs) {
        gbt.n = n_regions;
        gbt.store = inline_bcs ? 0 : 1;   // the gradient pass's ghost states are stored once, after the loop
        for (int r = 0; r <= n_regions; ++r) gbt.start[r] = mi->num.region_start[r];
        for (int r = 0; r < n_regions; ++r) gbt.type[r] = -1;
        for (int b = 0; b < n_bc; ++b) {   // a later condition on the same region replaces an earlier one
            const int r = (int)bcs[b].region_id;
            gbt.type[r] = bcs[b].type;
            gbt.mach[r] = make_float3(bcs[b].mach.x, bcs[b].mach.y, bcs[b].mach.z);
            gbt.p[r] = bcs[b].pressure;
            gbt.temp[r] = bcs[b].temperature;
        }
        for (int k = 0; k < 2; ++k) {
            gbt.rho[k] = (float*)impl(rho)->val[k];
            gbt.rhou[k] = (float4*)impl(rhou)->val[k];
            gbt.rhoe[k] = (float*)impl(rhoe)->val[k];
        }
    }
    // what the captured launches bake in
    const bool transposed = g_transposed.load() != 0;
    std::vector<uint64_t> key;
    for (const FvmField* f : {rho, rhou, rhoe, error}) key_field(key, f);
    key.push_back((uint64_t)ei->cur);
    key.push_back((uint64_t)transposed);
    key_bytes(key, &cfl, sizeof(cfl));
    key.push_back((uint64_t)n_bc);
    if (n_bc > 0) key_bytes(key, bcs, sizeof(gbBc) * (size_t)n_bc);
    key_bytes(key, &tolerance, sizeof(tolerance));
    key.push_back((uint64_t)density);
    // one graph per value buffer parity: BCs, gradients+limiters, flux+update, residual
    auto enqueue = [&](int k, cudaStream_t cap, const DevMesh& dh, RunCtl* ctl, double* hist,
                       unsigned long long hcap) {
        if (table_bcs && !inline_bcs && n_bc > 0) launch_bc_table(dh, gbt, k, cap);
        for (int b = 0; b < n_bc && !table_bcs; ++b) {
            if (bcs[b].type == 0) enqueue_slip(mesh, rho, rhou, rhoe, (int)bcs[b].region_id, k, cap, &dh);
            else enqueue_farfield(mesh, rho, rhou, rhoe, (int)bcs[b].region_id, k, bcs[b].mach, bcs[b].pressure,
                                  bcs[b].temperature, cap, &dh);
        }
        launch_grad_lim(dh, state_of(rho, rhou, rhoe, k), grad_of(rho, rhou, rhoe, false), transposed, cap,
                        inline_bcs ? &gbt : nullptr);
        enqueue_flux(mesh, rho, rhou, rhoe, error, cfl, k, cap, &dh, density ? ei->partials + nb : nullptr);
        if (density) launch_reduce_history(nb, ei->partials + nb, ctl, hist + hcap, hcap, cap);
        launch_reduce_final(nb, ei->partials, out, cap, ctl, hist, hcap, tolerance);
    };
    const int per_iter = (inline_bcs ? 0 : (table_bcs ? (n_bc > 0 ? 1 : 0) : n_bc)) + 3 + (density ? 1 : 0);
    if (!ensure_run_graphs(mi, mi->euler_run, key, std::min<int64_t>(check_every, n_iter), per_iter, enqueue,
                           "gbEulerRun", density ? 2 : 1))
        return -1;
    int cur = impl(rho)->cur;
    std::vector<double> hist((size_t)n_iter, 0.0), hist_rho(density ? (size_t)n_iter : 0, 0.0);
    const int64_t done = replay_run_graphs(mi->euler_run, cur, n_iter, check_every, hist, s, "gbEulerRun",
                                           density ? &hist_rho : nullptr);
    if (done > 0 && inline_bcs) {
        // the ghost states of the last gradient pass, from the state it read
        // (the buffer before the last update), into both value buffers
        launch_bc_table(mi->dev, gbt, 1 - cur, s);
        if (!launch_ok("gbEulerRun")) return -1;
    }
    impl(rho)->cur = impl(rhou)->cur = impl(rhoe)->cur = cur;
    ei->partials_valid = true;
    if (residual_history && done > 0) memcpy(residual_history, hist.data(), (size_t)done * sizeof(double));
    if (density_history && done > 0) memcpy(density_history, hist_rho.data(), (size_t)done * sizeof(double));
    return done;
}

int64_t gbEulerRun(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, FvmField* error, gb_scalar cfl,
                   int64_t n_iter, const gbBc* bcs, int n_bc, double tolerance, int check_every,
                   double* residual_history) {
    return euler_run(mesh, rho, rhou, rhoe, error, cfl, n_iter, bcs, n_bc, tolerance, check_every, residual_history,
                     nullptr);
}

int64_t gbEulerRunDensityResidual(cuMesh* mesh, FvmField* rho, FvmField* rhou, FvmField* rhoe, FvmField* error,
                                  gb_scalar cfl, int64_t n_iter, const gbBc* bcs, int n_bc, double tolerance,
                                  int check_every, double* residual_history, double* density_history) {
    if (!density_history) {
        clear_error();
        set_error("gbEulerRunDensityResidual: null density history");
        return -1;
    }
    return euler_run(mesh, rho, rhou, rhoe, error, cfl, n_iter, bcs, n_bc, tolerance, check_every, residual_history,
                     density_history);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Incompressible Navier-Stokes by artificial compressibility (nsi.cu).  The
// reference's src/models/nsi.cu drives FvmNSIInit / FvmNSISlipBc /
// FvmNSIInletOutletBc / FvmNSIStepPrepare / FvmNSIStep with fields
// "velocity" (vector) and "pressure" (scalar) but defines none of them; they
// are defined here with those names and argument meanings, plus a no-slip
// wall condition, a replayed-graph loop and the wall force.
namespace gb {
void launch_nsi_init(int64_t n, float* p, float4* u, float p0, float3 u0, cudaStream_t s);
void launch_nsi_bc(const DevMesh& m, uint32_t g0, uint32_t g1, int type, float* p[2], float4* u[2], int cur,
                   float3 vinf, float pinf, cudaStream_t s);
void launch_nsi_grad(const DevMesh& m, const float* p, const float4* u, float4* gp, float4* gu, int limited,
                     cudaStream_t s, const NsiGhostTable* ghosts = nullptr);
void launch_nsi_flux(const DevMesh& m, const float* p, const float4* u, const float4* gp, const float4* gu, float* p_n,
                     float4* u_n, float* err, double* partials, float cfl, float nu, float beta2, int corrected,
                     cudaStream_t s);
int launch_nsi_force(const DevMesh& m, uint32_t g0, uint32_t g1, const float* p, const float4* u, const float4* gu,
                     float nu, int corrected, double density, double* partials, double* out, cudaStream_t s);

namespace {

struct NsiConstants {
    double density = 1.0;
    double viscosity = 0.025;   // Re = 40 for a unit diameter and unit speed
    double beta = 2.0;          // artificial sound speed
    int corrected = 1;
    int limited = 0;
};
thread_local NsiConstants t_nsi;

bool nsi_fields(cuMesh* mesh, FvmField* velocity, FvmField* pressure, const char* what) {
    if (!check_mesh(mesh)) return false;
    if (!bind(mesh, velocity, 3, what) || !bind(mesh, pressure, 1, what)) return false;
    if (impl(velocity)->cur != impl(pressure)->cur) {
        set_error(std::string(what) + ": velocity and pressure were not updated together");
        return false;
    }
    return true;
}

bool nsi_grad(cuMesh* mesh, FvmField* f) {
    FieldImpl* fi = impl(f);
    if (fi->grad) return true;
    const int64_t N = impl(mesh)->topo.N;
    return dalloc(fi->grad, (size_t)N * fi->comps, "alloc gradient") &&
           cuda_ok(cudaMemsetAsync(fi->grad, 0, (size_t)N * fi->comps * sizeof(float4), t_stream), "zero gradient");
}

void enqueue_nsi_bc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, int r, int type, int cur, gb_vector v,
                    float pinf, cudaStream_t s, const DevMesh* dm = nullptr) {
    MeshImpl* mi = impl(mesh);
    float* pp[2] = {(float*)impl(pressure)->val[0], (float*)impl(pressure)->val[1]};
    float4* pu[2] = {(float4*)impl(velocity)->val[0], (float4*)impl(velocity)->val[1]};
    launch_nsi_bc(dm ? *dm : mi->dev, mi->num.region_start[r], mi->num.region_start[r + 1], type, pp, pu, cur,
                  make_float3(v.x, v.y, v.z), pinf, s);
}

void enqueue_nsi_step(cuMesh* mesh, FvmField* velocity, FvmField* pressure, FvmField* error, float cfl, int cur,
                      cudaStream_t s, const NsiGhostTable* ghosts = nullptr, const DevMesh* dm = nullptr) {
    MeshImpl* mi = impl(mesh);
    const DevMesh& d = dm ? *dm : mi->dev;
    FieldImpl *vi = impl(velocity), *pi = impl(pressure), *ei = impl(error);
    launch_nsi_grad(d, (const float*)pi->val[cur], (const float4*)vi->val[cur], pi->grad, vi->grad,
                    t_nsi.limited, s, ghosts);
    launch_nsi_flux(d, (const float*)pi->val[cur], (const float4*)vi->val[cur], pi->grad, vi->grad,
                    (float*)pi->val[1 - cur], (float4*)vi->val[1 - cur], (float*)ei->val[ei->cur], ei->partials, cfl,
                    (float)t_nsi.viscosity, (float)(t_nsi.beta * t_nsi.beta), t_nsi.corrected, s);
}

int nsi_bc_call(cuMesh* mesh, FvmField* velocity, FvmField* pressure, const char* region, int type, gb_vector v,
                float p, const char* what) {
    clear_error();
    if (!nsi_fields(mesh, velocity, pressure, what)) return 1;
    const int r = region_lookup(mesh, region);
    if (r < 0) return 1;
    enqueue_nsi_bc(mesh, velocity, pressure, r, type, impl(pressure)->cur, v, p, t_stream);
    return launch_ok(what) ? 0 : 1;
}

}  // namespace
}  // namespace gb

extern "C" {

int gbNSISetConstants(gb_scalar density, gb_scalar viscosity, gb_scalar beta, int corrected_laplacian, int limited) {
    clear_error();
    if (!(density > 0.f) || !(viscosity >= 0.f) || !(beta > 0.f)) {
        set_error("gbNSISetConstants: density and beta must be positive, viscosity non-negative");
        return 1;
    }
    t_nsi.density = density;
    t_nsi.viscosity = viscosity;
    t_nsi.beta = beta;
    t_nsi.corrected = corrected_laplacian ? 1 : 0;
    t_nsi.limited = limited ? 1 : 0;
    return 0;
}

int FvmNSIInit(cuMesh* mesh, FvmField* velocity, FvmField* pressure, gb_vector init_velocity, gb_scalar init_pressure) {
    clear_error();
    if (!nsi_fields(mesh, velocity, pressure, "FvmNSIInit")) return 1;
    const int64_t n = (int64_t)impl(pressure)->size;
    for (int k = 0; k < 2; ++k)
        launch_nsi_init(n, (float*)impl(pressure)->val[k], (float4*)impl(velocity)->val[k], init_pressure,
                        make_float3(init_velocity.x, init_velocity.y, init_velocity.z), t_stream);
    return launch_ok("FvmNSIInit") ? 0 : 1;
}

int FvmNSISlipBc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, const char* region) {
    return nsi_bc_call(mesh, velocity, pressure, region, 0, gb_vector{0.f, 0.f, 0.f}, 0.f, "FvmNSISlipBc");
}

int FvmNSIWallBc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, const char* region) {
    return nsi_bc_call(mesh, velocity, pressure, region, 2, gb_vector{0.f, 0.f, 0.f}, 0.f, "FvmNSIWallBc");
}

int FvmNSIInletOutletBc(cuMesh* mesh, FvmField* velocity, FvmField* pressure, gb_vector inlet_velocity,
                        gb_scalar outlet_pressure, const char* region) {
    return nsi_bc_call(mesh, velocity, pressure, region, 1, inlet_velocity, outlet_pressure, "FvmNSIInletOutletBc");
}

int FvmNSIStepPrepare(cuMesh* mesh, FvmField* velocity, FvmField* pressure) {
    clear_error();
    if (!nsi_fields(mesh, velocity, pressure, "FvmNSIStepPrepare")) return 1;
    if (!nsi_grad(mesh, velocity) || !nsi_grad(mesh, pressure)) return 1;
    const int cur = impl(pressure)->cur;
    launch_nsi_grad(impl(mesh)->dev, (const float*)impl(pressure)->val[cur], (const float4*)impl(velocity)->val[cur],
                    impl(pressure)->grad, impl(velocity)->grad, t_nsi.limited, t_stream);
    return launch_ok("FvmNSIStepPrepare") ? 0 : 1;
}

int FvmNSIStep(cuMesh* mesh, FvmField* velocity, FvmField* pressure, gb_scalar cfl, const char* time_scheme,
               FvmField* dt, FvmField* error) {
    (void)dt;
    clear_error();
    if (!time_scheme || strcmp(time_scheme, "steady") != 0) {
        set_error("FvmNSIStep: only the \"steady\" scheme exists");
        return 1;
    }
    if (!nsi_fields(mesh, velocity, pressure, "FvmNSIStep") || !bind(mesh, error, 1, "FvmNSIStep")) return 1;
    if (!impl(velocity)->grad || !impl(pressure)->grad) {
        set_error("FvmNSIStep: call FvmNSIStepPrepare first");
        return 1;
    }
    MeshImpl* mi = impl(mesh);
    FieldImpl* ei = impl(error);
    const int nb = (int)((mi->dev.N + kBlock - 1) / kBlock);
    if (!ensure_partials(ei, std::max(nb, 1))) return 1;
    const int cur = impl(pressure)->cur;
    FieldImpl *vi = impl(velocity), *pi = impl(pressure);
    launch_nsi_flux(mi->dev, (const float*)pi->val[cur], (const float4*)vi->val[cur], pi->grad, vi->grad,
                    (float*)pi->val[1 - cur], (float4*)vi->val[1 - cur], (float*)ei->val[ei->cur], ei->partials, cfl,
                    (float)t_nsi.viscosity, (float)(t_nsi.beta * t_nsi.beta), t_nsi.corrected, t_stream);
    if (!launch_ok("FvmNSIStep")) return 1;
    vi->cur = pi->cur = 1 - cur;
    ei->partials_valid = true;
    return 0;
}

int64_t gbNSIRun(cuMesh* mesh, FvmField* velocity, FvmField* pressure, FvmField* error, gb_scalar cfl, int64_t n_iter,
                 const gbBc* bcs, int n_bc, double tolerance, int check_every, double* residual_history) {
    clear_error();
    if (n_iter < 0 || n_bc < 0 || (n_bc > 0 && !bcs)) { set_error("gbNSIRun: bad arguments"); return -1; }
    if (!nsi_fields(mesh, velocity, pressure, "gbNSIRun") || !bind(mesh, error, 1, "gbNSIRun")) return -1;
    MeshImpl* mi = impl(mesh);
    for (int b = 0; b < n_bc; ++b)
        if (bcs[b].region_id >= mi->topo.regions.size() || bcs[b].type < 0 || bcs[b].type > 2) {
            set_error("gbNSIRun: bad boundary condition " + std::to_string(b));
            return -1;
        }
    if (n_iter == 0) return 0;
    if (!nsi_grad(mesh, velocity) || !nsi_grad(mesh, pressure)) return -1;
    FieldImpl* ei = impl(error);
    const int nb = (int)((mi->dev.N + kBlock - 1) / kBlock);
    if (!ensure_partials(ei, std::max(nb, 1))) return -1;
    if (check_every <= 0) check_every = 100;
    cudaStream_t s = t_stream;
    double* out = mi->dev.red + mi->dev.n_red_max;
    // On ghost-heavy meshes (one-layer extrusions carry two span ghosts per
    // cell) the gradient kernel applies the boundary conditions itself
    // (NsiGhostTable); on the others the ghost kernels cost less than the
    // extra work in the gradient pass.
    const int n_regions = (int)mi->topo.regions.size();
    const bool inline_bcs = n_regions > 0 && n_regions <= kMaxNsiRegions && 4 * mi->dev.G >= mi->dev.N;
    NsiGhostTable gt{};
    if (inline_bcs) {
        gt.n = n_regions;
        for (int r = 0; r <= n_regions; ++r) gt.start[r] = mi->num.region_start[r];
        for (int r = 0; r < n_regions; ++r) gt.type[r] = -1;
        for (int b = 0; b < n_bc; ++b) {   // a later condition on the same region replaces an earlier one
            const int r = (int)bcs[b].region_id;
            gt.type[r] = bcs[b].type == 1 ? 1 : (bcs[b].type == 2 ? 2 : 0);
            gt.vinf[r] = make_float3(bcs[b].mach.x, bcs[b].mach.y, bcs[b].mach.z);
            gt.pinf[r] = bcs[b].pressure;
        }
        for (int k = 0; k < 2; ++k) {
            gt.p[k] = (float*)impl(pressure)->val[k];
            gt.u[k] = (float4*)impl(velocity)->val[k];
        }
    }
    std::vector<uint64_t> key;
    for (const FvmField* f : {velocity, pressure, error}) key_field(key, f);
    key.push_back((uint64_t)ei->cur);
    key_bytes(key, &cfl, sizeof(cfl));
    key.push_back((uint64_t)n_bc);
    if (n_bc > 0) key_bytes(key, bcs, sizeof(gbBc) * (size_t)n_bc);
    key_bytes(key, &t_nsi, sizeof(t_nsi));
    key_bytes(key, &tolerance, sizeof(tolerance));
    auto enqueue = [&](int k, cudaStream_t cap, const DevMesh& dh, RunCtl* ctl, double* hist,
                       unsigned long long hcap) {
        for (int b = 0; b < n_bc && !inline_bcs; ++b) {
            const int type = bcs[b].type == 1 ? 1 : (bcs[b].type == 2 ? 2 : 0);
            enqueue_nsi_bc(mesh, velocity, pressure, (int)bcs[b].region_id, type, k, bcs[b].mach, bcs[b].pressure, cap,
                           &dh);
        }
        enqueue_nsi_step(mesh, velocity, pressure, error, cfl, k, cap, inline_bcs ? &gt : nullptr, &dh);
        launch_reduce_final(nb, ei->partials, out, cap, ctl, hist, hcap, tolerance);
    };
    const int per_iter = (inline_bcs ? 0 : n_bc) + 3;
    if (!ensure_run_graphs(mi, mi->nsi_run, key, std::min<int64_t>(check_every, n_iter), per_iter, enqueue,
                           "gbNSIRun"))
        return -1;
    int cur = impl(pressure)->cur;
    std::vector<double> hist((size_t)n_iter, 0.0);
    const int64_t done = replay_run_graphs(mi->nsi_run, cur, n_iter, check_every, hist, s, "gbNSIRun");
    impl(velocity)->cur = impl(pressure)->cur = cur;
    ei->partials_valid = true;
    if (residual_history && done > 0) memcpy(residual_history, hist.data(), (size_t)done * sizeof(double));
    return done;
}

int gbNSIWallForce(cuMesh* mesh, FvmField* velocity, FvmField* pressure, unsigned region_id, double* force) {
    clear_error();
    if (!force) { set_error("gbNSIWallForce: null output"); return 1; }
    if (!nsi_fields(mesh, velocity, pressure, "gbNSIWallForce")) return 1;
    MeshImpl* mi = impl(mesh);
    if (region_id >= mi->topo.regions.size()) { set_error("gbNSIWallForce: unknown region"); return 1; }
    if (!impl(velocity)->grad) { set_error("gbNSIWallForce: call FvmNSIStepPrepare or gbNSIRun first"); return 1; }
    const uint32_t g0 = mi->num.region_start[region_id], g1 = mi->num.region_start[region_id + 1];
    force[0] = force[1] = force[2] = 0.0;
    if (g1 <= g0) return 0;
    const int blocks = (int)((g1 - g0 + kBlock - 1) / kBlock);
    double* d = nullptr;
    if (!dalloc(d, (size_t)3 * blocks + 3, "gbNSIWallForce")) return 1;
    const int cur = impl(pressure)->cur;
    cudaStream_t s = t_stream;
    // the gradient of the current state (the one stored may be a step old)
    launch_nsi_grad(mi->dev, (const float*)impl(pressure)->val[cur], (const float4*)impl(velocity)->val[cur],
                    impl(pressure)->grad, impl(velocity)->grad, t_nsi.limited, s);
    launch_nsi_force(mi->dev, g0, g1, (const float*)impl(pressure)->val[cur], (const float4*)impl(velocity)->val[cur],
                     impl(velocity)->grad, (float)t_nsi.viscosity, t_nsi.corrected, t_nsi.density, d, d + 3 * blocks,
                     s);
    const bool ok = launch_ok("gbNSIWallForce") &&
                    cuda_ok(cudaMemcpyAsync(force, d + 3 * blocks, 3 * sizeof(double), cudaMemcpyDeviceToHost, s),
                            "gbNSIWallForce") &&
                    cuda_ok(cudaStreamSynchronize(s), "gbNSIWallForce");
    dfree(d);
    return ok ? 0 : 1;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Generic finite-volume operators (fvmops.cu).
namespace gb {
void launch_fvm_grad(const DevMesh& m, int comps, const float* s, const float4* v, float4* grad, cudaStream_t st);
void launch_field_init(int64_t n, int comps, void* val0, void* val1, float4 value, int64_t n_grad, float4* grad,
                       cudaStream_t st);
void launch_field_bc(const DevMesh& m, uint32_t g0, uint32_t g1, int comps, int zero_grad, int cur, void* val0,
                     void* val1, float4 value, cudaStream_t st);
void launch_field_axpy(const DevMesh& m, int comps, float a, const void* x, void* y, cudaStream_t st);
void launch_fvm_apply(const DevMesh& m, int op, const float* s, const float4* v, const float4* g, const float4* phi,
                      float3 phi_c, float* out, cudaStream_t st);
}  // namespace gb

extern "C" {

int gbFieldInit(cuMesh* mesh, FvmField* u, gb_vector value) {
    clear_error();
    if (!check_mesh(mesh)) return 1;
    FieldImpl* fi = impl(u);
    if (!fi || !bind(mesh, u, fi->comps, "gbFieldInit") || !flush_for(u)) return 1;
    const int64_t n_grad = fi->grad ? impl(mesh)->dev.N * fi->comps : 0;
    launch_field_init((int64_t)fi->size, fi->comps, fi->val[0], fi->val[1], make_float4(value.x, value.y, value.z, 0.f),
                      n_grad, fi->grad, t_stream);
    return launch_ok("gbFieldInit") ? 0 : 1;
}

static int field_bc(cuMesh* mesh, FvmField* u, unsigned int region_id, int zero_grad, gb_vector value,
                    const char* what) {
    clear_error();
    if (!check_mesh(mesh)) return 1;
    FieldImpl* fi = impl(u);
    if (!fi || !bind(mesh, u, fi->comps, what) || !flush_for(u)) return 1;
    MeshImpl* mi = impl(mesh);
    if (region_id >= mi->topo.regions.size()) {
        set_error(std::string(what) + ": no region " + std::to_string(region_id));
        return 1;
    }
    launch_field_bc(mi->dev, mi->num.region_start[region_id], mi->num.region_start[region_id + 1], fi->comps, zero_grad,
                    fi->cur, fi->val[0], fi->val[1], make_float4(value.x, value.y, value.z, 0.f), t_stream);
    return launch_ok(what) ? 0 : 1;
}

int gbFieldBcFixed(cuMesh* mesh, FvmField* u, gb_vector value, unsigned int region_id) {
    return field_bc(mesh, u, region_id, 0, value, "gbFieldBcFixed");
}

int gbFieldBcZeroGrad(cuMesh* mesh, FvmField* u, unsigned int region_id) {
    return field_bc(mesh, u, region_id, 1, gb_vector{0.f, 0.f, 0.f}, "gbFieldBcZeroGrad");
}

int gbFieldAxpy(cuMesh* mesh, FvmField* y, gb_scalar a, FvmField* x) {
    clear_error();
    if (!check_mesh(mesh)) return 1;
    FieldImpl* fy = impl(y);
    FieldImpl* fx = impl(x);
    if (!fy || !fx) { set_error("gbFieldAxpy: null field"); return 1; }
    if (x == y) { set_error("gbFieldAxpy: x and y are the same field"); return 1; }
    if (!bind(mesh, y, fy->comps, "gbFieldAxpy") || !bind(mesh, x, fy->comps, "gbFieldAxpy") || !flush_for(x) ||
        !flush_for(y))
        return 1;
    launch_field_axpy(impl(mesh)->dev, fy->comps, a, fx->val[fx->cur], fy->val[fy->cur], t_stream);
    return launch_ok("gbFieldAxpy") ? 0 : 1;
}

int gbFvmGradient(cuMesh* mesh, FvmField* u) {
    clear_error();
    if (!check_mesh(mesh)) return 1;
    FieldImpl* fi = impl(u);
    if (!fi || !bind(mesh, u, fi->comps, "gbFvmGradient") || !flush_for(u) || !nsi_grad(mesh, u)) return 1;
    launch_fvm_grad(impl(mesh)->dev, fi->comps, fi->comps == 1 ? (const float*)fi->val[fi->cur] : nullptr,
                    fi->comps == 3 ? (const float4*)fi->val[fi->cur] : nullptr, fi->grad, t_stream);
    return launch_ok("gbFvmGradient") ? 0 : 1;
}

}  // extern "C"

namespace {
// by operator id (GB_FVM_*): components of the input field and of the
// output, whether the operator reads the input's gradient
constexpr int kFvmOps = 11;
const int kOpInComps[kFvmOps] = {1, 1, 1, 3, 1, 3, 3, 1, 1, 1, 3};
const int kOpOutComps[kFvmOps] = {1, 3, 3, 9, 3, 9, 1, 1, 1, 1, 3};
const bool kOpNeedsGrad[kFvmOps] = {true, false, true, false, false, false, false, false, true, false, false};
}  // namespace

extern "C" {

int gbFvmApplyTerms(cuMesh* mesh, int n_terms, const gbFvmTerm* terms, FvmField* out) {
    clear_error();
    const char* what = "gbFvmApplyTerms";
    if (!check_mesh(mesh)) return 1;
    if (!terms || n_terms < 1 || n_terms > kFvmMaxTerms) {
        set_error("gbFvmApplyTerms: between 1 and " + std::to_string(kFvmMaxTerms) + " terms");
        return 1;
    }
    FvmTermDev dt[kFvmMaxTerms];
    int oc = 0;
    for (int q = 0; q < n_terms; ++q) {
        const gbFvmTerm& t = terms[q];
        const std::string tq = "gbFvmApplyTerms: term " + std::to_string(q);
        if (t.op < 0 || t.op >= kFvmOps) { set_error(tq + ": unknown operator"); return 1; }
        if (kOpOutComps[t.op] == 9) { set_error(tq + ": tensor-valued operators have no field form"); return 1; }
        if (q > 0 && kOpOutComps[t.op] != oc) { set_error(tq + ": every term must give the same kind of value"); return 1; }
        oc = kOpOutComps[t.op];
        FieldImpl* fi = impl(t.u);
        if (!fi) { set_error(tq + ": null field"); return 1; }
        if (!bind(mesh, t.u, kOpInComps[t.op], what) || !flush_for(t.u)) return 1;
        if (kOpNeedsGrad[t.op] && !fi->grad) { set_error(tq + ": the operator needs the field's gradient (gbFvmGradient)"); return 1; }
        const float4* phi_v = nullptr;
        if (t.op == 9 || t.op == 10) {
            if (!t.phi) { set_error(tq + ": the operator needs a vector field phi"); return 1; }
            if (!bind(mesh, t.phi, 3, what) || !flush_for(t.phi)) return 1;
            phi_v = (const float4*)impl(t.phi)->val[impl(t.phi)->cur];
        }
        if (out == t.u || out == t.phi) { set_error(tq + ": the output field is also an input"); return 1; }
        dt[q] = FvmTermDev{t.op, t.coef, fi->comps == 1 ? (const float*)fi->val[fi->cur] : nullptr,
                           fi->comps == 3 ? (const float4*)fi->val[fi->cur] : nullptr, fi->grad, phi_v,
                           make_float3(t.phi_const.x, t.phi_const.y, t.phi_const.z)};
    }
    if (!out) { set_error("gbFvmApplyTerms: null output field"); return 1; }
    if (!bind(mesh, out, oc, what) || !flush_for(out)) return 1;
    FieldImpl* fo = impl(out);
    launch_fvm_terms(impl(mesh)->dev, oc, n_terms, dt, oc == 1 ? (float*)fo->val[fo->cur] : nullptr,
                     oc == 3 ? (float4*)fo->val[fo->cur] : nullptr, t_stream);
    return launch_ok(what) ? 0 : 1;
}

int gbFvmApply(cuMesh* mesh, int op, FvmField* u, FvmField* phi, gb_vector phi_const, float* out) {
    clear_error();
    if (!check_mesh(mesh) || !out) { if (!out) set_error("gbFvmApply: null output"); return 1; }
    FieldImpl* fi = impl(u);
    if (!fi) { set_error("gbFvmApply: null field"); return 1; }
    const int* in_comps = kOpInComps;
    const int* out_comps = kOpOutComps;
    const bool* needs_grad = kOpNeedsGrad;
    if (op < 0 || op >= kFvmOps) { set_error("gbFvmApply: unknown operator"); return 1; }
    if (!bind(mesh, u, in_comps[op], "gbFvmApply") || !flush_for(u)) return 1;
    if (needs_grad[op] && !fi->grad) { set_error("gbFvmApply: the operator needs the field's gradient (gbFvmGradient)"); return 1; }
    const float4* phi_v = nullptr;
    if (op == 9 || op == 10) {
        if (!phi || !bind(mesh, phi, 3, "gbFvmApply") || !flush_for(phi)) { if (!phi) set_error("gbFvmApply: the operator needs a vector field phi"); return 1; }
        phi_v = (const float4*)impl(phi)->val[impl(phi)->cur];
    }
    MeshImpl* mi = impl(mesh);
    const int64_t N = mi->dev.N;
    const int oc = out_comps[op];
    float *d_out = nullptr, *d_ref = nullptr;
    if (!dalloc(d_out, (size_t)oc * N, "gbFvmApply") || !dalloc(d_ref, (size_t)oc * N, "gbFvmApply")) {
        dfree(d_out); dfree(d_ref);
        return 1;
    }
    cudaStream_t s = t_stream;
    launch_fvm_apply(mi->dev, op, fi->comps == 1 ? (const float*)fi->val[fi->cur] : nullptr,
                     fi->comps == 3 ? (const float4*)fi->val[fi->cur] : nullptr, fi->grad, phi_v,
                     make_float3(phi_const.x, phi_const.y, phi_const.z), d_out, s);
    for (int q = 0; q < oc; ++q) launch_gather_scalar(N, d_out + (size_t)q * N, mi->d_cell_new, d_ref + (size_t)q * N, s);
    std::vector<float> h((size_t)oc * N);
    const bool ok = launch_ok("gbFvmApply") &&
                    cuda_ok(cudaMemcpyAsync(h.data(), d_ref, h.size() * sizeof(float), cudaMemcpyDeviceToHost, s),
                            "gbFvmApply") &&
                    cuda_ok(cudaStreamSynchronize(s), "gbFvmApply");
    dfree(d_out);
    dfree(d_ref);
    if (!ok) return 1;
    for (int64_t i = 0; i < N; ++i)
        for (int q = 0; q < oc; ++q) out[i * oc + q] = h[(size_t)q * N + i];
    return 0;
}

}  // extern "C"
