// fvm_oracle.cpp -- CPU oracle for the explicit second-order unstructured
// finite-volume Euler iteration of Alexsimulation/graphite.
//
// TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.  Only tests/, the smoke check
// in __graft_entry__.py and bench.py's CPU-baseline leg load this library
// (oracle/_build/liboracle.so), and only to check results against / as the
// timed CPU restatement.  The product path (graphite_b200/) never calls it.
//
// It restates, function by function, the reference's algorithm in plain C++
// (templated on float/double, OpenMP over cells):
//   * mesh conversion semantics of cuMeshFromSu2   src/meshio.cu:713-764, 978-1136
//       - per-element local face lists               src/meshio.cu:315-475
//       - a face keeps the node order of the first element that lists it
//       - ghost cell per boundary face, ids n_elems + region offset + i
//       - cell->face CSR in element-local face order, connect = other cell
//   * metrics  cuMeshComputeFaces/Cells/GhostCells/CellMatrices  src/mesh.cu:44-219
//   * LSQ gradients (scalar / vector)              src/fvmops.cu:51-111
//   * limiter and limiter kernels                  src/fvmops.cu:118-266
//   * ghost gradient/limiter copy                  src/fvmops.cu:272-304
//   * euler_init / euler_slip_bc / euler_inletoutlet_bc  src/models/euler.cu:385-520
//   * fvmEulerSteadyOp + euler_steady_step         src/models/euler.cu:236-381,
//     with the per-face setup of fvmOpVoidSetup    include/fvmops.cuh:61-72
//   * FvmFieldReduceSum                            src/fvmops.cu:369-383
//   * vector helpers outer_normal / tensor*vector / lsqrt
//                                                  include/datatypes.cuh:144-150,296-302,375-377
//
// Deliberate differences, all documented at their use:
//   * the update is Jacobi (reads the old state, writes a new one); the
//     reference updates in place while neighbours read (a data race), which
//     has the same fixed point;
//   * arithmetic is done in T throughout (the reference mixes float with
//     double literals and is built with --use_fast_math), so float results
//     agree with the reference to rounding, not bitwise;
//   * sign(0) is +1 in both precisions (the reference's double overload
//     returns 0, include/datatypes.cuh:209-211);
//   * the residual sum accumulates in double.
//
// Parity of this oracle is pinned against outputs of the reference itself
// (tests/golden/*.npz, produced by tests/golden/make_golden.py running the
// headless reference build oracle/_ref/ref_driver on a GPU).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T> inline V3<T> mk(T x, T y, T z) { return {x, y, z}; }
template <typename T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline V3<T> operator*(V3<T> a, T b) { return {a.x * b, a.y * b, a.z * b}; }
template <typename T> inline V3<T> operator/(V3<T> a, T b) { return {a.x / b, a.y / b, a.z / b}; }
template <typename T> inline V3<T> mul(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <typename T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline T norm(V3<T> a) { return std::sqrt(dot(a, a)); }
template <typename T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// include/datatypes.cuh:144-150 (float overload): sign(x) = +1 for x >= 0.
template <typename T> inline T sgn(T x) { return (T)(x >= 0) - (T)(x < 0); }
template <typename T> inline V3<T> outer_normal(V3<T> n, V3<T> d) { return n * sgn(dot(n, d)); }
// include/datatypes.cuh:375-377
template <typename T> inline T lsqrt(T x) { return std::sqrt(std::fmax((T)1e-12, std::fmin((T)1e30, x))); }

// Tensor stored as three columns u, v, w (include/datatypes.cuh:52-54);
// tensor * vector is the column combination u*x.x + v*x.y + w*x.z
// (include/datatypes.cuh:296-302).
template <typename T>
struct T3 {
    V3<T> u, v, w;
};
template <typename T> inline V3<T> tmul(const T3<T>& a, V3<T> x) {
    return {a.u.x * x.x + a.v.x * x.y + a.w.x * x.z,
            a.u.y * x.x + a.v.y * x.y + a.w.y * x.z,
            a.u.z * x.x + a.v.z * x.y + a.w.z * x.z};
}

// Local faces per SU2 element kind, as listed by su2KindToFaces
// (src/meshio.cu:315-475); -1 pads triangles.
bool local_faces(int kind, std::vector<std::vector<int>>& out) {
    out.clear();
    switch (kind) {
    case 5: out = {{0, 1, 2}}; return true;
    case 9: out = {{0, 1, 2, 3}}; return true;
    case 10: out = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}}; return true;
    case 12: out = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}, {3, 2, 1, 0}, {4, 5, 6, 7}}; return true;
    case 13: out = {{0, 1, 2}, {3, 5, 4}, {0, 2, 5, 3}, {1, 4, 5, 2}, {1, 0, 3, 4}}; return true;
    case 14: out = {{0, 1, 2, 3}, {0, 4, 3}, {0, 1, 4}, {1, 2, 4}, {2, 3, 4}}; return true;
    }
    return false;
}

struct KeyHash {
    size_t operator()(const std::vector<int64_t>& k) const {
        uint64_t h = 1469598103934665603ull;
        for (int64_t v : k) { h ^= (uint64_t)v; h *= 1099511628211ull; }
        return (size_t)h;
    }
};

struct Mesh {
    int64_t N = 0, G = 0, F = 0, n_nodes = 0, n_regions = 0;
    std::vector<double> nodes;                 // 3 per node
    std::vector<int64_t> cfs, cf, cc;          // cell_faces_starts, cell_faces, cell_connects
    std::vector<int64_t> fns, fn;              // face_nodes_starts, face_nodes
    std::vector<int64_t> ghost_ids, ghost_starts;
    std::vector<std::string> region_names;
    // metrics, stored in double whatever precision computed them
    std::vector<double> face_area, face_normal, face_center, cell_volume, cell_center, cell_matrix;
    int metric_bits = 64;
};

template <typename M>
void compute_metrics(Mesh& m) {
    const int64_t F = m.F, N = m.N, G = m.G;
    auto node = [&](int64_t i) { return mk<M>((M)m.nodes[3 * i], (M)m.nodes[3 * i + 1], (M)m.nodes[3 * i + 2]); };
    std::vector<V3<M>> fc(F), fnrm(F);
    std::vector<M> fa(F);
    // cuMeshComputeFaces, src/mesh.cu:44-97
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < F; ++i) {
        const int64_t s = m.fns[i], e = m.fns[i + 1];
        V3<M> center = mk<M>(0, 0, 0);
        for (int64_t n = s; n < e; ++n) center = center + node(m.fn[n]);
        center = center / (M)(e - s);
        V3<M> new_center = mk<M>(0, 0, 0), normal = mk<M>(0, 0, 0);
        M area = 0;
        for (int64_t n0 = s; n0 < e; ++n0) {
            const int64_t n1 = (n0 + 1 < e) ? n0 + 1 : s;   // last edge closes the fan
            V3<M> d0 = center - node(m.fn[n0]);
            V3<M> d1 = center - node(m.fn[n1]);
            V3<M> new_cn = (node(m.fn[n0]) + node(m.fn[n1]) + center) / (M)3;
            V3<M> c = cross(d0, d1);
            M nc = norm(c);
            area += nc * (M)0.5;
            normal = normal + c;
            new_center = new_center + new_cn * nc * (M)0.5;
        }
        fc[i] = new_center / area;
        fnrm[i] = normal / norm(normal);
        fa[i] = area;
    }
    std::vector<V3<M>> cc(N + G);
    std::vector<M> cv(N + G);
    // cuMeshComputeCells, src/mesh.cu:102-143 (an approximate centroid:
    // area-weighted face centres, then a 0.75-pyramid-centroid correction)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        const int64_t s = m.cfs[i], e = m.cfs[i + 1];
        V3<M> center = mk<M>(0, 0, 0);
        M weight = 0;
        for (int64_t k = s; k < e; ++k) {
            const int64_t f = m.cf[k];
            center = center + fc[f] * fa[f];
            weight += fa[f];
        }
        center = center / weight;
        V3<M> new_center = mk<M>(0, 0, 0);
        weight = 0;
        for (int64_t k = s; k < e; ++k) {
            const int64_t f = m.cf[k];
            V3<M> d = fc[f] - center;
            M w = norm(d) * fa[f];
            V3<M> pc = center + d * (M)0.75;
            new_center = new_center + pc * w;
            weight += w;
        }
        new_center = new_center / weight;
        cc[i] = new_center;
        M volume = 0;
        for (int64_t k = s; k < e; ++k) {
            const int64_t f = m.cf[k];
            V3<M> ctf = fc[f] - new_center;
            V3<M> nrm = outer_normal(fnrm[f], ctf);
            volume += dot(ctf, nrm) * fa[f];
        }
        cv[i] = volume / (M)3;
    }
    // cuMeshComputeGhostCells, src/mesh.cu:148-173
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < G; ++t) {
        const int64_t i = m.ghost_ids[t];
        const int64_t other = m.cc[m.cfs[i]];
        const int64_t f = m.cf[m.cfs[i]];
        V3<M> oc = cc[other];
        M dx = norm(fc[f] - oc);
        cc[i] = fc[f] + outer_normal(fnrm[f], fc[f] - oc) * dx;
        cv[i] = fa[f] * (M)2 * dx;
    }
    std::vector<T3<M>> mat(N);
    // cuMeshComputeCellMatrices, src/mesh.cu:178-219: inverse of
    // sum_j d d^T / |d|^2 by adjugate / determinant.
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        T3<M> A{mk<M>(0, 0, 0), mk<M>(0, 0, 0), mk<M>(0, 0, 0)};
        for (int64_t k = m.cfs[i]; k < m.cfs[i + 1]; ++k) {
            V3<M> d = cc[m.cc[k]] - cc[i];
            M w = (M)1 / norm(d);
            // outer(d, d) = columns d*d.x, d*d.y, d*d.z
            A.u = A.u + d * d.x * w * w;
            A.v = A.v + d * d.y * w * w;
            A.w = A.w + d * d.z * w * w;
        }
        T3<M> Mx;
        Mx.u.x = A.v.y * A.w.z - A.v.z * A.w.y;
        Mx.u.y = A.w.y * A.u.z - A.w.z * A.u.y;
        Mx.u.z = A.u.y * A.v.z - A.u.z * A.v.y;
        Mx.v.x = A.w.x * A.v.z - A.w.z * A.v.x;
        Mx.v.y = A.u.x * A.w.z - A.u.z * A.w.x;
        Mx.v.z = A.v.x * A.u.z - A.v.z * A.u.x;
        Mx.w.x = A.v.x * A.w.y - A.v.y * A.w.x;
        Mx.w.y = A.w.x * A.u.y - A.w.y * A.u.x;
        Mx.w.z = A.u.x * A.v.y - A.u.y * A.v.x;
        M det = A.u.x * Mx.u.x + A.v.x * Mx.u.y + A.w.x * Mx.u.z;
        mat[i] = T3<M>{Mx.u / det, Mx.v / det, Mx.w / det};
    }
    m.face_area.resize(F);
    m.face_normal.resize(3 * F);
    m.face_center.resize(3 * F);
    for (int64_t i = 0; i < F; ++i) {
        m.face_area[i] = fa[i];
        m.face_normal[3 * i] = fnrm[i].x; m.face_normal[3 * i + 1] = fnrm[i].y; m.face_normal[3 * i + 2] = fnrm[i].z;
        m.face_center[3 * i] = fc[i].x; m.face_center[3 * i + 1] = fc[i].y; m.face_center[3 * i + 2] = fc[i].z;
    }
    m.cell_volume.resize(N + G);
    m.cell_center.resize(3 * (N + G));
    for (int64_t i = 0; i < N + G; ++i) {
        m.cell_volume[i] = cv[i];
        m.cell_center[3 * i] = cc[i].x; m.cell_center[3 * i + 1] = cc[i].y; m.cell_center[3 * i + 2] = cc[i].z;
    }
    m.cell_matrix.resize(9 * N);
    for (int64_t i = 0; i < N; ++i) {
        const M* p = &mat[i].u.x;
        for (int k = 0; k < 9; ++k) m.cell_matrix[9 * i + k] = p[k];
    }
}

// Conversion semantics of cuMeshFromSu2, src/meshio.cu:713-764 and 978-1136.
Mesh* build_mesh(int64_t n_nodes, const double* nodes, int64_t n_elems, const int32_t* kinds,
                 const int64_t* eoff, const int64_t* enodes, int64_t n_regions, const char* names,
                 const int64_t* roff, const int32_t* bkinds, const int64_t* boff, const int64_t* bnodes,
                 int metric_bits) {
    Mesh* m = new Mesh();
    m->n_nodes = n_nodes;
    m->nodes.assign(nodes, nodes + 3 * n_nodes);
    m->N = n_elems;
    m->n_regions = n_regions;
    m->G = roff[n_regions];
    const int64_t NG = m->N + m->G;
    const char* p = names;
    for (int64_t r = 0; r < n_regions; ++r) {
        m->region_names.emplace_back(p);
        p += strlen(p) + 1;
    }
    std::unordered_map<std::vector<int64_t>, int64_t, KeyHash> index;
    std::vector<std::vector<int64_t>> face_cells;
    std::vector<std::vector<int>> lf;
    std::vector<int64_t> key;
    m->fns.push_back(0);
    // su2ComputeFaces, src/meshio.cu:713-764: faces of interior elements in
    // element order; a new face keeps this element's node order.
    for (int64_t e = 0; e < n_elems; ++e) {
        if (!local_faces(kinds[e], lf) || kinds[e] == 5 || kinds[e] == 9) {
            g_err = "unknown or non-volume element kind " + std::to_string(kinds[e]);
            delete m;
            return nullptr;
        }
        for (auto& f : lf) {
            key.clear();
            for (int v : f) key.push_back(enodes[eoff[e] + v]);
            std::vector<int64_t> sk = key;
            std::sort(sk.begin(), sk.end());
            auto it = index.find(sk);
            if (it == index.end()) {
                int64_t id = (int64_t)face_cells.size();
                index.emplace(sk, id);
                face_cells.push_back({e});
                for (int64_t v : key) m->fn.push_back(v);
                m->fns.push_back((int64_t)m->fn.size());
            } else {
                face_cells[it->second].push_back(e);
            }
        }
    }
    m->F = (int64_t)face_cells.size();
    // Ghost cells: src/meshio.cu:978-1007, gid = n_elems + region start + i.
    for (int64_t r = 0; r < n_regions; ++r) {
        for (int64_t b = roff[r]; b < roff[r + 1]; ++b) {
            key.assign(bnodes + boff[b], bnodes + boff[b + 1]);
            std::sort(key.begin(), key.end());
            auto it = index.find(key);
            if (it == index.end()) {
                g_err = "boundary face " + std::to_string(b) + " matches no element face";
                delete m;
                return nullptr;
            }
            face_cells[it->second].push_back(n_elems + b);
            m->ghost_ids.push_back(n_elems + b);
        }
    }
    m->ghost_starts.assign(roff, roff + n_regions + 1);
    for (int64_t f = 0; f < m->F; ++f) {
        if (face_cells[f].size() != 2) {  // src/meshio.cu:1115-1128
            g_err = "face " + std::to_string(f) + " has " + std::to_string(face_cells[f].size()) + " cells, must be 2";
            delete m;
            return nullptr;
        }
    }
    // Cell->face CSR in element-local face order, src/meshio.cu:1044-1136.
    m->cfs.push_back(0);
    for (int64_t c = 0; c < NG; ++c) {
        int kind;
        const int64_t* en;
        if (c < n_elems) { kind = kinds[c]; en = enodes + eoff[c]; }
        else { kind = bkinds[c - n_elems]; en = bnodes + boff[c - n_elems]; }
        local_faces(kind, lf);
        for (auto& f : lf) {
            key.clear();
            for (int v : f) key.push_back(en[v]);
            std::sort(key.begin(), key.end());
            int64_t fid = index.at(key);
            const auto& cs = face_cells[fid];
            m->cf.push_back(fid);
            m->cc.push_back(cs[0] == c ? cs[1] : cs[0]);
        }
        m->cfs.push_back((int64_t)m->cf.size());
    }
    m->metric_bits = metric_bits;
    if (metric_bits == 32) compute_metrics<float>(*m);
    else compute_metrics<double>(*m);
    return m;
}

// ---------------------------------------------------------------------------
// Solver state and operators.
// ---------------------------------------------------------------------------
struct SolverBase {
    virtual ~SolverBase() {}
};

template <typename T>
struct Solver : SolverBase {
    const Mesh* m;
    int64_t N, G, NG;
    bool transposed;          // reference-compatible momentum reconstruction
    std::vector<V3<T>> cc, fc, fn;
    std::vector<T> cv, fa;
    std::vector<T3<T>> mat;
    std::vector<T> rho, rhoe, rho_n, rhoe_n, err, err_rho;   // err_rho: the density part F_rho^2 V
    std::vector<V3<T>> rhou, rhou_n;
    std::vector<V3<T>> g_rho, g_rhoe;   // gradients
    std::vector<T3<T>> g_rhou;
    std::vector<T> l_rho, l_rhoe;        // limiters
    std::vector<V3<T>> l_rhou;

    Solver(const Mesh* mesh, bool transposed_) : m(mesh), transposed(transposed_) {
        N = m->N; G = m->G; NG = N + G;
        cc.resize(NG); cv.resize(NG);
        for (int64_t i = 0; i < NG; ++i) {
            cc[i] = mk<T>((T)m->cell_center[3 * i], (T)m->cell_center[3 * i + 1], (T)m->cell_center[3 * i + 2]);
            cv[i] = (T)m->cell_volume[i];
        }
        fc.resize(m->F); fn.resize(m->F); fa.resize(m->F);
        for (int64_t f = 0; f < m->F; ++f) {
            fc[f] = mk<T>((T)m->face_center[3 * f], (T)m->face_center[3 * f + 1], (T)m->face_center[3 * f + 2]);
            fn[f] = mk<T>((T)m->face_normal[3 * f], (T)m->face_normal[3 * f + 1], (T)m->face_normal[3 * f + 2]);
            fa[f] = (T)m->face_area[f];
        }
        mat.resize(N);
        for (int64_t i = 0; i < N; ++i) {
            const double* p = &m->cell_matrix[9 * i];
            mat[i] = T3<T>{mk<T>((T)p[0], (T)p[1], (T)p[2]), mk<T>((T)p[3], (T)p[4], (T)p[5]),
                           mk<T>((T)p[6], (T)p[7], (T)p[8])};
        }
        rho.assign(NG, 0); rhoe.assign(NG, 0); rhou.assign(NG, mk<T>(0, 0, 0));
        rho_n = rho; rhoe_n = rhoe; rhou_n = rhou;
        err.assign(NG, 0);
        err_rho.assign(NG, 0);
        g_rho.assign(NG, mk<T>(0, 0, 0)); g_rhoe = g_rho;
        g_rhou.assign(NG, T3<T>{mk<T>(0, 0, 0), mk<T>(0, 0, 0), mk<T>(0, 0, 0)});
        l_rho.assign(NG, 1); l_rhoe.assign(NG, 1); l_rhou.assign(NG, mk<T>(1, 1, 1));
    }

    // euler_init, src/models/euler.cu:385-409 (cells and ghosts)
    void init(V3<T> mach, T p, T t) {
        T rv = p / t;
        V3<T> vel = mach * std::sqrt((T)1.4 * p / rv);
        V3<T> ru = vel * rv;
        T re = p / (T)0.4 + (T)0.5 * rv * dot(vel, vel);
        for (int64_t i = 0; i < NG; ++i) { rho[i] = rv; rhou[i] = ru; rhoe[i] = re; }
    }

    // Ghost c0, interior c1, the ghost's face and the outward unit normal
    // (src/models/euler.cu:422-434).
    void ghost_geom(int64_t t, int64_t& c0, int64_t& c1, V3<T>& n) const {
        c0 = m->ghost_ids[t];
        c1 = m->cc[m->cfs[c0]];
        const int64_t face = m->cf[m->cfs[c0]];
        V3<T> d1 = fc[face] - cc[c1];
        n = outer_normal(fn[face], d1);
    }

    // euler_slip_bc, src/models/euler.cu:412-442
    void bc_slip(int64_t region) {
        for (int64_t t = m->ghost_starts[region]; t < m->ghost_starts[region + 1]; ++t) {
            int64_t c0, c1; V3<T> n;
            ghost_geom(t, c0, c1, n);
            rhou[c0] = rhou[c1] - n * ((T)2 * dot(n, rhou[c1]));
            rho[c0] = rho[c1];
            rhoe[c0] = rhoe[c1];
        }
    }

    // euler_inletoutlet_bc, src/models/euler.cu:446-520
    void bc_farfield(int64_t region, V3<T> imach, T ip, T it) {
        for (int64_t t = m->ghost_starts[region]; t < m->ghost_starts[region + 1]; ++t) {
            int64_t c0, c1; V3<T> n;
            ghost_geom(t, c0, c1, n);
            V3<T> u = rhou[c1] / rho[c1];
            T p = (T)0.4 * (rhoe[c1] - (T)0.5 / rho[c1] * dot(rhou[c1], rhou[c1]));
            T tt = p / rho[c1];
            T mach = std::sqrt(dot(u, u) / ((T)1.4 * p / rho[c1]));
            T idens = ip / it;
            V3<T> ivel = imach * std::sqrt((T)1.4 * ip / idens);
            T ien = ip / (T)0.4 + (T)0.5 * idens * dot(ivel, ivel);
            if (dot(u, n) < 0) {
                if (mach > (T)1) {
                    T ic = std::sqrt((T)1.4 * ip / idens);
                    rho[c0] = idens;
                    rhou[c0] = imach * ic * idens;
                    rhoe[c0] = ien;
                } else {
                    rho[c0] = p / it;
                    T ic = std::sqrt((T)1.4 * p / rho[c0]);
                    V3<T> v = imach * ic;
                    rhou[c0] = v * rho[c0];
                    rhoe[c0] = p / (T)0.4 + (T)0.5 * rho[c0] * dot(v, v);
                }
            } else {
                if (mach > (T)1) {
                    rho[c0] = rho[c1]; rhou[c0] = rhou[c1]; rhoe[c0] = rhoe[c1];
                } else {
                    rho[c0] = ip / tt;
                    rhou[c0] = u * rho[c0];
                    rhoe[c0] = ip / (T)0.4 + (T)0.5 * rho[c0] * dot(u, u);
                }
            }
        }
    }

    // limiter(), src/fvmops.cu:118-169 (Michalak function, K = 1, x0.8)
    static T limiter(T u, V3<T> ug, T umin, T umax, V3<T> d) {
        const T tol = sizeof(T) == 4 ? (T)1e-6 : (T)1e-12;
        T delta = dot(ug, d);
        T du = umax - u, dd = umin - u;
        T dmm2 = (du - dd) * (du - dd);
        T k3v = norm(d);
        k3v *= k3v * k3v;
        T sig;
        if (dmm2 <= k3v) sig = 1;
        else if (dmm2 <= 2 * k3v) {
            T y = dmm2 / k3v - (T)1;
            sig = (T)2 * y * y * y - (T)3 * y * y + (T)1;
        } else sig = 0;
        T lim = 1;
        auto f = [](T y) { return y < (T)2 ? y - (T)0.25 * y * y : (T)1; };
        if (delta > tol) lim = f(du / delta);
        else if (delta < -tol) lim = f(dd / delta);
        lim *= (T)0.8;
        return sig + ((T)1 - sig) * lim;
    }

    // FvmEulerStepPrepare, src/models/euler.cu:597-647: gradient, limiter
    // and ghost copy for rho, rhou, rhoe; cells [c0, c1) only when c1 > c0
    // (a bounded sample for timing).
    void prepare(int64_t c0 = 0, int64_t c1 = -1) {
        if (c1 < 0) c1 = N;
#pragma omp parallel for schedule(static)
        for (int64_t i = c0; i < c1; ++i) {
            // ScalarVarComputeGradient / VectorVarComputeGradient, src/fvmops.cu:51-111
            V3<T> gr = mk<T>(0, 0, 0), ge = gr;
            T3<T> gu{gr, gr, gr};
            for (int64_t k = m->cfs[i]; k < m->cfs[i + 1]; ++k) {
                const int64_t c = m->cc[k];
                V3<T> d = cc[c] - cc[i];
                T w2 = (T)1 / dot(d, d);
                gr = gr + d * (rho[c] - rho[i]) * w2;
                ge = ge + d * (rhoe[c] - rhoe[i]) * w2;
                gu.u = gu.u + d * (rhou[c].x - rhou[i].x) * w2;
                gu.v = gu.v + d * (rhou[c].y - rhou[i].y) * w2;
                gu.w = gu.w + d * (rhou[c].z - rhou[i].z) * w2;
            }
            g_rho[i] = tmul(mat[i], gr);
            g_rhoe[i] = tmul(mat[i], ge);
            g_rhou[i] = T3<T>{tmul(mat[i], gu.u), tmul(mat[i], gu.v), tmul(mat[i], gu.w)};
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = c0; i < c1; ++i) {
            // ScalarVarComputeLimiters / VectorVarComputeLimiters, src/fvmops.cu:175-266
            T rmin = rho[i], rmax = rho[i], emin = rhoe[i], emax = rhoe[i];
            V3<T> umin = rhou[i], umax = rhou[i];
            for (int64_t k = m->cfs[i]; k < m->cfs[i + 1]; ++k) {
                const int64_t c = m->cc[k];
                rmin = std::fmin(rmin, rho[c]); rmax = std::fmax(rmax, rho[c]);
                emin = std::fmin(emin, rhoe[c]); emax = std::fmax(emax, rhoe[c]);
                umin = mk<T>(std::fmin(umin.x, rhou[c].x), std::fmin(umin.y, rhou[c].y), std::fmin(umin.z, rhou[c].z));
                umax = mk<T>(std::fmax(umax.x, rhou[c].x), std::fmax(umax.y, rhou[c].y), std::fmax(umax.z, rhou[c].z));
            }
            T lr = 2, le = 2;
            V3<T> lu = mk<T>(2, 2, 2);
            for (int64_t k = m->cfs[i]; k < m->cfs[i + 1]; ++k) {
                V3<T> d = fc[m->cf[k]] - cc[i];
                lr = std::fmin(lr, limiter(rho[i], g_rho[i], rmin, rmax, d));
                le = std::fmin(le, limiter(rhoe[i], g_rhoe[i], emin, emax, d));
                lu.x = std::fmin(lu.x, limiter(rhou[i].x, g_rhou[i].u, umin.x, umax.x, d));
                lu.y = std::fmin(lu.y, limiter(rhou[i].y, g_rhou[i].v, umin.y, umax.y, d));
                lu.z = std::fmin(lu.z, limiter(rhou[i].z, g_rhou[i].w, umin.z, umax.z, d));
            }
            l_rho[i] = lr; l_rhoe[i] = le; l_rhou[i] = lu;
        }
        // fvmScalGradLimBc / fvmVecGradLimBc, src/fvmops.cu:272-304
        for (int64_t t = 0; t < G; ++t) {
            const int64_t c = m->ghost_ids[t];
            const int64_t o = m->cc[m->cfs[c]];
            g_rho[c] = g_rho[o]; g_rhoe[c] = g_rhoe[o]; g_rhou[c] = g_rhou[o];
            l_rho[c] = l_rho[o]; l_rhoe[c] = l_rhoe[o]; l_rhou[c] = l_rhou[o];
        }
    }

    V3<T> mom_delta(int64_t c, V3<T> d) const {
        // Reference-compatible: dot(tensor, d) is the column combination,
        // i.e. G^T d with G[a][b] = d(rhou_a)/dx_b (src/models/euler.cu:252-253,
        // include/datatypes.cuh:296-302).  Otherwise the true G d.
        if (transposed) return tmul(g_rhou[c], d);
        return mk<T>(dot(g_rhou[c].u, d), dot(g_rhou[c].v, d), dot(g_rhou[c].w, d));
    }

    // fvmEulerSteadyOp + euler_steady_step, src/models/euler.cu:236-381,
    // with a Jacobi update into the *_n arrays; cells [b0, b1) only when
    // b1 > b0.
    void step(T cfl, int64_t b0 = 0, int64_t b1 = -1) {
        if (b1 < 0) b1 = N;
#pragma omp parallel for schedule(static)
        for (int64_t c0 = b0; c0 < b1; ++c0) {
            T dt = 0, fr = 0, fe = 0;
            V3<T> fu = mk<T>(0, 0, 0);
            const T v = cv[c0];
            for (int64_t k = m->cfs[c0]; k < m->cfs[c0 + 1]; ++k) {
                // fvmOpVoidSetup, include/fvmops.cuh:61-72
                const int64_t f = m->cf[k], c1 = m->cc[k];
                V3<T> d0 = fc[f] - cc[c0];
                V3<T> d1 = fc[f] - cc[c1];
                V3<T> n = outer_normal(fn[f], d0);
                T ds = fa[f] / v;
                T r0 = rho[c0] + dot(g_rho[c0], d0) * l_rho[c0];
                T r1 = rho[c1] + dot(g_rho[c1], d1) * l_rho[c1];
                V3<T> u0 = rhou[c0] + mul(mom_delta(c0, d0), l_rhou[c0]);
                V3<T> u1 = rhou[c1] + mul(mom_delta(c1, d1), l_rhou[c1]);
                T e0 = rhoe[c0] + dot(g_rhoe[c0], d0) * l_rhoe[c0];
                T e1 = rhoe[c1] + dot(g_rhoe[c1], d1) * l_rhoe[c1];
                T p0 = (T)0.4 * (e0 - (T)0.5 / r0 * dot(u0, u0));
                T p1 = (T)0.4 * (e1 - (T)0.5 / r1 * dot(u1, u1));
                T V0 = dot(u0, n) / r0;
                T V1 = dot(u1, n) / r1;
                T frf0 = V0 * r0, frf1 = V1 * r1;
                V3<T> fuf0 = u0 * V0 + n * p0, fuf1 = u1 * V1 + n * p1;
                T fef0 = V0 * (e0 + p0), fef1 = V1 * (e1 + p1);
                fr += (frf0 + frf1) * ds * (T)0.5;
                fu = fu + (fuf0 + fuf1) * ds * (T)0.5;
                fe += (fef0 + fef1) * ds * (T)0.5;
                T eig = std::fmax(norm(u0 / r0) + lsqrt((T)1.4 * p0 / r0), norm(u1 / r1) + lsqrt((T)1.4 * p1 / r1));
                fr -= eig * (r1 - r0) * (T)0.5 * ds;
                fu = fu - (u1 - u0) * (eig * (T)0.5 * ds);
                fe -= eig * (e1 - e0) * (T)0.5 * ds;
                dt += eig * ds;
            }
            dt = cfl / dt;
            rho_n[c0] = rho[c0] - fr * dt;
            rhou_n[c0] = rhou[c0] - fu * dt;
            rhoe_n[c0] = rhoe[c0] - fe * dt;
            err[c0] = (fr * fr + dot(fu, fu) + fe * fe) * v;
            err_rho[c0] = fr * fr * v;
        }
        for (int64_t c = b0; c < b1; ++c) { rho[c] = rho_n[c]; rhou[c] = rhou_n[c]; rhoe[c] = rhoe_n[c]; }
    }

    // FvmFieldReduceSum, src/fvmops.cu:369-383 (accumulated in double here)
    double reduce_error() const {
        double s = 0;
        for (int64_t i = 0; i < N; ++i) s += (double)err[i];
        return s;
    }
};

template <typename Fn>
auto dispatch(void* s, int bits, Fn fn) {
    if (bits == 32) return fn(static_cast<Solver<float>*>(s));
    return fn(static_cast<Solver<double>*>(s));
}

struct Handle {
    int bits;
    SolverBase* s;
};

}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void* orc_mesh_new(int64_t n_nodes, const double* nodes, int64_t n_elems, const int32_t* kinds,
                   const int64_t* eoff, const int64_t* enodes, int64_t n_regions, const char* names,
                   const int64_t* roff, const int32_t* bkinds, const int64_t* boff, const int64_t* bnodes,
                   int metric_bits) {
    return build_mesh(n_nodes, nodes, n_elems, kinds, eoff, enodes, n_regions, names, roff, bkinds, boff,
                      bnodes, metric_bits);
}

void orc_mesh_free(void* h) { delete static_cast<Mesh*>(h); }

// sizes: N, G, F, S (cell-face entries incl. ghosts), n_nodes, n_regions, face-node entries
void orc_mesh_sizes(void* h, int64_t* out) {
    Mesh* m = static_cast<Mesh*>(h);
    out[0] = m->N; out[1] = m->G; out[2] = m->F; out[3] = (int64_t)m->cf.size();
    out[4] = m->n_nodes; out[5] = m->n_regions; out[6] = (int64_t)m->fn.size();
}

// Copies a named mesh array; returns the element count (0 if unknown).
int64_t orc_mesh_get(void* h, const char* name, void* out) {
    Mesh* m = static_cast<Mesh*>(h);
    std::string n(name);
    auto cpy_i = [&](const std::vector<int64_t>& v) {
        if (out) memcpy(out, v.data(), v.size() * 8);
        return (int64_t)v.size();
    };
    auto cpy_d = [&](const std::vector<double>& v) {
        if (out) memcpy(out, v.data(), v.size() * 8);
        return (int64_t)v.size();
    };
    if (n == "cell_faces_starts") return cpy_i(m->cfs);
    if (n == "cell_faces") return cpy_i(m->cf);
    if (n == "cell_connects") return cpy_i(m->cc);
    if (n == "face_nodes_starts") return cpy_i(m->fns);
    if (n == "face_nodes") return cpy_i(m->fn);
    if (n == "ghost_cell_ids") return cpy_i(m->ghost_ids);
    if (n == "ghost_cell_starts") return cpy_i(m->ghost_starts);
    if (n == "face_areas") return cpy_d(m->face_area);
    if (n == "face_normals") return cpy_d(m->face_normal);
    if (n == "face_centers") return cpy_d(m->face_center);
    if (n == "cell_volumes") return cpy_d(m->cell_volume);
    if (n == "cell_centers") return cpy_d(m->cell_center);
    if (n == "cell_matrices") return cpy_d(m->cell_matrix);
    return 0;
}

int64_t orc_region_id(void* h, const char* name) {
    Mesh* m = static_cast<Mesh*>(h);
    for (size_t i = 0; i < m->region_names.size(); ++i)
        if (m->region_names[i] == name) return (int64_t)i;
    return -1;
}

void* orc_solver_new(void* mesh, int bits, int transposed) {
    Handle* h = new Handle();
    h->bits = bits;
    if (bits == 32) h->s = new Solver<float>(static_cast<Mesh*>(mesh), transposed != 0);
    else h->s = new Solver<double>(static_cast<Mesh*>(mesh), transposed != 0);
    return h;
}

void orc_solver_free(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    delete h->s;
    delete h;
}

void orc_init(void* hp, double mx, double my, double mz, double p, double t) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) {
        using T = std::remove_reference_t<decltype(s->rho[0])>;
        s->init(mk<T>((T)mx, (T)my, (T)mz), (T)p, (T)t);
        return 0;
    });
}

// state arrays are float64, n = N + G: rho[n], rhou[3n], rhoe[n]
void orc_set_state(void* hp, const double* rho, const double* rhou, const double* rhoe) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) {
        using T = std::remove_reference_t<decltype(s->rho[0])>;
        for (int64_t i = 0; i < s->NG; ++i) {
            s->rho[i] = (T)rho[i];
            s->rhou[i] = mk<T>((T)rhou[3 * i], (T)rhou[3 * i + 1], (T)rhou[3 * i + 2]);
            s->rhoe[i] = (T)rhoe[i];
        }
        return 0;
    });
}

// Named solver arrays in reference layout, as float64 (n = N + G entries):
// rho, rhoe, err, err_rho, lim_rho, lim_rhoe (1 per cell); rhou, lim_rhou, grad_rho,
// grad_rhoe (3); grad_rhou (9: columns u, v, w = gradients of each component).
int64_t orc_get(void* hp, const char* name, double* out) {
    Handle* h = static_cast<Handle*>(hp);
    std::string n(name);
    return dispatch(h->s, h->bits, [&](auto* s) -> int64_t {
        const int64_t NG = s->NG;
        auto s1 = [&](const auto& v) { for (int64_t i = 0; i < NG; ++i) out[i] = (double)v[i]; return NG; };
        auto s3 = [&](const auto& v) {
            for (int64_t i = 0; i < NG; ++i) { out[3 * i] = v[i].x; out[3 * i + 1] = v[i].y; out[3 * i + 2] = v[i].z; }
            return 3 * NG;
        };
        if (n == "rho") return s1(s->rho);
        if (n == "rhoe") return s1(s->rhoe);
        if (n == "err") return s1(s->err);
        if (n == "err_rho") return s1(s->err_rho);
        if (n == "lim_rho") return s1(s->l_rho);
        if (n == "lim_rhoe") return s1(s->l_rhoe);
        if (n == "rhou") return s3(s->rhou);
        if (n == "lim_rhou") return s3(s->l_rhou);
        if (n == "grad_rho") return s3(s->g_rho);
        if (n == "grad_rhoe") return s3(s->g_rhoe);
        if (n == "grad_rhou") {
            for (int64_t i = 0; i < NG; ++i) {
                const auto& g = s->g_rhou[i];
                double v[9] = {g.u.x, g.u.y, g.u.z, g.v.x, g.v.y, g.v.z, g.w.x, g.w.y, g.w.z};
                for (int k = 0; k < 9; ++k) out[9 * i + k] = v[k];
            }
            return 9 * NG;
        }
        return 0;
    });
}

void orc_bc_slip(void* hp, int64_t region) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) { s->bc_slip(region); return 0; });
}

void orc_bc_farfield(void* hp, int64_t region, double mx, double my, double mz, double p, double t) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) {
        using T = std::remove_reference_t<decltype(s->rho[0])>;
        s->bc_farfield(region, mk<T>((T)mx, (T)my, (T)mz), (T)p, (T)t);
        return 0;
    });
}

void orc_prepare(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) { s->prepare(); return 0; });
}

void orc_step(void* hp, double cfl) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) {
        using T = std::remove_reference_t<decltype(s->rho[0])>;
        s->step((T)cfl);
        return 0;
    });
}

double orc_reduce_error(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    return dispatch(h->s, h->bits, [&](auto* s) { return s->reduce_error(); });
}

// Gradients/limiters and the flux/update for the interior cells [c0, c1)
// only: a bounded sample of one iteration, for CPU timing.
void orc_sample_step(void* hp, double cfl, int64_t c0, int64_t c1) {
    Handle* h = static_cast<Handle*>(hp);
    dispatch(h->s, h->bits, [&](auto* s) {
        using T = std::remove_reference_t<decltype(s->rho[0])>;
        s->prepare(c0, c1);
        s->step((T)cfl, c0, c1);
        return 0;
    });
}

// The PhysicsEuler::step loop (src/models/euler.cu:99-175) for n_iter
// iterations: boundary conditions in the given order, prepare, step, and the
// residual sum into hist[it].  bc_type: 0 slip, 1 farfield; bc_param: 5 per
// condition (mx, my, mz, p, T).
void orc_run(void* hp, int64_t n_iter, double cfl, int64_t n_bc, const int32_t* bc_type,
             const int64_t* bc_region, const double* bc_param, double* hist) {
    for (int64_t it = 0; it < n_iter; ++it) {
        for (int64_t b = 0; b < n_bc; ++b) {
            const double* q = bc_param + 5 * b;
            if (bc_type[b] == 0) orc_bc_slip(hp, bc_region[b]);
            else orc_bc_farfield(hp, bc_region[b], q[0], q[1], q[2], q[3], q[4]);
        }
        orc_prepare(hp);
        orc_step(hp, cfl);
        double e = orc_reduce_error(hp);
        if (hist) hist[it] = e;
    }
}

}  // extern "C"
