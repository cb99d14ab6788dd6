// Host-side mesh construction: SU2 parsing, face de-duplication into the
// reference's cell/face/ghost topology, the .fvm file format, and the device
// numbering (reverse Cuthill-McKee).
#include <algorithm>
#include <mutex>
#include <thread>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "gb_internal.h"

namespace gb {

namespace {

// Local faces of each SU2 element kind, in the order the reference's
// su2KindToFaces lists them (src/meshio.cu:315-475).  The order decides the
// per-cell face order, hence the order in which a cell sums its fluxes.
struct LocalFaces {
    int n;
    int size[6];
    int node[6][4];
};

const LocalFaces* local_faces(int kind) {
    static const LocalFaces tri = {1, {3}, {{0, 1, 2}}};
    static const LocalFaces quad = {1, {4}, {{0, 1, 2, 3}}};
    static const LocalFaces tet = {4, {3, 3, 3, 3}, {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}}};
    static const LocalFaces hex = {6, {4, 4, 4, 4, 4, 4},
                                   {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}, {3, 2, 1, 0}, {4, 5, 6, 7}}};
    static const LocalFaces prism = {5, {3, 3, 4, 4, 4},
                                     {{0, 1, 2}, {3, 5, 4}, {0, 2, 5, 3}, {1, 4, 5, 2}, {1, 0, 3, 4}}};
    static const LocalFaces pyr = {5, {4, 3, 3, 3, 3}, {{0, 1, 2, 3}, {0, 4, 3}, {0, 1, 4}, {1, 2, 4}, {2, 3, 4}}};
    switch (kind) {
    case 5: return &tri;
    case 9: return &quad;
    case 10: return &tet;
    case 12: return &hex;
    case 13: return &prism;
    case 14: return &pyr;
    }
    return nullptr;
}

int nodes_of_kind(int kind) {
    switch (kind) {
    case 5: return 3;
    case 9: return 4;
    case 10: return 4;
    case 12: return 8;
    case 13: return 6;
    case 14: return 5;
    }
    return 0;
}

// Whole-file line reader.
struct Lines {
    std::vector<char> buf;
    size_t pos = 0;
    bool load(const char* path) {
        FILE* f = fopen(path, "rb");
        if (!f) return false;
        fseek(f, 0, SEEK_END);
        long n = ftell(f);
        fseek(f, 0, SEEK_SET);
        buf.resize((size_t)n + 1);
        size_t got = fread(buf.data(), 1, (size_t)n, f);
        fclose(f);
        buf[got] = '\0';
        buf.resize(got + 1);
        return true;
    }
    // Next non-empty, non-comment line (NUL-terminated in place), or nullptr.
    char* next() {
        while (pos + 1 < buf.size()) {
            char* s = buf.data() + pos;
            char* e = (char*)memchr(s, '\n', buf.size() - 1 - pos);
            if (e) { *e = '\0'; pos = (size_t)(e - buf.data()) + 1; }
            else { pos = buf.size() - 1; }
            while (*s == ' ' || *s == '\t' || *s == '\r') ++s;
            if (*s == '\0' || *s == '%') continue;
            return s;
        }
        return nullptr;
    }
};

// Runs fn(lo, hi) over [0, n) split into contiguous ranges, one per host
// thread (at most 32).
template <typename Fn>
void parallel_ranges(int64_t n, Fn fn) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int64_t parts = std::max<int64_t>(1, std::min<int64_t>({(int64_t)(hw ? hw : 1), 32, n / 65536}));
    if (parts == 1) {
        fn((int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int64_t p = 0; p < parts; ++p) th.emplace_back(fn, n * p / parts, n * (p + 1) / parts);
    for (auto& t : th) t.join();
}

bool keyword(char* line, const char* kw, char** rest) {
    size_t n = strlen(kw);
    if (strncmp(line, kw, n) != 0) return false;
    *rest = line + n;
    return true;
}

bool parse_count(const char* s, int64_t& v) {
    char* end;
    errno = 0;
    long long x = strtoll(s, &end, 10);
    if (end == s || errno != 0 || x < 0) return false;
    v = x;
    return true;
}

}  // namespace

bool parse_su2(const char* path, ElementSet& es) {
    Lines L;
    if (!L.load(path)) { set_error(std::string("cannot open mesh file ") + path); return false; }
    es = ElementSet();
    es.eoff.push_back(0);
    es.boff.push_back(0);
    es.roff.push_back(0);
    int64_t ndime = 0, npoin = -1;
    char* line;
    char* rest;
    auto bad = [&](const std::string& m) { set_error(std::string(path) + ": " + m); return false; };
    while ((line = L.next())) {
        if (keyword(line, "NDIME=", &rest)) {
            if (!parse_count(rest, ndime)) return bad("bad NDIME");
            if (ndime != 3) return bad("mesh must be 3D (NDIME= 3)");
        } else if (keyword(line, "NELEM=", &rest)) {
            int64_t n;
            if (!parse_count(rest, n)) return bad("bad NELEM");
            // line pointers in order, then each element's kind and nodes parsed
            // on all host threads into a fixed-stride scratch array (at most 8
            // nodes), then compacted; an error names the first bad element,
            // with the check that fails first on its line (kind, then nodes)
            std::vector<char*> lines((size_t)n);
            for (int64_t e = 0; e < n; ++e)
                if (!(lines[e] = L.next())) return bad("unexpected end of file in NELEM block");
            es.kinds.resize(n);
            std::vector<uint32_t> scratch((size_t)n * 8);
            int64_t first_bad = n;
            bool bad_kind = false;
            std::mutex bad_mu;
            parallel_ranges(n, [&](int64_t e0, int64_t e1) {
                for (int64_t e = e0; e < e1; ++e) {
                    char* p = lines[e];
                    const long kind = strtol(p, &p, 10);
                    const int k = nodes_of_kind((int)kind);
                    bool kind_fails = k == 0 || kind == 5 || kind == 9, nodes_fail = false;
                    for (int j = 0; j < k && !kind_fails; ++j) {
                        char* q;
                        const unsigned long v = strtoul(p, &q, 10);
                        if (q == p) { nodes_fail = true; break; }
                        p = q;
                        scratch[8 * e + j] = (uint32_t)v;
                    }
                    if (kind_fails || nodes_fail) {   // the first failure of this range
                        std::lock_guard<std::mutex> g(bad_mu);
                        if (e < first_bad) { first_bad = e; bad_kind = kind_fails; }
                        return;
                    }
                    es.kinds[e] = (int8_t)kind;
                }
            });
            if (first_bad < n) {
                const int64_t e = first_bad;
                if (bad_kind)
                    return bad("element " + std::to_string(e) + ": unsupported volume element kind " +
                               std::to_string(strtol(lines[e], nullptr, 10)));
                return bad("element " + std::to_string(e) + ": too few nodes");
            }
            es.eoff.resize(n + 1);
            es.eoff[0] = 0;
            for (int64_t e = 0; e < n; ++e) es.eoff[e + 1] = es.eoff[e] + nodes_of_kind(es.kinds[e]);
            es.enodes.resize(es.eoff[n]);
            parallel_ranges(n, [&](int64_t e0, int64_t e1) {
                for (int64_t e = e0; e < e1; ++e)
                    for (int64_t j = es.eoff[e]; j < es.eoff[e + 1]; ++j) es.enodes[j] = scratch[8 * e + (j - es.eoff[e])];
            });
        } else if (keyword(line, "NPOIN=", &rest)) {
            if (!parse_count(rest, npoin)) return bad("bad NPOIN");
            es.nodes.resize(3 * npoin);
            std::vector<char*> lines((size_t)npoin);
            for (int64_t i = 0; i < npoin; ++i)
                if (!(lines[i] = L.next())) return bad("unexpected end of file in NPOIN block");
            std::vector<int64_t> bad_at(1, npoin);
            std::mutex bad_mu;
            parallel_ranges(npoin, [&](int64_t i0, int64_t i1) {
                for (int64_t i = i0; i < i1; ++i) {
                    char* p = lines[i];
                    for (int c = 0; c < 3; ++c) {
                        char* q;
                        const double v = strtod(p, &q);
                        if (q == p) {
                            std::lock_guard<std::mutex> g(bad_mu);
                            bad_at[0] = std::min(bad_at[0], i);
                            return;
                        }
                        es.nodes[3 * i + c] = v;
                        p = q;
                    }
                }
            });
            if (bad_at[0] < npoin) return bad("point " + std::to_string(bad_at[0]) + ": expected 3 coordinates");
        } else if (keyword(line, "NMARK=", &rest)) {
            int64_t m;
            if (!parse_count(rest, m)) return bad("bad NMARK");
            for (int64_t r = 0; r < m; ++r) {
                char* l = L.next();
                if (!l || !keyword(l, "MARKER_TAG=", &rest)) return bad("expected MARKER_TAG=");
                while (*rest == ' ' || *rest == '\t') ++rest;
                char* e = rest + strlen(rest);
                while (e > rest && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\r')) --e;
                std::string name(rest, e);
                if (name.empty() || name.size() > 127) return bad("bad marker name");
                l = L.next();
                int64_t k;
                if (!l || !keyword(l, "MARKER_ELEMS=", &rest) || !parse_count(rest, k)) return bad("expected MARKER_ELEMS=");
                es.regions.push_back(name);
                for (int64_t b = 0; b < k; ++b) {
                    char* bl = L.next();
                    if (!bl) return bad("unexpected end of file in marker " + name);
                    char* p = bl;
                    long kind = strtol(p, &p, 10);
                    if (kind != 5 && kind != 9) return bad("marker " + name + ": boundary element kind must be 5 or 9");
                    int nn = nodes_of_kind((int)kind);
                    for (int j = 0; j < nn; ++j) {
                        char* q;
                        unsigned long v = strtoul(p, &q, 10);
                        if (q == p) return bad("marker " + name + ": too few nodes");
                        p = q;
                        es.bnodes.push_back((uint32_t)v);
                    }
                    es.bkinds.push_back((int8_t)kind);
                    es.boff.push_back((int64_t)es.bnodes.size());
                }
                es.roff.push_back((int64_t)es.bkinds.size());
            }
        }
    }
    if (npoin < 0) return bad("no NPOIN block");
    if (es.kinds.empty()) return bad("no elements");
    for (uint32_t v : es.enodes)
        if ((int64_t)v >= npoin) return bad("element node index out of range");
    for (uint32_t v : es.bnodes)
        if ((int64_t)v >= npoin) return bad("marker node index out of range");
    return true;
}

namespace {

struct FaceRec {
    uint64_t k0, k1;   // sorted node ids, padded with 0xffffffff
    uint32_t cell;
    uint32_t lf;
};


inline bool rec_less(const FaceRec& x, const FaceRec& y) {
    if (x.k0 != y.k0) return x.k0 < y.k0;
    if (x.k1 != y.k1) return x.k1 < y.k1;
    if (x.cell != y.cell) return x.cell < y.cell;   // records in (element, local face) order
    return x.lf < y.lf;
}

// Sorts v by less on the host's hardware threads: chunks sorted in parallel,
// then merged pairwise, in parallel, log2(chunks) rounds.  With a total order
// (no two records equal) the result is the same as a serial sort's.
template <typename T, typename Less>
void parallel_sort_by(std::vector<T>& v, Less less) {
    const size_t n = v.size();
    unsigned hw = std::thread::hardware_concurrency();
    size_t chunks = 1;
    while (chunks * 2 <= std::min<size_t>(hw ? hw : 1, 32) && n / (chunks * 2) >= 65536) chunks *= 2;
    if (chunks == 1) {
        std::sort(v.begin(), v.end(), less);
        return;
    }
    std::vector<size_t> cut(chunks + 1);
    for (size_t c = 0; c <= chunks; ++c) cut[c] = n * c / chunks;
    {
        std::vector<std::thread> th;
        for (size_t c = 0; c < chunks; ++c)
            th.emplace_back([&, c] { std::sort(v.begin() + cut[c], v.begin() + cut[c + 1], less); });
        for (auto& t : th) t.join();
    }
    for (size_t w = 1; w < chunks; w *= 2) {
        std::vector<std::thread> th;
        for (size_t c = 0; c + w < chunks; c += 2 * w) {
            const size_t lo = cut[c], mid = cut[c + w], hi = cut[std::min(c + 2 * w, chunks)];
            th.emplace_back([&, lo, mid, hi] {
                std::inplace_merge(v.begin() + lo, v.begin() + mid, v.begin() + hi, less);
            });
        }
        for (auto& t : th) t.join();
    }
}

inline void make_key(const uint32_t* nodes, int n, uint64_t& k0, uint64_t& k1) {
    uint32_t s[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
    for (int i = 0; i < n; ++i) s[i] = nodes[i];
    // 4-input sorting network; a triangle's padding (all ones) stays last
    auto cx = [&](int a, int b) {
        const uint32_t lo = std::min(s[a], s[b]), hi = std::max(s[a], s[b]);
        s[a] = lo;
        s[b] = hi;
    };
    cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
    k0 = ((uint64_t)s[0] << 32) | s[1];
    k1 = ((uint64_t)s[2] << 32) | s[3];
}

}  // namespace

// Conversion semantics of cuMeshFromSu2 (src/meshio.cu:713-764, 978-1136),
// done by a parallel sort of the face keys instead of a serial hash map.
bool build_topology(const ElementSet& es, Topology& t) {
    const int64_t N = (int64_t)es.kinds.size();
    const int64_t G = (int64_t)es.bkinds.size();
    t = Topology();
    t.N = N;
    t.G = G;
    t.nodes = es.nodes;
    t.regions = es.regions;
    // element face records
    std::vector<int64_t> rec_off(N + 1, 0);
    for (int64_t e = 0; e < N; ++e) rec_off[e + 1] = rec_off[e] + local_faces(es.kinds[e])->n;
    const int64_t S = rec_off[N];
    std::vector<FaceRec> srt(S);
    parallel_ranges(N, [&](int64_t e0, int64_t e1) {
        for (int64_t e = e0; e < e1; ++e) {
            const LocalFaces* lf = local_faces(es.kinds[e]);
            const uint32_t* en = es.enodes.data() + es.eoff[e];
            for (int f = 0; f < lf->n; ++f) {
                uint32_t fnodes[4];
                for (int j = 0; j < lf->size[f]; ++j) fnodes[j] = en[lf->node[f][j]];
                FaceRec& r = srt[rec_off[e] + f];
                make_key(fnodes, lf->size[f], r.k0, r.k1);
                r.cell = (uint32_t)e;
                r.lf = (uint32_t)f;
            }
        }
    });
    parallel_sort_by(srt, rec_less);
    auto rec_index = [&](const FaceRec& r) { return (uint32_t)(rec_off[r.cell] + r.lf); };
    // groups of equal keys: a group starts where the key changes; group ids
    // by a prefix sum over the starts; each group's arrays filled by its own
    // records (the first writes the key, creator and count, the second the
    // other cell), all in parallel.  A third record in a group is an error,
    // reported for the first such record in key order.
    std::vector<uint32_t> gid(S);
    parallel_ranges(S, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i)
            gid[i] = (i == 0 || srt[i].k0 != srt[i - 1].k0 || srt[i].k1 != srt[i - 1].k1) ? 1u : 0u;
    });
    int64_t n_groups = 0;
    for (int64_t i = 0; i < S; ++i) {
        const uint32_t start = gid[i];
        n_groups += start;
        gid[i] = (uint32_t)(n_groups - 1);
    }
    std::vector<uint32_t> group_of(S);
    std::vector<uint64_t> gk0(n_groups), gk1(n_groups);
    std::vector<uint32_t> g_first(n_groups);                  // record index of the first (creating) element face
    std::vector<uint32_t> g_cells(2 * n_groups, 0xffffffffu); // 2 per group
    std::vector<uint8_t> g_count(n_groups);
    int64_t third = S;
    std::mutex third_mu;
    parallel_ranges(S, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
            const FaceRec& r = srt[i];
            const uint32_t ri = rec_index(r);
            const uint32_t g = gid[i];
            group_of[ri] = g;
            if (i == 0 || gid[i - 1] != g) {
                gk0[g] = r.k0;
                gk1[g] = r.k1;
                g_first[g] = ri;
                g_cells[2 * g] = r.cell;
                g_count[g] = (i + 1 < S && gid[i + 1] == g) ? 2 : 1;
            } else if (i < 2 || gid[i - 2] != g) {
                g_cells[2 * g + 1] = r.cell;
            } else {
                std::lock_guard<std::mutex> lock(third_mu);
                third = std::min(third, i);
                return;
            }
        }
    });
    if (third < S) {
        set_error("non-manifold mesh: a face is shared by more than two elements (element " +
                  std::to_string(srt[third].cell) + ")");
        return false;
    }
    std::vector<FaceRec>().swap(srt);
    const int64_t F = (int64_t)gk0.size();
    t.F = F;
    // ghosts: one per boundary face, ids N + (running index), by region
    std::vector<uint32_t> bgroup(G);
    for (int64_t b = 0; b < G; ++b) {
        const int n = es.bkinds[b] == 5 ? 3 : 4;
        uint64_t k0, k1;
        make_key(es.bnodes.data() + es.boff[b], n, k0, k1);
        int64_t lo = 0, hi = F;
        while (lo < hi) {
            int64_t mid = (lo + hi) / 2;
            if (gk0[mid] < k0 || (gk0[mid] == k0 && gk1[mid] < k1)) lo = mid + 1;
            else hi = mid;
        }
        if (lo >= F || gk0[lo] != k0 || gk1[lo] != k1) {
            set_error("boundary face " + std::to_string(b) + " matches no element face");
            return false;
        }
        if (g_count[lo] != 1) {
            set_error("boundary face " + std::to_string(b) + " lies on a face that already has two cells");
            return false;
        }
        g_cells[2 * lo + 1] = (uint32_t)(N + b);
        g_count[lo] = 2;
        bgroup[b] = (uint32_t)lo;
    }
    for (int64_t g = 0; g < F; ++g) {
        if (g_count[g] != 2) {   // src/meshio.cu:1115-1128
            set_error("face of element " + std::to_string(g_cells[2 * g]) +
                      " has one cell and no boundary marker (open mesh)");
            return false;
        }
    }
    // face ids in order of first appearance; node order of the creator.
    // Pass 1 counts each element range's creating faces and their nodes, a
    // prefix sum gives each range its first face id and node offset, pass 2
    // writes them.
    const unsigned hw = std::thread::hardware_concurrency();
    const int64_t parts = std::max<int64_t>(1, std::min<int64_t>({(int64_t)(hw ? hw : 1), 32, N / 65536}));
    std::vector<int64_t> p_faces(parts + 1, 0), p_nodes(parts + 1, 0);
    auto creates = [&](int64_t e, int f) {
        const uint32_t ri = (uint32_t)(rec_off[e] + f);
        return g_first[group_of[ri]] == ri;
    };
    auto over_parts = [&](auto fn) {
        std::vector<std::thread> th;
        for (int64_t p = 0; p < parts; ++p) th.emplace_back(fn, p, N * p / parts, N * (p + 1) / parts);
        for (auto& x : th) x.join();
    };
    over_parts([&](int64_t p, int64_t e0, int64_t e1) {
        int64_t nf = 0, nn = 0;
        for (int64_t e = e0; e < e1; ++e) {
            const LocalFaces* lf = local_faces(es.kinds[e]);
            for (int f = 0; f < lf->n; ++f)
                if (creates(e, f)) { ++nf; nn += lf->size[f]; }
        }
        p_faces[p + 1] = nf;
        p_nodes[p + 1] = nn;
    });
    for (int64_t p = 0; p < parts; ++p) {
        p_faces[p + 1] += p_faces[p];
        p_nodes[p + 1] += p_nodes[p];
    }
    if (p_faces[parts] != F) {
        set_error("internal error: face count mismatch in the topology builder");
        return false;
    }
    std::vector<uint32_t> fid(F, 0xffffffffu);
    t.fns.assign(F + 1, 0);
    t.fn.assign(p_nodes[parts], 0);
    over_parts([&](int64_t p, int64_t e0, int64_t e1) {
        int64_t next = p_faces[p], pos = p_nodes[p];
        for (int64_t e = e0; e < e1; ++e) {
            const LocalFaces* lf = local_faces(es.kinds[e]);
            const uint32_t* en = es.enodes.data() + es.eoff[e];
            for (int f = 0; f < lf->n; ++f) {
                if (!creates(e, f)) continue;
                fid[group_of[rec_off[e] + f]] = (uint32_t)next;
                for (int j = 0; j < lf->size[f]; ++j) t.fn[pos++] = en[lf->node[f][j]];
                t.fns[++next] = (uint32_t)pos;
            }
        }
    });
    // CSR, element-local face order (src/meshio.cu:1044-1136)
    t.cfs.assign(N + G + 1, 0);
    t.cf.assign(S + G, 0);
    t.cc.assign(S + G, 0);
    parallel_ranges(N, [&](int64_t e0, int64_t e1) {
        for (int64_t e = e0; e < e1; ++e) {
            for (int64_t r = rec_off[e]; r < rec_off[e + 1]; ++r) {
                const uint32_t g = group_of[r];
                t.cf[r] = fid[g];
                const uint32_t a = g_cells[2 * g], b = g_cells[2 * g + 1];
                t.cc[r] = a == (uint32_t)e ? b : a;
            }
            t.cfs[e + 1] = (uint32_t)rec_off[e + 1];
        }
    });
    for (int64_t b = 0; b < G; ++b) {
        const uint32_t g = bgroup[b];
        t.cf[S + b] = fid[g];
        t.cc[S + b] = g_cells[2 * g];
        t.cfs[N + b + 1] = (uint32_t)(S + b + 1);
    }
    t.ghost_ids.resize(G);
    for (int64_t b = 0; b < G; ++b) t.ghost_ids[b] = (uint32_t)(N + b);
    t.ghost_starts.assign(es.roff.begin(), es.roff.end());
    return true;
}

// .fvm layout, src/meshio.cu:1150-1216 (writer) and 166-292 (reader), float
// node coordinates as in the reference's float build.
bool write_fvm(const char* path, const Topology& t) {
    // the whole file laid out in memory, then written at once
    const uint32_t nn = (uint32_t)(t.nodes.size() / 3);
    const int64_t NG = t.N + t.G;
    const size_t nr = t.regions.size();
    const size_t bytes = 4 + 12 * (size_t)nn + 8 + 4 * ((size_t)t.F + t.fns[t.F]) + 8 + 4 * ((size_t)NG + 2 * (size_t)t.cfs[NG]) +
                         8 + nr * (128 + 4) + 4 * (size_t)t.G;
    std::vector<char> out(bytes);
    char* w = out.data();
    auto w32 = [&](uint32_t v) { memcpy(w, &v, 4); w += 4; };
    auto warr = [&](const uint32_t* p, size_t n) { if (n) memcpy(w, p, 4 * n); w += 4 * n; };
    w32(nn);
    for (size_t i = 0; i < t.nodes.size(); ++i) {
        const float x = (float)t.nodes[i];
        memcpy(w, &x, 4);
        w += 4;
    }
    w32((uint32_t)t.F);
    w32(t.fns[t.F]);
    for (int64_t i = 0; i < t.F; ++i) {
        w32(t.fns[i + 1] - t.fns[i]);
        warr(t.fn.data() + t.fns[i], t.fns[i + 1] - t.fns[i]);
    }
    w32((uint32_t)NG);
    w32(t.cfs[NG]);
    for (int64_t i = 0; i < NG; ++i) {
        const uint32_t s = t.cfs[i], n = t.cfs[i + 1] - s;
        w32(n);
        warr(t.cf.data() + s, n);
        warr(t.cc.data() + s, n);
    }
    w32((uint32_t)nr);
    w32((uint32_t)t.G);
    for (size_t r = 0; r < nr; ++r) {
        char name[128] = {0};
        strncpy(name, t.regions[r].c_str(), 127);
        memcpy(w, name, 128);
        w += 128;
        const uint32_t s = t.ghost_starts[r], e = t.ghost_starts[r + 1];
        w32(e - s);
        warr(t.ghost_ids.data() + s, e - s);
    }
    FILE* f = fopen(path, "wb");
    if (!f) { set_error(std::string("cannot write ") + path); return false; }
    bool ok = (size_t)(w - out.data()) == bytes && fwrite(out.data(), 1, bytes, f) == bytes;
    ok = (fclose(f) == 0) && ok;
    if (!ok) set_error(std::string("write error on ") + path);
    return ok;
}

bool read_fvm(const char* path, Topology& t) {
    // the whole file read at once, then parsed from memory with every read
    // checked against the bytes left
    FILE* f = fopen(path, "rb");
    if (!f) { set_error(std::string("cannot open mesh file ") + path); return false; }
    std::vector<char> data;
    {
        fseek(f, 0, SEEK_END);
        const long n = ftell(f);
        fseek(f, 0, SEEK_SET);
        data.resize(n > 0 ? (size_t)n : 0);
        const size_t got = data.empty() ? 0 : fread(data.data(), 1, data.size(), f);
        data.resize(got);
        fclose(f);
    }
    t = Topology();
    size_t pos = 0;
    auto left = [&]() { return data.size() - pos; };
    auto r32 = [&](uint32_t& v) {
        if (left() < 4) return false;
        memcpy(&v, data.data() + pos, 4);
        pos += 4;
        return true;
    };
    auto rarr = [&](uint32_t* p, size_t n) {
        if (left() / 4 < n) return false;
        if (n) memcpy(p, data.data() + pos, 4 * n);
        pos += 4 * n;
        return true;
    };
    auto fail = [&](const char* m) { set_error(std::string(path) + ": " + m); return false; };
    uint32_t nn;
    if (!r32(nn)) return fail("truncated header");
    if (left() / 12 < nn) return fail("truncated nodes");
    std::vector<float> xyz((size_t)nn * 3);
    rarr(reinterpret_cast<uint32_t*>(xyz.data()), xyz.size());
    t.nodes.assign(xyz.begin(), xyz.end());
    uint32_t nf, nfn;
    if (!r32(nf) || !r32(nfn)) return fail("truncated faces header");
    if (left() / 4 < (uint64_t)nf + nfn) return fail("truncated face nodes");
    t.F = nf;
    t.fns.resize((size_t)nf + 1);
    t.fn.resize(nfn);
    uint32_t off = 0;
    for (uint32_t i = 0; i < nf; ++i) {
        uint32_t s;
        if (!r32(s) || s < 3 || (uint64_t)off + s > nfn) return fail("bad face record");
        t.fns[i] = off;
        if (!rarr(t.fn.data() + off, s)) return fail("truncated face nodes");
        off += s;
    }
    t.fns[nf] = off;
    uint32_t ncg, ncf;
    if (!r32(ncg) || !r32(ncf)) return fail("truncated cells header");
    if (left() / 4 < (uint64_t)ncg + 2 * (uint64_t)ncf) return fail("truncated cell record");
    t.cfs.resize((size_t)ncg + 1);
    t.cf.resize(ncf);
    t.cc.resize(ncf);
    off = 0;
    for (uint32_t i = 0; i < ncg; ++i) {
        uint32_t s;
        if (!r32(s) || s == 0 || (uint64_t)off + s > ncf) return fail("bad cell record");
        t.cfs[i] = off;
        if (!rarr(t.cf.data() + off, s) || !rarr(t.cc.data() + off, s)) return fail("truncated cell record");
        off += s;
    }
    t.cfs[ncg] = off;
    uint32_t nr, ng;
    if (!r32(nr) || !r32(ng) || ng > ncg) return fail("bad regions header");
    t.G = ng;
    t.N = (int64_t)ncg - ng;
    t.ghost_ids.resize(ng);
    t.ghost_starts.assign(1, 0);
    off = 0;
    for (uint32_t r = 0; r < nr; ++r) {
        char name[129] = {0};
        uint32_t s;
        if (left() < 128) return fail("bad region record");
        memcpy(name, data.data() + pos, 128);
        pos += 128;
        if (!r32(s) || (uint64_t)off + s > ng) return fail("bad region record");
        t.regions.emplace_back(name);
        if (!rarr(t.ghost_ids.data() + off, s)) return fail("truncated region");
        off += s;
        t.ghost_starts.push_back(off);
    }
    if (off != ng) { set_error(std::string(path) + ": region sizes do not add up to the ghost count"); return false; }
    // validation the reference does not do
    for (uint32_t v : t.fn) if (v >= nn) { set_error(std::string(path) + ": face node out of range"); return false; }
    for (uint32_t v : t.cf) if (v >= nf) { set_error(std::string(path) + ": cell face out of range"); return false; }
    for (uint32_t v : t.cc) if (v >= ncg) { set_error(std::string(path) + ": connected cell out of range"); return false; }
    std::vector<uint8_t> seen(t.G, 0);
    for (int64_t g = 0; g < t.G; ++g) {
        const uint32_t c = t.ghost_ids[g];
        if (c < t.N || c >= ncg || t.cfs[c + 1] - t.cfs[c] != 1 || seen[c - t.N]) {
            set_error(std::string(path) + ": ghost cells must be the last cells, listed once, with one face");
            return false;
        }
        seen[c - t.N] = 1;
    }
    return true;
}

// Reverse Cuthill-McKee over the interior-cell graph, ghosts by region,
// faces by (lower, higher) new cell index.
void number_cells(const Topology& t, bool rcm, Numbering& num) {
    const int64_t N = t.N, G = t.G, NG = N + G;
    num = Numbering();
    num.cell_new.assign(NG, 0);
    num.cell_old.assign(NG, 0);
    std::vector<uint32_t> order;
    order.reserve(N);
    if (rcm && N > 0) {
        std::vector<uint32_t> deg(N, 0);
        for (int64_t i = 0; i < N; ++i)
            for (uint32_t k = t.cfs[i]; k < t.cfs[i + 1]; ++k)
                if (t.cc[k] < (uint32_t)N) ++deg[i];
        std::vector<int32_t> level(N, -1);
        std::vector<uint32_t> queue;
        queue.reserve(N);
        std::vector<uint8_t> done(N, 0);
        std::vector<uint32_t> nbrs;
        auto bfs_last = [&](uint32_t s, int& depth) {
            // BFS levels from s over the not-yet-numbered component; returns a
            // minimum-degree node of the last level.
            queue.clear();
            queue.push_back(s);
            level[s] = 0;
            size_t h = 0;
            while (h < queue.size()) {
                uint32_t u = queue[h++];
                for (uint32_t k = t.cfs[u]; k < t.cfs[u + 1]; ++k) {
                    uint32_t v = t.cc[k];
                    if (v < (uint32_t)N && level[v] < 0 && !done[v]) { level[v] = level[u] + 1; queue.push_back(v); }
                }
            }
            depth = level[queue.back()];
            uint32_t best = queue.back();
            for (size_t i = queue.size(); i-- > 0;) {
                if (level[queue[i]] != depth) break;
                if (deg[queue[i]] < deg[best]) best = queue[i];
            }
            for (uint32_t u : queue) level[u] = -1;
            return best;
        };
        for (int64_t seed = 0; seed < N; ++seed) {
            if (done[seed]) continue;
            // pseudo-peripheral start node
            int depth = 0, prev = -1;
            uint32_t s = (uint32_t)seed;
            for (int it = 0; it < 6 && depth > prev; ++it) {
                prev = depth;
                uint32_t c = bfs_last(s, depth);
                if (depth > prev) s = c;
            }
            // Cuthill-McKee from s, neighbours by increasing degree
            size_t h = order.size();
            order.push_back(s);
            done[s] = 1;
            while (h < order.size()) {
                uint32_t u = order[h++];
                nbrs.clear();
                for (uint32_t k = t.cfs[u]; k < t.cfs[u + 1]; ++k) {
                    uint32_t v = t.cc[k];
                    if (v < (uint32_t)N && !done[v]) { done[v] = 1; nbrs.push_back(v); }
                }
                // at most a handful: insertion sort by (degree, index)
                for (size_t x = 1; x < nbrs.size(); ++x) {
                    const uint32_t v = nbrs[x];
                    size_t y = x;
                    for (; y > 0 && (deg[nbrs[y - 1]] != deg[v] ? deg[nbrs[y - 1]] > deg[v] : nbrs[y - 1] > v); --y)
                        nbrs[y] = nbrs[y - 1];
                    nbrs[y] = v;
                }
                for (uint32_t v : nbrs) order.push_back(v);
            }
        }
        std::reverse(order.begin(), order.end());
    } else {
        for (int64_t i = 0; i < N; ++i) order.push_back((uint32_t)i);
    }
    for (int64_t i = 0; i < N; ++i) {
        num.cell_old[i] = order[i];
        num.cell_new[order[i]] = (uint32_t)i;
    }
    // ghosts: region by region, ordered by the new index of their interior cell
    const size_t nr = t.regions.size();
    num.region_start.assign(1, (uint32_t)N);
    uint32_t next = (uint32_t)N;
    std::vector<uint32_t> gl;
    for (size_t r = 0; r < nr; ++r) {
        gl.assign(t.ghost_ids.begin() + t.ghost_starts[r], t.ghost_ids.begin() + t.ghost_starts[r + 1]);
        std::stable_sort(gl.begin(), gl.end(), [&](uint32_t a, uint32_t b) {
            return num.cell_new[t.cc[t.cfs[a]]] < num.cell_new[t.cc[t.cfs[b]]];
        });
        for (uint32_t g : gl) { num.cell_new[g] = next; num.cell_old[next] = g; ++next; }
        num.region_start.push_back(next);
    }
    // faces by (lower, higher) new cell
    const int64_t F = t.F;
    std::vector<uint32_t> fa(F), fb(F);
    for (int64_t c = 0; c < NG; ++c)
        for (uint32_t k = t.cfs[c]; k < t.cfs[c + 1]; ++k) {
            const uint32_t f = t.cf[k];
            const uint32_t a = num.cell_new[c], b = num.cell_new[t.cc[k]];
            fa[f] = std::min(a, b);
            fb[f] = std::max(a, b);
        }
    // sort (lower, higher, face id) as one 64-bit key plus the id: direct
    // comparisons on contiguous records, in parallel chunks
    std::vector<std::pair<uint64_t, uint32_t>> keyed(F);
    parallel_ranges(F, [&](int64_t f0, int64_t f1) {
        for (int64_t f = f0; f < f1; ++f) keyed[f] = {((uint64_t)fa[f] << 32) | fb[f], (uint32_t)f};
    });
    parallel_sort_by(keyed, [](const std::pair<uint64_t, uint32_t>& x, const std::pair<uint64_t, uint32_t>& y) {
        return x.first != y.first ? x.first < y.first : x.second < y.second;
    });
    num.face_old.resize(F);
    for (int64_t i = 0; i < F; ++i) num.face_old[i] = keyed[i].second;
    num.face_new.resize(F);
    for (int64_t i = 0; i < F; ++i) num.face_new[num.face_old[i]] = (uint32_t)i;
    // interior CSR in new order, element-local face order kept
    num.start.assign(1, 0);
    num.start.reserve(N + 1);
    num.nb_face.reserve(t.cfs[N]);
    num.nb_cell.reserve(t.cfs[N]);
    int64_t bw = 0;
    for (int64_t i = 0; i < N; ++i) {
        const uint32_t o = num.cell_old[i];
        for (uint32_t k = t.cfs[o]; k < t.cfs[o + 1]; ++k) {
            const uint32_t nb = num.cell_new[t.cc[k]];
            num.nb_face.push_back(num.face_new[t.cf[k]]);
            num.nb_cell.push_back(nb);
            if (nb < (uint32_t)N) bw = std::max<int64_t>(bw, std::llabs((int64_t)nb - i));
        }
        num.start.push_back((uint32_t)num.nb_face.size());
    }
    num.bandwidth = bw;
    num.ghost_cell.resize(G);
    num.ghost_face.resize(G);
    for (int64_t g = 0; g < G; ++g) {
        const uint32_t o = num.cell_old[N + g];
        num.ghost_cell[g] = num.cell_new[t.cc[t.cfs[o]]];
        num.ghost_face[g] = num.face_new[t.cf[t.cfs[o]]];
    }
}

}  // namespace gb
