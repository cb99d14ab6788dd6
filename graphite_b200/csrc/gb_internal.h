// Internal declarations of libgraphite_b200.so.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "graphite_b200.h"

namespace gb {

// Last error of the calling thread (gbGetLastError).
void set_error(const std::string& msg);
void clear_error();

// Volume and boundary elements as read from a mesh file (SU2 order).
struct ElementSet {
    std::vector<double> nodes;            // 3 per node
    std::vector<int8_t> kinds;            // SU2 kind per element
    std::vector<int64_t> eoff;            // n_elems + 1
    std::vector<uint32_t> enodes;
    std::vector<std::string> regions;     // marker names, file order
    std::vector<int64_t> roff;            // n_regions + 1 (boundary element ranges)
    std::vector<int8_t> bkinds;
    std::vector<int64_t> boff;            // n_bfaces + 1
    std::vector<uint32_t> bnodes;
};

// Reference-semantics topology (the content of a .fvm file): cells in
// element order, then one ghost per boundary face grouped by region; the
// cell->face CSR lists faces in element-local order (src/meshio.cu:315-475)
// and the connected cell of each; a face keeps the node order of the first
// element that lists it.
struct Topology {
    int64_t N = 0, G = 0, F = 0;
    std::vector<double> nodes;
    std::vector<uint32_t> cfs, cf, cc;    // N+G+1, S, S
    std::vector<uint32_t> fns, fn;        // F+1, face-node entries
    std::vector<uint32_t> ghost_ids;      // G
    std::vector<uint32_t> ghost_starts;   // n_regions + 1
    std::vector<std::string> regions;
};

bool parse_su2(const char* path, ElementSet& es);
bool build_topology(const ElementSet& es, Topology& t);
bool write_fvm(const char* path, const Topology& t);
bool read_fvm(const char* path, Topology& t);

// Device numbering.  Interior cells are renumbered (reverse Cuthill-McKee or
// identity), ghosts follow region by region, each region ordered by the new
// index of its interior cell; faces are ordered by (lower, higher) new cell.
struct Numbering {
    std::vector<uint32_t> cell_new;       // old -> new, N+G
    std::vector<uint32_t> cell_old;       // new -> old
    std::vector<uint32_t> face_new;       // old -> new, F
    std::vector<uint32_t> face_old;
    // new-order interior CSR: per interior cell the faces in the reference's
    // element-local order as (new face, new neighbour)
    std::vector<uint32_t> start;          // N+1
    std::vector<uint32_t> nb_face, nb_cell;
    std::vector<uint32_t> ghost_cell, ghost_face;   // per new ghost (index - N)
    std::vector<uint32_t> region_start;   // new ghost ranges per region, n_regions+1
    int64_t bandwidth = 0;                // max |new(i) - new(j)| over interior neighbours
};

void number_cells(const Topology& t, bool rcm, Numbering& num);

}  // namespace gb
