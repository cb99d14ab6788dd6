// VTU output of a mesh and its fields (FieldsWriteVtu, src/fvmfieldsio.cu:5-287).
//
// Cells are written as VTK polyhedra (type 42) with their unique nodes in
// ascending order and their face lists, as the reference does; cell data are
// the fields' host values (call VarGpuToCpu / VarAllGpuToCpu first, as
// PhysicsEuler::finish does), one value per interior cell -- the reference
// writes the ghosts' values too, more values than NumberOfCells.
// FieldsWriteVtu writes ASCII like the reference; gbFieldsWriteVtuBinary
// writes the same arrays as raw appended binary (UInt64 block headers).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gb_internal.h"

namespace gb {
namespace {

struct Cells {
    std::vector<int64_t> conn, offsets, faces, faceoffsets;
};

Cells polyhedra(const cuMeshBase* m) {
    Cells c;
    c.offsets.reserve(m->n_cells);
    c.faceoffsets.reserve(m->n_cells);
    std::vector<uint32_t> nodes;
    for (size_t e = 0; e < m->n_cells; ++e) {
        nodes.clear();
        const uint32_t f0 = m->cell_faces_starts[e], f1 = m->cell_faces_starts[e + 1];
        c.faces.push_back(f1 - f0);
        for (uint32_t k = f0; k < f1; ++k) {
            const uint32_t f = m->cell_faces[k];
            const uint32_t n0 = m->face_nodes_starts[f], n1 = m->face_nodes_starts[f + 1];
            c.faces.push_back(n1 - n0);
            for (uint32_t n = n0; n < n1; ++n) {
                nodes.push_back(m->face_nodes[n]);
                c.faces.push_back(m->face_nodes[n]);
            }
        }
        std::sort(nodes.begin(), nodes.end());
        nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
        for (uint32_t n : nodes) c.conn.push_back(n);
        c.offsets.push_back((int64_t)c.conn.size());
        c.faceoffsets.push_back((int64_t)c.faces.size());
    }
    return c;
}

bool check_args(const char* filename, cuMesh* mesh, const FvmField** vars, size_t nvars, const char* what) {
    if (!filename || !mesh || !mesh->_cpu || (nvars && !vars)) {
        set_error(std::string(what) + ": bad arguments");
        return false;
    }
    for (size_t i = 0; i < nvars; ++i) {
        const FvmField* v = vars[i];
        if (!v || !v->_cpu || !v->_cpu->value || (v->_cpu->elem_size != 4 && v->_cpu->elem_size != 12) ||
            v->_cpu->size < mesh->_cpu->n_cells) {
            set_error(std::string(what) + ": field " + std::to_string(i) +
                      " is not a scalar or vector field of this mesh");
            return false;
        }
    }
    return true;
}

void put_float(FILE* f, float v) {
    if (std::isnan(v)) fprintf(f, " nan");
    else fprintf(f, " %.9g", v);
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int FieldsWriteVtu(const char* filename, cuMesh* mesh, const FvmField** vars, const size_t nvars) {
    clear_error();
    if (!check_args(filename, mesh, vars, nvars, "FieldsWriteVtu")) return 1;
    const cuMeshBase* m = mesh->_cpu;
    FILE* f = fopen(filename, "wt");
    if (!f) { set_error(std::string("FieldsWriteVtu: cannot open ") + filename); return 1; }
    const Cells c = polyhedra(m);
    fprintf(f, "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
    fprintf(f, "  <UnstructuredGrid>\n    <Piece NumberOfPoints=\"%zu\" NumberOfCells=\"%zu\">\n", m->n_nodes, m->n_cells);
    fprintf(f, "      <CellData>\n");
    for (size_t i = 0; i < nvars; ++i) {
        const FvmField* v = vars[i];
        const int comps = v->_cpu->elem_size == 4 ? 1 : 3;
        if (comps == 1) fprintf(f, "        <DataArray type=\"Float32\" Name=\"%s\" format=\"ascii\">\n", v->name);
        else fprintf(f, "        <DataArray type=\"Float32\" Name=\"%s\" NumberOfComponents=\"3\" format=\"ascii\">\n", v->name);
        const float* val = (const float*)v->_cpu->value;
        for (size_t e = 0; e < m->n_cells; ++e) {
            fprintf(f, "         ");
            for (int k = 0; k < comps; ++k) put_float(f, val[comps * e + k]);
            fprintf(f, "\n");
        }
        fprintf(f, "        </DataArray>\n");
    }
    fprintf(f, "      </CellData>\n      <Points>\n");
    fprintf(f, "        <DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (size_t i = 0; i < m->n_nodes; ++i)
        fprintf(f, "          %.9g %.9g %.9g\n", m->nodes[i].x, m->nodes[i].y, m->nodes[i].z);
    fprintf(f, "        </DataArray>\n      </Points>\n      <Cells>\n");
    auto ints = [&](const char* name, const std::vector<int64_t>& a, size_t per_line) {
        fprintf(f, "        <DataArray type=\"Int64\" Name=\"%s\" format=\"ascii\">\n", name);
        for (size_t i = 0; i < a.size(); ++i)
            fprintf(f, "%s%lld%s", i % per_line ? " " : "          ", (long long)a[i],
                    (i % per_line == per_line - 1 || i + 1 == a.size()) ? "\n" : "");
        fprintf(f, "        </DataArray>\n");
    };
    ints("connectivity", c.conn, 8);
    ints("offsets", c.offsets, 8);
    ints("types", std::vector<int64_t>(m->n_cells, 42), 16);
    ints("faces", c.faces, 16);
    ints("faceoffsets", c.faceoffsets, 8);
    fprintf(f, "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
    const bool ok = fclose(f) == 0;
    if (!ok) set_error("FieldsWriteVtu: write failed");
    return ok ? 0 : 1;
}

int gbFieldsWriteVtuBinary(const char* filename, cuMesh* mesh, const FvmField** vars, const size_t nvars) {
    clear_error();
    if (!check_args(filename, mesh, vars, nvars, "gbFieldsWriteVtuBinary")) return 1;
    const cuMeshBase* m = mesh->_cpu;
    FILE* f = fopen(filename, "wb");
    if (!f) { set_error(std::string("gbFieldsWriteVtuBinary: cannot open ") + filename); return 1; }
    const Cells c = polyhedra(m);
    // appended blocks: each a UInt64 byte count, then the raw array
    struct Block { const void* data; uint64_t bytes; std::vector<float> own_f; std::vector<int64_t> own_i; };
    std::vector<Block> blocks;
    std::string xml;
    char buf[512];
    uint64_t off = 0;
    auto add = [&](Block b, const std::string& head) {
        snprintf(buf, sizeof(buf), "%s format=\"appended\" offset=\"%llu\"/>\n", head.c_str(), (unsigned long long)off);
        xml += buf;
        off += 8 + b.bytes;
        blocks.push_back(std::move(b));
    };
    xml += "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
           "header_type=\"UInt64\">\n  <UnstructuredGrid>\n";
    snprintf(buf, sizeof(buf), "    <Piece NumberOfPoints=\"%zu\" NumberOfCells=\"%zu\">\n      <CellData>\n", m->n_nodes,
             m->n_cells);
    xml += buf;
    for (size_t i = 0; i < nvars; ++i) {
        const FvmField* v = vars[i];
        const int comps = v->_cpu->elem_size == 4 ? 1 : 3;
        Block b{v->_cpu->value, (uint64_t)m->n_cells * comps * 4, {}, {}};
        std::string head = std::string("        <DataArray type=\"Float32\" Name=\"") + v->name + "\"" +
                           (comps == 3 ? " NumberOfComponents=\"3\"" : "");
        add(std::move(b), head);
    }
    xml += "      </CellData>\n      <Points>\n";
    {
        Block b{nullptr, (uint64_t)m->n_nodes * 12, {}, {}};
        b.own_f.resize(3 * m->n_nodes);
        for (size_t i = 0; i < m->n_nodes; ++i) {
            b.own_f[3 * i] = m->nodes[i].x;
            b.own_f[3 * i + 1] = m->nodes[i].y;
            b.own_f[3 * i + 2] = m->nodes[i].z;
        }
        add(std::move(b), "        <DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\"");
    }
    xml += "      </Points>\n      <Cells>\n";
    auto add_ints = [&](const char* name, std::vector<int64_t> a) {
        Block b{nullptr, (uint64_t)a.size() * 8, {}, std::move(a)};
        add(std::move(b), std::string("        <DataArray type=\"Int64\" Name=\"") + name + "\"");
    };
    add_ints("connectivity", c.conn);
    add_ints("offsets", c.offsets);
    add_ints("types", std::vector<int64_t>(m->n_cells, 42));
    add_ints("faces", c.faces);
    add_ints("faceoffsets", c.faceoffsets);
    xml += "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">\n   _";
    bool ok = fwrite(xml.data(), 1, xml.size(), f) == xml.size();
    for (const Block& b : blocks) {
        const void* p = b.data ? b.data : (!b.own_f.empty() ? (const void*)b.own_f.data() : (const void*)b.own_i.data());
        ok = ok && fwrite(&b.bytes, 8, 1, f) == 1 && (b.bytes == 0 || fwrite(p, 1, b.bytes, f) == b.bytes);
    }
    const char* tail = "\n  </AppendedData>\n</VTKFile>\n";
    ok = ok && fwrite(tail, 1, strlen(tail), f) == strlen(tail);
    ok = (fclose(f) == 0) && ok;
    if (!ok) set_error("gbFieldsWriteVtuBinary: write failed");
    return ok ? 0 : 1;
}

}  // extern "C"
