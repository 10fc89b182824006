// Mesh I/O in place of the reference's absent meshProcessor library: a
// reader of Netgen's ".vol" meshes (the format of the reference's meshfile
// key, radiation.cfg.example) and a writer of legacy VTK unstructured grids
// with the fields main.cpp:209-216 saves (cell vectors, point scalars and
// symmetric point tensors).
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "meshdata.h"

namespace transfer {

// Netgen .vol: keyword sections, 1-based vertex numbers.
//   points            N, then N lines "x y z"
//   volumeelements    N, then N lines "matnr np p1 .. p_np" (first four = tet)
//   surfaceelements   N, then "surfnr bcnr domin domout np p1 .. p_np"
//   surfaceelementsgi the same followed by np geometry numbers per line
// The region of a tetrahedron is its matnr; a boundary face's bcnr is kept
// in face_bcnr (matched by its vertex set).  Other sections are skipped.
MeshData MeshData::read_vol(const std::string &path, const RegionParams &rp) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open vol mesh " + path);
    std::vector<double> xyz;
    std::vector<tr_idx> tets;
    std::vector<int32_t> reg;
    std::map<std::array<tr_idx, 3>, int32_t> bcnr;
    std::string tok;
    bool have_points = false, have_tets = false;
    while (in >> tok) {
        if (tok == "points") {
            size_t n = 0;
            in >> n;
            xyz.resize(3 * n);
            for (size_t i = 0; i < 3 * n; ++i) in >> xyz[i];
            have_points = true;
        } else if (tok == "volumeelements") {
            size_t n = 0;
            in >> n;
            tets.resize(4 * n);
            reg.resize(n);
            for (size_t t = 0; t < n; ++t) {
                int mat = 0, np = 0;
                in >> mat >> np;
                if (np < 4) throw std::runtime_error("vol mesh: volume element with fewer than 4 points");
                for (int k = 0; k < np; ++k) {
                    long long p = 0;
                    in >> p;
                    if (k < 4) {
                        if (p < 1) throw std::runtime_error("vol mesh: bad vertex number");
                        tets[4 * t + k] = static_cast<tr_idx>(p - 1);
                    }
                }
                reg[t] = mat;
            }
            have_tets = true;
        } else if (tok == "surfaceelements" || tok == "surfaceelementsgi") {
            const bool gi = tok == "surfaceelementsgi";
            size_t n = 0;
            in >> n;
            for (size_t f = 0; f < n; ++f) {
                int surfnr = 0, bc = 0, din = 0, dout = 0, np = 0;
                in >> surfnr >> bc >> din >> dout >> np;
                std::vector<long long> p(np);
                for (int k = 0; k < np; ++k) in >> p[k];
                if (gi)
                    for (int k = 0; k < np; ++k) {
                        long long skip;
                        in >> skip;
                    }
                if (np >= 3) {
                    std::array<tr_idx, 3> key = {static_cast<tr_idx>(p[0] - 1), static_cast<tr_idx>(p[1] - 1),
                                                 static_cast<tr_idx>(p[2] - 1)};
                    std::sort(key.begin(), key.end());
                    bcnr[key] = bc;
                }
            }
        } else if (tok == "endmesh") {
            break;
        }
        if (!in) throw std::runtime_error("truncated vol mesh " + path);
    }
    if (!have_points || !have_tets) throw std::runtime_error("vol mesh without points or volume elements: " + path);
    const size_t nP = xyz.size() / 3;
    for (tr_idx v : tets)
        if (v >= nP) throw std::runtime_error("vol mesh: vertex number out of range");
    MeshData md = from_tets(static_cast<tr_idx>(nP), xyz.data(), static_cast<tr_idx>(reg.size()), tets.data(),
                            reg.data(), rp);
    md.face_bcnr.assign(md.nF, -1);
    for (tr_idx f = 0; f < md.nF; ++f) {
        std::array<tr_idx, 3> key = {md.bnd[f].p[0], md.bnd[f].p[1], md.bnd[f].p[2]};
        std::sort(key.begin(), key.end());
        auto it = bcnr.find(key);
        if (it != bcnr.end()) md.face_bcnr[f] = it->second;
    }
    return md;
}

namespace {
void put_be(std::ostream &o, const void *p, size_t bytes) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = bytes; i-- > 0;) o.put(static_cast<char>(b[i]));
}
void put_real(std::ostream &o, double v, int real_bytes) {
    if (real_bytes == 4) {
        const float f = static_cast<float>(v);
        put_be(o, &f, 4);
    } else {
        put_be(o, &v, 8);
    }
}
void put_i32(std::ostream &o, int32_t v) { put_be(o, &v, 4); }
}  // namespace

// Legacy VTK, binary (big-endian), reals of real_bytes (4 or 8).
void write_vtk(const std::string &path, const MeshData &md, int real_bytes, int nfields, const tr_vtk_field *fields) {
    if (real_bytes != 4 && real_bytes != 8) throw std::runtime_error("write_vtk: real_bytes must be 4 or 8");
    if (md.coords.size() != 3ull * md.nP) throw std::runtime_error("write_vtk: mesh without vertex coordinates");
    std::ofstream o(path, std::ios::binary);
    if (!o) throw std::runtime_error("cannot write " + path);
    const char *rt = real_bytes == 4 ? "float" : "double";
    o << "# vtk DataFile Version 3.0\ntransfer_b200 solution\nBINARY\nDATASET UNSTRUCTURED_GRID\n";
    o << "POINTS " << md.nP << " " << rt << "\n";
    for (size_t i = 0; i < 3ull * md.nP; ++i) put_real(o, md.coords[i], real_bytes);
    o << "\nCELLS " << md.nT << " " << 5ull * md.nT << "\n";
    for (tr_idx t = 0; t < md.nT; ++t) {
        put_i32(o, 4);
        for (int k = 0; k < 4; ++k) put_i32(o, static_cast<int32_t>(md.mesh[t].p[k]));
    }
    o << "\nCELL_TYPES " << md.nT << "\n";
    for (tr_idx t = 0; t < md.nT; ++t) put_i32(o, 10);  // VTK_TETRA
    o << "\n";
    for (int pass = 0; pass < 2; ++pass) {  // cell data, then point data
        const int loc = pass == 0 ? TR_VTK_CELL : TR_VTK_POINT;
        const size_t n = loc == TR_VTK_CELL ? md.nT : md.nP;
        bool header = false;
        for (int i = 0; i < nfields; ++i) {
            const tr_vtk_field &f = fields[i];
            if (f.location != loc) continue;
            if (!f.name || !f.data || (f.kind != TR_VTK_SCALAR && f.kind != TR_VTK_VECTOR && f.kind != TR_VTK_TENSOR))
                throw std::runtime_error("write_vtk: bad field");
            if (!header) {
                o << (loc == TR_VTK_CELL ? "CELL_DATA " : "POINT_DATA ") << n << "\n";
                header = true;
            }
            if (f.kind == TR_VTK_SCALAR) {
                o << "SCALARS " << f.name << " " << rt << " 1\nLOOKUP_TABLE default\n";
                for (size_t j = 0; j < n; ++j) put_real(o, f.data[j], real_bytes);
            } else if (f.kind == TR_VTK_VECTOR) {
                o << "VECTORS " << f.name << " " << rt << "\n";
                for (size_t j = 0; j < n; ++j)
                    for (int c = 0; c < 3; ++c) put_real(o, f.data[c * n + j], real_bytes);
            } else {
                // symmetric tensor from its 6 components xx xy xz yy yz zz
                static const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
                o << "TENSORS " << f.name << " " << rt << "\n";
                for (size_t j = 0; j < n; ++j)
                    for (int c = 0; c < 9; ++c) put_real(o, f.data[sym[c] * n + j], real_bytes);
            }
            o << "\n";
        }
    }
    if (!o) throw std::runtime_error("write error on " + path);
}

}  // namespace transfer
