// MeshData: the reference's host problem data (MeshData.h:13-32,
// MeshData.cpp:9-94) built from a tetrahedral mesh, plus the mesh sources
// this project has in place of the absent meshProcessor library: a
// Kuhn-split box / ball generator and a plain-text tetrahedral mesh reader.
//
// Record conventions (identical to what MeshData.cpp:56-93 produces from a
// mesh whose tet-face normals point inward):
//   tetrahedron.s[j]  = OUTWARD area normal of the face opposite local vertex
//                       j, so grad(lambda_j) = -s[j] / (3V) and sum_j s[j] = 0;
//   kappa_volume      = kappa(region) * V,  I_p = Ip(region);
//   face.p[0..2]      = the owning tet's vertices except the opposite one,
//                       in local order; face.s = outward area normal;
//   tetstart/tetidx/tetpos: vertex -> (tet, local index), tets ascending;
//   facestart/faceidx/facepos: vertex -> (boundary face, 0..2), ascending.
// Boundary faces are listed in (tet, local face) order of their owner.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/transfer_b200.h"

namespace transfer {

class Config;

struct RegionParams {
    std::vector<double> kappa, Ip, albedo;   // [nreg+1], index 0 unused
};

struct KuhnParams {
    int n[3] = {1, 1, 1};
    double box[6] = {0, 1, 0, 1, 0, 1};
    double jitter = 0.0;
    uint64_t seed = 20261203ULL;
    int region_kind = 0;          // 0 uniform(1), 1 sphere, 2 half space
    double region_arg[4] = {0, 0, 0, 0};
    bool ball = false;
    double ball_center[3] = {0, 0, 0};
    double ball_radius = 1.0;
};

struct MeshData {
    tr_idx nP = 0, nF = 0, nT = 0;
    std::vector<tr_idx> tetstart, tetidx, tetpos;
    std::vector<tr_tetrahedron> mesh;
    std::vector<tr_idx> facestart, faceidx, facepos;
    std::vector<tr_face> bnd;

    std::vector<double> coords;             // [nP][3]
    std::vector<int32_t> region;            // [nT]
    std::vector<double> kappa_abs_volume;   // [nT] or empty (no scattering)
    std::vector<int32_t> face_side;         // [nF] box side 0..5 or -1
    std::vector<int32_t> face_bcnr;         // [nF] bc number of a .vol surface element, -1 if none

    MeshData() {}
    // MeshData(const Config &) (MeshData.cpp:9): meshfile is a Netgen mesh
    // ("*.vol", the reference's format), a plain-text mesh ("*.tmesh") or a
    // Kuhn box spec "kuhn:nx,ny,nz:x0,x1,y0,y1,z0,z1:jitter:seed"; regions of
    // a Kuhn box come from the additive keys region_kind
    // (uniform|sphere|halfspace) and region_arg (4 numbers).
    explicit MeshData(const Config &cfg);

    static MeshData from_tets(tr_idx nP, const double *xyz, tr_idx nT, const tr_idx *tets,
                              const int32_t *region, const RegionParams &rp,
                              const int32_t *vertex_side_mask = nullptr);
    static MeshData kuhn(const KuhnParams &kp, const RegionParams &rp);
    static MeshData read_tmesh(const std::string &path, const RegionParams &rp);
    static MeshData read_vol(const std::string &path, const RegionParams &rp);  // meshio.cpp

    tr_mesh_view view() const;
};

// splitmix64 (Steele, Lea & Flood 2014): the generator's jitter source.
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// legacy VTK writer (meshio.cpp)
void write_vtk(const std::string &path, const MeshData &md, int real_bytes, int nfields, const tr_vtk_field *fields);

}  // namespace transfer
