// MeshData construction (see meshdata.h).
#include "meshdata.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

#include "config.h"

namespace transfer {

namespace {
struct V3 {
    double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct TriKey {
    tr_idx a, b, c;
    bool operator==(const TriKey &o) const { return a == o.a && b == o.b && c == o.c; }
};
struct TriHash {
    size_t operator()(const TriKey &k) const {
        uint64_t h = k.a * 0x9E3779B97F4A7C15ULL;
        h ^= (k.b + 0x632BE59BD9B4E019ULL) + (h << 6) + (h >> 2);
        h ^= (k.c + 0x85EBCA77C2B2AE63ULL) + (h << 6) + (h >> 2);
        return static_cast<size_t>(h);
    }
};
TriKey make_key(tr_idx a, tr_idx b, tr_idx c) {
    tr_idx v[3] = {a, b, c};
    std::sort(v, v + 3);
    return {v[0], v[1], v[2]};
}
}  // namespace

MeshData MeshData::from_tets(tr_idx nP, const double *xyz, tr_idx nT, const tr_idx *tets,
                             const int32_t *region, const RegionParams &rp,
                             const int32_t *vertex_side_mask) {
    if (nP == 0 || nT == 0) throw std::invalid_argument("empty mesh");
    MeshData md;
    md.nP = nP;
    md.nT = nT;
    md.coords.assign(xyz, xyz + 3 * static_cast<size_t>(nP));
    md.region.assign(region, region + nT);
    md.mesh.resize(nT);
    int nreg = static_cast<int>(rp.kappa.size()) - 1;
    bool scatter = false;
    for (size_t r = 1; r < rp.albedo.size(); ++r)
        if (rp.albedo[r] != 0.0) scatter = true;
    if (scatter) md.kappa_abs_volume.resize(nT);
    auto P = [&](tr_idx v) { return V3{xyz[3 * v], xyz[3 * v + 1], xyz[3 * v + 2]}; };

    for (tr_idx t = 0; t < nT; ++t) {
        tr_tetrahedron &T = md.mesh[t];
        for (int k = 0; k < 4; ++k) {
            T.p[k] = tets[4 * t + k];
            if (T.p[k] >= nP) throw std::invalid_argument("tet vertex index out of range");
        }
        int reg = region[t];
        if (reg < 1 || reg > nreg) throw std::invalid_argument("tet region out of range");
        V3 x0 = P(T.p[0]), e1 = sub(P(T.p[1]), x0), e2 = sub(P(T.p[2]), x0), e3 = sub(P(T.p[3]), x0);
        double vol = std::fabs(dot(e1, cross(e2, e3))) / 6.0;
        if (!(vol > 0.0)) throw std::invalid_argument("degenerate tetrahedron");
        T.kappa_volume = vol * rp.kappa[reg];
        T.I_p = rp.Ip[reg];
        if (scatter) {
            double alb = reg < static_cast<int>(rp.albedo.size()) ? rp.albedo[reg] : 0.0;
            md.kappa_abs_volume[t] = vol * rp.kappa[reg] * (1.0 - alb);
        }
        for (int j = 0; j < 4; ++j) {
            tr_idx q[3];
            int c = 0;
            for (int k = 0; k < 4; ++k)
                if (k != j) q[c++] = T.p[k];
            V3 a = P(q[0]), n = cross(sub(P(q[1]), a), sub(P(q[2]), a));
            n = {0.5 * n.x, 0.5 * n.y, 0.5 * n.z};
            if (dot(n, sub(a, P(T.p[j]))) < 0) n = {-n.x, -n.y, -n.z};
            T.s[j][0] = n.x;
            T.s[j][1] = n.y;
            T.s[j][2] = n.z;
        }
    }

    // vertex -> tet CSR (tets ascending)
    md.tetstart.assign(nP + 1, 0);
    for (tr_idx t = 0; t < nT; ++t)
        for (int k = 0; k < 4; ++k) md.tetstart[md.mesh[t].p[k] + 1]++;
    for (tr_idx v = 0; v < nP; ++v) md.tetstart[v + 1] += md.tetstart[v];
    md.tetidx.resize(md.tetstart[nP]);
    md.tetpos.resize(md.tetstart[nP]);
    {
        std::vector<tr_idx> fill(md.tetstart.begin(), md.tetstart.end() - 1);
        for (tr_idx t = 0; t < nT; ++t)
            for (int k = 0; k < 4; ++k) {
                tr_idx v = md.mesh[t].p[k];
                md.tetidx[fill[v]] = t;
                md.tetpos[fill[v]] = static_cast<tr_idx>(k);
                fill[v]++;
            }
    }

    // boundary faces: faces owned by exactly one tet
    std::unordered_map<TriKey, int, TriHash> count;
    count.reserve(static_cast<size_t>(nT) * 3);
    for (tr_idx t = 0; t < nT; ++t) {
        const tr_idx *p = md.mesh[t].p;
        for (int j = 0; j < 4; ++j) {
            tr_idx q[3];
            int c = 0;
            for (int k = 0; k < 4; ++k)
                if (k != j) q[c++] = p[k];
            count[make_key(q[0], q[1], q[2])]++;
        }
    }
    for (tr_idx t = 0; t < nT; ++t) {
        const tr_tetrahedron &T = md.mesh[t];
        for (int j = 0; j < 4; ++j) {
            tr_idx q[3];
            int c = 0;
            for (int k = 0; k < 4; ++k)
                if (k != j) q[c++] = T.p[k];
            auto it = count.find(make_key(q[0], q[1], q[2]));
            if (it->second > 2) throw std::invalid_argument("non-manifold mesh: face shared by >2 tets");
            if (it->second != 1) continue;
            tr_face F;
            F.p[0] = q[0];
            F.p[1] = q[1];
            F.p[2] = q[2];
            F.p[3] = 0;
            F.s[0] = T.s[j][0];
            F.s[1] = T.s[j][1];
            F.s[2] = T.s[j][2];
            F._pad[0] = F._pad[1] = F._pad[2] = 0.0;
            md.bnd.push_back(F);
            int side = -1;
            if (vertex_side_mask) {
                int m = vertex_side_mask[q[0]] & vertex_side_mask[q[1]] & vertex_side_mask[q[2]];
                for (int b = 0; b < 6; ++b)
                    if (m == (1 << b)) side = b;
            }
            md.face_side.push_back(side);
        }
    }
    md.nF = static_cast<tr_idx>(md.bnd.size());

    md.facestart.assign(nP + 1, 0);
    for (const tr_face &F : md.bnd)
        for (int k = 0; k < 3; ++k) md.facestart[F.p[k] + 1]++;
    for (tr_idx v = 0; v < nP; ++v) md.facestart[v + 1] += md.facestart[v];
    md.faceidx.resize(md.facestart[nP]);
    md.facepos.resize(md.facestart[nP]);
    {
        std::vector<tr_idx> fill(md.facestart.begin(), md.facestart.end() - 1);
        for (tr_idx f = 0; f < md.nF; ++f)
            for (int k = 0; k < 3; ++k) {
                tr_idx v = md.bnd[f].p[k];
                md.faceidx[fill[v]] = f;
                md.facepos[fill[v]] = static_cast<tr_idx>(k);
                fill[v]++;
            }
    }
    return md;
}

MeshData MeshData::kuhn(const KuhnParams &kp, const RegionParams &rp) {
    const int nx = kp.n[0], ny = kp.n[1], nz = kp.n[2];
    if (nx < 1 || ny < 1 || nz < 1) throw std::invalid_argument("kuhn: n must be >= 1");
    const double hx = (kp.box[1] - kp.box[0]) / nx, hy = (kp.box[3] - kp.box[2]) / ny,
                 hz = (kp.box[5] - kp.box[4]) / nz;
    if (!(hx > 0 && hy > 0 && hz > 0)) throw std::invalid_argument("kuhn: empty box");
    if (kp.jitter < 0 || kp.jitter >= 0.5) throw std::invalid_argument("kuhn: jitter must be in [0,0.5)");
    const size_t NX = nx + 1, NY = ny + 1, NZ = nz + 1;
    const size_t nPall = NX * NY * NZ;
    if (nPall > 0xFFFFFFF0ULL || 6ULL * nx * ny * nz > 0x3FFFFFFFULL)
        throw std::invalid_argument("kuhn: mesh too large for 32-bit indices");
    std::vector<double> xyz(3 * nPall);
    std::vector<int32_t> side(nPall);
    SplitMix64 rng(kp.seed);
    for (size_t k = 0; k < NZ; ++k)
        for (size_t j = 0; j < NY; ++j)
            for (size_t i = 0; i < NX; ++i) {
                size_t v = i + NX * (j + NY * k);
                double x = kp.box[0] + i * hx, y = kp.box[2] + j * hy, z = kp.box[4] + k * hz;
                int m = 0;
                if (i == 0) m |= 1;
                if (i == NX - 1) m |= 2;
                if (j == 0) m |= 4;
                if (j == NY - 1) m |= 8;
                if (k == 0) m |= 16;
                if (k == NZ - 1) m |= 32;
                if (m == 0 && kp.jitter > 0) {
                    x += (2.0 * rng.uniform() - 1.0) * kp.jitter * hx;
                    y += (2.0 * rng.uniform() - 1.0) * kp.jitter * hy;
                    z += (2.0 * rng.uniform() - 1.0) * kp.jitter * hz;
                }
                xyz[3 * v] = x;
                xyz[3 * v + 1] = y;
                xyz[3 * v + 2] = z;
                side[v] = m;
            }
    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const size_t stride[3] = {1, NX, NX * NY};
    std::vector<tr_idx> tets;
    std::vector<int32_t> reg;
    tets.reserve(24ULL * nx * ny * nz);
    reg.reserve(6ULL * nx * ny * nz);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t v0 = i + NX * (j + NY * k);
                for (int q = 0; q < 6; ++q) {
                    size_t v1 = v0 + stride[perm[q][0]];
                    size_t v2 = v1 + stride[perm[q][1]];
                    size_t v3 = v0 + stride[0] + stride[1] + stride[2];
                    size_t vv[4] = {v0, v1, v2, v3};
                    double c[3] = {0, 0, 0};
                    for (int a = 0; a < 4; ++a)
                        for (int d = 0; d < 3; ++d) c[d] += 0.25 * xyz[3 * vv[a] + d];
                    if (kp.ball) {
                        double dx = c[0] - kp.ball_center[0], dy = c[1] - kp.ball_center[1],
                               dz = c[2] - kp.ball_center[2];
                        if (dx * dx + dy * dy + dz * dz > kp.ball_radius * kp.ball_radius) continue;
                    }
                    int r = 1;
                    if (kp.region_kind == 1) {
                        double dx = c[0] - kp.region_arg[0], dy = c[1] - kp.region_arg[1],
                               dz = c[2] - kp.region_arg[2];
                        r = (dx * dx + dy * dy + dz * dz < kp.region_arg[3] * kp.region_arg[3]) ? 1 : 2;
                    } else if (kp.region_kind == 2) {
                        r = (c[0] < kp.region_arg[0]) ? 1 : 2;
                    }
                    for (int a = 0; a < 4; ++a) tets.push_back(static_cast<tr_idx>(vv[a]));
                    reg.push_back(r);
                }
            }
    if (tets.empty()) throw std::invalid_argument("kuhn: no tetrahedra kept");
    if (!kp.ball) {
        return from_tets(static_cast<tr_idx>(nPall), xyz.data(), static_cast<tr_idx>(reg.size()), tets.data(),
                         reg.data(), rp, side.data());
    }
    // compact the vertices the kept tets use (ascending old index)
    std::vector<int64_t> newid(nPall, -1);
    for (tr_idx v : tets) newid[v] = 0;
    std::vector<double> cxyz;
    tr_idx nP = 0;
    for (size_t v = 0; v < nPall; ++v)
        if (newid[v] == 0) {
            newid[v] = nP++;
            cxyz.push_back(xyz[3 * v]);
            cxyz.push_back(xyz[3 * v + 1]);
            cxyz.push_back(xyz[3 * v + 2]);
        }
    for (tr_idx &v : tets) v = static_cast<tr_idx>(newid[v]);
    return from_tets(nP, cxyz.data(), static_cast<tr_idx>(reg.size()), tets.data(), reg.data(), rp, nullptr);
}

MeshData MeshData::read_tmesh(const std::string &path, const RegionParams &rp) {
    std::ifstream in(path);
    std::string magic;
    int version = 0;
    if (!(in >> magic >> version) || magic != "tmesh") throw std::runtime_error("cannot read tmesh " + path);
    size_t nP = 0, nT = 0;
    in >> nP;
    std::vector<double> xyz(3 * nP);
    for (size_t i = 0; i < 3 * nP; ++i) in >> xyz[i];
    in >> nT;
    std::vector<tr_idx> tets(4 * nT);
    std::vector<int32_t> reg(nT);
    for (size_t t = 0; t < nT; ++t) in >> tets[4 * t] >> tets[4 * t + 1] >> tets[4 * t + 2] >> tets[4 * t + 3] >> reg[t];
    if (!in) throw std::runtime_error("truncated tmesh " + path);
    return from_tets(static_cast<tr_idx>(nP), xyz.data(), static_cast<tr_idx>(nT), tets.data(), reg.data(), rp);
}

static RegionParams region_params(const Config &cfg) {
    RegionParams rp;
    int n = cfg.numRegions();
    if (n < 1) throw ConfigError("numregs must be >= 1");
    rp.kappa.assign(n + 1, 0.0);
    rp.Ip.assign(n + 1, 0.0);
    rp.albedo.assign(n + 1, 0.0);
    for (int r = 1; r <= n; ++r) {
        rp.kappa[r] = cfg.getKappa(r);
        rp.Ip[r] = cfg.getIp(r);
        rp.albedo[r] = cfg.region_double(r, "albedo", 0.0);
    }
    return rp;
}

MeshData::MeshData(const Config &cfg) {
    RegionParams rp = region_params(cfg);
    std::string fn = cfg.getMeshFilename();
    if (fn.compare(0, 5, "kuhn:") == 0) {
        KuhnParams kp;
        std::string spec = fn.substr(5);
        for (char &c : spec)
            if (c == ':' || c == ',') c = ' ';
        std::istringstream is(spec);
        if (!(is >> kp.n[0] >> kp.n[1] >> kp.n[2] >> kp.box[0] >> kp.box[1] >> kp.box[2] >> kp.box[3] >>
              kp.box[4] >> kp.box[5] >> kp.jitter))
            throw ConfigError("bad kuhn mesh spec: " + fn);
        unsigned long long seed;
        if (is >> seed) kp.seed = seed;
        std::string rk = cfg.get_string("region_kind", "uniform");
        kp.region_kind = rk == "sphere" ? 1 : rk == "halfspace" ? 2 : 0;
        std::istringstream ra(cfg.get_string("region_arg", "0 0 0 0"));
        ra >> kp.region_arg[0] >> kp.region_arg[1] >> kp.region_arg[2] >> kp.region_arg[3];
        *this = kuhn(kp, rp);
    } else if (fn.size() > 4 && fn.compare(fn.size() - 4, 4, ".vol") == 0) {
        *this = read_vol(fn, rp);
    } else {
        *this = read_tmesh(fn, rp);
    }
}

tr_mesh_view MeshData::view() const {
    tr_mesh_view v;
    v.nP = nP;
    v.nF = nF;
    v.nT = nT;
    v.tetstart = tetstart.data();
    v.tetidx = tetidx.data();
    v.tetpos = tetpos.data();
    v.mesh = mesh.data();
    v.facestart = facestart.data();
    v.faceidx = faceidx.data();
    v.facepos = facepos.data();
    v.bnd = bnd.data();
    return v;
}

}  // namespace transfer
