// tr_ctx creation (CudaContext::CudaContext + DeviceMeshData +
// DeviceAngularData, CudaContext.cpp:24-50, DeviceMeshData.cpp:8-52,
// DeviceAngularData.cpp:7-67): validates the reference's MeshData /
// AngularData arrays, assembles the vertex-pair operator described in
// internal.h on the host, and uploads it in FP64 and FP32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "solver.h"

namespace transfer {

namespace {

struct Edge {
    uint32_t u;
    double k9[9];             // K[i][j] before symmetrisation
    double c[kCoefStride];
};

// reference axis choice for a boundary face (kernels.cu:419-425)
inline int face_axis(const tr_face &f, double *surf) {
    double s = std::fabs(f.s[0] + f.s[1] + f.s[2]);
    *surf = s;
    if (2 * std::fabs(f.s[0]) > s) return 0;
    if (2 * std::fabs(f.s[1]) > s) return 1;
    return 2;
}

std::string validate(const tr_mesh_view *m, const tr_angular_view *a) {
    if (!m || !a) return "null mesh or angular view";
    if (m->nP == 0 || m->nT == 0) return "empty mesh";
    if (!m->tetstart || !m->tetidx || !m->tetpos || !m->mesh) return "null tet arrays";
    if (m->nF && (!m->bnd)) return "null boundary face array";
    if (!m->facestart || !m->faceidx || !m->facepos) return "null boundary CSR arrays";
    if (!a->omega || !a->omega_pos || !a->Ox || !a->Oy || !a->Oz) return "null angular tables";
    bool slm_ok = false;
    for (int k = 0; k <= TR_MAXK_MAX; ++k)
        if (a->slm == static_cast<tr_idx>((1 + k) * (1 + 2 * k))) slm_ok = true;
    if (!slm_ok) return "slm is not (1+maxk)(1+2maxk) for maxk <= 7";
    if (static_cast<uint64_t>(m->nP) * 128 >= 0xFFFFFFFFULL) return "mesh too large for 32-bit vector offsets";
    if (m->tetstart[0] != 0) return "tetstart[0] != 0";
    for (tr_idx v = 0; v < m->nP; ++v)
        if (m->tetstart[v + 1] < m->tetstart[v]) return "tetstart not monotonic";
    for (tr_idx j = 0; j < m->tetstart[m->nP]; ++j) {
        if (m->tetidx[j] >= m->nT) return "tetidx out of range";
        if (m->tetpos[j] > 3) return "tetpos out of range";
    }
    for (tr_idx t = 0; t < m->nT; ++t) {
        const tr_tetrahedron &T = m->mesh[t];
        for (int k = 0; k < 4; ++k)
            if (T.p[k] >= m->nP) return "tetrahedron vertex out of range";
        if (!(T.kappa_volume > 0.0) || !std::isfinite(T.kappa_volume)) return "kappa_volume must be positive";
        for (int k = 0; k < 4; ++k)
            for (int d = 0; d < 3; ++d)
                if (!std::isfinite(T.s[k][d])) return "non-finite face normal";
    }
    for (tr_idx v = 0; v < m->nP; ++v)
        for (tr_idx j = m->tetstart[v]; j < m->tetstart[v + 1]; ++j)
            if (m->mesh[m->tetidx[j]].p[m->tetpos[j]] != v) return "tetidx/tetpos inconsistent with tet vertices";
    if (m->facestart[0] != 0) return "facestart[0] != 0";
    for (tr_idx v = 0; v < m->nP; ++v)
        if (m->facestart[v + 1] < m->facestart[v]) return "facestart not monotonic";
    for (tr_idx j = 0; j < m->facestart[m->nP]; ++j) {
        if (m->faceidx[j] >= m->nF) return "faceidx out of range";
        if (m->facepos[j] > 2) return "facepos out of range";
    }
    for (tr_idx f = 0; f < m->nF; ++f)
        for (int k = 0; k < 3; ++k)
            if (m->bnd[f].p[k] >= m->nP) return "face vertex out of range";
    const size_t n3 = 3ULL * a->slm * a->slm;
    for (size_t i = 0; i < n3; ++i)
        if (a->omega_pos[i] > 2) return "omega_pos out of range";
    return "";
}

template <typename T>
cudaError_t upload(tr_ctx *c, T **dst, const void *src, size_t bytes) {
    if (bytes == 0) bytes = sizeof(T);
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dst), bytes);
    if (e != cudaSuccess) return e;
    c->allocations.push_back(*dst);
    c->device_bytes += bytes;
    if (src) return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    return cudaMemset(*dst, 0, bytes);
}

template <typename T>
std::vector<T> to_type(const std::vector<double> &v) {
    std::vector<T> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = static_cast<T>(v[i]);
    return o;
}

// The contraction rounds (the Runs layout of internal.h) of the lists
// lists[lm] = {(q * 256 + lms, weight)} for L lanes, offsets q * sa + lms
// into a table of `word`-byte elements.  schedule_runs lays out one choice
// (the harmonics taken in `order`, chunks of R) and prices it in
// shared-memory wavefronts; make_runs keeps the cheapest over R and a few
// harmonic orders.  Within a chunk the entries may come in any order; the
// order is chosen so that the lanes of a step read distinct banks (word 4:
// bank = offset mod 32 over the warp; word 8: bank pair = offset mod 16
// within each half-warp, a 64-bit access being served per 16 lanes).
struct RunsHost {
    uint32_t rounds = 0, R = 0, L = 0;
    std::vector<unsigned char> tab;
    std::vector<uint32_t> span;  // [slm]: first chunk | end chunk << 16
    uint64_t cost = UINT64_MAX;  // shared-memory wavefronts of one contraction
};
typedef std::pair<uint32_t, double> RunEnt;
RunsHost schedule_runs(const std::vector<std::vector<RunEnt>> &lists, const std::vector<uint32_t> &order, uint32_t L,
                       uint32_t sa, int word, uint32_t R) {
    const uint32_t slm = static_cast<uint32_t>(lists.size());
    RunsHost H;
    H.L = L;
    H.R = R;
    // chunks of consecutive entries, harmonic after harmonic in `order`
    std::vector<std::vector<RunEnt>> chunk;
    H.span.assign(slm, 0u);
    for (uint32_t lm : order) {
        const uint32_t c0 = static_cast<uint32_t>(chunk.size());
        for (size_t i = 0; i < lists[lm].size(); i += R)
            chunk.emplace_back(lists[lm].begin() + static_cast<std::ptrdiff_t>(i),
                               lists[lm].begin() + static_cast<std::ptrdiff_t>(std::min(lists[lm].size(), i + R)));
        H.span[lm] = c0 | static_cast<uint32_t>(chunk.size()) << 16;
    }
    H.rounds = std::max<uint32_t>(1, static_cast<uint32_t>((chunk.size() + L - 1) / L));
    const size_t n = static_cast<size_t>(H.rounds) * R * L;
    std::vector<double> w(n, 0.0);
    std::vector<uint32_t> o(n, 0u);
    // Per round and bank group (FP64: each half-warp; FP32: the warp), the
    // entries are the edges of a bipartite multigraph lanes x banks, and the
    // steps 0..R-1 its colours: a proper edge colouring is a schedule whose
    // every step hits distinct banks.  Edges are coloured one by one; when
    // the lane's first free colour a is taken at the bank, the bank's free
    // colour b is swapped with a along the a/b alternating path from the
    // bank (which cannot reach the lane, the graph being bipartite) --
    // Konig's construction, which succeeds whenever no bank has more than R
    // entries.  Entries of a bank that has more take any free step of their
    // lane (a conflict).  Unused steps (weight 0) read a cell on a bank that
    // step leaves free, among the cells every vertex writes (rows q < 6,
    // columns lms < slm): a row's pad column is never written, and 0 times
    // whatever it holds need not be 0.
    const uint32_t nbank = word == 8 ? 16 : 32, group = std::min<uint32_t>(L, nbank);
    std::vector<int> readable(nbank, -1);  // per bank, a written cell on it
    for (uint32_t q = 0; q < static_cast<uint32_t>(kSymRows); ++q)
        for (uint32_t lms = 0; lms < slm; ++lms)
            if (readable[(q * sa + lms) % nbank] < 0) readable[(q * sa + lms) % nbank] = static_cast<int>(q * sa + lms);
    struct BankEdge {
        uint32_t lane, bank, off;
        double w;
        int colour;
    };
    for (uint32_t r = 0; r < H.rounds; ++r)
        for (uint32_t g0 = 0; g0 < L; g0 += group) {
            std::vector<BankEdge> ed;
            for (uint32_t l = g0; l < g0 + group; ++l) {
                const size_t c = static_cast<size_t>(r) * L + l;
                if (c >= chunk.size()) continue;
                for (const RunEnt &x : chunk[c]) {
                    const uint32_t off = (x.first >> 8) * sa + (x.first & 255u);
                    ed.push_back(BankEdge{l - g0, off % nbank, off, x.second, -1});
                }
            }
            std::vector<int> at_lane(static_cast<size_t>(group) * R, -1), at_bank(static_cast<size_t>(nbank) * R, -1);
            auto set = [&](int e, int col) {
                ed[e].colour = col;
                at_lane[ed[e].lane * R + col] = e;
                at_bank[ed[e].bank * R + col] = e;
            };
            auto unset = [&](int e) {
                at_lane[ed[e].lane * R + ed[e].colour] = -1;
                at_bank[ed[e].bank * R + ed[e].colour] = -1;
            };
            std::vector<int> leftover;
            for (int e = 0; e < static_cast<int>(ed.size()); ++e) {
                const uint32_t l = ed[e].lane, bk = ed[e].bank;
                int ca = -1, cb = -1;
                for (uint32_t c = 0; c < R && ca < 0; ++c)
                    if (at_lane[l * R + c] < 0) ca = static_cast<int>(c);
                for (uint32_t c = 0; c < R && cb < 0; ++c)
                    if (at_bank[bk * R + c] < 0) cb = static_cast<int>(c);
                if (cb < 0) {
                    leftover.push_back(e);
                    continue;
                }
                if (at_bank[bk * R + ca] >= 0) {
                    // swap ca and cb along the path bank -ca- lane -cb- bank ...
                    std::vector<int> path;
                    uint32_t node = bk;
                    bool on_bank = true;
                    int col = ca;
                    for (;;) {
                        const int f = on_bank ? at_bank[node * R + col] : at_lane[node * R + col];
                        if (f < 0) break;
                        path.push_back(f);
                        node = on_bank ? ed[f].lane : ed[f].bank;
                        on_bank = !on_bank;
                        col = col == ca ? cb : ca;
                    }
                    for (int f : path) unset(f);
                    for (int f : path) set(f, ed[f].colour == ca ? cb : ca);
                }
                set(e, ca);
            }
            for (int e : leftover)
                for (uint32_t c = 0; c < R; ++c)
                    if (at_lane[ed[e].lane * R + c] < 0) {
                        ed[e].colour = static_cast<int>(c);
                        at_lane[ed[e].lane * R + c] = e;
                        break;
                    }
            for (const BankEdge &x : ed) {
                const size_t at = (static_cast<size_t>(r) * R + static_cast<uint32_t>(x.colour)) * L + g0 + x.lane;
                w[at] = x.w;
                o[at] = x.off;
            }
            for (uint32_t c = 0; c < R; ++c)
                for (uint32_t l = 0; l < group; ++l) {
                    if (at_lane[l * R + c] >= 0) continue;
                    uint32_t off = 0;  // offset 0 (S[0][0]) when no free bank has a readable cell
                    for (uint32_t bk = 0; bk < nbank; ++bk)
                        if (at_bank[bk * R + c] < 0 && readable[bk] >= 0) {
                            off = static_cast<uint32_t>(readable[bk]);
                            at_bank[bk * R + c] = static_cast<int>(ed.size());  // taken by this unused step
                            break;
                        }
                    o[(static_cast<size_t>(r) * R + c) * L + g0 + l] = off;
                }
        }
    // price: per step the entry loads (FP32 one 8-byte pair: 2 wavefronts;
    // FP64 weight and offset: 3) and the table reads (the most distinct
    // addresses on one bank, per bank group); per round the chunk-sum store
    const uint32_t nbk = word == 8 ? 16 : 32;
    uint64_t cost = 0;
    for (size_t k = 0; k < static_cast<size_t>(H.rounds) * R; ++k) {
        cost += word == 8 ? 3 : 2;
        for (uint32_t g0 = 0; g0 < L; g0 += nbk) {
            std::vector<std::vector<uint32_t>> seen(nbk);
            uint64_t most = 1;
            for (uint32_t l = g0; l < std::min(L, g0 + nbk); ++l) {
                const uint32_t off = o[k * L + l];
                auto &v = seen[off % nbk];
                if (std::find(v.begin(), v.end(), off) == v.end()) v.push_back(off);
                most = std::max<uint64_t>(most, v.size());
            }
            cost += most;
        }
    }
    H.cost = cost + 2ull * H.rounds;
    // storage: FP32 (w, o) pairs; FP64 weights then offsets
    if (word == 4) {
        H.tab.resize(n * 8);
        for (size_t i = 0; i < n; ++i) {
            const float wf = static_cast<float>(w[i]);
            std::memcpy(&H.tab[8 * i], &wf, 4);
            std::memcpy(&H.tab[8 * i + 4], &o[i], 4);
        }
    } else {
        H.tab.resize(n * 12);
        std::memcpy(H.tab.data(), w.data(), n * 8);
        std::memcpy(H.tab.data() + n * 8, o.data(), n * 4);
    }
    return H;
}

// The cheapest schedule with at most `cap` chunks (the kernel's room for
// chunk sums): R over the multiples of 4 up to the longest list, harmonic
// order the natural one or one of 31 fixed shuffles (SplitMix64 from a
// constant seed, Fisher-Yates), so that the chunks sharing a round come
// from harmonics whose lists load different banks.  rounds = 0 when no
// schedule fits.
RunsHost make_runs(const std::vector<std::vector<RunEnt>> &lists, uint32_t L, uint32_t sa, int word, uint32_t cap) {
    const uint32_t slm = static_cast<uint32_t>(lists.size());
    size_t longest = 0;
    for (const auto &l : lists) longest = std::max(longest, l.size());
    std::vector<std::vector<uint32_t>> orders(1, std::vector<uint32_t>(slm));
    for (uint32_t i = 0; i < slm; ++i) orders[0][i] = i;
    uint64_t state = 0x5DEECE66Dull;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    for (int k = 0; k < 31; ++k) {
        std::vector<uint32_t> p = orders[0];
        for (uint32_t i = slm; i > 1; --i) std::swap(p[i - 1], p[next() % i]);
        orders.push_back(p);
    }
    RunsHost best;
    best.L = L;
    if (L > 32) return best;
    for (uint32_t R = 4; R < longest + 4; R += 4) {
        uint64_t chunks = 0;
        for (const auto &l : lists) chunks += (l.size() + R - 1) / R;
        if (chunks > cap || chunks >= 0xFFFFu) continue;
        for (const auto &ord : orders) {
            RunsHost h = schedule_runs(lists, ord, L, sa, word, R);
            if (h.cost < best.cost) best = std::move(h);
        }
    }
    if (best.cost == UINT64_MAX) best.rounds = 0;
    return best;
}

template <typename T>
cudaError_t upload_runs(tr_ctx *c, const RunsHost &h, uint32_t slm, Runs<T> &r) {
    if (h.rounds == 0 || h.tab.size() != static_cast<size_t>(h.rounds) * h.R * h.L * (sizeof(T) + 4))
        return cudaErrorInvalidValue;
    unsigned char *tab = nullptr;
    uint32_t *st = nullptr;
    cudaError_t e = upload(c, &tab, h.tab.data(), h.tab.size());
    if (e == cudaSuccess) e = upload(c, &st, h.span.data(), slm * sizeof(uint32_t));
    if (e != cudaSuccess) return e;
    r.rounds = h.rounds;
    r.R = h.R;
    r.L = h.L;
    r.tab = tab;
    r.span = st;
    return cudaSuccess;
}

}  // namespace

cudaError_t operator_init_attributes();

void ctx_free(tr_ctx *c) {
    if (!c) return;
    for (auto &g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (void *p : c->allocations) cudaFree(p);
    if (c->host_pinned) cudaFreeHost(c->host_pinned);
    if (c->stage_in) cudaFreeHost(c->stage_in);
    if (c->stage_out) cudaFreeHost(c->stage_out);
    for (cudaEvent_t e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

tr_status ctx_create(int device, const tr_mesh_view *m, const tr_angular_view *a, const tr_physics_view *ph,
                     tr_ctx **out, std::string &err) {
    err = validate(m, a);
    if (!err.empty()) return TR_ERR_MESH;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        err = "no CUDA device available (this library has no CPU fallback)";
        return TR_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) {
        err = "device index out of range";
        return TR_ERR_INVALID_ARG;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        err = "cudaSetDevice failed";
        return TR_ERR_NO_DEVICE;
    }
    const tr_idx nP = m->nP, nT = m->nT, nF = m->nF, slm = a->slm;
    const int32_t *bc = ph ? ph->face_bc : nullptr;
    const double *finc = ph ? ph->face_incident : nullptr;
    const double *kva = ph ? ph->kappa_abs_volume : nullptr;
    if (ph && ph->surface_mode != TR_SURFACE_AXIS) {
        err = "surface_mode other than TR_SURFACE_AXIS is not supported";
        return TR_ERR_UNSUPPORTED;
    }
    if (bc)
        for (tr_idx f = 0; f < nF; ++f)
            if (bc[f] < 0 || bc[f] > 2) {
                err = "face_bc value out of range";
                return TR_ERR_INVALID_ARG;
            }
    if (bc)
        for (tr_idx f = 0; f < nF; ++f)
            if (bc[f] == TR_BC_INCIDENT && !finc) {
                err = "TR_BC_INCIDENT faces need face_incident";
                return TR_ERR_INVALID_ARG;
            }
    if (bc)
        for (tr_idx f = 0; f < nF; ++f)
            if (bc[f] == TR_BC_REFLECTIVE) {
                err = "TR_BC_REFLECTIVE is not supported by this build";
                return TR_ERR_UNSUPPORTED;
            }

    tr_ctx *c = new tr_ctx();
    c->device = device;
    c->nP = nP;
    c->nT = nT;
    c->nF = nF;
    c->slm = slm;
    c->aslm = (slm + 7) & ~7u;
    c->aslm32 = (slm + 15) & ~15u;
    auto bail = [&](const std::string &msg, tr_status st) {
        err = msg;
        ctx_free(c);
        return st;
    };
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail("cudaGetDeviceProperties failed", TR_ERR_CUDA);
    c->num_sms = prop.multiProcessorCount;

    // ---------------------------------------------------- assembled operator
    std::vector<uint32_t> row(nP + 1, 0);
    std::vector<std::vector<Edge>> edges(nP);
    std::vector<double> inflow;
    bool any_inflow = false;
    if (bc)
        for (tr_idx f = 0; f < nF; ++f)
            if (bc[f] == TR_BC_INCIDENT) any_inflow = true;
    if (any_inflow) inflow.assign(3ULL * nP, 0.0);
#pragma omp parallel for schedule(dynamic, 256)
    for (long vv = 0; vv < static_cast<long>(nP); ++vv) {
        const tr_idx v = static_cast<tr_idx>(vv);
        std::vector<Edge> &E = edges[v];
        auto find = [&](uint32_t u) -> Edge & {
            for (Edge &e : E)
                if (e.u == u) return e;
            Edge ne;
            ne.u = u;
            std::memset(ne.k9, 0, sizeof(ne.k9));
            std::memset(ne.c, 0, sizeof(ne.c));
            E.push_back(ne);
            return E.back();
        };
        for (tr_idx j = m->tetstart[v]; j < m->tetstart[v + 1]; ++j) {
            const tr_idx t = m->tetidx[j], loc = m->tetpos[j];
            const tr_tetrahedron &T = m->mesh[t];
            const double kv = T.kappa_volume, ka = kva ? kva[t] : kv;
            for (int k = 0; k < 4; ++k) {
                Edge &e = find(T.p[k]);
                for (int i = 0; i < 3; ++i)
                    for (int jj = 0; jj < 3; ++jj) e.k9[3 * i + jj] += T.s[loc][i] / kv * (1.0 / 9.0) * T.s[k][jj];
                const double mult = (k == static_cast<int>(loc)) ? 2.0 : 1.0;
                e.c[kRowM] += kv * mult * (1.0 / 20.0);
                e.c[kRowM0] += ka * mult * (1.0 / 20.0);
            }
        }
        for (tr_idx j = m->facestart[v]; j < m->facestart[v + 1]; ++j) {
            const tr_idx fi = m->faceidx[j], loc = m->facepos[j];
            const int kind = bc ? bc[fi] : TR_BC_VACUUM;
            if (kind == TR_BC_REFLECTIVE) continue;
            const tr_face &F = m->bnd[fi];
            double surf;
            const int ax = face_axis(F, &surf);
            if (kind == TR_BC_INCIDENT) inflow[3ULL * v + ax] += finc[fi] * surf * (1.0 / 3.0);
            for (int k = 0; k < 3; ++k)
                find(F.p[k]).c[kRowE + ax] += surf * ((k == static_cast<int>(loc)) ? 2.0 : 1.0) * (1.0 / 12.0);
        }
        for (Edge &e : E) {  // symmetric stiffness rows
            e.c[0] = e.k9[0];
            e.c[1] = e.k9[4];
            e.c[2] = e.k9[8];
            e.c[3] = e.k9[1] + e.k9[3];
            e.c[4] = e.k9[2] + e.k9[6];
            e.c[5] = e.k9[5] + e.k9[7];
        }
        std::sort(E.begin(), E.end(), [](const Edge &x, const Edge &y) { return x.u < y.u; });
    }
    for (tr_idx v = 0; v < nP; ++v) row[v + 1] = row[v] + static_cast<uint32_t>(edges[v].size());
    const size_t nnz = row[nP];
    c->n_edges = nnz;
    std::vector<uint32_t> col(nnz);
    std::vector<double> coef(nnz * kCoefStride);
    std::vector<uint8_t> bmask(nP, 0);
    uint64_t nb = 0;
    for (tr_idx v = 0; v < nP; ++v) {
        size_t o = row[v];
        for (const Edge &e : edges[v]) {
            col[o] = e.u;
            std::memcpy(&coef[o * kCoefStride], e.c, sizeof(e.c));
            bool any = false;
            for (int n = 0; n < 3; ++n)
                if (e.c[kRowE + n] != 0.0) {
                    bmask[v] |= static_cast<uint8_t>(1u << n);
                    any = true;
                }
            nb += any;
            ++o;
        }
    }
    c->n_bnd_edges = nb;

    // ---------------------------------------------------- angular tables
    const size_t ss = static_cast<size_t>(slm) * slm;
    double maxabs = 0.0;
    for (size_t i = 0; i < 3 * ss; ++i) maxabs = std::max(maxabs, std::fabs(a->omega[i]));
    const double drop = 1e-14 * maxabs;
    // per harmonic lm: sum_q,lms W[q][lms] S_sym[q][lms], merging (i,j) and
    // (j,i) into the symmetric row q (kernels.cu:276-282 reads
    // omega[i][lms][lm] and omega_pos[i][lms][lm])
    auto sym_row = [](int i, int j) { return i == j ? i : (i + j == 1 ? 3 : (i + j == 2 ? 4 : 5)); };
    std::vector<std::vector<std::pair<uint32_t, double>>> lists(slm);  // (q * 256 + lms, w)
    for (tr_idx lm = 0; lm < slm; ++lm) {
        std::vector<double> wsum(kSymRows * slm, 0.0);
        std::vector<char> used(kSymRows * slm, 0);
        for (int i = 0; i < 3; ++i)
            for (tr_idx lms = 0; lms < slm; ++lms) {
                const size_t q = (static_cast<size_t>(i) * slm + lms) * slm + lm;
                const double w = a->omega[q];
                if (std::fabs(w) <= drop) continue;
                const int r = sym_row(i, static_cast<int>(a->omega_pos[q]));
                wsum[r * slm + lms] += (r < 3) ? w : 0.5 * w;  // S_sym = S_ij + S_ji
                used[r * slm + lms] = 1;
            }
        for (int r = 0; r < kSymRows; ++r)
            for (tr_idx lms = 0; lms < slm; ++lms)
                if (used[r * slm + lms]) lists[lm].push_back({static_cast<uint32_t>(r * 256 + lms), wsum[r * slm + lms]});
    }
    const uint32_t aslm_max = std::max((slm + 7) & ~7u, (slm + 15) & ~15u);
    const uint32_t cls = (aslm_max + 31) & ~31u;
    const uint32_t a64 = (slm + 7) & ~7u, a32 = (slm + 15) & ~15u;
    const uint32_t satc = (slm + 7) / 8 * 8 + 1;
    // chunk-sum room: the SIMT group slab's part table (runs_part_elems),
    // rows 11-15 of the tensor-core C table
    const RunsHost rs64 = make_runs(lists, group_width(a64), s_row_stride(a64), 8,
                                    runs_part_elems(group_width(a64), harm_per_lane(a64)));
    const RunsHost rs32 = make_runs(lists, group_width(a32), s_row_stride(a32), 4,
                                    runs_part_elems(group_width(a32), harm_per_lane(a32)));
    const RunsHost rt64 = make_runs(lists, 32, satc, 8, 5 * satc);
    const RunsHost rt32 = make_runs(lists, 32, satc, 4, 5 * satc);
    std::vector<double> O(3 * ss), ang_diag(3 * slm), O_diag(3 * slm);
    const double *On[3] = {a->Ox, a->Oy, a->Oz};
    for (int n = 0; n < 3; ++n) {
        std::memcpy(&O[n * ss], On[n], ss * sizeof(double));
        for (tr_idx lm = 0; lm < slm; ++lm) {
            ang_diag[n * slm + lm] = a->omega[(static_cast<size_t>(n) * slm + lm) * slm + lm];
            O_diag[n * slm + lm] = On[n][static_cast<size_t>(lm) * slm + lm];
        }
    }
    // Jacobi: 1 / diag(A)
    std::vector<double> dinv(static_cast<size_t>(nP) * c->aslm, 0.0);
    std::vector<float> dinv32(static_cast<size_t>(nP) * c->aslm32, 0.0f);
    for (tr_idx v = 0; v < nP; ++v) {
        const double *cv = nullptr;
        for (uint32_t e = row[v]; e < row[v + 1]; ++e)
            if (col[e] == v) cv = &coef[static_cast<size_t>(e) * kCoefStride];
        for (tr_idx lm = 0; lm < slm; ++lm) {
            double d = 0.0;
            if (cv) {
                d += (lm == 0) ? cv[kRowM0] : cv[kRowM];
                for (int i = 0; i < 3; ++i) {  // omega_pos[i][lm][lm] = i: the K_ii rows
                    const size_t q = (static_cast<size_t>(i) * slm + lm) * slm + lm;
                    d += a->omega[q] * cv[i];
                }
            }
            if (cv)
                for (int n = 0; n < 3; ++n) d += O_diag[n * slm + lm] * cv[kRowE + n];
            const double inv = (d != 0.0) ? 1.0 / d : 0.0;
            dinv[static_cast<size_t>(v) * c->aslm + lm] = inv;
            dinv32[static_cast<size_t>(v) * c->aslm32 + lm] = static_cast<float>(inv);
        }
    }
    // moments: omega_i[lm][0] and its j (MeshData.cpp:105-110)
    std::vector<double> mom_w(3 * slm);
    std::vector<uint32_t> mom_pos(3 * slm);
    for (int i = 0; i < 3; ++i)
        for (tr_idx lm = 0; lm < slm; ++lm) {
            mom_w[i * slm + lm] = a->omega[(static_cast<size_t>(i) * slm + lm) * slm];
            mom_pos[i * slm + lm] = a->omega_pos[(static_cast<size_t>(i) * slm + lm) * slm];
        }
    // per-tet data for the right-hand side and the flux
    std::vector<uint32_t> tetp(4ULL * nT);
    std::vector<double> tets(12ULL * nT), tetkv(nT), tetq(nT);
    for (tr_idx t = 0; t < nT; ++t) {
        const tr_tetrahedron &T = m->mesh[t];
        for (int k = 0; k < 4; ++k) tetp[4ULL * t + k] = T.p[k];
        for (int k = 0; k < 4; ++k)
            for (int d = 0; d < 3; ++d) tets[12ULL * t + 3 * k + d] = T.s[k][d];
        tetkv[t] = T.kappa_volume;
        tetq[t] = T.kappa_volume * T.I_p;
    }

    // ---------------------------------------------------- upload
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
        return e == cudaSuccess;
    };
    DeviceOp<double> &o64 = c->op64;
    DeviceOp<float> &o32 = c->op32;
    o64.aslm = c->aslm;
    o32.aslm = c->aslm32;
    // the fastest solves measured on B200: FP64 DMMA edge sums, FP32 FMA edge
    // sums (split-TF32 tensor-core sums drop the lo*lo product, which costs
    // the mixed solve more inner iterations than the faster operator saves)
    o64.kind = TR_OPERATOR_TENSOR;
    o32.kind = TR_OPERATOR_SIMT;
    ok(upload(c, &o64.row, row.data(), row.size() * 4));
    ok(upload(c, &o64.col, col.data(), col.size() * 4));
    o64.cls = o32.cls = cls;
    ok(upload_runs(c, rs64, slm, o64.rs));
    ok(upload_runs(c, rt64, slm, o64.rt));
    ok(upload_runs(c, rs32, slm, o32.rs));
    ok(upload_runs(c, rt32, slm, o32.rt));
    // device records in two halves: rows 0-7 of every edge, then rows 8-15
    std::vector<double> coef_split(coef.size());
    for (size_t e = 0; e < nnz; ++e)
        for (int q = 0; q < kCoefStride; ++q)
            coef_split[(q < kCoefHalf ? e : nnz + e) * kCoefHalf + q % kCoefHalf] = coef[e * kCoefStride + q];
    o64.nnz = o32.nnz = nnz;
    ok(upload(c, &o64.coef, coef_split.data(), coef_split.size() * 8));
    // operator copy of O_n, rows lms padded to the lane stride cls
    std::vector<double> Opad(3 * static_cast<size_t>(slm) * cls, 0.0);
    for (int n = 0; n < 3; ++n)
        for (tr_idx lms = 0; lms < slm; ++lms)
            for (tr_idx lm = 0; lm < slm; ++lm)
                Opad[(static_cast<size_t>(n) * slm + lms) * cls + lm] = On[n][static_cast<size_t>(lms) * slm + lm];
    ok(upload(c, &o64.O, Opad.data(), Opad.size() * 8));
    ok(upload(c, &o64.ang_diag, ang_diag.data(), ang_diag.size() * 8));
    ok(upload(c, &o64.O_diag, O_diag.data(), O_diag.size() * 8));
    ok(upload(c, &o64.dinv, dinv.data(), dinv.size() * 8));
    ok(upload(c, &o64.bmask, bmask.data(), bmask.size()));
    o32.row = o64.row;
    o32.col = o64.col;
    o32.bmask = o64.bmask;
    {
        auto c32 = to_type<float>(coef_split);
        ok(upload(c, &o32.coef, c32.data(), c32.size() * 4));
        auto O32 = to_type<float>(Opad);
        ok(upload(c, &o32.O, O32.data(), O32.size() * 4));
        auto d32 = to_type<float>(ang_diag);
        ok(upload(c, &o32.ang_diag, d32.data(), d32.size() * 4));
        auto od32 = to_type<float>(O_diag);
        ok(upload(c, &o32.O_diag, od32.data(), od32.size() * 4));
        ok(upload(c, &o32.dinv, dinv32.data(), dinv32.size() * 4));
    }
    ok(upload(c, &c->vt_start, m->tetstart, (nP + 1) * 4ULL));
    ok(upload(c, &c->vt_tet, m->tetidx, std::max<size_t>(m->tetstart[nP], 1) * 4ULL));
    ok(upload(c, &c->tet_q, tetq.data(), tetq.size() * 8));
    if (any_inflow) ok(upload(c, &c->inflow, inflow.data(), inflow.size() * 8));
    ok(upload(c, &c->O64, O.data(), O.size() * 8));
    ok(upload(c, reinterpret_cast<uint32_t **>(&c->tet_p), tetp.data(), tetp.size() * 4));
    ok(upload(c, &c->tet_s, tets.data(), tets.size() * 8));
    ok(upload(c, &c->tet_kv, tetkv.data(), tetkv.size() * 8));
    ok(upload(c, &c->mom_w, mom_w.data(), mom_w.size() * 8));
    ok(upload(c, &c->mom_pos, mom_pos.data(), mom_pos.size() * 4));
    ok(upload(c, &c->partials, nullptr, 4 * kMaxGrid * sizeof(double)));
    ok(upload(c, &c->counters, nullptr, 16 * sizeof(unsigned int)));
    ok(upload(c, &c->bar, nullptr, 2 * sizeof(unsigned int)));
    ok(upload(c, &c->bar_err, nullptr, sizeof(int)));
    ok(upload(c, &c->red_out, nullptr, 16 * sizeof(double)));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&c->host_pinned), 16 * sizeof(double));
    if (e == cudaSuccess) e = cudaStreamCreate(&c->own_stream);
    if (e == cudaSuccess) e = operator_init_attributes();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bail(std::string("device setup failed: ") + cudaGetErrorString(e),
                    e == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA);
    }
    // grids: whole waves of resident 256-thread blocks, capped by the work
    const size_t n64 = static_cast<size_t>(nP) * c->aslm;
    // (up to 4 resident blocks per SM; the grid-reduction tickets scale with it)
    const size_t waves = static_cast<size_t>(c->num_sms) * 4;
    auto cap = [&](size_t need) { return static_cast<int>(std::max<size_t>(1, std::min(waves, need))); };
    c->grid_vec = cap((n64 + kBlock - 1) / kBlock);
    c->grid_vec64 = cap((n64 / 2 + kBlock - 1) / kBlock);
    c->grid_vec32 = cap((static_cast<size_t>(nP) * c->aslm32 / 4 + kBlock - 1) / kBlock);
    const uint32_t G = c->aslm <= 8 ? 8 : c->aslm <= 16 ? 16 : 32;
    const size_t groups_per_block = kBlock / G;
    c->grid_op = cap((nP + groups_per_block - 1) / groups_per_block);
    *out = c;
    return TR_OK;
}

}  // namespace transfer
