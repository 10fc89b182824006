// TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own host code (compiled from the reference sources
// by oracle/Makefile into oracle/_ref/) and writes its outputs as raw
// little-endian binaries, from which tests/golden/make_golden.py builds the
// committed golden fixtures.  Modes:
//   angular  <maxk> <out>           AngularData (AngularData.cpp:9-67)
//   lebedev  <mindegree> <out>      LebedevQuad (LebedevQuad.cpp:6269)
//   hemi     <mindegree> <out>      HemiQuad (HemiQuad.cpp:265)
//   sph      <topow> <out>          Spherical::value on fixed points
//   xe1      <out>                  xE1 (E1.cpp:136-160) on fixed points
//   trieig   <out>                  trieig (Eigenvalue.cpp:5-51), fixed cases
//   config   <cfg> <nreg>           Config (Config.cpp:8-131), printed
//   meshdata <cfg> <out>            MeshData (MeshData.cpp:9-94) + moments/flux
#include "AngularData.h"
#include "Config.h"
#include "HemiQuad.h"
#include "LebedevQuad.h"
#include "MeshData.h"
#include "Spherical.h"
#include "util.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

double trieig(REAL *a, REAL *b, idx N);   // Eigenvalue.cpp:5
double xE1(double x);                      // E1.cpp:136

static FILE *open_out(const char *fn) {
    FILE *f = std::fopen(fn, "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", fn);
        std::exit(2);
    }
    return f;
}
template <class T> static void put(FILE *f, const T *p, size_t n) { std::fwrite(p, sizeof(T), n, f); }
static void put_i(FILE *f, int v) { put(f, &v, 1); }

// deterministic test directions (not on a symmetry axis)
static void points(std::vector<double> &x, std::vector<double> &y, std::vector<double> &z) {
    for (int i = 0; i < 64; i++) {
        double t = std::acos(1.0 - 2.0 * (i + 0.5) / 64.0), p = 2.399963229728653 * i + 0.1;
        x.push_back(std::sin(t) * std::cos(p));
        y.push_back(std::sin(t) * std::sin(p));
        z.push_back(std::cos(t));
    }
}

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: ref_dump <mode> ...\n");
        return 1;
    }
    const char *mode = argv[1];
    if (!std::strcmp(mode, "angular") && argc == 4) {
        int maxk = std::atoi(argv[2]);
        AngularData ad(maxk);
        int n = ad.slm;
        FILE *f = open_out(argv[3]);
        put_i(f, n);
        put(f, ad.omega, 3 * n * n);
        put(f, ad.omega_pos, 3 * n * n);
        put(f, ad.Ox, n * n);
        put(f, ad.Oy, n * n);
        put(f, ad.Oz, n * n);
        std::fclose(f);
        return 0;
    }
    if ((!std::strcmp(mode, "lebedev") || !std::strcmp(mode, "hemi")) && argc == 4) {
        int deg = std::atoi(argv[2]);
        FILE *f = open_out(argv[3]);
        if (mode[0] == 'l') {
            LebedevQuad q(deg);
            put_i(f, q.order);
            put(f, q.x, q.order); put(f, q.y, q.order); put(f, q.z, q.order); put(f, q.w, q.order);
        } else {
            HemiQuad q(deg);
            put_i(f, q.order);
            put(f, q.x, q.order); put(f, q.y, q.order); put(f, q.z, q.order); put(f, q.w, q.order);
        }
        std::fclose(f);
        return 0;
    }
    if (!std::strcmp(mode, "sph") && argc == 4) {
        int L = std::atoi(argv[2]);
        Spherical s(L);
        std::vector<double> x, y, z;
        points(x, y, z);
        FILE *f = open_out(argv[3]);
        put_i(f, L);
        put_i(f, (int)x.size());
        put(f, x.data(), x.size()); put(f, y.data(), y.size()); put(f, z.data(), z.size());
        for (int l = 0; l <= L; l++)
            for (int m = -l; m <= l; m++)
                for (size_t p = 0; p < x.size(); p++) {
                    double v = s.value(l, m, x[p], y[p], z[p]);
                    put(f, &v, 1);
                }
        std::fclose(f);
        return 0;
    }
    if (!std::strcmp(mode, "xe1")) {
        FILE *f = open_out(argv[2]);
        std::vector<double> xs;
        for (int i = 0; i < 200; i++) xs.push_back(0.005 + i * 0.05);
        put_i(f, (int)xs.size());
        put(f, xs.data(), xs.size());
        for (size_t i = 0; i < xs.size(); i++) {
            double v = xE1(xs[i]);
            put(f, &v, 1);
        }
        std::fclose(f);
        return 0;
    }
    if (!std::strcmp(mode, "trieig")) {
        FILE *f = open_out(argv[2]);
        unsigned long long st = 12345;
        int ncase = 40;
        put_i(f, ncase);
        for (int c = 0; c < ncase; c++) {
            int N = 1 + c % 30;
            std::vector<REAL> a(N), b(N);
            for (int i = 0; i < N; i++) {
                st = st * 6364136223846793005ULL + 1442695040888963407ULL;
                a[i] = 1.0 + (double)(st >> 11) * (1.0 / 9007199254740992.0);
                st = st * 6364136223846793005ULL + 1442695040888963407ULL;
                b[i] = 0.5 * (double)(st >> 11) * (1.0 / 9007199254740992.0);
            }
            double lm = trieig(a.data(), b.data(), N);
            put_i(f, N);
            put(f, a.data(), N);
            put(f, b.data(), N);
            put(f, &lm, 1);
        }
        std::fclose(f);
        return 0;
    }
    if (!std::strcmp(mode, "config") && argc == 4) {
        try {
            Config cfg(argv[2]);
            int nreg = std::atoi(argv[3]);
            std::printf("RESULT maxk=%d device=%d dump=%d prec=%d soltype=%d\n", cfg.getMaxK(),
                        cfg.getDevice(), (int)cfg.doDump(), (int)cfg.usePrec(), cfg.solType());
            std::printf("RESULT meshfile=%s\n", cfg.getMeshFilename());
            std::printf("RESULT outfile=%s\n", cfg.getOutFilename());
            for (int r = 1; r <= nreg; r++)
                std::printf("RESULT region=%d kappa=%.17g Ip=%.17g\n", r, cfg.getKappa(r), cfg.getIp(r));
        } catch (int) {
            std::printf("RESULT error\n");
            return 3;
        }
        return 0;
    }
    if (!std::strcmp(mode, "meshdata") && argc == 4) {
        Config cfg(argv[2]);
        MeshData md(cfg);
        if (!md.tetstart) return 4;
        AngularData ad(cfg.getMaxK());
        FILE *f = open_out(argv[3]);
        idx nP = md.nP, nT = md.nT, nF = md.nF;
        idx ntc = md.tetstart[nP], nfc = md.facestart[nP];
        put(f, &nP, 1); put(f, &nT, 1); put(f, &nF, 1);
        put(f, md.tetstart, nP + 1); put(f, md.tetidx, ntc); put(f, md.tetpos, ntc);
        put(f, md.mesh, nT);
        put(f, md.facestart, nP + 1); put(f, md.faceidx, nfc); put(f, md.facepos, nfc);
        put(f, md.bnd, nF);
        // moments / flux of a fixed synthetic intensity field
        idx slm = ad.slm;
        std::vector<REAL *> I(slm);
        for (idx k = 0; k < slm; k++) {
            I[k] = new REAL[nP];
            for (idx i = 0; i < nP; i++) I[k][i] = std::sin(0.37 * i + 1.3 * k) + 0.1 * k;
        }
        std::vector<REAL> U(nP);
        REAL *T[3][3], *W[3];
        for (int i = 0; i < 3; i++) {
            W[i] = new REAL[nT];
            for (int j = 0; j < 3; j++) T[i][j] = new REAL[nP];
        }
        md.ComputeMoments(ad, I.data(), U.data(), T);
        md.ComputeFlux(T, W);
        put(f, &slm, 1);
        for (idx k = 0; k < slm; k++) put(f, I[k], nP);
        put(f, U.data(), nP);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) put(f, T[i][j], nP);
        for (int i = 0; i < 3; i++) put(f, W[i], nT);
        std::fclose(f);
        return 0;
    }
    std::fprintf(stderr, "bad mode/arguments\n");
    return 1;
}
