// TEST INFRASTRUCTURE ONLY: implementation of the meshProcessor stand-in
// declared in meshProcessor/mesh.h.
//
// Input format (plain text, written by tests/refrun.py):
//   tmesh 1
//   <nP>
//   x y z                       (nP lines)
//   <nT>
//   p0 p1 p2 p3 region          (nT lines, region >= 1)
#include "meshProcessor/mesh.h"
#include "meshProcessor/tetrahedron.h"
#include "meshProcessor/tri_face.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <string>

static Vector sub(const Vector &a, const Vector &b) { return Vector(a.x - b.x, a.y - b.y, a.z - b.z); }
static Vector cross(const Vector &a, const Vector &b) {
    return Vector(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static double dot(const Vector &a, const Vector &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Area-weighted normal of triangle (a,b,c) oriented away from point o.
static void face_normal(const Vector &a, const Vector &b, const Vector &c, const Vector &o,
                        Vector &unit, double &area) {
    Vector n = cross(sub(b, a), sub(c, a));
    n.scale(0.5);
    if (dot(n, sub(a, o)) < 0) n.scale(-1.0);
    area = n.norm();
    unit = n;
    unit.scale(1.0 / area);
}

Mesh::Mesh(std::ostream &log, const char *filename) : nVert(0), nElems(0), nFaces(0), nBndFaces(0), ok_(false) {
    std::ifstream in(filename);
    std::string magic;
    int version = 0;
    if (!(in >> magic >> version) || magic != "tmesh") {
        log << "stub Mesh: cannot read " << filename << "\n";
        return;
    }
    in >> nVert;
    for (int i = 0; i < nVert; i++) {
        Vertex *v = new Vertex();
        v->index = i;
        in >> v->r.x >> v->r.y >> v->r.z;
        vertices.push_back(v);
    }
    in >> nElems;
    std::vector<int> cnt;
    std::map<std::vector<int>, int> owners;
    for (int t = 0; t < nElems; t++) {
        Tetrahedron *T = new Tetrahedron();
        int q[4], reg;
        in >> q[0] >> q[1] >> q[2] >> q[3] >> reg;
        T->index = t;
        T->region = reg;
        for (int k = 0; k < 4; k++) T->p[k] = vertices.at(q[k]);
        Vector e1 = sub(T->p[1]->r, T->p[0]->r), e2 = sub(T->p[2]->r, T->p[0]->r), e3 = sub(T->p[3]->r, T->p[0]->r);
        T->volume = std::fabs(dot(e1, cross(e2, e3))) / 6.0;
        elements.push_back(T);
        for (int k = 0; k < 4; k++) T->p[k]->elems.push_back(std::make_pair((Element *)T, k));
        for (int j = 0; j < 4; j++) {
            TriFace *F = new TriFace();
            int c = 0;
            for (int k = 0; k < 4; k++)
                if (k != j) F->p[c++] = T->p[k];
            Vector unit;
            double area;
            face_normal(F->p[0]->r, F->p[1]->r, F->p[2]->r, T->p[j]->r, unit, area);
            unit.scale(-1.0);            // inward for the tet's own face
            F->normal = unit;
            F->surface = area;
            F->bnd_index = -1;
            T->f[j] = F;
            faces.push_back(F);
            std::vector<int> key;
            for (int k = 0; k < 3; k++) key.push_back(F->p[k]->index);
            std::sort(key.begin(), key.end());
            owners[key]++;
        }
    }
    // boundary faces: keys seen once, in (tet, local face) order
    int nb = 0;
    for (int t = 0; t < nElems; t++) {
        Tetrahedron *T = (Tetrahedron *)elements[t];
        for (int j = 0; j < 4; j++) {
            TriFace *F = (TriFace *)T->f[j];
            std::vector<int> key;
            for (int k = 0; k < 3; k++) key.push_back(F->p[k]->index);
            std::sort(key.begin(), key.end());
            if (owners[key] != 1) continue;
            TriFace *B = new TriFace();
            for (int k = 0; k < 3; k++) B->p[k] = F->p[k];
            B->normal = F->normal;
            B->normal.scale(-1.0);       // outward
            B->surface = F->surface;
            B->bnd_index = nb++;
            faces.push_back(B);
            for (int k = 0; k < 3; k++) B->p[k]->bnds.push_back(std::make_pair((Face *)B, k));
        }
    }
    nBndFaces = nb;
    nFaces = (int)faces.size();
    ok_ = true;
}

Mesh::~Mesh() {
    for (size_t i = 0; i < vertices.size(); i++) delete vertices[i];
    for (size_t i = 0; i < elements.size(); i++) delete elements[i];
    for (size_t i = 0; i < faces.size(); i++) delete faces[i];
}

bool Mesh::check(std::ostream &log) {
    if (!ok_) return false;
    for (int t = 0; t < nElems; t++)
        if (!(((Tetrahedron *)elements[t])->volume > 0)) {
            log << "stub Mesh: degenerate tet " << t << "\n";
            return false;
        }
    return true;
}

void Mesh::saveVtk(std::ostream &log, const char *filename, int realsize, const char *cellfmt,
                   const char *pointfmt, ...) {
    FILE *out = std::fopen(filename, "w");
    if (!out) {
        log << "stub Mesh: cannot write " << filename << "\n";
        return;
    }
    va_list ap;
    va_start(ap, pointfmt);
    const char *fmts[2] = {cellfmt, pointfmt};
    int counts[2] = {nElems, nVert};
    const char *kinds[2] = {"cell", "point"};
    for (int s = 0; s < 2; s++) {
        const char *p = fmts[s];
        while (*p) {
            std::string name;
            while (*p && *p != '%') name += *p++;
            if (!*p) break;
            char ty = *++p;
            ++p;
            int ncomp = ty == 's' ? 1 : ty == 'v' ? 3 : ty == 't' ? 6 : 0;
            std::fprintf(out, "%s %s %d %d\n", kinds[s], name.c_str(), ncomp, counts[s]);
            for (int c = 0; c < ncomp; c++) {
                void *arr = va_arg(ap, void *);
                for (int i = 0; i < counts[s]; i++) {
                    double v = realsize == 8 ? ((double *)arr)[i] : (double)((float *)arr)[i];
                    std::fprintf(out, "%.17g\n", v);
                }
            }
        }
    }
    va_end(ap);
    std::fclose(out);
}
