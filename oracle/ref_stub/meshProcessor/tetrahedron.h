// TEST INFRASTRUCTURE ONLY: see mesh.h.
#ifndef TR_STUB_TETRAHEDRON_H
#define TR_STUB_TETRAHEDRON_H
#include "mesh.h"

struct Tetrahedron : public Element {
    Vertex *p[4];
    Face *f[4];       // f[j] is opposite p[j]; normal points inward
    double volume;
};

#endif
