// TEST INFRASTRUCTURE ONLY: see mesh.h.
#ifndef TR_STUB_TRI_FACE_H
#define TR_STUB_TRI_FACE_H
#include "mesh.h"

struct TriFace : public Face {
    Vertex *p[3];
};

#endif
