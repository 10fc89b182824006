// TEST INFRASTRUCTURE ONLY.
//
// Minimal stand-in for the `meshProcessor` submodule of the reference
// (.gitmodules:1-3; absent from the reference tree and pinned to no
// version).  It provides exactly the members the reference's MeshData.cpp
// (lines 9-94) and main.cpp (lines 192-216) use, so that those reference
// sources compile unmodified for the oracle/_ref builds.
//
// Mesh(std::ostream&, const char *file) reads the plain-text tetrahedral
// mesh that tests write (see mesh.cpp for the format); it computes faces,
// areas and volumes itself.  Tet face j is the face opposite local vertex j
// and its `normal` points INTO the tetrahedron, so MeshData.cpp's
// s = -normal * surface is the outward area normal of that face.  Boundary
// faces carry the outward normal.
#ifndef TR_STUB_MESH_H
#define TR_STUB_MESH_H

#include <cmath>
#include <cstdarg>
#include <ostream>
#include <utility>
#include <vector>

struct Vector {
    double x, y, z;
    Vector() : x(0), y(0), z(0) {}
    Vector(double a, double b, double c) : x(a), y(b), z(c) {}
    void scale(double s) { x *= s; y *= s; z *= s; }
    void add(const Vector &o) { x += o.x; y += o.y; z += o.z; }
    double norm() const { return std::sqrt(x * x + y * y + z * z); }
};

struct Element;
struct Face;

struct Vertex {
    int index;
    Vector r;
    std::vector<std::pair<Element *, int> > elems;
    std::vector<std::pair<Face *, int> > bnds;
};

struct Element {
    int index;
    int region;
    virtual ~Element() {}
};

struct Face {
    int bnd_index;          // index among boundary faces, -1 for interior
    Vector normal;          // unit normal
    double surface;         // area
    virtual ~Face() {}
};

class Mesh {
public:
    int nVert, nElems, nFaces, nBndFaces;
    std::vector<Vertex *> vertices;
    std::vector<Element *> elements;
    std::vector<Face *> faces;
    Mesh(std::ostream &log, const char *filename);
    ~Mesh();
    bool check(std::ostream &log);
    // Writes the named fields as plain text (one "name count" header line
    // followed by the values); replaces the VTK writer used at main.cpp:209.
    void saveVtk(std::ostream &log, const char *filename, int realsize,
                 const char *cellfmt, const char *pointfmt, ...);
private:
    bool ok_;
};

#endif
