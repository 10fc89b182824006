// TEST INFRASTRUCTURE ONLY.
//
// A CPU implementation of the reference's `struct CudaContext`
// (CudaContext.h:9-50) on top of the FP64 oracle kernels.  Linked with the
// reference's own host sources (main.cpp, MeshData.cpp, DeviceMeshData.cpp,
// DeviceAngularData.cpp, Eigenvalue.cpp, ...) it runs the reference's driver
// logic -- CG, invprec, eigest, ComputeMoments/ComputeFlux -- on the CPU,
// with "device" memory being host memory.  Built with -DUSE_DOUBLE only.
#include "CudaContext.h"
#include "common.cuh"
#include "transfer_oracle.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

static_assert(sizeof(REAL) == 8, "the CPU context is FP64 only");
static_assert(sizeof(tetrahedron) == sizeof(or_tet), "tetrahedron layout");
static_assert(sizeof(face) == sizeof(or_face), "face layout");

static or_mesh view_mesh(const DeviceMeshData *m) {
    or_mesh o;
    std::memset(&o, 0, sizeof(o));
    o.nP = m->nP;
    o.tetstart = m->tetstart;
    o.tetidx = m->tetidx;
    o.tetpos = m->tetpos;
    o.mesh = reinterpret_cast<const or_tet *>(m->mesh);
    o.facestart = m->facestart;
    o.faceidx = m->faceidx;
    o.facepos = m->facepos;
    o.bnd = reinterpret_cast<const or_face *>(m->bnd);
    return o;
}
static or_ang view_ang(const DeviceAngularData *a) {
    or_ang o;
    o.slm = a->slm;
    o.aslm = a->aslm;
    o.omega = a->omega;
    o.omega_pos = a->omega_pos;
    o.Ox = a->Ox;
    o.Oy = a->Oy;
    o.Oz = a->Oz;
    return o;
}

CudaContext::CudaContext(const int dev, const MeshData &dmd, const AngularData &dad) {
    (void)dev;
    std::printf("CPU oracle context\n");
    meshdata = new DeviceMeshData(this, dmd);
    angdata = new DeviceAngularData(this, dad);
    red = (REAL *)deviceAlloc(sizeof(REAL));
}
CudaContext::~CudaContext() {
    deviceFree(red);
    delete meshdata;
    delete angdata;
}
void *CudaContext::deviceAlloc(size_t size) const { return std::calloc(size ? size : 1, 1); }
idx CudaContext::N() const { return meshdata->nP * angdata->aslm; }
REAL *CudaContext::allocVector() const { return (REAL *)deviceAlloc(N() * sizeof(REAL)); }
void CudaContext::deviceFree(void *mem) const { std::free(mem); }
void CudaContext::copyToDev(void *dst, void *src, size_t sz) const { std::memcpy(dst, src, sz); }
void CudaContext::copyToHost(void *dst, void *src, size_t sz) const { std::memcpy(dst, src, sz); }
REAL *CudaContext::getHostSmall(void *src) const {
    idx nP = meshdata->nP, slm = angdata->slm, aslm = angdata->aslm;
    REAL *p = (REAL *)std::malloc(sizeof(REAL) * nP * slm);
    const REAL *q = (const REAL *)src;
    for (idx i = 0; i < nP; i++)
        for (idx j = 0; j < slm; j++) p[i * slm + j] = q[i * aslm + j];
    return p;
}
void CudaContext::computeLhs(REAL *f, REAL *Af) const {
    or_mesh m = view_mesh(meshdata);
    or_ang a = view_ang(angdata);
    oracle_compute_lhs(&m, &a, f, Af);
}
void CudaContext::computeLhsDiag(REAL *f, REAL *Af) const {
    or_mesh m = view_mesh(meshdata);
    or_ang a = view_ang(angdata);
    oracle_compute_lhs_diag(&m, &a, f, Af);
}
void CudaContext::computeRhs(REAL *b) const {
    or_mesh m = view_mesh(meshdata);
    or_ang a = view_ang(angdata);
    oracle_rhs(&m, &a, b);
}
void CudaContext::scale(REAL *x, const REAL wx) const { oracle_scale(N(), x, wx); }
void CudaContext::addProd(REAL *x, const REAL *y, const REAL wy) const { oracle_add_prod(N(), x, y, wy); }
void CudaContext::mulAdd(REAL *x, const REAL wx, const REAL *y) const { oracle_mul_add(N(), x, wx, y); }
void CudaContext::mulAddProd(REAL *x, const REAL wx, const REAL *y, const REAL wy) const {
    oracle_mul_add_prod(N(), x, wx, y, wy);
}
REAL CudaContext::norm(const REAL *x) const {
    return oracle_norm(meshdata->nP, angdata->aslm, angdata->slm, x);
}
REAL CudaContext::dot(const REAL *x, const REAL *y) const {
    return oracle_dot(meshdata->nP, angdata->aslm, angdata->slm, x, y);
}
