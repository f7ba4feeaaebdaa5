// ref_sdf.cpp -- TEST INFRASTRUCTURE ONLY.
//
// KamiSimulator's body SDF bake compiled from the reference sources in place (oracle/ref/Makefile)
// into oracle/_ref/libkami_ref_cpu.so, CPU only: Kami::SDF (utilities/Geometry.cpp:5-35), which
// builds Discregrid's TriangleMeshDistance and a CubicLagrangeDiscreteGrid of it, and the per-node
// loop of PNMesh::StoreSDFQueries (PNMesh.cpp:109-173), restated here because PNMesh.cpp needs the
// rest of the application.  Tests use it to pin the CPU oracle and the GPU bake.
#include <array>
#include <cstdint>
#include <vector>

#include "utilities/Geometry.h"

extern "C" {

// Discregrid's exact signed distance (TriangleMeshDistance::signed_distance) at np points.
int ref_sdf_signed_distance(int32_t nv, const float* verts, int32_t nt, const int32_t* tris, int64_t np,
                            const double* pts, double* out) {
    std::vector<Eigen::Vector3d> pos(nv);
    std::vector<std::array<unsigned int, 3>> tri(nt);
    for (int32_t i = 0; i < nv; i++) pos[i] = Eigen::Vector3d(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    for (int32_t t = 0; t < nt; t++) tri[t] = {(unsigned)tris[3 * t], (unsigned)tris[3 * t + 1], (unsigned)tris[3 * t + 2]};
    Discregrid::TriangleMesh mesh(pos, tri);
    Discregrid::TriangleMeshDistance md(mesh);
    for (int64_t i = 0; i < np; i++) out[i] = md.signed_distance({pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}).distance;
    return 0;
}

// Kami::SDF::Init at resolution dims, then StoreSDFQueries' loop over the nodes of the grid
// [gmin, gmax] (the mesh's bounding box there): phi and grad, x fastest.
int ref_sdf_bake(int32_t nv, const float* verts, int32_t nt, const int32_t* tris, const int32_t* dims, const float* gmin,
                 const float* gmax, float* phi, float* grad) {
    unq_ptr<glm::vec3[]> vp(new glm::vec3[nv]);
    unq_ptr<glm::uvec3[]> ti(new glm::uvec3[nt]);
    for (int32_t i = 0; i < nv; i++) vp[i] = glm::vec3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    for (int32_t t = 0; t < nt; t++) ti[t] = glm::uvec3(tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]);
    Kami::SDF sdf;
    const glm::uvec3 dim(dims[0], dims[1], dims[2]);
    sdf.Init(vp, ti, (uint32_t)nv, (uint32_t)nt, dim);
    const glm::vec3 lo(gmin[0], gmin[1], gmin[2]), hi(gmax[0], gmax[1], gmax[2]);
    const glm::vec3 ds((hi.x - lo.x) / dim.x, (hi.y - lo.y) / dim.y, (hi.z - lo.z) / dim.z);
    const int total = (int)(dim.x * dim.y * dim.z);
    for (int i = 0; i < total; i++) {
        glm::vec3 pos = lo;
        const int ix = i % dim.x, iy = (i / dim.x) % dim.y, iz = i / (dim.x * dim.y);
        pos += ds.x * (ix) * glm::vec3(1.f, 0.f, 0.f);
        pos += ds.y * (iy) * glm::vec3(0.f, 1.f, 0.f);
        pos += ds.z * (iz) * glm::vec3(0.f, 0.f, 1.f);
        glm::vec3 cp, n;
        float dist;
        if (sdf.CollisionTest(pos, cp, n, dist)) {
            phi[i] = dist;
        } else {
            phi[i] = (float)sdf.Distance(pos);
            glm::vec3 centre = (hi + lo) / 2.f;
            glm::vec3 to = centre - pos;
            float l = glm::length(to);
            n = glm::vec3(-to.x / l, -to.y / l, -to.z / l);
        }
        grad[3 * i] = n.x;
        grad[3 * i + 1] = n.y;
        grad[3 * i + 2] = n.z;
    }
    return 0;
}

}  // extern "C"
