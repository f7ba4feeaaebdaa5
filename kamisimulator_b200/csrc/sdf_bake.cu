// sdf_bake.cu -- the body SDF grid baked from a closed triangle mesh on the GPU.
//
// KamiSimulator bakes the head's SDF on the CPU: Discregrid's TriangleMeshDistance resampled by a
// CubicLagrangeDiscreteGrid (utilities/Geometry.cpp:5-35), then sampled at the grid nodes by
// PNMesh::StoreSDFQueries (PNMesh.cpp:109-173).  Here every node gets the exact signed distance
// to the mesh, the function that grid approximates:
//   * nearest point: every triangle is tested (tiles of triangles staged in shared memory, one
//     node per thread); closest point on a triangle and its Voronoi feature (vertex, edge or
//     face) after Ericson, Real-Time Collision Detection (2005), 5.1.5;
//   * sign: the angle-weighted pseudonormal of that feature (Baerentzen and Aanaes, "Signed
//     distance computation using the angle weighted pseudonormal", IEEE TVCG 11(3), 2005), the
//     sign rule of TriangleMeshDistance::signed_distance;
//   * gradient: inside (distance < 0) the unit gradient of the distance, (nearest - x) / |d|;
//     elsewhere the unit direction from the grid centre, as StoreSDFQueries sets it (zero at a
//     node exactly at the centre, where the reference divides 0 by 0).
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "kami_vbd.h"
#include "vbd_common.cuh"
#include "vbd_host.h"

namespace kami {
namespace {

constexpr int BAKE_THREADS = 256;
constexpr int BAKE_TILE = 256;  // triangles per shared-memory tile (9 floats each)

// Closest point on triangle (a, b, c) to p and its feature: 0, 1, 2 = vertex a, b, c; 3, 4, 5 =
// edge ab, bc, ca; 6 = face.  Returns the squared distance.
__device__ __forceinline__ float closest_on_triangle(float3 p, float3 a, float3 b, float3 c, float3& cp, int& f) {
    const float3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) {
        cp = a;
        f = 0;
    } else {
        const float3 bp = p - b;
        const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
        if (d3 >= 0.f && d4 <= d3) {
            cp = b;
            f = 1;
        } else {
            const float vc = d1 * d4 - d3 * d2;
            if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
                cp = a + (d1 / (d1 - d3)) * ab;
                f = 3;
            } else {
                const float3 cpp = p - c;
                const float d5 = dot3(ab, cpp), d6 = dot3(ac, cpp);
                if (d6 >= 0.f && d5 <= d6) {
                    cp = c;
                    f = 2;
                } else {
                    const float vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
                        cp = a + (d2 / (d2 - d6)) * ac;
                        f = 5;
                    } else {
                        const float va = d3 * d6 - d5 * d4;
                        if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
                            cp = b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
                            f = 4;
                        } else {
                            const float den = 1.f / (va + vb + vc);
                            cp = a + (vb * den) * ab + (vc * den) * ac;
                            f = 6;
                        }
                    }
                }
            }
        }
    }
    const float3 d = p - cp;
    return dot3(d, d);
}

__global__ void __launch_bounds__(BAKE_THREADS) sdf_bake_kernel(const float* __restrict__ tv, int nt,
                                                                const int32_t* __restrict__ tris,
                                                                const float4* __restrict__ face_n,
                                                                const float4* __restrict__ edge_n,
                                                                const float4* __restrict__ vert_n, int nx, int ny, int nz,
                                                                float3 lo, float3 ds, float3 centre,
                                                                float* __restrict__ phi, float* __restrict__ grad) {
    __shared__ float sv[BAKE_TILE * 9];
    const int64_t total = (int64_t)nx * ny * nz;
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = node < total;
    const int64_t i = node % nx, j = (node / nx) % ny, k = node / ((int64_t)nx * ny);
    const float3 x = f3(lo.x + ds.x * (float)i, lo.y + ds.y * (float)j, lo.z + ds.z * (float)k);
    float best = INFINITY;
    int bt = -1, bf = 0;
    float3 bcp = x;
    for (int base = 0; base < nt; base += BAKE_TILE) {
        const int cnt = min(BAKE_TILE, nt - base);
        __syncthreads();
        for (int q = threadIdx.x; q < cnt * 9; q += blockDim.x) sv[q] = tv[(int64_t)base * 9 + q];
        __syncthreads();
        if (active) {
            for (int t = 0; t < cnt; t++) {
                const float* T = sv + 9 * t;
                float3 cp;
                int f;
                const float d2 = closest_on_triangle(x, f3(T[0], T[1], T[2]), f3(T[3], T[4], T[5]), f3(T[6], T[7], T[8]), cp, f);
                if (d2 < best) {
                    best = d2;
                    bt = base + t;
                    bf = f;
                    bcp = cp;
                }
            }
        }
    }
    if (!active) return;
    if (bt < 0) {  // no finite distance (the host rejects non-finite vertices, so this is a guard)
        phi[node] = NAN;
        grad[3 * node] = grad[3 * node + 1] = grad[3 * node + 2] = 0.f;
        return;
    }
    const float dist = sqrtf(best);
    float4 pn;
    if (bf < 3)
        pn = vert_n[tris[3 * bt + bf]];
    else if (bf < 6)
        pn = edge_n[3 * bt + (bf - 3)];
    else
        pn = face_n[bt];
    const float3 u = x - bcp;
    const float s = (u.x * pn.x + u.y * pn.y + u.z * pn.z) >= 0.f ? 1.f : -1.f;
    const float d = s * dist;
    phi[node] = d;
    float3 g;
    if (d < 0.f) {
        g = (bcp - x) * (1.f / dist);
    } else {
        const float3 r = x - centre;
        const float l = sqrtf(dot3(r, r));
        g = l > 0.f ? r * (1.f / l) : f3(0.f, 0.f, 0.f);
    }
    grad[3 * node] = g.x;
    grad[3 * node + 1] = g.y;
    grad[3 * node + 2] = g.z;
}

struct D3 {
    double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 mul(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 crossd(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double lend(D3 a) { return std::sqrt(dotd(a, a)); }

kami_status bake_fail(kami_status st, const std::string& msg) {
    set_last_error(msg.c_str());
    return st;
}

}  // namespace
}  // namespace kami

using namespace kami;

extern "C" kami_status kami_sdf_bake(const float* vertices, int32_t num_vertices, const int32_t* triangles,
                                     int32_t num_triangles, const int32_t dims[3], const float grid_min[3],
                                     const float grid_max[3], float* phi, float* grad, int32_t memory, int32_t device) {
    if (!vertices || !triangles || !dims || !grid_min || !grid_max || !phi || !grad || num_vertices < 3 || num_triangles < 1)
        return bake_fail(KAMI_ERR_INVALID_ARGUMENT, "need a mesh of >= 3 vertices and >= 1 triangle, dims, bounds and outputs");
    if (memory != KAMI_MEMORY_HOST && memory != KAMI_MEMORY_DEVICE) return bake_fail(KAMI_ERR_INVALID_ARGUMENT, "bad memory kind");
    for (int a = 0; a < 3; a++) {
        if (dims[a] <= 0) return bake_fail(KAMI_ERR_INVALID_ARGUMENT, "dims must be > 0");
        if (!(grid_max[a] > grid_min[a])) return bake_fail(KAMI_ERR_INVALID_ARGUMENT, "grid_max must exceed grid_min");
    }
    const int64_t total = (int64_t)dims[0] * dims[1] * dims[2];
    for (int64_t q = 0; q < 3LL * num_vertices; q++)
        if (!std::isfinite(vertices[q])) return bake_fail(KAMI_ERR_INVALID_ARGUMENT, "non-finite mesh vertex");
    // pseudonormals, in double: faces; vertices weighted by the incident angles; edges the sum of
    // their faces' normals (TriangleMeshDistance.h:364-421 builds the same three sets)
    const int32_t nv = num_vertices, nt = num_triangles;
    auto vert = [&](int32_t i) { return D3{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]}; };
    std::vector<D3> fn(nt), vn(nv, D3{0, 0, 0});
    std::map<std::pair<int32_t, int32_t>, D3> edge_sum;
    for (int32_t t = 0; t < nt; t++) {
        const int32_t* T = triangles + 3 * t;
        for (int q = 0; q < 3; q++)
            if (T[q] < 0 || T[q] >= nv) return bake_fail(KAMI_ERR_INVALID_ARGUMENT, "triangle index out of range");
        const D3 p[3] = {vert(T[0]), vert(T[1]), vert(T[2])};
        D3 n = crossd(sub(p[1], p[0]), sub(p[2], p[0]));
        const double ln = lend(n);
        if (!(ln > 0) || !std::isfinite(ln))
            return bake_fail(KAMI_ERR_GEOMETRY, "triangle " + std::to_string(t) + " has zero area");
        n = mul(1.0 / ln, n);
        fn[t] = n;
        for (int q = 0; q < 3; q++) {
            const D3 e1 = sub(p[(q + 1) % 3], p[q]), e2 = sub(p[(q + 2) % 3], p[q]);
            const double c = dotd(e1, e2) / (lend(e1) * lend(e2));
            vn[T[q]] = add(vn[T[q]], mul(std::acos(std::max(-1.0, std::min(1.0, c))), n));
            const int32_t i0 = T[q], i1 = T[(q + 1) % 3];
            auto key = std::make_pair(std::min(i0, i1), std::max(i0, i1));
            auto it = edge_sum.find(key);
            if (it == edge_sum.end())
                edge_sum[key] = n;
            else
                it->second = add(it->second, n);
        }
    }
    std::vector<float> tv(9 * (size_t)nt);
    std::vector<float4> hf(nt), he(3 * (size_t)nt), hv(nv);
    for (int32_t t = 0; t < nt; t++) {
        for (int q = 0; q < 9; q++) tv[9 * t + q] = vertices[3 * triangles[3 * t + q / 3] + q % 3];
        hf[t] = make_float4((float)fn[t].x, (float)fn[t].y, (float)fn[t].z, 0.f);
        for (int q = 0; q < 3; q++) {
            const int32_t i0 = triangles[3 * t + q], i1 = triangles[3 * t + (q + 1) % 3];
            D3 e = edge_sum[std::make_pair(std::min(i0, i1), std::max(i0, i1))];
            const double le = lend(e);
            e = le > 0 ? mul(1.0 / le, e) : fn[t];
            he[3 * t + q] = make_float4((float)e.x, (float)e.y, (float)e.z, 0.f);
        }
    }
    for (int32_t i = 0; i < nv; i++) {
        const double l = lend(vn[i]);
        const D3 n = l > 0 ? mul(1.0 / l, vn[i]) : D3{0, 0, 0};
        hv[i] = make_float4((float)n.x, (float)n.y, (float)n.z, 0.f);
    }

    if (device >= 0) {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return bake_fail(KAMI_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    float* d_tv = nullptr;
    int32_t* d_tris = nullptr;
    float4 *d_f = nullptr, *d_e = nullptr, *d_v = nullptr;
    float *d_phi = nullptr, *d_grad = nullptr;
    cudaError_t e = cudaMalloc(&d_tv, sizeof(float) * tv.size());
    if (e == cudaSuccess) e = cudaMalloc(&d_tris, sizeof(int32_t) * 3 * (size_t)nt);
    if (e == cudaSuccess) e = cudaMalloc(&d_f, sizeof(float4) * hf.size());
    if (e == cudaSuccess) e = cudaMalloc(&d_e, sizeof(float4) * he.size());
    if (e == cudaSuccess) e = cudaMalloc(&d_v, sizeof(float4) * hv.size());
    if (e == cudaSuccess && memory == KAMI_MEMORY_HOST) e = cudaMalloc(&d_phi, sizeof(float) * total);
    if (e == cudaSuccess && memory == KAMI_MEMORY_HOST) e = cudaMalloc(&d_grad, sizeof(float) * 3 * total);
    if (e == cudaSuccess) e = cudaMemcpy(d_tv, tv.data(), sizeof(float) * tv.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_tris, triangles, sizeof(int32_t) * 3 * (size_t)nt, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_f, hf.data(), sizeof(float4) * hf.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_e, he.data(), sizeof(float4) * he.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_v, hv.data(), sizeof(float4) * hv.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        float* out_phi = memory == KAMI_MEMORY_HOST ? d_phi : phi;
        float* out_grad = memory == KAMI_MEMORY_HOST ? d_grad : grad;
        const float3 lo = f3(grid_min[0], grid_min[1], grid_min[2]);
        // node spacing and grid centre as SDFBodyCollisionSolver / StoreSDFQueries compute them
        const float3 ds = f3((grid_max[0] - grid_min[0]) / (1.f * dims[0]), (grid_max[1] - grid_min[1]) / (1.f * dims[1]),
                             (grid_max[2] - grid_min[2]) / (1.f * dims[2]));
        const float3 centre = f3((grid_max[0] + grid_min[0]) / 2.f, (grid_max[1] + grid_min[1]) / 2.f,
                                 (grid_max[2] + grid_min[2]) / 2.f);
        const unsigned blocks = (unsigned)((total + BAKE_THREADS - 1) / BAKE_THREADS);
        sdf_bake_kernel<<<blocks, BAKE_THREADS>>>(d_tv, nt, d_tris, d_f, d_e, d_v, dims[0], dims[1], dims[2], lo, ds, centre,
                                                  out_phi, out_grad);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess && memory == KAMI_MEMORY_HOST) {
            e = cudaMemcpy(phi, d_phi, sizeof(float) * total, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(grad, d_grad, sizeof(float) * 3 * total, cudaMemcpyDeviceToHost);
        }
    }
    void* bufs[] = {d_tv, d_tris, d_f, d_e, d_v, d_phi, d_grad};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (e != cudaSuccess)
        return bake_fail(e == cudaErrorMemoryAllocation ? KAMI_ERR_OUT_OF_MEMORY : KAMI_ERR_CUDA,
                         std::string("SDF bake: ") + cudaGetErrorString(e));
    return KAMI_OK;
}
