// vbd_math.cuh -- the per-vertex and per-segment updates of the Stable Cosserat Rods VBD step,
// as device functions on plain values.  Both step forms (sweep and fused) call these, so they
// compute identical arithmetic and differ only in where the operands come from.
#pragma once
#include "vbd_common.cuh"

namespace kami {

// Inertial predict + initial guess of one vertex: initItr, YarnBall/sim/iteration.cu:8-59.
// Returns dx (initial guess of the displacement) and y (= y - x, the inertial target displacement;
// the reference keeps it in d_vels).  Pinned vertices keep dx = h v and y = v.
__device__ __forceinline__ void vbd_predict(float3 x, float3 v, float3 vlast, float inv_mass, const PhysParams& pp,
                                            float h, float last_h, float time, float3& dx, float3& y) {
    float windx = 0.f;
    if (pp.wind_peak != 0.f) {
        // the reference evaluates the cosines in double (2 * M_PI promotes), iteration.cu:22-25
        float wy = x.y > 0.f ? (float)cos(2.0 * 3.14159265358979323846 * (double)(pp.wind_yf * x.y + pp.wind_tf * time)) : 0.f;
        float wz = (float)cos(2.0 * 3.14159265358979323846 * (double)(pp.wind_zf * fabsf(x.z) + pp.wind_tf * time));
        float prod = wy * wz;
        float sg = prod > 0.f ? 1.f : (prod < 0.f ? -1.f : 0.f);
        float pw = powf(prod, pp.wind_sharp) * sg;
        windx = pp.wind_peak * ((0.f < pw) ? pw : 0.f);
    }
    float3 ext = f3(pp.gx + windx, pp.gy, pp.gz) * pp.ext_mult;
    dx = h * v;
    y = v;
    if (inv_mass != 0.f) {
        y = dx + (h * h) * ext;
        float ext2 = dot3(ext, ext);
        if (ext2 > 0.f) {
            float3 acc = (v - vlast) * (1.f / last_h);
            float s = dot3(acc, ext) / ext2;
            s = fminf(fmaxf(s, 0.f), 1.f);
            dx = dx + (h * h * s) * ext;
        }
    }
}

// Constants of one vertex's 3x3 Newton block for one substep.  cosseratItr builds
// H = hess3(m/h^2) + sum_segments d (1 + damping) I, where hess3(float) fills all six packed
// entries (KittenEngine SymMat.h:16-18, cosserat.cu:117), i.e. H = a * ones(3,3) + s * I with
// a = 1 / (invMass h^2).  Its inverse is  delta = (f - m 1) / s + m / (s + 3a) 1,  m = mean(f),
// so the block solve needs only the two reciprocals kept here.
struct BlockConst {
    float a;       // 1 / (invMass h^2), 0 for pinned vertices
    float inv_s;   // 1 / s
    float inv_s3a; // 1 / (s + 3a)
};

__device__ __forceinline__ BlockConst vbd_block_const(float inv_mass, uint32_t fl, float dd_next, float dd_prev, float h,
                                                      float damp) {
    BlockConst b;
    if (inv_mass == 0.f) {
        b.a = 0.f;
        b.inv_s = 0.f;
        b.inv_s3a = 0.f;
        return b;
    }
    b.a = 1.f / (inv_mass * h * h);
    float s = 0.f;
    if (fl & F_HAS_NEXT) s += dd_next * (1.f + damp);
    if (fl & F_HAS_PREV) s += dd_prev * (1.f + damp);
    b.inv_s = 1.f / s;
    b.inv_s3a = 1.f / (s + 3.f * b.a);
    return b;
}

// vbd_block_const for a vertex tied by a connection spring of stiffness k_tie: k_tie (1 + damp) on
// the diagonal, added before the segments' terms as cosseratItr adds it (cosserat.cu:130).
__device__ __forceinline__ BlockConst vbd_block_const_tied(float inv_mass, uint32_t fl, float dd_next, float dd_prev,
                                                           float h, float damp, float k_tie) {
    BlockConst b;
    b.a = 1.f / (inv_mass * h * h);
    float s = k_tie * (1.f + damp);
    if (fl & F_HAS_NEXT) s += dd_next * (1.f + damp);
    if (fl & F_HAS_PREV) s += dd_prev * (1.f + damp);
    b.inv_s = 1.f / s;
    b.inv_s3a = 1.f / (s + 3.f * b.a);
    return b;
}

// Position block solve of one vertex: cosseratItr, YarnBall/sim/cosserat.cu:112-161 and
// :254-285, without the hair-hair collision terms (:163-227) and with the step limit at
// infinity (recomputeStepLimitKernel<false,*>, collision.cu:95-131).
//   segment i   (next): e_n = x_{i+1} - x_i, 1/l, k = kStretch/l, d = k/l, d3 = q_i e_x q_i*
//   segment i-1 (prev): the same for the previous segment.
// vbd_position_from starts from the force f: the inertial force bc.a (y - dx), to which a tied
// vertex has added its connection spring's force.
__device__ __forceinline__ float3 vbd_position_from(float3 f, float3 dx, uint32_t fl, BlockConst bc, float3 e_n,
                                                    float invl_n, float kk_n, float dd_n, float3 d3_n, float3 dx_next,
                                                    float3 e_p, float invl_p, float kk_p, float dd_p, float3 d3_p,
                                                    float3 dx_prev, float damp, float accel) {
    if (fl & F_HAS_NEXT) {
        float3 c = (e_n + (dx_next - dx)) * invl_n - d3_n;
        f = f + (kk_n * c - (damp * dd_n) * dx);
    }
    if (fl & F_HAS_PREV) {
        float3 c = (e_p + (dx - dx_prev)) * invl_p - d3_p;
        f = f + ((-kk_p) * c - (damp * dd_p) * dx);
    }
    float m = (f.x + f.y + f.z) * (1.f / 3.f);
    float mb = m * bc.inv_s3a;
    float3 delta = f3((f.x - m) * bc.inv_s + mb, (f.y - m) * bc.inv_s + mb, (f.z - m) * bc.inv_s + mb);
    return dx + accel * delta;
}
__device__ __forceinline__ float3 vbd_position(float3 dx, float3 y, uint32_t fl, BlockConst bc, float3 e_n, float invl_n,
                                               float kk_n, float dd_n, float3 d3_n, float3 dx_next, float3 e_p,
                                               float invl_p, float kk_p, float dd_p, float3 d3_p, float3 dx_prev,
                                               float damp, float accel) {
    return vbd_position_from(bc.a * (y - dx), dx, fl, bc, e_n, invl_n, kk_n, dd_n, d3_n, dx_next, e_p, invl_p, kk_p,
                             dd_p, d3_p, dx_prev, damp, accel);
}

// Closed-form segment orientation: quaternionLambdaItr, YarnBall/sim/cosserat.cu:290-337
// (SCR Eq. 15-22).  m2k = -2 kStretch / lRest.  Both neighbour terms use the identity
// <conj(a) b, r> = <a r, b> (and <conj(a) b, r> = <b conj(r), a>), so the sign test of each
// term reuses the product that the term adds to b.
__device__ __forceinline__ float4 vbd_orientation(float4 q, uint32_t fl, float3 e, float3 dx, float3 dx_next, float m2k,
                                                  float4 q_prev, float4 qr_prev, float4 q_next, float4 qr) {
    float3 V = (e + (dx_next - dx)) * m2k;
    float4 b = make_float4(0.f, 0.f, 0.f, 0.f);
    if (fl & F_HAS_PREV) {
        float4 P = qmul(q_prev, qr_prev);
        float phi = dot4(q, P) > 0.f ? 1.f : -1.f;
        b = add4(b, scale4(phi, P));
    }
    if (fl & F_HAS_NEXT_ORIENTATION) {
        float4 P = qmul_conj(q_next, qr);
        float phi = dot4(q, P) > 0.f ? 1.f : -1.f;
        b = add4(b, scale4(phi, P));
    }
    float lambda = sqrtf(dot3(V, V)) + sqrtf(dot4(b, b));
    // (V (x) b (x) e_x).v with V = (V, 0):  P = V b;  P e_x = (P.w, P.z, -P.y, -P.x)
    float3 bq = f3(b.x, b.y, b.z);
    float3 Pq = b.w * V + cross3(V, bq);
    float Pw = -dot3(V, bq);
    float4 R = make_float4(Pw + lambda * b.x, Pq.z + lambda * b.y, -Pq.y + lambda * b.z, -Pq.x + lambda * b.w);
    return scale4(rsqrtf(dot4(R, R)), R);
}

// Velocity update and advection: endItr, YarnBall/sim/iteration.cu:62-74.
__device__ __forceinline__ void vbd_finish(float3& x, float3& v, float3 dx, float inv_mass, float h, float decay) {
    if (inv_mass != 0.f) v = dx * (1.f / h) * (1.f - decay * h);
    x = x + dx;
}

// Body SDF projection of one non-root vertex: SDFHeadCollision + TriInterpSDF + index helpers,
// SDFCollisionSolver/cudaSDFCollision.cu:88-155 and :205-268.  The nearest-node index is
// truncated toward zero from (p/ds + 0.5) and the interpolation weights are measured from
// (idx - 0.5) ds, both in double, as there.  Outside-grid corners contribute a zero gradient and
// the border value of phi (zero-Neumann, :102-118).
__device__ __forceinline__ void vbd_sdf(float3& x, float3& v, const SdfParams& sp, const StepParams& st) {
    float4 invq = make_float4(-st.rot_x, -st.rot_y, -st.rot_z, st.rot_w);
    float3 lp = qrotate(invq, x - f3(st.tr_x, st.tr_y, st.tr_z)) - f3(sp.min_x, sp.min_y, sp.min_z);
    int ix = (int)((double)(lp.x * sp.inv_x) + 0.5);
    int iy = (int)((double)(lp.y * sp.inv_y) + 0.5);
    int iz = (int)((double)(lp.z * sp.inv_z) + 0.5);
    if (ix < 0 || ix >= sp.nx || iy < 0 || iy >= sp.ny || iz < 0 || iz >= sp.nz) return;
    const int jx = min(ix + 1, sp.nx - 1), jy = min(iy + 1, sp.ny - 1), jz = min(iz + 1, sp.nz - 1);
    const bool ox = ix + 1 < sp.nx, oy = iy + 1 < sp.ny, oz = iz + 1 < sp.nz;
    const int64_t sy = sp.nx, sz = (int64_t)sp.nx * sp.ny;
    auto ld = [&](int cx, int cy, int cz, bool inside) {
        float4 c = __ldg(sp.grid + (cx + cy * sy + cz * sz));
        if (!inside) c.x = c.y = c.z = 0.f;
        return c;
    };
    float4 c000 = ld(ix, iy, iz, true);
    float4 c100 = ld(jx, iy, iz, ox);
    float4 c010 = ld(ix, jy, iz, oy);
    float4 c110 = ld(jx, jy, iz, ox && oy);
    float4 c001 = ld(ix, iy, jz, oz);
    float4 c101 = ld(jx, iy, jz, ox && oz);
    float4 c011 = ld(ix, jy, jz, oy && oz);
    float4 c111 = ld(jx, jy, jz, ox && oy && oz);
    float ux = (float)((double)sp.inv_x * ((double)lp.x - ((double)ix - 0.5) * (double)sp.ds_x));
    float uy = (float)((double)sp.inv_y * ((double)lp.y - ((double)iy - 0.5) * (double)sp.ds_y));
    float uz = (float)((double)sp.inv_z * ((double)lp.z - ((double)iz - 0.5) * (double)sp.ds_z));
    auto lerp4 = [](float4 a, float4 b, float t) {
        return make_float4(a.x * (1.f - t) + b.x * t, a.y * (1.f - t) + b.y * t, a.z * (1.f - t) + b.z * t,
                           a.w * (1.f - t) + b.w * t);
    };
    float4 c00 = lerp4(c000, c100, ux), c01 = lerp4(c001, c101, ux);
    float4 c10 = lerp4(c010, c110, ux), c11 = lerp4(c011, c111, ux);
    float4 c0 = lerp4(c00, c10, uy), c1 = lerp4(c01, c11, uy);
    float4 r = lerp4(c0, c1, uz);
    float3 n = f3(r.x, r.y, r.z) * rsqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
    float phi = r.w - sp.thresh;
    if (phi < 0.f) {
        x = x - phi * n;
        float vl = sqrtf(dot3(v, v));
        if (vl >= 1e-6f) {
            float3 vn = v * (1.f / vl);
            v = v - dot3(vn, n) * n;
        }
    }
}

__device__ __forceinline__ bool finite3(float3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ bool finite4(float4 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(a.w); }

}  // namespace kami
