// vbd_adjoint.cu -- reverse-mode adjoint of the fused colour2 VBD step (one substep per step).
//
// The forward step is recorded by fused_step_kernel<C, false, true> (vbd_fused.cuh): the start
// state and, after the predict and after every iteration, every slot's displacement iterate dx and
// segment orientation q.  adjoint_step_kernel<C> walks one recorded step backwards, one warp per
// tile as in the forward:
//
//   SDF pass  ->  velocity update  ->  iterations N..1, each as
//     orientation sweep odd segments, even segments, position sweep odd vertices, even vertices
//   ->  predict.
//
// Each Gauss-Seidel colour sweep updates only its own colour from the other colour's values, so
// its adjoint is local: the slots of the swept colour turn their output adjoint into contributions
// to themselves and to their two neighbours, and the neighbours (the other colour) pull those
// contributions from registers or, across lanes, by warp shuffles.  Position block (see
// vbd_fused.cuh): dx' = dx + M f with M = isA (I - 11^T/3) + isB 11^T/3 symmetric, so
// fbar = M dx'bar and every linear term of f passes fbar on with its coefficient.  Orientation block
// (quaternionLambdaItr, YarnBall/sim/cosserat.cu:290-337): the sign tests are constants; the
// normalisation, the lambda norms and both quaternion products are differentiated by hand, using
// <a b, c> = <b, conj(a) c> = <a, c conj(b)> for the product adjoints.  The segment vectors
// e = x_{i+1} - x_i enter through the folded force constant and through V, the start velocity
// through the inertial target and the initial guess (iteration.cu:8-59), and with wind the start
// position's y and z through the wind force in both.  The parameter gradient
// d loss / d qRest accumulates in AdjointState::gqr.
#include "vbd_fused.cuh"
#include "vbd_kernels.h"

namespace kami {

__device__ __forceinline__ float4 qconj(float4 a) { return make_float4(-a.x, -a.y, -a.z, a.w); }

// 16-byte asynchronous global -> shared copies (each lane copies and later reads only its own cells).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_but_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ float3 zero3() { return f3(0.f, 0.f, 0.f); }

// J(q)^T g for d3 = q e_x q*  =  (w^2+x^2-y^2-z^2, 2(xy+wz), 2(xz-wy)).
__device__ __forceinline__ float4 d3_vjp(float4 q, float3 g) {
    return make_float4(2.f * (q.x * g.x + q.y * g.y + q.z * g.z), 2.f * (-q.y * g.x + q.x * g.y - q.w * g.z),
                       2.f * (-q.z * g.x + q.w * g.y + q.x * g.z), 2.f * (q.w * g.x + q.z * g.y - q.y * g.z));
}

// fbar = M g for the position block's symmetric M (isA, isB include the acceleration ratio).
__device__ __forceinline__ float3 pos_fbar(float3 g, float isA, float isB) {
    const float m = (g.x + g.y + g.z) * (1.f / 3.f);
    const float mb = m * isB;
    return f3((g.x - m) * isA + mb, (g.y - m) * isA + mb, (g.z - m) * isA + mb);
}

struct OrientationAdjoint {
    float4 p1bar;   // d loss / d (q_{k-1} qr_{k-1}): the previous segment turns it into q and qRest adjoints
    float4 q_next;  // contribution to the next segment's orientation adjoint
    float3 vt;      // m2k * Vbar: + to dx_{k+1}, - to dx_k, + to e_k
    float4 gqr;     // contribution to this segment's qRest adjoint
};

// Adjoint of one orientation update (fused_orientation) given the adjoint qbar of its output.
__device__ __forceinline__ OrientationAdjoint orientation_adjoint(float4 qbar, float4 q, bool upd, bool pre, bool nxt,
                                                                  float3 e, float m2k, float3 dx, float3 dxN,
                                                                  float4 qPrev, float4 qrPrev, float4 qNext,
                                                                  float4 qr) {
    OrientationAdjoint o;
    o.p1bar = zero4();
    o.q_next = zero4();
    o.vt = zero3();
    o.gqr = zero4();
    if (!upd) return o;
    const float3 V = m2k * (e + (dxN - dx));
    qPrev = pre ? qPrev : q;
    qNext = nxt ? qNext : q;
    const float4 P1 = qmul_fma(qPrev, qrPrev);  // as the forward step rounds them
    const float4 P2 = qmul_conj_fma(qNext, qr);
    float s1 = dot4(q, P1) > 0.f ? 1.f : -1.f;
    float s2 = dot4(q, P2) > 0.f ? 1.f : -1.f;
    s1 = pre ? s1 : 0.f;
    s2 = nxt ? s2 : 0.f;
    const float4 b = make_float4(s1 * P1.x + s2 * P2.x, s1 * P1.y + s2 * P2.y, s1 * P1.z + s2 * P2.z,
                                 s1 * P1.w + s2 * P2.w);
    // |V|, |b| and 1 / |R| as fused_orientation takes them (rsqrt forms), with the reciprocals the
    // reverse needs: 1 / |V| = iV and 1 / |b| = ib wherever the norm is above 1e-15
    const float vv = dot3(V, V), bb2 = dot4(b, b);
    const float iV = rsqrt_ftz(fmaxf(vv, 1e-30f)), ib = rsqrt_ftz(fmaxf(bb2, 1e-30f));
    const float nV = vv * iV, nb = bb2 * ib;
    const float lambda = nV + nb;
    const float3 bq = f3(b.x, b.y, b.z);
    const float3 Pq = b.w * V + cross3(V, bq);
    const float Pw = -dot3(V, bq);
    const float4 R = make_float4(Pw + lambda * b.x, Pq.z + lambda * b.y, -Pq.y + lambda * b.z, -Pq.x + lambda * b.w);
    const float iR = rsqrt_ftz(dot4(R, R));
    const float4 n = scale4(iR, R);
    // normalisation
    const float nq = dot4(n, qbar);
    const float4 Rb = scale4(iR, make_float4(qbar.x - n.x * nq, qbar.y - n.y * nq, qbar.z - n.z * nq, qbar.w - n.w * nq));
    // R = (Pw + l b.x, Pq.z + l b.y, -Pq.y + l b.z, -Pq.x + l b.w)
    const float Pwb = Rb.x;
    const float3 Pqb = f3(-Rb.w, -Rb.z, Rb.y);
    const float lb = dot4(Rb, b);
    float4 bb = scale4(lambda, Rb);
    // Pw = -V.bq ;  Pq = b.w V + V x bq
    float3 Vb = (-Pwb) * bq + b.w * Pqb + cross3(bq, Pqb);
    const float3 bqb = (-Pwb) * V + cross3(Pqb, V);
    bb.x += bqb.x;
    bb.y += bqb.y;
    bb.z += bqb.z;
    bb.w += dot3(V, Pqb);
    // lambda = |V| + |b|
    if (nV > 0.f) Vb = Vb + (lb * iV) * V;
    if (nb > 0.f) bb = add4(bb, scale4(lb * ib, b));
    const float4 P1b = scale4(s1, bb), P2b = scale4(s2, bb);
    o.p1bar = P1b;
    o.q_next = qmul_fma(P2b, qr);         // d/d qNext of qNext conj(qr)
    o.gqr = qmul_fma(qconj(P2b), qNext);  // d/d qr of qNext conj(qr)
    o.vt = m2k * Vb;
    return o;
}

// Adjoint of vbd_sdf: (gx, gv) = adjoint of the projected (x, v) -> adjoint of the unprojected ones.
__device__ __forceinline__ void sdf_adjoint(float3 x, float3 v, float3& gx, float3& gv, const SdfParams& sp,
                                            const StepParams& st) {
    const float4 rot = make_float4(st.rot_x, st.rot_y, st.rot_z, st.rot_w);
    const float4 invq = qconj(rot);
    const float3 lp = qrotate(invq, x - f3(st.tr_x, st.tr_y, st.tr_z)) - f3(sp.min_x, sp.min_y, sp.min_z);
    const int ix = (int)((double)(lp.x * sp.inv_x) + 0.5);
    const int iy = (int)((double)(lp.y * sp.inv_y) + 0.5);
    const int iz = (int)((double)(lp.z * sp.inv_z) + 0.5);
    if (ix < 0 || ix >= sp.nx || iy < 0 || iy >= sp.ny || iz < 0 || iz >= sp.nz) return;
    const int jx = min(ix + 1, sp.nx - 1), jy = min(iy + 1, sp.ny - 1), jz = min(iz + 1, sp.nz - 1);
    const bool ox = ix + 1 < sp.nx, oy = iy + 1 < sp.ny, oz = iz + 1 < sp.nz;
    const int64_t sy = sp.nx, sz = (int64_t)sp.nx * sp.ny;
    auto ld = [&](int cx, int cy, int cz, bool inside) {
        float4 c = __ldg(sp.grid + (cx + cy * sy + cz * sz));
        if (!inside) c.x = c.y = c.z = 0.f;
        return c;
    };
    const float4 c000 = ld(ix, iy, iz, true), c100 = ld(jx, iy, iz, ox), c010 = ld(ix, jy, iz, oy),
                 c110 = ld(jx, jy, iz, ox && oy), c001 = ld(ix, iy, jz, oz), c101 = ld(jx, iy, jz, ox && oz),
                 c011 = ld(ix, jy, jz, oy && oz), c111 = ld(jx, jy, jz, ox && oy && oz);
    const float ux = (float)((double)sp.inv_x * ((double)lp.x - ((double)ix - 0.5) * (double)sp.ds_x));
    const float uy = (float)((double)sp.inv_y * ((double)lp.y - ((double)iy - 0.5) * (double)sp.ds_y));
    const float uz = (float)((double)sp.inv_z * ((double)lp.z - ((double)iz - 0.5) * (double)sp.ds_z));
    auto lerp4 = [](float4 a, float4 b, float t) {
        return make_float4(a.x * (1.f - t) + b.x * t, a.y * (1.f - t) + b.y * t, a.z * (1.f - t) + b.z * t,
                           a.w * (1.f - t) + b.w * t);
    };
    auto sub4 = [](float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); };
    const float4 c00 = lerp4(c000, c100, ux), c01 = lerp4(c001, c101, ux);
    const float4 c10 = lerp4(c010, c110, ux), c11 = lerp4(c011, c111, ux);
    const float4 c0 = lerp4(c00, c10, uy), c1 = lerp4(c01, c11, uy);
    const float4 r = lerp4(c0, c1, uz);
    const float3 g = f3(r.x, r.y, r.z);
    const float gn = sqrtf(dot3(g, g));
    const float3 n = g * (1.f / gn);
    const float phi = r.w - sp.thresh;
    if (!(phi < 0.f)) return;
    // x' = x - phi n
    const float phib = -dot3(n, gx);
    float3 nb = (-phi) * gx;
    // v' = v - (v/|v| . n) n
    const float vl = sqrtf(dot3(v, v));
    if (vl >= 1e-6f) {
        const float3 vh = v * (1.f / vl);
        const float s = dot3(vh, n);
        const float sb = -dot3(n, gv);
        nb = nb + (-s) * gv + sb * vh;
        const float3 vhb = sb * n;
        gv = gv + (vhb - dot3(vh, vhb) * vh) * (1.f / vl);
    }
    // n = g / |g|
    const float3 gb = (nb - dot3(n, nb) * n) * (1.f / gn);
    const float4 cb = make_float4(gb.x, gb.y, gb.z, phib);
    // trilinear interpolation derivatives
    const float4 dux = add4(scale4(1.f - uz, add4(scale4(1.f - uy, sub4(c100, c000)), scale4(uy, sub4(c110, c010)))),
                            scale4(uz, add4(scale4(1.f - uy, sub4(c101, c001)), scale4(uy, sub4(c111, c011)))));
    const float4 duy = add4(scale4(1.f - uz, sub4(c10, c00)), scale4(uz, sub4(c11, c01)));
    const float4 duz = sub4(c1, c0);
    const float3 ub = f3(dot4(cb, dux) * sp.inv_x, dot4(cb, duy) * sp.inv_y, dot4(cb, duz) * sp.inv_z);
    gx = gx + qrotate(rot, ub);
}

// initItr's wind (iteration.cu:18-30), windx = peak * max(0, pow(cY cZ, sharp) sign(cY cZ)) with
// cY = cos 2 pi (fY y + fT t) for y > 0 (else 0) and cZ = cos 2 pi (fZ |z| + fT t), evaluated as
// vbd_predict does, and its derivatives d windx / d y, d windx / d z.  Where windx > 0,
// d windx / d (cY cZ) = peak sharp pw / (cY cZ) (pw = pow(cY cZ, sharp) sign(cY cZ), which holds for
// either sign of cY cZ); elsewhere windx is 0 and so is its derivative.
__device__ __forceinline__ float wind_with_grad(float3 x, const PhysParams& pp, float time, float& dwy, float& dwz) {
    const double two_pi = 2.0 * 3.14159265358979323846;
    const double ay = two_pi * (double)(pp.wind_yf * x.y + pp.wind_tf * time);
    const double az = two_pi * (double)(pp.wind_zf * fabsf(x.z) + pp.wind_tf * time);
    const float wy = x.y > 0.f ? (float)cos(ay) : 0.f;
    const float wz = (float)cos(az);
    const float prod = wy * wz;
    const float sg = prod > 0.f ? 1.f : (prod < 0.f ? -1.f : 0.f);
    const float pw = powf(prod, pp.wind_sharp) * sg;
    dwy = 0.f;
    dwz = 0.f;
    if (!(0.f < pw)) return 0.f;
    const float dprod = pp.wind_peak * pp.wind_sharp * pw / prod;
    const float dy = x.y > 0.f ? (float)(-two_pi * (double)pp.wind_yf * sin(ay)) : 0.f;
    const float zs = x.z > 0.f ? 1.f : (x.z < 0.f ? -1.f : 0.f);
    const float dz = (float)(-two_pi * (double)pp.wind_zf * sin(az)) * zs;
    dwy = dprod * wz * dy;
    dwz = dprod * wy * dz;
    return pp.wind_peak * pw;
}

// Adjoint values a group's warps hand across their tile boundaries (GROUPED: one CTA of NW = K warps
// per group of tiles, as GroupExchange in vbd_fused.cuh): `up` from lane 31 of warp w to lane 0 of
// warp w + 1, `down` from lane 0 of warp w to lane 31 of warp w - 1.  Each slot is written once per
// iteration and the next write comes after further __syncthreads that its readers have passed.
enum : int { AU_QR, AU_DD, AU_TQ, AU_TV, AU_QO, AU_F0, AU_GE, AU_N };
enum : int { AD_X, AD_QN, AD_DXN, AD_PN, AD_FN, AD_N };
template <int NW>
struct AdjointExchange {
    float4 up[NW][AU_N];
    float4 down[NW][AD_N];
};

// MINB blocks of NT threads per SM: (128, 4) caps the registers at 128 so 16 warps share an SM.
// NT = 256 is the instantiation for groups of 8 tiles; its prefetch buffer is dynamic shared memory.
template <int C, int MINB, bool GROUPED = false, int NT = 128>
__global__ void __launch_bounds__(NT, MINB) adjoint_step_kernel(DeviceState st, PhysParams pp, StepParams sp,
                                                                SdfParams sdf, TapeView tp, AdjointState ad) {
    const int lane = threadIdx.x & 31;
    const int64_t tile = tp.tile_begin + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tile >= st.num_tiles) return;  // uniform per warp (per CTA for groups)
    const int gw = threadIdx.x >> 5, gK = blockDim.x >> 5;
    AdjointExchange<NT / 32>* gx_ = nullptr;
    if constexpr (GROUPED) {
        __shared__ AdjointExchange<NT / 32> adjoint_exchange;
        gx_ = &adjoint_exchange;
    }
    // neighbours across the warps of a group; at a group's ends (and without groups) the previous /
    // next lane of lane 0 / 31 is another strand or nothing, and gets `edge`
    auto xsync = [&]() {
        if (GROUPED) __syncthreads();
    };
    auto up_put = [&](int slot, float4 v) {
        if (GROUPED && lane == 31) gx_->up[gw][slot] = v;
    };
    auto down_put = [&](int slot, float4 v) {
        if (GROUPED && lane == 0) gx_->down[gw][slot] = v;
    };
    auto up_get = [&](int slot, float4 v, float4 edge) {
        if (lane != 0) return v;
        return (GROUPED && gw > 0) ? gx_->up[gw - 1][slot] : edge;
    };
    auto down_get = [&](int slot, float4 v, float4 edge) {
        if (lane != 31) return v;
        return (GROUPED && gw < gK - 1) ? gx_->down[gw + 1][slot] : edge;
    };
    auto f4 = [](float3 a) { return make_float4(a.x, a.y, a.z, 0.f); };
    const int64_t base = tile * (32LL * C) + lane;
    const int64_t S = tp.slots;
    const int N = tp.num_itr;
    const int64_t tslot = base - tp.tile_begin * 32LL * C;  // this lane's slot in the tape window
    const int64_t row0 = ((int64_t)tp.step * (N + 1)) * S + tslot;
    const int64_t srow = (int64_t)tp.step * S + tslot;

    float3 x[C], v[C], vl[C], e[C], gdx[C], ge[C], gy[C], gx[C], gv[C], gvl[C], gd3[C];
    float4 qr[C], gq[C], gqr[C];
    float im[C], kk[C], ddN[C], kkN[C], as_[C], isA[C], isB[C], a_[C];
    uint32_t fl[C];
    bool mov[C];

#pragma unroll
    for (int k = 0; k < C; k++) {
        const int64_t g = base + 32LL * k;
        const float4 xm = tp.x[srow + 32LL * k];
        x[k] = xyz(xm);
        im[k] = xm.w;
        v[k] = xyz(tp.v[srow + 32LL * k]);
        vl[k] = xyz(tp.vl[srow + 32LL * k]);
        qr[k] = st.qr[g];
        const float4 p = st.prm[g];
        const float invl = 1.f / p.x;
        kk[k] = p.y * invl;
        fl[k] = __float_as_uint(p.w);
        mov[k] = im[k] != 0.f;
        ddN[k] = (fl[k] & F_HAS_NEXT) ? kk[k] * invl : 0.f;
        kkN[k] = (fl[k] & F_HAS_NEXT) ? kk[k] : 0.f;
    }
    float4 qrH = shfl_up4(qr[C - 1], 1);
    float ddH = __shfl_up_sync(0xffffffffu, ddN[C - 1], 1);
    if (GROUPED) {
        up_put(AU_QR, qr[C - 1]);
        up_put(AU_DD, make_float4(ddN[C - 1], 0.f, 0.f, 0.f));
        xsync();
        qrH = up_get(AU_QR, qrH, qrH);
        ddH = up_get(AU_DD, make_float4(ddH, 0.f, 0.f, 0.f), make_float4(ddH, 0.f, 0.f, 0.f)).x;
    }
    const float h = sp.h;
    const float damp = pp.damping / h;
    const float accel = pp.accel_ratio;
#pragma unroll
    for (int k = 0; k < C - 1; k++) e[k] = x[k + 1] - x[k];
    float3 xN0 = shfl_down3(x[0], 1);
    if (GROUPED) {
        down_put(AD_X, f4(x[0]));
        xsync();
        xN0 = xyz(down_get(AD_X, f4(xN0), f4(xN0)));
    }
    e[C - 1] = xN0 - x[C - 1];
#pragma unroll
    for (int k = 0; k < C; k++) {
        e[k] = (fl[k] & F_HAS_NEXT) ? e[k] : zero3();
        const float ddP = k > 0 ? ddN[k > 0 ? k - 1 : 0] : ddH;
        const float a = mov[k] ? 1.f / (im[k] * h * h) : 0.f;
        const float sk = (ddN[k] + ddP) * (1.f + damp);
        a_[k] = a;
        as_[k] = a + sk;
        isA[k] = mov[k] ? accel / sk : 0.f;
        isB[k] = mov[k] ? accel / (sk + 3.f * a) : 0.f;
    }

    // adjoint of the step's output, through the SDF pass and the velocity update (endItr)
    const float vscale = (1.f / h) * (1.f - pp.velocity_decay * h);
#pragma unroll
    for (int k = 0; k < C; k++) {
        const int64_t g = base + 32LL * k;
        const float3 dxN = xyz(tp.dx[row0 + (int64_t)N * S + 32LL * k]);
        const float3 xpre = x[k] + dxN;
        const float3 vpre = mov[k] ? dxN * vscale : v[k];
        float3 gxo = xyz(ad.gx[g]), gvo = xyz(ad.gv[g]);
        if (sdf.grid && (fl[k] & F_VALID) && !(fl[k] & F_ROOT)) sdf_adjoint(xpre, vpre, gxo, gvo, sdf, sp);
        gdx[k] = mov[k] ? gxo + gvo * vscale : gxo;
        gx[k] = gxo;
        gv[k] = (mov[k] ? zero3() : gvo) + xyz(ad.gvl[g]);  // the step's vlast output is its start velocity
        gvl[k] = zero3();
        gq[k] = ad.gq[g];
        ge[k] = zero3();
        gy[k] = zero3();
        gd3[k] = zero3();
        gqr[k] = zero4();
    }

    // iterate values after (n) and before (o) the iteration being reversed; the "before" values of
    // one iteration are the "after" values of the next one down, so each tape row is read once.  The
    // row of the next iteration down is prefetched into shared memory (double buffer per warp) while
    // the current one is reversed.
    float4 (*mine)[2][C][32];  // this warp's [buffer][dx | q][slot row][lane]
    if constexpr (NT <= 128) {
        __shared__ float4 pref[4][2][2][C][32];  // [warp in CTA][buffer][dx | q][slot row][lane]
        mine = pref[threadIdx.x >> 5];
    } else {  // 8 warps: 32 KB (C = 2) or 64 KB (C = 4), in dynamic shared memory
        extern __shared__ float4 adjoint_pref[];
        mine = reinterpret_cast<float4 (*)[2][C][32]>(adjoint_pref + (size_t)(threadIdx.x >> 5) * 2 * 2 * C * 32);
    }
    float3 dxn[C], dxo[C];
    float4 qn[C], qo[C];
#pragma unroll
    for (int k = 0; k < C; k++) {
        dxn[k] = xyz(tp.dx[row0 + (int64_t)N * S + 32LL * k]);
        qn[k] = tp.q[row0 + (int64_t)N * S + 32LL * k];
        if (N >= 1) {
            cp_async16(&mine[0][0][k][lane], &tp.dx[row0 + (int64_t)(N - 1) * S + 32LL * k]);
            cp_async16(&mine[0][1][k][lane], &tp.q[row0 + (int64_t)(N - 1) * S + 32LL * k]);
        }
    }
    cp_async_commit();
    for (int it = N; it >= 1; it--) {
        const int buf = (N - it) & 1;
        if (it >= 2) {
#pragma unroll
            for (int k = 0; k < C; k++) {
                cp_async16(&mine[buf ^ 1][0][k][lane], &tp.dx[row0 + (int64_t)(it - 2) * S + 32LL * k]);
                cp_async16(&mine[buf ^ 1][1][k][lane], &tp.q[row0 + (int64_t)(it - 2) * S + 32LL * k]);
            }
        }
        cp_async_commit();
        cp_async_wait_all_but_one();  // this iteration's row has landed
#pragma unroll
        for (int k = 0; k < C; k++) {
            dxo[k] = xyz(mine[buf][0][k][lane]);
            qo[k] = mine[buf][1][k][lane];
        }
        float4 p1b[C], tq[C];
        float3 tv[C];
        // ---- orientations, odd segments (read even neighbours' new values)
        {
            float4 qnN0 = shfl_down4(qn[0], 1);
            float3 dxnN0 = shfl_down3(dxn[0], 1);
            if (GROUPED) {
                down_put(AD_QN, qn[0]);
                down_put(AD_DXN, f4(dxn[0]));
                xsync();
                qnN0 = down_get(AD_QN, qnN0, qnN0);
                dxnN0 = xyz(down_get(AD_DXN, f4(dxnN0), f4(dxnN0)));
            }
#pragma unroll
            for (int k = 1; k < C; k += 2) {
                const int kn = k + 1 < C ? k + 1 : k;
                const uint32_t f = fl[k];
                const bool upd = (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION);
                OrientationAdjoint o =
                    orientation_adjoint(gq[k], qo[k], upd, f & F_HAS_PREV, f & F_HAS_NEXT_ORIENTATION, e[k], -2.f * kk[k],
                                        dxn[k], k == C - 1 ? dxnN0 : dxn[kn], qn[k - 1], qr[k - 1],
                                        k == C - 1 ? qnN0 : qn[kn], qr[k]);
                p1b[k] = o.p1bar;
                tq[k] = o.q_next;
                tv[k] = o.vt;
                gqr[k] = add4(gqr[k], o.gqr);
                gdx[k] = gdx[k] - o.vt;
                ge[k] = ge[k] + o.vt;
                gq[k] = upd ? zero4() : gq[k];
            }
            float4 tq0 = shfl_up4(tq[C - 1], 1);
            float3 tv0 = shfl_up3(tv[C - 1], 1);
            up_put(AU_TQ, tq[C - 1]);
            up_put(AU_TV, f4(tv[C - 1]));
            xsync();
            tq0 = up_get(AU_TQ, tq0, zero4());
            tv0 = xyz(up_get(AU_TV, f4(tv0), zero4()));
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const float4 P = p1b[j + 1];
                gq[j] = add4(gq[j], qmul_conj_fma(P, qr[j]));
                gqr[j] = add4(gqr[j], qmul_fma(qconj(qn[j]), P));
                gq[j] = add4(gq[j], j ? tq[j > 0 ? j - 1 : 0] : tq0);
                gdx[j] = gdx[j] + (j ? tv[j > 0 ? j - 1 : 0] : tv0);
            }
        }
        // ---- orientations, even segments (read odd neighbours' old values)
        {
            float4 qoP = shfl_up4(qo[C - 1], 1);
            if (GROUPED) {
                up_put(AU_QO, qo[C - 1]);
                xsync();
                qoP = up_get(AU_QO, qoP, qoP);
            }
#pragma unroll
            for (int k = 0; k < C; k += 2) {
                const int kp = k > 0 ? k - 1 : 0;
                const uint32_t f = fl[k];
                const bool upd = (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION);
                OrientationAdjoint o =
                    orientation_adjoint(gq[k], qo[k], upd, f & F_HAS_PREV, f & F_HAS_NEXT_ORIENTATION, e[k], -2.f * kk[k],
                                        dxn[k], dxn[k + 1], k ? qo[kp] : qoP, k ? qr[kp] : qrH, qo[k + 1], qr[k]);
                p1b[k] = o.p1bar;
                tq[k] = o.q_next;
                tv[k] = o.vt;
                gqr[k] = add4(gqr[k], o.gqr);
                gdx[k] = gdx[k] - o.vt;
                ge[k] = ge[k] + o.vt;
                gq[k] = upd ? zero4() : gq[k];
            }
            float4 pN = shfl_down4(p1b[0], 1);
            down_put(AD_PN, p1b[0]);
            xsync();
            pN = down_get(AD_PN, pN, zero4());
#pragma unroll
            for (int j = 1; j < C; j += 2) {
                const int jn = j + 1 < C ? j + 1 : j;
                gq[j] = add4(gq[j], tq[j - 1]);
                gdx[j] = gdx[j] + tv[j - 1];
                const float4 P = j == C - 1 ? pN : p1b[jn];
                gq[j] = add4(gq[j], qmul_conj_fma(P, qr[j]));
                gqr[j] = add4(gqr[j], qmul_fma(qconj(qo[j]), P));
            }
        }
        float3 fb[C];
        // ---- positions, odd vertices (read even neighbours' new values)
        {
#pragma unroll
            for (int k = 1; k < C; k += 2) {
                fb[k] = mov[k] ? pos_fbar(gdx[k], isA[k], isB[k]) : zero3();
                gdx[k] = gdx[k] - as_[k] * fb[k];
                gd3[k] = gd3[k] - kkN[k] * fb[k];
                gy[k] = gy[k] + a_[k] * fb[k];
                ge[k] = ge[k] + ddN[k] * fb[k];
            }
            float3 f0 = shfl_up3(fb[C - 1], 1);
            up_put(AU_F0, f4(fb[C - 1]));
            xsync();
            f0 = xyz(up_get(AU_F0, f4(f0), zero4()));
#pragma unroll
            for (int j = 0; j < C; j += 2) {
                const float3 fn = fb[j + 1];  // from the next vertex (its previous-segment terms)
                gdx[j] = gdx[j] + ddN[j] * fn;
                gd3[j] = gd3[j] + kkN[j] * fn;
                ge[j] = ge[j] - ddN[j] * fn;
                const float3 fp = j ? fb[j > 0 ? j - 1 : 0] : f0;  // from the previous vertex (its next-segment terms)
                gdx[j] = gdx[j] + (j ? ddN[j > 0 ? j - 1 : 0] : ddH) * fp;
            }
        }
        // ---- positions, even vertices (read odd neighbours' old values)
        {
#pragma unroll
            for (int k = 0; k < C; k += 2) {
                fb[k] = mov[k] ? pos_fbar(gdx[k], isA[k], isB[k]) : zero3();
                gdx[k] = gdx[k] - as_[k] * fb[k];
                gd3[k] = gd3[k] - kkN[k] * fb[k];
                gy[k] = gy[k] + a_[k] * fb[k];
                ge[k] = ge[k] + ddN[k] * fb[k];
            }
            float3 fN = shfl_down3(fb[0], 1);
            down_put(AD_FN, f4(fb[0]));
            xsync();
            fN = xyz(down_get(AD_FN, f4(fN), zero4()));
#pragma unroll
            for (int j = 1; j < C; j += 2) {
                const int jn = j + 1 < C ? j + 1 : j;
                gdx[j] = gdx[j] + ddN[j - 1] * fb[j - 1];
                const float3 fn = j == C - 1 ? fN : fb[jn];
                gdx[j] = gdx[j] + ddN[j] * fn;
                gd3[j] = gd3[j] + kkN[j] * fn;
                ge[j] = ge[j] - ddN[j] * fn;
            }
        }
#pragma unroll
        for (int k = 0; k < C; k++) {
            gq[k] = add4(gq[k], d3_vjp(qo[k], gd3[k]));
            gd3[k] = zero3();
            dxn[k] = dxo[k];
            qn[k] = qo[k];
        }
    }

    // ---- predict (initItr): dx0 = h v [+ h^2 s ext], y = h v + h^2 ext, vlast_out = v, where
    // ext = (g + (windx(x), 0, 0)) * ext_mult and s = clamp(acc . ext / |ext|^2, 0, 1)
#pragma unroll
    for (int k = 0; k < C; k++) {
        gv[k] = gv[k] + h * gdx[k];
        if (mov[k]) {
            float dwy = 0.f, dwz = 0.f;
            const float windx = pp.wind_peak != 0.f ? wind_with_grad(x[k], pp, sp.time, dwy, dwz) : 0.f;
            const float3 ext = f3(pp.gx + windx, pp.gy, pp.gz) * pp.ext_mult;
            const float ext2 = dot3(ext, ext);
            gv[k] = gv[k] + h * gy[k];
            float gex = h * h * gy[k].x;  // d loss / d ext.x
            if (ext2 > 0.f) {
                const float3 acc = (v[k] - vl[k]) * (1.f / sp.last_h);
                const float sr = dot3(acc, ext) / ext2;
                gex += h * h * fminf(fmaxf(sr, 0.f), 1.f) * gdx[k].x;
                if (sr > 0.f && sr < 1.f) {
                    const float eg = h * h * dot3(ext, gdx[k]);
                    const float c = eg / (sp.last_h * ext2);
                    gv[k] = gv[k] + c * ext;
                    gvl[k] = gvl[k] - c * ext;
                    gex += eg / ext2 * (acc.x - 2.f * sr * ext.x);  // d s / d ext = (acc - 2 s ext) / |ext|^2
                }
            }
            const float gwind = gex * pp.ext_mult;  // d loss / d windx
            gx[k].y += gwind * dwy;
            gx[k].z += gwind * dwz;
        }
    }
    // ---- segment vectors e_k = x_{k+1} - x_k
    float3 geP = shfl_up3(ge[C - 1], 1);
    up_put(AU_GE, f4(ge[C - 1]));
    xsync();
    geP = xyz(up_get(AU_GE, f4(geP), zero4()));
#pragma unroll
    for (int k = 0; k < C; k++) {
        gx[k] = gx[k] - ge[k] + (k ? ge[k > 0 ? k - 1 : 0] : geP);
        const int64_t g = base + 32LL * k;
        ad.gx[g] = make_float4(gx[k].x, gx[k].y, gx[k].z, 0.f);
        ad.gv[g] = make_float4(gv[k].x, gv[k].y, gv[k].z, 0.f);
        ad.gvl[g] = make_float4(gvl[k].x, gvl[k].y, gvl[k].z, 0.f);
        ad.gq[g] = gq[k];
        ad.gqr[g] = add4(ad.gqr[g], gqr[k]);
    }
}

// ------------------------------------------------------------------------------------------
cudaError_t launch_fused_record(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                                const TapeView& tp, int C, int warps_per_block, cudaStream_t s, int group) {
    if (group > 1) {  // one CTA of `group` warps per group of tiles (the window is whole groups)
        const int64_t tiles = st.num_tiles - tp.tile_begin;
        if (group > 8 || tiles % group != 0 || tp.tile_begin % group != 0) return cudaErrorInvalidValue;
        if (tiles == 0) return cudaSuccess;
        const unsigned gblocks = (unsigned)(tiles / group);
        if (C == 2)
            fused_record_group_kernel<2><<<gblocks, 32 * group, 0, s>>>(st, pp, sp, sdf, tp);
        else if (C == 4)
            fused_record_group_kernel<4><<<gblocks, 32 * group, 0, s>>>(st, pp, sp, sdf, tp);
        else
            return cudaErrorInvalidValue;
        return cudaGetLastError();
    }
    const int threads = 32 * warps_per_block;
    const int64_t tiles = st.num_tiles - tp.tile_begin;
    const unsigned blocks = (unsigned)((tiles + warps_per_block - 1) / warps_per_block);
    if (blocks == 0) return cudaSuccess;
    if (C == 2)
        fused_step_kernel<2, false, true><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, tp, nullptr, 1);
    else if (C == 4)
        fused_step_kernel<4, false, true><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, tp, nullptr, 1);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_adjoint_step(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                                const TapeView& tp, const AdjointState& ad, int C, cudaStream_t s, int group) {
    if (group > 1) {  // one CTA of `group` warps per group of tiles
        const int64_t tiles = st.num_tiles - tp.tile_begin;
        if ((group != 2 && group != 4 && group != 8) || tiles % group != 0 || tp.tile_begin % group != 0)
            return cudaErrorInvalidValue;
        if (tiles == 0) return cudaSuccess;
        const unsigned gblocks = (unsigned)(tiles / group);
        if (group == 8) {
            const size_t smem = sizeof(float4) * 8 * 2 * 2 * C * 32;  // the per-warp prefetch buffers
            if (C == 2) {
                adjoint_step_kernel<2, 2, true, 256><<<gblocks, 256, smem, s>>>(st, pp, sp, sdf, tp, ad);
            } else if (C == 4) {
                // per launch: the attribute belongs to the current device, and a process may drive several
                const cudaError_t attr = cudaFuncSetAttribute(adjoint_step_kernel<4, 1, true, 256>,
                                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (attr != cudaSuccess) return attr;
                adjoint_step_kernel<4, 1, true, 256><<<gblocks, 256, smem, s>>>(st, pp, sp, sdf, tp, ad);
            } else {
                return cudaErrorInvalidValue;
            }
            return cudaGetLastError();
        }
        if (C == 2)
            adjoint_step_kernel<2, 4, true><<<gblocks, 32 * group, 0, s>>>(st, pp, sp, sdf, tp, ad);
        else if (C == 4)
            adjoint_step_kernel<4, 2, true><<<gblocks, 32 * group, 0, s>>>(st, pp, sp, sdf, tp, ad);
        else
            return cudaErrorInvalidValue;
        return cudaGetLastError();
    }
    const int wpb = 4;
    const int64_t tiles = st.num_tiles - tp.tile_begin;
    const unsigned blocks = (unsigned)((tiles + wpb - 1) / wpb);
    if (blocks == 0) return cudaSuccess;
    if (C == 2)
        adjoint_step_kernel<2, 4><<<blocks, 32 * wpb, 0, s>>>(st, pp, sp, sdf, tp, ad);
    else if (C == 4)
        adjoint_step_kernel<4, 2><<<blocks, 32 * wpb, 0, s>>>(st, pp, sp, sdf, tp, ad);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace kami
