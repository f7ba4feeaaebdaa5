// vbd_fused.cuh -- the fused step kernel: one warp per tile, all substeps and iterations of one
// KamiSimulator step in registers.
//
// Per substep every slot folds its step-constant terms into a few coefficients, so that an
// iteration only touches the iterated state (dx, q, d3 = q e_x q*):
//   position block (cosseratItr, YarnBall/sim/cosserat.cu:112-161, 246-285), with the segment
//   constraint c = (e + dx_next - dx)/l - d3 expanded,
//     f  = F0 + ddN dx_next + ddP dx_prev - (a + s) dx - kkN d3_i + kkP d3_{i-1}
//     F0 = a y + ddN e_i - ddP e_{i-1},  kk = kStretch / l,  dd = kk / l,  s = (ddN + ddP)(1 + damping/h)
//   (ddN/kkN are zero for a vertex without a next segment, ddP/kkP are the previous slot's),
//   then dx += (f - mean f) accel/s + mean f accel/(s + 3a)   (the exact inverse of a 1 1^T + s I),
//   evaluated as dx + f isA + mean f isD with isA = accel/s, isD = accel/(s + 3a) - isA;
//   orientation (quaternionLambdaItr, cosserat.cu:290-337) with V = -2 kk (e_i + dx_next - dx).
// Missing neighbours enter as zero coefficients or are discarded by selects, so the iteration
// loop has no data-dependent branches.
#pragma once
#include "vbd_math.cuh"

namespace kami {

// PTX rsqrt.approx.ftz.f32: rsqrtf's approximation without the input scaling that the non-ftz form
// adds for subnormal inputs.  Every input here is a normal float (or clamped to one), where the two
// give the same result.
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float sqrt_nonneg(float x) { return x * rsqrt_ftz(fmaxf(x, 1e-30f)); }

// The Hamilton product of qmul (vbd_common.cuh) as FMA chains: the same product in 16 instead of
// 20 instructions, rounded differently.  qmul_conj_fma(l, r) = l * conj(r).
__device__ __forceinline__ float4 qmul_fma(float4 l, float4 r) {
    return make_float4(fmaf(l.w, r.x, fmaf(r.w, l.x, fmaf(l.y, r.z, -r.y * l.z))),
                       fmaf(l.w, r.y, fmaf(r.w, l.y, fmaf(l.z, r.x, -r.z * l.x))),
                       fmaf(l.w, r.z, fmaf(r.w, l.z, fmaf(l.x, r.y, -r.x * l.y))),
                       fmaf(l.w, r.w, -fmaf(l.x, r.x, fmaf(l.y, r.y, l.z * r.z))));
}
__device__ __forceinline__ float4 qmul_conj_fma(float4 l, float4 r) {
    return qmul_fma(l, make_float4(-r.x, -r.y, -r.z, r.w));
}

// One position update with folded coefficients (see the file comment).  Neighbour operands from
// another strand (no segment in between: hn / hp false) are replaced by the vertex's own values
// before they meet their zero coefficient, and vertices that do not move (upd false) keep dx, so a
// non-finite strand cannot leak into the strands or padding that share its tile, as the
// reference's flag tests guarantee.  Strands start at even tile positions, so only the previous
// neighbour of an even slot and the next neighbour of an odd slot can belong to another strand;
// the others are the same strand or padding (always finite), and guard_next / guard_prev say
// which operands need the replacement (the results are the same bit for bit either way).  Padding
// and pinned slots keep their dx through the final select: padding must stay finite, as the
// strand before it reads it unguarded and a restored state does not rewrite padding.
__device__ __forceinline__ float3 fused_position(float3 dx, float3 F0, float ddN, float kkN, float3 d3N, float3 dxN,
                                                 float ddP, float kkP, float3 d3P, float3 dxP, float as_, float isA,
                                                 float isD, bool hn, bool hp, bool upd, bool guard_next,
                                                 bool guard_prev) {
    if (guard_next) dxN = hn ? dxN : dx;
    if (guard_prev) {
        dxP = hp ? dxP : dx;
        d3P = hp ? d3P : d3N;
    }
    float3 f;
    f.x = F0.x + ddN * dxN.x + ddP * dxP.x - as_ * dx.x - kkN * d3N.x + kkP * d3P.x;
    f.y = F0.y + ddN * dxN.y + ddP * dxP.y - as_ * dx.y - kkN * d3N.y + kkP * d3P.y;
    f.z = F0.z + ddN * dxN.z + ddP * dxP.z - as_ * dx.z - kkN * d3N.z + kkP * d3P.z;
    const float m = (f.x + f.y + f.z) * (1.f / 3.f);
    const float3 n = f3(fmaf(m, isD, fmaf(f.x, isA, dx.x)), fmaf(m, isD, fmaf(f.y, isA, dx.y)),
                        fmaf(m, isD, fmaf(f.z, isA, dx.z)));
    return upd ? n : dx;
}

// One orientation update (quaternionLambdaItr), branch-free: pre/nxt say whether the previous /
// next segment exists, upd whether this segment is updated at all; guard_prev / guard_next as in
// fused_position.
__device__ __forceinline__ float4 fused_orientation(float4 q, bool upd, bool pre, bool nxt, float3 Ve, float m2k,
                                                    float3 dx, float3 dxN, float4 qPrev, float4 qrPrev, float4 qNext,
                                                    float4 qr, bool guard_prev, bool guard_next) {
    const float3 V = Ve + m2k * (dxN - dx);
    if (guard_prev) qPrev = pre ? qPrev : q;  // operands from another strand never meet arithmetic
    if (guard_next) qNext = nxt ? qNext : q;
    const float4 P1 = qmul_fma(qPrev, qrPrev);
    const float4 P2 = qmul_conj_fma(qNext, qr);
    float s1 = dot4(q, P1) > 0.f ? 1.f : -1.f;
    float s2 = dot4(q, P2) > 0.f ? 1.f : -1.f;
    s1 = pre ? s1 : 0.f;
    s2 = nxt ? s2 : 0.f;
    const float4 b = make_float4(s1 * P1.x + s2 * P2.x, s1 * P1.y + s2 * P2.y, s1 * P1.z + s2 * P2.z,
                                 s1 * P1.w + s2 * P2.w);
    const float lambda = sqrt_nonneg(dot3(V, V)) + sqrt_nonneg(dot4(b, b));
    const float3 bq = f3(b.x, b.y, b.z);
    const float3 Pq = b.w * V + cross3(V, bq);
    const float Pw = -dot3(V, bq);
    const float4 R = make_float4(Pw + lambda * b.x, Pq.z + lambda * b.y, -Pq.y + lambda * b.z, -Pq.x + lambda * b.w);
    const float4 n = scale4(rsqrt_ftz(dot4(R, R)), R);
    return upd ? n : q;
}

// ---- packed FP32x2 form (sm_100 FFMA2 / FADD2 / FMUL2) ---------------------------------------------
// With 4 slots per lane, slots {0, 2} and {1, 3} are each one colour, and every operand of a colour's
// update pairs up with the same operand of the other slot of that colour.  The x2 kernel variant
// keeps each pair in a float2 and updates both slots with one packed instruction per operation.
struct F2x3 {
    float2 x, y, z;
};
struct F2x4 {
    float2 x, y, z, w;
};
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 sel2(bool cx, bool cy, float2 a, float2 b) {
    return make_float2(cx ? a.x : b.x, cy ? a.y : b.y);
}
__device__ __forceinline__ F2x3 sel23(bool cx, bool cy, F2x3 a, F2x3 b) {
    return {sel2(cx, cy, a.x, b.x), sel2(cx, cy, a.y, b.y), sel2(cx, cy, a.z, b.z)};
}
__device__ __forceinline__ F2x4 sel24(bool cx, bool cy, F2x4 a, F2x4 b) {
    return {sel2(cx, cy, a.x, b.x), sel2(cx, cy, a.y, b.y), sel2(cx, cy, a.z, b.z), sel2(cx, cy, a.w, b.w)};
}
__device__ __forceinline__ F2x3 pack3(float3 a, float3 b) {
    return {make_float2(a.x, b.x), make_float2(a.y, b.y), make_float2(a.z, b.z)};
}
__device__ __forceinline__ F2x4 pack4(float4 a, float4 b) {
    return {make_float2(a.x, b.x), make_float2(a.y, b.y), make_float2(a.z, b.z), make_float2(a.w, b.w)};
}
__device__ __forceinline__ float3 lo3(F2x3 a) { return f3(a.x.x, a.y.x, a.z.x); }
__device__ __forceinline__ float3 hi3(F2x3 a) { return f3(a.x.y, a.y.y, a.z.y); }
__device__ __forceinline__ float4 lo4(F2x4 a) { return make_float4(a.x.x, a.y.x, a.z.x, a.w.x); }
__device__ __forceinline__ float4 hi4(F2x4 a) { return make_float4(a.x.y, a.y.y, a.z.y, a.w.y); }

// d3 = q e_x q* for a pair (d3_of, vbd_common.cuh)
__device__ __forceinline__ F2x3 d3_of2(F2x4 q) {
    F2x3 d;
    d.x = sub2(fma2(q.w, q.w, mul2(q.x, q.x)), fma2(q.y, q.y, mul2(q.z, q.z)));
    const float2 s1 = fma2(q.x, q.y, mul2(q.w, q.z));
    d.y = add2(s1, s1);
    const float2 s2 = fma2(q.x, q.z, mul2(neg2(q.w), q.y));
    d.z = add2(s2, s2);
    return d;
}

// Hamilton product l r with the scalar last (qmul), and l conj(r) (qmul_conj), for pairs
__device__ __forceinline__ F2x4 qmul2(F2x4 l, F2x4 r) {
    F2x4 o;
    o.x = fma2(l.w, r.x, fma2(r.w, l.x, fma2(l.y, r.z, neg2(mul2(r.y, l.z)))));
    o.y = fma2(l.w, r.y, fma2(r.w, l.y, fma2(l.z, r.x, neg2(mul2(r.z, l.x)))));
    o.z = fma2(l.w, r.z, fma2(r.w, l.z, fma2(l.x, r.y, neg2(mul2(r.x, l.y)))));
    o.w = fma2(l.w, r.w, neg2(fma2(l.x, r.x, fma2(l.y, r.y, mul2(l.z, r.z)))));
    return o;
}
__device__ __forceinline__ F2x4 qmul_conj2(F2x4 l, F2x4 r) {
    return qmul2(l, F2x4{neg2(r.x), neg2(r.y), neg2(r.z), r.w});
}
__device__ __forceinline__ float2 dot42(F2x4 a, F2x4 b) {
    return fma2(a.x, b.x, fma2(a.y, b.y, fma2(a.z, b.z, mul2(a.w, b.w))));
}
__device__ __forceinline__ float2 dot32(F2x3 a, F2x3 b) { return fma2(a.x, b.x, fma2(a.y, b.y, mul2(a.z, b.z))); }
__device__ __forceinline__ float2 sqrt_nonneg2(float2 x) {
    return make_float2(sqrt_nonneg(x.x), sqrt_nonneg(x.y));
}

// fused_position for a pair of same-colour slots; nkkN = -kkN, nas = -(a + s) are precomputed.
// guard_next / guard_prev as in fused_position (even pair: previous; odd pair: next).
__device__ __forceinline__ F2x3 fused_position2(F2x3 dx, F2x3 F0, float2 ddN, float2 nkkN, F2x3 d3N, F2x3 dxN,
                                                float2 ddP, float2 kkP, F2x3 d3P, F2x3 dxP, float2 nas, float2 isA,
                                                float2 isD, const bool* hn, const bool* hp, const bool* upd,
                                                bool guard_next, bool guard_prev) {
    if (guard_next) dxN = sel23(hn[0], hn[1], dxN, dx);
    if (guard_prev) {
        dxP = sel23(hp[0], hp[1], dxP, dx);
        d3P = sel23(hp[0], hp[1], d3P, d3N);
    }
    F2x3 f;
    f.x = fma2(kkP, d3P.x, fma2(nkkN, d3N.x, fma2(nas, dx.x, fma2(ddP, dxP.x, fma2(ddN, dxN.x, F0.x)))));
    f.y = fma2(kkP, d3P.y, fma2(nkkN, d3N.y, fma2(nas, dx.y, fma2(ddP, dxP.y, fma2(ddN, dxN.y, F0.y)))));
    f.z = fma2(kkP, d3P.z, fma2(nkkN, d3N.z, fma2(nas, dx.z, fma2(ddP, dxP.z, fma2(ddN, dxN.z, F0.z)))));
    const float2 m = mul2(add2(add2(f.x, f.y), f.z), make_float2(1.f / 3.f, 1.f / 3.f));
    F2x3 n;
    n.x = fma2(m, isD, fma2(f.x, isA, dx.x));
    n.y = fma2(m, isD, fma2(f.y, isA, dx.y));
    n.z = fma2(m, isD, fma2(f.z, isA, dx.z));
    return sel23(upd[0], upd[1], n, dx);
}

// fused_orientation for a pair of same-colour segments; guard_prev / guard_next as in fused_position.
__device__ __forceinline__ F2x4 fused_orientation2(F2x4 q, const bool* upd, const bool* pre, const bool* nxt, F2x3 Ve,
                                                   float2 m2k, F2x3 dx, F2x3 dxN, F2x4 qPrev, F2x4 qrPrev,
                                                   F2x4 qNext, F2x4 qr, bool guard_prev, bool guard_next) {
    F2x3 V;
    V.x = fma2(m2k, sub2(dxN.x, dx.x), Ve.x);
    V.y = fma2(m2k, sub2(dxN.y, dx.y), Ve.y);
    V.z = fma2(m2k, sub2(dxN.z, dx.z), Ve.z);
    if (guard_prev) qPrev = sel24(pre[0], pre[1], qPrev, q);
    if (guard_next) qNext = sel24(nxt[0], nxt[1], qNext, q);
    const F2x4 P1 = qmul2(qPrev, qrPrev);
    const F2x4 P2 = qmul_conj2(qNext, qr);
    const float2 d1 = dot42(q, P1), d2 = dot42(q, P2);
    const float2 s1 = make_float2(pre[0] ? (d1.x > 0.f ? 1.f : -1.f) : 0.f, pre[1] ? (d1.y > 0.f ? 1.f : -1.f) : 0.f);
    const float2 s2 = make_float2(nxt[0] ? (d2.x > 0.f ? 1.f : -1.f) : 0.f, nxt[1] ? (d2.y > 0.f ? 1.f : -1.f) : 0.f);
    F2x4 b;
    b.x = fma2(s1, P1.x, mul2(s2, P2.x));
    b.y = fma2(s1, P1.y, mul2(s2, P2.y));
    b.z = fma2(s1, P1.z, mul2(s2, P2.z));
    b.w = fma2(s1, P1.w, mul2(s2, P2.w));
    const float2 lambda = add2(sqrt_nonneg2(dot32(V, V)), sqrt_nonneg2(dot42(b, b)));
    // P = V b e_x with V = (V, 0): R = (Pw + l b.x, Pq.z + l b.y, -Pq.y + l b.z, -Pq.x + l b.w),
    // Pq = b.w V + V x bq, Pw = -V . bq
    const float2 Pqx = fma2(b.w, V.x, sub2(mul2(V.y, b.z), mul2(b.y, V.z)));
    const float2 Pqy = fma2(b.w, V.y, sub2(mul2(V.z, b.x), mul2(b.z, V.x)));
    const float2 Pqz = fma2(b.w, V.z, sub2(mul2(V.x, b.y), mul2(b.x, V.y)));
    const float2 Pw = neg2(fma2(V.x, b.x, fma2(V.y, b.y, mul2(V.z, b.z))));
    F2x4 R;
    R.x = fma2(lambda, b.x, Pw);
    R.y = fma2(lambda, b.y, Pqz);
    R.z = fma2(lambda, b.z, neg2(Pqy));
    R.w = fma2(lambda, b.w, neg2(Pqx));
    const float2 rr = dot42(R, R);
    const float2 inv = make_float2(rsqrt_ftz(rr.x), rsqrt_ftz(rr.y));
    const F2x4 n = {mul2(inv, R.x), mul2(inv, R.y), mul2(inv, R.z), mul2(inv, R.w)};
    return sel24(upd[0], upd[1], n, q);
}

// Values a group's warps hand across their tile boundaries (GROUPED: one CTA of K <= 8 warps per
// group of K tiles, warp w on tile group * K + w): `up` from lane 31 of warp w to lane 0 of warp
// w + 1 (its previous lane), `down` from lane 0 of warp w to lane 31 of warp w - 1 (its next lane).
// Each slot is written once per substep or iteration and read after the __syncthreads that follows;
// the next write to it comes after at least one more __syncthreads, which every reader has passed.
enum : int { XU_QR, XU_DK, XU_E, XU_DX, XU_Q, XU_D3, XU_N };
enum : int { XD_X, XD_DX, XD_Q, XD_DX2, XD_N };
struct GroupExchange {
    float4 up[8][XU_N];
    float4 down[8][XD_N];
};

// One launch runs `nsteps` consecutive steps, step j with clock and body transform steps[j] (or
// `sp` when steps is null), keeping the tile's state in registers between them.  RECORD (colour2,
// one step of one substep) additionally writes the step's start state and the iterates to a tape
// for the adjoint (vbd_adjoint.cuh).  HOSTIO steps tile `tile` of a host frame (fused_frame_kernel):
// `stage` holds the tile's positions then velocities from the host buffers of `hio`, 3 floats per
// tile position p = lane * C + k, and the step writes its results back to the host buffers
// through the same area, as well as to the device state.
// EXPLICIT_TILE steps tile `frame_tile` (the persistent kernels' tile loop) instead of the launch's own.
template <int C, bool JACOBI, bool RECORD, bool PAIRED = false, bool HOSTIO = false, bool GROUPED = false,
          bool EXPLICIT_TILE = false>
__device__ __forceinline__ void fused_step_body(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                TapeView tp, const StepParams* __restrict__ steps, int nsteps,
                                                HostIO hio = HostIO{}, int64_t frame_tile = 0, float* stage = nullptr) {
    static_assert(!GROUPED || !PAIRED, "tile groups run the plain step");
    static_assert(!PAIRED || (C == 4 && !JACOBI && !RECORD), "the packed form is the colour2 step with 4 slots per lane");
    static_assert(!(HOSTIO && RECORD), "recorded steps keep their state on the device");
    static_assert(!(RECORD && JACOBI), "the tape records the colour2 schedule");
    static_assert(C % 2 == 0, "slots per lane must be even");
    const int lane = threadIdx.x & 31;
    const int64_t tile = (HOSTIO || EXPLICIT_TILE)
                             ? frame_tile
                             : (RECORD ? tp.tile_begin : 0) + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tile >= st.num_tiles) return;  // uniform per warp (per CTA for groups: num_tiles is a multiple of K)
    const int64_t base = tile * (32LL * C) + lane;
    // tile groups: neighbours across the warps of the CTA (see GroupExchange)
    const int gw = threadIdx.x >> 5, gK = blockDim.x >> 5;
    GroupExchange* gx = nullptr;
    if constexpr (GROUPED) {
        __shared__ GroupExchange group_exchange;
        gx = &group_exchange;
    }
    auto up_put = [&](int slot, float4 v) {
        if (GROUPED && lane == 31) gx->up[gw][slot] = v;
    };
    auto up_get = [&](int slot, float4 v) { return (GROUPED && lane == 0 && gw > 0) ? gx->up[gw - 1][slot] : v; };
    auto down_put = [&](int slot, float4 v) {
        if (GROUPED && lane == 0) gx->down[gw][slot] = v;
    };
    auto down_get = [&](int slot, float4 v) { return (GROUPED && lane == 31 && gw < gK - 1) ? gx->down[gw + 1][slot] : v; };
    auto group_sync = [&]() {
        if (GROUPED) __syncthreads();
    };
    auto f4 = [](float3 a) { return make_float4(a.x, a.y, a.z, 0.f); };

    float3 x[C], v[C], vl[C], dx[C], d3[C], F0[C], Ve[C];
    float4 q[C], qr[C];
    float im[C], invl[C], kk[C], ddN[C], kkN[C], as_[C], isA[C], isD[C];
    uint32_t fl[C];
    bool mov[C];  // the vertex's position is updated (not pinned, not padding)

#pragma unroll
    for (int k = 0; k < C; k++) {
        const int64_t g = base + 32LL * k;
        const float4 a = st.xm[g];
        x[k] = xyz(a);
        im[k] = a.w;
        v[k] = xyz(st.vel[g]);
        vl[k] = xyz(st.vlast[g]);
        q[k] = st.q[g];
        qr[k] = st.qr[g];
        const float4 p = st.prm[g];
        invl[k] = 1.f / p.x;
        kk[k] = p.y * invl[k];
        fl[k] = __float_as_uint(p.w);
        mov[k] = im[k] != 0.f;
        ddN[k] = (fl[k] & F_HAS_NEXT) ? kk[k] * invl[k] : 0.f;
        kkN[k] = (fl[k] & F_HAS_NEXT) ? kk[k] : 0.f;
    }
    float* const sx = stage;
    float* const sv = stage + 3 * 32 * C;
    if (HOSTIO && hio.x_in) {  // (no input buffers: the frame starts from the device state)
#pragma unroll
        for (int k = 0; k < C; k++) {
            if (fl[k] & F_VALID) {  // padding slots keep their device values
                const int o = 3 * (lane * C + k);
                x[k] = f3(sx[o], sx[o + 1], sx[o + 2]);
                v[k] = f3(sv[o], sv[o + 1], sv[o + 2]);
            }
        }
        __syncwarp();
    }
    const int64_t tS = tp.slots;
    const int64_t tslot = base - (RECORD ? tp.tile_begin * 32LL * C : 0);  // this lane's slot in the tape window
    const int64_t tbase = ((int64_t)tp.step * (tp.num_itr + 1)) * tS + tslot;  // tape row of iteration 0
    if (RECORD) {
#pragma unroll
        for (int k = 0; k < C; k++) {
            const int64_t o = (int64_t)tp.step * tS + tslot + 32LL * k;
            tp.x[o] = make_float4(x[k].x, x[k].y, x[k].z, im[k]);
            tp.v[o] = make_float4(v[k].x, v[k].y, v[k].z, 0.f);
            tp.vl[o] = make_float4(vl[k].x, vl[k].y, vl[k].z, 0.f);
        }
    }
    // constants of the previous lane's last segment (segment i-1 of slot 0)
    float4 qrH = shfl_up4(qr[C - 1], 1);
    float ddH = __shfl_up_sync(0xffffffffu, ddN[C - 1], 1);
    float kkH = __shfl_up_sync(0xffffffffu, kkN[C - 1], 1);
    if (GROUPED) {
        up_put(XU_QR, qr[C - 1]);
        up_put(XU_DK, make_float4(ddN[C - 1], kkN[C - 1], 0.f, 0.f));
        group_sync();
        qrH = up_get(XU_QR, qrH);
        const float4 dk = up_get(XU_DK, make_float4(ddH, kkH, 0.f, 0.f));
        ddH = dk.x;
        kkH = dk.y;
    }

    const float accel = pp.accel_ratio;
    bool bad = false;
    for (int step = 0; step < nsteps; step++) {
    if (steps) sp = steps[step];
    const float h = sp.h;
    const float damp = pp.damping / h;

    for (int s = 0; s < sp.substeps; s++) {
        {
            float3 e[C];
#pragma unroll
            for (int k = 0; k < C - 1; k++) e[k] = x[k + 1] - x[k];
            float3 xN0 = shfl_down3(x[0], 1);
            if (GROUPED) {
                down_put(XD_X, f4(x[0]));
                group_sync();
                xN0 = xyz(down_get(XD_X, f4(xN0)));
            }
            e[C - 1] = xN0 - x[C - 1];
#pragma unroll
            for (int k = 0; k < C; k++) e[k] = (fl[k] & F_HAS_NEXT) ? e[k] : f3(0.f, 0.f, 0.f);
            float3 eH = shfl_up3(e[C - 1], 1);
            if (GROUPED) {
                up_put(XU_E, f4(e[C - 1]));
                group_sync();
                eH = xyz(up_get(XU_E, f4(eH)));
            }
#pragma unroll
            for (int k = 0; k < C; k++) {
                float3 y;
                vbd_predict(x[k], v[k], vl[k], im[k], pp, h, sp.last_h, sp.time, dx[k], y);
                vl[k] = v[k];
                const float ddP = k > 0 ? ddN[k > 0 ? k - 1 : 0] : ddH;
                const float3 eP = k > 0 ? e[k > 0 ? k - 1 : 0] : eH;
                const float a = im[k] != 0.f ? 1.f / (im[k] * h * h) : 0.f;
                const float sk = (ddN[k] + ddP) * (1.f + damp);
                as_[k] = a + sk;
                isA[k] = im[k] != 0.f ? accel / sk : 0.f;
                isD[k] = im[k] != 0.f ? accel / (sk + 3.f * a) - isA[k] : 0.f;
                F0[k] = a * y + ddN[k] * e[k] - ddP * eP;
                Ve[k] = (-2.f * kk[k]) * e[k];
                d3[k] = d3_of(q[k]);
            }
        }
        float4 qP = shfl_up4(q[C - 1], 1);
        float3 d3P = shfl_up3(d3[C - 1], 1);  // the previous lane's d3_of(qP)
        if (RECORD) {
#pragma unroll
            for (int k = 0; k < C; k++) {
                tp.dx[tbase + 32LL * k] = make_float4(dx[k].x, dx[k].y, dx[k].z, 0.f);
                tp.q[tbase + 32LL * k] = q[k];
            }
        }

        if constexpr (PAIRED) {
            // pairs of same-colour slots: A = {0, 2}, B = {1, 3}.  A's neighbours are B's slots
            // (and the previous lane's slot 3 for slot 0); B's are A's (and the next lane's slot 0
            // for slot 3).
            F2x3 dxA = pack3(dx[0], dx[2]), dxB = pack3(dx[1], dx[3]);
            F2x4 qA = pack4(q[0], q[2]), qB = pack4(q[1], q[3]);
            F2x3 d3A = pack3(d3[0], d3[2]), d3B = pack3(d3[1], d3[3]);
            const F2x3 F0A = pack3(F0[0], F0[2]), F0B = pack3(F0[1], F0[3]);
            const F2x3 VeA = pack3(Ve[0], Ve[2]), VeB = pack3(Ve[1], Ve[3]);
            const float2 ddNA = make_float2(ddN[0], ddN[2]), ddNB = make_float2(ddN[1], ddN[3]);
            const float2 nkkNA = make_float2(-kkN[0], -kkN[2]), nkkNB = make_float2(-kkN[1], -kkN[3]);
            const float2 ddPA = make_float2(ddH, ddN[1]), kkPA = make_float2(kkH, kkN[1]);
            const float2 kkPB = make_float2(kkN[0], kkN[2]);
            const float2 nasA = make_float2(-as_[0], -as_[2]), nasB = make_float2(-as_[1], -as_[3]);
            const float2 isAA = make_float2(isA[0], isA[2]), isAB = make_float2(isA[1], isA[3]);
            const float2 isDA = make_float2(isD[0], isD[2]), isDB = make_float2(isD[1], isD[3]);
            const float2 m2kA = make_float2(-2.f * kk[0], -2.f * kk[2]), m2kB = make_float2(-2.f * kk[1], -2.f * kk[3]);
            const F2x4 qrA = pack4(qr[0], qr[2]), qrB = pack4(qr[1], qr[3]), qrPA = pack4(qrH, qr[1]);
            bool hnA[2], hpA[2], mvA[2], uoA[2], nxA[2], hnB[2], hpB[2], mvB[2], uoB[2], nxB[2];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const uint32_t fa = fl[2 * j], fb = fl[2 * j + 1];
                hnA[j] = fa & F_HAS_NEXT;
                hpA[j] = fa & F_HAS_PREV;
                mvA[j] = mov[2 * j];
                uoA[j] = (fa & F_HAS_NEXT) && !(fa & F_FIX_ORIENTATION);
                nxA[j] = fa & F_HAS_NEXT_ORIENTATION;
                hnB[j] = fb & F_HAS_NEXT;
                hpB[j] = fb & F_HAS_PREV;
                mvB[j] = mov[2 * j + 1];
                uoB[j] = (fb & F_HAS_NEXT) && !(fb & F_FIX_ORIENTATION);
                nxB[j] = fb & F_HAS_NEXT_ORIENTATION;
            }
            for (int it = 0; it < pp.num_itr; it++) {
                // positions, even slots
                const F2x3 dxPA = pack3(shfl_up3(hi3(dxB), 1), lo3(dxB));
                const F2x3 d3PA = pack3(shfl_up3(hi3(d3B), 1), lo3(d3B));
                dxA = fused_position2(dxA, F0A, ddNA, nkkNA, d3A, dxB, ddPA, kkPA, d3PA, dxPA, nasA, isAA, isDA, hnA,
                                      hpA, mvA, false, true);
                // positions, odd slots
                const F2x3 dxNB = pack3(hi3(dxA), shfl_down3(lo3(dxA), 1));
                dxB = fused_position2(dxB, F0B, ddNB, nkkNB, d3B, dxNB, ddNA, kkPB, d3A, dxA, nasB, isAB, isDB, hnB, hpB,
                                      mvB, true, false);
                // orientations, even segments
                const F2x4 qPA = pack4(shfl_up4(hi4(qB), 1), lo4(qB));
                qA = fused_orientation2(qA, uoA, hpA, nxA, VeA, m2kA, dxA, dxB, qPA, qrPA, qB, qrA, true, false);
                d3A = d3_of2(qA);
                // orientations, odd segments
                const F2x4 qNB = pack4(hi4(qA), shfl_down4(lo4(qA), 1));
                qB = fused_orientation2(qB, uoB, hpB, nxB, VeB, m2kB, dxB, dxNB, qA, qrA, qNB, qrB, false, true);
                d3B = d3_of2(qB);
            }
            dx[0] = lo3(dxA);
            dx[2] = hi3(dxA);
            dx[1] = lo3(dxB);
            dx[3] = hi3(dxB);
            q[0] = lo4(qA);
            q[2] = hi4(qA);
            q[1] = lo4(qB);
            q[3] = hi4(qB);
        } else {  // (braced: an unbraced discarded `else for` also dropped the loop after it)
        for (int it = 0; it < pp.num_itr; it++) {
            if (!JACOBI) {
                float3 dxP = shfl_up3(dx[C - 1], 1);
                if (GROUPED) {  // the previous lane's odd values, unchanged until the odd sweeps
                    up_put(XU_DX, f4(dx[C - 1]));
                    up_put(XU_Q, q[C - 1]);
                    up_put(XU_D3, f4(d3[C - 1]));
                    group_sync();
                    dxP = xyz(up_get(XU_DX, f4(dxP)));
                    qP = up_get(XU_Q, qP);
                    d3P = xyz(up_get(XU_D3, f4(d3P)));
                }
                // positions, even slots (neighbours are odd: own registers or the previous lane)
                {
#pragma unroll
                    for (int k = 0; k < C; k += 2) {
                        const int kp = k > 0 ? k - 1 : 0;
                        dx[k] = fused_position(dx[k], F0[k], ddN[k], kkN[k], d3[k], dx[k + 1], k ? ddN[kp] : ddH,
                                               k ? kkN[kp] : kkH, k ? d3[kp] : d3P, k ? dx[kp] : dxP, as_[k], isA[k],
                                               isD[k], fl[k] & F_HAS_NEXT, fl[k] & F_HAS_PREV, mov[k], false, true);
                    }
                }
                // positions, odd slots
                float3 dxN0 = shfl_down3(dx[0], 1);
                if (GROUPED) {
                    down_put(XD_DX, f4(dx[0]));
                    group_sync();
                    dxN0 = xyz(down_get(XD_DX, f4(dxN0)));
                }
#pragma unroll
                for (int k = 1; k < C; k += 2) {
                    const int kn = k + 1 < C ? k + 1 : k;
                    dx[k] = fused_position(dx[k], F0[k], ddN[k], kkN[k], d3[k], k == C - 1 ? dxN0 : dx[kn], ddN[k - 1],
                                           kkN[k - 1], d3[k - 1], dx[k - 1], as_[k], isA[k], isD[k],
                                           fl[k] & F_HAS_NEXT, fl[k] & F_HAS_PREV, mov[k], true, false);
                }
                // orientations, even segments
#pragma unroll
                for (int k = 0; k < C; k += 2) {
                    const int kp = k > 0 ? k - 1 : 0;
                    const uint32_t f = fl[k];
                    q[k] = fused_orientation(q[k], (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION), f & F_HAS_PREV,
                                             f & F_HAS_NEXT_ORIENTATION, Ve[k], -2.f * kk[k], dx[k], dx[k + 1],
                                             k ? q[kp] : qP, k ? qr[kp] : qrH, q[k + 1], qr[k], true, false);
                    d3[k] = d3_of(q[k]);
                }
                // orientations, odd segments
                float4 qN0 = shfl_down4(q[0], 1);
                if (GROUPED) {
                    down_put(XD_Q, q[0]);
                    group_sync();
                    qN0 = down_get(XD_Q, qN0);
                }
#pragma unroll
                for (int k = 1; k < C; k += 2) {
                    const int kn = k + 1 < C ? k + 1 : k;
                    const uint32_t f = fl[k];
                    q[k] = fused_orientation(q[k], (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION), f & F_HAS_PREV,
                                             f & F_HAS_NEXT_ORIENTATION, Ve[k], -2.f * kk[k], dx[k],
                                             k == C - 1 ? dxN0 : dx[kn], q[k - 1], qr[k - 1],
                                             k == C - 1 ? qN0 : q[kn], qr[k], false, true);
                    d3[k] = d3_of(q[k]);
                }
                qP = shfl_up4(q[C - 1], 1);
                d3P = shfl_up3(d3[C - 1], 1);
                if (RECORD) {
                    const int64_t row = tbase + (int64_t)(it + 1) * tS;
#pragma unroll
                    for (int k = 0; k < C; k++) {
                        tp.dx[row + 32LL * k] = make_float4(dx[k].x, dx[k].y, dx[k].z, 0.f);
                        tp.q[row + 32LL * k] = q[k];
                    }
                }
            } else {
                // positions, every slot from the previous sweep
                float3 dxP = shfl_up3(dx[C - 1], 1);
                float3 dxN0 = shfl_down3(dx[0], 1);
                if (GROUPED) {
                    up_put(XU_DX, f4(dx[C - 1]));
                    up_put(XU_Q, q[C - 1]);
                    up_put(XU_D3, f4(d3[C - 1]));
                    down_put(XD_DX, f4(dx[0]));
                    group_sync();
                    dxP = xyz(up_get(XU_DX, f4(dxP)));
                    qP = up_get(XU_Q, qP);
                    d3P = xyz(up_get(XU_D3, f4(d3P)));
                    dxN0 = xyz(down_get(XD_DX, f4(dxN0)));
                }
                float3 nd[C];
#pragma unroll
                for (int k = 0; k < C; k++) {
                    const int kp = k > 0 ? k - 1 : 0, kn = k + 1 < C ? k + 1 : k;
                    nd[k] = fused_position(dx[k], F0[k], ddN[k], kkN[k], d3[k], k == C - 1 ? dxN0 : dx[kn],
                                           k ? ddN[kp] : ddH, k ? kkN[kp] : kkH, k ? d3[kp] : d3P, k ? dx[kp] : dxP,
                                           as_[k], isA[k], isD[k], fl[k] & F_HAS_NEXT, fl[k] & F_HAS_PREV, mov[k],
                                           (k & 1) != 0, (k & 1) == 0);
                }
#pragma unroll
                for (int k = 0; k < C; k++) dx[k] = nd[k];
                // orientations, every segment from the previous sweep
                float3 dxN1 = shfl_down3(dx[0], 1);
                float4 qN0 = shfl_down4(q[0], 1);
                if (GROUPED) {
                    down_put(XD_DX2, f4(dx[0]));
                    down_put(XD_Q, q[0]);
                    group_sync();
                    dxN1 = xyz(down_get(XD_DX2, f4(dxN1)));
                    qN0 = down_get(XD_Q, qN0);
                }
                float4 nq[C];
#pragma unroll
                for (int k = 0; k < C; k++) {
                    const int kp = k > 0 ? k - 1 : 0, kn = k + 1 < C ? k + 1 : k;
                    const uint32_t f = fl[k];
                    nq[k] = fused_orientation(q[k], (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION), f & F_HAS_PREV,
                                              f & F_HAS_NEXT_ORIENTATION, Ve[k], -2.f * kk[k], dx[k],
                                              k == C - 1 ? dxN1 : dx[kn], k ? q[kp] : qP, k ? qr[kp] : qrH,
                                              k == C - 1 ? qN0 : q[kn], qr[k], (k & 1) == 0, (k & 1) != 0);
                }
#pragma unroll
                for (int k = 0; k < C; k++) {
                    q[k] = nq[k];
                    d3[k] = d3_of(q[k]);
                }
                qP = shfl_up4(q[C - 1], 1);
                d3P = shfl_up3(d3[C - 1], 1);
            }
        }
        }  // scalar iterations
#pragma unroll
        for (int k = 0; k < C; k++) vbd_finish(x[k], v[k], dx[k], im[k], h, pp.velocity_decay);
    }
#pragma unroll
    for (int k = 0; k < C; k++) {
        if (sdf.grid && (fl[k] & F_VALID) && !(fl[k] & F_ROOT)) vbd_sdf(x[k], v[k], sdf, sp);
        bad |= !finite3(x[k]) || !finite3(v[k]) || !finite4(q[k]);
    }
    }  // steps

#pragma unroll
    for (int k = 0; k < C; k++) {
        const int64_t g = base + 32LL * k;
        st.xm[g] = make_float4(x[k].x, x[k].y, x[k].z, im[k]);
        st.vel[g] = make_float4(v[k].x, v[k].y, v[k].z, 0.f);
        st.vlast[g] = make_float4(vl[k].x, vl[k].y, vl[k].z, 0.f);
        st.q[g] = q[k];
    }
    if (HOSTIO && hio.x_out) {  // (no output buffers: the results stay on the device)
#pragma unroll
        for (int k = 0; k < C; k++) {
            const int o = 3 * (lane * C + k);
            sx[o] = x[k].x;
            sx[o + 1] = x[k].y;
            sx[o + 2] = x[k].z;
            sv[o] = v[k].x;
            sv[o + 1] = v[k].y;
            sv[o + 2] = v[k].z;
        }
        __syncwarp();
        const int r_end = hio.run_begin[tile + 1];
        for (int r = hio.run_begin[tile]; r < r_end; r++) {
            const int4 run = hio.runs[r];
            float* gx = hio.x_out + 3LL * run.y;
            float* gv = hio.v_out + 3LL * run.y;
            for (int j = lane; j < 3 * run.z; j += 32) {
                gx[j] = sx[3 * run.x + j];
                gv[j] = sv[3 * run.x + j];
            }
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(st.status, STATUS_NONFINITE);
}

template <int C, bool JACOBI, bool RECORD>
__global__ void __launch_bounds__(256) fused_step_kernel(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                         TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, RECORD>(st, pp, sp, sdf, tp, steps, nsteps);
}

// The colour2 step with 4 slots per lane in the packed FP32x2 form (the `x2` kernel variant).
template <int C>
__global__ void __launch_bounds__(256) fused_step_kernel_x2(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                            TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, false, false, true>(st, pp, sp, sdf, tp, steps, nsteps);
}

// ---- host frames: one launch uploads, steps and downloads ---------------------------------------------

// One upload-step-download frame in one launch: each warp copies its tile's strands from the host
// buffers into its staging area (6 * 32C floats of dynamic shared memory; coalesced 4-byte loads
// over PCIe), steps the tile and writes it back (fused_step_body, HOSTIO).  The waves of tiles keep
// the host reads of one wave apart from the host writes of the wave before, which is faster here
// than interleaving them: SM-issued reads and writes over PCIe slow each other down.
template <int C, bool JACOBI, bool PAIRED, bool GROUPED = false>
__device__ __forceinline__ void fused_frame(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf, HostIO hio) {
    extern __shared__ float kami_frame_stage[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + w;
    if (t >= st.num_tiles) return;  // uniform per warp (per CTA for groups)
    float* const stage = kami_frame_stage + w * (6 * 32 * C);
    const int r_end = hio.x_in ? hio.run_begin[t + 1] : 0;
    for (int r = hio.run_begin[t]; r < r_end; r++) {
        const int4 run = hio.runs[r];
        const float* gx = hio.x_in + 3LL * run.y;
        const float* gv = hio.v_in + 3LL * run.y;
        for (int j = lane; j < 3 * run.z; j += 32) {
            stage[3 * run.x + j] = gx[j];
            stage[3 * 32 * C + 3 * run.x + j] = gv[j];
        }
    }
    __syncwarp();
    fused_step_body<C, JACOBI, false, PAIRED, true, GROUPED>(st, pp, sp, sdf, TapeView{}, nullptr, 1, hio, t, stage);
}
template <int C, bool JACOBI, bool PAIRED>
__global__ void __launch_bounds__(256) fused_frame_kernel(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                          HostIO hio) {
    fused_frame<C, JACOBI, PAIRED>(st, pp, sp, sdf, hio);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(120) fused_frame_kernel_r120(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                        HostIO hio) {
    fused_frame<C, JACOBI, false>(st, pp, sp, sdf, hio);
}
// The same over groups of tiles: one CTA of K warps per group.
template <int C, bool JACOBI>
__global__ void __launch_bounds__(256) fused_frame_group_kernel(DeviceState st, PhysParams pp, StepParams sp,
                                                                SdfParams sdf, HostIO hio) {
    fused_frame<C, JACOBI, false, true>(st, pp, sp, sdf, hio);
}

// The step with 4 slots per lane at most 168 registers per thread (a few bytes of spills): 12 instead
// of 8 warps share an SM, which hides more of the colour sweeps' dependency latency.
template <int C, bool JACOBI>
__global__ void __maxnreg__(168) fused_step_kernel_r168(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                       TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, false>(st, pp, sp, sdf, tp, steps, nsteps);
}

// The step over groups of K tiles (strands longer than a tile): one CTA of K warps per group, plain
// and with the register caps of the single-tile variants.
template <int C, bool JACOBI>
__global__ void __launch_bounds__(256) fused_group_kernel(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                          const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, false, false, false, true>(st, pp, sp, sdf, TapeView{}, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(120) fused_group_kernel_r120(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                        const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, false, false, false, true>(st, pp, sp, sdf, TapeView{}, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(168) fused_group_kernel_r168(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                        const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, false, false, false, true>(st, pp, sp, sdf, TapeView{}, steps, nsteps);
}

// The recorded step (kami_vbd_step_record) over groups of tiles: one CTA of K warps per group.
template <int C>
__global__ void __launch_bounds__(256) fused_record_group_kernel(DeviceState st, PhysParams pp, StepParams sp,
                                                                 SdfParams sdf, TapeView tp) {
    fused_step_body<C, false, true, false, false, true>(st, pp, sp, sdf, tp, nullptr, 1);
}

// The same step with at most 120 registers per thread, so 17 warps (instead of 16) share an SM: a
// launch whose tile count is just above a multiple of 16 warps per SM then needs one wave less.
template <int C, bool JACOBI>
__global__ void __maxnreg__(120) fused_step_kernel_r120(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                       TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, false>(st, pp, sp, sdf, tp, steps, nsteps);
}

// ---- persistent form ----------------------------------------------------------------------------
// A grid of at most as many CTAs as stay resident: CTA b's warp w steps tiles u * W + w for
// u = b, b + gridDim.x, ... (W warps per CTA), or, for groups of K tiles (GROUPED, W = K), the groups
// b, b + gridDim.x, ...  With the grid at the resident count, the SMs' shares differ by one unit.
template <int C, bool JACOBI, bool GROUPED>
__device__ __forceinline__ void fused_persistent(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                 const StepParams* __restrict__ steps, int nsteps) {
    // only the 32-bit unit index stays live across the step body (register pressure)
    for (int u = blockIdx.x; (int64_t)u * (blockDim.x >> 5) < st.num_tiles; u += gridDim.x) {
        fused_step_body<C, JACOBI, false, false, false, GROUPED, true>(
            st, pp, sp, sdf, TapeView{}, steps, nsteps, HostIO{}, (int64_t)u * (blockDim.x >> 5) + (threadIdx.x >> 5));
        if (GROUPED) __syncthreads();  // the group exchange area is reused by the next group
    }
}
template <int C, bool JACOBI>
__global__ void __launch_bounds__(256) fused_persistent_kernel(DeviceState st, PhysParams pp, StepParams sp,
                                                               SdfParams sdf, const StepParams* __restrict__ steps,
                                                               int nsteps) {
    fused_persistent<C, JACOBI, false>(st, pp, sp, sdf, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(120) fused_persistent_kernel_r120(DeviceState st, PhysParams pp, StepParams sp,
                                                              SdfParams sdf, const StepParams* __restrict__ steps,
                                                              int nsteps) {
    fused_persistent<C, JACOBI, false>(st, pp, sp, sdf, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(168) fused_persistent_kernel_r168(DeviceState st, PhysParams pp, StepParams sp,
                                                              SdfParams sdf, const StepParams* __restrict__ steps,
                                                              int nsteps) {
    fused_persistent<C, JACOBI, false>(st, pp, sp, sdf, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __launch_bounds__(256) fused_persistent_group_kernel(DeviceState st, PhysParams pp, StepParams sp,
                                                                     SdfParams sdf, const StepParams* __restrict__ steps,
                                                                     int nsteps) {
    fused_persistent<C, JACOBI, true>(st, pp, sp, sdf, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(120) fused_persistent_group_kernel_r120(DeviceState st, PhysParams pp, StepParams sp,
                                                                    SdfParams sdf,
                                                                    const StepParams* __restrict__ steps, int nsteps) {
    fused_persistent<C, JACOBI, true>(st, pp, sp, sdf, steps, nsteps);
}
template <int C, bool JACOBI>
__global__ void __maxnreg__(168) fused_persistent_group_kernel_r168(DeviceState st, PhysParams pp, StepParams sp,
                                                                    SdfParams sdf,
                                                                    const StepParams* __restrict__ steps, int nsteps) {
    fused_persistent<C, JACOBI, true>(st, pp, sp, sdf, steps, nsteps);
}

}  // namespace kami
