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
//   then dx += (f - mean f) accel/s + mean f accel/(s + 3a)   (the exact inverse of a 1 1^T + s I);
//   orientation (quaternionLambdaItr, cosserat.cu:290-337) with V = -2 kk (e_i + dx_next - dx).
// Missing neighbours enter as zero coefficients or are discarded by selects, so the iteration
// loop has no data-dependent branches.
#pragma once
#include "vbd_math.cuh"

namespace kami {

__device__ __forceinline__ float sqrt_nonneg(float x) { return x * rsqrtf(fmaxf(x, 1e-30f)); }

// One position update with folded coefficients (see the file comment).  Neighbour operands from
// another strand (no segment in between: hn / hp false) are replaced by the vertex's own values
// before they meet their zero coefficient, and vertices that do not move (upd false) keep dx, so a
// non-finite strand cannot leak into the strands or padding that share its tile, as the
// reference's flag tests guarantee.
__device__ __forceinline__ float3 fused_position(float3 dx, float3 F0, float ddN, float kkN, float3 d3N, float3 dxN,
                                                 float ddP, float kkP, float3 d3P, float3 dxP, float as_, float isA,
                                                 float isB, bool hn, bool hp, bool upd) {
    dxN = hn ? dxN : dx;
    dxP = hp ? dxP : dx;
    d3P = hp ? d3P : d3N;
    float3 f;
    f.x = F0.x + ddN * dxN.x + ddP * dxP.x - as_ * dx.x - kkN * d3N.x + kkP * d3P.x;
    f.y = F0.y + ddN * dxN.y + ddP * dxP.y - as_ * dx.y - kkN * d3N.y + kkP * d3P.y;
    f.z = F0.z + ddN * dxN.z + ddP * dxP.z - as_ * dx.z - kkN * d3N.z + kkP * d3P.z;
    const float m = (f.x + f.y + f.z) * (1.f / 3.f);
    const float mb = m * isB;
    const float3 n = f3(dx.x + (f.x - m) * isA + mb, dx.y + (f.y - m) * isA + mb, dx.z + (f.z - m) * isA + mb);
    return upd ? n : dx;
}

// One orientation update (quaternionLambdaItr), branch-free: pre/nxt say whether the previous /
// next segment exists, upd whether this segment is updated at all.
__device__ __forceinline__ float4 fused_orientation(float4 q, bool upd, bool pre, bool nxt, float3 Ve, float m2k,
                                                    float3 dx, float3 dxN, float4 qPrev, float4 qrPrev, float4 qNext,
                                                    float4 qr) {
    const float3 V = Ve + m2k * (dxN - dx);
    qPrev = pre ? qPrev : q;  // operands from another strand never meet arithmetic
    qNext = nxt ? qNext : q;
    const float4 P1 = qmul(qPrev, qrPrev);
    const float4 P2 = qmul_conj(qNext, qr);
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
    const float4 n = scale4(rsqrtf(dot4(R, R)), R);
    return upd ? n : q;
}

// One launch runs `nsteps` consecutive steps, step j with clock and body transform steps[j] (or
// `sp` when steps is null), keeping the tile's state in registers between them.  RECORD (colour2,
// one step of one substep) additionally writes the step's start state and the iterates to a tape
// for the adjoint (vbd_adjoint.cuh).
template <int C, bool JACOBI, bool RECORD>
__device__ __forceinline__ void fused_step_body(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    static_assert(!(RECORD && JACOBI), "the tape records the colour2 schedule");
    static_assert(C % 2 == 0, "slots per lane must be even");
    const int lane = threadIdx.x & 31;
    const int64_t tile = (RECORD ? tp.tile_begin : 0) + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tile >= st.num_tiles) return;  // uniform per warp
    const int64_t base = tile * (32LL * C) + lane;

    float3 x[C], v[C], vl[C], dx[C], d3[C], F0[C], Ve[C];
    float4 q[C], qr[C];
    float im[C], invl[C], kk[C], ddN[C], kkN[C], as_[C], isA[C], isB[C];
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
    const float4 qrH = shfl_up4(qr[C - 1], 1);
    const float ddH = __shfl_up_sync(0xffffffffu, ddN[C - 1], 1);
    const float kkH = __shfl_up_sync(0xffffffffu, kkN[C - 1], 1);

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
            e[C - 1] = shfl_down3(x[0], 1) - x[C - 1];
#pragma unroll
            for (int k = 0; k < C; k++) e[k] = (fl[k] & F_HAS_NEXT) ? e[k] : f3(0.f, 0.f, 0.f);
            const float3 eH = shfl_up3(e[C - 1], 1);
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
                isB[k] = im[k] != 0.f ? accel / (sk + 3.f * a) : 0.f;
                F0[k] = a * y + ddN[k] * e[k] - ddP * eP;
                Ve[k] = (-2.f * kk[k]) * e[k];
                d3[k] = d3_of(q[k]);
            }
        }
        float4 qP = shfl_up4(q[C - 1], 1);
        float3 d3P = d3_of(qP);
        if (RECORD) {
#pragma unroll
            for (int k = 0; k < C; k++) {
                tp.dx[tbase + 32LL * k] = make_float4(dx[k].x, dx[k].y, dx[k].z, 0.f);
                tp.q[tbase + 32LL * k] = q[k];
            }
        }

        for (int it = 0; it < pp.num_itr; it++) {
            if (!JACOBI) {
                // positions, even slots (neighbours are odd: own registers or the previous lane)
                {
                    const float3 dxP = shfl_up3(dx[C - 1], 1);
#pragma unroll
                    for (int k = 0; k < C; k += 2) {
                        const int kp = k > 0 ? k - 1 : 0;
                        dx[k] = fused_position(dx[k], F0[k], ddN[k], kkN[k], d3[k], dx[k + 1], k ? ddN[kp] : ddH,
                                               k ? kkN[kp] : kkH, k ? d3[kp] : d3P, k ? dx[kp] : dxP, as_[k], isA[k],
                                               isB[k], fl[k] & F_HAS_NEXT, fl[k] & F_HAS_PREV, mov[k]);
                    }
                }
                // positions, odd slots
                const float3 dxN0 = shfl_down3(dx[0], 1);
#pragma unroll
                for (int k = 1; k < C; k += 2) {
                    const int kn = k + 1 < C ? k + 1 : k;
                    dx[k] = fused_position(dx[k], F0[k], ddN[k], kkN[k], d3[k], k == C - 1 ? dxN0 : dx[kn], ddN[k - 1],
                                           kkN[k - 1], d3[k - 1], dx[k - 1], as_[k], isA[k], isB[k],
                                           fl[k] & F_HAS_NEXT, fl[k] & F_HAS_PREV, mov[k]);
                }
                // orientations, even segments
#pragma unroll
                for (int k = 0; k < C; k += 2) {
                    const int kp = k > 0 ? k - 1 : 0;
                    const uint32_t f = fl[k];
                    q[k] = fused_orientation(q[k], (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION), f & F_HAS_PREV,
                                             f & F_HAS_NEXT_ORIENTATION, Ve[k], -2.f * kk[k], dx[k], dx[k + 1],
                                             k ? q[kp] : qP, k ? qr[kp] : qrH, q[k + 1], qr[k]);
                    d3[k] = d3_of(q[k]);
                }
                // orientations, odd segments
                const float4 qN0 = shfl_down4(q[0], 1);
#pragma unroll
                for (int k = 1; k < C; k += 2) {
                    const int kn = k + 1 < C ? k + 1 : k;
                    const uint32_t f = fl[k];
                    q[k] = fused_orientation(q[k], (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION), f & F_HAS_PREV,
                                             f & F_HAS_NEXT_ORIENTATION, Ve[k], -2.f * kk[k], dx[k],
                                             k == C - 1 ? dxN0 : dx[kn], q[k - 1], qr[k - 1],
                                             k == C - 1 ? qN0 : q[kn], qr[k]);
                    d3[k] = d3_of(q[k]);
                }
                qP = shfl_up4(q[C - 1], 1);
                d3P = d3_of(qP);
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
                const float3 dxP = shfl_up3(dx[C - 1], 1);
                const float3 dxN0 = shfl_down3(dx[0], 1);
                float3 nd[C];
#pragma unroll
                for (int k = 0; k < C; k++) {
                    const int kp = k > 0 ? k - 1 : 0, kn = k + 1 < C ? k + 1 : k;
                    nd[k] = fused_position(dx[k], F0[k], ddN[k], kkN[k], d3[k], k == C - 1 ? dxN0 : dx[kn],
                                           k ? ddN[kp] : ddH, k ? kkN[kp] : kkH, k ? d3[kp] : d3P, k ? dx[kp] : dxP,
                                           as_[k], isA[k], isB[k], fl[k] & F_HAS_NEXT, fl[k] & F_HAS_PREV, mov[k]);
                }
#pragma unroll
                for (int k = 0; k < C; k++) dx[k] = nd[k];
                // orientations, every segment from the previous sweep
                const float3 dxN1 = shfl_down3(dx[0], 1);
                const float4 qN0 = shfl_down4(q[0], 1);
                float4 nq[C];
#pragma unroll
                for (int k = 0; k < C; k++) {
                    const int kp = k > 0 ? k - 1 : 0, kn = k + 1 < C ? k + 1 : k;
                    const uint32_t f = fl[k];
                    nq[k] = fused_orientation(q[k], (f & F_HAS_NEXT) && !(f & F_FIX_ORIENTATION), f & F_HAS_PREV,
                                              f & F_HAS_NEXT_ORIENTATION, Ve[k], -2.f * kk[k], dx[k],
                                              k == C - 1 ? dxN1 : dx[kn], k ? q[kp] : qP, k ? qr[kp] : qrH,
                                              k == C - 1 ? qN0 : q[kn], qr[k]);
                }
#pragma unroll
                for (int k = 0; k < C; k++) {
                    q[k] = nq[k];
                    d3[k] = d3_of(q[k]);
                }
                qP = shfl_up4(q[C - 1], 1);
                d3P = d3_of(qP);
            }
        }
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
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(st.status, STATUS_NONFINITE);
}

template <int C, bool JACOBI, bool RECORD>
__global__ void __launch_bounds__(256) fused_step_kernel(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                         TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, RECORD>(st, pp, sp, sdf, tp, steps, nsteps);
}

// The same step with at most 120 registers per thread, so 17 warps (instead of 16) share an SM: a
// launch whose tile count is just above a multiple of 16 warps per SM then needs one wave less.
template <int C, bool JACOBI>
__global__ void __maxnreg__(120) fused_step_kernel_r120(DeviceState st, PhysParams pp, StepParams sp, SdfParams sdf,
                                                       TapeView tp, const StepParams* __restrict__ steps, int nsteps) {
    fused_step_body<C, JACOBI, false>(st, pp, sp, sdf, tp, steps, nsteps);
}

}  // namespace kami
