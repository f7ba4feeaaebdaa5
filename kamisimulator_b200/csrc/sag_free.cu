// sag_free.cu -- sag-free initialisation on the GPU: Sim::SagFree / SingleSagFree
// (YarnBall/YBSimulator.cu:480-674), which the reference runs on the host strand after strand.
// Strands are independent, so one thread takes one strand and walks it twice with the
// reference's float / double mix:
//   1. tip to root, each segment's rest length becomes the root of the quadratic that cancels the
//      stretch force of the mass below it (the root nearer the old length; 1.5 x when there is
//      none; clamped to [1e-6, 1.5 x]);
//   2. root to tip, each segment's orientation turns, in the plane of its axis and the bending
//      force, to the angle whose bending torque cancels that force's torque (bracketed within
//      1e-4 rad of the force's direction); the turns accumulate towards the tip and the previous
//      segment's rest Darboux is re-aimed keeping its magnitude (the bend/twist stiffness).
// Positions do not change.  Part 1's stretch forces, which part 2 needs, go through `fs`, one
// float per slot.
#include "vbd_kernels.h"

namespace kami {
namespace {

__device__ __forceinline__ double sag_fmod(double x, double y) {  // my_fmod, YBSimulator.cu:59-72 (in double here)
    return y != 0 ? x - (double)(long long)(x / y) * y : 0.0;
}
__device__ __forceinline__ double fit_angle(double a) {  // fitAngle, YBSimulator.cu:74-79
    const double pi = 3.141592653589793238462643, two_pi = 6.2831853071795864769252867665590057683943;
    return sag_fmod(sag_fmod(a + pi, two_pi) + two_pi, two_pi) - pi;
}
__device__ __forceinline__ double sgn(double x) { return (double)((0.0 < x) - (x < 0.0)); }
__device__ __forceinline__ float3 nrm3(float3 a) { return (1.f / sqrtf(dot3(a, a))) * a; }
__device__ __forceinline__ float3 d3_unit(float4 q) { return nrm3(qrotate(q, f3(1.f, 0.f, 0.f))); }  // getD3, Rotor.h:206

__global__ void sag_free_kernel(DeviceState st, float3 g, const int32_t* __restrict__ strand_begin,
                                const int64_t* __restrict__ slot_of, int32_t ns, float* __restrict__ fs) {
    const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    // the steps only read rest lengths and rest Darboux; this initialisation rewrites them
    float4* prm = const_cast<float4*>(st.prm);
    float4* qrw = const_cast<float4*>(st.qr);
    const int32_t b = strand_begin[s], e = strand_begin[s + 1], n = e - b;
    auto G = [&](int v) { return slot_of[b + v]; };  // slot of the strand's v-th vertex
    const float eps = 1e-6f;
    // 1. rest lengths, tip to root
    float total_from_tip = 1 / st.xm[G(n - 1)].w;
    for (int v = n - 2; v >= 0; v--) {
        const int64_t gi = G(v), gn = G(v + 1);
        const float3 axis = d3_unit(st.q[gi]);
        float4 p = st.prm[gi];
        const float ks = p.y, old_len = p.x;
        const float im = st.xm[gi].w;
        if (im != 0.f)
            total_from_tip = (float)((double)total_from_tip + 0.5 / (double)im);
        else
            total_from_tip = (float)((double)total_from_tip +
                                     0.5 * (double)(old_len / st.prm[gn].x) / (double)st.xm[gn].w);
        const double f_s = -(double)(dot3(axis, g) * total_from_tip);
        float len;
        if (f_s == 0) {
            len = old_len;
        } else if (1 - 4 * f_s * old_len / ks < 0) {
            len = 1.5f * old_len;
        } else {
            const double fsk = f_s / ks, fskinv = ks / f_s;
            const double r = sqrt(1 - 4 * old_len * fsk);
            const double ans1 = (1 + r) * 0.5f * fskinv, ans2 = (1 - r) * 0.5f * fskinv;
            len = (float)(fabs(old_len - ans1) >= fabs(old_len - ans2) ? ans2 : ans1);
        }
        p.x = fminf(fmaxf(len, eps), 1.5f * old_len);
        prm[gi] = p;
        fs[gi] = (float)-f_s;
        total_from_tip = (float)((double)total_from_tip + 0.5 / (double)im);
    }
    // 2. rest angles, root to tip
    const float nearest = 1e-4f;
    float total_to_tip = 0.f;
    for (int v = 1; v < n; v++) {
        const float im = st.xm[G(v)].w;
        if (im != 0.f)
            total_to_tip += 1 / im;
        else
            total_to_tip += (st.prm[G(v)].x / st.prm[G(v - 1)].x) / st.xm[G(v - 1)].w;
    }
    float4 acc = make_float4(0.f, 0.f, 0.f, 1.f);
    for (int v = 1; v < n - 1; v++) {
        const int64_t gi = G(v), gn = G(v + 1), gp = G(v - 1);
        const float4 qv = st.q[gi];
        const float4 cqk = qmul(acc, qv);
        const float im = st.xm[gi].w;
        if (im != 0.f)
            total_to_tip = (float)((double)total_to_tip - 0.5 / (double)im);
        else
            total_to_tip = (float)((double)total_to_tip - 0.5 * (double)(st.prm[gi].x / st.prm[gn].x) / (double)st.xm[gn].w);
        const float3 axisk = d3_unit(cqk);
        // the stretch force of the next segment (none past the last segment)
        const float3 f_sr = (v + 1 <= n - 2) ? fs[gn] * d3_unit(st.q[gn]) : f3(0.f, 0.f, 0.f);
        const float3 f_b = f_sr + total_to_tip * g;
        if (dot3(f_b, axisk) < 1 - nearest) {
            const float4 qr = st.qr[gi];
            const float kbend = sqrtf(dot4(qr, qr));
            const float3 pn = nrm3(cross3(axisk, f_b));
            const float3 tdir = cross3(pn, axisk);
            const float3 seg = xyz(st.xm[gn]) - xyz(st.xm[gi]);
            const float T = dot3(tdir, f_b) * sqrtf(dot3(seg, seg)) / kbend;
            const float lfb = sqrtf(dot3(f_b, f_b));
            const double fx = f_b.x / lfb, fy = f_b.y / lfb, fz = f_b.z / lfb;
            const double maxrad = acos(-((double)axisk.x * fx + (double)axisk.y * fy + (double)axisk.z * fz));
            const double m1 = fit_angle(maxrad + nearest), m2 = fit_angle(maxrad - nearest);
            const double max_theta = fabs(m1) >= fabs(m2) ? m2 : m1;
            const float left = max_theta >= 0 ? 0.f : (float)max_theta;
            const float right = max_theta >= 0 ? (float)max_theta : 0.f;
            double res = 0;
            if (fabs(T) > 2) {
                res = max_theta;
            } else {
                const double half_pi = 1.5707963267948966192313216916397;
                const double t1 = fit_angle(2 * acos(1 - (0.5 * T * T)));
                const double t2 = fit_angle(2 * acos(-1 + (0.5 * T * T)));
                double c1 = -sgn(max_theta) * 100, c2 = -sgn(max_theta) * 100;
                if (fabs(t1) <= half_pi) c1 = t1;
                if (fabs(t2) > half_pi) c2 = t2;
                if (sgn(c1) == sgn(max_theta) && sgn(c2) == sgn(max_theta)) {
                    res = fmin(c1, c2);
                } else {
                    if (sgn(c1) == sgn(max_theta)) res = c1;
                    if (sgn(c2) == sgn(max_theta)) res = c2;
                }
            }
            res = fmin(fmax(res, (double)left), (double)right);
            const float half = 0.5f * (float)res;  // Rotor::angleAxis, Rotor.h:51-54
            const float sh = sinf(half);
            acc = qmul(acc, make_float4(sh * pn.x, sh * pn.y, sh * pn.z, cosf(half)));
            const float4 nq = qmul(acc, qv);
            st.q[gi] = nq;
            const float4 pq = st.q[gp];
            const float4 d = qmul(make_float4(-pq.x, -pq.y, -pq.z, pq.w), nq);
            const float4 pr = st.qr[gp];
            const float len = sqrtf(dot4(pr, pr));
            const float dl = 1.f / sqrtf(dot4(d, d));
            qrw[gp] = make_float4(d.x * dl * len, d.y * dl * len, d.z * dl * len, d.w * dl * len);
        }
        total_to_tip = (float)((double)total_to_tip - 0.5 / (double)im);
    }
}

}  // namespace

cudaError_t launch_sag_free(const DeviceState& st, float3 gravity, const int32_t* strand_begin, const int64_t* slot_of,
                            int32_t num_strands, float* fs, int iterations, cudaStream_t s) {
    if (num_strands == 0) return cudaSuccess;
    for (int it = 0; it < iterations; it++) {
        sag_free_kernel<<<(num_strands + 127) / 128, 128, 0, s>>>(st, gravity, strand_begin, slot_of, num_strands, fs);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace kami
