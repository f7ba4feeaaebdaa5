// hair_prep.cu -- Hair preprocessing that KamiSimulator's StableCosseratRods solver runs before it
// builds the simulation, done on the GPU with one thread per strand:
//   * kami_hair_subdivide = Kami::HairMods::DivideHair (utilities/HairModification.cpp:12-80):
//     SubdivCoeff - 1 evenly spaced points inserted into every segment (positions and velocities);
//   * kami_hair_resample = the EnableResample branch of BuildYarnBallHair
//     (StableCosseratRodsSolver.cpp:141-163) with Resample::resampleCMR (YarnBall/io/resample.h):
//     uniform Catmull-Rom samples (Kit::cmrSpline, KittenEngine Common.h:625-635) marched at
//     parameter steps of 0.2 and refined by eight secant steps to the target segment length, from
//     both ends and merged at the closest pair of samples when both have more than 32; done for the
//     target length and again for the average length of the first result, keeping the one whose
//     segment lengths vary less; a result longer than the Hair's row is subsampled to it.
// This file is compiled without FMA contraction so that its double arithmetic rounds as the
// reference's host code does.  Entries the reference would write outside its lists (a pass with
// fewer than 9 samples, or a merge point within 8 samples of an end) are skipped.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "kami_vbd.h"
#include "vbd_host.h"

namespace kami {
namespace {

struct DV {
    double x, y, z;
};
__device__ __forceinline__ DV dmix(DV a, DV b, double t) {  // glm::mix: a (1 - t) + b t
    return {a.x * (1.0 - t) + b.x * t, a.y * (1.0 - t) + b.y * t, a.z * (1.0 - t) + b.z * t};
}
__device__ __forceinline__ double dlen2(DV a, DV b) {
    const double x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
    return x * x + y * y + z * z;
}
__device__ __forceinline__ double glm_clamp(double x, double lo, double hi) {
    x = (x < lo) ? lo : x;
    return (hi < x) ? hi : x;
}

struct Curve {
    const float* p;  // n points xyz
    int n;
    __device__ DV at(int i) const { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
    __device__ DV sample(double t) const {  // sampleCurve, resample.h:10-18
        int si = (int)floor(t);
        si = si < 1 ? 1 : (si > n - 3 ? n - 3 : si);
        const DV p0 = at(si - 1), p1 = at(si), p2 = at(si + 1), p3 = at(si + 2);
        const double u = t - si;
        const DV a0 = dmix(p0, p1, u + 1), a1 = dmix(p1, p2, u + 0), a2 = dmix(p2, p3, u - 1);
        const DV b0 = dmix(a0, a1, (u + 1) * 0.5f), b1 = dmix(a1, a2, (u + 0) * 0.5f);
        return dmix(b0, b1, u);
    }
};

// A bounded list of parameters in scratch memory; push past the capacity sets `over`.
struct List {
    double* d;
    int64_t cap, n;
    bool* over;
    __device__ void push(double v) {
        if (n < cap)
            d[n++] = v;
        else
            *over = true;
    }
};

// resampleCMRCoords, resample.h:20-82
__device__ void cmr_coords(const Curve& c, double start, double end, double tar, List& ts) {
    ts.n = 0;
    const double step = end > start ? 0.2 : -0.2;
    const double r2 = tar * tar;
    double i = start;
    DV last = c.sample(i);
    ts.push(i);
    while (((end > start) ? i < end : i > end) && !*ts.over) {
        i += step;
        const DV pos = c.sample(i);
        double l0 = dlen2(pos, last);
        if (l0 > r2) {
            l0 = sqrt(l0);
            double lo = i - step, hi = i;
            if (lo > hi) {
                const double t = lo;
                lo = hi;
                hi = t;
            }
            const double t0 = i;
            i -= 0.5 * step;
            for (int k = 0; k < 8; k++) {
                const double d = sqrt(dlen2(c.sample(i), last));
                i += (i - t0) * (tar - d) / (d - l0);
            }
            i = glm_clamp(i, lo, hi);
            ts.push(i);
            last = c.sample(i);
        }
    }
    if (*ts.over) return;
    if (ts.n == 1) {
        ts.push(end);
    } else {
        const double d = sqrt(dlen2(c.sample(ts.d[ts.n - 1]), c.sample(end)));
        double dt = ts.d[ts.n - 1] - ts.d[ts.n - 2];
        if (d > 0.5f * tar)
            ts.push(end);
        else
            ts.d[ts.n - 1] = end;
        if (*ts.over) return;
        dt -= ts.d[ts.n - 1] - ts.d[ts.n - 2];
        const int64_t N = ts.n < 8 ? ts.n : 8;
        for (int64_t k = 0; k < N; k++) {
            const int64_t idx = ts.n - 2 - k;
            if (idx >= 0) ts.d[idx] -= dt * (N - k) / (double)N;
        }
    }
}

// twoDirectionResampleCMRCoords, resample.h:84-140: the merged list goes to m.
__device__ void cmr_two_way(const Curve& c, double start, double end, double tar, List& F, List& B, List& m) {
    cmr_coords(c, start, end, tar, F);
    cmr_coords(c, end, start, tar, B);
    m.n = 0;
    if (*F.over) return;
    const int BORDER = 8;
    if (F.n > 4 * BORDER && B.n > 4 * BORDER) {
        double min_err = INFINITY;
        int64_t sx = 2 * BORDER, sy = 2 * BORDER;
        for (int64_t i = BORDER, j = B.n - 1 - BORDER; i < F.n - 8; i++) {
            const double t = F.d[i];
            while (j > 0 && B.d[j] < t) j--;
            const double t0 = B.d[j + 1];
            if (min_err > fabs(t - t0)) {
                min_err = fabs(t - t0);
                sx = i;
                sy = j + 1;
            }
            const double t1 = B.d[j];
            if (min_err > fabs(t1 - t)) {
                min_err = fabs(t1 - t);
                sx = i;
                sy = j;
            }
        }
        for (int64_t k = 0; k < sx; k++) m.push(F.d[k]);
        const double mid = 0.5 * (F.d[sx] + B.d[sy]);
        m.push(mid);
        for (int64_t k = sy - 1; k >= 0; k--) m.push(B.d[k]);
        if (*m.over) return;
        double dt = F.d[sx] - mid;
        for (int k = 0; k < BORDER; k++) {
            const int64_t idx = sx - k - 1;
            if (idx >= 0 && idx < m.n) m.d[idx] -= dt * (BORDER - k) / (1. + BORDER);
        }
        dt = B.d[sy] - mid;
        for (int k = 0; k < BORDER; k++) {
            const int64_t idx = sx + k + 1;
            if (idx >= 0 && idx < m.n) m.d[idx] -= dt * (BORDER - k) / (1. + BORDER);
        }
    } else {
        for (int64_t k = 0; k < F.n; k++) m.push(F.d[k]);
    }
}

__device__ void seg_stats(const Curve& c, const List& ts, double tar, double& total, double& err) {
    total = 0;
    err = 0;
    DV last = c.sample(ts.d[0]);
    for (int64_t i = 1; i < ts.n; i++) {
        const DV pos = c.sample(ts.d[i]);
        const double len = sqrt(dlen2(pos, last));
        err = fmax(err, fabs(len - tar));
        total += len;
        last = pos;
    }
}

// One strand per thread: strands first .. first + count of the batch.  `in` holds each strand's
// original points (row s at s * max_verts); the result is written into `out` (same rows) and its
// count into `counts`.  Scratch: 6 lists per strand at scratch + offsets[s].
__global__ void resample_kernel(int32_t first, int32_t count, int32_t* __restrict__ counts, int32_t max_verts,
                                const float* __restrict__ in, float* __restrict__ out, double tar,
                                double* __restrict__ scratch, const int64_t* __restrict__ offsets,
                                const int64_t* __restrict__ caps, int* __restrict__ error) {
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int32_t s = first + k;
    const int32_t n = counts[s];
    const float* src = in + (int64_t)s * max_verts * 3;
    float* dst = out + (int64_t)s * max_verts * 3;
    if (n < 4) {  // left as it is (BuildYarnBallHair skips such strands)
        for (int32_t q = 0; q < 3 * n; q++) dst[q] = src[q];
        return;
    }
    bool over = false;
    const int64_t cap = caps[k];
    double* base = scratch + offsets[k];
    List F{base, cap, 0, &over}, B{base + cap, cap, 0, &over};
    List m0{base + 2 * cap, 2 * cap, 0, &over}, m1{base + 4 * cap, 2 * cap, 0, &over};
    const Curve c{src, n};
    const double start = 1, end = n - 2;
    cmr_two_way(c, start, end, tar, F, B, m0);
    double total0 = 0, err0 = 0, total1 = 0, err1 = 0;
    if (!over) seg_stats(c, m0, tar, total0, err0);
    const double avg = over ? tar : total0 / (m0.n - 1);
    if (!over) cmr_two_way(c, start, end, avg, F, B, m1);
    if (!over) seg_stats(c, m1, avg, total1, err1);
    if (over) {
        atomicExch(error, 1);
        return;
    }
    const List& ts = err0 < err1 ? m0 : m1;
    const int64_t m = ts.n;
    if (m <= max_verts) {
        for (int64_t i = 0; i < m; i++) {
            const DV p = c.sample(ts.d[i]);
            dst[3 * i] = (float)p.x;
            dst[3 * i + 1] = (float)p.y;
            dst[3 * i + 2] = (float)p.z;
        }
        counts[s] = (int32_t)m;
    } else {
        // the resampled strand is longer than the Hair's row: keep its ends and every stride-th
        // point between them (StableCosseratRodsSolver.cpp:147-158)
        const float stride = (float)(m - 2) / (float)(max_verts - 2);
        for (int32_t v = 0; v < max_verts; v++) {
            const int64_t j = v == 0 ? 0 : (v == max_verts - 1 ? m - 1 : (int64_t)(uint32_t)(stride * v));
            const DV p = c.sample(ts.d[j]);
            dst[3 * v] = (float)p.x;
            dst[3 * v + 1] = (float)p.y;
            dst[3 * v + 2] = (float)p.z;
        }
        counts[s] = max_verts;
    }
}

// DivideHair's interpolate(x, y, den, num) = ((den - num) x + num y) / den, in float.
__device__ __forceinline__ float lerp_div(float x, float y, int den, int num) {
    const float fden = (float)den, fnum = (float)num;
    return ((fden - fnum) * x + fnum * y) / fden;
}

__global__ void subdivide_kernel(int32_t ns, const int32_t* __restrict__ counts, int32_t max_verts,
                                 const float* __restrict__ x, const float* __restrict__ v, int32_t mul,
                                 int32_t out_verts, float* __restrict__ ox, float* __restrict__ ov) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t s = t / out_verts;
    const int32_t w = (int32_t)(t - s * out_verts);
    if (s >= ns) return;
    const int32_t n = counts[s];
    if (n <= 0 || w > (n - 1) * mul) return;
    const int64_t in_row = s * (int64_t)max_verts * 3, out_row = s * (int64_t)out_verts * 3;
    const int32_t seg = w / mul, i = w - seg * mul;
    for (int a = 0; a < 3; a++) {
        if (seg == n - 1) {  // the strand's last point
            ox[out_row + 3 * w + a] = x[in_row + 3 * seg + a];
            if (v) ov[out_row + 3 * w + a] = v[in_row + 3 * seg + a];
        } else {
            ox[out_row + 3 * w + a] = lerp_div(x[in_row + 3 * seg + a], x[in_row + 3 * (seg + 1) + a], mul, i);
            if (v) ov[out_row + 3 * w + a] = lerp_div(v[in_row + 3 * seg + a], v[in_row + 3 * (seg + 1) + a], mul, i);
        }
    }
}

#define KAMI_TRY_PREP(expr)              \
    do {                                 \
        kami_status s_ = (expr);         \
        if (s_ != KAMI_OK) return s_;    \
    } while (0)

kami_status prep_fail(kami_status st, const std::string& msg) {
    set_last_error(msg.c_str());
    return st;
}

kami_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return KAMI_OK;
    return prep_fail(e == cudaErrorMemoryAllocation ? KAMI_ERR_OUT_OF_MEMORY : KAMI_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace kami

using namespace kami;

extern "C" kami_status kami_hair_subdivide(int32_t num_strands, const int32_t* counts, int32_t max_verts, const float* xyz,
                                           const float* vxyz, int32_t mul, int32_t* out_counts, float* out_xyz,
                                           float* out_vxyz, int32_t device) {
    if (num_strands < 0 || max_verts < 1 || mul < 1 || !counts || !xyz || !out_counts || !out_xyz || (vxyz && !out_vxyz))
        return prep_fail(KAMI_ERR_INVALID_ARGUMENT, "bad arguments to kami_hair_subdivide");
    for (int32_t s = 0; s < num_strands; s++)
        if (counts[s] < 0 || counts[s] > max_verts)
            return prep_fail(KAMI_ERR_INVALID_ARGUMENT, "a strand count is negative or exceeds max_verts");
    const int64_t out_verts = (int64_t)(max_verts - 1) * mul + 1;
    if (out_verts > INT32_MAX) return prep_fail(KAMI_ERR_INVALID_ARGUMENT, "subdivided rows too long");
    for (int32_t s = 0; s < num_strands; s++) out_counts[s] = counts[s] > 0 ? (counts[s] - 1) * mul + 1 : 0;
    if (num_strands == 0) return KAMI_OK;
    if (device >= 0) KAMI_TRY_PREP(cuda_status(cudaSetDevice(device), "cudaSetDevice"));
    const size_t in_b = sizeof(float) * 3 * (size_t)num_strands * max_verts;
    const size_t out_b = sizeof(float) * 3 * (size_t)num_strands * out_verts;
    int32_t* dc = nullptr;
    float *dx = nullptr, *dv = nullptr, *dox = nullptr, *dov = nullptr;
    cudaError_t e = cudaMalloc(&dc, sizeof(int32_t) * num_strands);
    if (e == cudaSuccess) e = cudaMalloc(&dx, in_b);
    if (e == cudaSuccess && vxyz) e = cudaMalloc(&dv, in_b);
    if (e == cudaSuccess) e = cudaMalloc(&dox, out_b);
    if (e == cudaSuccess && vxyz) e = cudaMalloc(&dov, out_b);
    if (e == cudaSuccess) e = cudaMemcpy(dc, counts, sizeof(int32_t) * num_strands, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dx, xyz, in_b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && vxyz) e = cudaMemcpy(dv, vxyz, in_b, cudaMemcpyHostToDevice);
    // rows past each strand's end keep the caller's values
    if (e == cudaSuccess) e = cudaMemcpy(dox, out_xyz, out_b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && vxyz) e = cudaMemcpy(dov, out_vxyz, out_b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int64_t threads = (int64_t)num_strands * out_verts;
        subdivide_kernel<<<(unsigned)((threads + 255) / 256), 256>>>(num_strands, dc, max_verts, dx, dv, mul,
                                                                     (int32_t)out_verts, dox, dov);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out_xyz, dox, out_b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && vxyz) e = cudaMemcpy(out_vxyz, dov, out_b, cudaMemcpyDeviceToHost);
    void* bufs[] = {dc, dx, dv, dox, dov};
    for (void* b : bufs)
        if (b) cudaFree(b);
    return cuda_status(e, "kami_hair_subdivide");
}

extern "C" kami_status kami_hair_resample(int32_t num_strands, int32_t* counts, int32_t max_verts, float* xyz,
                                          float target_len, int32_t device) {
    if (num_strands < 0 || max_verts < 4 || !counts || !xyz || !(target_len > 0.f) || !std::isfinite(target_len))
        return prep_fail(KAMI_ERR_INVALID_ARGUMENT, "bad arguments to kami_hair_resample (max_verts >= 4, target > 0)");
    for (int32_t s = 0; s < num_strands; s++)
        if (counts[s] < 0 || counts[s] > max_verts)
            return prep_fail(KAMI_ERR_INVALID_ARGUMENT, "a strand count is negative or exceeds max_verts");
    if (num_strands == 0) return KAMI_OK;
    // scratch per strand: 6 lists of a capacity bounded by the parameter steps (5 per segment) plus
    // the samples the arc length needs (polyline length / target, doubled for the spline's excess)
    std::vector<int64_t> caps(num_strands, 0);
    for (int32_t s = 0; s < num_strands; s++) {
        const int32_t n = counts[s];
        if (n < 4) continue;
        double L = 0;
        const float* p = xyz + (size_t)s * max_verts * 3;
        for (int32_t i = 0; i + 1 < n; i++) {
            const double dx = p[3 * i + 3] - p[3 * i], dy = p[3 * i + 4] - p[3 * i + 1], dz = p[3 * i + 5] - p[3 * i + 2];
            L += std::sqrt(dx * dx + dy * dy + dz * dz);
        }
        if (!std::isfinite(L)) return prep_fail(KAMI_ERR_INVALID_ARGUMENT, "non-finite strand point");
        caps[s] = 5LL * (n - 3) + 16 + 2 * (int64_t)std::ceil(L / target_len);
    }
    if (device >= 0) KAMI_TRY_PREP(cuda_status(cudaSetDevice(device), "cudaSetDevice"));
    const size_t rows_b = sizeof(float) * 3 * (size_t)num_strands * max_verts;
    int32_t* dc = nullptr;
    float *din = nullptr, *dout = nullptr;
    int* derr = nullptr;
    cudaError_t e = cudaMalloc(&dc, sizeof(int32_t) * num_strands);
    if (e == cudaSuccess) e = cudaMalloc(&din, rows_b);
    if (e == cudaSuccess) e = cudaMalloc(&dout, rows_b);
    if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(dc, counts, sizeof(int32_t) * num_strands, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(din, xyz, rows_b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dout, xyz, rows_b, cudaMemcpyHostToDevice);  // padding keeps its values
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    // batches of strands whose scratch stays within 1 GiB
    const int64_t budget = (1LL << 30) / (int64_t)sizeof(double);
    double* dscratch = nullptr;
    int64_t *doff = nullptr, *dcap = nullptr;
    int64_t scratch_cap = 0;
    for (int32_t first = 0; first < num_strands && e == cudaSuccess;) {
        int32_t last = first;
        int64_t total = 0;
        std::vector<int64_t> offs, cps;
        while (last < num_strands && (last == first || total + 6 * caps[last] <= budget)) {
            offs.push_back(total);
            cps.push_back(caps[last]);
            total += 6 * caps[last];
            last++;
        }
        const int32_t count = last - first;
        if (total > scratch_cap) {
            if (dscratch) cudaFree(dscratch);
            dscratch = nullptr;
            e = cudaMalloc(&dscratch, sizeof(double) * std::max<int64_t>(total, 1));
            scratch_cap = total;
        }
        if (doff) cudaFree(doff);
        if (dcap) cudaFree(dcap);
        doff = dcap = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&doff, sizeof(int64_t) * count);
        if (e == cudaSuccess) e = cudaMalloc(&dcap, sizeof(int64_t) * count);
        if (e == cudaSuccess) e = cudaMemcpy(doff, offs.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dcap, cps.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            resample_kernel<<<(count + 63) / 64, 64>>>(first, count, dc, max_verts, din, dout, (double)target_len,
                                                       dscratch, doff, dcap, derr);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        first = last;
    }
    int err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&err, derr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && !err) e = cudaMemcpy(counts, dc, sizeof(int32_t) * num_strands, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && !err) e = cudaMemcpy(xyz, dout, rows_b, cudaMemcpyDeviceToHost);
    void* bufs[] = {dc, din, dout, derr, dscratch, doff, dcap};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (e != cudaSuccess) return cuda_status(e, "kami_hair_resample");
    if (err) return prep_fail(KAMI_ERR_UNSUPPORTED, "a strand needed more samples than its scratch bound (nothing was changed)");
    return KAMI_OK;
}
