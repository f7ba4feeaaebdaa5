// kami_vbd_noalloc.cu -- kami_vbd_step_noalloc: one solver step that allocates no device memory.
//
// Who needs it: a host engine that owns every byte of device memory itself (a fixed pool or a
// hard budget, so a library may not cudaMalloc behind its back), and real-time frame loops in
// which a cudaMalloc/cudaFree, which can synchronise the whole device, would blow the frame
// budget.  Such a caller keeps the solver state in its own device buffers, in boundary order,
// and calls this entry point each step; the handle-based API (kami_vbd_create) cannot serve it
// because creating a handle allocates.
//
// What runs: the sweep form of the step (predict; per iteration the even-vertex, odd-vertex,
// even-segment and odd-segment colour sweeps; velocity update), with the same per-vertex
// arithmetic as the handle's kernels (vbd_math.cuh), indexed directly in boundary order.  There
// is no SDF pass and no finiteness status word in this variant.
//
// Scratch: the inertial targets, the displacement iterate and the derived vertex flags live in
// g_noalloc_scratch, a file-scope __device__ array sized for KAMI_NOALLOC_MAX_VERTICES vertices
// (12 MiB), which every device that loads the library keeps until the process exits.  Host code
// cannot use the symbol itself as a device address, so each call, with the caller's device
// current, resolves it with cudaGetSymbolAddress (the set-up) unless its stream is capturing; make
// the first call on each device, and the first after a cudaDeviceReset, outside any stream
// capture.  All calls share the one array and it keeps the last call's contents; every call
// writes each scratch entry before reading it, so nothing needs clearing.  Calls whose work
// overlaps on the GPU (different streams, or concurrent host threads) race on the scratch.
//
// The strand offsets are device data, so the host cannot check them: the flags kernel clamps each
// strand to the vertex range, and malformed offsets give wrong flags but no access out of bounds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "kami_vbd.h"
#include "vbd_host.h"
#include "vbd_math.cuh"

namespace kami {
namespace {

constexpr int64_t kMaxV = KAMI_NOALLOC_MAX_VERTICES;

// rows: [0, kMaxV) inertial target y (xyz); [kMaxV, 2 kMaxV) displacement iterate dx (xyz);
// [2 kMaxV, 3 kMaxV) vertex flags in .x (bit pattern)
static __device__ __align__(256) float4 g_noalloc_scratch[3 * kMaxV];

constexpr uint32_t F_ODD = 128u;  // odd index inside its strand (colour 1)

__device__ __forceinline__ float3 ld3(const float* a, int64_t i) { return f3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
__device__ __forceinline__ void st3(float* a, int64_t i, float3 v) {
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}
__device__ __forceinline__ float4 ld4(const float* a, int64_t i) {
    return make_float4(a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]);
}

struct NoAllocArgs {
    int64_t nv;
    int32_t ns;
    const int32_t* sb;
    float* x;
    float* v;
    float* vl;
    float* q;
    const float* qr;
    const float* im;
    const float* lr;
    const float* ks;
    float4* scratch;
};

// Flags of each vertex from the strand offsets, as Sim::configure sets them (YBSimulator.cu:170-186).
__global__ void noalloc_flags_kernel(NoAllocArgs a) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nv) return;
    int lo = 0, hi = a.ns - 1;  // last strand s with sb[s] <= i
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (a.sb[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    // The offsets are the caller's and are not checked on the host (they live on the device), so
    // the strand's range is clamped to [0, nv): no flag can then point a neighbour read past either
    // end of the arrays, whatever the offsets hold.  A vertex outside every clamped range gets no
    // flags and moves as a free particle.
    const int64_t b = max((int64_t)a.sb[lo], (int64_t)0);
    const int64_t n = min((int64_t)a.sb[lo + 1], a.nv) - b;
    const int64_t local = i - b;
    if (local < 0 || local >= n) {
        a.scratch[2 * kMaxV + i] = make_float4(__uint_as_float(0u), 0.f, 0.f, 0.f);
        return;
    }
    uint32_t f = F_VALID;
    if (local == 0) f |= F_ROOT;
    if (local > 0) f |= F_HAS_PREV;
    if (local + 1 < n) f |= F_HAS_NEXT;
    if (local + 2 < n) f |= F_HAS_NEXT_ORIENTATION;
    if (local + 1 == n && i + 1 < a.nv) f |= F_FIX_ORIENTATION;
    if (local & 1) f |= F_ODD;
    a.scratch[2 * kMaxV + i] = make_float4(__uint_as_float(f), 0.f, 0.f, 0.f);
}

__global__ void noalloc_predict_kernel(NoAllocArgs a, PhysParams pp, StepParams sp) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nv) return;
    float3 x = ld3(a.x, i), v = ld3(a.v, i), vl = ld3(a.vl, i);
    float3 dx, y;
    vbd_predict(x, v, vl, a.im[i], pp, sp.h, sp.last_h, sp.time, dx, y);
    st3(a.vl, i, v);
    a.scratch[i] = make_float4(y.x, y.y, y.z, 0.f);
    a.scratch[kMaxV + i] = make_float4(dx.x, dx.y, dx.z, 0.f);
}

__device__ __forceinline__ uint32_t flags_of(const NoAllocArgs& a, int64_t i) {
    return __float_as_uint(a.scratch[2 * kMaxV + i].x);
}

__global__ void noalloc_position_kernel(NoAllocArgs a, PhysParams pp, float h, int colour) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nv) return;
    const uint32_t fl = flags_of(a, i);
    if (((fl & F_ODD) ? 1 : 0) != colour || a.im[i] == 0.f) return;
    const float damp = pp.damping / h;
    const float4* dxs = a.scratch + kMaxV;
    const float3 dx = xyz(dxs[i]);
    float3 en = f3(0.f, 0.f, 0.f), ep = en, d3n = en, d3p = en, dxn = en, dxp = en;
    float invln = 0.f, kkn = 0.f, ddn = 0.f, invlp = 0.f, kkp = 0.f, ddp = 0.f;
    if (fl & F_HAS_NEXT) {
        en = ld3(a.x, i + 1) - ld3(a.x, i);
        invln = 1.f / a.lr[i];
        kkn = a.ks[i] * invln;
        ddn = kkn * invln;
        d3n = d3_of(ld4(a.q, i));
        dxn = xyz(dxs[i + 1]);
    }
    if (fl & F_HAS_PREV) {
        ep = ld3(a.x, i) - ld3(a.x, i - 1);
        invlp = 1.f / a.lr[i - 1];
        kkp = a.ks[i - 1] * invlp;
        ddp = kkp * invlp;
        d3p = d3_of(ld4(a.q, i - 1));
        dxp = xyz(dxs[i - 1]);
    }
    BlockConst bc = vbd_block_const(a.im[i], fl, ddn, ddp, h, damp);
    float3 nd = vbd_position(dx, xyz(a.scratch[i]), fl, bc, en, invln, kkn, ddn, d3n, dxn, ep, invlp, kkp, ddp, d3p,
                             dxp, damp, pp.accel_ratio);
    a.scratch[kMaxV + i] = make_float4(nd.x, nd.y, nd.z, 0.f);
}

__global__ void noalloc_orientation_kernel(NoAllocArgs a, int colour) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nv) return;
    const uint32_t fl = flags_of(a, i);
    if (((fl & F_ODD) ? 1 : 0) != colour) return;
    if (!(fl & F_HAS_NEXT) || (fl & F_FIX_ORIENTATION)) return;
    const float4* dxs = a.scratch + kMaxV;
    float3 e = ld3(a.x, i + 1) - ld3(a.x, i);
    float4 qp = make_float4(0.f, 0.f, 0.f, 1.f), qrp = qp, qn = qp;
    if (fl & F_HAS_PREV) {
        qp = ld4(a.q, i - 1);
        qrp = ld4(a.qr, i - 1);
    }
    if (fl & F_HAS_NEXT_ORIENTATION) qn = ld4(a.q, i + 1);
    float m2k = -2.f * a.ks[i] * (1.f / a.lr[i]);
    float4 nq = vbd_orientation(ld4(a.q, i), fl, e, xyz(dxs[i]), xyz(dxs[i + 1]), m2k, qp, qrp, qn, ld4(a.qr, i));
    a.q[4 * i] = nq.x;
    a.q[4 * i + 1] = nq.y;
    a.q[4 * i + 2] = nq.z;
    a.q[4 * i + 3] = nq.w;
}

__global__ void noalloc_finish_kernel(NoAllocArgs a, float h, float decay) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nv) return;
    float3 x = ld3(a.x, i), v = ld3(a.v, i);
    vbd_finish(x, v, xyz(a.scratch[kMaxV + i]), a.im[i], h, decay);
    st3(a.x, i, x);
    st3(a.v, i, v);
}

// Device address of g_noalloc_scratch, resolved once per device.
std::mutex g_scratch_mutex;
constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};

// the message is reported through kami_vbd_last_error_string
kami_status noalloc_fail(kami_status st, const char* msg, cudaError_t e = cudaSuccess) {
    char buf[512];
    if (e != cudaSuccess)
        snprintf(buf, sizeof(buf), "%s: %s", msg, cudaGetErrorString(e));
    else
        snprintf(buf, sizeof(buf), "%s", msg);
    set_last_error(buf);
    return st;
}

}  // namespace
}  // namespace kami

using namespace kami;

extern "C" kami_status kami_vbd_step_noalloc(const kami_vbd_desc* settings, kami_vbd_noalloc_args* a, float dt,
                                             void* stream) {
    if (!settings || !a) return noalloc_fail(KAMI_ERR_INVALID_ARGUMENT, "null settings or arguments");
    if (a->num_vertices < 3 || a->num_strands <= 0)
        return noalloc_fail(KAMI_ERR_INVALID_ARGUMENT, "need at least 3 vertices and 1 strand");
    if (a->num_vertices > KAMI_NOALLOC_MAX_VERTICES)
        return noalloc_fail(KAMI_ERR_UNSUPPORTED,
                            "kami_vbd_step_noalloc holds at most KAMI_NOALLOC_MAX_VERTICES (262144) vertices; use the "
                            "handle API (kami_vbd_create) for larger sets");
    if (!a->strand_begin || !a->positions || !a->velocities || !a->last_velocities || !a->orientations ||
        !a->rest_darboux || !a->inv_mass || !a->rest_length || !a->stretch_stiffness)
        return noalloc_fail(KAMI_ERR_INVALID_ARGUMENT, "a device array pointer is null");
    if (settings->schedule != KAMI_SCHEDULE_COLOUR2)
        return noalloc_fail(KAMI_ERR_UNSUPPORTED, "kami_vbd_step_noalloc runs the colour2 schedule only");
    if (settings->connection_index)
        return noalloc_fail(KAMI_ERR_UNSUPPORTED, "kami_vbd_step_noalloc has no connection springs");
    if (settings->num_itr < 0 || !(settings->max_h > 0.f))
        return noalloc_fail(KAMI_ERR_INVALID_ARGUMENT, "num_itr must be >= 0 and max_h > 0");
    if (!std::isfinite(dt)) return noalloc_fail(KAMI_ERR_INVALID_ARGUMENT, "dt must be finite");
    if (!(dt > 0.f)) return KAMI_OK;  // Sim::advance returns for h <= 0
    // Sim::advance's substep count (step.cpp:38-62), bounded before the conversion to int
    const float ratio = std::ceil(dt / settings->max_h);
    if (!(ratio <= (float)KAMI_MAX_SUBSTEPS))
        return noalloc_fail(KAMI_ERR_INVALID_ARGUMENT, "dt / max_h needs more than KAMI_MAX_SUBSTEPS substeps");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(KAMI_ERR_CUDA, "cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(KAMI_ERR_UNSUPPORTED, "device ordinal out of range");
    cudaStream_t s = (cudaStream_t)stream;
    // The symbol's device address belongs to the module loaded in the device's current context, and
    // a cudaDeviceReset makes a new one, so it is looked up again on every call made outside a stream
    // capture.  A call made while its stream captures takes the address of the last call made
    // outside one on this device.
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &capture);
    if (e != cudaSuccess) return noalloc_fail(KAMI_ERR_CUDA, "cudaStreamIsCapturing", e);
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (capture == cudaStreamCaptureStatusNone) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return noalloc_fail(KAMI_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch)", e);
            g_scratch_ptr[dev] = p;
        } else if (!g_scratch_ptr[dev]) {
            return noalloc_fail(KAMI_ERR_STATE,
                                "the first kami_vbd_step_noalloc call on a device must come outside a stream capture");
        }
        scratch = g_scratch_ptr[dev];
    }

    PhysParams pp;
    pp.gx = settings->gravity[0];
    pp.gy = settings->gravity[1];
    pp.gz = settings->gravity[2];
    pp.damping = settings->damping;
    pp.velocity_decay = settings->velocity_decay;
    pp.accel_ratio = settings->acceleration_ratio;
    pp.ext_mult = settings->external_force_multiplier;
    pp.wind_peak = settings->wind_peak;
    pp.wind_yf = settings->wind_y_freq;
    pp.wind_zf = settings->wind_z_freq;
    pp.wind_tf = settings->wind_time_freq;
    pp.wind_sharp = settings->wind_sharpness;
    pp.num_itr = settings->num_itr;

    // Sim::advance (step.cpp:38-62): clock = {h of the previous call, lastH, time}
    const int steps = std::max(1, (int)ratio);
    StepParams sp{};
    sp.last_h = a->clock[0];
    sp.h = dt / (float)steps;
    sp.time = a->clock[2];
    sp.substeps = steps;

    NoAllocArgs k;
    k.nv = a->num_vertices;
    k.ns = a->num_strands;
    k.sb = a->strand_begin;
    k.x = a->positions;
    k.v = a->velocities;
    k.vl = a->last_velocities;
    k.q = a->orientations;
    k.qr = a->rest_darboux;
    k.im = a->inv_mass;
    k.lr = a->rest_length;
    k.ks = a->stretch_stiffness;
    k.scratch = (float4*)scratch;
    const unsigned threads = 256, blocks = (unsigned)((k.nv + threads - 1) / threads);
    noalloc_flags_kernel<<<blocks, threads, 0, s>>>(k);
    for (int sub = 0; sub < steps; sub++) {
        noalloc_predict_kernel<<<blocks, threads, 0, s>>>(k, pp, sp);
        for (int it = 0; it < pp.num_itr; it++) {
            noalloc_position_kernel<<<blocks, threads, 0, s>>>(k, pp, sp.h, 0);
            noalloc_position_kernel<<<blocks, threads, 0, s>>>(k, pp, sp.h, 1);
            noalloc_orientation_kernel<<<blocks, threads, 0, s>>>(k, 0);
            noalloc_orientation_kernel<<<blocks, threads, 0, s>>>(k, 1);
        }
        noalloc_finish_kernel<<<blocks, threads, 0, s>>>(k, sp.h, pp.velocity_decay);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(KAMI_ERR_CUDA, "kernel launch", e);
    a->clock[0] = sp.h;
    a->clock[1] = sp.last_h;
    a->clock[2] = a->clock[2] + dt;
    return KAMI_OK;
}
