// vbd_collision.cu -- hair-hair collision of the sweep form (EnableHairHairColl).
//
// Detection (once every detectionPeriod substeps, after the predict, as Sim::advance calls
// detectCollisions, YarnBall/sim/step.cpp:53):
//   1. every segment's box around its two end points, padded by scaledDetectionRadius plus its
//      velocity radius (buildAABBs, collision.cu:8-32), and the largest box extent;
//   2. a spatial hash of the box centres on cells of that extent: bucket counts, an exclusive scan
//      and a scatter group the segments by bucket;
//   3. each segment scans the 27 cells around its centre and keeps the partners that pass the
//      distance test of buildCollisionList (collision.cu:36-92), in ascending partner order.
// Two boxes that overlap have centres less than one extent apart on every axis, so the 27 cells
// find every pair the reference's LBVH query finds (KittenGpuLBVH/lbvh.cu:197-292); the distance
// test, evaluated once per pair with the lower vertex index first, then decides.
//
// The step limit (recomputeStepLimitKernel, collision.cu:95-131) runs on every substep, and the
// position sweep adds each contact's IPC barrier and friction terms (cosseratItr,
// cosserat.cu:163-227).  The partner segment's displacement is read from a snapshot taken at the
// start of the iteration, so the sweep does not race on the partner's vertices.
#include "vbd_kernels.h"
#include "vbd_math.cuh"

namespace kami {
namespace {

constexpr uint32_t NO_CELL = 0xffffffffu;

__device__ __forceinline__ float len2(float3 a) { return dot3(a, a); }
// glm::mix(x, y, t) = x (1 - t) + y t
__device__ __forceinline__ float3 mixv(float3 a, float3 b, float t) { return a * (1.f - t) + b * t; }
__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.f), 1.f); }
__device__ __forceinline__ bool finite3c(float3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// Kit::segmentClosestPoints (KittenEngine/includes/modules/Common.h:294-312): the closest points
// are mix(a0, a1, u) and mix(b0, b1, w).
__device__ __forceinline__ float2 seg_closest(float3 a0, float3 a1, float3 b0, float3 b1) {
    const float3 A0 = a1 - a0, A1 = b1 - b0;
    const float a = len2(A0), b = dot3(A0, A1), c = len2(A1);
    const float3 diff = b0 - a0;
    float w = b * dot3(A0, diff) - a * dot3(A1, diff);
    w /= a * c - b * b;
    if (!isfinite(w)) w = 0.5f;
    w = clamp01(w);
    const float u = clamp01(dot3(mixv(b0, b1, w) - a0, A0) / a);
    w = clamp01(dot3(mixv(a0, a1, u) - b0, A1) / c);
    return make_float2(u, w);
}

// Spatial hash of a cell (the three large primes of Teschner et al., "Optimized Spatial Hashing
// for Collision Detection of Deformable Objects", VMV 2003).
__device__ __forceinline__ uint32_t cell_hash(uint32_t x, uint32_t y, uint32_t z, uint32_t mask) {
    return ((x * 73856093u) ^ (y * 19349663u) ^ (z * 83492791u)) & mask;
}

__device__ __forceinline__ float cell_size(const CollParams& cp) { return __uint_as_float(*cp.ext_bits) * 1.01f; }

// glm::inverse(mat3) of the packed symmetric Hessian (hess3::operator mat3, SymMat.h:66-75)
// applied to f: the adjugate over the determinant.
__device__ __forceinline__ float3 solve_sym3(const float H[6], float3 f) {
    const float m00 = H[0], m11 = H[1], m22 = H[2], m01 = H[3], m02 = H[4], m12 = H[5];
    const float det = m00 * (m11 * m22 - m12 * m12) - m01 * (m01 * m22 - m12 * m02) + m02 * (m01 * m12 - m11 * m02);
    const float od = 1.f / det;
    const float i00 = (m11 * m22 - m12 * m12) * od;
    const float i10 = -(m01 * m22 - m02 * m12) * od;
    const float i20 = (m01 * m12 - m02 * m11) * od;
    const float i01 = -(m01 * m22 - m12 * m02) * od;
    const float i11 = (m00 * m22 - m02 * m02) * od;
    const float i21 = -(m00 * m12 - m02 * m01) * od;
    const float i02 = (m01 * m12 - m11 * m02) * od;
    const float i12 = -(m00 * m12 - m01 * m02) * od;
    const float i22 = (m00 * m11 - m01 * m01) * od;
    return f3(i00 * f.x + i10 * f.y + i20 * f.z, i01 * f.x + i11 * f.y + i21 * f.z, i02 * f.x + i12 * f.y + i22 * f.z);
}

// ---- detection --------------------------------------------------------------------------------

__global__ void coll_box_kernel(DeviceState st, const float4* __restrict__ dx4, CollParams cp) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float ext = 0.f;
    if (g < cp.num_slots) {
        const uint32_t fl = __float_as_uint(st.prm[g].w);
        if (fl & F_HAS_NEXT) {
            const int64_t gn = next_slot(g, cp.C);
            const float3 p0 = xyz(st.xm[g]), p1 = xyz(st.xm[gn]);
            float vr = 0.f;
            if (cp.use_vel) vr = sqrtf(fmaxf(len2(xyz(dx4[g])), len2(xyz(dx4[gn]))));
            const float pad = cp.scaled_r + vr;
            const float3 lo = f3(fminf(p0.x, p1.x) - pad, fminf(p0.y, p1.y) - pad, fminf(p0.z, p1.z) - pad);
            const float3 hi = f3(fmaxf(p0.x, p1.x) + pad, fmaxf(p0.y, p1.y) + pad, fmaxf(p0.z, p1.z) + pad);
            cp.bmin[g] = make_float4(lo.x, lo.y, lo.z, vr);
            cp.bmax[g] = make_float4(hi.x, hi.y, hi.z, 1.f);
            const float e = fmaxf(fmaxf(hi.x - lo.x, hi.y - lo.y), hi.z - lo.z);
            if (isfinite(e)) ext = e;
        } else {
            cp.bmax[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    for (int o = 16; o; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomicMax(cp.ext_bits, __float_as_uint(ext));
}

__device__ __forceinline__ bool box_cell_of(const CollParams& cp, float4 lo, float4 hi, int3& ci) {
    if (hi.w == 0.f) return false;
    const float3 c = f3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
    const float cs = cell_size(cp);
    if (!finite3c(c) || !(cs > 0.f)) return false;
    const float inv = 1.f / cs;
    ci = make_int3(__float2int_rd(c.x * inv), __float2int_rd(c.y * inv), __float2int_rd(c.z * inv));
    return true;
}
__device__ __forceinline__ bool box_cell(const CollParams& cp, int64_t g, int3& ci) {
    return box_cell_of(cp, cp.bmin[g], cp.bmax[g], ci);
}

__global__ void coll_hash_kernel(CollParams cp) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= cp.num_slots) return;
    int3 ci;
    if (!box_cell(cp, g, ci)) {
        cp.cell[g] = NO_CELL;
        return;
    }
    const uint32_t mask = (1u << cp.table_bits) - 1u;
    const uint32_t h = cell_hash((uint32_t)ci.x, (uint32_t)ci.y, (uint32_t)ci.z, mask);
    cp.cell[g] = h;
    atomicAdd(&cp.count[h], 1);
}

__global__ void coll_scatter_kernel(CollParams cp) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= cp.num_slots) return;
    const uint32_t h = cp.cell[g];
    if (h == NO_CELL) return;
    const int32_t pos = atomicAdd(&cp.cursor[h], 1);
    // the query's per-candidate values in bucket order: one contiguous read per candidate instead of
    // a gather through the slot index
    cp.srec[pos] = make_int4((int32_t)g, cp.vid[g], cp.gid[g], 0);
    cp.sbmin[pos] = cp.bmin[g];
    cp.sbmax[pos] = cp.bmax[g];
}

// buildCollisionList's query for one segment per warp.  Lanes 0-26 take the 27 cells around the
// segment's box centre; a lane whose bucket a lower lane already has drops it (every segment sits in
// exactly one bucket, so this removes exactly the repeated candidates).  A warp prefix sum of the
// bucket sizes numbers the candidates, and the lanes test them 32 at a time: groom, the
// |i - j| <= 2 exemption (collision.cu:52), box overlap, then the distance test once per pair with
// the lower boundary index first.  Accepted partners are compacted with a ballot into a shared list
// of at most 16, then sorted by partner vertex index, so the list does not depend on the order in
// which lanes found them.
constexpr int kQueryWarps = 4;
__global__ void __launch_bounds__(32 * kQueryWarps, 9) coll_query_kernel(DeviceState st, CollParams cp) {
    __shared__ int32_t s_beg[kQueryWarps][27], s_pre[kQueryWarps][28];
    __shared__ int32_t s_lst[kQueryWarps][MAX_CONTACTS], s_key[kQueryWarps][MAX_CONTACTS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t g = (int64_t)blockIdx.x * kQueryWarps + w;
    if (g >= cp.num_slots) return;  // uniform per warp
    // the segment's own operands are loaded before the bucket look-ups, so that they are in flight
    // beside them instead of after them
    const float4 loa = cp.bmin[g], hia = cp.bmax[g];
    const int32_t va = cp.vid[g], ga = cp.gid[g];
    int3 ci;
    if (!box_cell_of(cp, loa, hia, ci)) {  // uniform per warp (one segment)
        if (lane == 0) cp.ncols[g] = 0;
        return;
    }
    // a segment with a box has a next vertex in its tile, so ga1 is in bounds
    const int64_t ga1 = next_slot(g, cp.C);
    const float3 xa0 = xyz(st.xm[g]), xa1 = xyz(st.xm[ga1]);
    const uint32_t mask = (1u << cp.table_bits) - 1u;
    uint32_t h = 0xffffffffu;
    int32_t beg = 0, cnt = 0;
    if (lane < 27) {
        const int dxc = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
        h = cell_hash((uint32_t)ci.x + (uint32_t)dxc, (uint32_t)ci.y + (uint32_t)dy, (uint32_t)ci.z + (uint32_t)dz, mask);
        beg = cp.start[h];
        cnt = cp.count[h];
    }
    // a bucket that a lower lane holds too is dropped: the lanes holding the same bucket, by one match
    if (__match_any_sync(0xffffffffu, h) & ((1u << lane) - 1u)) cnt = 0;
    int32_t inc = cnt;  // inclusive prefix sum of the bucket sizes
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    const int32_t total = __shfl_sync(0xffffffffu, inc, 31);
    if (lane < 27) {
        s_beg[w][lane] = beg;
        s_pre[w][lane] = inc - cnt;
    }
    if (lane == 0) s_pre[w][27] = total;
    __syncwarp();

    const float slack = 1e-3f * cell_size(cp);  // box overlap is a pre-filter: never reject a pair the distance test keeps
    int n = 0;  // accepted so far (uniform)
    for (int32_t t0 = 0; t0 < total; t0 += 32) {
        const int32_t t = t0 + lane;
        bool hit = false;
        int32_t j = -1, vb = 0;
        if (t < total) {
            // the bucket of candidate t: the last c with s_pre[c] <= t (a binary search over the 27
            // non-decreasing prefix sums; an empty bucket shares its start with the next one)
            int c = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1)
                if (c + step <= 26 && s_pre[w][c + step] <= t) c += step;
            const int32_t k = s_beg[w][c] + (t - s_pre[w][c]);
            // the candidate's record and box in one round of loads (the box is read whether or not the
            // record's tests pass)
            const int4 rec = cp.srec[k];
            const float4 lob = cp.sbmin[k], hib = cp.sbmax[k];
            j = rec.x;
            vb = rec.y;
            bool glued = false;
            if (st.conn && j != g) {  // glued pairs are exempt (collision.cu:47-48), tested from either segment
                const int64_t ja = next_slot(j, cp.C), ta0 = st.conn[g], ta1 = st.conn[ga1], tb0 = st.conn[j],
                              tb1 = st.conn[ja];
                glued = ta0 == j || ta1 == j || ta0 == ja || ta1 == ja || tb0 == g || tb1 == g || tb0 == ga1 ||
                        tb1 == ga1;
            }
            const bool apart = (lob.x > hia.x + slack) | (loa.x > hib.x + slack) | (lob.y > hia.y + slack) |
                               (loa.y > hib.y + slack) | (lob.z > hia.z + slack) | (loa.z > hib.z + slack);
            if ((j != g) & (rec.z == ga) & (abs(vb - va) > 2) & !glued & !apart) {
                {
                    const float3 xb0 = xyz(st.xm[j]), xb1 = xyz(st.xm[next_slot(j, cp.C)]);
                    const bool af = va < vb;
                    const float3 p0 = af ? xa0 : xb0, p1 = af ? xa1 : xb1, q0 = af ? xb0 : xa0, q1 = af ? xb1 : xa1;
                    const float3 A1 = p1 - p0, B0 = q0 - p0, B1 = q1 - p0;
                    const float2 uv = seg_closest(f3(0.f, 0.f, 0.f), A1, B0, B1);
                    const float3 nrm = uv.x * A1 - mixv(B0, B1, uv.y);
                    const float d2 = len2(nrm);
                    float r = 2.f * cp.scaled_r;
                    if (cp.use_vel) {
                        r += af ? loa.w : lob.w;
                        r += af ? lob.w : loa.w;
                    }
                    hit = d2 < r * r;
                }
            }
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int slot = n + __popc(ballot & ((1u << lane) - 1u));
            if (slot < MAX_CONTACTS) {
                s_lst[w][slot] = j;
                s_key[w][slot] = vb;
            }
        }
        n += __popc(ballot);
    }
    __syncwarp();
    const int m = min(n, MAX_CONTACTS);
    if (lane == 0) {
        int32_t* lst = s_lst[w];
        int32_t* key = s_key[w];
        for (int i = 1; i < m; i++) {  // ascending partner vertex index
            const int32_t kk = key[i], vv = lst[i];
            int q = i - 1;
            while (q >= 0 && key[q] > kk) {
                key[q + 1] = key[q];
                lst[q + 1] = lst[q];
                q--;
            }
            key[q + 1] = kk;
            lst[q + 1] = vv;
        }
        cp.ncols[g] = m;
        if (n > MAX_CONTACTS) atomicOr(st.status, STATUS_CONTACTS);
    }
    __syncwarp();
    if (lane < m) cp.cols[(int64_t)lane * cp.num_slots + g] = s_lst[w][lane];
}

// Exclusive scan of int32 counts, 4096 per block (1024 threads x 4): per-block scan + block sums.
__global__ void __launch_bounds__(1024) scan_block_kernel(const int32_t* in, int32_t* out, int32_t* sums, int64_t n) {
    __shared__ int32_t warp_tot[32];
    const int64_t base = (int64_t)blockIdx.x * 4096 + (int64_t)threadIdx.x * 4;
    int32_t v[4];
    for (int i = 0; i < 4; i++) v[i] = (base + i < n) ? in[base + i] : 0;
    const int32_t tsum = v[0] + v[1] + v[2] + v[3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t incl = tsum;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int32_t wv = warp_tot[lane];
        int32_t wi = wv;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        warp_tot[lane] = wi - wv;  // exclusive offset of each warp
        if (lane == 31) sums[blockIdx.x] = wi;
    }
    __syncthreads();
    int32_t run = warp_tot[warp] + incl - tsum;
    for (int i = 0; i < 4; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

__global__ void scan_add_kernel(int32_t* out, const int32_t* offs, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / 4096];
}

cudaError_t exclusive_scan(const int32_t* in, int32_t* out, int64_t n, int32_t* tmp, cudaStream_t s) {
    const int64_t blocks = (n + 4095) / 4096;
    scan_block_kernel<<<(unsigned)blocks, 1024, 0, s>>>(in, out, tmp, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || blocks == 1) return e;
    e = exclusive_scan(tmp, tmp, blocks, tmp + blocks, s);
    if (e != cudaSuccess) return e;
    scan_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, tmp, n);
    return cudaGetLastError();
}

// ---- step limit ---------------------------------------------------------------------------------

__global__ void coll_steplimit_kernel(DeviceState st, const float4* __restrict__ dx4, CollParams cp) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= cp.num_slots) return;
    const uint32_t fl = __float_as_uint(st.prm[g].w);
    float min_dist = INFINITY;
    if (cp.limit && (fl & F_HAS_NEXT)) {
        const float margin = (1.f - 0.1f) * 0.5f;  // (1 - SAFETY_MARGIN) / 2, collision.cu:102, :126
        const float3 a0 = xyz(st.xm[g]);
        const float3 A1 = xyz(st.xm[next_slot(g, cp.C)]) - a0;
        min_dist = cp.det_r * (cp.scaler - 1.f);
        if (cp.use_vel) min_dist += sqrtf(len2(xyz(dx4[g])));
        const int n = cp.ncols[g];
        for (int k = 0; k < n; k++) {
            const int64_t o = cp.cols[(int64_t)k * cp.num_slots + g];
            const float3 B0 = xyz(st.xm[o]) - a0, B1 = xyz(st.xm[next_slot(o, cp.C)]) - a0;
            const float2 uv = seg_closest(f3(0.f, 0.f, 0.f), A1, B0, B1);
            const float l = sqrtf(len2(uv.x * A1 - mixv(B0, B1, uv.y)));
            min_dist = fminf(min_dist, margin * l);
        }
    }
    cp.maxstep[g] = min_dist;
}

// ---- position sweep with contacts -----------------------------------------------------------------

// The partner segment of one contact: its end points and their displacements at the start of the
// iteration.
struct ContactOperands {
    float3 b0, b1, db0, db1;
};
__device__ __forceinline__ ContactOperands load_contact(const DeviceState& st, const CollParams& cp,
                                                       const float4* __restrict__ snap, int64_t o) {
    const int64_t on = next_slot(o, cp.C);
    return ContactOperands{xyz(st.xm[o]), xyz(st.xm[on]), xyz(snap[o]), xyz(snap[on])};
}

// One contact of segment (x0, x1) (displacements d0, d1) with the partner segment c: the IPC barrier
// and friction terms of cosserat.cu:177-226, for the segment's first vertex (own) or its second
// vertex.  contact_eval computes everything that does not depend on the running sums (f, H);
// contact_apply adds the result to them in the reference's order: the barrier's force and Hessian,
// then friction's.  A pair that does not touch (d > 1), or has no tangential slip, carries zero
// coefficients, and contact_term skips its application.
struct ContactOut {
    float3 nrm, u;            // contact normal; tangential relative displacement
    float cf, sH, cfr, sfr;  // force along nrm, Hessian weight of nrm nrm^T; friction force along u, its Hessian weight
    bool touch;
};
__device__ __forceinline__ ContactOut contact_eval(const CollParams& cp, const ContactOperands& c, float3 x0, float3 x1,
                                                  float3 d0, float3 d1, bool own, float damp) {
    ContactOut o;
    o.nrm = f3(0.f, 0.f, 0.f);
    o.u = f3(0.f, 0.f, 0.f);
    o.cf = o.sH = o.cfr = o.sfr = 0.f;
    o.touch = false;
    const float3 b0 = c.b0, b1 = c.b1, db0 = c.db0, db1 = c.db1;
    const float2 uv = seg_closest(f3(0.f, 0.f, 0.f), (x1 - x0) + (d1 - d0), (b0 - x0) + (db0 - d0), (b1 - x0) + (db1 - d0));
    const float3 dpos = mixv(x0, x1, uv.x) - mixv(b0, b1, uv.y);
    const float3 ddpos = mixv(d0, d1, uv.x) - mixv(db0, db1, uv.y);
    float3 nrm = dpos + ddpos;
    float d = sqrtf(len2(nrm));
    nrm = nrm * (1.f / d);
    const float wt = own ? 1.f - uv.x : uv.x;
    d = d - cp.radius2;
    d *= cp.invb;
    if (d > 1.f) return o;  // not touching
    d = fmaxf(d, 1e-3f);
    const float invd = 1.f / d;
    const float logd = logf(d);
    float dH = (-3.f + (2.f + invd) * invd - 2.f * logd) * cp.kcol * cp.invb;
    const float ff = -(1.f - d) * (d - 1.f + 2.f * d * logd) * invd * cp.kcol;
    const float3 mydx = own ? d0 : d1;
    o.touch = true;
    o.nrm = nrm;
    o.cf = ff * wt - damp * dH * wt * wt * dot3(nrm, mydx);
    dH *= 1.f + damp;
    o.sH = dH * wt * wt;
    const float3 u = ddpos - dot3(nrm, ddpos) * nrm;
    const float ul = sqrtf(len2(u));
    if (ul > 0.f) {
        const float f1 = fminf(cp.kfric, cp.mu * ff / ul);
        o.u = u;
        o.cfr = f1 * wt;
        o.sfr = wt * wt * f1;
    }
    return o;
}
__device__ __forceinline__ void contact_apply(const ContactOut& o, float3& f, float H[6]) {
    const float3 nrm = o.nrm;
    f = f + o.cf * nrm;
    float op[6] = {nrm.x * nrm.x, nrm.y * nrm.y, nrm.z * nrm.z, nrm.x * nrm.y, nrm.x * nrm.z, nrm.y * nrm.z};
#pragma unroll
    for (int k = 0; k < 6; k++) H[k] += op[k] * o.sH;
    op[0] -= 1.f;
    op[1] -= 1.f;
    op[2] -= 1.f;
    f = f - o.cfr * o.u;
#pragma unroll
    for (int k = 0; k < 6; k++) H[k] -= op[k] * o.sfr;
}
__device__ __forceinline__ void contact_term(const CollParams& cp, const ContactOperands& c, float3 x0, float3 x1,
                                             float3 d0, float3 d1, bool own, float damp, float3& f, float H[6]) {
    const ContactOut o = contact_eval(cp, c, x0, x1, d0, d1, own, damp);
    if (o.touch) contact_apply(o, f, H);
}

// Every contact of the segment starting at slot g, in list order (the order of the sums is that of
// one contact at a time).  The next contact's operands are loaded before the current one is
// evaluated, so each gather overlaps the arithmetic of the contact before it.
// The per-segment contact data (count, first partner, step limit) of the vertex's segment (g) and of
// the previous one (gp) come from the caller, which can read them ahead of the sweep.
struct SegContacts {
    int n;
    int32_t first;
    float limit;
    int cached;                  // how many of the n partners' operands `part` holds (the first ones)
    const ContactOperands* part;  // shared memory (coll_iteration_kernel), or null
};
__device__ __forceinline__ SegContacts seg_contacts(const CollParams& cp, int64_t g) {
    const int n = cp.ncols[g];
    return SegContacts{n, n > 0 ? cp.cols[g] : 0, cp.maxstep[g], 0, nullptr};
}
__device__ __forceinline__ SegContacts no_contacts() { return SegContacts{0, 0, INFINITY, 0, nullptr}; }

// The segment's contacts past the first `cached` (whose partner operands the caller holds in shared
// memory), read from global memory: the next contact's operands are loaded before the current one is
// evaluated, so each gather overlaps the arithmetic of the contact before it.
__device__ __forceinline__ void contact_terms_global(const DeviceState& st, const CollParams& cp,
                                                     const float4* __restrict__ snap, int64_t g, const SegContacts& co,
                                                     float3 x0, float3 x1, float3 d0, float3 d1, bool own, float damp,
                                                     float3& f, float H[6]) {
    const int n = co.n;
    if (co.cached >= n) return;
    ContactOperands cur = load_contact(st, cp, snap, co.cached == 0 ? co.first
                                                                     : cp.cols[(int64_t)co.cached * cp.num_slots + g]);
    for (int m = co.cached; m < n; m++) {
        ContactOperands nxt = cur;
        if (m + 1 < n) nxt = load_contact(st, cp, snap, cp.cols[(int64_t)(m + 1) * cp.num_slots + g]);
        contact_term(cp, cur, x0, x1, d0, d1, own, damp, f, H);
        cur = nxt;
    }
}

// The segment's contacts (count, first partner read ahead by the caller); the first `cached` of
// them have their partner operands in shared memory already.
__device__ __forceinline__ void contact_terms(const DeviceState& st, const CollParams& cp, const float4* __restrict__ snap,
                                              int64_t g, const SegContacts& co, float3 x0, float3 x1, float3 d0,
                                              float3 d1, bool own, float damp, float3& f, float H[6]) {
    for (int m = 0; m < co.cached; m++) contact_term(cp, co.part[m], x0, x1, d0, d1, own, damp, f, H);
    contact_terms_global(st, cp, snap, g, co, x0, x1, d0, d1, own, damp, f, H);
}

// cosseratItr with contacts for one vertex (cosserat.cu:112-285), in three parts:
//  * coll_terms_next: hess3(m/h^2) and the inertial force, the connection spring, and the stretch of
//    the vertex's own segment (to the next vertex xj, dxj, orientation qg); the step limit of that
//    segment;
//  * coll_terms_prev: the stretch of the previous segment (vertex xp, dp, its prm pp4, orientation
//    qgp), into separate sums;
//  * coll_solve: the two sums added, the full 3x3 block solved with glm's adjugate inverse, and the
//    update clamped to the segments' step limit.
// Each segment's contacts (IPC barrier and friction, both ends) are added to its sums between the
// parts; coll_position does it for one vertex, the one-warp tiles of coll_iteration_kernel for the
// whole tile at once.
__device__ __forceinline__ void coll_terms_next(const DeviceState& st, const float4* snap, int64_t g, uint32_t fl,
                                                float4 xm, float4 prm, float3 vi_dx, float3 yv, float3 xj, float3 vj_dx,
                                                float4 qg, float h, const PhysParams& pp, float3& f, float H[6]) {
    const float damp = pp.damping / h;
    const float im = xm.w;
    const float3 vi = xyz(xm);
    const float inert = 1.f / (im * h * h);
#pragma unroll
    for (int n = 0; n < 6; n++) H[n] = inert;  // hess3(float) fills all six entries (SymMat.h:16-18)
    f = (1.f / (h * h * im)) * (yv - vi_dx);
    if (st.conn) {
        const int64_t t = st.conn[g];
        if (t >= 0) {  // connection spring (cosserat.cu:123-131), the partner's dx from `snap`
            constexpr float k_tie = 4e1f;
            f = f - k_tie * ((vi - xyz(st.xm[t])) + (vi_dx - xyz(__ldcg(snap + t))) + damp * vi_dx);
            const float d = k_tie * (1.f + damp);
            H[0] += d;
            H[1] += d;
            H[2] += d;
        }
    }
    if (fl & F_HAS_NEXT) {
        const float invl = 1.f / prm.x;
        const float3 cc = ((xj - vi) + (vj_dx - vi_dx)) * invl - d3_of(qg);
        const float kk = prm.y * invl;
        float dd = kk * invl;
        f = f + (kk * cc - (damp * dd) * vi_dx);
        dd *= 1.f + damp;
        H[0] += dd;
        H[1] += dd;
        H[2] += dd;
    }
}
__device__ __forceinline__ void coll_terms_prev(float3 vi, float3 vi_dx, float3 xp, float3 dp, float4 qgp, float4 pp4,
                                                float damp, float3& f2, float H2[6]) {
    const float invl = 1.f / pp4.x;
    const float3 cc = ((vi - xp) + (vi_dx - dp)) * invl - d3_of(qgp);
    const float kk = pp4.y * invl;
    float dd = kk * invl;
    f2 = (-kk) * cc - (damp * dd) * vi_dx;
    dd *= 1.f + damp;
    H2[0] = dd;
    H2[1] = dd;
    H2[2] = dd;
    H2[3] = 0.f;
    H2[4] = 0.f;
    H2[5] = 0.f;
}
__device__ __forceinline__ float3 coll_solve(float3 vi_dx, float3 f, float H[6], bool has_prev, float3 f2,
                                             const float H2[6], float step_limit, const PhysParams& pp) {
    if (has_prev) {
        f = f + f2;
#pragma unroll
        for (int q = 0; q < 6; q++) H[q] += H2[q];
    }
    const float3 delta = pp.accel_ratio * solve_sym3(H, f);
    float3 out = vi_dx + delta;
    const float l = sqrtf(len2(out));
    if (l > step_limit && l > 0.f) out = out * (step_limit / l);
    return out;
}

// cosseratItr with contacts for one vertex: the three parts with each segment's contacts, in list order
// (the order of the sums is that of one contact at a time).  The in-strand operands are the current
// iterate: the next vertex (xj, dxj), this segment's orientation qg, the previous vertex (xp, dp, its
// prm pp4) and its segment's orientation qgp; gn / gp are read only when the flags say the neighbour
// exists.  Partners' dx come from `snap`.
__device__ __forceinline__ float3 coll_position(const DeviceState& st, const CollParams& cp, const float4* snap,
                                                int64_t g, int64_t gp, uint32_t fl, float4 xm, float4 prm, float3 vi_dx,
                                                float3 yv, float3 xj, float3 vj_dx, float4 qg, float3 xp, float3 dp,
                                                float4 qgp, float4 pp4, SegContacts co, SegContacts cop, float h,
                                                const PhysParams& pp) {
    const float damp = pp.damping / h;
    const float3 vi = xyz(xm);
    float3 f;
    float H[6];
    coll_terms_next(st, snap, g, fl, xm, prm, vi_dx, yv, xj, vj_dx, qg, h, pp, f, H);
    float step_limit = INFINITY;
    if (fl & F_HAS_NEXT) {
        step_limit = co.limit;
        contact_terms(st, cp, snap, g, co, vi, xj, vi_dx, vj_dx, true, damp, f, H);
    }
    float3 f2 = f3(0.f, 0.f, 0.f);
    float H2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (fl & F_HAS_PREV) {
        coll_terms_prev(vi, vi_dx, xp, dp, qgp, pp4, damp, f2, H2);
        contact_terms(st, cp, snap, gp, cop, xp, vi, dp, vi_dx, false, damp, f2, H2);
        step_limit = fminf(step_limit, cop.limit);
    }
    return coll_solve(vi_dx, f, H, (fl & F_HAS_PREV) != 0, f2, H2, step_limit, pp);
}

// The position sweep of the sweep form with hair-hair contacts (one thread per slot of one colour,
// or of all slots under jacobi), in place (colour2) or double-buffered (jacobi) as in
// sweep_position_kernel; `snap` holds the partners' dx.
template <bool JACOBI>
__global__ void sweep_position_coll_kernel(DeviceState st, const float4* __restrict__ y4, const float4* __restrict__ qcur,
                                           const float4* dx_in, float4* dx_out, const float4* snap,
                                           const StepParams* __restrict__ spp, PhysParams pp, CollParams cp, int colour,
                                           int64_t num_threads) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_threads) return;
    const int C = cp.C;
    const int rows = JACOBI ? C : C / 2;
    // thread t: tile t / 32 rows, row r, lane t mod 32 (a 32-bit division: t / 32 < 2^32)
    const uint32_t trow = (uint32_t)((uint64_t)t >> 5);
    const int64_t tile = trow / (uint32_t)rows;
    const int r = (int)(trow - (uint32_t)tile * (uint32_t)rows), lane = (int)(t & 31);
    const int k = JACOBI ? r : 2 * r + colour;
    const int64_t g = tile * 32LL * C + (int64_t)k * 32 + lane;
    const float4 prm = st.prm[g];
    const uint32_t fl = __float_as_uint(prm.w);
    const float4 d4 = dx_in[g];
    const float4 xm = st.xm[g];
    if (!(fl & F_VALID) || xm.w == 0.f) {
        if (JACOBI) dx_out[g] = d4;
        return;
    }
    const float3 zero = f3(0.f, 0.f, 0.f);
    const float4 unit = make_float4(0.f, 0.f, 0.f, 1.f);
    float3 xj = zero, vj_dx = zero, xp = zero, dp = zero;
    float4 qgp = unit, pp4 = make_float4(1.f, 0.f, 0.f, 0.f);
    int64_t gp = g;
    if (fl & F_HAS_NEXT) {
        const int64_t gn = next_slot(g, C);
        xj = xyz(st.xm[gn]);
        vj_dx = xyz(dx_in[gn]);
    }
    if (fl & F_HAS_PREV) {
        gp = prev_slot(g, C);
        pp4 = st.prm[gp];
        xp = xyz(st.xm[gp]);
        dp = xyz(dx_in[gp]);
        qgp = qcur[gp];
    }
    const SegContacts co = (fl & F_HAS_NEXT) ? seg_contacts(cp, g) : no_contacts();
    const SegContacts cop = (fl & F_HAS_PREV) ? seg_contacts(cp, gp) : no_contacts();
    const float3 out = coll_position(st, cp, snap, g, gp, fl, xm, prm, xyz(d4), xyz(y4[g]), xj, vj_dx,
                                     (fl & F_HAS_NEXT) ? qcur[g] : unit, xp, dp, qgp, pp4, co, cop, spp->h, pp);
    dx_out[g] = make_float4(out.x, out.y, out.z, 0.f);
}

// Contacts whose partner operands coll_iteration_kernel holds in shared memory, per tile of T slots
// (2.5 per slot: at T = 64 the block's shared memory stays under 15 KB, so 14 blocks fit on an SM and
// the 2,000 tiles of a 2,000-strand groom run in one wave; one per slot at T = 1024, which keeps the
// block under the 227 KB limit).
__host__ __device__ constexpr int coll_contact_cap(int T) { return T <= 512 ? T * 5 / 2 : T; }
// Shared memory of coll_iteration_kernel: x | dx | q | prm | qr (T float4 each), the slots' contact
// data (T SegContacts), the cached contacts' operands, partner slots and segments (coll_contact_cap(T)
// each), the warps' totals; then, for tiles of several warps, the cached contacts' evaluations
// (coll_contact_cap(T) ContactOut from coll_out_offset(T), 16-byte aligned).
__host__ __device__ constexpr size_t coll_out_offset(int T) {
    return ((sizeof(float4) * 5 + sizeof(SegContacts)) * T +
            (sizeof(ContactOperands) + sizeof(int32_t) + sizeof(int16_t)) * coll_contact_cap(T) +
            sizeof(int32_t) * (T / 64) + 15) / 16 * 16;
}
__host__ __device__ constexpr size_t coll_iteration_smem(int T) {
    return T == 64 ? coll_out_offset(T) : coll_out_offset(T) + sizeof(ContactOut) * coll_contact_cap(T);
}

// A contact's evaluation passed from the lane that computed it to the lane whose sums take it.
__device__ __forceinline__ ContactOut shfl_contact(const ContactOut& o, int src) {
    ContactOut r;
    r.nrm = f3(__shfl_sync(0xffffffffu, o.nrm.x, src), __shfl_sync(0xffffffffu, o.nrm.y, src),
               __shfl_sync(0xffffffffu, o.nrm.z, src));
    r.u = f3(__shfl_sync(0xffffffffu, o.u.x, src), __shfl_sync(0xffffffffu, o.u.y, src),
             __shfl_sync(0xffffffffu, o.u.z, src));
    r.cf = __shfl_sync(0xffffffffu, o.cf, src);
    r.sH = __shfl_sync(0xffffffffu, o.sH, src);
    r.cfr = __shfl_sync(0xffffffffu, o.cfr, src);
    r.sfr = __shfl_sync(0xffffffffu, o.sfr, src);
    r.touch = __shfl_sync(0xffffffffu, (int)o.touch, src) != 0;
    return r;
}

// One colour2 iteration of the sweep form with contacts, one tile per block (T = 32 C slots, T <= 1024)
// and one thread per slot pair: thread (r, lane) owns the slots of rows 2r and 2r + 1 of that lane,
// one of each colour, so every thread works in every half-sweep.  The even and odd position sweeps,
// then the even and odd orientation sweeps, run on the tile's positions, displacements and
// orientations in shared memory, separated by __syncthreads.  Partners (other tiles) read the
// displacement the iteration started from in `snap`, which the launch does not write, so the launch
// stands for the snapshot copy and the four sweep launches (same operands and arithmetic).
// Displacements go to dx_out, orientations are updated in place.  Everything a slot's updates read
// that does not change in the launch (its parameters, rest Darboux, inertial target, contact count,
// first partner and step limit) is read once at the start.  So are the partners' operands (the
// partner segments' end points and their `snap` displacements, neither written in the launch): the
// tile's contact lists are laid end to end in shared memory, first their partner indices, then the
// operands gathered cooperatively (every thread a share of the tile's contacts, all loads
// independent), up to coll_contact_cap(T) contacts per tile; a slot's contacts past the cap are read
// from global memory in the sweep as before.  Each segment's list serves two vertices (its first as
// `own`, its second as the previous segment), so the gather halves the partner reads and takes them
// out of the sweeps' dependency chains.  The operands and the order of the sums are unchanged.
//
// ONE_WARP (tiles of 64 slots, one warp per block): a position half-sweep evaluates the tile's cached
// contacts 32 at a time, one per lane, each from its segment's end point of the half-sweep's colour
// (the first end point as `own`, the second as the previous segment), and every vertex then adds its
// own segment's and its previous segment's evaluations to its two sums in list order, taking them from
// the evaluating lanes by shuffles.  The operands, the arithmetic and the order of each sum are those
// of coll_position; what changes is that a vertex with many contacts no longer evaluates them one
// after another while the other lanes of its warp wait.  The tiles of a groom run in one wave when
// they fit, so the iteration takes as long as its slowest tile, which is the one with the most
// contacts on one vertex.  Tiles of several warps (!ONE_WARP) do the same with the block's threads
// over the tile's cached contacts and the evaluations in shared memory (coll_out_offset).
template <bool ONE_WARP>
__global__ void __launch_bounds__(512) coll_iteration_kernel(DeviceState st, const float4* __restrict__ y4, float4* q,
                                                             const float4* __restrict__ snap,
                                                             float4* __restrict__ dx_out,
                                                             const StepParams* __restrict__ spp, PhysParams pp,
                                                             CollParams cp) {
    extern __shared__ float4 coll_tile[];  // x | dx | q | prm | qr, T entries each, then the contact data
    const int C = cp.C;
    const int T = 32 * C;
    float4* sx = coll_tile;
    float4* sdx = sx + T;
    float4* sq = sdx + T;
    float4* sprm = sq + T;
    float4* sqr = sprm + T;
    SegContacts* sco = reinterpret_cast<SegContacts*>(sqr + T);
    const int ncap = coll_contact_cap(T);
    ContactOperands* spart = reinterpret_cast<ContactOperands*>(sco + T);
    int32_t* spidx = reinterpret_cast<int32_t*>(spart + ncap);  // the partners' slots, then the warps' totals
    int32_t* swarp = spidx + ncap;
    int16_t* sown = reinterpret_cast<int16_t*>(swarp + T / 64);  // each cached contact's segment (its first slot)
    const int lane = threadIdx.x & 31, row2 = (threadIdx.x >> 5) * 2;  // rows row2 (even) and row2 + 1 (odd)
    const int64_t base = (int64_t)blockIdx.x * T;
    float3 yown[2];
    SegContacts own[2];
    int32_t second[2];  // each slot's second partner (read ahead, like the first)
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;  // storage offset in the tile
        const int64_t g = base + p;
        sx[p] = st.xm[g];
        sdx[p] = snap[g];
        sq[p] = q[g];
        const float4 prm = st.prm[g];
        sprm[p] = prm;
        sqr[p] = st.qr[g];
        // the segment's contact count, first two partners and step limit, read together with the slot's
        // state instead of after its flags and count (the arrays have an entry for every slot, and the
        // query leaves no contacts on a slot without a segment)
        const int n = cp.ncols[g];
        const int32_t c0 = cp.cols[g], c1 = cp.cols[cp.num_slots + g];
        const float lim = cp.maxstep[g];
        const bool seg = __float_as_uint(prm.w) & F_HAS_NEXT;
        own[c] = seg ? SegContacts{n, n > 0 ? c0 : 0, lim, 0, nullptr} : no_contacts();
        second[c] = c1;
        yown[c] = xyz(y4[g]);
    }
    // the tile's contact lists end to end, in thread order (thread t: its even slot's list, then its
    // odd slot's): an exclusive scan of the threads' contact counts, within each warp by shuffles and
    // across the warps through swarp
    const int cnt = own[0].n + own[1].n;
    int incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    const int warp = threadIdx.x >> 5;
    if (lane == 31) swarp[warp] = incl;
    __syncthreads();
    int first_off = incl - cnt;
    for (int k = 0; k < warp; k++) first_off += swarp[k];
    int total = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) total += swarp[k];
    total = min(total, ncap);
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;
        const int off = first_off + (c ? own[0].n : 0);
        const int cached = max(0, min(own[c].n, ncap - off));
        for (int m = 0; m < cached; m++) {
            spidx[off + m] = m == 0 ? own[c].first : m == 1 ? second[c] : cp.cols[(int64_t)m * cp.num_slots + base + p];
            sown[off + m] = (int16_t)p;
        }
        own[c].cached = cached;
        own[c].part = spart + min(off, ncap);
        sco[p] = own[c];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x) spart[k] = load_contact(st, cp, snap, spidx[k]);
    const float h = spp->h;
    __syncthreads();
    if constexpr (ONE_WARP) {
        const float damp = pp.damping / h;
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
            const int p = c * 32 + lane;  // rows 0 (even) and 1 (odd): the row is the colour
            const int64_t g = base + p;
            const float4 xm = sx[p], prm = sprm[p];
            const uint32_t fl = __float_as_uint(prm.w);
            const bool act = (fl & F_VALID) && xm.w != 0.f;
            const bool hn = act && (fl & F_HAS_NEXT), hp = act && (fl & F_HAS_PREV);
            const int pn = hn ? (int)(next_slot(g, C) - base) : p;
            const int pq = hp ? (int)(prev_slot(g, C) - base) : p;
            const float3 vi = xyz(xm), vi_dx = xyz(sdx[p]), xj = xyz(sx[pn]), vj_dx = xyz(sdx[pn]);
            const float3 xp = xyz(sx[pq]), dp = xyz(sdx[pq]);
            const SegContacts co = sco[p];
            const SegContacts cop = hp ? sco[pq] : no_contacts();
            float3 f = f3(0.f, 0.f, 0.f), f2 = f3(0.f, 0.f, 0.f);
            float H[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, H2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            float step_limit = INFINITY;
            if (act) {
                coll_terms_next(st, snap, g, fl, xm, prm, vi_dx, c ? yown[1] : yown[0], xj, vj_dx, sq[p], h, pp, f, H);
                if (hn) step_limit = co.limit;
                if (hp) coll_terms_prev(vi, vi_dx, xp, dp, sq[pq], sprm[pq], damp, f2, H2);
            }
            // this vertex's cached entries: [a0, a0 + n0) of its own segment, [a1, a1 + n1) of the previous one
            const int a0 = hn ? (int)(co.part - spart) : 0, n0 = hn ? co.cached : 0;
            const int a1 = hp ? (int)(cop.part - spart) : 0, n1 = hp ? cop.cached : 0;
            for (int r0 = 0; r0 < total; r0 += 32) {  // (total is uniform)
                ContactOut o;
                o.touch = false;
                o.nrm = o.u = f3(0.f, 0.f, 0.f);
                o.cf = o.sH = o.cfr = o.sfr = 0.f;
                const int e = r0 + lane;
                if (e < total) {
                    const int s0 = sown[e];  // the contact's segment: its end points s0 and s1
                    const int s1 = (int)(next_slot(base + s0, C) - base);
                    o = contact_eval(cp, spart[e], xyz(sx[s0]), xyz(sx[s1]), xyz(sdx[s0]), xyz(sdx[s1]), (s0 >> 5) == c,
                                     damp);
                }
                const int lo0 = max(a0, r0), k0 = max(0, min(a0 + n0, r0 + 32) - lo0);
                const int lo1 = max(a1, r0), k1 = max(0, min(a1 + n1, r0 + 32) - lo1);
                const int kmax = __reduce_max_sync(0xffffffffu, max(k0, k1));
                for (int j = 0; j < kmax; j++) {
                    const ContactOut e0 = shfl_contact(o, (lo0 + j - r0) & 31);
                    const ContactOut e1 = shfl_contact(o, (lo1 + j - r0) & 31);
                    if (j < k0 && e0.touch) contact_apply(e0, f, H);
                    if (j < k1 && e1.touch) contact_apply(e1, f2, H2);
                }
            }
            if (act) {
                // contacts past the tile's cap, from global memory, after the cached ones
                if (hn) contact_terms_global(st, cp, snap, g, co, vi, xj, vi_dx, vj_dx, true, damp, f, H);
                if (hp) {
                    contact_terms_global(st, cp, snap, base + pq, cop, xp, vi, dp, vi_dx, false, damp, f2, H2);
                    step_limit = fminf(step_limit, cop.limit);
                }
                const float3 out = coll_solve(vi_dx, f, H, hp, f2, H2, step_limit, pp);
                sdx[p] = make_float4(out.x, out.y, out.z, 0.f);
            }
            __syncwarp();
        }
    } else {
        // several warps per tile: the evaluations go through shared memory (after the owner array)
        ContactOut* sout = reinterpret_cast<ContactOut*>(coll_out_offset(T) + reinterpret_cast<char*>(coll_tile));
        const float damp = pp.damping / h;
#pragma unroll 1
        for (int c = 0; c < 2; c++) {
            // the tile's cached contacts, each from its segment's end point of colour c
            for (int e = threadIdx.x; e < total; e += blockDim.x) {
                const int s0 = sown[e];
                const int s1 = (int)(next_slot(base + s0, C) - base);
                sout[e] = contact_eval(cp, spart[e], xyz(sx[s0]), xyz(sx[s1]), xyz(sdx[s0]), xyz(sdx[s1]),
                                       ((s0 >> 5) & 1) == c, damp);
            }
            __syncthreads();
            const int p = (row2 + c) * 32 + lane;
            const int64_t g = base + p;
            const float4 xm = sx[p], prm = sprm[p];
            const uint32_t fl = __float_as_uint(prm.w);
            if ((fl & F_VALID) && xm.w != 0.f) {
                // in-tile neighbours (strands never cross tiles in the sweep form)
                const bool hn = fl & F_HAS_NEXT, hp = fl & F_HAS_PREV;
                const int pn = hn ? (int)(next_slot(g, C) - base) : p;
                const int pq = hp ? (int)(prev_slot(g, C) - base) : p;
                const float3 vi = xyz(xm), vi_dx = xyz(sdx[p]), xj = xyz(sx[pn]), vj_dx = xyz(sdx[pn]);
                const float3 xp = xyz(sx[pq]), dp = xyz(sdx[pq]);
                const SegContacts co = sco[p];
                const SegContacts cop = hp ? sco[pq] : no_contacts();
                float3 f, f2 = f3(0.f, 0.f, 0.f);
                float H[6], H2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                coll_terms_next(st, snap, g, fl, xm, prm, vi_dx, c ? yown[1] : yown[0], xj, vj_dx, sq[p], h, pp, f, H);
                float step_limit = INFINITY;
                if (hn) {
                    step_limit = co.limit;
                    const ContactOut* ev = sout + (co.part - spart);
                    for (int m = 0; m < co.cached; m++)
                        if (ev[m].touch) contact_apply(ev[m], f, H);
                    contact_terms_global(st, cp, snap, g, co, vi, xj, vi_dx, vj_dx, true, damp, f, H);
                }
                if (hp) {
                    coll_terms_prev(vi, vi_dx, xp, dp, sq[pq], sprm[pq], damp, f2, H2);
                    const ContactOut* ev = sout + (cop.part - spart);
                    for (int m = 0; m < cop.cached; m++)
                        if (ev[m].touch) contact_apply(ev[m], f2, H2);
                    contact_terms_global(st, cp, snap, base + pq, cop, xp, vi, dp, vi_dx, false, damp, f2, H2);
                    step_limit = fminf(step_limit, cop.limit);
                }
                const float3 out = coll_solve(vi_dx, f, H, hp, f2, H2, step_limit, pp);
                sdx[p] = make_float4(out.x, out.y, out.z, 0.f);
            }
            __syncthreads();
        }
    }
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;
        const int64_t g = base + p;
        const float4 prm = sprm[p];
        const uint32_t fl = __float_as_uint(prm.w);
        if ((fl & F_HAS_NEXT) && !(fl & F_FIX_ORIENTATION)) {
            const int pn = (int)(next_slot(g, C) - base);
            const int pq = (fl & F_HAS_PREV) ? (int)(prev_slot(g, C) - base) : p;
            const float4 unit = make_float4(0.f, 0.f, 0.f, 1.f);
            const float4 qp = (fl & F_HAS_PREV) ? sq[pq] : unit;
            const float4 qrp = (fl & F_HAS_PREV) ? sqr[pq] : unit;
            const float4 qn = (fl & F_HAS_NEXT_ORIENTATION) ? sq[pn] : unit;
            const float m2k = -2.f * prm.y * (1.f / prm.x);
            sq[p] = vbd_orientation(sq[p], fl, xyz(sx[pn]) - xyz(sx[p]), xyz(sdx[p]), xyz(sdx[pn]), m2k, qp, qrp, qn,
                                    sqr[p]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;
        dx_out[base + p] = sdx[p];
        q[base + p] = sq[p];
    }
}

inline unsigned blocks_of(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int64_t coll_scan_tmp_size(int64_t n) {
    int64_t total = 0;
    while (n > 4096) {
        n = (n + 4095) / 4096;
        total += n;
    }
    return total + 1;
}

cudaError_t launch_coll_detect(const DeviceState& st, const float4* dx4, const CollParams& cp, cudaStream_t s) {
    const int64_t S = cp.num_slots;
    const int64_t table = 1LL << cp.table_bits;
    cudaError_t e = cudaMemsetAsync(cp.ext_bits, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    coll_box_kernel<<<blocks_of(S, 256), 256, 0, s>>>(st, dx4, cp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(cp.count, 0, sizeof(int32_t) * table, s)) != cudaSuccess) return e;
    coll_hash_kernel<<<blocks_of(S, 256), 256, 0, s>>>(cp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = exclusive_scan(cp.count, cp.start, table, cp.scan_tmp, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(cp.cursor, cp.start, sizeof(int32_t) * table, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return e;
    coll_scatter_kernel<<<blocks_of(S, 256), 256, 0, s>>>(cp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    coll_query_kernel<<<blocks_of(S, kQueryWarps), 32 * kQueryWarps, 0, s>>>(st, cp);
    return cudaGetLastError();
}

cudaError_t launch_coll_steplimit(const DeviceState& st, const float4* dx4, const CollParams& cp, cudaStream_t s) {
    coll_steplimit_kernel<<<blocks_of(cp.num_slots, 256), 256, 0, s>>>(st, dx4, cp);
    return cudaGetLastError();
}

bool coll_iteration_supported(int C) { return C % 2 == 0 && C >= 2 && 32 * C <= 1024; }

cudaError_t launch_coll_iteration(const DeviceState& st, const float4* y4, float4* q, const float4* snap, float4* dx_out,
                                  const StepParams* d_sp, const PhysParams& pp, const CollParams& cp, cudaStream_t s) {
    if (!coll_iteration_supported(cp.C)) return cudaErrorInvalidValue;
    if (!y4 || !q || !snap || !dx_out || !d_sp || snap == dx_out || !cp.cols || !cp.ncols || !cp.maxstep)
        return cudaErrorInvalidValue;
    if (st.num_tiles == 0) return cudaSuccess;
    const int T = 32 * cp.C;
    const size_t smem = coll_iteration_smem(T);
    if (cp.C == 2) {  // one warp per tile
        coll_iteration_kernel<true><<<(unsigned)st.num_tiles, T / 2, smem, s>>>(st, y4, q, snap, dx_out, d_sp, pp, cp);
        return cudaGetLastError();
    }
    if (smem > 48 * 1024) {  // the opt-in dynamic shared memory limit is set per device, so on every launch
        cudaError_t e =
            cudaFuncSetAttribute(coll_iteration_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    coll_iteration_kernel<false><<<(unsigned)st.num_tiles, T / 2, smem, s>>>(st, y4, q, snap, dx_out, d_sp, pp, cp);
    return cudaGetLastError();
}

cudaError_t launch_sweep_position_coll(const DeviceState& st, const float4* y4, const float4* q, const float4* dx_in,
                                       float4* dx_out, const float4* snap, const StepParams* d_sp, const PhysParams& pp,
                                       const CollParams& cp, int colour, bool jacobi, cudaStream_t s) {
    const int64_t n = st.num_tiles * 32LL * (jacobi ? cp.C : cp.C / 2);
    if (jacobi)
        sweep_position_coll_kernel<true><<<blocks_of(n, 128), 128, 0, s>>>(st, y4, q, dx_in, dx_out, snap, d_sp, pp, cp,
                                                                          colour, n);
    else
        sweep_position_coll_kernel<false><<<blocks_of(n, 128), 128, 0, s>>>(st, y4, q, dx_in, dx_out, snap, d_sp, pp, cp,
                                                                           colour, n);
    return cudaGetLastError();
}

}  // namespace kami
