// vbd_kernels.cu -- sm_100a kernels of the Stable Cosserat Rods VBD step.
//
// Two forms share the tile-major float4 structure-of-arrays layout of vbd_common.cuh:
//
//  * sweep form: one kernel per phase (predict; per iteration: even-vertex, odd-vertex,
//    even-segment, odd-segment sweeps; finish + SDF), each thread owning one slot and reading
//    its neighbours from global memory: the reference's kernel-per-sweep structure.  The host
//    replays the whole step from a CUDA graph, as Sim::rebuildCUDAGraph does (step.cpp:9-36).
//
//  * fused form: one kernel per step.  Each warp owns one tile (a strand, or several short
//    strands, of up to 32*C vertices) in registers for every substep and iteration; neighbour
//    coupling across lanes goes through warp shuffles.  Predict, all iterations, the velocity
//    update and the SDF projection run back to back, so HBM sees each vertex twice per step
//    (one float4 load per array, one store per dynamic array).
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "vbd_fused.cuh"
#include "vbd_kernels.h"
#include "vbd_math.cuh"

namespace kami {

// ==========================================================================================
// sweep form
// ==========================================================================================

// initItr for every slot; writes y4 = (y, 1/(invMass h^2)), dx4 = (dx, 0), vlast = v.
__global__ void sweep_predict_kernel(DeviceState st, float4* __restrict__ y4, float4* __restrict__ dx4,
                                     const StepParams* __restrict__ spp, PhysParams pp, int64_t num_slots) {
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= num_slots) return;
    const StepParams sp = *spp;
    float4 xm = st.xm[g];
    float3 v = xyz(st.vel[g]);
    float3 vl = xyz(st.vlast[g]);
    float3 dx, y;
    vbd_predict(xyz(xm), v, vl, xm.w, pp, sp.h, sp.last_h, sp.time, dx, y);
    st.vlast[g] = make_float4(v.x, v.y, v.z, 0.f);
    y4[g] = make_float4(y.x, y.y, y.z, 0.f);
    dx4[g] = make_float4(dx.x, dx.y, dx.z, 0.f);
}

// Segment constants of the segment starting at slot g (whose next slot is gn).
struct SegData {
    float3 e;
    float invl, kk, dd;
    float3 d3;
};
__device__ __forceinline__ SegData seg_data(const DeviceState& st, const float4* q, int64_t g, int64_t gn, float4 prm) {
    SegData s;
    s.e = xyz(st.xm[gn]) - xyz(st.xm[g]);
    s.invl = 1.f / prm.x;
    s.kk = prm.y * s.invl;
    s.dd = s.kk * s.invl;
    s.d3 = d3_of(q[g]);
    return s;
}

// Position sweep.  COLOUR2: threads cover the rows of one colour (k = 2r + colour), read and
// write dx in place.  JACOBI: threads cover every row, read dx_in and write dx_out.
// Tied vertices (st.conn): the connection spring of cosseratItr (cosserat.cu:123-131), stiffness 40,
// to the partner's position at the start of the step (positions do not move within it) and the
// partner's dx in conn_dx, the iteration's starting values.
template <bool JACOBI>
__global__ void sweep_position_kernel(DeviceState st, const float4* __restrict__ y4, const float4* __restrict__ qcur,
                                      const float4* dx_in, float4* dx_out, const StepParams* __restrict__ spp,
                                      PhysParams pp, int C, int colour, int64_t num_threads, const float4* conn_dx) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_threads) return;
    int rows = JACOBI ? C : C / 2;
    // thread t: tile t / 32 rows, row r, lane t mod 32 (a 32-bit division: t / 32 < 2^32)
    const uint32_t trow = (uint32_t)((uint64_t)t >> 5);
    int64_t tile = trow / (uint32_t)rows;
    int r = (int)(trow - (uint32_t)tile * (uint32_t)rows), lane = (int)(t & 31);
    int k = JACOBI ? r : 2 * r + colour;
    int64_t g = tile * 32LL * C + (int64_t)k * 32 + lane;
    float4 prm = st.prm[g];
    uint32_t fl = __float_as_uint(prm.w);
    float4 d = dx_in[g];
    float3 dx = xyz(d);
    float4 xm = st.xm[g];
    if (!(fl & F_VALID) || xm.w == 0.f) {
        if (JACOBI) dx_out[g] = d;
        return;
    }
    const float h = spp->h;
    const float damp = pp.damping / h;
    SegData sn{}, sp{};
    float3 dxn = f3(0.f, 0.f, 0.f), dxp = f3(0.f, 0.f, 0.f);
    if (fl & F_HAS_NEXT) {
        int64_t gn = next_slot(g, C);
        sn = seg_data(st, qcur, g, gn, prm);
        dxn = xyz(dx_in[gn]);
    }
    if (fl & F_HAS_PREV) {
        int64_t gp = prev_slot(g, C);
        sp = seg_data(st, qcur, gp, g, st.prm[gp]);
        dxp = xyz(dx_in[gp]);
    }
    const int64_t tie = st.conn ? st.conn[g] : -1;
    float3 nd;
    if (tie >= 0) {
        constexpr float k_tie = 4e1f;  // cosserat.cu:125
        const BlockConst bc = vbd_block_const_tied(xm.w, fl, sn.dd, sp.dd, h, damp, k_tie);
        const float3 f0 = bc.a * (xyz(y4[g]) - dx) -
                          k_tie * ((xyz(xm) - xyz(st.xm[tie])) + (dx - xyz(conn_dx[tie])) + damp * dx);
        nd = vbd_position_from(f0, dx, fl, bc, sn.e, sn.invl, sn.kk, sn.dd, sn.d3, dxn, sp.e, sp.invl, sp.kk, sp.dd,
                               sp.d3, dxp, damp, pp.accel_ratio);
    } else {
        const BlockConst bc = vbd_block_const(xm.w, fl, sn.dd, sp.dd, h, damp);
        nd = vbd_position(dx, xyz(y4[g]), fl, bc, sn.e, sn.invl, sn.kk, sn.dd, sn.d3, dxn, sp.e, sp.invl, sp.kk, sp.dd,
                          sp.d3, dxp, damp, pp.accel_ratio);
    }
    dx_out[g] = make_float4(nd.x, nd.y, nd.z, 0.f);
}

// Orientation sweep, same thread mapping as the position sweep.
template <bool JACOBI>
__global__ void sweep_orientation_kernel(DeviceState st, const float4* __restrict__ dx4, const float4* q_in,
                                         float4* q_out, int C, int colour, int64_t num_threads) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_threads) return;
    int rows = JACOBI ? C : C / 2;
    // thread t: tile t / 32 rows, row r, lane t mod 32 (a 32-bit division: t / 32 < 2^32)
    const uint32_t trow = (uint32_t)((uint64_t)t >> 5);
    int64_t tile = trow / (uint32_t)rows;
    int r = (int)(trow - (uint32_t)tile * (uint32_t)rows), lane = (int)(t & 31);
    int k = JACOBI ? r : 2 * r + colour;
    int64_t g = tile * 32LL * C + (int64_t)k * 32 + lane;
    float4 prm = st.prm[g];
    uint32_t fl = __float_as_uint(prm.w);
    float4 q = q_in[g];
    if (!(fl & F_HAS_NEXT) || (fl & F_FIX_ORIENTATION)) {
        if (JACOBI) q_out[g] = q;
        return;
    }
    int64_t gn = next_slot(g, C);
    float3 e = xyz(st.xm[gn]) - xyz(st.xm[g]);
    float3 dx = xyz(dx4[g]), dxn = xyz(dx4[gn]);
    float4 qp = make_float4(0.f, 0.f, 0.f, 1.f), qrp = qp, qn = qp;
    if (fl & F_HAS_PREV) {
        int64_t gp = prev_slot(g, C);
        qp = q_in[gp];
        qrp = st.qr[gp];
    }
    if (fl & F_HAS_NEXT_ORIENTATION) qn = q_in[gn];
    float m2k = -2.f * prm.y * (1.f / prm.x);
    q_out[g] = vbd_orientation(q, fl, e, dx, dxn, m2k, qp, qrp, qn, st.qr[g]);
}

// One colour2 iteration of the sweep form in one launch, one block per tile (T = 32 C slots,
// T <= 1024) and one thread per slot pair (rows 2r and 2r + 1 of its lane, one of each colour): the
// even and odd position sweeps of sweep_position_kernel, then the even and odd orientation sweeps of
// sweep_orientation_kernel, on the tile's positions, displacements and orientations in shared
// memory, separated by __syncthreads.  The sweep form's strands never leave their tile, so within
// an iteration a tile needs nothing of another tile but its tied partners' dx, which it reads from
// dx_in: the iteration's starting values, which the launch does not write (the snapshot the four
// launches copy).  Same operands and arithmetic as those launches, so the same results bit for bit;
// the state is read once per iteration instead of once per sweep.  dx goes to dx_out, q is updated
// in place.
__global__ void __launch_bounds__(512) sweep_iteration_kernel(DeviceState st, const float4* __restrict__ y4, float4* q,
                                                              const float4* __restrict__ dx_in,
                                                              float4* __restrict__ dx_out,
                                                              const StepParams* __restrict__ spp, PhysParams pp, int C) {
    extern __shared__ float4 sweep_tile[];  // x | dx | q | prm | qr, T entries each
    const int T = 32 * C;
    float4* sx = sweep_tile;
    float4* sdx = sx + T;
    float4* sq = sdx + T;
    float4* sprm = sq + T;
    float4* sqr = sprm + T;
    const int lane = threadIdx.x & 31, row2 = (threadIdx.x >> 5) * 2;  // rows row2 (even) and row2 + 1 (odd)
    const int64_t base = (int64_t)blockIdx.x * T;
    float3 yown[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;  // storage offset in the tile
        const int64_t g = base + p;
        sx[p] = st.xm[g];
        sdx[p] = dx_in[g];
        sq[p] = q[g];
        sprm[p] = st.prm[g];
        sqr[p] = st.qr[g];
        yown[c] = xyz(y4[g]);
    }
    const float h = spp->h;
    const float damp = pp.damping / h;
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 2; c++) {  // position sweeps: even rows, then odd rows
        const int p = (row2 + c) * 32 + lane;
        const int64_t g = base + p;
        const float4 prm = sprm[p], xm = sx[p];
        const uint32_t fl = __float_as_uint(prm.w);
        if ((fl & F_VALID) && xm.w != 0.f) {
            const float3 dx = xyz(sdx[p]);
            SegData sn{}, sp{};
            float3 dxn = f3(0.f, 0.f, 0.f), dxp = f3(0.f, 0.f, 0.f);
            if (fl & F_HAS_NEXT) {  // seg_data of the segment at g, from the tile
                const int pn = (int)(next_slot(g, C) - base);
                sn.e = xyz(sx[pn]) - xyz(xm);
                sn.invl = 1.f / prm.x;
                sn.kk = prm.y * sn.invl;
                sn.dd = sn.kk * sn.invl;
                sn.d3 = d3_of(sq[p]);
                dxn = xyz(sdx[pn]);
            }
            if (fl & F_HAS_PREV) {
                const int pq = (int)(prev_slot(g, C) - base);
                const float4 pp4 = sprm[pq];
                sp.e = xyz(xm) - xyz(sx[pq]);
                sp.invl = 1.f / pp4.x;
                sp.kk = pp4.y * sp.invl;
                sp.dd = sp.kk * sp.invl;
                sp.d3 = d3_of(sq[pq]);
                dxp = xyz(sdx[pq]);
            }
            const int64_t tie = st.conn ? st.conn[g] : -1;
            float3 nd;
            if (tie >= 0) {  // as sweep_position_kernel: the partner's dx at the start of the iteration
                constexpr float k_tie = 4e1f;  // cosserat.cu:125
                const BlockConst bc = vbd_block_const_tied(xm.w, fl, sn.dd, sp.dd, h, damp, k_tie);
                const float3 f0 = bc.a * (yown[c] - dx) -
                                  k_tie * ((xyz(xm) - xyz(st.xm[tie])) + (dx - xyz(dx_in[tie])) + damp * dx);
                nd = vbd_position_from(f0, dx, fl, bc, sn.e, sn.invl, sn.kk, sn.dd, sn.d3, dxn, sp.e, sp.invl, sp.kk,
                                       sp.dd, sp.d3, dxp, damp, pp.accel_ratio);
            } else {
                const BlockConst bc = vbd_block_const(xm.w, fl, sn.dd, sp.dd, h, damp);
                nd = vbd_position(dx, yown[c], fl, bc, sn.e, sn.invl, sn.kk, sn.dd, sn.d3, dxn, sp.e, sp.invl, sp.kk,
                                  sp.dd, sp.d3, dxp, damp, pp.accel_ratio);
            }
            sdx[p] = make_float4(nd.x, nd.y, nd.z, 0.f);
        }
        __syncthreads();
    }
    for (int c = 0; c < 2; c++) {  // orientation sweeps: even rows, then odd rows
        const int p = (row2 + c) * 32 + lane;
        const int64_t g = base + p;
        const float4 prm = sprm[p];
        const uint32_t fl = __float_as_uint(prm.w);
        if ((fl & F_HAS_NEXT) && !(fl & F_FIX_ORIENTATION)) {
            const int pn = (int)(next_slot(g, C) - base);
            const float4 unit = make_float4(0.f, 0.f, 0.f, 1.f);
            float4 qp = unit, qrp = unit, qn = unit;
            if (fl & F_HAS_PREV) {
                const int pq = (int)(prev_slot(g, C) - base);
                qp = sq[pq];
                qrp = sqr[pq];
            }
            if (fl & F_HAS_NEXT_ORIENTATION) qn = sq[pn];
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

// One Jacobi iteration of the sweep form in one launch, as sweep_iteration_kernel does colour2: every
// position from the previous iterate, then every orientation from the new displacements and the
// previous orientations (double-buffered in shared memory), as the two Jacobi launches
// (sweep_position_kernel<true>, sweep_orientation_kernel<true>) do.  Tied partners' dx come from
// dx_in, the previous iterate.  dx goes to dx_out, q to q_out.
__global__ void __launch_bounds__(512) sweep_iteration_jacobi_kernel(DeviceState st, const float4* __restrict__ y4,
                                                                     const float4* __restrict__ q_in,
                                                                     float4* __restrict__ q_out,
                                                                     const float4* __restrict__ dx_in,
                                                                     float4* __restrict__ dx_out,
                                                                     const StepParams* __restrict__ spp, PhysParams pp,
                                                                     int C) {
    extern __shared__ float4 sweep_tile[];  // x | dx | q | prm | qr | new dx | new q, T entries each
    const int T = 32 * C;
    float4* sx = sweep_tile;
    float4* sdx = sx + T;
    float4* sq = sdx + T;
    float4* sprm = sq + T;
    float4* sqr = sprm + T;
    float4* sdx2 = sqr + T;
    float4* sq2 = sdx2 + T;
    const int lane = threadIdx.x & 31, row2 = (threadIdx.x >> 5) * 2;
    const int64_t base = (int64_t)blockIdx.x * T;
    float3 yown[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;
        const int64_t g = base + p;
        sx[p] = st.xm[g];
        sdx[p] = dx_in[g];
        sq[p] = q_in[g];
        sprm[p] = st.prm[g];
        sqr[p] = st.qr[g];
        yown[c] = xyz(y4[g]);
    }
    const float h = spp->h;
    const float damp = pp.damping / h;
    __syncthreads();
    // (the updates are written out as in sweep_iteration_kernel, so that they compile to the same
    // arithmetic as the per-sweep kernels)
#pragma unroll
    for (int c = 0; c < 2; c++) {  // every position from the previous iterate
        const int p = (row2 + c) * 32 + lane;
        const int64_t g = base + p;
        const float4 prm = sprm[p], xm = sx[p];
        const uint32_t fl = __float_as_uint(prm.w);
        if ((fl & F_VALID) && xm.w != 0.f) {
            const float3 dx = xyz(sdx[p]);
            SegData sn{}, sp{};
            float3 dxn = f3(0.f, 0.f, 0.f), dxp = f3(0.f, 0.f, 0.f);
            if (fl & F_HAS_NEXT) {  // seg_data of the segment at g, from the tile
                const int pn = (int)(next_slot(g, C) - base);
                sn.e = xyz(sx[pn]) - xyz(xm);
                sn.invl = 1.f / prm.x;
                sn.kk = prm.y * sn.invl;
                sn.dd = sn.kk * sn.invl;
                sn.d3 = d3_of(sq[p]);
                dxn = xyz(sdx[pn]);
            }
            if (fl & F_HAS_PREV) {
                const int pq = (int)(prev_slot(g, C) - base);
                const float4 pp4 = sprm[pq];
                sp.e = xyz(xm) - xyz(sx[pq]);
                sp.invl = 1.f / pp4.x;
                sp.kk = pp4.y * sp.invl;
                sp.dd = sp.kk * sp.invl;
                sp.d3 = d3_of(sq[pq]);
                dxp = xyz(sdx[pq]);
            }
            const int64_t tie = st.conn ? st.conn[g] : -1;
            float3 nd;
            if (tie >= 0) {  // as sweep_position_kernel: the partner's dx at the start of the iteration
                constexpr float k_tie = 4e1f;  // cosserat.cu:125
                const BlockConst bc = vbd_block_const_tied(xm.w, fl, sn.dd, sp.dd, h, damp, k_tie);
                const float3 f0 = bc.a * (yown[c] - dx) -
                                  k_tie * ((xyz(xm) - xyz(st.xm[tie])) + (dx - xyz(dx_in[tie])) + damp * dx);
                nd = vbd_position_from(f0, dx, fl, bc, sn.e, sn.invl, sn.kk, sn.dd, sn.d3, dxn, sp.e, sp.invl, sp.kk,
                                       sp.dd, sp.d3, dxp, damp, pp.accel_ratio);
            } else {
                const BlockConst bc = vbd_block_const(xm.w, fl, sn.dd, sp.dd, h, damp);
                nd = vbd_position(dx, yown[c], fl, bc, sn.e, sn.invl, sn.kk, sn.dd, sn.d3, dxn, sp.e, sp.invl, sp.kk,
                                  sp.dd, sp.d3, dxp, damp, pp.accel_ratio);
            }
            sdx2[p] = make_float4(nd.x, nd.y, nd.z, 0.f);
        } else {
            sdx2[p] = sdx[p];
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 2; c++) {  // every orientation from the new dx and the previous q
        const int p = (row2 + c) * 32 + lane;
        const int64_t g = base + p;
        const float4 prm = sprm[p];
        const uint32_t fl = __float_as_uint(prm.w);
        if ((fl & F_HAS_NEXT) && !(fl & F_FIX_ORIENTATION)) {
            const int pn = (int)(next_slot(g, C) - base);
            const float4 unit = make_float4(0.f, 0.f, 0.f, 1.f);
            float4 qp = unit, qrp = unit, qn = unit;
            if (fl & F_HAS_PREV) {
                const int pq = (int)(prev_slot(g, C) - base);
                qp = sq[pq];
                qrp = sqr[pq];
            }
            if (fl & F_HAS_NEXT_ORIENTATION) qn = sq[pn];
            const float m2k = -2.f * prm.y * (1.f / prm.x);
            sq2[p] = vbd_orientation(sq[p], fl, xyz(sx[pn]) - xyz(sx[p]), xyz(sdx2[p]), xyz(sdx2[pn]), m2k, qp, qrp, qn,
                                     sqr[p]);
        } else {
            sq2[p] = sq[p];
        }
    }
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int p = (row2 + c) * 32 + lane;
        dx_out[base + p] = sdx2[p];
        q_out[base + p] = sq2[p];
    }
}

bool sweep_iteration_supported(int C) { return C % 2 == 0 && C >= 2 && 32 * C <= 1024; }

cudaError_t launch_sweep_iteration(const DeviceState& st, const float4* y4, const float4* q_in, float4* q_out,
                                   const float4* dx_in, float4* dx_out, const StepParams* d_sp, const PhysParams& pp,
                                   int C, bool jacobi, cudaStream_t s) {
    if (!sweep_iteration_supported(C) || !y4 || !q_in || !q_out || !dx_in || !dx_out || dx_in == dx_out || !d_sp)
        return cudaErrorInvalidValue;
    if (jacobi == (q_in == q_out)) return cudaErrorInvalidValue;  // colour2 in place, jacobi into another buffer
    if (st.num_tiles == 0) return cudaSuccess;
    const int T = 32 * C;
    const size_t smem = sizeof(float4) * (jacobi ? 7 : 5) * T;
    if (smem > 48 * 1024) {  // the opt-in limit is set per device, so on every launch
        cudaError_t e = jacobi ? cudaFuncSetAttribute(sweep_iteration_jacobi_kernel,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                               : cudaFuncSetAttribute(sweep_iteration_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)smem);
        if (e != cudaSuccess) return e;
    }
    if (jacobi)
        sweep_iteration_jacobi_kernel<<<(unsigned)st.num_tiles, T / 2, smem, s>>>(st, y4, q_in, q_out, dx_in, dx_out,
                                                                                  d_sp, pp, C);
    else
        sweep_iteration_kernel<<<(unsigned)st.num_tiles, T / 2, smem, s>>>(st, y4, q_out, dx_in, dx_out, d_sp, pp, C);
    return cudaGetLastError();
}

// endItr for every slot, then (on the last substep) the SDF pass and the finiteness check.
__global__ void sweep_finish_kernel(DeviceState st, const float4* __restrict__ dx4, const StepParams* __restrict__ spp,
                                    PhysParams pp, SdfParams sdf, int apply_sdf, int64_t num_slots) {
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (g < num_slots) {
        const StepParams sp = *spp;
        float4 xm = st.xm[g];
        uint32_t fl = __float_as_uint(st.prm[g].w);
        float3 x = xyz(xm), v = xyz(st.vel[g]);
        vbd_finish(x, v, xyz(dx4[g]), xm.w, sp.h, pp.velocity_decay);
        if (apply_sdf && sdf.grid && (fl & F_VALID) && !(fl & F_ROOT)) vbd_sdf(x, v, sdf, sp);
        st.xm[g] = make_float4(x.x, x.y, x.z, xm.w);
        st.vel[g] = make_float4(v.x, v.y, v.z, 0.f);
        if (apply_sdf) bad = !finite3(x) || !finite3(v) || !finite4(st.q[g]);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(st.status, STATUS_NONFINITE);
}

// ==========================================================================================
// fused form
// ==========================================================================================

// fused_step_kernel: see vbd_fused.cuh

// ==========================================================================================
// boundary gather / scatter (API vertex order <-> tile slots)
// ==========================================================================================
__global__ void scatter3_kernel(const float* __restrict__ src, float4* __restrict__ dst,
                                const int64_t* __restrict__ slot_of, int64_t nv) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    float4* d = dst + slot_of[i];
    float4 o = *d;
    *d = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], o.w);
}
__global__ void gather3_kernel(const float4* __restrict__ src, float* __restrict__ dst,
                               const int64_t* __restrict__ slot_of, int64_t nv) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    float4 a = src[slot_of[i]];
    dst[3 * i] = a.x;
    dst[3 * i + 1] = a.y;
    dst[3 * i + 2] = a.z;
}
__global__ void scatter4_kernel(const float4* __restrict__ src, float4* __restrict__ dst,
                                const int64_t* __restrict__ slot_of, int64_t nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    dst[slot_of[i]] = src[i];
}
__global__ void gather4_kernel(const float4* __restrict__ src, float4* __restrict__ dst,
                               const int64_t* __restrict__ slot_of, int64_t nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    dst[i] = src[slot_of[i]];
}
// Tape windows: the slots [s0, s0 + n) of a window and the boundary vertices they hold (vert_of: the
// vertex of each slot, -1 for padding).  Slot side in tile order, boundary side read and written as
// floats (its 4-vectors need not start on 16-byte boundaries, e.g. the orientations inside a state
// buffer).  `comps` is 3 (the slot's .w is kept) or 4.
__global__ void vert_of_kernel(const int64_t* __restrict__ slot_of, int64_t* __restrict__ vert_of, int64_t nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nv) vert_of[slot_of[i]] = i;
}
__global__ void scatter_slots_kernel(const float* __restrict__ src, float4* __restrict__ dst,
                                     const int64_t* __restrict__ vert_of, int64_t s0, int64_t n, int comps) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t s = s0 + t, v = vert_of[s];
    if (v < 0) return;
    if (comps == 3)
        dst[s] = make_float4(src[3 * v], src[3 * v + 1], src[3 * v + 2], dst[s].w);
    else
        dst[s] = make_float4(src[4 * v], src[4 * v + 1], src[4 * v + 2], src[4 * v + 3]);
}
__global__ void gather_slots_kernel(const float4* __restrict__ src, float* __restrict__ dst,
                                    const int64_t* __restrict__ vert_of, int64_t s0, int64_t n, int comps) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t s = s0 + t, v = vert_of[s];
    if (v < 0) return;
    const float4 a = src[s];
    dst[comps * v] = a.x;
    dst[comps * v + 1] = a.y;
    dst[comps * v + 2] = a.z;
    if (comps == 4) dst[4 * v + 3] = a.w;
}

// ==========================================================================================
// launchers
// ==========================================================================================
static inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

cudaError_t launch_sweep_predict(const DeviceState& st, float4* y4, float4* dx4, const StepParams* d_sp,
                                 const PhysParams& pp, int64_t num_slots, cudaStream_t s) {
    sweep_predict_kernel<<<blocks_for(num_slots, 256), 256, 0, s>>>(st, y4, dx4, d_sp, pp, num_slots);
    return cudaGetLastError();
}

cudaError_t launch_sweep_position(const DeviceState& st, const float4* y4, const float4* q, const float4* dx_in,
                                  float4* dx_out, const StepParams* d_sp, const PhysParams& pp, int C, int colour,
                                  bool jacobi, cudaStream_t s, const float4* conn_dx) {
    if (st.conn && !conn_dx) return cudaErrorInvalidValue;
    int64_t n = st.num_tiles * 32LL * (jacobi ? C : C / 2);
    if (jacobi)
        sweep_position_kernel<true><<<blocks_for(n, 256), 256, 0, s>>>(st, y4, q, dx_in, dx_out, d_sp, pp, C, colour, n,
                                                                       conn_dx);
    else
        sweep_position_kernel<false><<<blocks_for(n, 256), 256, 0, s>>>(st, y4, q, dx_in, dx_out, d_sp, pp, C, colour,
                                                                        n, conn_dx);
    return cudaGetLastError();
}

cudaError_t launch_sweep_orientation(const DeviceState& st, const float4* dx4, const float4* q_in, float4* q_out, int C,
                                     int colour, bool jacobi, cudaStream_t s) {
    int64_t n = st.num_tiles * 32LL * (jacobi ? C : C / 2);
    if (jacobi)
        sweep_orientation_kernel<true><<<blocks_for(n, 256), 256, 0, s>>>(st, dx4, q_in, q_out, C, colour, n);
    else
        sweep_orientation_kernel<false><<<blocks_for(n, 256), 256, 0, s>>>(st, dx4, q_in, q_out, C, colour, n);
    return cudaGetLastError();
}

cudaError_t launch_sweep_finish(const DeviceState& st, const float4* dx4, const StepParams* d_sp, const PhysParams& pp,
                                const SdfParams& sdf, bool apply_sdf, int64_t num_slots, cudaStream_t s) {
    sweep_finish_kernel<<<blocks_for(num_slots, 256), 256, 0, s>>>(st, dx4, d_sp, pp, sdf, apply_sdf ? 1 : 0, num_slots);
    return cudaGetLastError();
}

// SDFBodyCollisionSolver's StrainLimiting (SDFCollisionSolver/cudaSDFCollision.cu:176-199): one
// thread per strand marches from the root to the tip; a segment whose length l differs from its rest
// length l0 by more than strain_error * l0 has its far vertex moved along the segment by (l - l0),
// towards the near vertex as already corrected (helper_math's length and normalize: sqrtf and rsqrtf
// of the dot product).  The next vertex's position is loaded before the current segment is
// corrected: loads do not depend on the corrections, so the march is one dependent chain of
// arithmetic, not of memory latencies.
__global__ void strain_limit_kernel(float4* xm, const float4* __restrict__ prm, const int64_t* __restrict__ root_slot,
                                    const int32_t* __restrict__ strand_len, int32_t num_strands, int C,
                                    float strain_error) {
    const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= num_strands) return;
    const int32_t n = strand_len[s];
    int64_t g = root_slot[s];
    float4 cur = xm[g];
    int64_t gn = n > 1 ? next_slot(g, C) : g;
    float4 nxt = xm[gn];
    for (int32_t i = 0; i + 1 < n; i++) {
        const float l0 = prm[g].x;
        const int64_t gnn = i + 2 < n ? next_slot(gn, C) : gn;
        const float4 after = xm[gnn];  // the vertex after next, loaded ahead
        const float3 pc = xyz(cur), pn = xyz(nxt);
        const float l = sqrtf(dot3(pn - pc, pn - pc));
        if (fabsf(l - l0) > strain_error * l0) {
            const float3 d = pc - pn;
            const float3 dir = d * rsqrtf(dot3(d, d));
            const float3 q = pn + (l - l0) * dir;
            nxt = make_float4(q.x, q.y, q.z, nxt.w);
            xm[gn] = nxt;
        }
        g = gn;
        gn = gnn;
        cur = nxt;
        nxt = after;
    }
}

// The same march with the state staged in shared memory: CTA b owns slots [b S, (b + 1) S) of whole
// tile groups (so every strand rooted there lies inside), loads their positions and rest lengths
// with coalesced loads, marches the strands rooted there (cta_begin[b] .. cta_begin[b + 1] in
// root_slot, ascending) in shared memory, one thread per strand, and writes the positions back.
__global__ void __launch_bounds__(128) strain_limit_staged_kernel(float4* xm, const float4* __restrict__ prm,
                                                                 const int64_t* __restrict__ root_slot,
                                                                 const int32_t* __restrict__ strand_len,
                                                                 const int32_t* __restrict__ cta_begin,
                                                                 int64_t num_slots, int slots_per_cta, int C,
                                                                 float strain_error) {
    extern __shared__ float4 staged[];  // positions, then rest lengths
    float* sl0 = reinterpret_cast<float*>(staged + slots_per_cta);
    const int64_t s0 = (int64_t)blockIdx.x * slots_per_cta;  // a multiple of the tile size
    const int n_here = (int)min((int64_t)slots_per_cta, num_slots - s0);
    for (int i = threadIdx.x; i < n_here; i += blockDim.x) {
        staged[i] = xm[s0 + i];
        sl0[i] = prm[s0 + i].x;
    }
    __syncthreads();
    for (int32_t k = cta_begin[blockIdx.x] + (int32_t)threadIdx.x; k < cta_begin[blockIdx.x + 1]; k += blockDim.x) {
        const int32_t n = strand_len[k];
        int64_t g = root_slot[k] - s0;  // local slots keep the tile arithmetic (s0 is tile-aligned)
        float3 cur = xyz(staged[g]);
        for (int32_t i = 0; i + 1 < n; i++) {
            const int64_t gn = next_slot(g, C);
            const float4 nx = staged[gn];
            const float l0 = sl0[g];
            const float3 pn = xyz(nx);
            const float l = sqrtf(dot3(pn - cur, pn - cur));
            if (fabsf(l - l0) > strain_error * l0) {
                const float3 d = cur - pn;
                const float3 dir = d * rsqrtf(dot3(d, d));
                cur = pn + (l - l0) * dir;
                staged[gn] = make_float4(cur.x, cur.y, cur.z, nx.w);
            } else {
                cur = pn;
            }
            g = gn;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_here; i += blockDim.x) xm[s0 + i] = staged[i];
}

cudaError_t launch_strain_limit_staged(float4* xm, const float4* prm, const int64_t* root_slot,
                                       const int32_t* strand_len, const int32_t* cta_begin, int32_t num_ctas,
                                       int64_t num_slots, int slots_per_cta, int C, float strain_error, cudaStream_t s) {
    if (num_ctas <= 0) return cudaSuccess;
    const size_t smem = (sizeof(float4) + sizeof(float)) * (size_t)slots_per_cta;
    if (smem > 48 * 1024) {  // the opt-in limit is set per device, so on every launch
        cudaError_t e =
            cudaFuncSetAttribute(strain_limit_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    strain_limit_staged_kernel<<<(unsigned)num_ctas, 128, smem, s>>>(xm, prm, root_slot, strand_len, cta_begin,
                                                                    num_slots, slots_per_cta, C, strain_error);
    return cudaGetLastError();
}

cudaError_t launch_strain_limit(float4* xm, const float4* prm, const int64_t* root_slot, const int32_t* strand_len,
                                int32_t num_strands, int C, float strain_error, cudaStream_t s) {
    if (num_strands <= 0) return cudaSuccess;
    strain_limit_kernel<<<blocks_for(num_strands, 128), 128, 0, s>>>(xm, prm, root_slot, strand_len, num_strands, C,
                                                                   strain_error);
    return cudaGetLastError();
}

bool fused_supported(int C) { return C == 2 || C == 4; }

namespace {
// Launches a frame kernel: one warp per tile, 6 * 32C floats of staging per warp.
template <typename K>
cudaError_t launch_frame(K kernel, int C, const DeviceState& st, const PhysParams& pp, const StepParams& sp,
                         const SdfParams& sdf, const HostIO& hio, int warps_per_block, cudaStream_t s) {
    const size_t smem = sizeof(float) * 6 * 32 * (size_t)C * warps_per_block;
    kernel<<<blocks_for(st.num_tiles, warps_per_block), 32 * warps_per_block, smem, s>>>(st, pp, sp, sdf, hio);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_fused_frame(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                               const HostIO& hio, int C, bool jacobi, int warps_per_block, cudaStream_t s, int reg_cap,
                               int group) {
    if (group > 1) {  // one CTA of `group` warps per group of tiles
        if (group > 8 || st.num_tiles % group != 0) return cudaErrorInvalidValue;
        if (st.num_tiles == 0) return cudaSuccess;
        if (C == 2)
            return jacobi ? launch_frame(fused_frame_group_kernel<2, true>, 2, st, pp, sp, sdf, hio, group, s)
                          : launch_frame(fused_frame_group_kernel<2, false>, 2, st, pp, sp, sdf, hio, group, s);
        if (C == 4)
            return jacobi ? launch_frame(fused_frame_group_kernel<4, true>, 4, st, pp, sp, sdf, hio, group, s)
                          : launch_frame(fused_frame_group_kernel<4, false>, 4, st, pp, sp, sdf, hio, group, s);
        return cudaErrorInvalidValue;
    }
    if (blocks_for(st.num_tiles, warps_per_block) == 0) return cudaSuccess;
    if (reg_cap == 2 && C == 4 && !jacobi)
        return launch_frame(fused_frame_kernel<4, false, true>, 4, st, pp, sp, sdf, hio, warps_per_block, s);
    if (reg_cap == 120 && C == 2)
        return jacobi ? launch_frame(fused_frame_kernel_r120<2, true>, 2, st, pp, sp, sdf, hio, warps_per_block, s)
                      : launch_frame(fused_frame_kernel_r120<2, false>, 2, st, pp, sp, sdf, hio, warps_per_block, s);
    if (C == 2)
        return jacobi ? launch_frame(fused_frame_kernel<2, true, false>, 2, st, pp, sp, sdf, hio, warps_per_block, s)
                      : launch_frame(fused_frame_kernel<2, false, false>, 2, st, pp, sp, sdf, hio, warps_per_block, s);
    if (C == 4)
        return jacobi ? launch_frame(fused_frame_kernel<4, true, false>, 4, st, pp, sp, sdf, hio, warps_per_block, s)
                      : launch_frame(fused_frame_kernel<4, false, false>, 4, st, pp, sp, sdf, hio, warps_per_block, s);
    return cudaErrorInvalidValue;
}

// Resident CTAs of `kernel` at `threads` threads on the current device (cached per device, kernel
// and block size), times the SM count.
static cudaError_t resident_ctas(const void* kernel, int threads, int64_t* out) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int>, int64_t> cache;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(dev, kernel, threads);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    *out = cache[key] = (int64_t)std::max(1, per_sm) * sms;
    return cudaSuccess;
}

// The persistent grid for `units` units of work: the resident CTA count, or fewer when there are
// fewer units.  (A smaller grid that gives every CTA the same number of units was measured slower:
// the SMs then hold unequal numbers of CTAs, and the SM with the most sets the time.)
static cudaError_t persistent_grid(const void* kernel, int threads, int64_t units, unsigned* grid) {
    int64_t resident = 0;
    cudaError_t e = resident_ctas(kernel, threads, &resident);
    if (e != cudaSuccess) return e;
    *grid = (unsigned)std::min<int64_t>(units, resident);
    return cudaSuccess;
}

template <typename K>
static cudaError_t launch_persistent(K kernel, int64_t units, int threads, cudaStream_t s, const DeviceState& st,
                                     const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                                     const StepParams* d_steps, int nsteps) {
    unsigned grid = 0;
    cudaError_t e = persistent_grid((const void*)kernel, threads, units, &grid);
    if (e != cudaSuccess) return e;
    kernel<<<grid, threads, 0, s>>>(st, pp, sp, sdf, d_steps, nsteps);
    return cudaGetLastError();
}

// The persistent form of launch_fused_step (LAUNCH_PERSISTENT).
static cudaError_t launch_fused_persistent(const DeviceState& st, const PhysParams& pp, const StepParams& sp,
                                           const SdfParams& sdf, int C, bool jacobi, int warps_per_block,
                                           cudaStream_t s, const StepParams* d_steps, int nsteps, int reg_cap,
                                           int group) {
    const int W = group > 1 ? group : warps_per_block;
    const int64_t units = (st.num_tiles + W - 1) / W;
    if (units == 0) return cudaSuccess;
    const int threads = 32 * W;
#define KAMI_PERSIST(KERNEL, CC)                                                                                 \
    return jacobi ? launch_persistent(KERNEL<CC, true>, units, threads, s, st, pp, sp, sdf, d_steps, nsteps) \
                  : launch_persistent(KERNEL<CC, false>, units, threads, s, st, pp, sp, sdf, d_steps, nsteps)
    if (group > 1) {
        if (group > 8 || st.num_tiles % group != 0) return cudaErrorInvalidValue;
        if (C == 2 && reg_cap == 120) KAMI_PERSIST(fused_persistent_group_kernel_r120, 2);
        if (C == 4 && reg_cap == 168) KAMI_PERSIST(fused_persistent_group_kernel_r168, 4);
        if (C == 2) KAMI_PERSIST(fused_persistent_group_kernel, 2);
        if (C == 4) KAMI_PERSIST(fused_persistent_group_kernel, 4);
        return cudaErrorInvalidValue;
    }
    if (C == 2 && reg_cap == 120) KAMI_PERSIST(fused_persistent_kernel_r120, 2);
    if (C == 4 && reg_cap == 168) KAMI_PERSIST(fused_persistent_kernel_r168, 4);
    if (C == 2) KAMI_PERSIST(fused_persistent_kernel, 2);
    if (C == 4) KAMI_PERSIST(fused_persistent_kernel, 4);
#undef KAMI_PERSIST
    return cudaErrorInvalidValue;
}

cudaError_t launch_fused_step(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                              int C, bool jacobi, int warps_per_block, cudaStream_t s, const StepParams* d_steps,
                              int nsteps, int reg_cap, int group, int launch_mode) {
    if ((launch_mode & LAUNCH_PERSISTENT) && !(reg_cap == 2 && C == 4 && !jacobi && group <= 1))
        return launch_fused_persistent(st, pp, sp, sdf, C, jacobi, warps_per_block, s, d_steps, nsteps, reg_cap, group);
    if (group > 1) {
        if (group > 8 || st.num_tiles % group != 0) return cudaErrorInvalidValue;
        const unsigned gblocks = (unsigned)(st.num_tiles / group);
        if (gblocks == 0) return cudaSuccess;
        const int gthreads = 32 * group;
#define KAMI_GROUP_LAUNCH(KERNEL, CC)                                                                   \
    do {                                                                                                \
        if (jacobi)                                                                                     \
            KERNEL<CC, true><<<gblocks, gthreads, 0, s>>>(st, pp, sp, sdf, d_steps, nsteps);             \
        else                                                                                            \
            KERNEL<CC, false><<<gblocks, gthreads, 0, s>>>(st, pp, sp, sdf, d_steps, nsteps);            \
    } while (0)
        if (C == 2 && reg_cap == 120)
            KAMI_GROUP_LAUNCH(fused_group_kernel_r120, 2);
        else if (C == 4 && reg_cap == 168)
            KAMI_GROUP_LAUNCH(fused_group_kernel_r168, 4);
        else if (C == 2)
            KAMI_GROUP_LAUNCH(fused_group_kernel, 2);
        else if (C == 4)
            KAMI_GROUP_LAUNCH(fused_group_kernel, 4);
        else
            return cudaErrorInvalidValue;
#undef KAMI_GROUP_LAUNCH
        return cudaGetLastError();
    }
    int threads = 32 * warps_per_block;
    unsigned blocks = blocks_for(st.num_tiles, warps_per_block);
    if (blocks == 0) return cudaSuccess;
    if (reg_cap == 2 && C == 4 && !jacobi) {
        fused_step_kernel_x2<4><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, TapeView{}, d_steps, nsteps);
        return cudaGetLastError();
    }
    if (reg_cap == 168 && C == 4) {
        if (jacobi)
            fused_step_kernel_r168<4, true><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, TapeView{}, d_steps, nsteps);
        else
            fused_step_kernel_r168<4, false><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, TapeView{}, d_steps, nsteps);
        return cudaGetLastError();
    }
    if (reg_cap == 120 && C == 2) {
        if (jacobi)
            fused_step_kernel_r120<2, true><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, TapeView{}, d_steps, nsteps);
        else
            fused_step_kernel_r120<2, false><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, TapeView{}, d_steps, nsteps);
        return cudaGetLastError();
    }
    const TapeView none{};
#define KAMI_FUSED_CASE(CC)                                                                        \
    if (C == CC) {                                                                                 \
        if (jacobi)                                                                                \
            fused_step_kernel<CC, true, false><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, none, d_steps, nsteps);  \
        else                                                                                       \
            fused_step_kernel<CC, false, false><<<blocks, threads, 0, s>>>(st, pp, sp, sdf, none, d_steps, nsteps); \
        return cudaGetLastError();                                                                 \
    }
    KAMI_FUSED_CASE(2)
    KAMI_FUSED_CASE(4)
#undef KAMI_FUSED_CASE
    return cudaErrorInvalidValue;
}

// KamiSimulator's padded Hair arrays (xyz of Hair strand u, vertex v at (u * max_verts + v) * 3,
// LinearUtil.cpp:159, :247-253) <-> tile slots; hair_index[i] is the padded entry of boundary vertex i.
__global__ void hair_in_kernel(const float* __restrict__ src, float4* __restrict__ dst, const int64_t* __restrict__ slot_of,
                               const int64_t* __restrict__ hair_index, int64_t nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const int64_t p = hair_index[i];
    float4* d = dst + slot_of[i];
    const float4 o = *d;
    *d = make_float4(src[3 * p], src[3 * p + 1], src[3 * p + 2], o.w);
}
__global__ void hair_out_kernel(const float4* __restrict__ src, float* __restrict__ dst, const int64_t* __restrict__ slot_of,
                                const int64_t* __restrict__ hair_index, int64_t nv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const int64_t p = hair_index[i];
    const float4 a = src[slot_of[i]];
    dst[3 * p] = a.x;
    dst[3 * p + 1] = a.y;
    dst[3 * p + 2] = a.z;
}

cudaError_t launch_hair_in(const float* src, float4* dst, const int64_t* slot_of, const int64_t* hair_index, int64_t nv,
                           cudaStream_t s) {
    if (nv == 0) return cudaSuccess;
    hair_in_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(src, dst, slot_of, hair_index, nv);
    return cudaGetLastError();
}
cudaError_t launch_hair_out(const float4* src, float* dst, const int64_t* slot_of, const int64_t* hair_index, int64_t nv,
                            cudaStream_t s) {
    if (nv == 0) return cudaSuccess;
    hair_out_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(src, dst, slot_of, hair_index, nv);
    return cudaGetLastError();
}

cudaError_t launch_scatter3(const float* src, float4* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s) {
    if (nv == 0) return cudaSuccess;
    scatter3_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(src, dst, slot_of, nv);
    return cudaGetLastError();
}
cudaError_t launch_gather3(const float4* src, float* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s) {
    if (nv == 0) return cudaSuccess;
    gather3_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(src, dst, slot_of, nv);
    return cudaGetLastError();
}
cudaError_t launch_scatter4(const float4* src, float4* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s) {
    if (nv == 0) return cudaSuccess;
    scatter4_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(src, dst, slot_of, nv);
    return cudaGetLastError();
}
cudaError_t launch_gather4(const float4* src, float4* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s) {
    if (nv == 0) return cudaSuccess;
    gather4_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(src, dst, slot_of, nv);
    return cudaGetLastError();
}
cudaError_t launch_vert_of(const int64_t* slot_of, int64_t* vert_of, int64_t nv, int64_t num_slots, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(vert_of, 0xff, sizeof(int64_t) * num_slots, s);  // -1: padding
    if (e != cudaSuccess || nv == 0) return e;
    vert_of_kernel<<<blocks_for(nv, 256), 256, 0, s>>>(slot_of, vert_of, nv);
    return cudaGetLastError();
}
cudaError_t launch_scatter_slots(const float* src, float4* dst, const int64_t* vert_of, int64_t s0, int64_t n, int comps,
                                 cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    scatter_slots_kernel<<<blocks_for(n, 256), 256, 0, s>>>(src, dst, vert_of, s0, n, comps);
    return cudaGetLastError();
}
cudaError_t launch_gather_slots(const float4* src, float* dst, const int64_t* vert_of, int64_t s0, int64_t n, int comps,
                                cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    gather_slots_kernel<<<blocks_for(n, 256), 256, 0, s>>>(src, dst, vert_of, s0, n, comps);
    return cudaGetLastError();
}

}  // namespace kami
