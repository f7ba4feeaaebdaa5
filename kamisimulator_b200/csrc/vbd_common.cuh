// vbd_common.cuh -- device data layout, parameter blocks and small vector/quaternion helpers
// shared by the solver's kernels.
//
// Device layout ("tiles"): the solver's vertices live in tiles of T = 32*C slots, one tile per
// warp in the fused kernel.  Lane j of a tile owns the C contiguous slots p = j*C .. j*C+C-1 and
// slot p is stored at index  tile*T + (p % C)*32 + (p / C),  so the warp's access to "its k-th
// slot" is one fully coalesced 32-element row.  Strands occupy contiguous slot ranges starting
// at an even slot and padding slots carry no flags.  A strand stays in one tile, or, in a layout
// of groups of K tiles (fused form, strands longer than a tile), in one group, running on from
// lane 31's last slot of a tile into lane 0's first slot of the next.  Because every strand starts
// at an even slot and C is even, the 2-colour class of a slot (its index parity inside the strand)
// is simply k & 1 (the row parity).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace kami {

// Vertex flags: bits 1..8 are YarnBall::VertexFlags (YarnBall/YarnBall.h:33-39).
enum : uint32_t {
    F_HAS_PREV = 1u,
    F_HAS_NEXT = 2u,
    F_HAS_NEXT_ORIENTATION = 4u,
    F_FIX_ORIENTATION = 8u,
    F_ROOT = 32u,   // first vertex of its strand (skipped by the SDF pass, cudaSDFCollision.cu:241)
    F_VALID = 64u,  // a real vertex (padding slots have no flags at all)
};

// Status word bits raised by the kernels.
enum : int {
    STATUS_NONFINITE = 1,
    STATUS_CONTACTS = 2,  // a segment found more than MAX_CONTACTS hair-hair contacts
};

// Partners a segment can hold: MAX_COLLISIONS_PER_SEGMENT, YarnBall/YarnBall.h:19.
constexpr int MAX_CONTACTS = 16;

// Per-solver physical constants (MetaData scalars, YarnBall/YarnBall.h:80-123).
struct PhysParams {
    float gx, gy, gz;
    float damping;             // MetaData::damping (divided by h inside the step)
    float velocity_decay;
    float accel_ratio;
    float ext_mult;
    float wind_peak, wind_yf, wind_zf, wind_tf, wind_sharp;
    int num_itr;
};

// Per-call clock: Sim::advance splits dt into `substeps` of h; lastH is the h of the previous
// advance call and time is MetaData::time before this call (step.cpp:38-62).
struct StepParams {
    float h, last_h, time;
    int substeps;
    float rot_x, rot_y, rot_z, rot_w;  // body rotation (x, y, z, w)
    float tr_x, tr_y, tr_z;            // body translation
};

// Body SDF: (grad.xyz, phi) packed per node, x fastest.
struct SdfParams {
    const float4* grid;  // nullptr: no body collision
    int nx, ny, nz;
    float min_x, min_y, min_z;
    float ds_x, ds_y, ds_z;
    float inv_x, inv_y, inv_z;
    float thresh;
};

// Device state arrays, all indexed by tile slot.
struct DeviceState {
    float4* xm;        // position xyz, inverse mass
    float4* vel;       // velocity xyz, 0
    float4* vlast;     // velocity at the start of the previous step, 0
    float4* q;         // segment orientation (x, y, z, w)
    const float4* qr;  // rest Darboux quaternion scaled by bend/twist stiffness
    const float4* prm; // lRest, kStretch, 0, flags (bit pattern)
    int64_t num_tiles;
    int* status;
    const int64_t* conn = nullptr;  // slot each slot is tied to by a connection spring, or -1 (sweep form)
};

// Iterates of recorded steps for the adjoint: for step s, iteration it (0 = after the predict) and
// slot g, dx at dx[(s*(N+1) + it)*S + g] and q at q[(s*(N+1) + it)*S + g]; the state at the start
// of step s at x/v/vl[s*S + g].  N = iterations per step, S = slots.
// A tape may cover a window of tiles [tile_begin, DeviceState::num_tiles): slot g of tile t is then
// tape slot g - tile_begin * 32C, and `slots` is the window's slot count.
struct TapeView {
    float4* dx;
    float4* q;
    float4* x;
    float4* v;
    float4* vl;
    int64_t slots;
    int num_itr;
    int step;
    int64_t tile_begin;
};

// Host buffers that a fused step reads and writes itself (page-locked and mapped, device-visible
// addresses): positions and velocities, 3 floats per boundary vertex.  Each strand of a tile is a
// run of consecutive tile positions p (slot (p % C) * 32 + p / C of the tile) holding consecutive
// boundary vertices; runs[r] = (first position, first boundary vertex, vertex count, 0), and the
// runs of tile t are [run_begin[t], run_begin[t + 1]).
struct HostIO {
    const float* x_in;
    const float* v_in;
    float* x_out;
    float* v_out;
    const int4* runs;
    const int32_t* run_begin;
};

// Adjoint state of the solver, tile slots: d loss / d (x, v, vlast, q), and the accumulated
// d loss / d qRest.
struct AdjointState {
    float4* gx;
    float4* gv;
    float4* gvl;
    float4* gq;
    float4* gqr;
};

// Hair-hair collision: constants (MetaData, YarnBall/YarnBall.h:93-114) and the device arrays of
// detection (padded segment boxes, a spatial hash of their centres, per-segment contact lists)
// and of the step limit.  Slots are int32 here: a handle with hair-hair collision has < 2^31 slots.
struct CollParams {
    float scaled_r;  // scaledDetectionRadius = (radius + barrier / 2) * detectionScaler
    float det_r;     // detectionRadius = radius + barrier / 2
    float scaler;    // detectionScaler
    float radius2;   // 2 * radius: the contact distance before the barrier
    float invb;      // 1 / barrierThickness
    float kcol;      // kCollision / barrierThickness
    float kfric;     // kFriction
    float mu;        // frictionCoeff
    int use_vel;     // useVelocityRadius
    int limit;       // useStepSizeLimit
    const int32_t* vid;  // boundary vertex index of each slot (-1: padding)
    const int32_t* gid;  // groom of each slot (batch handles)
    int32_t* cols;       // [MAX_CONTACTS][S] partner segment (first slot), ascending by partner vid
    int32_t* ncols;      // [S]
    float* maxstep;      // [S] step limit of the segment starting at the slot
    float4* bmin;        // [S] padded box: min xyz, velocity radius
    float4* bmax;        // [S] padded box: max xyz, 1 when the slot starts a segment
    uint32_t* cell;      // [S] hash bucket of the segment's box centre
    int32_t* count;      // [table] segments per bucket
    int32_t* start;      // [table] first entry of each bucket in the bucket-ordered arrays
    int32_t* cursor;     // [table] scatter cursor
    int4* srec;          // [S] segments grouped by bucket: slot, boundary vertex index, groom
    float4* sbmin;       // [S] bmin of the same entries (bucket order)
    float4* sbmax;       // [S] bmax of the same entries (bucket order)
    unsigned* ext_bits;  // largest padded box extent (float bits): the cell size
    int32_t* scan_tmp;   // block sums of the bucket scan
    int table_bits;
    int64_t num_slots;
    int C;
};

// ---- tile slot neighbours ----------------------------------------------------------------------
// Storage index of slot p+1 / p-1 of the strand slot stored at g (the caller knows it exists).  In
// a group of tiles a strand runs on from lane 31's last slot of a tile into lane 0's first slot of
// the next tile.  Slot g sits in row (g / 32) mod C of its tile, at lane g mod 32; the row index
// needs only a 32-bit remainder (g / 32 < 2^32 for any slot count a device can hold), a mask when C
// is a power of two, instead of a 64-bit division by the tile size.
__host__ __device__ __forceinline__ int tile_row(int64_t g, int C) {
    const uint32_t row = (uint32_t)((uint64_t)g >> 5);
    return (int)((C & (C - 1)) == 0 ? row & (uint32_t)(C - 1) : row % (uint32_t)C);
}
__host__ __device__ __forceinline__ int64_t next_slot(int64_t g, int C) {
    const int k = tile_row(g, C), lane = (int)(g & 31);
    if (k < C - 1) return g + 32;
    const int64_t tile_base = g - lane - 32LL * k;
    return lane < 31 ? tile_base + lane + 1 : tile_base + 32LL * C;
}
__host__ __device__ __forceinline__ int64_t prev_slot(int64_t g, int C) {
    const int k = tile_row(g, C), lane = (int)(g & 31);
    if (k > 0) return g - 32;
    const int64_t tile_base = g - lane;
    return lane > 0 ? tile_base + 32LL * (C - 1) + lane - 1 : tile_base - 1;
}

// ---- small helpers ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
__host__ __device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__host__ __device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__host__ __device__ __forceinline__ float4 scale4(float s, float4 a) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }
__host__ __device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

// Hamilton product with the scalar last (Kit::Rotor operator*, Rotor.h:210-212).
__host__ __device__ __forceinline__ float4 qmul(float4 l, float4 r) {
    return make_float4(l.w * r.x + r.w * l.x + (l.y * r.z - r.y * l.z), l.w * r.y + r.w * l.y + (l.z * r.x - r.z * l.x),
                       l.w * r.z + r.w * l.z + (l.x * r.y - r.x * l.y), l.w * r.w - (l.x * r.x + l.y * r.y + l.z * r.z));
}
// l * conj(r)
__host__ __device__ __forceinline__ float4 qmul_conj(float4 l, float4 r) {
    return qmul(l, make_float4(-r.x, -r.y, -r.z, r.w));
}
// Material axis d3 = q e_x q* (Rotor::rotate applied to e_x, Rotor.h:114-123, expanded).
__host__ __device__ __forceinline__ float3 d3_of(float4 q) {
    return f3(q.w * q.w + q.x * q.x - q.y * q.y - q.z * q.z, 2.f * (q.x * q.y + q.w * q.z), 2.f * (q.x * q.z - q.w * q.y));
}
// Rotor::rotate (Rotor.h:114-123) for a general vector.
__host__ __device__ __forceinline__ float3 qrotate(float4 r, float3 v) {
    float3 qv = f3(r.x, r.y, r.z);
    float3 a = r.w * v + cross3(qv, v);
    float c = dot3(v, qv);
    return r.w * a + cross3(qv, a) + c * qv;
}

__device__ __forceinline__ float3 shfl_up3(float3 v, int d) {
    return f3(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d), __shfl_up_sync(0xffffffffu, v.z, d));
}
__device__ __forceinline__ float3 shfl_down3(float3 v, int d) {
    return f3(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d),
              __shfl_down_sync(0xffffffffu, v.z, d));
}
__device__ __forceinline__ float4 shfl_up4(float4 v, int d) {
    return make_float4(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d),
                       __shfl_up_sync(0xffffffffu, v.z, d), __shfl_up_sync(0xffffffffu, v.w, d));
}
__device__ __forceinline__ float4 shfl_down4(float4 v, int d) {
    return make_float4(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d),
                       __shfl_down_sync(0xffffffffu, v.z, d), __shfl_down_sync(0xffffffffu, v.w, d));
}

}  // namespace kami
