// kami_vbd.cpp -- implementation of the C ABI in include/kami_vbd.h.
#include "kami_vbd.h"

#include <cuda.h>  // CUpointer_attribute; the driver call is looked up at run time
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vbd_host.h"
#include "vbd_kernels.h"

using namespace kami;

namespace {

thread_local std::string g_last_error;

kami_status fail(kami_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

kami_status cuda_fail(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) return fail(KAMI_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(KAMI_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define KAMI_CUDA(call, what)                          \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

}  // namespace

namespace kami {
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace kami

struct kami_vbd_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;

    int64_t nv = 0;
    int32_t ns = 0;
    std::vector<int32_t> strand_begin;
    std::vector<int32_t> groom_strand_begin;  // strand offsets of the grooms of a batch handle
    TileLayout layout;
    int64_t* d_slot_of = nullptr;

    // device state (tile slots)
    float4 *d_xm = nullptr, *d_vel = nullptr, *d_vlast = nullptr, *d_q = nullptr, *d_qr = nullptr, *d_prm = nullptr;
    // sweep-form scratch
    float4 *d_y = nullptr, *d_dx = nullptr, *d_dx2 = nullptr, *d_q2 = nullptr;
    StepParams* d_step = nullptr;
    StepParams h_step{};
    // boundary staging (4 floats per boundary vertex)
    float* d_stage = nullptr;
    // frames over mapped host buffers (kami_vbd_step_host): the runs of each tile's strands, built
    // for tiles of 32 * runs_C slots
    int4* d_runs = nullptr;
    int32_t* d_run_begin = nullptr;
    int runs_C = 0;
    // the same runs addressed in the padded Hair arrays (kami_vbd_set_hair_layout): .y is the padded
    // entry of the run's first vertex; null when there is no Hair layout or it has 2^31 entries or more
    int4* d_hair_runs = nullptr;
    int* d_status = nullptr;
    float4* d_sdf = nullptr;
    SdfParams sdf{};

    PhysParams pp{};
    float h = 0.f, last_h = 0.f, time = 0.f, max_h = 4e-4f;
    float rot[4] = {0.f, 0.f, 0.f, 1.f};
    float tr[3] = {0.f, 0.f, 0.f};
    int schedule = KAMI_SCHEDULE_COLOUR2;
    int form = KAMI_FORM_FUSED;
    int warps_per_block = 4;

    cudaGraphExec_t graph = nullptr;
    int graph_substeps = -1;

    // multi-step launches (kami_vbd_step_n) and tuning
    int steps_per_launch = 8;
    int reg_cap = 0;  // 0: fused kernel without a register cap; 120 / 168: the capped variants (C = 2 / 4); 2: packed
    int launch_mode = 0;  // KAMI_LAUNCH_*: hardware-scheduled tile grid, or persistent resident CTAs
    StepParams* d_steps = nullptr;
    int d_steps_cap = 0;
    std::vector<StepParams> h_steps;
    cudaGraphExec_t graph_n = nullptr;
    int graph_n_steps = -1, graph_n_F = -1;

    // hair-hair collision (sweep form): parameters and arrays, the substep counter that paces
    // detection (Sim::stepCounter, step.cpp:52), and whether the contact lists must be rebuilt
    bool hair_hair = false;
    int detection_period = 1;
    CollParams cp{};
    int64_t counter = 0;
    bool coll_stale = true;
    float4* d_snap = nullptr;
    std::vector<char> graph_detect;  // substeps of the cached sweep graph that run detection

    // connection springs: the slot each slot is tied to (-1: none), null when no vertex is tied
    int64_t* d_conn = nullptr;

    // strain limiting (kami_vbd_strain_limit): root slot and vertex count of each strand, built on
    // the first call for the current tile layout
    int64_t* d_strand_root = nullptr;
    int32_t* d_strand_len = nullptr;
    int32_t* d_strand_cta = nullptr;  // staged form: first strand (in root order) of each CTA's slot range
    int32_t strain_ctas = 0, strain_slots_per_cta = 0;  // 0 CTAs: one thread per strand over global memory

    // device-resident Hair: padded entry of each boundary vertex, and a staging copy of a padded
    // array for host transfers
    int64_t* d_hair_index = nullptr;
    std::vector<int64_t> hair_index;  // host copy of d_hair_index
    float* d_hair_stage = nullptr;
    int64_t hair_entries = 0;  // Hair strands x max_verts

    // differentiable stepping: the tape of recorded steps and the adjoint state
    int tape_capacity = 0;
    int64_t tape_tiles = 0;               // tiles the tape holds per step
    int64_t win_begin = 0, win_end = 0;   // tile window that recording and the adjoint cover
    // the boundary vertex of every slot, -1 for padding (built when a window smaller than the groom is
    // first used, for the layout it was built on)
    int64_t* d_vert_of = nullptr;
    int vert_of_C = 0, vert_of_K = 0;
    struct TapeStep {
        StepParams sp;  // one substep (sp.substeps == 1) of a recorded advance
        bool sdf;       // the advance's last substep, which ends with the body pass
    };
    std::vector<TapeStep> tape_steps;
    float4 *d_tdx = nullptr, *d_tq = nullptr, *d_tx = nullptr, *d_tv = nullptr, *d_tvl = nullptr;
    float4 *d_gx = nullptr, *d_gv = nullptr, *d_gvl = nullptr, *d_gq = nullptr, *d_gqr = nullptr;

    TapeView tape(int step) const {
        TapeView t;
        t.dx = d_tdx;
        t.q = d_tq;
        t.x = d_tx;
        t.v = d_tv;
        t.vl = d_tvl;
        t.slots = tape_tiles * 32LL * layout.C;
        t.num_itr = pp.num_itr;
        t.step = step;
        t.tile_begin = win_begin;
        return t;
    }
    DeviceState window_state() const {  // the device state seen through the tape window
        DeviceState s = dstate();
        s.num_tiles = win_end;
        return s;
    }

    DeviceState dstate() const {
        DeviceState s;
        s.xm = d_xm;
        s.vel = d_vel;
        s.vlast = d_vlast;
        s.q = d_q;
        s.qr = d_qr;
        s.conn = d_conn;
        s.prm = d_prm;
        s.num_tiles = layout.num_tiles;
        s.status = d_status;
        return s;
    }
};

namespace {

void release(kami_vbd_solver* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->graph_n) cudaGraphExecDestroy(h->graph_n);
    if (h->d_steps) cudaFree(h->d_steps);
    void* ptrs[] = {h->d_slot_of, h->d_xm, h->d_vel, h->d_vlast, h->d_q,     h->d_qr,    h->d_prm,
                    h->d_y,       h->d_dx, h->d_dx2, h->d_q2,    h->d_step,  h->d_stage, h->d_status,
                    h->d_sdf,     h->d_tdx, h->d_tq, h->d_tx,    h->d_tv,    h->d_tvl,   h->d_gx,
                    h->d_gv,      h->d_gvl, h->d_gq, h->d_gqr,   h->d_vert_of};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    const CollParams& c = h->cp;
    void* cptrs[] = {(void*)c.vid, (void*)c.gid, c.cols,   c.ncols,  c.maxstep,  c.bmin,    c.bmax,
                     c.cell,       c.count,      c.start,  c.cursor, c.srec,     c.sbmin,    c.sbmax,
                     c.ext_bits,   c.scan_tmp,
                     h->d_snap,    h->d_hair_index, h->d_hair_stage, h->d_strand_root, h->d_strand_len, h->d_conn,
                     h->d_strand_cta};
    for (void* p : cptrs)
        if (p) cudaFree(p);
    if (h->ev_a) cudaEventDestroy(h->ev_a);
    if (h->ev_b) cudaEventDestroy(h->ev_b);
    if (h->d_runs) cudaFree(h->d_runs);
    if (h->d_run_begin) cudaFree(h->d_run_begin);
    if (h->d_hair_runs) cudaFree(h->d_hair_runs);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, sizeof(T) * (count > 0 ? count : 1));
}

// Runs `body` on the caller's stream if one is given, ordered after and before the handle's own
// stream so every other entry point (which uses the handle's stream) stays ordered with it.
template <typename F>
kami_status on_stream(kami_vbd_solver* h, void* user_stream, F body) {
    cudaStream_t us = (cudaStream_t)user_stream;
    if (!us || us == h->stream) return body(h->stream);
    KAMI_CUDA(cudaEventRecord(h->ev_a, h->stream), "cudaEventRecord");
    KAMI_CUDA(cudaStreamWaitEvent(us, h->ev_a, 0), "cudaStreamWaitEvent");
    kami_status st = body(us);
    if (st != KAMI_OK) return st;
    KAMI_CUDA(cudaEventRecord(h->ev_b, us), "cudaEventRecord");
    KAMI_CUDA(cudaStreamWaitEvent(h->stream, h->ev_b, 0), "cudaStreamWaitEvent");
    return KAMI_OK;
}

kami_status check_status_word(kami_vbd_solver* h) {
    int word = 0;
    KAMI_CUDA(cudaMemcpyAsync(&word, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "status read");
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    if (word != 0) {
        KAMI_CUDA(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream), "status reset");
        if (word & STATUS_NONFINITE)
            return fail(KAMI_ERR_NONFINITE, "non-finite position, velocity or orientation produced by a step");
        if (word & STATUS_CONTACTS)
            return fail(KAMI_ERR_CONTACTS,
                        "a segment has more than 16 hair-hair contacts (MAX_COLLISIONS_PER_SEGMENT exceeded); "
                        "the step dropped the extra contacts");
        return fail(KAMI_ERR_CUDA, "device status word 0x%x", word);
    }
    return KAMI_OK;
}

// Copies 3*nv (or 4*nv) boundary floats into the staging buffer, from host or device memory.
kami_status stage_in(kami_vbd_solver* h, const float* src, int comps, int32_t memory) {
    size_t bytes = sizeof(float) * comps * (size_t)h->nv;
    cudaMemcpyKind kind = memory == KAMI_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    KAMI_CUDA(cudaMemcpyAsync(h->d_stage, src, bytes, kind, h->stream), "copy in");
    return KAMI_OK;
}
kami_status stage_out(kami_vbd_solver* h, float* dst, int comps, int32_t memory) {
    size_t bytes = sizeof(float) * comps * (size_t)h->nv;
    cudaMemcpyKind kind = memory == KAMI_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    KAMI_CUDA(cudaMemcpyAsync(dst, h->d_stage, bytes, kind, h->stream), "copy out");
    return KAMI_OK;
}

kami_status valid_handle(kami_vbd_solver* h) {
    if (!h) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle");
    KAMI_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    return KAMI_OK;
}

#define KAMI_TRY(expr)                      \
    do {                                    \
        kami_status s_ = (expr);            \
        if (s_ != KAMI_OK) return s_;       \
    } while (0)

// Which substeps of the next step run collision detection: every detectionPeriod-th substep of the
// handle's life (step.cpp:53), and the first one after the contact lists went stale.
static std::vector<char> detect_pattern(const kami_vbd_solver* h, int substeps) {
    std::vector<char> d(substeps, 0);
    if (!h->hair_hair) return d;
    for (int sub = 0; sub < substeps; sub++)
        d[sub] = h->detection_period > 0 && (h->counter + sub) % h->detection_period == 0;
    if (h->coll_stale && h->detection_period > 0 && substeps > 0) d[0] = 1;
    return d;
}

kami_status build_sweep_graph(kami_vbd_solver* h, int substeps) {
    const std::vector<char> detect = detect_pattern(h, substeps);
    if (h->graph && h->graph_substeps == substeps && h->graph_detect == detect) return KAMI_OK;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    const DeviceState st = h->dstate();
    const bool jac = h->schedule == KAMI_SCHEDULE_JACOBI;
    const int C = h->layout.C;
    cudaStream_t s = h->stream;
    KAMI_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaError_t err = cudaSuccess;
    const size_t b4 = sizeof(float4) * h->layout.num_slots;
    for (int sub = 0; sub < substeps && err == cudaSuccess; sub++) {
        err = launch_sweep_predict(st, h->d_y, h->d_dx, h->d_step, h->pp, h->layout.num_slots, s);
        if (h->hair_hair) {
            if (err == cudaSuccess && detect[sub]) err = launch_coll_detect(st, h->d_dx, h->cp, s);
            if (err == cudaSuccess) err = launch_coll_steplimit(st, h->d_dx, h->cp, s);
        }
        float4* dx_cur = h->d_dx;
        float4* dx_alt = h->d_dx2;
        float4* q_cur = h->d_q;
        float4* q_alt = h->d_q2;
        for (int it = 0; it < h->pp.num_itr && err == cudaSuccess; it++) {
            if (jac && !h->hair_hair && h->layout.K == 1 && sweep_iteration_supported(C)) {
                // the whole iteration in one launch: dx_cur -> dx_alt, q_cur -> q_alt
                err = launch_sweep_iteration(st, h->d_y, q_cur, q_alt, dx_cur, dx_alt, h->d_step, h->pp, C, true, s);
                std::swap(dx_cur, dx_alt);
                std::swap(q_cur, q_alt);
            } else if (jac) {
                if (h->hair_hair)
                    err = launch_sweep_position_coll(st, h->d_y, q_cur, dx_cur, dx_alt, dx_cur, h->d_step, h->pp, h->cp, 0,
                                                     true, s);
                else
                    err = launch_sweep_position(st, h->d_y, q_cur, dx_cur, dx_alt, h->d_step, h->pp, C, 0, true, s,
                                                dx_cur);
                std::swap(dx_cur, dx_alt);
                if (err == cudaSuccess) err = launch_sweep_orientation(st, dx_cur, q_cur, q_alt, C, 0, true, s);
                std::swap(q_cur, q_alt);
            } else if (h->hair_hair && h->layout.K == 1 && coll_iteration_supported(C)) {
                // the whole iteration in one launch: partners read dx_cur, the result goes to the other of
                // d_dx and d_snap (a colour2 handle has no d_dx2; its snapshot buffer is free here)
                float4* other = dx_cur == h->d_dx ? h->d_snap : h->d_dx;
                err = launch_coll_iteration(st, h->d_y, q_cur, dx_cur, other, h->d_step, h->pp, h->cp, s);
                dx_cur = other;
            } else if (h->hair_hair) {
                err = cudaMemcpyAsync(h->d_snap, dx_cur, b4, cudaMemcpyDeviceToDevice, s);  // partners' dx
                for (int c = 0; c < 2 && err == cudaSuccess; c++)
                    err = launch_sweep_position_coll(st, h->d_y, q_cur, dx_cur, dx_cur, h->d_snap, h->d_step, h->pp, h->cp,
                                                     c, false, s);
                for (int c = 0; c < 2 && err == cudaSuccess; c++)
                    err = launch_sweep_orientation(st, dx_cur, q_cur, q_cur, C, c, false, s);
            } else if (h->layout.K == 1 && sweep_iteration_supported(C) && h->d_snap) {
                // the whole iteration in one launch, from dx_cur into the other of d_dx and d_snap
                float4* other = dx_cur == h->d_dx ? h->d_snap : h->d_dx;
                err = launch_sweep_iteration(st, h->d_y, q_cur, q_cur, dx_cur, other, h->d_step, h->pp, C, false, s);
                dx_cur = other;
            } else {
                if (h->d_conn)  // the tied partners' dx at the start of the iteration
                    err = cudaMemcpyAsync(h->d_snap, dx_cur, b4, cudaMemcpyDeviceToDevice, s);
                for (int c = 0; c < 2 && err == cudaSuccess; c++)
                    err = launch_sweep_position(st, h->d_y, q_cur, dx_cur, dx_cur, h->d_step, h->pp, C, c, false, s,
                                                h->d_snap);
                for (int c = 0; c < 2 && err == cudaSuccess; c++)
                    err = launch_sweep_orientation(st, dx_cur, q_cur, q_cur, C, c, false, s);
            }
        }
        if (err == cudaSuccess && q_cur != h->d_q)
            err = cudaMemcpyAsync(h->d_q, q_cur, sizeof(float4) * h->layout.num_slots, cudaMemcpyDeviceToDevice, s);
        if (err == cudaSuccess)
            err = launch_sweep_finish(st, dx_cur, h->d_step, h->pp, h->sdf, sub == substeps - 1, h->layout.num_slots, s);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (err != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(err, "capturing the sweep graph");
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
    cudaError_t e3 = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
    h->graph_substeps = substeps;
    h->graph_detect = detect;
    return KAMI_OK;
}

}  // namespace

extern "C" {

kami_status kami_vbd_desc_init(kami_vbd_desc* d) {
    if (!d) return fail(KAMI_ERR_INVALID_ARGUMENT, "null descriptor");
    std::memset(d, 0, sizeof(*d));
    d->radius = 4e-5f;
    d->density = 1300.f;
    d->stiffness_mode = KAMI_STIFFNESS_YOUNG;
    d->young = 5.f;
    d->deviation = 1.f;
    d->k_stretch = 3e3f;
    d->k_bend = 6e-4f;
    d->gravity[0] = 0.f;
    d->gravity[1] = -9.8f;
    d->gravity[2] = 0.f;
    d->damping = 1e-6f;
    d->velocity_decay = 0.05f;
    d->acceleration_ratio = 1.f;
    d->external_force_multiplier = 1.f;
    d->wind_peak = 0.f;
    d->wind_y_freq = 1.f;
    d->wind_z_freq = 0.7f;
    d->wind_time_freq = 0.4f;
    d->wind_sharpness = 3.f;
    d->num_itr = 8;
    d->max_h = 4e-4f;
    d->schedule = KAMI_SCHEDULE_COLOUR2;
    d->form = KAMI_FORM_AUTO;
    d->pin_roots = 1;
    d->device = -1;
    d->sdf = nullptr;
    d->hair_hair = 0;
    d->barrier_thickness = 2.f * (1.f - 0.05f) * 4e-5f;  // StableCosseratRodsSolver.cpp:176-180 at CurveRadius 4e-5
    d->k_collision = 1e-5f;                               // Sim::Sim, YBSimulator.cu:91-102
    d->k_friction = 5.f;
    d->friction_coeff = 0.1f;
    d->detection_scaler = 1.2f;
    d->detection_period = 1;
    d->step_limit = 1;  // StableCosseratRodsSolver.cpp:184: useStepSizeLimit = EnableHairHairColl
    d->velocity_radius = 1;
    return KAMI_OK;
}

static kami_status validate_desc(const kami_vbd_desc* d) {
    if (d->num_strands <= 0 || !d->strand_begin || !d->positions)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "need num_strands > 0, strand_begin and positions");
    if (d->strand_begin[0] != 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "strand_begin[0] must be 0");
    for (int32_t s = 0; s < d->num_strands; s++)
        if (d->strand_begin[s + 1] - d->strand_begin[s] < 2)
            return fail(KAMI_ERR_GEOMETRY, "strand %d has fewer than 2 vertices (dangling segment)", s);
    if (d->num_itr < 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "num_itr must be >= 0");
    if (!(d->max_h > 0.f)) return fail(KAMI_ERR_INVALID_ARGUMENT, "max_h must be > 0");
    if (!(d->radius > 0.f) || !(d->density > 0.f)) return fail(KAMI_ERR_INVALID_ARGUMENT, "radius and density must be > 0");
    if (d->schedule != KAMI_SCHEDULE_COLOUR2 && d->schedule != KAMI_SCHEDULE_JACOBI)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "unknown schedule %d", d->schedule);
    if (d->form < KAMI_FORM_AUTO || d->form > KAMI_FORM_FUSED) return fail(KAMI_ERR_INVALID_ARGUMENT, "unknown form %d", d->form);
    if (d->stiffness_mode != KAMI_STIFFNESS_YOUNG && d->stiffness_mode != KAMI_STIFFNESS_K)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "unknown stiffness mode %d", d->stiffness_mode);
    if (d->sdf) {
        const kami_vbd_sdf_desc* s = d->sdf;
        if (s->dims[0] <= 0 || s->dims[1] <= 0 || s->dims[2] <= 0 || !s->phi || !s->grad)
            return fail(KAMI_ERR_INVALID_ARGUMENT, "SDF needs positive dims and phi/grad arrays");
        for (int a = 0; a < 3; a++)
            if (!(s->grid_max[a] > s->grid_min[a])) return fail(KAMI_ERR_INVALID_ARGUMENT, "SDF grid_max must exceed grid_min");
    }
    if (d->sag_free_itr < 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "sag_free_itr must be >= 0");
    if (d->connection_index) {
        const int32_t nv = d->strand_begin[d->num_strands];
        bool tied = false;
        for (int32_t i = 0; i < nv; i++) {
            const int32_t c = d->connection_index[i];
            if (c < -1 || c >= nv || c == i)
                return fail(KAMI_ERR_INVALID_ARGUMENT,
                            "connection_index[%d] = %d: must be -1 or another vertex of the groom (0..%d)", i, c, nv - 1);
            tied |= c >= 0;
        }
        if (tied && d->form == KAMI_FORM_FUSED)
            return fail(KAMI_ERR_UNSUPPORTED, "connection springs run on the sweep form (a tie may join two tiles)");
    }
    if (d->hair_hair) {
        if (!(d->barrier_thickness > 0.f)) return fail(KAMI_ERR_INVALID_ARGUMENT, "barrier_thickness must be > 0");
        if (!(d->detection_scaler > 1.f))  // Sim::uploadMeta, YBSimulator.cu:326
            return fail(KAMI_ERR_INVALID_ARGUMENT, "detection_scaler must be greater than 1");
        if (!(d->k_collision >= 0.f) || !(d->k_friction >= 0.f) || !(d->friction_coeff >= 0.f))
            return fail(KAMI_ERR_INVALID_ARGUMENT, "collision stiffness and friction must be >= 0");
        if (d->form == KAMI_FORM_FUSED)
            return fail(KAMI_ERR_UNSUPPORTED, "hair-hair collision runs on the sweep form (strands of one warp tile "
                                              "meet partners in other tiles)");
    }
    return KAMI_OK;
}

// The settings one handle applies to all its strands: grooms of a batch must agree on them.
static const char* differing_setting(const kami_vbd_desc* a, const kami_vbd_desc* b) {
    for (int i = 0; i < 3; i++)
        if (a->gravity[i] != b->gravity[i]) return "gravity";
    if (a->damping != b->damping) return "damping";
    if (a->velocity_decay != b->velocity_decay) return "velocity_decay";
    if (a->acceleration_ratio != b->acceleration_ratio) return "acceleration_ratio";
    if (a->external_force_multiplier != b->external_force_multiplier) return "external_force_multiplier";
    if (a->wind_peak != b->wind_peak || a->wind_y_freq != b->wind_y_freq || a->wind_z_freq != b->wind_z_freq ||
        a->wind_time_freq != b->wind_time_freq || a->wind_sharpness != b->wind_sharpness)
        return "wind";
    if (a->num_itr != b->num_itr) return "num_itr";
    if (a->max_h != b->max_h) return "max_h";
    if (a->schedule != b->schedule) return "schedule";
    if (a->form != b->form) return "form";
    if (a->device != b->device) return "device";
    if (a->slots_per_lane != b->slots_per_lane || a->warps_per_block != b->warps_per_block) return "tile shape";
    if (a->hair_hair != b->hair_hair) return "hair_hair";
    if (a->sag_free_itr != b->sag_free_itr) return "sag_free_itr";
    if (a->hair_hair &&
        (a->radius != b->radius || a->barrier_thickness != b->barrier_thickness || a->k_collision != b->k_collision ||
         a->k_friction != b->k_friction || a->friction_coeff != b->friction_coeff ||
         a->detection_scaler != b->detection_scaler || a->detection_period != b->detection_period ||
         a->step_limit != b->step_limit || a->velocity_radius != b->velocity_radius))
        return "radius or hair-hair collision settings";
    if ((a->sdf == nullptr) != (b->sdf == nullptr)) return "sdf";
    if (a->sdf && a->sdf != b->sdf) {
        const kami_vbd_sdf_desc *x = a->sdf, *y = b->sdf;
        for (int i = 0; i < 3; i++)
            if (x->dims[i] != y->dims[i] || x->grid_min[i] != y->grid_min[i] || x->grid_max[i] != y->grid_max[i])
                return "sdf";
        if (x->threshold != y->threshold || x->phi != y->phi || x->grad != y->grad) return "sdf";
    }
    return nullptr;
}

// Hair-hair collision arrays: per-slot boundary vertex and groom indices, contact lists, step
// limits, boxes and the spatial hash (a power-of-two table of at least twice the slot count).
static kami_status setup_collisions(kami_vbd_solver* h, const kami_vbd_desc* d) {
    const int64_t S = h->layout.num_slots;
    if (S >= INT32_MAX) return fail(KAMI_ERR_UNSUPPORTED, "hair-hair collision supports fewer than 2^31 slots");
    h->hair_hair = true;
    h->detection_period = d->detection_period;
    CollParams& c = h->cp;
    c.det_r = d->radius + 0.5f * d->barrier_thickness;  // Sim::uploadMeta, YBSimulator.cu:323-324
    c.scaled_r = c.det_r * d->detection_scaler;
    c.scaler = d->detection_scaler;
    c.radius2 = 2.f * d->radius;
    c.invb = 1.f / d->barrier_thickness;
    c.kcol = d->k_collision * c.invb;
    c.kfric = d->k_friction;
    c.mu = d->friction_coeff;
    c.use_vel = d->velocity_radius != 0;
    c.limit = d->step_limit != 0;
    c.num_slots = S;
    c.C = h->layout.C;
    int bits = 10;
    while ((1LL << bits) < 2 * S && bits < 30) bits++;
    c.table_bits = bits;
    const int64_t table = 1LL << bits;
    std::vector<int32_t> vid(S, -1), gid(S, -1);
    const int32_t ng = (int32_t)h->groom_strand_begin.size() - 1;
    for (int32_t g = 0; g < ng; g++)
        for (int64_t i = h->strand_begin[h->groom_strand_begin[g]]; i < h->strand_begin[h->groom_strand_begin[g + 1]]; i++) {
            vid[h->layout.slot_of[i]] = (int32_t)i;
            gid[h->layout.slot_of[i]] = g;
        }
    int32_t *dvid = nullptr, *dgid = nullptr;
    cudaError_t e = dalloc(&dvid, S);
    if (e == cudaSuccess) e = dalloc(&dgid, S);
    c.vid = dvid;
    c.gid = dgid;
    if (e == cudaSuccess) e = dalloc(&c.cols, (size_t)MAX_CONTACTS * S);
    if (e == cudaSuccess) e = dalloc(&c.ncols, S);
    if (e == cudaSuccess) e = dalloc(&c.maxstep, S);
    if (e == cudaSuccess) e = dalloc(&c.bmin, S);
    if (e == cudaSuccess) e = dalloc(&c.bmax, S);
    if (e == cudaSuccess) e = dalloc(&c.cell, S);
    if (e == cudaSuccess) e = dalloc(&c.count, table);
    if (e == cudaSuccess) e = dalloc(&c.start, table);
    if (e == cudaSuccess) e = dalloc(&c.cursor, table);
    if (e == cudaSuccess) e = dalloc(&c.srec, S);
    if (e == cudaSuccess) e = dalloc(&c.sbmin, S);
    if (e == cudaSuccess) e = dalloc(&c.sbmax, S);
    if (e == cudaSuccess) e = dalloc(&c.ext_bits, 1);
    if (e == cudaSuccess) e = dalloc(&c.scan_tmp, coll_scan_tmp_size(table));
    if (e == cudaSuccess && h->schedule == KAMI_SCHEDULE_COLOUR2 && !h->d_snap) e = dalloc(&h->d_snap, S);
    if (e != cudaSuccess) return cuda_fail(e, "allocating hair-hair collision arrays");
    e = cudaMemcpy(dvid, vid.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dgid, gid.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(c.ncols, 0, sizeof(int32_t) * S);
    if (e != cudaSuccess) return cuda_fail(e, "uploading hair-hair collision arrays");
    h->coll_stale = true;
    return KAMI_OK;
}

// Builds one handle over the strands of n descriptors (n = 1: kami_vbd_create).  Each groom's
// material is set up on its own, as one YarnBall::Sim per groom would do it; the solver-wide
// settings come from the first descriptor.
static kami_status create_impl(const kami_vbd_desc* descs, int32_t n, kami_vbd_handle* out) {
    if (!descs || !out || n <= 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "null descriptor or output handle");
    *out = nullptr;
    for (int32_t g = 0; g < n; g++) {
        KAMI_TRY(validate_desc(&descs[g]));
        if (const char* what = differing_setting(&descs[0], &descs[g]))
            return fail(KAMI_ERR_INVALID_ARGUMENT, "groom %d differs from groom 0 in %s", g, what);
    }
    const kami_vbd_desc* d = &descs[0];

    kami_vbd_solver* h = new (std::nothrow) kami_vbd_solver();
    if (!h) return fail(KAMI_ERR_OUT_OF_MEMORY, "host allocation failed");
    auto bail = [&](kami_status st) {
        release(h);
        return st;
    };
    int64_t total_strands = 0, total_vertices = 0;
    for (int32_t g = 0; g < n; g++) {
        total_strands += descs[g].num_strands;
        total_vertices += descs[g].strand_begin[descs[g].num_strands];
    }
    if (total_strands > INT32_MAX || total_vertices > INT32_MAX)
        return bail(fail(KAMI_ERR_UNSUPPORTED, "a handle holds at most 2^31 - 1 strands and vertices"));
    h->ns = (int32_t)total_strands;
    h->strand_begin.assign(1, 0);
    h->strand_begin.reserve(total_strands + 1);
    h->groom_strand_begin.assign(1, 0);

    // per-vertex positions, velocities and material in boundary order, groom after groom
    std::vector<float> positions, velocities;
    positions.reserve(3 * total_vertices);
    velocities.reserve(3 * total_vertices);
    Material m;
    std::vector<int32_t> ties;  // boundary vertex each vertex is tied to, or -1 (empty: no tie)
    for (int32_t g = 0; g < n; g++) {
        const kami_vbd_desc* e = &descs[g];
        const int32_t base = h->strand_begin.back();
        if (e->connection_index) {
            const int32_t nvg = e->strand_begin[e->num_strands];
            for (int32_t i = 0; i < nvg; i++)
                if (e->connection_index[i] >= 0) {
                    if (ties.empty()) ties.assign(total_vertices, -1);
                    ties[base + i] = base + e->connection_index[i];
                }
        }
        for (int32_t s = 1; s <= e->num_strands; s++) h->strand_begin.push_back(base + e->strand_begin[s]);
        h->groom_strand_begin.push_back(h->groom_strand_begin.back() + e->num_strands);
        const int32_t nvg = e->strand_begin[e->num_strands];
        positions.insert(positions.end(), e->positions, e->positions + 3 * (size_t)nvg);
        if (e->velocities)
            velocities.insert(velocities.end(), e->velocities, e->velocities + 3 * (size_t)nvg);
        else
            velocities.insert(velocities.end(), 3 * (size_t)nvg, 0.f);
        MaterialDesc md;
        md.radius = e->radius;
        md.density = e->density;
        md.stiffness_mode = e->stiffness_mode;
        md.strand_young = e->strand_young;
        md.strand_dev = e->strand_deviation;
        md.young = e->young;
        md.deviation = e->deviation;
        md.k_stretch = e->k_stretch;
        md.k_bend = e->k_bend;
        md.pin_roots = e->pin_roots != 0;
        Material mg;
        std::string err;
        int rc = build_material(e->strand_begin, e->num_strands, e->positions, md, mg, err);
        if (rc != 0) {
            if (n > 1) err = "groom " + std::to_string(g) + ": " + err;
            return bail(fail(rc == 1 ? KAMI_ERR_INVALID_ARGUMENT : KAMI_ERR_GEOMETRY, "%s", err.c_str()));
        }
        m.inv_mass.insert(m.inv_mass.end(), mg.inv_mass.begin(), mg.inv_mass.end());
        m.l_rest.insert(m.l_rest.end(), mg.l_rest.begin(), mg.l_rest.end());
        m.k_stretch.insert(m.k_stretch.end(), mg.k_stretch.begin(), mg.k_stretch.end());
        m.flags.insert(m.flags.end(), mg.flags.begin(), mg.flags.end());
        m.q.insert(m.q.end(), mg.q.begin(), mg.q.end());
        m.q_rest.insert(m.q_rest.end(), mg.q_rest.begin(), mg.q_rest.end());
    }
    h->nv = h->strand_begin.back();
    std::string err;

    // tile layout and form
    int C = slots_per_lane_for(h->strand_begin.data(), h->ns);
    if (d->slots_per_lane != 0) {
        if (d->slots_per_lane < C || (d->slots_per_lane & 1))
            return bail(fail(KAMI_ERR_INVALID_ARGUMENT, "slots_per_lane %d must be even and >= %d for these strands",
                             d->slots_per_lane, C));
        C = d->slots_per_lane;
    }
    if (d->warps_per_block < 0 || d->warps_per_block > 32 || (d->warps_per_block & (d->warps_per_block - 1)))
        return bail(fail(KAMI_ERR_INVALID_ARGUMENT, "warps_per_block must be 0 or a power of two <= 32"));
    if (d->warps_per_block > 0) h->warps_per_block = d->warps_per_block;
    // the fused form runs strands longer than a tile of 4 slots per lane on groups of up to 8 tiles
    int K = 1;
    if (!fused_supported(C) && d->slots_per_lane == 0 && tiles_per_group_for(h->strand_begin.data(), h->ns, 4) > 0) {
        if (d->form != KAMI_FORM_SWEEP && !d->hair_hair && ties.empty()) {
            C = 4;
            K = tiles_per_group_for(h->strand_begin.data(), h->ns, 4);
        }
    }
    int form = d->form;
    if (form == KAMI_FORM_AUTO)
        form = (fused_supported(C) && !d->hair_hair && ties.empty()) ? KAMI_FORM_FUSED : KAMI_FORM_SWEEP;
    if (d->hair_hair) {
        // Sim::uploadMeta (YBSimulator.cu:328-332): contacts must fit between a segment's ends
        float min_seg = FLT_MAX;
        for (int64_t i = 0; i < h->nv; i++)
            if (m.flags[i] & F_HAS_NEXT) min_seg = std::min(min_seg, m.l_rest[i]);
        if (2.f * min_seg < 2.f * d->radius + d->barrier_thickness)
            return bail(fail(KAMI_ERR_GEOMETRY,
                             "use thinner strands or longer segments: 2 x shortest segment (%g) must be >= "
                             "2 x radius + barrier_thickness (%g)",
                             2.0 * min_seg, 2.0 * d->radius + d->barrier_thickness));
    }
    if (form == KAMI_FORM_FUSED && !fused_supported(C))
        return bail(fail(KAMI_ERR_UNSUPPORTED, "fused form supports strands of up to 1024 vertices (8 tiles of 128)"));
    h->form = form;
    if (!pack_tiles(h->strand_begin.data(), h->ns, C, h->layout, err, form == KAMI_FORM_FUSED ? K : 1))
        return bail(fail(KAMI_ERR_UNSUPPORTED, "%s", err.c_str()));
    const int64_t S = h->layout.num_slots;

    // everything above is host-only validation; device work starts here
    if (d->device >= 0) {
        cudaError_t e = cudaSetDevice(d->device);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaSetDevice"));
        h->device = d->device;
    } else {
        cudaError_t e = cudaGetDevice(&h->device);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaGetDevice"));
    }

    // host images of the device arrays (padding slots: lRest 1, no flags, zero mass)
    std::vector<float4> xm(S, make_float4(0.f, 0.f, 0.f, 0.f)), vel(S, make_float4(0.f, 0.f, 0.f, 0.f)),
        vlast(S, make_float4(0.f, 0.f, 0.f, 0.f)), q(S, make_float4(0.f, 0.f, 0.f, 1.f)),
        qr(S, make_float4(0.f, 0.f, 0.f, 1.f)), prm(S, make_float4(1.f, 0.f, 0.f, 0.f));
    for (int64_t i = 0; i < h->nv; i++) {
        const int64_t g = h->layout.slot_of[i];
        xm[g] = make_float4(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], m.inv_mass[i]);
        vel[g] = make_float4(velocities[3 * i], velocities[3 * i + 1], velocities[3 * i + 2], 0.f);
        q[g] = make_float4(m.q[4 * i], m.q[4 * i + 1], m.q[4 * i + 2], m.q[4 * i + 3]);
        qr[g] = make_float4(m.q_rest[4 * i], m.q_rest[4 * i + 1], m.q_rest[4 * i + 2], m.q_rest[4 * i + 3]);
        uint32_t fl = m.flags[i];
        float flf;
        std::memcpy(&flf, &fl, 4);
        prm[g] = make_float4(m.l_rest[i], m.k_stretch[i], 0.f, flf);
    }

    // physical parameters and clock (meta.h starts at maxH, YBSimulator.cu:85)
    h->pp.gx = d->gravity[0];
    h->pp.gy = d->gravity[1];
    h->pp.gz = d->gravity[2];
    h->pp.damping = d->damping;
    h->pp.velocity_decay = d->velocity_decay;
    h->pp.accel_ratio = d->acceleration_ratio;
    h->pp.ext_mult = d->external_force_multiplier;
    h->pp.wind_peak = d->wind_peak;
    h->pp.wind_yf = d->wind_y_freq;
    h->pp.wind_zf = d->wind_z_freq;
    h->pp.wind_tf = d->wind_time_freq;
    h->pp.wind_sharp = d->wind_sharpness;
    h->pp.num_itr = d->num_itr;
    h->max_h = d->max_h;
    h->h = d->max_h;
    h->schedule = d->schedule;

    // a blocking stream, so work on the legacy default stream (e.g. a torch producer) orders with ours
    cudaError_t e = cudaStreamCreate(&h->stream);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_a, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_b, cudaEventDisableTiming);
    if (e == cudaSuccess) e = dalloc(&h->d_slot_of, h->nv);
    if (e == cudaSuccess) e = dalloc(&h->d_xm, S);
    if (e == cudaSuccess) e = dalloc(&h->d_vel, S);
    if (e == cudaSuccess) e = dalloc(&h->d_vlast, S);
    if (e == cudaSuccess) e = dalloc(&h->d_q, S);
    if (e == cudaSuccess) e = dalloc(&h->d_qr, S);
    if (e == cudaSuccess) e = dalloc(&h->d_prm, S);
    if (e == cudaSuccess) e = dalloc(&h->d_stage, 4 * h->nv);
    if (e == cudaSuccess) e = dalloc(&h->d_status, 1);
    if (e == cudaSuccess && form == KAMI_FORM_SWEEP) {
        e = dalloc(&h->d_y, S);
        if (e == cudaSuccess) e = dalloc(&h->d_dx, S);
        if (e == cudaSuccess) e = dalloc(&h->d_step, 1);
        if (e == cudaSuccess && h->schedule == KAMI_SCHEDULE_JACOBI) e = dalloc(&h->d_dx2, S);
        if (e == cudaSuccess && h->schedule == KAMI_SCHEDULE_JACOBI) e = dalloc(&h->d_q2, S);
        // colour2: the other dx buffer of the one-launch iterations (and the partners' snapshot)
        if (e == cudaSuccess && h->schedule == KAMI_SCHEDULE_COLOUR2) e = dalloc(&h->d_snap, S);
    }
    if (e != cudaSuccess) return bail(cuda_fail(e, "allocating solver state"));
    const size_t b4 = sizeof(float4) * S;
    e = cudaMemcpy(h->d_slot_of, h->layout.slot_of.data(), sizeof(int64_t) * h->nv, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_xm, xm.data(), b4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_vel, vel.data(), b4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_vlast, vlast.data(), b4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_q, q.data(), b4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_qr, qr.data(), b4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_prm, prm.data(), b4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->d_status, 0, sizeof(int));
    if (e == cudaSuccess && !ties.empty()) {  // connection springs, by slot; colour2 snapshots the partners' dx
        std::vector<int64_t> conn(S, -1);
        for (int64_t i = 0; i < h->nv; i++)
            if (ties[i] >= 0) conn[h->layout.slot_of[i]] = h->layout.slot_of[ties[i]];
        e = dalloc(&h->d_conn, S);
        if (e == cudaSuccess) e = cudaMemcpy(h->d_conn, conn.data(), sizeof(int64_t) * S, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return bail(cuda_fail(e, "uploading solver state"));

    if (d->sdf) {
        const kami_vbd_sdf_desc* s = d->sdf;
        const int64_t n = (int64_t)s->dims[0] * s->dims[1] * s->dims[2];
        std::vector<float4> grid(n);
        for (int64_t i = 0; i < n; i++) grid[i] = make_float4(s->grad[3 * i], s->grad[3 * i + 1], s->grad[3 * i + 2], s->phi[i]);
        e = dalloc(&h->d_sdf, n);
        if (e == cudaSuccess) e = cudaMemcpy(h->d_sdf, grid.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bail(cuda_fail(e, "uploading the SDF grid"));
        // grid spacing as SDFBodyCollisionSolver::InitParams computes it (SDFBodyCollisionSolver.cpp:142-159)
        SdfParams& sp = h->sdf;
        sp.grid = h->d_sdf;
        sp.nx = s->dims[0];
        sp.ny = s->dims[1];
        sp.nz = s->dims[2];
        sp.min_x = s->grid_min[0];
        sp.min_y = s->grid_min[1];
        sp.min_z = s->grid_min[2];
        sp.ds_x = (s->grid_max[0] - s->grid_min[0]) / (1.f * sp.nx);
        sp.ds_y = (s->grid_max[1] - s->grid_min[1]) / (1.f * sp.ny);
        sp.ds_z = (s->grid_max[2] - s->grid_min[2]) / (1.f * sp.nz);
        sp.inv_x = 1.f / sp.ds_x;
        sp.inv_y = 1.f / sp.ds_y;
        sp.inv_z = 1.f / sp.ds_z;
        sp.thresh = s->threshold;
    }
    if (d->hair_hair) {
        kami_status cs = setup_collisions(h, d);
        if (cs != KAMI_OK) return bail(cs);
    }
    if (d->sag_free_itr > 0) {
        kami_status ss = kami_vbd_sag_free(h, d->sag_free_itr);
        if (ss != KAMI_OK) return bail(ss);
    }
    *out = h;
    return KAMI_OK;
}

kami_status kami_vbd_create(const kami_vbd_desc* desc, kami_vbd_handle* out) { return create_impl(desc, 1, out); }

kami_status kami_vbd_batch_create(int32_t num_grooms, const kami_vbd_desc* descs, kami_vbd_handle* out) {
    if (num_grooms <= 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "num_grooms must be > 0");
    return create_impl(descs, num_grooms, out);
}

kami_status kami_vbd_batch_count(kami_vbd_handle h, int32_t* num_grooms) {
    if (!h || !num_grooms) return fail(KAMI_ERR_INVALID_ARGUMENT, "null argument");
    *num_grooms = (int32_t)h->groom_strand_begin.size() - 1;
    return KAMI_OK;
}

kami_status kami_vbd_batch_groom_range(kami_vbd_handle h, int32_t groom, int32_t* strand_begin, int32_t* num_strands,
                                       int64_t* vertex_begin, int64_t* num_vertices) {
    if (!h) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle");
    const int32_t n = (int32_t)h->groom_strand_begin.size() - 1;
    if (groom < 0 || groom >= n) return fail(KAMI_ERR_INVALID_ARGUMENT, "groom %d out of range [0, %d)", groom, n);
    const int32_t s0 = h->groom_strand_begin[groom], s1 = h->groom_strand_begin[groom + 1];
    if (strand_begin) *strand_begin = s0;
    if (num_strands) *num_strands = s1 - s0;
    if (vertex_begin) *vertex_begin = h->strand_begin[s0];
    if (num_vertices) *num_vertices = (int64_t)h->strand_begin[s1] - h->strand_begin[s0];
    return KAMI_OK;
}

kami_status kami_vbd_batch_step(kami_vbd_handle h, float dt, int32_t n, const float* body_transforms, void* stream) {
    return kami_vbd_step_n(h, dt, n, body_transforms, stream);
}

kami_status kami_vbd_destroy(kami_vbd_handle h) {
    if (!h) return KAMI_OK;
    release(h);
    return KAMI_OK;
}

kami_status kami_vbd_get_sizes(kami_vbd_handle h, int64_t* num_vertices, int32_t* num_strands, int32_t* slots_per_lane) {
    if (!h) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle");
    if (num_vertices) *num_vertices = h->nv;
    if (num_strands) *num_strands = h->ns;
    if (slots_per_lane) *slots_per_lane = h->layout.C;
    return KAMI_OK;
}

kami_status kami_vbd_set_positions_velocities(kami_vbd_handle h, const float* xyz, const float* vxyz, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (memory != KAMI_MEMORY_HOST && memory != KAMI_MEMORY_DEVICE) return fail(KAMI_ERR_INVALID_ARGUMENT, "bad memory kind");
    if (xyz) {
        KAMI_TRY(stage_in(h, xyz, 3, memory));
        KAMI_CUDA(launch_scatter3(h->d_stage, h->d_xm, h->d_slot_of, h->nv, h->stream), "scatter positions");
    }
    if (vxyz) {
        KAMI_TRY(stage_in(h, vxyz, 3, memory));
        KAMI_CUDA(launch_scatter3(h->d_stage, h->d_vel, h->d_slot_of, h->nv, h->stream), "scatter velocities");
    }
    return KAMI_OK;
}

kami_status kami_vbd_get_positions_velocities(kami_vbd_handle h, float* xyz, float* vxyz, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (memory != KAMI_MEMORY_HOST && memory != KAMI_MEMORY_DEVICE) return fail(KAMI_ERR_INVALID_ARGUMENT, "bad memory kind");
    if (xyz) {
        KAMI_CUDA(launch_gather3(h->d_xm, h->d_stage, h->d_slot_of, h->nv, h->stream), "gather positions");
        KAMI_TRY(stage_out(h, xyz, 3, memory));
    }
    if (vxyz) {
        KAMI_CUDA(launch_gather3(h->d_vel, h->d_stage, h->d_slot_of, h->nv, h->stream), "gather velocities");
        KAMI_TRY(stage_out(h, vxyz, 3, memory));
    }
    return check_status_word(h);
}

static kami_status get4(kami_vbd_solver* h, const float4* src, float* dst, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (!dst) return fail(KAMI_ERR_INVALID_ARGUMENT, "null output");
    KAMI_CUDA(launch_gather4(src, (float4*)h->d_stage, h->d_slot_of, h->nv, h->stream), "gather");
    KAMI_TRY(stage_out(h, dst, 4, memory));
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    return KAMI_OK;
}
static kami_status set4(kami_vbd_solver* h, float4* dst, const float* src, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (!src) return fail(KAMI_ERR_INVALID_ARGUMENT, "null input");
    KAMI_TRY(stage_in(h, src, 4, memory));
    KAMI_CUDA(launch_scatter4((const float4*)h->d_stage, dst, h->d_slot_of, h->nv, h->stream), "scatter");
    return KAMI_OK;
}

kami_status kami_vbd_get_orientations(kami_vbd_handle h, float* xyzw, int32_t memory) { return get4(h, h ? h->d_q : nullptr, xyzw, memory); }
kami_status kami_vbd_set_orientations(kami_vbd_handle h, const float* xyzw, int32_t memory) { return set4(h, h ? h->d_q : nullptr, xyzw, memory); }
kami_status kami_vbd_get_rest_darboux(kami_vbd_handle h, float* xyzw, int32_t memory) { return get4(h, h ? h->d_qr : nullptr, xyzw, memory); }
kami_status kami_vbd_set_rest_darboux(kami_vbd_handle h, const float* xyzw, int32_t memory) { return set4(h, h ? h->d_qr : nullptr, xyzw, memory); }

kami_status kami_vbd_set_body_transform(kami_vbd_handle h, const float rotation_xyzw[4], const float translate[3]) {
    if (!h) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle");
    if (rotation_xyzw)
        for (int i = 0; i < 4; i++) h->rot[i] = rotation_xyzw[i];
    if (translate)
        for (int i = 0; i < 3; i++) h->tr[i] = translate[i];
    return KAMI_OK;
}

// A step's dt: finite, and at most KAMI_MAX_SUBSTEPS substeps of max_h (ceil(dt / max_h) is bounded
// before it is converted to int).  dt <= 0 passes: Sim::advance returns for it (step.cpp:38-39).
static kami_status check_dt(const kami_vbd_solver* h, float dt) {
    if (!std::isfinite(dt)) return fail(KAMI_ERR_INVALID_ARGUMENT, "dt must be finite");
    if (dt > 0.f && !(std::ceil(dt / h->max_h) <= (float)KAMI_MAX_SUBSTEPS))
        return fail(KAMI_ERR_INVALID_ARGUMENT, "dt / max_h needs more than %d substeps", KAMI_MAX_SUBSTEPS);
    return KAMI_OK;
}

static StepParams advance_clock(kami_vbd_solver* h, float dt) {
    const int steps = std::max(1, (int)std::ceil(dt / h->max_h));
    h->last_h = h->h;
    h->h = dt / (float)steps;
    StepParams sp;
    sp.h = h->h;
    sp.last_h = h->last_h;
    sp.time = h->time;
    sp.substeps = steps;
    sp.rot_x = h->rot[0];
    sp.rot_y = h->rot[1];
    sp.rot_z = h->rot[2];
    sp.rot_w = h->rot[3];
    sp.tr_x = h->tr[0];
    sp.tr_y = h->tr[1];
    sp.tr_z = h->tr[2];
    return sp;
}

kami_status kami_vbd_step(kami_vbd_handle h, float dt, void* stream) {
    KAMI_TRY(valid_handle(h));
    KAMI_TRY(check_dt(h, dt));
    if (!(dt > 0.f)) return KAMI_OK;  // Sim::advance returns for h <= 0 (step.cpp:38-39)
    const StepParams sp = advance_clock(h, dt);
    const int steps = sp.substeps;
    kami_status st = on_stream(h, stream, [&](cudaStream_t s) -> kami_status {
        if (h->form == KAMI_FORM_FUSED) {
            KAMI_CUDA(launch_fused_step(h->dstate(), h->pp, sp, h->sdf, h->layout.C, h->schedule == KAMI_SCHEDULE_JACOBI,
                                        h->warps_per_block, s, nullptr, 1, h->reg_cap, h->layout.K, h->launch_mode),
                      "fused step launch");
        } else {
            KAMI_TRY(build_sweep_graph(h, steps));
            h->h_step = sp;
            KAMI_CUDA(cudaMemcpyAsync(h->d_step, &h->h_step, sizeof(StepParams), cudaMemcpyHostToDevice, s), "step params");
            KAMI_CUDA(cudaGraphLaunch(h->graph, s), "cudaGraphLaunch");
            if (h->hair_hair) h->coll_stale = false;
        }
        return KAMI_OK;
    });
    if (st != KAMI_OK) return st;
    h->time += dt;
    h->counter += steps;
    return KAMI_OK;
}

// ---- multi-step launches, tile shape and autotuning --------------------------------------------------

static void drop_graphs(kami_vbd_solver* h) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->graph_n) cudaGraphExecDestroy(h->graph_n);
    h->graph = h->graph_n = nullptr;
    h->graph_substeps = h->graph_n_steps = h->graph_n_F = -1;
}

// ---- frames over host buffers -------------------------------------------------------------------------

// Runs of each tile's strands for the fused frame kernel (HostIO): strand s is one run of
// consecutive tile positions starting at the position of its first vertex.
static kami_status build_host_runs(kami_vbd_solver* h) {
    const int C = h->layout.C;
    const int64_t T = 32LL * C, tiles = h->layout.num_tiles;
    // a strand is one run of consecutive tile positions in each tile it occupies (more than one
    // when it runs on across the tiles of a group): the kernel stages positions [p0, p0 + n) < T
    struct Piece {
        int64_t tile;
        int4 run;
    };
    std::vector<Piece> pieces;
    pieces.reserve(h->ns);
    for (int32_t s = 0; s < h->ns; s++) {
        const int32_t v1 = h->strand_begin[s + 1];
        for (int32_t j = h->strand_begin[s]; j < v1;) {
            const int64_t g = h->layout.slot_of[j];
            const int64_t t = g / T, q = g % T;  // q = (p % C) * 32 + p / C
            const int p0 = (int)((q % 32) * C + q / 32);
            int32_t n = 1;
            while (j + n < v1) {
                const int p = p0 + n;
                if (p >= T || h->layout.slot_of[j + n] != t * T + (int64_t)(p % C) * 32 + p / C) break;
                n++;
            }
            pieces.push_back({t, make_int4(p0, j, n, 0)});
            j += n;
        }
    }
    std::vector<int32_t> begin(tiles + 1, 0);
    for (const Piece& pc : pieces) begin[pc.tile + 1]++;
    for (int64_t t = 0; t < tiles; t++) begin[t + 1] += begin[t];
    std::vector<int32_t> next(begin.begin(), begin.end() - 1);
    std::vector<int4> runs(pieces.size());
    for (const Piece& pc : pieces) runs[next[pc.tile]++] = pc.run;
    // with a Hair layout, the runs again with their first vertex's padded Hair entry (a strand's
    // vertices are consecutive there too)
    const bool hair = !h->hair_index.empty() && h->hair_entries < ((int64_t)1 << 31);
    std::vector<int4> hruns;
    if (hair) {
        hruns = runs;
        for (int4& r : hruns) r.y = (int32_t)h->hair_index[r.y];
    }
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    if (h->d_runs) cudaFree(h->d_runs);
    if (h->d_run_begin) cudaFree(h->d_run_begin);
    if (h->d_hair_runs) cudaFree(h->d_hair_runs);
    h->d_runs = nullptr;
    h->d_run_begin = nullptr;
    h->d_hair_runs = nullptr;
    h->runs_C = 0;
    KAMI_CUDA(dalloc(&h->d_runs, runs.size()), "strand runs");
    KAMI_CUDA(dalloc(&h->d_run_begin, begin.size()), "strand runs");
    KAMI_CUDA(cudaMemcpy(h->d_runs, runs.data(), sizeof(int4) * runs.size(), cudaMemcpyHostToDevice), "strand runs");
    if (hair) {
        KAMI_CUDA(dalloc(&h->d_hair_runs, hruns.size()), "Hair runs");
        KAMI_CUDA(cudaMemcpy(h->d_hair_runs, hruns.data(), sizeof(int4) * hruns.size(), cudaMemcpyHostToDevice),
                  "Hair runs");
    }
    KAMI_CUDA(cudaMemcpy(h->d_run_begin, begin.data(), sizeof(int32_t) * begin.size(), cudaMemcpyHostToDevice),
              "strand runs");
    h->runs_C = C;
    return KAMI_OK;
}

// The device address of host array [p, p + n floats) when the whole range lies in one page-locked
// allocation mapped into the device's address space; null otherwise.
static float* mapped_range(const void* p, int64_t n) {
    using PtrAttr = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
    static PtrAttr ptr_attr = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PtrAttr) nullptr;
        }
        return (PtrAttr)f;
    }();
    if (!ptr_attr || !p || ((uintptr_t)p & 3) != 0 || n <= 0) return nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
    CUdeviceptr start = 0;
    size_t size = 0;
    const CUdeviceptr d = (CUdeviceptr)(uintptr_t)a.devicePointer;
    if (ptr_attr(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS ||
        ptr_attr(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS)
        return nullptr;
    if (d < start || d + sizeof(float) * (size_t)n > start + size) return nullptr;
    return (float*)a.devicePointer;
}

kami_status kami_vbd_step_host(kami_vbd_handle h, float dt, const float* xyz, const float* vxyz, float* xyz_out,
                               float* vxyz_out) {
    KAMI_TRY(valid_handle(h));
    if (!xyz || !vxyz || !xyz_out || !vxyz_out) return fail(KAMI_ERR_INVALID_ARGUMENT, "null position or velocity array");
    KAMI_TRY(check_dt(h, dt));
    HostIO io{};
    const int64_t n = 3 * h->nv;
    bool direct = dt > 0.f && h->form == KAMI_FORM_FUSED && !h->hair_hair;
    if (direct) {
        io.x_in = mapped_range(xyz, n);
        io.v_in = mapped_range(vxyz, n);
        io.x_out = mapped_range(xyz_out, n);
        io.v_out = mapped_range(vxyz_out, n);
        direct = io.x_in && io.v_in && io.x_out && io.v_out;
    }
    if (!direct) {
        // pageable buffers, no step, or strands coupled within the step: upload, step and download in turn
        KAMI_TRY(kami_vbd_set_positions_velocities(h, xyz, vxyz, KAMI_MEMORY_HOST));
        KAMI_TRY(kami_vbd_step(h, dt, nullptr));
        return kami_vbd_get_positions_velocities(h, xyz_out, vxyz_out, KAMI_MEMORY_HOST);
    }
    if (h->runs_C != h->layout.C) KAMI_TRY(build_host_runs(h));
    io.runs = h->d_runs;
    io.run_begin = h->d_run_begin;
    const StepParams sp = advance_clock(h, dt);
    KAMI_CUDA(launch_fused_frame(h->dstate(), h->pp, sp, h->sdf, io, h->layout.C, h->schedule == KAMI_SCHEDULE_JACOBI,
                                 h->warps_per_block, h->stream, h->reg_cap, h->layout.K),
              "fused frame launch");
    h->time += dt;
    h->counter += sp.substeps;
    return check_status_word(h);
}

kami_status kami_vbd_step_hair(kami_vbd_handle h, float dt, const float* hair_xyz_in, const float* hair_vxyz_in,
                               float* hair_xyz_out, float* hair_vxyz_out) {
    KAMI_TRY(valid_handle(h));
    if (h->hair_index.empty()) return fail(KAMI_ERR_STATE, "call kami_vbd_set_hair_layout first");
    if (!hair_xyz_in != !hair_vxyz_in || !hair_xyz_out != !hair_vxyz_out)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "give both Hair input arrays or neither, and both outputs or neither");
    KAMI_TRY(check_dt(h, dt));
    const int64_t n = 3 * h->hair_entries;
    HostIO io{};
    bool direct = dt > 0.f && h->form == KAMI_FORM_FUSED && !h->hair_hair && h->hair_entries < ((int64_t)1 << 31);
    if (direct && hair_xyz_in) {
        io.x_in = mapped_range(hair_xyz_in, n);
        io.v_in = mapped_range(hair_vxyz_in, n);
        direct = io.x_in && io.v_in;
    }
    if (direct && hair_xyz_out) {
        io.x_out = mapped_range(hair_xyz_out, n);
        io.v_out = mapped_range(hair_vxyz_out, n);
        direct = io.x_out && io.v_out;
    }
    if (!direct) {  // UploadHair, SolveNextStep, DownloadHair in turn
        if (hair_xyz_in) KAMI_TRY(kami_vbd_upload_hair(h, hair_xyz_in, hair_vxyz_in, KAMI_MEMORY_HOST));
        KAMI_TRY(kami_vbd_step(h, dt, nullptr));
        if (hair_xyz_out) return kami_vbd_download_hair(h, hair_xyz_out, hair_vxyz_out, KAMI_MEMORY_HOST);
        return kami_vbd_synchronize(h);
    }
    if (h->runs_C != h->layout.C) KAMI_TRY(build_host_runs(h));
    if (!h->d_hair_runs) return fail(KAMI_ERR_STATE, "no Hair runs for this layout");
    io.runs = h->d_hair_runs;
    io.run_begin = h->d_run_begin;
    const StepParams sp = advance_clock(h, dt);
    KAMI_CUDA(launch_fused_frame(h->dstate(), h->pp, sp, h->sdf, io, h->layout.C, h->schedule == KAMI_SCHEDULE_JACOBI,
                                 h->warps_per_block, h->stream, h->reg_cap, h->layout.K),
              "fused Hair frame launch");
    h->time += dt;
    h->counter += sp.substeps;
    return check_status_word(h);  // blocks: the host may touch the Hair arrays once this returns
}

kami_status kami_host_register(void* p, size_t bytes) {
    if (!p || bytes == 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "null pointer or zero size");
    KAMI_CUDA(cudaHostRegister(p, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable), "cudaHostRegister");
    return KAMI_OK;
}

kami_status kami_host_unregister(void* p) {
    if (!p) return fail(KAMI_ERR_INVALID_ARGUMENT, "null pointer");
    KAMI_CUDA(cudaHostUnregister(p), "cudaHostUnregister");
    return KAMI_OK;
}

// Moves the live state to tiles of 32*C slots (gathered to boundary order and scattered back); the
// fused form takes groups of as many tiles as the longest strand needs.
static kami_status relayout(kami_vbd_solver* h, int C) {
    if (C == h->layout.C) return KAMI_OK;
    const int K = h->form == KAMI_FORM_FUSED ? tiles_per_group_for(h->strand_begin.data(), h->ns, C) : 1;
    if (K == 0) return fail(KAMI_ERR_UNSUPPORTED, "a strand is longer than 8 tiles of %d slots", 32 * C);
    std::string err;
    TileLayout nl;
    if (!pack_tiles(h->strand_begin.data(), h->ns, C, nl, err, K)) return fail(KAMI_ERR_UNSUPPORTED, "%s", err.c_str());
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    const int64_t nv = h->nv, S = nl.num_slots;
    float4* tmp = nullptr;
    KAMI_CUDA(dalloc(&tmp, 6 * nv), "relayout buffer");
    float4* olds[6] = {h->d_xm, h->d_vel, h->d_vlast, h->d_q, h->d_qr, h->d_prm};
    cudaError_t e = cudaSuccess;
    for (int a = 0; a < 6 && e == cudaSuccess; a++) e = launch_gather4(olds[a], tmp + a * nv, h->d_slot_of, nv, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    // padding slots: zero position/mass, identity orientations, lRest 1 and no flags
    std::vector<float4> zero(S, make_float4(0.f, 0.f, 0.f, 0.f)), ident(S, make_float4(0.f, 0.f, 0.f, 1.f)),
        pad(S, make_float4(1.f, 0.f, 0.f, 0.f));
    const std::vector<float4>* init[6] = {&zero, &zero, &zero, &ident, &ident, &pad};
    float4* news[6] = {};
    for (int a = 0; a < 6 && e == cudaSuccess; a++) {
        e = dalloc(&news[a], S);
        if (e == cudaSuccess) e = cudaMemcpy(news[a], init[a]->data(), sizeof(float4) * S, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(h->d_slot_of, nl.slot_of.data(), sizeof(int64_t) * nv, cudaMemcpyHostToDevice);
    for (int a = 0; a < 6 && e == cudaSuccess; a++) e = launch_scatter4(tmp + a * nv, news[a], h->d_slot_of, nv, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) {
        for (float4* p : news)
            if (p) cudaFree(p);
        return cuda_fail(e, "relayout");
    }
    for (float4* p : olds) cudaFree(p);
    h->d_xm = news[0];
    h->d_vel = news[1];
    h->d_vlast = news[2];
    h->d_q = news[3];
    h->d_qr = news[4];
    h->d_prm = news[5];
    // slot-indexed scratch follows the new layout; the tape and adjoint buffers are dropped
    float4** scratch[] = {&h->d_y, &h->d_dx, &h->d_dx2, &h->d_q2, &h->d_tdx, &h->d_tq, &h->d_tx, &h->d_tv, &h->d_tvl,
                          &h->d_gx, &h->d_gv, &h->d_gvl, &h->d_gq, &h->d_gqr};
    bool had[14];
    for (int i = 0; i < 14; i++) {
        had[i] = *scratch[i] != nullptr;
        if (*scratch[i]) cudaFree(*scratch[i]);
        *scratch[i] = nullptr;
    }
    h->tape_capacity = 0;
    h->tape_tiles = 0;
    h->tape_steps.clear();
    for (int i = 0; i < 4 && e == cudaSuccess; i++)
        if (had[i]) e = dalloc(scratch[i], S);
    h->layout = nl;
    if (h->d_strand_root) cudaFree(h->d_strand_root);  // slots of the old layout
    if (h->d_strand_len) cudaFree(h->d_strand_len);
    if (h->d_strand_cta) cudaFree(h->d_strand_cta);
    h->d_strand_root = nullptr;
    h->d_strand_len = nullptr;
    h->d_strand_cta = nullptr;
    drop_graphs(h);
    if (e != cudaSuccess) return cuda_fail(e, "relayout scratch");
    return KAMI_OK;
}

kami_status kami_vbd_set_tuning(kami_vbd_handle h, int32_t slots_per_lane, int32_t warps_per_block,
                                int32_t steps_per_launch, int32_t register_cap) {
    KAMI_TRY(valid_handle(h));
    if (slots_per_lane != 0 && h->hair_hair && slots_per_lane != h->layout.C)
        return fail(KAMI_ERR_UNSUPPORTED, "the tile shape of a handle with hair-hair collision is fixed at creation");
    if (slots_per_lane != 0 && h->d_conn && slots_per_lane != h->layout.C)
        return fail(KAMI_ERR_UNSUPPORTED, "the tile shape of a handle with connection springs is fixed at creation");
    if (slots_per_lane != 0) {
        const int cmin = slots_per_lane_for(h->strand_begin.data(), h->ns);
        if (h->form == KAMI_FORM_FUSED) {  // longer strands take groups of tiles
            if (!fused_supported(slots_per_lane))
                return fail(KAMI_ERR_UNSUPPORTED, "the fused form supports 2 or 4 slots per lane");
        } else if (slots_per_lane < cmin || (slots_per_lane & 1)) {
            return fail(KAMI_ERR_INVALID_ARGUMENT, "slots_per_lane must be even and >= %d", cmin);
        }
        KAMI_TRY(relayout(h, slots_per_lane));
    }
    if (warps_per_block != 0) {
        if (warps_per_block < 0 || warps_per_block > 8 || (warps_per_block & (warps_per_block - 1)))
            return fail(KAMI_ERR_INVALID_ARGUMENT, "warps_per_block must be 1, 2, 4 or 8");
        if (warps_per_block != h->warps_per_block) drop_graphs(h);
        h->warps_per_block = warps_per_block;
    }
    if (steps_per_launch != 0) {
        if (steps_per_launch < 1 || steps_per_launch > 1024)
            return fail(KAMI_ERR_INVALID_ARGUMENT, "steps_per_launch must be in [1, 1024]");
        if (steps_per_launch != h->steps_per_launch) drop_graphs(h);
        h->steps_per_launch = steps_per_launch;
    }
    if (register_cap != 0) {
        if (register_cap != 1 && register_cap != 2 && register_cap != 120 && register_cap != 168)
            return fail(KAMI_ERR_INVALID_ARGUMENT,
                        "register_cap must be 0 (unchanged), 1 (none), 2 (packed x2), 120 or 168");
        if (register_cap == 2 && (h->layout.C != 4 || h->layout.K != 1 || h->schedule != KAMI_SCHEDULE_COLOUR2))
            return fail(KAMI_ERR_UNSUPPORTED,
                        "the packed FP32x2 variant runs the colour2 step with 4 slots per lane on single tiles");
        const int cap = register_cap == 1 ? 0 : register_cap;
        if (cap != h->reg_cap) drop_graphs(h);
        h->reg_cap = cap;
    }
    return KAMI_OK;
}

kami_status kami_vbd_get_tuning(kami_vbd_handle h, int32_t* slots_per_lane, int32_t* warps_per_block,
                                int32_t* steps_per_launch, int32_t* register_cap) {
    if (!h) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle");
    if (slots_per_lane) *slots_per_lane = h->layout.C;
    if (warps_per_block) *warps_per_block = h->warps_per_block;
    if (steps_per_launch) *steps_per_launch = h->steps_per_launch;
    if (register_cap) *register_cap = h->reg_cap ? h->reg_cap : 1;
    return KAMI_OK;
}

static_assert(KAMI_LAUNCH_PERSISTENT == LAUNCH_PERSISTENT, "the C ABI's launch mode is the launcher's");

kami_status kami_vbd_set_launch_mode(kami_vbd_handle h, int32_t mode) {
    KAMI_TRY(valid_handle(h));
    if (mode != 0 && mode != KAMI_LAUNCH_PERSISTENT)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "the launch mode is 0 or KAMI_LAUNCH_PERSISTENT");
    if (mode != h->launch_mode) drop_graphs(h);
    h->launch_mode = mode;
    return KAMI_OK;
}

kami_status kami_vbd_get_launch_mode(kami_vbd_handle h, int32_t* mode) {
    if (!h || !mode) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle or output");
    *mode = h->launch_mode;
    return KAMI_OK;
}

kami_status kami_vbd_step_n(kami_vbd_handle h, float dt, int32_t n, const float* body_transforms, void* stream) {
    KAMI_TRY(valid_handle(h));
    if (n < 1) return fail(KAMI_ERR_INVALID_ARGUMENT, "n must be >= 1");
    KAMI_TRY(check_dt(h, dt));
    if (!(dt > 0.f)) return fail(KAMI_ERR_INVALID_ARGUMENT, "dt must be > 0");
    if (h->form != KAMI_FORM_FUSED) {
        for (int j = 0; j < n; j++) {
            if (body_transforms) kami_vbd_set_body_transform(h, body_transforms + 7 * j, body_transforms + 7 * j + 4);
            KAMI_TRY(kami_vbd_step(h, dt, stream));
        }
        return KAMI_OK;
    }
    if (n > h->d_steps_cap) {
        KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        if (h->d_steps) cudaFree(h->d_steps);
        h->d_steps = nullptr;
        h->d_steps_cap = 0;
        KAMI_CUDA(dalloc(&h->d_steps, (size_t)n), "step parameter array");
        h->d_steps_cap = n;
        drop_graphs(h);
    }
    h->h_steps.resize(n);
    for (int j = 0; j < n; j++) {
        if (body_transforms) kami_vbd_set_body_transform(h, body_transforms + 7 * j, body_transforms + 7 * j + 4);
        h->h_steps[j] = advance_clock(h, dt);
        h->time += dt;
        h->counter += h->h_steps[j].substeps;
    }
    const int F = std::min(h->steps_per_launch, n);
    if (!h->graph_n || h->graph_n_steps != n || h->graph_n_F != F) {
        if (h->graph_n) cudaGraphExecDestroy(h->graph_n);
        h->graph_n = nullptr;
        KAMI_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        cudaError_t err = cudaSuccess;
        for (int j0 = 0; j0 < n && err == cudaSuccess; j0 += F)
            err = launch_fused_step(h->dstate(), h->pp, h->h_steps[0], h->sdf, h->layout.C,
                                    h->schedule == KAMI_SCHEDULE_JACOBI, h->warps_per_block, h->stream, h->d_steps + j0,
                                    std::min(F, n - j0), h->reg_cap, h->layout.K, h->launch_mode);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
        if (err != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(err != cudaSuccess ? err : e2, "capturing the multi-step graph");
        }
        cudaError_t e3 = cudaGraphInstantiate(&h->graph_n, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) return cuda_fail(e3, "cudaGraphInstantiate");
        h->graph_n_steps = n;
        h->graph_n_F = F;
    }
    return on_stream(h, stream, [&](cudaStream_t s) -> kami_status {
        KAMI_CUDA(cudaMemcpyAsync(h->d_steps, h->h_steps.data(), sizeof(StepParams) * n, cudaMemcpyHostToDevice, s),
                  "step parameters");
        KAMI_CUDA(cudaGraphLaunch(h->graph_n, s), "cudaGraphLaunch");
        return KAMI_OK;
    });
}

kami_status kami_vbd_autotune(kami_vbd_handle h, float dt, int32_t trial_steps, int32_t best[4], double* best_rate) {
    KAMI_TRY(valid_handle(h));
    if (h->form != KAMI_FORM_FUSED) return fail(KAMI_ERR_UNSUPPORTED, "the autotuner tunes the fused form");
    if (trial_steps < 1 || !(dt > 0.f)) return fail(KAMI_ERR_INVALID_ARGUMENT, "need trial_steps >= 1 and dt > 0");
    // snapshot of the simulation state and clock, restored after every trial
    size_t bytes = 0;
    kami_vbd_state_size(h, &bytes);
    void* snap = nullptr;
    KAMI_CUDA(cudaMalloc(&snap, bytes), "autotune snapshot");
    kami_status st = kami_vbd_get_state(h, snap, bytes, KAMI_MEMORY_DEVICE);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (st == KAMI_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        st = fail(KAMI_ERR_CUDA, "cudaEventCreate");
    const int Fs[3] = {1, 4, 16};
    double rate_best = -1.0;
    int pick[4] = {h->layout.C, h->warps_per_block, h->steps_per_launch, h->reg_cap ? h->reg_cap : 1};
    const bool colour2 = h->schedule == KAMI_SCHEDULE_COLOUR2;
    for (int C = 2; C <= 4 && st == KAMI_OK; C += 2) {  // both, in groups of tiles where strands need them
        // tiles per group for this C (strands longer than a tile); groups fix the CTA shape
        const int K = tiles_per_group_for(h->strand_begin.data(), h->ns, C);
        if (K == 0) continue;
        // kernel variants: C = 2 plain or 120 registers; C = 4 plain, 168 registers or packed FP32x2
        // (colour2, single tiles)
        const int caps[3] = {1, C == 2 ? 120 : 168, 2};
        for (int R = 0; R < (C == 4 && colour2 && K == 1 ? 3 : 2) && st == KAMI_OK; R++) {
        const int cap = caps[R];
        for (int W = 1; W <= (K == 1 ? 8 : 1) && st == KAMI_OK; W *= 2) {
            for (int fi = 0; fi < 3 && st == KAMI_OK; fi++) {
                const int F = std::min(Fs[fi], trial_steps);
                st = kami_vbd_set_tuning(h, C, W, F, cap);
                if (st == KAMI_OK) st = kami_vbd_set_state(h, snap, bytes, KAMI_MEMORY_DEVICE);
                if (st == KAMI_OK) st = kami_vbd_step_n(h, dt, trial_steps, nullptr, nullptr);  // warm-up, builds the graph
                if (st == KAMI_OK) st = kami_vbd_set_state(h, snap, bytes, KAMI_MEMORY_DEVICE);
                if (st != KAMI_OK) break;
                cudaEventRecord(e0, h->stream);
                st = kami_vbd_step_n(h, dt, trial_steps, nullptr, nullptr);
                cudaEventRecord(e1, h->stream);
                if (st != KAMI_OK) break;
                if (cudaEventSynchronize(e1) != cudaSuccess) {
                    st = fail(KAMI_ERR_CUDA, "autotune timing");
                    break;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                const double rate = (double)h->nv * h->pp.num_itr * trial_steps / (ms * 1e-3);
                if (rate > rate_best) {
                    rate_best = rate;
                    pick[0] = C;
                    pick[1] = W;
                    pick[2] = F;
                    pick[3] = cap;
                }
                if (Fs[fi] >= trial_steps) break;
            }
        }
        }
    }
    if (st == KAMI_OK) st = kami_vbd_set_tuning(h, pick[0], pick[1], pick[2], pick[3]);
    // the launch modes on the fastest shape (the packed variant has no persistent form)
    int mode_best = 0;
    const int modes[2] = {0, KAMI_LAUNCH_PERSISTENT};
    for (int mi = 0; mi < (pick[3] == 2 ? 1 : 2) && st == KAMI_OK; mi++) {
        st = kami_vbd_set_launch_mode(h, modes[mi]);
        if (st == KAMI_OK) st = kami_vbd_set_state(h, snap, bytes, KAMI_MEMORY_DEVICE);
        if (st == KAMI_OK) st = kami_vbd_step_n(h, dt, trial_steps, nullptr, nullptr);
        if (st == KAMI_OK) st = kami_vbd_set_state(h, snap, bytes, KAMI_MEMORY_DEVICE);
        if (st != KAMI_OK) break;
        cudaEventRecord(e0, h->stream);
        st = kami_vbd_step_n(h, dt, trial_steps, nullptr, nullptr);
        cudaEventRecord(e1, h->stream);
        if (st != KAMI_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            st = fail(KAMI_ERR_CUDA, "autotune timing");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double rate = (double)h->nv * h->pp.num_itr * trial_steps / (ms * 1e-3);
        if (mi == 0 || rate > rate_best) {
            rate_best = rate;
            mode_best = modes[mi];
        }
    }
    if (st == KAMI_OK) st = kami_vbd_set_launch_mode(h, mode_best);
    if (st == KAMI_OK) st = kami_vbd_set_state(h, snap, bytes, KAMI_MEMORY_DEVICE);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(snap);
    if (st != KAMI_OK) return st;
    if (best)
        for (int i = 0; i < 4; i++) best[i] = pick[i];
    if (best_rate) *best_rate = rate_best;
    return KAMI_OK;
}

// ---- differentiable stepping ----------------------------------------------------------------------

static kami_status adjoint_supported(kami_vbd_solver* h) {
    if (h->form != KAMI_FORM_FUSED || h->schedule != KAMI_SCHEDULE_COLOUR2)
        return fail(KAMI_ERR_UNSUPPORTED, "the adjoint covers the fused form with the colour2 schedule");
    return KAMI_OK;
}

kami_status kami_vbd_tape_reserve(kami_vbd_handle h, int32_t max_steps, int64_t max_tiles) {
    KAMI_TRY(valid_handle(h));
    KAMI_TRY(adjoint_supported(h));
    if (max_steps <= 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "max_steps must be > 0");
    if (max_tiles < 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "max_tiles must be >= 0");
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    const int64_t K = h->layout.K;  // windows are whole groups of tiles
    int64_t tiles = (max_tiles == 0 || max_tiles > h->layout.num_tiles) ? h->layout.num_tiles : max_tiles;
    tiles = std::min<int64_t>(h->layout.num_tiles, (tiles + K - 1) / K * K);
    if (h->tape_capacity == max_steps && h->tape_tiles == tiles) {  // already the requested size
        h->tape_steps.clear();
        h->win_begin = 0;
        h->win_end = tiles;
        return KAMI_OK;
    }
    const size_t S = (size_t)h->layout.num_slots, N1 = (size_t)h->pp.num_itr + 1;
    const size_t TS = (size_t)tiles * 32 * h->layout.C;  // tape slots per step
    float4** tape_arrays[] = {&h->d_tdx, &h->d_tq, &h->d_tx, &h->d_tv, &h->d_tvl};
    for (float4** p : tape_arrays)
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    h->tape_capacity = 0;
    h->tape_tiles = 0;
    h->tape_steps.clear();
    cudaError_t e = dalloc(&h->d_tdx, (size_t)max_steps * N1 * TS);
    if (e == cudaSuccess) e = dalloc(&h->d_tq, (size_t)max_steps * N1 * TS);
    if (e == cudaSuccess) e = dalloc(&h->d_tx, (size_t)max_steps * TS);
    if (e == cudaSuccess) e = dalloc(&h->d_tv, (size_t)max_steps * TS);
    if (e == cudaSuccess) e = dalloc(&h->d_tvl, (size_t)max_steps * TS);
    float4** adj_arrays[] = {&h->d_gx, &h->d_gv, &h->d_gvl, &h->d_gq, &h->d_gqr};
    for (float4** p : adj_arrays)
        if (e == cudaSuccess && !*p) {
            e = dalloc(p, S);
            if (e == cudaSuccess) e = cudaMemset(*p, 0, sizeof(float4) * S);
        }
    if (e != cudaSuccess) return cuda_fail(e, "allocating the tape");
    h->tape_capacity = max_steps;
    h->tape_tiles = tiles;
    h->win_begin = 0;
    h->win_end = tiles;
    return KAMI_OK;
}

kami_status kami_vbd_get_tile_count(kami_vbd_handle h, int64_t* num_tiles) {
    if (!h || !num_tiles) return fail(KAMI_ERR_INVALID_ARGUMENT, "null argument");
    *num_tiles = h->layout.num_tiles;
    return KAMI_OK;
}

kami_status kami_vbd_get_tiles_per_group(kami_vbd_handle h, int32_t* tiles_per_group) {
    if (!h || !tiles_per_group) return fail(KAMI_ERR_INVALID_ARGUMENT, "null argument");
    *tiles_per_group = h->layout.K;
    return KAMI_OK;
}

// The tape window's slots [s0, s0 + n) and the slot -> vertex map for the scatters and gathers of
// kami_vbd_backward and kami_vbd_restore_tape_window; *vert_of stays null when the window covers the
// whole groom.
static kami_status window_slots(kami_vbd_solver* h, const int64_t** vert_of, int64_t* s0, int64_t* n) {
    *vert_of = nullptr;
    if (h->win_begin == 0 && h->win_end >= h->layout.num_tiles) return KAMI_OK;
    if (!h->d_vert_of || h->vert_of_C != h->layout.C || h->vert_of_K != h->layout.K) {
        if (h->d_vert_of) cudaFree(h->d_vert_of);
        h->d_vert_of = nullptr;
        KAMI_CUDA(dalloc(&h->d_vert_of, (size_t)h->layout.num_slots), "allocating the slot -> vertex map");
        KAMI_CUDA(launch_vert_of(h->d_slot_of, h->d_vert_of, h->nv, h->layout.num_slots, h->stream), "slot -> vertex map");
        h->vert_of_C = h->layout.C;
        h->vert_of_K = h->layout.K;
    }
    const int64_t T = 32LL * h->layout.C;
    *vert_of = h->d_vert_of;
    *s0 = h->win_begin * T;
    *n = (h->win_end - h->win_begin) * T;
    return KAMI_OK;
}

kami_status kami_vbd_set_tape_window(kami_vbd_handle h, int64_t tile_begin, int64_t tile_end) {
    if (!h) return fail(KAMI_ERR_INVALID_ARGUMENT, "null handle");
    if (h->tape_capacity == 0) return fail(KAMI_ERR_STATE, "call kami_vbd_tape_reserve first");
    if (!h->tape_steps.empty()) return fail(KAMI_ERR_STATE, "the tape holds recorded steps; run kami_vbd_backward first");
    if (tile_begin < 0 || tile_end <= tile_begin || tile_end > h->layout.num_tiles)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "bad tile window [%lld, %lld)", (long long)tile_begin, (long long)tile_end);
    if (tile_end - tile_begin > h->tape_tiles)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "the tape holds %lld tiles per step", (long long)h->tape_tiles);
    if (tile_begin % h->layout.K != 0 || tile_end % h->layout.K != 0)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "tape windows are whole groups of %d tiles", h->layout.K);
    h->win_begin = tile_begin;
    h->win_end = tile_end;
    return KAMI_OK;
}

kami_status kami_vbd_step_record(kami_vbd_handle h, float dt, void* stream) {
    KAMI_TRY(valid_handle(h));
    if (h->tape_capacity == 0) return fail(KAMI_ERR_STATE, "call kami_vbd_tape_reserve first");
    KAMI_TRY(check_dt(h, dt));
    if (!(dt > 0.f)) return fail(KAMI_ERR_INVALID_ARGUMENT, "dt must be > 0");
    const int substeps = std::max(1, (int)std::ceil(dt / h->max_h));
    if ((int)h->tape_steps.size() + substeps > h->tape_capacity)
        return fail(KAMI_ERR_STATE, "the tape holds %d substeps, %d are recorded and this step takes %d; run "
                    "kami_vbd_backward first or reserve more", h->tape_capacity, (int)h->tape_steps.size(), substeps);
    const StepParams sp = advance_clock(h, dt);
    // Sim::advance keeps h, lastH, time and the body fixed over its substeps and runs the body pass once
    // after them (step.cpp:38-62), so each substep is recorded as a one-substep launch of its own and
    // only the last one ends with the SDF pass
    StepParams sp1 = sp;
    sp1.substeps = 1;
    SdfParams no_sdf = h->sdf;
    no_sdf.grid = nullptr;
    const int first = (int)h->tape_steps.size();
    kami_status st = on_stream(h, stream, [&](cudaStream_t s) -> kami_status {
        for (int k = 0; k < substeps; k++)
            KAMI_CUDA(launch_fused_record(h->window_state(), h->pp, sp1, k == substeps - 1 ? h->sdf : no_sdf,
                                          h->tape(first + k), h->layout.C, h->warps_per_block, s, h->layout.K),
                      "recorded step launch");
        return KAMI_OK;
    });
    if (st != KAMI_OK) return st;
    for (int k = 0; k < substeps; k++) h->tape_steps.push_back({sp1, k == substeps - 1});
    h->time += dt;
    h->counter += sp.substeps;
    return KAMI_OK;
}

kami_status kami_vbd_backward(kami_vbd_handle h, float* adj_x, float* adj_v, float* adj_vlast, float* adj_q,
                              int32_t memory, void* stream) {
    KAMI_TRY(valid_handle(h));
    if (h->tape_capacity == 0 || h->tape_steps.empty()) return fail(KAMI_ERR_STATE, "no recorded steps to differentiate");
    if (!adj_x || !adj_v || !adj_vlast || !adj_q) return fail(KAMI_ERR_INVALID_ARGUMENT, "null adjoint array");
    if (memory != KAMI_MEMORY_HOST && memory != KAMI_MEMORY_DEVICE) return fail(KAMI_ERR_INVALID_ARGUMENT, "bad memory kind");
    const size_t S = (size_t)h->layout.num_slots;
    AdjointState ad;
    ad.gx = h->d_gx;
    ad.gv = h->d_gv;
    ad.gvl = h->d_gvl;
    ad.gq = h->d_gq;
    ad.gqr = h->d_gqr;
    float* ins3[] = {adj_x, adj_v, adj_vlast};
    float4* adj3[] = {h->d_gx, h->d_gv, h->d_gvl};
    // A window smaller than the groom, with the adjoints in device memory, moves only its own strands'
    // entries: the slots of its tiles are reset and its vertices scattered straight from the caller's
    // arrays and gathered back into them (the other entries of those arrays are left as they are,
    // which is what the whole-groom copies would write back too).
    const int64_t* wv = nullptr;
    int64_t ws0 = 0, wn = 0;
    if (memory == KAMI_MEMORY_DEVICE) KAMI_TRY(window_slots(h, &wv, &ws0, &wn));
    if (wv) {
        for (int a = 0; a < 3; a++) {
            KAMI_CUDA(cudaMemsetAsync(adj3[a] + ws0, 0, sizeof(float4) * wn, h->stream), "adjoint reset");
            KAMI_CUDA(launch_scatter_slots(ins3[a], adj3[a], wv, ws0, wn, 3, h->stream), "scatter adjoint");
        }
        KAMI_CUDA(launch_scatter_slots(adj_q, h->d_gq, wv, ws0, wn, 4, h->stream), "scatter adjoint");
    } else {
        for (int a = 0; a < 3; a++) {
            KAMI_CUDA(cudaMemsetAsync(adj3[a], 0, sizeof(float4) * S, h->stream), "adjoint reset");
            KAMI_TRY(stage_in(h, ins3[a], 3, memory));
            KAMI_CUDA(launch_scatter3(h->d_stage, adj3[a], h->d_slot_of, h->nv, h->stream), "scatter adjoint");
        }
        KAMI_CUDA(cudaMemsetAsync(h->d_gq, 0, sizeof(float4) * S, h->stream), "adjoint reset");
        KAMI_TRY(stage_in(h, adj_q, 4, memory));
        KAMI_CUDA(launch_scatter4((const float4*)h->d_stage, h->d_gq, h->d_slot_of, h->nv, h->stream), "scatter adjoint");
    }
    kami_status st = on_stream(h, stream, [&](cudaStream_t s) -> kami_status {
        SdfParams no_sdf = h->sdf;
        no_sdf.grid = nullptr;
        for (int step = (int)h->tape_steps.size() - 1; step >= 0; step--) {
            const auto& ts = h->tape_steps[step];
            KAMI_CUDA(launch_adjoint_step(h->window_state(), h->pp, ts.sp, ts.sdf ? h->sdf : no_sdf, h->tape(step), ad,
                                          h->layout.C, s, h->layout.K),
                      "adjoint step launch");
        }
        return KAMI_OK;
    });
    if (st != KAMI_OK) return st;
    h->tape_steps.clear();
    if (wv) {
        for (int a = 0; a < 3; a++)
            KAMI_CUDA(launch_gather_slots(adj3[a], ins3[a], wv, ws0, wn, 3, h->stream), "gather adjoint");
        KAMI_CUDA(launch_gather_slots(h->d_gq, adj_q, wv, ws0, wn, 4, h->stream), "gather adjoint");
    } else {
        for (int a = 0; a < 3; a++) {
            KAMI_CUDA(launch_gather3(adj3[a], h->d_stage, h->d_slot_of, h->nv, h->stream), "gather adjoint");
            KAMI_TRY(stage_out(h, ins3[a], 3, memory));
        }
        KAMI_CUDA(launch_gather4(h->d_gq, (float4*)h->d_stage, h->d_slot_of, h->nv, h->stream), "gather adjoint");
        KAMI_TRY(stage_out(h, adj_q, 4, memory));
    }
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    return KAMI_OK;
}

kami_status kami_vbd_get_rest_darboux_grad(kami_vbd_handle h, float* xyzw, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (!h->d_gqr) return fail(KAMI_ERR_STATE, "call kami_vbd_tape_reserve first");
    return get4(h, h->d_gqr, xyzw, memory);
}

kami_status kami_vbd_zero_rest_darboux_grad(kami_vbd_handle h) {
    KAMI_TRY(valid_handle(h));
    if (!h->d_gqr) return fail(KAMI_ERR_STATE, "call kami_vbd_tape_reserve first");
    KAMI_CUDA(cudaMemsetAsync(h->d_gqr, 0, sizeof(float4) * h->layout.num_slots, h->stream), "gradient reset");
    return KAMI_OK;
}

kami_status kami_vbd_sag_free(kami_vbd_handle h, int32_t iterations) {
    KAMI_TRY(valid_handle(h));
    if (iterations < 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "iterations must be >= 0");
    if (iterations == 0) return KAMI_OK;
    int32_t* d_sb = nullptr;
    float* d_fs = nullptr;
    cudaError_t e = dalloc(&d_sb, (size_t)h->ns + 1);
    if (e == cudaSuccess) e = dalloc(&d_fs, (size_t)h->layout.num_slots);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_sb, h->strand_begin.data(), sizeof(int32_t) * (h->ns + 1), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = launch_sag_free(h->dstate(), make_float3(h->pp.gx, h->pp.gy, h->pp.gz), d_sb, h->d_slot_of, h->ns, d_fs,
                            iterations, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (d_sb) cudaFree(d_sb);
    if (d_fs) cudaFree(d_fs);
    if (e != cudaSuccess) return cuda_fail(e, "sag-free initialisation");
    return KAMI_OK;
}

kami_status kami_vbd_set_hair_layout(kami_vbd_handle h, int32_t hair_strands, int32_t max_verts,
                                     const int32_t* strand_refs) {
    KAMI_TRY(valid_handle(h));
    if (hair_strands <= 0 || max_verts <= 0) return fail(KAMI_ERR_INVALID_ARGUMENT, "hair_strands and max_verts must be > 0");
    std::vector<char> used(hair_strands, 0);
    std::vector<int64_t> index(h->nv);
    for (int32_t s = 0; s < h->ns; s++) {
        const int32_t u = strand_refs ? strand_refs[s] : s;
        if (u < 0 || u >= hair_strands) return fail(KAMI_ERR_INVALID_ARGUMENT, "strand_refs[%d] = %d is not a Hair strand", s, u);
        if (used[u]) return fail(KAMI_ERR_INVALID_ARGUMENT, "Hair strand %d is referenced twice", u);
        used[u] = 1;
        const int32_t len = h->strand_begin[s + 1] - h->strand_begin[s];
        if (len > max_verts)
            return fail(KAMI_ERR_INVALID_ARGUMENT, "strand %d has %d vertices, more than max_verts = %d", s, len, max_verts);
        for (int32_t v = 0; v < len; v++) index[h->strand_begin[s] + v] = (int64_t)u * max_verts + v;
    }
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    if (h->d_hair_index) cudaFree(h->d_hair_index);
    if (h->d_hair_stage) cudaFree(h->d_hair_stage);
    h->d_hair_index = nullptr;
    h->d_hair_stage = nullptr;
    h->hair_entries = 0;
    KAMI_CUDA(dalloc(&h->d_hair_index, h->nv), "Hair layout");
    KAMI_CUDA(cudaMemcpy(h->d_hair_index, index.data(), sizeof(int64_t) * h->nv, cudaMemcpyHostToDevice), "Hair layout");
    h->hair_entries = (int64_t)hair_strands * max_verts;
    h->hair_index.swap(index);
    h->runs_C = 0;  // the host-frame runs are rebuilt with the Hair's entries
    return KAMI_OK;
}

static kami_status hair_stage(kami_vbd_solver* h) {
    if (!h->d_hair_stage) KAMI_CUDA(dalloc(&h->d_hair_stage, 3 * h->hair_entries), "Hair staging buffer");
    return KAMI_OK;
}

kami_status kami_vbd_upload_hair(kami_vbd_handle h, const float* xyz, const float* vxyz, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (!h->d_hair_index) return fail(KAMI_ERR_STATE, "call kami_vbd_set_hair_layout first");
    if (memory != KAMI_MEMORY_HOST && memory != KAMI_MEMORY_DEVICE) return fail(KAMI_ERR_INVALID_ARGUMENT, "bad memory kind");
    const float* srcs[2] = {xyz, vxyz};
    float4* dsts[2] = {h->d_xm, h->d_vel};
    const size_t bytes = sizeof(float) * 3 * h->hair_entries;
    for (int a = 0; a < 2; a++) {
        if (!srcs[a]) continue;
        const float* src = srcs[a];
        const float* mapped = memory == KAMI_MEMORY_HOST ? mapped_range(src, 3 * h->hair_entries) : nullptr;
        if (mapped) {  // page-locked and mapped: the scatter kernel reads the Hair over PCIe itself
            src = mapped;
        } else if (memory == KAMI_MEMORY_HOST) {
            KAMI_TRY(hair_stage(h));
            KAMI_CUDA(cudaMemcpyAsync(h->d_hair_stage, src, bytes, cudaMemcpyHostToDevice, h->stream), "Hair copy in");
            src = h->d_hair_stage;
        }
        KAMI_CUDA(launch_hair_in(src, dsts[a], h->d_slot_of, h->d_hair_index, h->nv, h->stream), "Hair scatter");
    }
    if (memory == KAMI_MEMORY_HOST) KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    return KAMI_OK;
}

kami_status kami_vbd_download_hair(kami_vbd_handle h, float* xyz, float* vxyz, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (!h->d_hair_index) return fail(KAMI_ERR_STATE, "call kami_vbd_set_hair_layout first");
    if (memory != KAMI_MEMORY_HOST && memory != KAMI_MEMORY_DEVICE) return fail(KAMI_ERR_INVALID_ARGUMENT, "bad memory kind");
    float* dsts[2] = {xyz, vxyz};
    const float4* srcs[2] = {h->d_xm, h->d_vel};
    const size_t bytes = sizeof(float) * 3 * h->hair_entries;
    for (int a = 0; a < 2; a++) {
        if (!dsts[a]) continue;
        float* mapped = memory == KAMI_MEMORY_HOST ? mapped_range(dsts[a], 3 * h->hair_entries) : nullptr;
        if (memory == KAMI_MEMORY_DEVICE || mapped) {
            // device memory, or page-locked and mapped: the gather kernel writes the owned entries in place
            KAMI_CUDA(launch_hair_out(srcs[a], mapped ? mapped : dsts[a], h->d_slot_of, h->d_hair_index, h->nv,
                                      h->stream),
                      "Hair gather");
        } else {
            // the padded entries the solver does not own (skipped strands, padding) keep their values
            KAMI_TRY(hair_stage(h));
            KAMI_CUDA(cudaMemcpyAsync(h->d_hair_stage, dsts[a], bytes, cudaMemcpyHostToDevice, h->stream), "Hair copy in");
            KAMI_CUDA(launch_hair_out(srcs[a], h->d_hair_stage, h->d_slot_of, h->d_hair_index, h->nv, h->stream), "Hair gather");
            KAMI_CUDA(cudaMemcpyAsync(dsts[a], h->d_hair_stage, bytes, cudaMemcpyDeviceToHost, h->stream), "Hair copy out");
        }
    }
    return check_status_word(h);
}

kami_status kami_vbd_strain_limit(kami_vbd_handle h, float strain_error, void* stream) {
    KAMI_TRY(valid_handle(h));
    if (!std::isfinite(strain_error) || strain_error < 0.f)
        return fail(KAMI_ERR_INVALID_ARGUMENT, "strain_error must be finite and >= 0");
    if (!h->tape_steps.empty())
        return fail(KAMI_ERR_STATE, "the tape holds recorded steps; strain limiting has no adjoint, run kami_vbd_backward "
                                    "first");
    if (!h->d_strand_root) {
        // strands in the order of their root slots; the staged form gives each CTA a slot range of whole
        // tile groups (at least 2,048 slots) and the strands rooted in it
        std::vector<int32_t> order(h->ns);
        for (int32_t k = 0; k < h->ns; k++) order[k] = k;
        std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
            return h->layout.slot_of[h->strand_begin[a]] < h->layout.slot_of[h->strand_begin[b]];
        });
        std::vector<int64_t> root(h->ns);
        std::vector<int32_t> len(h->ns);
        for (int32_t k = 0; k < h->ns; k++) {
            root[k] = h->layout.slot_of[h->strand_begin[order[k]]];
            len[k] = h->strand_begin[order[k] + 1] - h->strand_begin[order[k]];
        }
        const int64_t unit = 32LL * h->layout.C * std::max(1, h->layout.K);  // slots of a tile group
        int64_t per_cta = unit * std::max<int64_t>(1, 2048 / unit);
        std::vector<int32_t> cta;
        if (per_cta <= kStrainStagedMaxSlots) {
            const int64_t n_cta = (h->layout.num_slots + per_cta - 1) / per_cta;
            cta.assign(n_cta + 1, 0);
            int32_t k = 0;
            for (int64_t c = 0; c <= n_cta; c++) {
                while (k < h->ns && root[k] < c * per_cta) k++;
                cta[c] = k;
            }
        } else {
            per_cta = 0;
        }
        KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        cudaError_t e = dalloc(&h->d_strand_root, (size_t)h->ns);
        if (e == cudaSuccess) e = dalloc(&h->d_strand_len, (size_t)h->ns);
        if (e == cudaSuccess && !cta.empty()) e = dalloc(&h->d_strand_cta, cta.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(h->d_strand_root, root.data(), sizeof(int64_t) * h->ns, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->d_strand_len, len.data(), sizeof(int32_t) * h->ns, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !cta.empty())
            e = cudaMemcpy(h->d_strand_cta, cta.data(), sizeof(int32_t) * cta.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            if (h->d_strand_root) cudaFree(h->d_strand_root);
            if (h->d_strand_len) cudaFree(h->d_strand_len);
            if (h->d_strand_cta) cudaFree(h->d_strand_cta);
            h->d_strand_root = nullptr;
            h->d_strand_len = nullptr;
            h->d_strand_cta = nullptr;
            return cuda_fail(e, "strain limiting strand table");
        }
        h->strain_ctas = cta.empty() ? 0 : (int32_t)(cta.size() - 1);
        h->strain_slots_per_cta = (int32_t)per_cta;
    }
    return on_stream(h, stream, [&](cudaStream_t s) -> kami_status {
        if (h->strain_ctas > 0)
            KAMI_CUDA(launch_strain_limit_staged(h->d_xm, h->d_prm, h->d_strand_root, h->d_strand_len, h->d_strand_cta,
                                                 h->strain_ctas, h->layout.num_slots, h->strain_slots_per_cta,
                                                 h->layout.C, strain_error, s),
                      "strain limiting launch");
        else
            KAMI_CUDA(launch_strain_limit(h->d_xm, h->d_prm, h->d_strand_root, h->d_strand_len, h->ns, h->layout.C,
                                          strain_error, s),
                      "strain limiting launch");
        return KAMI_OK;
    });
}

kami_status kami_vbd_synchronize(kami_vbd_handle h) {
    KAMI_TRY(valid_handle(h));
    return check_status_word(h);
}

kami_status kami_vbd_state_size(kami_vbd_handle h, size_t* bytes) {
    if (!h || !bytes) return fail(KAMI_ERR_INVALID_ARGUMENT, "null argument");
    *bytes = sizeof(float) * 13 * (size_t)h->nv + 4 * sizeof(float);
    return KAMI_OK;
}

kami_status kami_vbd_get_state(kami_vbd_handle h, void* dst, size_t bytes, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    size_t need = 0;
    kami_vbd_state_size(h, &need);
    if (!dst || bytes < need) return fail(KAMI_ERR_INVALID_ARGUMENT, "state buffer must hold %zu bytes", need);
    float* f = (float*)dst;
    const int64_t nv = h->nv;
    cudaMemcpyKind kind = memory == KAMI_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const float4* srcs[3] = {h->d_xm, h->d_vel, h->d_vlast};
    for (int a = 0; a < 3; a++) {
        KAMI_CUDA(launch_gather3(srcs[a], h->d_stage, h->d_slot_of, nv, h->stream), "gather state");
        KAMI_CUDA(cudaMemcpyAsync(f + 3 * nv * a, h->d_stage, sizeof(float) * 3 * nv, kind, h->stream), "state copy");
    }
    KAMI_CUDA(launch_gather4(h->d_q, (float4*)h->d_stage, h->d_slot_of, nv, h->stream), "gather state");
    KAMI_CUDA(cudaMemcpyAsync(f + 9 * nv, h->d_stage, sizeof(float) * 4 * nv, kind, h->stream), "state copy");
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    // the fourth word holds the substep counter (uint32 bits), which paces hair-hair detection
    const uint32_t ctr = (uint32_t)h->counter;
    float ctr_f;
    std::memcpy(&ctr_f, &ctr, 4);
    const float clk[4] = {h->h, h->last_h, h->time, ctr_f};
    if (memory == KAMI_MEMORY_DEVICE)
        KAMI_CUDA(cudaMemcpy(f + 13 * nv, clk, sizeof(clk), cudaMemcpyHostToDevice), "state clock");
    else
        std::memcpy(f + 13 * nv, clk, sizeof(clk));
    return KAMI_OK;
}

kami_status kami_vbd_set_state(kami_vbd_handle h, const void* src, size_t bytes, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    size_t need = 0;
    kami_vbd_state_size(h, &need);
    if (!src || bytes < need) return fail(KAMI_ERR_INVALID_ARGUMENT, "state buffer must hold %zu bytes", need);
    const float* f = (const float*)src;
    const int64_t nv = h->nv;
    cudaMemcpyKind kind = memory == KAMI_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    float4* dsts[3] = {h->d_xm, h->d_vel, h->d_vlast};
    for (int a = 0; a < 3; a++) {
        KAMI_CUDA(cudaMemcpyAsync(h->d_stage, f + 3 * nv * a, sizeof(float) * 3 * nv, kind, h->stream), "state copy");
        KAMI_CUDA(launch_scatter3(h->d_stage, dsts[a], h->d_slot_of, nv, h->stream), "scatter state");
    }
    KAMI_CUDA(cudaMemcpyAsync(h->d_stage, f + 9 * nv, sizeof(float) * 4 * nv, kind, h->stream), "state copy");
    KAMI_CUDA(launch_scatter4((const float4*)h->d_stage, h->d_q, h->d_slot_of, nv, h->stream), "scatter state");
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    float clk[4];
    if (memory == KAMI_MEMORY_DEVICE)
        KAMI_CUDA(cudaMemcpy(clk, f + 13 * nv, sizeof(clk), cudaMemcpyDeviceToHost), "state clock");
    else
        std::memcpy(clk, f + 13 * nv, sizeof(clk));
    h->h = clk[0];
    h->last_h = clk[1];
    h->time = clk[2];
    uint32_t ctr;
    std::memcpy(&ctr, &clk[3], 4);
    h->counter = ctr;
    h->coll_stale = true;  // the contact lists belong to the state before
    return KAMI_OK;
}

kami_status kami_vbd_restore_tape_window(kami_vbd_handle h, const void* src, size_t bytes, int32_t memory) {
    KAMI_TRY(valid_handle(h));
    if (h->tape_capacity == 0) return fail(KAMI_ERR_STATE, "call kami_vbd_tape_reserve first");
    const int64_t* wv = nullptr;
    int64_t ws0 = 0, wn = 0;
    if (memory == KAMI_MEMORY_DEVICE) KAMI_TRY(window_slots(h, &wv, &ws0, &wn));
    if (!wv) return kami_vbd_set_state(h, src, bytes, memory);  // the whole groom, or host memory
    size_t need = 0;
    kami_vbd_state_size(h, &need);
    if (!src || bytes < need) return fail(KAMI_ERR_INVALID_ARGUMENT, "state buffer must hold %zu bytes", need);
    const float* f = (const float*)src;
    const int64_t nv = h->nv;
    float4* dsts[3] = {h->d_xm, h->d_vel, h->d_vlast};
    for (int a = 0; a < 3; a++)
        KAMI_CUDA(launch_scatter_slots(f + 3 * nv * a, dsts[a], wv, ws0, wn, 3, h->stream), "scatter state");
    KAMI_CUDA(launch_scatter_slots(f + 9 * nv, h->d_q, wv, ws0, wn, 4, h->stream), "scatter state");
    float clk[4];
    KAMI_CUDA(cudaMemcpyAsync(clk, f + 13 * nv, sizeof(clk), cudaMemcpyDeviceToHost, h->stream), "state clock");
    KAMI_CUDA(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    h->h = clk[0];
    h->last_h = clk[1];
    h->time = clk[2];
    uint32_t ctr;
    std::memcpy(&ctr, &clk[3], 4);
    h->counter = ctr;
    h->coll_stale = true;
    return KAMI_OK;
}

const char* kami_vbd_last_error_string(void) { return g_last_error.c_str(); }

const char* kami_vbd_version(void) { return "kami-vbd-b200 0.1 (sm_100a)"; }

}  // extern "C"
