// vbd_kernels.h -- host-side launchers of the solver's kernels (vbd_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vbd_common.cuh"

namespace kami {

cudaError_t launch_sweep_predict(const DeviceState& st, float4* y4, float4* dx4, const StepParams* d_sp,
                                 const PhysParams& pp, int64_t num_slots, cudaStream_t s);
// conn_dx: the partners' dx for tied vertices (st.conn), the iteration's starting values
cudaError_t launch_sweep_position(const DeviceState& st, const float4* y4, const float4* q, const float4* dx_in,
                                  float4* dx_out, const StepParams* d_sp, const PhysParams& pp, int C, int colour,
                                  bool jacobi, cudaStream_t s, const float4* conn_dx = nullptr);
// One iteration (colour2: both position sweeps, both orientation sweeps; jacobi: the position and
// the orientation sweep) in one launch, one block per tile of up to 1024 slots: reads dx_in, writes
// dx_out; q in place for colour2 (q_in == q_out), into q_out for jacobi (sweep_iteration_supported).
bool sweep_iteration_supported(int C);
cudaError_t launch_sweep_iteration(const DeviceState& st, const float4* y4, const float4* q_in, float4* q_out,
                                   const float4* dx_in, float4* dx_out, const StepParams* d_sp, const PhysParams& pp,
                                   int C, bool jacobi, cudaStream_t s);
cudaError_t launch_sweep_orientation(const DeviceState& st, const float4* dx4, const float4* q_in, float4* q_out, int C,
                                     int colour, bool jacobi, cudaStream_t s);
cudaError_t launch_sweep_finish(const DeviceState& st, const float4* dx4, const StepParams* d_sp, const PhysParams& pp,
                                const SdfParams& sdf, bool apply_sdf, int64_t num_slots, cudaStream_t s);

bool fused_supported(int C);
// nsteps consecutive steps in one launch: parameters from d_steps[0..nsteps) (device), or sp when
// d_steps is null (then nsteps must be 1).  group > 1: the layout's groups of `group` tiles, one CTA
// of `group` warps each (warps_per_block and the packed variant do not apply).
// launch_mode: 0 = one CTA per W tiles (or per group), scheduled by the hardware; LAUNCH_PERSISTENT =
// resident CTAs loop over the tiles (fused_persistent_kernel; the packed variant has no persistent form).
enum : int { LAUNCH_PERSISTENT = 1 };
cudaError_t launch_fused_step(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                              int C, bool jacobi, int warps_per_block, cudaStream_t s, const StepParams* d_steps = nullptr,
                              int nsteps = 1, int reg_cap = 0, int group = 1, int launch_mode = 0);

// One step as an upload-step-download frame over the host buffers of hio (fused_frame_kernel);
// same tile shapes and register variants as launch_fused_step.
cudaError_t launch_fused_frame(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                               const HostIO& hio, int C, bool jacobi, int warps_per_block, cudaStream_t s, int reg_cap,
                               int group = 1);

// group > 1: groups of tiles, one CTA of `group` warps each (2, 4 or 8);
// the tape window must be whole groups.
cudaError_t launch_fused_record(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                                const TapeView& tp, int C, int warps_per_block, cudaStream_t s, int group = 1);
cudaError_t launch_adjoint_step(const DeviceState& st, const PhysParams& pp, const StepParams& sp, const SdfParams& sdf,
                                const TapeView& tp, const AdjointState& ad, int C, cudaStream_t s, int group = 1);

// Hair-hair collision (vbd_collision.cu).  coll_scan_tmp_size: int32 elements of scratch the
// bucket scan of a table of n buckets needs.
int64_t coll_scan_tmp_size(int64_t n);
cudaError_t launch_coll_detect(const DeviceState& st, const float4* dx4, const CollParams& cp, cudaStream_t s);
cudaError_t launch_coll_steplimit(const DeviceState& st, const float4* dx4, const CollParams& cp, cudaStream_t s);
// One colour2 iteration of the sweep form with contacts in one launch (one block per tile, one
// thread per slot): reads the iteration's starting displacements from snap, writes dx_out, updates
// q in place.  Tiles of up to 1024 slots (coll_iteration_supported).
bool coll_iteration_supported(int C);
cudaError_t launch_coll_iteration(const DeviceState& st, const float4* y4, float4* q, const float4* snap, float4* dx_out,
                                  const StepParams* d_sp, const PhysParams& pp, const CollParams& cp, cudaStream_t s);
cudaError_t launch_sweep_position_coll(const DeviceState& st, const float4* y4, const float4* q, const float4* dx_in,
                                       float4* dx_out, const float4* snap, const StepParams* d_sp, const PhysParams& pp,
                                       const CollParams& cp, int colour, bool jacobi, cudaStream_t s);

// Strain limiting after the step (strain_limit_kernel): root slot and vertex count of each strand.
cudaError_t launch_strain_limit(float4* xm, const float4* prm, const int64_t* root_slot, const int32_t* strand_len,
                                int32_t num_strands, int C, float strain_error, cudaStream_t s);
// The same with the state staged in shared memory (strain_limit_staged_kernel): slots_per_cta is a
// multiple of the tile group (tiles_per_group x 32 C slots), root_slot ascending, cta_begin[num_ctas
// + 1] the first strand of each CTA's slot range.
constexpr int kStrainStagedMaxSlots = 11000;  // 20 B of shared memory per slot
cudaError_t launch_strain_limit_staged(float4* xm, const float4* prm, const int64_t* root_slot,
                                       const int32_t* strand_len, const int32_t* cta_begin, int32_t num_ctas,
                                       int64_t num_slots, int slots_per_cta, int C, float strain_error, cudaStream_t s);

// sag-free initialisation (sag_free.cu): `iterations` passes, one thread per strand; fs: a float per slot
cudaError_t launch_sag_free(const DeviceState& st, float3 gravity, const int32_t* strand_begin, const int64_t* slot_of,
                            int32_t num_strands, float* fs, int iterations, cudaStream_t s);

// padded Hair arrays <-> tile slots (hair_index: padded entry of each boundary vertex)
cudaError_t launch_hair_in(const float* src, float4* dst, const int64_t* slot_of, const int64_t* hair_index, int64_t nv,
                           cudaStream_t s);
cudaError_t launch_hair_out(const float4* src, float* dst, const int64_t* slot_of, const int64_t* hair_index, int64_t nv,
                            cudaStream_t s);

cudaError_t launch_scatter3(const float* src, float4* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s);
cudaError_t launch_gather3(const float4* src, float* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s);
cudaError_t launch_scatter4(const float4* src, float4* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s);
cudaError_t launch_gather4(const float4* src, float4* dst, const int64_t* slot_of, int64_t nv, cudaStream_t s);

// Tape windows: vert_of (num_slots entries) = the boundary vertex of every slot, -1 for padding; and
// slots [s0, s0 + n) <-> their vertices in a caller's boundary array of `comps` (3 or 4) floats per
// vertex, any 4-byte alignment (a 3-component scatter keeps the slot's .w).
cudaError_t launch_vert_of(const int64_t* slot_of, int64_t* vert_of, int64_t nv, int64_t num_slots, cudaStream_t s);
cudaError_t launch_scatter_slots(const float* src, float4* dst, const int64_t* vert_of, int64_t s0, int64_t n, int comps,
                                 cudaStream_t s);
cudaError_t launch_gather_slots(const float4* src, float* dst, const int64_t* vert_of, int64_t s0, int64_t n, int comps,
                                cudaStream_t s);

}  // namespace kami
