// vbd_host.h -- host-side preparation of a solver: strand-to-tile packing and the per-vertex
// material/orientation set-up of YarnBall::Sim.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace kami {

// Placement of strands into warp tiles of 32*C slots (see vbd_common.cuh for the slot layout).
struct TileLayout {
    int C = 2;
    int K = 1;  // tiles per group: a strand may run on from one tile of its group into the next
    int64_t num_tiles = 0;
    int64_t num_slots = 0;
    std::vector<int64_t> slot_of;  // storage index of each boundary-order vertex
};

// Packs strands (CSR offsets sb[0..ns]) into groups of K tiles of 32*C slots.  A group's positions
// p = 0 .. 32*C*K-1 run through its tiles in order (position p is slot (p' % C) * 32 + p' / C of the
// group's tile p / (32*C), p' = p % (32*C)), so a strand may continue from lane 31's last slot of
// one tile into lane 0's first slot of the next.  Each strand takes a contiguous run of positions
// starting at an even one (its length rounded up to even).  Strands are placed longest first into
// the fullest group that still has room (best fit decreasing), so uneven strands share groups.
// Returns false when a strand is longer than a group.
bool pack_tiles(const int32_t* sb, int32_t ns, int C, TileLayout& out, std::string& err, int K = 1);

// Smallest power of two K (<= 8) whose groups of K tiles of 32*C slots hold the longest strand;
// 0 when even 8 tiles are too short.
int tiles_per_group_for(const int32_t* sb, int32_t ns, int C);

// Smallest even C whose tile (32*C slots) holds the longest strand.
int slots_per_lane_for(const int32_t* sb, int32_t ns);

// Per-vertex set-up in boundary order, as YarnBall::Sim ends up after createFromCurves +
// configure + setYoung (or setKStretch/setKBend) + root pinning.
struct Material {
    std::vector<float> inv_mass, l_rest, k_stretch;
    std::vector<uint32_t> flags;  // YarnBall::VertexFlags bits plus F_ROOT / F_VALID
    std::vector<float> q;         // 4 per vertex (x, y, z, w)
    std::vector<float> q_rest;    // 4 per vertex, scaled by the bend/twist stiffness
};

struct MaterialDesc {
    float radius;
    float density;
    int stiffness_mode;        // 0 = Young's modulus, 1 = explicit stretch / bend constants
    const float* strand_young; // per strand, may be null (then `young`)
    const float* strand_dev;   // per strand, may be null (then `deviation`)
    float young, deviation, k_stretch, k_bend;
    bool pin_roots;
};

// Returns 0 on success, 2 for a dangling segment, 3 for a zero-length or non-finite segment,
// 1 for too few vertices.
int build_material(const int32_t* sb, int32_t ns, const float* pos, const MaterialDesc& md, Material& out,
                   std::string& err);

// Sets the message returned by kami_vbd_last_error_string on the calling thread.
void set_last_error(const char* msg);

}  // namespace kami
