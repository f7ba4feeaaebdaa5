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
    int64_t num_tiles = 0;
    int64_t num_slots = 0;
    std::vector<int64_t> slot_of;  // storage index of each boundary-order vertex
};

// Packs strands (CSR offsets sb[0..ns]) into tiles of 32*C slots.  Each strand takes a
// contiguous run of slots starting at an even slot (its length rounded up to even).  Strands are
// placed longest first into the fullest tile that still has room (best fit decreasing), so
// uneven strands share tiles.  Returns false when a strand is longer than a tile.
bool pack_tiles(const int32_t* sb, int32_t ns, int C, TileLayout& out, std::string& err);

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
