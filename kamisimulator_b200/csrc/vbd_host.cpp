// vbd_host.cpp -- strand-to-tile packing and per-vertex set-up (see vbd_host.h).
#include "vbd_host.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "vbd_common.cuh"

namespace kami {

int slots_per_lane_for(const int32_t* sb, int32_t ns) {
    int32_t longest = 0;
    for (int32_t s = 0; s < ns; s++) longest = std::max(longest, sb[s + 1] - sb[s]);
    int C = (longest + 31) / 32;
    C += C & 1;
    return std::max(C, 2);
}

int tiles_per_group_for(const int32_t* sb, int32_t ns, int C) {
    int32_t longest = 0;
    for (int32_t s = 0; s < ns; s++) longest = std::max(longest, sb[s + 1] - sb[s]);
    longest += longest & 1;
    for (int K = 1; K <= 8; K *= 2)
        if (longest <= 32 * C * K) return K;
    return 0;
}

bool pack_tiles(const int32_t* sb, int32_t ns, int C, TileLayout& out, std::string& err, int K) {
    const int Tt = 32 * C;  // slots per tile
    const int T = Tt * K;   // positions per group
    out.C = C;
    out.K = K;
    out.slot_of.assign(ns > 0 ? (size_t)sb[ns] : 0, -1);
    std::vector<int32_t> order(ns);
    std::iota(order.begin(), order.end(), 0);
    auto need = [&](int32_t s) { int n = sb[s + 1] - sb[s]; return n + (n & 1); };
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return need(a) > need(b); });
    // open groups bucketed by free positions; each bucket is a stack of group ids
    std::vector<std::vector<int64_t>> bucket(T + 1);
    std::vector<int> used;  // positions used per group
    for (int32_t s : order) {
        const int n = need(s);
        if (n > T) {
            err = "strand " + std::to_string(s) + " has " + std::to_string(sb[s + 1] - sb[s]) +
                  " vertices, more than a group of " + std::to_string(T) + " slots";
            return false;
        }
        int64_t tile = -1;
        for (int r = n; r <= T; r++) {
            if (!bucket[r].empty()) {
                tile = bucket[r].back();
                bucket[r].pop_back();
                break;
            }
        }
        if (tile < 0) {
            tile = (int64_t)used.size();
            used.push_back(0);
        }
        const int p0 = used[tile];  // `tile` numbers groups here
        for (int32_t j = 0; j < sb[s + 1] - sb[s]; j++) {
            const int p = p0 + j, pt = p % Tt;
            out.slot_of[sb[s] + j] = (tile * K + p / Tt) * Tt + (int64_t)(pt % C) * 32 + pt / C;
        }
        used[tile] += n;
        const int free_slots = T - used[tile];
        if (free_slots >= 2) bucket[free_slots].push_back(tile);
    }
    out.num_tiles = (int64_t)used.size() * K;
    out.num_slots = out.num_tiles * Tt;
    return true;
}

namespace {
constexpr double kPi = 3.141592653589793238462643;  // YBSimulator.cu:55

struct Q {
    float x, y, z, w;
};
inline Q qmul(Q l, Q r) {
    return {l.w * r.x + r.w * l.x + (l.y * r.z - r.y * l.z), l.w * r.y + r.w * l.y + (l.z * r.x - r.z * l.x),
            l.w * r.z + r.w * l.z + (l.x * r.y - r.x * l.y), l.w * r.w - (l.x * r.x + l.y * r.y + l.z * r.z)};
}
inline Q qnormalize(Q a) {
    float s = 1.f / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w);
    return {a.x * s, a.y * s, a.z * s, a.w * s};
}
// Rotor::fromTo(e_x, to) (KittenEngine Rotor.h:79-88); `to` is a unit vector.  The antiparallel
// case takes the second axis of orthoBasisX(e_x) (Common.h:220-232), which is (0, 1, 0).
inline Q from_ex(float tx, float ty, float tz) {
    float hx = (1.f + tx) * 0.5f, hy = ty * 0.5f, hz = tz * 0.5f;
    float l = hx * hx + hy * hy + hz * hz;
    if (l > 0.f) {
        float s = 1.f / std::sqrt(l);
        hx *= s;
        hy *= s;
        hz *= s;
    } else {
        hx = 0.f;
        hy = 1.f;
        hz = 0.f;
    }
    // cross(e_x, h) = (0, -h.z, h.y); dot(e_x, h) = h.x
    return {0.f, -hz, hy, hx};
}
}  // namespace

int build_material(const int32_t* sb, int32_t ns, const float* pos, const MaterialDesc& md, Material& m,
                   std::string& err) {
    const int64_t nv = ns > 0 ? sb[ns] : 0;
    if (nv < 3) {
        err = "too few vertices (the solver needs at least 3)";
        return 1;
    }
    m.inv_mass.assign(nv, 1.f);
    m.l_rest.assign(nv, 1.f / (float)nv);
    m.k_stretch.assign(nv, 100.f);
    m.flags.assign(nv, 0u);
    m.q.assign(4 * nv, 0.f);
    m.q_rest.assign(4 * nv, 0.f);
    // segment flags: a vertex has a next vertex unless it ends its strand (createFromCurves)
    for (int32_t s = 0; s < ns; s++) {
        const int32_t a = sb[s], b = sb[s + 1];
        for (int32_t i = a; i < b; i++) {
            uint32_t f = F_VALID;
            if (i == a) f |= F_ROOT;
            if (i + 1 < b) f |= F_HAS_NEXT;
            if (i > a) f |= F_HAS_PREV;
            if (i + 2 < b) f |= F_HAS_NEXT_ORIENTATION;
            if (i + 1 == b) f |= F_FIX_ORIENTATION;
            m.flags[i] = f;
        }
    }
    // the reference only marks fixOrientation below the last vertex of the whole set
    m.flags[nv - 1] &= ~F_FIX_ORIENTATION;
    for (int64_t i = 0; i < nv; i++)
        if (!(m.flags[i] & (F_HAS_PREV | F_HAS_NEXT))) {
            err = "dangling segment at vertex " + std::to_string(i) + ": strands need at least 2 vertices";
            return 2;
        }
    // rest lengths, orientations, masses (Sim::configure, YBSimulator.cu:168-237)
    const float r = md.radius;
    const double mass_scale = (double)(r * r) * kPi * (double)md.density * 0.5;
    Q last_q = {0.f, 0.f, 0.f, 1.f};
    for (int64_t i = 0; i < nv; i++) {
        float mass = 0.f;
        if (m.flags[i] & F_HAS_PREV) mass += m.l_rest[i - 1];
        if (m.flags[i] & F_HAS_NEXT) {
            float sx = pos[3 * i + 3] - pos[3 * i], sy = pos[3 * i + 4] - pos[3 * i + 1], sz = pos[3 * i + 5] - pos[3 * i + 2];
            float len = std::sqrt(sx * sx + sy * sy + sz * sz);
            if (len == 0.f || !std::isfinite(len)) {
                err = "zero-length or non-finite segment at vertex " + std::to_string(i);
                return 3;
            }
            m.l_rest[i] = len;
            float inv = 1.f / std::sqrt(sx * sx + sy * sy + sz * sz);
            last_q = from_ex(sx * inv, sy * inv, sz * inv);
            mass += len;
        }
        m.q[4 * i] = last_q.x;
        m.q[4 * i + 1] = last_q.y;
        m.q[4 * i + 2] = last_q.z;
        m.q[4 * i + 3] = last_q.w;
        mass = (float)((double)mass * mass_scale);
        if (mass != 0.f)
            m.inv_mass[i] *= 1.f / mass;
        else
            m.inv_mass[i] = 0.f;
    }
    // rest Darboux quaternions, normalize(q_i^-1 q_{i+1}) (YBSimulator.cu:241); the last keeps identity
    for (int64_t i = 0; i < nv; i++) {
        Q rq = {0.f, 0.f, 0.f, 1.f};
        if (i + 1 < nv) {
            Q qi = {-m.q[4 * i], -m.q[4 * i + 1], -m.q[4 * i + 2], m.q[4 * i + 3]};
            Q qj = {m.q[4 * i + 4], m.q[4 * i + 5], m.q[4 * i + 6], m.q[4 * i + 7]};
            rq = qnormalize(qmul(qi, qj));
        }
        m.q_rest[4 * i] = rq.x;
        m.q_rest[4 * i + 1] = rq.y;
        m.q_rest[4 * i + 2] = rq.z;
        m.q_rest[4 * i + 3] = rq.w;
    }
    // stiffness
    if (md.stiffness_mode == 0) {  // setYoung (YBSimulator.cu:300-320), strand by strand
        const float mmrad = md.radius * 1000.f;
        for (int32_t s = 0; s < ns; s++) {
            const float young = md.strand_young ? md.strand_young[s] : md.young;
            const float dev = md.strand_dev ? md.strand_dev[s] : md.deviation;
            const float ss = (float)((double)young * kPi * (double)mmrad * (double)mmrad);
            for (int32_t i = sb[s]; i < sb[s + 1]; i++) {
                const float len = m.l_rest[i];
                const float bt = (float)((double)(ss * dev * mmrad * mmrad) * 0.25 / (double)(len * len));
                m.k_stretch[i] = ss;
                for (int c = 0; c < 4; c++) m.q_rest[4 * i + c] *= bt;
            }
        }
    } else {  // setKBend (:286-298) and setKStretch (:276-284)
        const float kb = md.k_bend * 4.f;
        for (int64_t i = 0; i < nv; i++) {
            Q rq = qnormalize({m.q_rest[4 * i], m.q_rest[4 * i + 1], m.q_rest[4 * i + 2], m.q_rest[4 * i + 3]});
            const float sc = kb / m.l_rest[i];
            m.q_rest[4 * i] = sc * rq.x;
            m.q_rest[4 * i + 1] = sc * rq.y;
            m.q_rest[4 * i + 2] = sc * rq.z;
            m.q_rest[4 * i + 3] = sc * rq.w;
            m.k_stretch[i] = md.k_stretch * m.l_rest[i];
        }
    }
    if (md.pin_roots)
        for (int32_t s = 0; s < ns; s++) m.inv_mass[sb[s]] = 0.f;
    return 0;
}

}  // namespace kami
