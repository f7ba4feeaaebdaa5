// kami_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the Stable Cosserat Rods vertex-block-descent (VBD) step of
// KamiSimulator's StableCosseratRods solver, templated on the scalar type so the
// same update runs in FP32 (parity checker) and FP64 (trajectory-error replay).
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
// library, always as the checker; no product code links or calls it.
//
// Each function names the reference file:line it restates (paths are relative to
// the KamiSimulator project root).  Arithmetic follows the reference's operation
// order where that is cheap to keep, including its quirks:
//   * hess3(float d) fills all six packed entries, so the inertia block is
//     (m/h^2) * ones(3,3), not (m/h^2) * I  (KittenEngine/includes/modules/SymMat.h:16-18,
//     used at YarnBall/sim/cosserat.cu:117);
//   * setYoung works in millimetre units (YarnBall/YBSimulator.cu:300-320);
//   * the SDF lookup rounds to the nearest node but interpolates from idx-0.5
//     (SDFCollisionSolver/cudaSDFCollision.cu:88-96 vs :139-142);
//   * the SDF velocity fix subtracts (v/|v| . n) n (cudaSDFCollision.cu:261-263);
//   * the initial guess uses lastH, the step of the previous advance() call
//     (YarnBall/sim/iteration.cu:49, YarnBall/sim/step.cpp:38-42).
//
// Two deterministic schedules are provided because the reference's own kernels
// race at block boundaries (cosserat.cu:142-143 vs :285, :316-335):
//   schedule 1 "jacobi":  every vertex/segment reads the previous sweep's values
//                         (the reference's intent);
//   schedule 0 "colour2": Gauss-Seidel over a 2-colouring by local index parity
//                         within each strand: even vertices, odd vertices, then
//                         even segments, odd segments.
// Vertices in another vertex's update that other threads may be writing -- hair-hair
// partners and connection-spring partners -- are read as they stood at the start of the
// iteration (a snapshot) under both schedules.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <array>
#include <limits>
#include <map>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

// ---- FLOP counting -------------------------------------------------------------------------------------
// A double that counts the arithmetic made with it: +, -, *, / and sqrt/log count one operation each
// (an FMA is two); negation, comparisons, min/max and conversions are free.  oracle_flop_count
// instantiates the per-vertex updates with it to pin the FLOPs per vertex-iteration of the reference
// update.  Its overloads are declared before the templates so that their qualified std:: calls see them.
struct Counted {
    double v = 0;
    static int64_t ops;  // single-threaded use only (oracle_flop_count)
    Counted() = default;
    Counted(double x) : v(x) {}
    explicit operator double() const { return v; }
};
int64_t Counted::ops = 0;
inline Counted operator+(Counted a, Counted b) { Counted::ops++; return a.v + b.v; }
inline Counted operator-(Counted a, Counted b) { Counted::ops++; return a.v - b.v; }
inline Counted operator*(Counted a, Counted b) { Counted::ops++; return a.v * b.v; }
inline Counted operator/(Counted a, Counted b) { Counted::ops++; return a.v / b.v; }
inline Counted operator-(Counted a) { return -a.v; }
inline Counted operator+(Counted a) { return a; }
inline Counted& operator+=(Counted& a, Counted b) { return a = a + b; }
inline Counted& operator-=(Counted& a, Counted b) { return a = a - b; }
inline Counted& operator*=(Counted& a, Counted b) { return a = a * b; }
inline Counted& operator/=(Counted& a, Counted b) { return a = a / b; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }
namespace std {
inline Counted sqrt(Counted a) { Counted::ops++; return std::sqrt(a.v); }
inline Counted log(Counted a) { Counted::ops++; return std::log(a.v); }
template <>
class numeric_limits<Counted> : public numeric_limits<double> {
   public:
    static Counted infinity() { return numeric_limits<double>::infinity(); }
};
}  // namespace std

namespace {

constexpr double kPi = 3.141592653589793238462643;  // myPi, YBSimulator.cu:55

// Vertex flags, YarnBall/YarnBall.h:33-39.
constexpr uint32_t HAS_PREV = 1, HAS_NEXT = 2, HAS_NEXT_ORIENTATION = 4, FIX_ORIENTATION = 8;

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T>
struct Q4 {  // Kit::Rotor layout: (x, y, z) bivector part, w scalar last (Rotor.h:39-48)
    T x, y, z, w;
};

template <typename T> inline V3<T> v3(T x, T y, T z) { return {x, y, z}; }
template <typename T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <typename T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <typename T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <typename T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <typename T> inline T dot4(Q4<T> a, Q4<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <typename T> inline T length4(Q4<T> a) { return std::sqrt(dot4(a, a)); }
template <typename T> inline Q4<T> qadd(Q4<T> a, Q4<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <typename T> inline Q4<T> qscale(T s, Q4<T> a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template <typename T> inline V3<T> qvec(Q4<T> a) { return {a.x, a.y, a.z}; }
template <typename T> inline Q4<T> qconj(Q4<T> a) { return {-a.x, -a.y, -a.z, a.w}; }  // Rotor::inverse, Rotor.h:109

// Rotor product, Rotor.h:210-212.
template <typename T>
inline Q4<T> qmul(Q4<T> l, Q4<T> r) {
    V3<T> q = l.w * qvec(r) + r.w * qvec(l) + cross(qvec(l), qvec(r));
    return {q.x, q.y, q.z, l.w * r.w - dot(qvec(l), qvec(r))};
}

// Rotor::rotate, Rotor.h:114-123.
template <typename T>
inline V3<T> qrotate(Q4<T> r, V3<T> v) {
    V3<T> qv = qvec(r);
    V3<T> a = r.w * v + cross(qv, v);
    T c = dot(v, qv);
    return r.w * a + cross(qv, a) + c * qv;
}

template <typename T>
inline V3<T> normalize3(V3<T> a) {  // glm::normalize: v * inversesqrt(dot(v, v))
    T s = T(1) / std::sqrt(dot(a, a));
    return a * s;
}
template <typename T>
inline Q4<T> normalize4(Q4<T> a) {
    T s = T(1) / std::sqrt(dot4(a, a));
    return qscale(s, a);
}

// Rotor::fromTo, Rotor.h:79-88, with orthoBasisX (KittenEngine Common.h:220-232).
template <typename T>
inline Q4<T> fromTo(V3<T> from, V3<T> to) {
    V3<T> h = (from + to) * T(0.5);
    T l = dot(h, h);
    if (l > 0) {
        h = h * (T(1) / std::sqrt(l));
    } else {
        V3<T> n = from;
        if (n.z >= n.y) {
            T a = T(1) / (T(1) + n.z);
            T b = -n.x * n.y * a;
            h = v3<T>(b, T(1) - n.y * n.y * a, -n.y);
        } else {
            T a = T(1) / (T(1) + n.y);
            T b = -n.x * n.z * a;
            h = v3<T>(T(1) - n.x * n.x * a, -n.x, b);
        }
    }
    V3<T> c = cross(from, h);
    return {c.x, c.y, c.z, dot(from, h)};
}

// glm::inverse(mat3) (extern/glm/glm/detail/func_matrix.inl compute_inverse<3,3>) applied to
// a packed symmetric hess3 converted with hess3::operator mat3 (SymMat.h:66-75), then mat3*vec3.
template <typename T>
inline V3<T> solveHess3(const T H[6], V3<T> f) {
    T m[3][3];  // m[col][row]
    m[0][0] = H[0];
    m[1][1] = H[1];
    m[2][2] = H[2];
    m[0][1] = m[1][0] = H[3];
    m[0][2] = m[2][0] = H[4];
    m[1][2] = m[2][1] = H[5];
    T det = +m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
            m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
    T od = T(1) / det;
    T inv[3][3];
    inv[0][0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * od;
    inv[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * od;
    inv[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * od;
    inv[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * od;
    inv[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * od;
    inv[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * od;
    inv[0][2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * od;
    inv[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * od;
    inv[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * od;
    return {inv[0][0] * f.x + inv[1][0] * f.y + inv[2][0] * f.z, inv[0][1] * f.x + inv[1][1] * f.y + inv[2][1] * f.z,
            inv[0][2] * f.x + inv[1][2] * f.y + inv[2][2] * f.z};
}

template <typename T> inline V3<T> ld3(const T* a, int64_t i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
template <typename T> inline void st3(T* a, int64_t i, V3<T> v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }
template <typename T> inline Q4<T> ld4(const T* a, int64_t i) { return {a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]}; }
template <typename T> inline void st4(T* a, int64_t i, Q4<T> q) { a[4 * i] = q.x; a[4 * i + 1] = q.y; a[4 * i + 2] = q.z; a[4 * i + 3] = q.w; }

}  // namespace

extern "C" {

// Parameters of one solver instance (scalars of YarnBall::MetaData, YarnBall.h:61-124,
// plus the SDFSimulationParams of cudaSDFCollision.cuh:23-48 that the SDF pass reads).
typedef struct oracle_params {
    float gravity[3];
    float damping;            // MetaData::damping (1e-6)
    float velocity_decay;     // MetaData::velocityDecay
    float acceleration_ratio; // MetaData::accelerationRatio (1)
    float ext_mult;           // MetaData::ExternalForceMultiplier
    float wind_peak, wind_y_freq, wind_z_freq, wind_time_freq, wind_sharpness;
    int32_t num_itr;
    int32_t schedule;  // 0 = colour2 Gauss-Seidel, 1 = jacobi
    float max_h;       // Sim::maxH
    int32_t sdf_enabled;
    int32_t sdf_dims[3];
    float sdf_min[3];
    float sdf_max[3];
    float sdf_threshold;
    const float* sdf_phi;   // [nz][ny][nx]
    const float* sdf_grad;  // [nz][ny][nx][3]
    float body_rot[4];      // (x, y, z, w)
    float body_trans[3];
    int32_t num_threads;    // <= 0: OpenMP default
    // hair-hair collision (MetaData, YarnBall.h:93-114; StableCosseratRodsSolver.cpp:176-186)
    int32_t hair_hair;        // enableHairHairColl
    float radius;             // MetaData::radius
    float barrier_thickness;  // barrierThickness
    float k_collision;        // kCollision
    float k_friction;         // kFriction
    float friction_coeff;     // frictionCoeff
    float detection_scaler;   // detectionScaler
    int32_t detection_period; // detectionPeriod
    int32_t step_limit;       // useStepSizeLimit
    int32_t velocity_radius;  // useVelocityRadius
    // Vertex::connectionIndex (YarnBall.h:56): per vertex the vertex it is tied to, or -1; null = none
    const int32_t* connection;
} oracle_params;

}  // extern "C"

namespace {

template <typename T>
struct Topology {
    int64_t nv;
    int32_t ns;
    const int32_t* sb;
    std::vector<int32_t> local;  // local index of each vertex inside its strand
    Topology(int64_t nv_, int32_t ns_, const int32_t* sb_) : nv(nv_), ns(ns_), sb(sb_), local(nv_) {
        for (int32_t s = 0; s < ns; s++)
            for (int32_t i = sb[s]; i < sb[s + 1]; i++) local[i] = i - sb[s];
    }
};

// createFromCurves (YarnBall/io/reader.cpp:16-50) + Sim::Sim (YBSimulator.cu:81-127) +
// Sim::configure (YBSimulator.cu:161-241) + setYoung (:300-320) / setKStretch (:276-284) /
// setKBend (:286-298) + root pinning (StableCosseratRods/StableCosseratRodsSolver.cpp:203-205).
// strand_young / strand_dev give one Young's modulus [GPa] / bend deviation per strand; the
// reference's setYoung applies a single pair to every vertex, and a per-strand pair is the same
// formula applied strand by strand.
template <typename T>
int configureT(int64_t nv, int32_t ns, const int32_t* sb, const float* pos, float radius, float density,
               int32_t stiffness_mode, const float* strand_young, const float* strand_dev, float k_stretch_in,
               float k_bend_in, int32_t pin_roots, T* inv_mass, T* l_rest, T* k_stretch, uint32_t* flags, T* q,
               T* q_rest) {
    if (nv < 3) return 1;  // Sim::Sim throws "Too little vertices"
    std::vector<uint32_t> fl(nv, HAS_NEXT);
    fl[nv - 1] = 0;
    for (int32_t s = 0; s < ns; s++) fl[sb[s + 1] - 1] = 0;  // cut off each curve end
    std::vector<T> im(nv, T(1)), lr(nv, T(1));
    std::vector<Q4<T>> qs(nv);
    Q4<T> lastQ = {0, 0, 0, 1};
    const T r = (T)radius;
    for (int64_t i = 0; i < nv; i++) {
        if (i < nv - 1) {
            bool hasNext = (fl[i] & HAS_NEXT) != 0;
            fl[i + 1] = hasNext ? (fl[i + 1] | HAS_PREV) : (fl[i + 1] & ~HAS_PREV);
            bool hasNextNext = hasNext && (fl[i + 1] & HAS_NEXT);
            fl[i] = hasNextNext ? (fl[i] | HAS_NEXT_ORIENTATION) : (fl[i] & ~HAS_NEXT_ORIENTATION);
            if (!hasNext) fl[i] |= FIX_ORIENTATION;
        }
        if (!(fl[i] & HAS_PREV) && !(fl[i] & HAS_NEXT)) return 2;  // dangling segment
        lr[i] = T(1) / (T)nv;
        T mass = 0;
        if (fl[i] & HAS_PREV) mass += lr[i - 1];
        if (fl[i] & HAS_NEXT) {
            V3<T> p0 = v3<T>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
            V3<T> p1 = v3<T>(pos[3 * i + 3], pos[3 * i + 4], pos[3 * i + 5]);
            V3<T> seg = p1 - p0;
            lr[i] = length(seg);
            if (lr[i] == 0 || !std::isfinite((double)lr[i])) return 3;  // 0 length segment
            lastQ = fromTo<T>(v3<T>(1, 0, 0), normalize3(seg));
            mass += lr[i];
        }
        qs[i] = lastQ;
        // mass = (l_{i-1} + l_i) r^2 pi rho / 2, YBSimulator.cu:227-229
        mass = (T)((double)mass * ((double)(r * r) * kPi * (double)density * 0.5));
        if (mass != 0)
            im[i] *= T(1) / mass;
        else
            im[i] = 0;
    }
    std::vector<Q4<T>> qr(nv, Q4<T>{0, 0, 0, 1});
    for (int64_t i = 0; i < nv - 1; i++) qr[i] = normalize4(qmul(qconj(qs[i]), qs[i + 1]));
    std::vector<T> ks(nv, T(100));
    // strand of each vertex
    std::vector<int32_t> strandOf(nv, 0);
    for (int32_t s = 0; s < ns; s++)
        for (int32_t i = sb[s]; i < sb[s + 1]; i++) strandOf[i] = s;
    if (stiffness_mode == 0) {
        const T mmrad = (T)radius * T(1000);
        for (int64_t i = 0; i < nv; i++) {
            T young = (T)strand_young[strandOf[i]];
            T dev = (T)strand_dev[strandOf[i]];
            T len = lr[i];
            T ss = (T)((double)young * kPi * (double)mmrad * (double)mmrad);
            T bt = (T)((double)(ss * dev * mmrad * mmrad) * 0.25 / (double)(len * len));
            ks[i] = ss;
            qr[i] = qscale(bt, qr[i]);
        }
    } else {
        for (int64_t i = 0; i < nv; i++) {
            T kb = (T)k_bend_in * T(4);
            qr[i] = qscale(kb / lr[i], normalize4(qr[i]));
            ks[i] = (T)k_stretch_in * lr[i];
        }
    }
    if (pin_roots)
        for (int32_t s = 0; s < ns; s++) im[sb[s]] = 0;
    for (int64_t i = 0; i < nv; i++) {
        inv_mass[i] = im[i];
        l_rest[i] = lr[i];
        k_stretch[i] = ks[i];
        flags[i] = fl[i];
        st4(q, i, qs[i]);
        st4(q_rest, i, qr[i]);
    }
    return 0;
}

constexpr int kMaxCollisions = 16;  // MAX_COLLISIONS_PER_SEGMENT, YarnBall.h:19

// Kit::segmentClosestPoints (KittenEngine/includes/modules/Common.h:294-312): closest points
// mix(a0, a1, uv.x) and mix(b0, b1, uv.y) of two segments.  glm::mix(x, y, t) = x (1 - t) + y t.
template <typename T>
inline void segClosest(V3<T> a0, V3<T> a1, V3<T> b0, V3<T> b1, T& u, T& w) {
    V3<T> A0 = a1 - a0, A1 = b1 - b0;
    T a = dot(A0, A0), b = dot(A0, A1), c = dot(A1, A1);
    V3<T> diff = b0 - a0;
    T vy = b * dot(A0, diff) - a * dot(A1, diff);
    vy /= a * c - b * b;
    if (!std::isfinite((double)vy)) vy = T(0.5);
    vy = std::min(std::max(vy, T(0)), T(1));
    V3<T> pb = b0 * (T(1) - vy) + b1 * vy;
    T vx = std::min(std::max(dot(pb - a0, A0) / a, T(0)), T(1));
    V3<T> pa = a0 * (T(1) - vx) + a1 * vx;
    vy = std::min(std::max(dot(pa - b0, A1) / c, T(0)), T(1));
    u = vx;
    w = vy;
}

template <typename T>
struct StepCtx {
    const oracle_params* p;
    int64_t nv;
    const T* im;
    const T* lr;
    const T* ks;
    const uint32_t* fl;
    const T* qr;
    const int32_t* local;
    T* x;
    T* v;
    T* vl;
    T* q;
    std::vector<T> y, dx, dxNew, qNew;
    // hair-hair collision state: partner segments of each segment (ascending), their count, the
    // step limit of each segment, and the partner dx snapshot of the current iteration
    std::vector<int32_t> cols, ncols;
    std::vector<T> maxStep, snap;
};

// The collision detection of detectCollisions (YBSimulator.cu:424-456): buildAABBs +
// LBVH query + buildCollisionList (collision.cu:8-92).  The LBVH only proposes pairs whose padded
// AABBs overlap, and every pair that passes the distance test below has overlapping padded
// AABBs, so the result is the set of segment pairs (a, b), |a - b| > 2, with
// |closest(a, b)| < 2 scaledDetectionRadius (+ the velocity radii).  Each pair is tested once,
// with the lower index as segment a; each segment lists its partners in ascending order.  Returns
// 1 when a segment has more than 16 partners (ERROR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED).
template <typename T>
int detectCollisions(StepCtx<T>& c) {
    const oracle_params* p = c.p;
    const T detR = (T)p->radius + T(0.5f) * (T)p->barrier_thickness;  // Sim::uploadMeta, YBSimulator.cu:323-324
    const T scaled = detR * (T)p->detection_scaler;
    const int64_t nv = c.nv;
    c.cols.assign(kMaxCollisions * nv, -1);
    c.ncols.assign(nv, 0);
    std::vector<T> vr(nv, T(0));  // velocity radius of each segment
    if (p->velocity_radius)
        for (int64_t i = 0; i < nv; i++)
            if (c.fl[i] & HAS_NEXT) {
                V3<T> d0 = ld3(c.dx.data(), i), d1 = ld3(c.dx.data(), i + 1);
                vr[i] = std::sqrt(std::max(dot(d0, d0), dot(d1, d1)));
            }
    int overflow = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : overflow)
    for (int64_t i = 0; i < nv; i++) {
        if (!(c.fl[i] & HAS_NEXT)) continue;
        int n = 0;
        for (int64_t j = 0; j < nv; j++) {
            if (j == i || !(c.fl[j] & HAS_NEXT) || std::llabs(j - i) <= 2) continue;
            const int64_t a = std::min(i, j), b = std::max(i, j);
            if (p->connection) {  // glued pairs are exempt (collision.cu:47-48), tested from either segment
                const int32_t* t = p->connection;
                if (t[a] == b || t[a + 1] == b || t[a] == b + 1 || t[a + 1] == b + 1 || t[b] == a || t[b + 1] == a ||
                    t[b] == a + 1 || t[b + 1] == a + 1)
                    continue;
            }
            V3<T> a0 = ld3(c.x, a);
            V3<T> A1 = ld3(c.x, a + 1) - a0, B0 = ld3(c.x, b) - a0, B1 = ld3(c.x, b + 1) - a0;
            T u, w;
            segClosest(v3<T>(0, 0, 0), A1, B0, B1, u, w);
            V3<T> nrm = u * A1 - (B0 * (T(1) - w) + B1 * w);
            T d2 = dot(nrm, nrm);
            T r = T(2) * scaled;
            if (p->velocity_radius) {
                r += vr[a];
                r += vr[b];
            }
            if (d2 < r * r) {
                if (n < kMaxCollisions)
                    c.cols[(int64_t)n * nv + i] = (int32_t)j;
                else
                    overflow = 1;
                n++;
            }
        }
        c.ncols[i] = std::min(n, kMaxCollisions);
    }
    return overflow;
}

// recomputeStepLimitKernel (collision.cu:95-131): the largest move of each segment's first
// vertex for which the detection above still sees every contact.
template <typename T>
void recomputeStepLimit(StepCtx<T>& c) {
    const oracle_params* p = c.p;
    const T detR = (T)p->radius + T(0.5f) * (T)p->barrier_thickness;
    c.maxStep.assign(c.nv, std::numeric_limits<T>::infinity());
    if (!p->step_limit) return;
    const T margin = (T)((1.f - 0.1f) * 0.5f);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c.nv; i++) {
        if (!(c.fl[i] & HAS_NEXT)) continue;
        V3<T> a0 = ld3(c.x, i);
        V3<T> A1 = ld3(c.x, i + 1) - a0;
        T minDist = detR * ((T)p->detection_scaler - T(1));
        if (p->velocity_radius) minDist += length(ld3(c.dx.data(), i));
        for (int k = 0; k < c.ncols[i]; k++) {
            int64_t o = c.cols[(int64_t)k * c.nv + i];
            V3<T> B0 = ld3(c.x, o) - a0, B1 = ld3(c.x, o + 1) - a0;
            T u, w;
            segClosest(v3<T>(0, 0, 0), A1, B0, B1, u, w);
            T l = length(u * A1 - (B0 * (T(1) - w) + B1 * w));
            minDist = std::min(minDist, margin * l);
        }
        c.maxStep[i] = minDist;
    }
}

// The IPC barrier + friction energy of one contact of segment s = (v0, v1) with partner segment
// (b0, b1), cosserat.cu:163-227, added to the force / Hessian of v0 (own = true, weight 1 - t) or
// of v1 (own = false, weight t).  x0/x1 and d0/d1 are the segment's positions and current dx; the
// partner's dx come from the iteration's snapshot.
template <typename T>
void contactTerm(const StepCtx<T>& c, V3<T> x0, V3<T> x1, V3<T> d0, V3<T> d1, int64_t o, bool own, T damping,
                 V3<T>& f, T H[6]) {
    const oracle_params* p = c.p;
    const T invb = T(1) / (T)p->barrier_thickness;
    const T radius = T(2) * (T)p->radius;
    const T kCol = (T)p->k_collision * invb;
    V3<T> b0 = ld3(c.x, o), b1 = ld3(c.x, o + 1);
    V3<T> db0 = ld3(c.snap.data(), o), db1 = ld3(c.snap.data(), o + 1);
    T u, w;
    segClosest(v3<T>(0, 0, 0), (x1 - x0) + (d1 - d0), (b0 - x0) + (db0 - d0), (b1 - x0) + (db1 - d0), u, w);
    V3<T> dpos = (x0 * (T(1) - u) + x1 * u) - (b0 * (T(1) - w) + b1 * w);
    V3<T> ddpos = (d0 * (T(1) - u) + d1 * u) - (db0 * (T(1) - w) + db1 * w);
    V3<T> nrm = dpos + ddpos;
    T d = length(nrm);
    nrm = nrm * (T(1) / d);
    const T wt = own ? T(1) - u : u;
    d = d - radius;
    d *= invb;
    if (d > 1) return;
    d = std::max(d, T(1e-3f));
    T invd = T(1) / d;
    T logd = std::log(d);
    T dH = (T(-3) + (T(2) + invd) * invd - T(2) * logd) * kCol * invb;
    T ff = -(T(1) - d) * (d - T(1) + T(2) * d * logd) * invd * kCol;
    V3<T> mydx = own ? d0 : d1;
    f = f + (ff * wt - damping * dH * wt * wt * dot(nrm, mydx)) * nrm;
    dH *= T(1) + damping;
    T op[6] = {nrm.x * nrm.x, nrm.y * nrm.y, nrm.z * nrm.z, nrm.x * nrm.y, nrm.x * nrm.z, nrm.y * nrm.z};
    for (int k = 0; k < 6; k++) H[k] += op[k] * (dH * wt * wt);
    V3<T> uu = ddpos - dot(nrm, ddpos) * nrm;
    T ul = length(uu);
    if (ul > 0) {
        T f1 = std::min((T)p->k_friction, (T)p->friction_coeff * ff / ul);
        op[0] -= 1;
        op[1] -= 1;
        op[2] -= 1;
        f = f - (f1 * wt) * uu;
        for (int k = 0; k < 6; k++) H[k] -= op[k] * (wt * wt * f1);
    }
}

// initItr, YarnBall/sim/iteration.cu:8-59.  y - x is kept in ctx.y (the reference keeps it in d_vels).
template <typename T>
void predict(StepCtx<T>& c, T h, T lastH, T time) {
    const oracle_params* p = c.p;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c.nv; i++) {
        V3<T> g = v3<T>(p->gravity[0], p->gravity[1], p->gravity[2]);
        V3<T> vel = ld3(c.v, i);
        T windx = 0;
        if (p->wind_peak != 0) {
            T ypos = c.x[3 * i + 1], zpos = c.x[3 * i + 2];
            T wy = ypos > 0 ? (T)std::cos(2 * M_PI * (double)((T)p->wind_y_freq * ypos + (T)p->wind_time_freq * time)) : T(0);
            T wz = (T)std::cos(2 * M_PI * (double)((T)p->wind_z_freq * std::abs(zpos) + (T)p->wind_time_freq * time));
            T prod = wy * wz;
            T sg = prod > 0 ? T(1) : (prod < 0 ? T(-1) : T(0));
            T pw = std::pow(prod, (T)p->wind_sharpness) * sg;
            windx = (T)p->wind_peak * ((T(0) < pw) ? pw : T(0));
        }
        V3<T> ext = (g + v3<T>(windx, 0, 0)) * (T)p->ext_mult;
        V3<T> dx = h * vel;
        V3<T> lastVel = ld3(c.vl, i);
        st3(c.vl, i, vel);
        V3<T> y = vel;  // roots keep the velocity in d_vels
        if (c.im[i] != 0) {
            y = dx + (h * h) * ext;
            T ext2 = dot(ext, ext);
            if (ext2 > 0) {
                V3<T> a = (vel - lastVel) / lastH;
                T s = dot(a, ext) / ext2;
                s = s < 0 ? T(0) : (s > 1 ? T(1) : s);
                dx = dx + (h * h * s) * ext;
            }
        }
        st3(c.y.data(), i, y);
        st3(c.dx.data(), i, dx);
    }
}

// cosseratItr, YarnBall/sim/cosserat.cu:112-161 and :246-285, for one vertex i.  With hair-hair
// collision on, each segment adds its contacts' barrier and friction terms (:163-227) and the move
// is clamped to the step limit of the vertex's segments (:157, :270, :281-282).  dxr is the dx
// array the vertex reads.  Returns the new dx_i (or the old one when the vertex is pinned).
template <typename T>
V3<T> positionUpdate(const StepCtx<T>& c, const T* dxr, int64_t i, T h) {
    const T damping = (T)c.p->damping / h;
    const bool coll = c.p->hair_hair != 0;
    V3<T> vi_dx = ld3(dxr, i);
    if (c.im[i] == 0) return vi_dx;
    T H[6];
    T inert = T(1) / (c.im[i] * h * h);
    for (int k = 0; k < 6; k++) H[k] = inert;  // hess3(float) fills all six entries (SymMat.h:16-18)
    V3<T> f = (T(1) / (h * h * c.im[i])) * (ld3(c.y.data(), i) - vi_dx);
    if (c.p->connection && c.p->connection[i] >= 0) {
        // the connection spring (cosserat.cu:123-131) to the partner's position at the start of the
        // step (x does not move within it) and its dx at the start of the iteration (the snapshot)
        const int64_t j = c.p->connection[i];
        const T stiffness = T(4e1);
        f = f - stiffness * ((ld3(c.x, i) - ld3(c.x, j)) + (vi_dx - ld3(c.snap.data(), j)) + damping * vi_dx);
        const T d = stiffness * (1 + damping);
        H[0] += d;
        H[1] += d;
        H[2] += d;
    }
    T stepLimit = std::numeric_limits<T>::infinity();
    if (c.fl[i] & HAS_NEXT) {  // segment i, as thread i computes it (:141-161)
        V3<T> xi = ld3(c.x, i), xj = ld3(c.x, i + 1), vj_dx = ld3(dxr, i + 1);
        T invl = T(1) / c.lr[i];
        V3<T> cc = ((xj - xi) + (vj_dx - vi_dx)) * invl - qrotate(ld4(c.q, i), v3<T>(1, 0, 0));
        T k = c.ks[i] * invl;
        T d = k * invl;
        f = f + (k * cc - (damping * d) * vi_dx);
        d *= 1 + damping;
        H[0] += d;
        H[1] += d;
        H[2] += d;
        if (coll) {
            stepLimit = c.maxStep[i];
            for (int n = 0; n < c.ncols[i]; n++)
                contactTerm(c, xi, xj, vi_dx, vj_dx, c.cols[(int64_t)n * c.nv + i], true, damping, f, H);
        }
    }
    if (c.fl[i] & HAS_PREV) {  // segment i-1, as thread i-1 computes f2/H2 and passes it on (:157, :269-274)
        int64_t j = i - 1;
        V3<T> xj = ld3(c.x, j), xi = ld3(c.x, i), dj = ld3(dxr, j);
        T invl = T(1) / c.lr[j];
        V3<T> cc = ((xi - xj) + (vi_dx - dj)) * invl - qrotate(ld4(c.q, j), v3<T>(1, 0, 0));
        T k = c.ks[j] * invl;
        T d = k * invl;
        V3<T> f2 = -k * cc - (damping * d) * vi_dx;
        d *= 1 + damping;
        T H2[6] = {d, d, d, 0, 0, 0};
        if (coll) {
            for (int n = 0; n < c.ncols[j]; n++)
                contactTerm(c, xj, xi, dj, vi_dx, c.cols[(int64_t)n * c.nv + j], false, damping, f2, H2);
            stepLimit = std::min(stepLimit, c.maxStep[j]);
        }
        f = f + f2;
        for (int n = 0; n < 6; n++) H[n] += H2[n];
    }
    V3<T> delta = (T)c.p->acceleration_ratio * solveHess3(H, f);
    V3<T> out = vi_dx + delta;
    if (coll) {
        T l = length(out);
        if (l > stepLimit && l > 0) out = out * (stepLimit / l);
    }
    return out;
}

// quaternionLambdaItr, YarnBall/sim/cosserat.cu:290-337, for one segment i.  qr_ is the q array
// it reads.  Returns the new q_i (or the old one when the segment is not updated).
template <typename T>
Q4<T> quaternionUpdate(const StepCtx<T>& c, const T* qread, int64_t i) {
    Q4<T> vi_q = ld4(qread, i);
    uint32_t fl = c.fl[i];
    if (!(!(fl & FIX_ORIENTATION) && (fl & HAS_NEXT))) return vi_q;
    V3<T> vi_dx = ld3(c.dx.data(), i);
    V3<T> vj_pos = ld3(c.x, i + 1);
    V3<T> vj_dx = ld3(c.dx.data(), i + 1);
    V3<T> vp = ((vj_pos - ld3(c.x, i)) + (vj_dx - vi_dx)) / c.lr[i];
    vp = vp * (T(-2) * c.ks[i]);
    Q4<T> b = {0, 0, 0, 0};
    if (fl & HAS_PREV) {
        Q4<T> qRest = ld4(c.qr, i - 1);
        Q4<T> vj_q = ld4(qread, i - 1);
        T phi = dot4(qmul(qconj(vj_q), vi_q), qRest) > 0 ? T(1) : T(-1);
        b = qadd(b, qscale(phi, qmul(vj_q, qRest)));
    }
    if (fl & HAS_NEXT_ORIENTATION) {
        Q4<T> qRest = ld4(c.qr, i);
        Q4<T> vj_q = ld4(qread, i + 1);
        T phi = dot4(qmul(qconj(vi_q), vj_q), qRest) > 0 ? T(1) : T(-1);
        b = qadd(b, qscale(phi, qmul(vj_q, qconj(qRest))));
    }
    T lambda = length(vp) + length4(b);
    Q4<T> V = {vp.x, vp.y, vp.z, 0};
    Q4<T> E = {1, 0, 0, 0};
    Q4<T> r = qadd(qmul(qmul(V, b), E), qscale(lambda, b));
    return normalize4(r);
}

// endItr, YarnBall/sim/iteration.cu:62-74.
template <typename T>
void finish(StepCtx<T>& c, T h) {
    const T invH = T(1) / h;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c.nv; i++) {
        V3<T> dx = ld3(c.dx.data(), i);
        if (c.im[i] != 0) st3(c.v, i, dx * invH * (T(1) - (T)c.p->velocity_decay * h));
        st3(c.x, i, ld3(c.x, i) + dx);
    }
}

// SDFHeadCollision + TriInterpSDF + index helpers, SDFCollisionSolver/cudaSDFCollision.cu:88-155 and
// :205-268; grid spacing from SDFBodyCollisionSolver::InitParams (SDFBodyCollisionSolver.cpp:46-82).
template <typename T>
void sdfProject(StepCtx<T>& c) {
    const oracle_params* p = c.p;
    const int nx = p->sdf_dims[0], ny = p->sdf_dims[1], nz = p->sdf_dims[2];
    T ds[3], invDs[3];
    for (int a = 0; a < 3; a++) {
        ds[a] = ((T)p->sdf_max[a] - (T)p->sdf_min[a]) / ((T)1 * (T)p->sdf_dims[a]);
        invDs[a] = T(1) / ds[a];
    }
    const Q4<T> invq = {-(T)p->body_rot[0], -(T)p->body_rot[1], -(T)p->body_rot[2], (T)p->body_rot[3]};
    const V3<T> tr = v3<T>(p->body_trans[0], p->body_trans[1], p->body_trans[2]);
    const V3<T> gmin = v3<T>(p->sdf_min[0], p->sdf_min[1], p->sdf_min[2]);
    const T thresh = (T)p->sdf_threshold;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c.nv; i++) {
        if (c.local[i] == 0) continue;  // strand root
        V3<T> pos = ld3(c.x, i);
        V3<T> lp = qrotate(invq, pos - tr) - gmin;
        int idx[3];
        T lpa[3] = {lp.x, lp.y, lp.z};
        for (int a = 0; a < 3; a++) idx[a] = (int)((double)(lpa[a] * invDs[a]) + 0.5);
        if (idx[0] < 0 || idx[0] >= nx || idx[1] < 0 || idx[1] >= ny || idx[2] < 0 || idx[2] >= nz) continue;
        T corner[2][2][2][4];
        for (int dz = 0; dz < 2; dz++)
            for (int dy = 0; dy < 2; dy++)
                for (int dx = 0; dx < 2; dx++) {
                    int cx = idx[0] + dx, cy = idx[1] + dy, cz = idx[2] + dz;
                    bool inside = cx >= 0 && cx < nx && cy >= 0 && cy < ny && cz >= 0 && cz < nz;
                    int qx = std::max(0, std::min(cx, nx - 1)), qy = std::max(0, std::min(cy, ny - 1)),
                        qz = std::max(0, std::min(cz, nz - 1));
                    int64_t li = (int64_t)qx + (int64_t)qy * nx + (int64_t)qz * nx * ny;
                    int64_t gi = (int64_t)cx + (int64_t)cy * nx + (int64_t)cz * nx * ny;
                    for (int a = 0; a < 3; a++) corner[dz][dy][dx][a] = inside ? (T)p->sdf_grad[3 * gi + a] : T(0);
                    corner[dz][dy][dx][3] = (T)p->sdf_phi[li];
                }
        T ud[3];
        for (int a = 0; a < 3; a++) ud[a] = (T)((double)invDs[a] * ((double)lpa[a] - ((double)idx[a] - 0.5) * (double)ds[a]));
        T res[4];
        for (int k = 0; k < 4; k++) {
            T c00 = corner[0][0][0][k] * (T(1) - ud[0]) + corner[0][0][1][k] * ud[0];
            T c01 = corner[1][0][0][k] * (T(1) - ud[0]) + corner[1][0][1][k] * ud[0];
            T c10 = corner[0][1][0][k] * (T(1) - ud[0]) + corner[0][1][1][k] * ud[0];
            T c11 = corner[1][1][0][k] * (T(1) - ud[0]) + corner[1][1][1][k] * ud[0];
            T c0 = c00 * (T(1) - ud[1]) + c10 * ud[1];
            T c1 = c01 * (T(1) - ud[1]) + c11 * ud[1];
            res[k] = c0 * (T(1) - ud[2]) + c1 * ud[2];
        }
        V3<T> n = normalize3(v3<T>(res[0], res[1], res[2]));
        T phi = res[3] - thresh;
        if (phi < 0) {
            st3(c.x, i, pos - phi * n);
            V3<T> vel = ld3(c.v, i);
            T vl = length(vel);
            if (vl >= T(1e-6)) {
                V3<T> vn = vel / vl;
                st3(c.v, i, vel - dot(vn, n) * n);
            }
        }
    }
}

// Sim::advance (YarnBall/sim/step.cpp:38-62) followed by the SDF pass that
// StableCosseratRodsSolver::SolveNextStep runs after it (StableCosseratRodsSolver.cpp:216-234).
// clock = {meta.h, meta.lastH, meta.time}; updated in place.
template <typename T>
int advanceT(const oracle_params* p, int64_t nv, int32_t ns, const int32_t* sb, const T* im, const T* lr,
             const T* ks, const uint32_t* fl, const T* qr, T* x, T* v, T* vl, T* q, double* clock, float dt) {
#ifdef _OPENMP
    if (p->num_threads > 0) omp_set_num_threads(p->num_threads);
#endif
    if (dt <= 0) return 0;
    Topology<T> topo(nv, ns, sb);
    int steps = std::max(1, (int)std::ceil(dt / p->max_h));
    T lastH = (T)clock[0];
    T h = (T)(dt / (float)steps);
    if (sizeof(T) == 8) h = (T)((double)dt / (double)steps);
    T time = (T)clock[2];
    StepCtx<T> c;
    c.p = p;
    c.nv = nv;
    c.im = im;
    c.lr = lr;
    c.ks = ks;
    c.fl = fl;
    c.qr = qr;
    c.local = topo.local.data();
    c.x = x;
    c.v = v;
    c.vl = vl;
    c.q = q;
    c.y.assign(3 * nv, T(0));
    c.dx.assign(3 * nv, T(0));
    c.dxNew.assign(3 * nv, T(0));
    c.qNew.assign(4 * nv, T(0));
    int64_t counter = (int64_t)clock[3];
    int rc = 0;
    if (p->hair_hair) {
        c.cols.assign(kMaxCollisions * nv, -1);
        c.ncols.assign(nv, 0);
    }
    for (int s = 0; s < steps; s++, counter++) {
        predict(c, h, lastH, time);
        if (p->hair_hair) {
            // Sim::advance: detection every detectionPeriod substeps (step.cpp:53), then the graph's
            // recomputeStepLimit (step.cpp:19)
            if (p->detection_period > 0 && counter % p->detection_period == 0) rc |= detectCollisions(c);
            recomputeStepLimit(c);
        }
        for (int it = 0; it < p->num_itr; it++) {
            if (p->hair_hair || p->connection) c.snap = c.dx;  // partner dx of this iteration (both schedules)
            if (p->schedule == 1) {
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < nv; i++) st3(c.dxNew.data(), i, positionUpdate(c, c.dx.data(), i, h));
                std::swap(c.dx, c.dxNew);
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < nv; i++) st4(c.qNew.data(), i, quaternionUpdate(c, c.q, i));
                std::memcpy(c.q, c.qNew.data(), sizeof(T) * 4 * nv);
            } else {
                for (int colour = 0; colour < 2; colour++) {
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < nv; i++)
                        if ((topo.local[i] & 1) == colour) st3(c.dx.data(), i, positionUpdate(c, c.dx.data(), i, h));
                }
                for (int colour = 0; colour < 2; colour++) {
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < nv; i++)
                        if ((topo.local[i] & 1) == colour) st4(c.q, i, quaternionUpdate(c, c.q, i));
                }
            }
        }
        finish(c, h);
    }
    if (p->sdf_enabled) sdfProject(c);
    clock[0] = (double)h;
    clock[1] = (double)lastH;
    clock[2] = (double)((T)clock[2] + (T)dt);
    clock[3] = (double)counter;
    return rc ? 4 : 0;
}

}  // namespace

extern "C" {

int oracle_configure_f32(int64_t nv, int32_t ns, const int32_t* sb, const float* pos, float radius, float density,
                         int32_t stiffness_mode, const float* strand_young, const float* strand_dev, float k_stretch,
                         float k_bend, int32_t pin_roots, float* inv_mass, float* l_rest, float* k_stretch_out,
                         uint32_t* flags, float* q, float* q_rest) {
    return configureT<float>(nv, ns, sb, pos, radius, density, stiffness_mode, strand_young, strand_dev, k_stretch,
                             k_bend, pin_roots, inv_mass, l_rest, k_stretch_out, flags, q, q_rest);
}

int oracle_configure_f64(int64_t nv, int32_t ns, const int32_t* sb, const float* pos, float radius, float density,
                         int32_t stiffness_mode, const float* strand_young, const float* strand_dev, float k_stretch,
                         float k_bend, int32_t pin_roots, double* inv_mass, double* l_rest, double* k_stretch_out,
                         uint32_t* flags, double* q, double* q_rest) {
    return configureT<double>(nv, ns, sb, pos, radius, density, stiffness_mode, strand_young, strand_dev, k_stretch,
                              k_bend, pin_roots, inv_mass, l_rest, k_stretch_out, flags, q, q_rest);
}

int oracle_advance_f32(const oracle_params* p, int64_t nv, int32_t ns, const int32_t* sb, const float* im,
                       const float* lr, const float* ks, const uint32_t* fl, const float* qr, float* x, float* v,
                       float* vl, float* q, double* clock, float dt) {
    return advanceT<float>(p, nv, ns, sb, im, lr, ks, fl, qr, x, v, vl, q, clock, dt);
}

int oracle_advance_f64(const oracle_params* p, int64_t nv, int32_t ns, const int32_t* sb, const double* im,
                       const double* lr, const double* ks, const uint32_t* fl, const double* qr, double* x, double* v,
                       double* vl, double* q, double* clock, float dt) {
    return advanceT<double>(p, nv, ns, sb, im, lr, ks, fl, qr, x, v, vl, q, clock, dt);
}

// Body SDF bake, FP64, by brute force over the triangles: the grid PNMesh::StoreSDFQueries fills
// (PNMesh.cpp:109-173) from the exact signed distance that Discregrid::TriangleMeshDistance gives
// (extern/Discregrid/geometry/TriangleMeshDistance.h:280-318) rather than from its cubic Lagrange
// resampling.  Closest point on a triangle with its Voronoi feature: Ericson, Real-Time Collision
// Detection (2005), 5.1.5.  Sign: the angle-weighted pseudonormal of that feature (Baerentzen and
// Aanaes, IEEE TVCG 11(3), 2005).  grad: inside (distance < 0), the unit gradient of the distance;
// otherwise the unit direction from the grid centre, as StoreSDFQueries sets it (zero at the centre
// node, where the reference divides 0 by 0).
int oracle_sdf_bake_f64(int32_t nv, const float* verts, int32_t nt, const int32_t* tris, const int32_t* dims,
                        const float* gmin, const float* gmax, double* phi, double* grad) {
    typedef V3<double> D3;
    auto vert = [&](int32_t i) { return v3<double>(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); };
    std::vector<D3> fn(nt), vn(nv, v3<double>(0, 0, 0));
    std::vector<std::array<D3, 3>> en(nt);
    std::map<std::pair<int32_t, int32_t>, D3> edge_sum;
    for (int32_t t = 0; t < nt; t++) {
        const int32_t* T = tris + 3 * t;
        D3 a = vert(T[0]), b = vert(T[1]), c = vert(T[2]);
        D3 n = cross(b - a, c - a);
        n = n / length(n);
        fn[t] = n;
        D3 p[3] = {a, b, c};
        for (int k = 0; k < 3; k++) {
            D3 e1 = p[(k + 1) % 3] - p[k], e2 = p[(k + 2) % 3] - p[k];
            double ang = std::acos(std::max(-1.0, std::min(1.0, dot(e1, e2) / (length(e1) * length(e2)))));
            vn[T[k]] = vn[T[k]] + ang * n;
            int32_t i0 = T[k], i1 = T[(k + 1) % 3];
            auto key = std::make_pair(std::min(i0, i1), std::max(i0, i1));
            auto it = edge_sum.find(key);
            if (it == edge_sum.end()) edge_sum[key] = n; else it->second = it->second + n;
        }
    }
    for (auto& n : vn) { double l = length(n); if (l > 0) n = n / l; }
    for (int32_t t = 0; t < nt; t++)
        for (int k = 0; k < 3; k++) {  // edge k joins corners k and k+1
            int32_t i0 = tris[3 * t + k], i1 = tris[3 * t + (k + 1) % 3];
            D3 e = edge_sum[std::make_pair(std::min(i0, i1), std::max(i0, i1))];
            en[t][k] = e / length(e);
        }
    const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
    D3 lo = v3<double>(gmin[0], gmin[1], gmin[2]);
    D3 ds = v3<double>(((double)gmax[0] - gmin[0]) / nx, ((double)gmax[1] - gmin[1]) / ny, ((double)gmax[2] - gmin[2]) / nz);
    D3 centre = v3<double>(0.5 * ((double)gmax[0] + gmin[0]), 0.5 * ((double)gmax[1] + gmin[1]), 0.5 * ((double)gmax[2] + gmin[2]));
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t node = 0; node < nx * ny * nz; node++) {
        const int64_t i = node % nx, j = (node / nx) % ny, k = node / (nx * ny);
        D3 x = v3<double>(lo.x + ds.x * i, lo.y + ds.y * j, lo.z + ds.z * k);
        double best = std::numeric_limits<double>::infinity();
        D3 bcp = x;
        int32_t bt = -1, bf = 0;
        for (int32_t t = 0; t < nt; t++) {
            const int32_t* T = tris + 3 * t;
            D3 a = vert(T[0]), b = vert(T[1]), c = vert(T[2]);
            D3 ab = b - a, ac = c - a, ap = x - a;
            double d1 = dot(ab, ap), d2 = dot(ac, ap);
            D3 cp;
            int f;  // 0,1,2 vertices; 3 edge ab, 4 edge bc, 5 edge ca; 6 face
            if (d1 <= 0 && d2 <= 0) { cp = a; f = 0; }
            else {
                D3 bp = x - b;
                double d3 = dot(ab, bp), d4 = dot(ac, bp);
                if (d3 >= 0 && d4 <= d3) { cp = b; f = 1; }
                else {
                    double vc = d1 * d4 - d3 * d2;
                    if (vc <= 0 && d1 >= 0 && d3 <= 0) { double v = d1 / (d1 - d3); cp = a + v * ab; f = 3; }
                    else {
                        D3 cpp = x - c;
                        double d5 = dot(ab, cpp), d6 = dot(ac, cpp);
                        if (d6 >= 0 && d5 <= d6) { cp = c; f = 2; }
                        else {
                            double vb = d5 * d2 - d1 * d6;
                            if (vb <= 0 && d2 >= 0 && d6 <= 0) { double w = d2 / (d2 - d6); cp = a + w * ac; f = 5; }
                            else {
                                double va = d3 * d6 - d5 * d4;
                                if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
                                    double w = (d4 - d3) / ((d4 - d3) + (d5 - d6)); cp = b + w * (c - b); f = 4;
                                } else {
                                    double den = 1.0 / (va + vb + vc);
                                    double v = vb * den, w = vc * den;
                                    cp = a + v * ab + w * ac; f = 6;
                                }
                            }
                        }
                    }
                }
            }
            D3 dd = x - cp;
            double q = dot(dd, dd);
            if (q < best) { best = q; bt = t; bf = f; bcp = cp; }
        }
        double dist = std::sqrt(best);
        D3 pn;
        if (bf < 3) pn = vn[tris[3 * bt + bf]];
        else if (bf == 3) pn = en[bt][0];
        else if (bf == 4) pn = en[bt][1];
        else if (bf == 5) pn = en[bt][2];
        else pn = fn[bt];
        D3 u = x - bcp;
        double sgn = dot(u, pn) >= 0 ? 1.0 : -1.0;
        phi[node] = sgn * dist;
        D3 g;
        if (sgn * dist < 0) g = (bcp - x) / dist;
        else {  // radial; the grid centre itself (0/0 there) gets a zero gradient
            D3 r = x - centre;
            double l = length(r);
            g = l > 0 ? r / l : v3<double>(0, 0, 0);
        }
        grad[3 * node] = g.x;
        grad[3 * node + 1] = g.y;
        grad[3 * node + 2] = g.z;
    }
    return 0;
}

// Signed distance (as oracle_sdf_bake_f64 computes it) at np arbitrary points: a bake on a
// 1 x 1 x 1 grid per point.
int oracle_sdf_points_f64(int32_t nv, const float* verts, int32_t nt, const int32_t* tris, int64_t np, const double* pts,
                          double* dist) {
    const int32_t one[3] = {1, 1, 1};
    for (int64_t i = 0; i < np; i++) {
        const float lo[3] = {(float)pts[3 * i], (float)pts[3 * i + 1], (float)pts[3 * i + 2]};
        const float hi[3] = {lo[0] + 1.f, lo[1] + 1.f, lo[2] + 1.f};
        double g[3];
        oracle_sdf_bake_f64(nv, verts, nt, tris, one, lo, hi, &dist[i], g);
    }
    return 0;
}

// Sim::SagFree / SingleSagFree (YarnBall/YBSimulator.cu:480-674), strand by strand with the
// reference's float / double mix.  Part 1, tip to root: each segment's rest length becomes the
// root of the quadratic that cancels the stretch force of the mass below it (the root nearer the
// old length; 1.5 x when there is none; clamped to [1e-6, 1.5 x]).  Part 2, root to tip: each
// segment's orientation turns in the plane of its axis and the bending force towards the angle
// whose bending torque cancels the force's torque, bracketed within 1e-4 rad of the force's
// direction; the rotations accumulate towards the tip, and the rest Darboux of the previous
// segment is re-aimed keeping its magnitude (the bend/twist stiffness).  Positions do not change.
namespace {
const double kSagPi = 3.141592653589793238462643;
const double kSag2Pi = 6.2831853071795864769252867665590057683943;
const double kSagPi2 = 1.5707963267948966192313216916397;

double sag_fmod(double x, double y) {  // my_fmod, YBSimulator.cu:59-72
    long double lx = x, ly = y;
    return ly != 0 ? (double)(lx - (long long int)(lx / ly) * ly) : 0.0;
}
double fit_angle(double a) { return sag_fmod(sag_fmod(a + kSagPi, kSag2Pi) + kSag2Pi, kSag2Pi) - kSagPi; }
double sgn(double x) { return (double)((0.0 < x) - (x < 0.0)); }

struct F3 {
    float x, y, z;
};
inline F3 f3m(float a, F3 v) { return {a * v.x, a * v.y, a * v.z}; }
inline F3 f3a(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 f3s(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float f3d(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 f3c(F3 a, F3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline F3 f3n(F3 a) { return f3m(1.f / std::sqrt(f3d(a, a)), a); }  // glm::normalize (v * inversesqrt(dot))
struct FQ {
    F3 q;
    float w;
};
inline FQ fqmul(FQ l, FQ r) {  // Rotor operator*, Rotor.h:210-212
    return {f3a(f3a(f3m(l.w, r.q), f3m(r.w, l.q)), f3c(l.q, r.q)), l.w * r.w - f3d(l.q, r.q)};
}
inline F3 fqrot(FQ r, F3 v) {  // Rotor::rotate, Rotor.h:114-123
    F3 a = f3a(f3m(r.w, v), f3c(r.q, v));
    float c = f3d(v, r.q);
    return f3a(f3a(f3m(r.w, a), f3c(r.q, a)), f3m(c, r.q));
}
inline F3 fqd3(FQ r) { return f3n(fqrot(r, F3{1.f, 0.f, 0.f})); }  // getD3, Rotor.h:206
}  // namespace

int oracle_sag_free_f32(int32_t ns, const int32_t* sb, const float* pos, const float* gravity, const float* inv_mass,
                        const float* k_stretch, float* l_rest, float* q, float* q_rest, int32_t iterations) {
    const F3 g = {gravity[0], gravity[1], gravity[2]};
    for (int32_t it = 0; it < iterations; it++) {
#pragma omp parallel for schedule(dynamic, 16)
        for (int32_t s = 0; s < ns; s++) {
            const int rootv = sb[s], nextv = sb[s + 1];
            const float eps = 1e-6f;
            auto Q = [&](int i) { return FQ{{q[4 * i], q[4 * i + 1], q[4 * i + 2]}, q[4 * i + 3]}; };
            std::vector<F3> f_srs(nextv - rootv, F3{0.f, 0.f, 0.f});
            // 1. rest lengths, tip to root
            float totalMassFromTip = 1 / inv_mass[nextv - 1];
            for (int v = 0; rootv + v < nextv - 1; ++v) {
                const int vId = nextv - 2 - v;
                const F3 axis = fqd3(Q(vId));
                const float kS = k_stretch[vId];
                const float oldRestLen = l_rest[vId];
                if (inv_mass[vId])
                    totalMassFromTip += 0.5 / inv_mass[vId];
                else
                    totalMassFromTip += 0.5 * (l_rest[vId] / l_rest[vId + 1]) / inv_mass[vId + 1];
                double f_s_g = f3d(axis, g) * totalMassFromTip;
                double f_s = -f_s_g;
                if (f_s == 0) {
                    l_rest[vId] = oldRestLen;
                } else if (1 - 4 * f_s * oldRestLen / kS < 0) {
                    l_rest[vId] = 1.5f * oldRestLen;
                } else {
                    double fsk = f_s / kS;
                    double fskinv = kS / f_s;
                    double ans1 = (1 + std::sqrt(1 - 4 * oldRestLen * fsk)) * 0.5f * fskinv;
                    double ans2 = (1 - std::sqrt(1 - 4 * oldRestLen * fsk)) * 0.5f * fskinv;
                    l_rest[vId] = std::abs(oldRestLen - ans1) >= std::abs(oldRestLen - ans2) ? ans2 : ans1;
                }
                l_rest[vId] = std::min(std::max(l_rest[vId], eps), 1.5f * oldRestLen);
                if (rootv + v < nextv - 2) f_srs[vId - rootv - 1] = f3m((float)-f_s, axis);
                totalMassFromTip += 0.5 / inv_mass[vId];
            }
            // 2. rest angles, root to tip
            const float nearestAngle = 1e-4f;
            float totalMassToTip = 0;
            for (int v = 1; rootv + v < nextv; ++v) {
                if (inv_mass[rootv + v])
                    totalMassToTip += 1 / inv_mass[rootv + v];
                else
                    totalMassToTip += (l_rest[rootv + v] / l_rest[rootv + v - 1]) / inv_mass[rootv + v - 1];
            }
            FQ accumQ = {{0.f, 0.f, 0.f}, 1.f};
            for (int v = 1; rootv + v < nextv - 1; ++v) {
                const int vId = rootv + v;
                const FQ cQk = fqmul(accumQ, Q(vId));
                if (inv_mass[vId])
                    totalMassToTip -= 0.5 / inv_mass[vId];
                else
                    totalMassToTip -= 0.5 * (l_rest[vId] / l_rest[vId + 1]) / inv_mass[vId + 1];
                const F3 axisk = fqd3(cQk);
                const F3 f_b = f3a(f_srs[v], f3m(totalMassToTip, g));
                if (f3d(f_b, axisk) < 1 - nearestAngle) {
                    const float* qr = q_rest + 4 * vId;
                    const float kBend = std::sqrt(qr[0] * qr[0] + qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
                    const F3 planeNormal = f3n(f3c(axisk, f_b));
                    const F3 torqueDir = f3c(planeNormal, axisk);
                    const F3 seg = f3s(F3{pos[3 * vId + 3], pos[3 * vId + 4], pos[3 * vId + 5]},
                                       F3{pos[3 * vId], pos[3 * vId + 1], pos[3 * vId + 2]});
                    const float torque = f3d(torqueDir, f_b) * std::sqrt(f3d(seg, seg));
                    const float T = torque / kBend;
                    const float lfb = std::sqrt(f3d(f_b, f_b));  // f_b / glm::length(f_b) in float, then dvec3
                    const double fbn[3] = {(double)(f_b.x / lfb), (double)(f_b.y / lfb), (double)(f_b.z / lfb)};
                    const double cosm = -((double)axisk.x * fbn[0] + (double)axisk.y * fbn[1] + (double)axisk.z * fbn[2]);
                    const double maxrad = std::acos(cosm);
                    const double maxTheta1 = fit_angle(maxrad + nearestAngle), maxTheta2 = fit_angle(maxrad - nearestAngle);
                    const double maxTheta = std::abs(maxTheta1) >= std::abs(maxTheta2) ? maxTheta2 : maxTheta1;
                    const float left = maxTheta >= 0 ? 0 : (float)maxTheta;
                    const float right = maxTheta >= 0 ? (float)maxTheta : 0;
                    double resTheta = 0;
                    if (std::abs(T) > 2) {
                        resTheta = maxTheta;
                    } else {
                        double theta1 = fit_angle(2 * std::acos(1 - (0.5 * T * T)));
                        double theta2 = fit_angle(2 * std::acos(-1 + (0.5 * T * T)));
                        double cT1 = -sgn(maxTheta) * 100, cT2 = -sgn(maxTheta) * 100;
                        if (std::abs(theta1) <= kSagPi2) cT1 = theta1;
                        if (std::abs(theta2) > kSagPi2) cT2 = theta2;
                        if (sgn(cT1) == sgn(maxTheta) && sgn(cT2) == sgn(maxTheta))
                            resTheta = std::min(cT1, cT2);
                        else {
                            if (sgn(cT1) == sgn(maxTheta)) resTheta = cT1;
                            if (sgn(cT2) == sgn(maxTheta)) resTheta = cT2;
                        }
                    }
                    resTheta = std::min(std::max(resTheta, (double)left), (double)right);
                    float half = (float)resTheta;  // Rotor::angleAxis(float rad, axis), Rotor.h:51-54
                    half *= 0.5f;
                    const FQ qTheta = {f3m(std::sin(half), planeNormal), std::cos(half)};
                    accumQ = fqmul(accumQ, qTheta);
                    const FQ nq = fqmul(accumQ, Q(vId));
                    q[4 * vId] = nq.q.x;
                    q[4 * vId + 1] = nq.q.y;
                    q[4 * vId + 2] = nq.q.z;
                    q[4 * vId + 3] = nq.w;
                    const FQ pq = Q(vId - 1);
                    const FQ d = fqmul(FQ{f3m(-1.f, pq.q), pq.w}, nq);
                    float* pr = q_rest + 4 * (vId - 1);
                    const float len = std::sqrt(pr[0] * pr[0] + pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
                    const float dl = 1.f / std::sqrt(d.q.x * d.q.x + d.q.y * d.q.y + d.q.z * d.q.z + d.w * d.w);
                    pr[0] = d.q.x * dl * len;
                    pr[1] = d.q.y * dl * len;
                    pr[2] = d.q.z * dl * len;
                    pr[3] = d.w * dl * len;
                }
                totalMassToTip -= 0.5 / inv_mass[vId];
            }
        }
    }
    return 0;
}

// Resample::resampleCMR (YarnBall/io/resample.h:10-170) for one strand, in double: uniform
// Catmull-Rom samples (Kit::cmrSpline, KittenEngine Common.h:625-635) marched at parameter steps of
// 0.2 and refined by eight secant steps to the target segment length, from both ends, merged at the
// closest pair of samples when both have more than 32; done for the target length and again for
// the average length of the first result, keeping the one whose segment lengths vary less.
// Entries the reference would write outside its lists (fewer than 9 samples, or a merge point
// within 8 samples of an end) are skipped.
namespace {
struct DV {
    double x, y, z;
};
inline DV dmix(DV a, DV b, double t) { return {a.x * (1.0 - t) + b.x * t, a.y * (1.0 - t) + b.y * t, a.z * (1.0 - t) + b.z * t}; }
inline double dlen2(DV a, DV b) { double x = a.x - b.x, y = a.y - b.y, z = a.z - b.z; return x * x + y * y + z * z; }
inline double glm_clamp(double x, double lo, double hi) {
    x = (x < lo) ? lo : x;
    return (hi < x) ? hi : x;
}
struct Curve {
    const float* p;
    int n;
    DV at(int i) const { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
    DV sample(double t) const {  // sampleCurve, resample.h:10-18
        int si = (int)std::floor(t);
        si = si < 1 ? 1 : (si > n - 3 ? n - 3 : si);
        DV p0 = at(si - 1), p1 = at(si), p2 = at(si + 1), p3 = at(si + 2);
        double u = t - si;
        DV a0 = dmix(p0, p1, u + 1), a1 = dmix(p1, p2, u + 0), a2 = dmix(p2, p3, u - 1);
        DV b0 = dmix(a0, a1, (u + 1) * 0.5f), b1 = dmix(a1, a2, (u + 0) * 0.5f);
        return dmix(b0, b1, u);
    }
};
std::vector<double> cmr_coords(const Curve& c, double start, double end, double tar) {
    std::vector<double> ts;
    const double step = end > start ? 0.2 : -0.2;
    const double r2 = tar * tar;
    double i = start;
    DV last = c.sample(i);
    ts.push_back(i);
    while ((end > start) ? i < end : i > end) {
        i += step;
        DV pos = c.sample(i);
        double l0 = dlen2(pos, last);
        if (l0 > r2) {
            l0 = std::sqrt(l0);
            double lo = i - step, hi = i;
            if (lo > hi) std::swap(lo, hi);
            const double t0 = i;
            i -= 0.5 * step;
            for (int k = 0; k < 8; k++) {
                double d = std::sqrt(dlen2(c.sample(i), last));
                i += (i - t0) * (tar - d) / (d - l0);
            }
            i = glm_clamp(i, lo, hi);
            ts.push_back(i);
            last = c.sample(i);
        }
    }
    if (ts.size() == 1) {
        ts.push_back(end);
    } else {
        double d = std::sqrt(dlen2(c.sample(ts.back()), c.sample(end)));
        double dt = ts.back() - ts[ts.size() - 2];
        if (d > 0.5f * tar)
            ts.push_back(end);
        else
            ts.back() = end;
        dt -= ts.back() - ts[ts.size() - 2];
        const int N = std::min((int)ts.size(), 8);
        for (int k = 0; k < N; k++) {
            long idx = (long)ts.size() - 2 - k;
            if (idx >= 0) ts[idx] -= dt * (N - k) / (double)N;
        }
    }
    return ts;
}
std::vector<double> cmr_coords_two_way(const Curve& c, double start, double end, double tar) {
    std::vector<double> F = cmr_coords(c, start, end, tar), B = cmr_coords(c, end, start, tar);
    const int BORDER = 8;
    if ((int)F.size() > 4 * BORDER && (int)B.size() > 4 * BORDER) {
        double minErr = std::numeric_limits<double>::infinity();
        int sx = 2 * BORDER, sy = 2 * BORDER;
        for (long i = BORDER, j = (long)B.size() - 1 - BORDER; i < (long)F.size() - 8; i++) {
            double t = F[i];
            while (j > 0 && B[j] < t) j--;
            double t0 = B[j + 1];
            if (minErr > std::abs(t - t0)) { minErr = std::abs(t - t0); sx = (int)i; sy = (int)j + 1; }
            double t1 = B[j];
            if (minErr > std::abs(t1 - t)) { minErr = std::abs(t1 - t); sx = (int)i; sy = (int)j; }
        }
        std::vector<double> m(F.begin(), F.begin() + sx);
        double mid = 0.5 * (F[sx] + B[sy]);
        m.push_back(mid);
        for (int k = sy - 1; k >= 0; k--) m.push_back(B[k]);
        double dt = F[sx] - mid;
        for (int k = 0; k < BORDER; k++) {
            long idx = sx - k - 1;
            if (idx >= 0 && idx < (long)m.size()) m[idx] -= dt * (BORDER - k) / (1. + BORDER);
        }
        dt = B[sy] - mid;
        for (int k = 0; k < BORDER; k++) {
            long idx = sx + k + 1;
            if (idx >= 0 && idx < (long)m.size()) m[idx] -= dt * (BORDER - k) / (1. + BORDER);
        }
        return m;
    }
    return F;
}
}  // namespace

// One strand's resampled points (float xyz) into out, at most max_out of them: returns the count
// resampleCMR produces (the caller resizes when it exceeds the Hair's row, as BuildYarnBallHair does).
int64_t oracle_resample_cmr(const float* pts, int32_t n, double tar, float* out, int64_t max_out) {
    if (n < 4) return -1;
    Curve c{pts, n};
    const double start = 1, end = n - 2;
    std::vector<double> ts0 = cmr_coords_two_way(c, start, end, tar);
    double total = 0, err0 = 0;
    DV last = c.sample(ts0[0]);
    for (size_t i = 1; i < ts0.size(); i++) {
        DV pos = c.sample(ts0[i]);
        double len = std::sqrt(dlen2(pos, last));
        err0 = std::max(err0, std::abs(len - tar));
        total += len;
        last = pos;
    }
    const double avg = total / (ts0.size() - 1);
    std::vector<double> ts1 = cmr_coords_two_way(c, start, end, avg);
    last = c.sample(ts1[0]);
    double err1 = 0;
    for (size_t i = 1; i < ts1.size(); i++) {
        DV pos = c.sample(ts1[i]);
        double len = std::sqrt(dlen2(pos, last));
        err1 = std::max(err1, std::abs(len - avg));
        last = pos;
    }
    const std::vector<double>& ts = err0 < err1 ? ts0 : ts1;
    for (size_t i = 0; i < ts.size() && (int64_t)i < max_out; i++) {
        DV p = c.sample(ts[i]);
        out[3 * i] = (float)p.x;
        out[3 * i + 1] = (float)p.y;
        out[3 * i + 2] = (float)p.z;
    }
    return (int64_t)ts.size();
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// FLOPs of one position update (cosseratItr for an interior vertex: both segments, no hair-hair)
// and one orientation update (quaternionLambdaItr for a segment with both neighbours), counted on
// the reference's operation order.  TEST INFRASTRUCTURE (the roofline's FLOP count).
void oracle_flop_count(int64_t* position_ops, int64_t* orientation_ops) {
    // a 4-vertex strand, slightly bent; vertex 1 / segment 1 have every neighbour
    const int nv = 4;
    std::vector<Counted> im(nv, Counted(1.0 / 3e-7)), lr(nv, Counted(2e-3)), ks(nv, Counted(3e3)), qr(4 * nv),
        x(3 * nv), v(3 * nv), vl(3 * nv), q(4 * nv);
    std::vector<uint32_t> fl = {HAS_NEXT | HAS_NEXT_ORIENTATION, HAS_PREV | HAS_NEXT | HAS_NEXT_ORIENTATION,
                                HAS_PREV | HAS_NEXT, HAS_PREV};
    for (int i = 0; i < nv; i++) {
        x[3 * i] = 2e-3 * i;
        x[3 * i + 1] = 1e-4 * i * i;
        q[4 * i + 3] = 1.0;
        qr[4 * i + 3] = 1e-6;
        qr[4 * i + 2] = 1e-7;
    }
    oracle_params prm{};
    prm.damping = 1e-6f;
    prm.acceleration_ratio = 1.f;
    prm.velocity_decay = 0.05f;
    StepCtx<Counted> c;
    c.p = &prm;
    c.nv = nv;
    c.im = im.data();
    c.lr = lr.data();
    c.ks = ks.data();
    c.fl = fl.data();
    c.qr = qr.data();
    c.x = x.data();
    c.v = v.data();
    c.vl = vl.data();
    c.q = q.data();
    c.y.assign(3 * nv, Counted(1e-5));
    c.dx.assign(3 * nv, Counted(2e-5));
    Counted::ops = 0;
    positionUpdate<Counted>(c, c.dx.data(), 1, Counted(1.0 / 120));
    *position_ops = Counted::ops;
    Counted::ops = 0;
    quaternionUpdate<Counted>(c, q.data(), 1);
    *orientation_ops = Counted::ops;
}

// StrainLimiting (SDFCollisionSolver/cudaSDFCollision.cu:176-199), FP32, over packed strands
// (x: 3 floats per vertex in strand order; l0: rest length of the segment starting at each vertex).
// Per strand, from the root: l = length(x[i+1] - x[i]); if |l - l0| > strain_error * l0 then
// x[i+1] += (l - l0) * normalize(x[i] - x[i+1]), with x[i] as already corrected.  helper_math's
// length is sqrtf(dot) and normalize is v * rsqrtf(dot), whose host form is 1 / sqrtf
// (extern/cuda_helpers/helper_math.h:66, :683, :694-697).
void oracle_strain_limit_f32(int32_t num_strands, const int32_t* strand_begin, const float* l0, float strain_error,
                             float* x) {
    for (int32_t s = 0; s < num_strands; s++) {
        for (int32_t i = strand_begin[s]; i + 1 < strand_begin[s + 1]; i++) {
            float* a = x + 3 * (int64_t)i;
            float* b = a + 3;
            const float ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2];
            const float l = std::sqrt(ux * ux + uy * uy + uz * uz);
            if (std::fabs(l - l0[i]) > strain_error * l0[i]) {
                const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
                const float inv = 1.0f / std::sqrt(dx * dx + dy * dy + dz * dz);
                const float k = l - l0[i];
                b[0] += k * (dx * inv);
                b[1] += k * (dy * inv);
                b[2] += k * (dz * inv);
            }
        }
    }
}

}  // extern "C"
