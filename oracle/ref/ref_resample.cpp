// ref_resample.cpp -- TEST INFRASTRUCTURE ONLY.
//
// KamiSimulator's strand resampling (Resample::resampleCMR, YarnBall/io/resample.h) compiled from
// the reference sources in place into oracle/_ref/libkami_ref_cpu.so (oracle/ref/Makefile), CPU only.
#include <cstdint>
#include <cstring>
#include <vector>

#include "glm/glm.hpp"
#include "KittenEngine/includes/modules/Common.h"
namespace Kit = Kitten;
#include "YarnBall/io/resample.h"

extern "C" {

// resampleCMR(curve, 1, n - 2, target) as BuildYarnBallHair calls it
// (StableCosseratRodsSolver.cpp:141-143); writes at most max_out points, returns the count.
int64_t ref_resample_cmr(const float* pts, int32_t n, double target, float* out, int64_t max_out) {
    std::vector<glm::vec3> curve(n);
    for (int32_t i = 0; i < n; i++) curve[i] = glm::vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    std::vector<glm::vec3> r = Resample::resampleCMR(curve, 1, curve.size() - 2, target);
    for (size_t i = 0; i < r.size() && (int64_t)i < max_out; i++) std::memcpy(out + 3 * i, &r[i], 12);
    return (int64_t)r.size();
}

}  // extern "C"
