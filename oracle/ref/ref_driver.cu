// ref_driver.cu -- TEST INFRASTRUCTURE ONLY.
//
// A thin C driver around KamiSimulator's own Stable Cosserat Rods code, compiled from the
// reference sources in place (oracle/ref/Makefile) into oracle/_ref/libkami_ref.so.  The tests use
// it on a GPU to pin the CPU oracle to the reference itself: material set-up (Sim::configure +
// setYoung, YarnBall/YBSimulator.cu:161-320), the racy Jacobi step (Sim::advance,
// YarnBall/sim/step.cpp:38-62, kernels in YarnBall/sim/{iteration,cosserat}.cu) and the SDF pass
// (SDFHeadCollision, SDFCollisionSolver/cudaSDFCollision.cu:205-268).  Nothing in the product loads it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "solvers/SDFCollisionSolver/cudaSDFCollision.cuh"
#include "solvers/StableCosseratRods/YarnBall/YBSimulator.h"

namespace YarnBall {
extern std::shared_ptr<Sim> createFromCurves(std::vector<std::vector<glm::vec3>>& curves, std::vector<bool>& isCurveClosed,
                                             int numVerts);
// the reference's step kernels (YarnBall/sim/{iteration,cosserat,collision}.cu), declared as
// YBSimulator.cu:29-50 declares them
extern __global__ void cosseratItr(MetaData* data);
extern __global__ void quaternionLambdaItr(MetaData* data);
extern __global__ void initItr(MetaData* data);
extern __global__ void endItr(MetaData* data);
template <bool USE_VEL_RADIUS>
extern __global__ void buildCollisionList(MetaData* data, int maxCols, int* errorReturn);
extern template __global__ void buildCollisionList<true>(MetaData* data, int maxCols, int* errorReturn);
template <bool LIMIT, bool USE_VEL_RADIUS>
extern __global__ void recomputeStepLimitKernel(MetaData* data);
extern template __global__ void recomputeStepLimitKernel<true, true>(MetaData* data);
}

namespace {
struct Holder {
    std::shared_ptr<YarnBall::Sim> sim;
};
}  // namespace

extern "C" {

// Builds a Sim the way StableCosseratRodsSolver::BuildYarnBallHair does (StableCosseratRodsSolver.cpp:112-212),
// with the radius given directly (MetaData::radius), one Young's modulus / deviation for all strands,
// maxH = max_h and meta.h = max_h, no hair-hair collision and no wind.
void* ref_create(int64_t nv, int32_t ns, const int32_t* sb, const float* pos, float radius, float density, float young,
                 float deviation, const float* gravity, float velocity_decay, int32_t num_itr, float max_h,
                 int32_t pin_roots) {
    try {
        std::vector<std::vector<glm::vec3>> curves(ns);
        std::vector<bool> closed(ns, false);
        for (int32_t s = 0; s < ns; s++)
            for (int32_t i = sb[s]; i < sb[s + 1]; i++) curves[s].push_back(glm::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
        auto sim = YarnBall::createFromCurves(curves, closed, (int)nv);
        sim->meta.radius = radius;
        sim->meta.barrierThickness = 1e-7f;  // only used by hair-hair collision (off); keeps uploadMeta's check quiet
        sim->meta.numItr = num_itr;
        sim->meta.velocityDecay = velocity_decay;
        sim->meta.gravity = glm::vec3(gravity[0], gravity[1], gravity[2]);
        sim->meta.useStepSizeLimit = false;
        sim->meta.enableHairHairColl = false;
        sim->meta.ExternalForceMultiplier = 1.f;
        sim->meta.windPeak = 0.f;
        sim->maxH = max_h;
        sim->meta.h = max_h;
        sim->printErrors = false;
        sim->configure(density);
        sim->setYoung(young, deviation);
        if (pin_roots)
            for (int32_t s = 0; s < ns; s++) sim->verts[sb[s]].invMass = 0;
        sim->upload();
        return new Holder{sim};
    } catch (...) {
        return nullptr;
    }
}

void ref_destroy(void* h) { delete (Holder*)h; }

// Sim::SagFree (YBSimulator.cu:480-674) on the host arrays, with every strand's first vertex as its
// root, as BuildYarnBallHair passes them (StableCosseratRodsSolver.cpp:208); ref_material reads
// the result.
int ref_sag_free(void* h, int32_t ns, const int32_t* sb, int32_t iterations) {
    auto& sim = ((Holder*)h)->sim;
    std::vector<int> roots(sb, sb + ns);
    sim->SagFree(roots, (uint32_t)iterations);
    return 0;
}

int ref_material(void* h, float* inv_mass, float* l_rest, float* k_stretch, uint32_t* flags, float* q, float* q_rest) {
    auto& sim = ((Holder*)h)->sim;
    const int nv = sim->meta.numVerts;
    for (int i = 0; i < nv; i++) {
        inv_mass[i] = sim->verts[i].invMass;
        l_rest[i] = sim->verts[i].lRest;
        k_stretch[i] = sim->verts[i].kStretch;
        flags[i] = sim->verts[i].flags;
        std::memcpy(q + 4 * i, &sim->qs[i].v, 4 * sizeof(float));
        std::memcpy(q_rest + 4 * i, &sim->qRests[i], 4 * sizeof(float));
    }
    return 0;
}

// Sets every vertex's connectionIndex (YarnBall.h:56; -1: none), as glueEndpoints and the closed-curve
// reader set it (jsonBuilder.cpp:165-185, reader.cpp:40-44), and uploads the vertices.
int ref_set_connections(void* h, const int32_t* conn) {
    auto& sim = ((Holder*)h)->sim;
    for (int i = 0; i < sim->meta.numVerts; i++) sim->verts[i].connectionIndex = conn[i];
    sim->upload();
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// Overwrites positions, velocities, last velocities, orientations and the clock.
int ref_set_state(void* h, const float* x, const float* v, const float* vlast, const float* q, const float* clock) {
    auto& sim = ((Holder*)h)->sim;
    const int nv = sim->meta.numVerts;
    for (int i = 0; i < nv; i++) {
        sim->verts[i].pos = glm::vec3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        sim->vels[i] = glm::vec3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        std::memcpy(&sim->qs[i].v, q + 4 * i, 4 * sizeof(float));
    }
    sim->upload();
    if (cudaMemcpy(sim->meta.d_lastVels, vlast, sizeof(float) * 3 * nv, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    sim->meta.h = clock[0];
    sim->meta.lastH = clock[1];
    sim->meta.time = clock[2];
    return 0;
}

// One substep of the reference's hair-hair path with its own kernels, in Sim::advance's order
// (step.cpp:44-58): initItr, detection, then the step graph (recomputeStepLimit, numItr x
// (cosseratItr, quaternionLambdaItr), endItr), with the launch shapes of YBSimulator.cu:414-420.
// Detection is buildCollisionList<true> (collision.cu:36-92) over every pair of segments instead of
// the LBVH query's overlapping pairs: the distance test decides either way, and the LBVH as shipped
// cannot run (LBVH::compute reads d_flags[0] before sizing it, KittenGpuLBVH/lbvh.cu:366-370).  Uses
// useStepSizeLimit and useVelocityRadius, as StableCosseratRodsSolver sets them.  Returns the
// reference's error word, or -1 when a CUDA call failed.
int ref_step_hair_hair(void* h, float dt, float barrier) {
    auto& sim = ((Holder*)h)->sim;
    YarnBall::MetaData m = sim->meta;
    const int nv = m.numVerts;
    m.barrierThickness = barrier;
    m.enableHairHairColl = true;
    m.useStepSizeLimit = true;
    m.useVelocityRadius = true;
    m.detectionRadius = m.radius + 0.5f * m.barrierThickness;  // Sim::uploadMeta, YBSimulator.cu:323-324
    m.scaledDetectionRadius = m.detectionRadius * m.detectionScaler;
    m.lastH = m.h;
    m.h = dt;
    std::vector<glm::ivec2> pairs;
    for (int i = 0; i < nv; i++)
        for (int j = i + 1; j < nv; j++)
            if ((sim->verts[i].flags & (uint32_t)YarnBall::VertexFlags::hasNext) &&
                (sim->verts[j].flags & (uint32_t)YarnBall::VertexFlags::hasNext))
                pairs.push_back(glm::ivec2(i, j));
    YarnBall::MetaData* dm = nullptr;
    glm::ivec2* dpairs = nullptr;
    int* derr = nullptr;
    int err[2] = {0, 0};
    bool ok = !pairs.empty() && cudaMalloc(&dm, sizeof(m)) == cudaSuccess &&
              cudaMalloc(&dpairs, sizeof(glm::ivec2) * pairs.size()) == cudaSuccess &&
              cudaMalloc(&derr, 2 * sizeof(int)) == cudaSuccess;
    if (ok) {
        m.d_boundColList = dpairs;
        ok = cudaMemcpy(dm, &m, sizeof(m), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(dpairs, pairs.data(), sizeof(glm::ivec2) * pairs.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemset(derr, 0, 2 * sizeof(int)) == cudaSuccess && cudaMemset(m.d_numCols, 0, sizeof(int) * nv) == cudaSuccess;
    }
    if (ok) {
        const int np = (int)pairs.size();
        YarnBall::initItr<<<(nv + 255) / 256, 256>>>(dm);
        YarnBall::buildCollisionList<true><<<(np + 127) / 128, 128>>>(dm, np, derr);
        YarnBall::recomputeStepLimitKernel<true, true><<<(nv + 127) / 128, 128>>>(dm);
        for (int it = 0; it < m.numItr; it++) {
            YarnBall::cosseratItr<<<((nv - 1) + (VERTEX_PER_BLOCK - 1)) / (VERTEX_PER_BLOCK - 1), BLOCK_SIZE>>>(dm);
            YarnBall::quaternionLambdaItr<<<(nv + 127) / 128, 128>>>(dm);
        }
        YarnBall::endItr<<<(nv + 255) / 256, 256>>>(dm);
        ok = cudaDeviceSynchronize() == cudaSuccess && cudaMemcpy(err, derr, sizeof(err), cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    if (dm) cudaFree(dm);
    if (dpairs) cudaFree(dpairs);
    if (derr) cudaFree(derr);
    if (!ok) return -1;
    sim->meta.lastH = m.lastH;
    sim->meta.h = m.h;
    sim->meta.time += dt;
    return err[0];
}

int ref_advance(void* h, float dt) {
    auto& sim = ((Holder*)h)->sim;
    try {
        sim->advance(dt);
    } catch (...) {
        return 2;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

int ref_download(void* h, float* x, float* v, float* q) {
    auto& sim = ((Holder*)h)->sim;
    sim->download();
    const int nv = sim->meta.numVerts;
    for (int i = 0; i < nv; i++) {
        std::memcpy(x + 3 * i, &sim->verts[i].pos, 3 * sizeof(float));
        std::memcpy(v + 3 * i, &sim->vels[i], 3 * sizeof(float));
        std::memcpy(q + 4 * i, &sim->qs[i].v, 4 * sizeof(float));
    }
    return 0;
}

// The SDF solver's StrainLimiting kernel (cudaSDFCollision.cu:176-199) over packed strands, set up
// as SDFBodyCollisionSolver::InitAdditionalHairData does (SDFBodyCollisionSolver.cpp:100-121): every
// particle's GlobalIdx and StrandLength, EdgeRestIdx.y naming its segment's rest length, and the
// roots' indices.  l0[i]: rest length of the segment starting at vertex i.
int ref_strain_limit(int32_t num_strands, const int32_t* strand_begin, const float* l0, float strain_error, float* x) {
    const int64_t np = strand_begin[num_strands];
    SDFSimulationParams p{};
    p.NumStrands = (size_t)num_strands;
    p.NumParticles = (size_t)np;
    p.StrainError = strain_error;
    p.UseStrainLimiting = true;
    KamiCopySDFSimParamsToDevice(&p);
    std::vector<ParticleForSDFColl> parts(np);
    std::vector<int> roots(num_strands);
    for (int32_t s = 0; s < num_strands; s++) {
        roots[s] = strand_begin[s];
        for (int32_t i = strand_begin[s]; i < strand_begin[s + 1]; i++) {
            parts[i].Position = make_float3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
            parts[i].StrandLength = strand_begin[s + 1] - strand_begin[s];
            parts[i].LocalIdx = i - strand_begin[s];
            parts[i].GlobalIdx = i;
            parts[i].EdgeRestIdx.y = i;
        }
    }
    SDFDeviceBuffers b{};
    if (cudaMalloc(&b.Particles, sizeof(ParticleForSDFColl) * np) != cudaSuccess) return 1;
    if (cudaMalloc(&b.restLenghts, sizeof(float) * np) != cudaSuccess) return 1;
    if (cudaMalloc(&b.rootIdx, sizeof(int) * num_strands) != cudaSuccess) return 1;
    cudaMemcpy(b.Particles, parts.data(), sizeof(ParticleForSDFColl) * np, cudaMemcpyHostToDevice);
    cudaMemcpy(b.restLenghts, l0, sizeof(float) * np, cudaMemcpyHostToDevice);
    cudaMemcpy(b.rootIdx, roots.data(), sizeof(int) * num_strands, cudaMemcpyHostToDevice);
    KamiLaunchKernelStrainLimitingAfterSDFCollision(make_int2((num_strands + 127) / 128, 128), b);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(parts.data(), b.Particles, sizeof(ParticleForSDFColl) * np, cudaMemcpyDeviceToHost);
    cudaFree(b.Particles);
    cudaFree(b.restLenghts);
    cudaFree(b.rootIdx);
    for (int64_t i = 0; i < np; i++) {
        x[3 * i] = parts[i].Position.x;
        x[3 * i + 1] = parts[i].Position.y;
        x[3 * i + 2] = parts[i].Position.z;
    }
    return e == cudaSuccess ? 0 : 1;
}

// One SDFHeadCollision pass over np particles, with the grid spacing SDFBodyCollisionSolver::InitParams
// computes (SDFBodyCollisionSolver.cpp:142-159).  local_idx[i] == 0 marks strand roots.
int ref_sdf_project(int64_t np, float* pos, float* vel, const int32_t* local_idx, const int32_t* dims, const float* gmin,
                    const float* gmax, float thresh, const float* phi, const float* grad, const float* rot,
                    const float* trans) {
    SDFSimulationParams p{};
    p.Dt = 1.f;
    p.InvDt = 1.f;
    p.SDFDim = make_int3(dims[0], dims[1], dims[2]);
    p.NumParticles = (size_t)np;
    p.NumSdfCells = (size_t)dims[0] * dims[1] * dims[2];
    p.ThreshSdf = thresh;
    p.HeadMin = make_float3(gmin[0], gmin[1], gmin[2]);
    p.HeadMax = make_float3(gmax[0], gmax[1], gmax[2]);
    float dxS = (gmax[0] - gmin[0]) / (1.f * dims[0]);
    float dyS = (gmax[1] - gmin[1]) / (1.f * dims[1]);
    float dzS = (gmax[2] - gmin[2]) / (1.f * dims[2]);
    p.SdfInvSqDs = make_float3(1.f / (dxS * dxS), 1.f / (dyS * dyS), 1.f / (dzS * dzS));
    p.SDFInvDs = make_float3(1.f / dxS, 1.f / dyS, 1.f / dzS);
    p.SdfDs = make_float3(dxS, dyS, dzS);
    p.rotation = make_float4(rot[0], rot[1], rot[2], rot[3]);
    p.translate = make_float3(trans[0], trans[1], trans[2]);
    KamiCopySDFSimParamsToDevice(&p);
    std::vector<ParticleForSDFColl> parts(np);
    for (int64_t i = 0; i < np; i++) {
        parts[i].Position = make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        parts[i].Velocity = make_float3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        parts[i].LocalIdx = local_idx[i];
        parts[i].GlobalIdx = (int)i;
    }
    SDFDeviceBuffers b{};
    size_t cells = p.NumSdfCells;
    if (cudaMalloc(&b.Particles, sizeof(ParticleForSDFColl) * np) != cudaSuccess) return 1;
    if (cudaMalloc(&b.SDF, sizeof(float) * cells) != cudaSuccess) return 1;
    if (cudaMalloc(&b.NablaSDF, sizeof(float3) * cells) != cudaSuccess) return 1;
    cudaMemcpy(b.Particles, parts.data(), sizeof(ParticleForSDFColl) * np, cudaMemcpyHostToDevice);
    cudaMemcpy(b.SDF, phi, sizeof(float) * cells, cudaMemcpyHostToDevice);
    cudaMemcpy(b.NablaSDF, grad, sizeof(float3) * cells, cudaMemcpyHostToDevice);
    int blocks = (int)((np + 255) / 256);
    KamiLaunchKernelSDFHeadCollision(make_int2(blocks, 256), b);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(parts.data(), b.Particles, sizeof(ParticleForSDFColl) * np, cudaMemcpyDeviceToHost);
    cudaFree(b.Particles);
    cudaFree(b.SDF);
    cudaFree(b.NablaSDF);
    for (int64_t i = 0; i < np; i++) {
        pos[3 * i] = parts[i].Position.x;
        pos[3 * i + 1] = parts[i].Position.y;
        pos[3 * i + 2] = parts[i].Position.z;
        vel[3 * i] = parts[i].Velocity.x;
        vel[3 * i + 1] = parts[i].Velocity.y;
        vel[3 * i + 2] = parts[i].Velocity.z;
    }
    return e == cudaSuccess ? 0 : 1;
}

}  // extern "C"
