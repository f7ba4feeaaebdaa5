// kami_plugin.h -- the C++ solver plugin that drops into KamiSimulator's Solver interface
// (src/solvers/Solver.h:13-85), on top of the C ABI in include/kami_vbd.h.
//
// Hair mirrors the part of KamiSimulator's Hair the StableCosseratRods solver reads and writes
// (src/Hair.h:10-52, LinearUtil.h:150-176): a padded [strand][vertex] array of positions and
// velocities plus the vertex count of each strand.  Solver mirrors the reference's abstract plugin
// (same method names and meanings: Construct(settings json), SolveNextStep(dt in seconds),
// UploadHair, DownloadHair, GetInfoString).
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "kami_vbd.h"

namespace kami {

struct Hair {
    uint32_t num_strands = 0;
    uint32_t max_verts = 0;                 // hairSize.y
    std::vector<uint32_t> strand_vert_count;
    std::vector<float> positions;           // num_strands * max_verts * 3
    std::vector<float> velocities;          // same layout
    float* pos(uint32_t s, uint32_t v) { return &positions[((size_t)s * max_verts + v) * 3]; }
    float* vel(uint32_t s, uint32_t v) { return &velocities[((size_t)s * max_verts + v) * 3]; }
};

class Solver {
   public:
    explicit Solver(std::shared_ptr<Hair> hair) : hair_(std::move(hair)) {}
    virtual ~Solver() = default;
    virtual void Construct(const std::string& settingJsonPath = "") = 0;
    virtual void SolveNextStep(float dt) = 0;  // dt in seconds (1 / (fps * internal steps))
    virtual void UploadHair() = 0;
    virtual void DownloadHair() = 0;
    virtual std::string GetInfoString() = 0;

   protected:
    std::shared_ptr<Hair> hair_;
};

// Body collision input: the head's signed-distance grid (as SDFBodyCollisionSolver builds it from
// the body mesh) and its rigid transform.
struct BodySDF {
    int32_t dims[3] = {0, 0, 0};
    float grid_min[3] = {0, 0, 0}, grid_max[3] = {0, 0, 0};
    std::vector<float> phi, grad;
};

// The StableCosseratRods solver on B200.  Settings keys are those of the reference's solver JSON
// (StableCosseratRodsSolver.h:41-112): NumItr, UseYoungsModule, YoungsModule,
// StiffnessDeviationCoeff, StretchK, BendK, CurveRadius (the simulated radius is 0.05 x CurveRadius,
// StableCosseratRodsSolver.cpp:177-179), Density, VelocityDecay, ExternalForceMultiplier, Wind*,
// EnableSDF, EnableHairHairColl, SagFreeItr, SubdivCoeff, EnableResample, plus the SDF solver's
// SDFThreshold, UseStrainLimiting and StrainError (SDFBodyCollisionSolver.h:25-27: strain limiting
// after each step, when EnableSDF) and the extensions MaxTimeStep (the reference fixes 4e-4 s),
// Gravity [x, y, z], Schedule ("colour2" | "jacobi") and Form ("auto" | "fused" | "sweep").
// SagFreeItr runs that many passes of sag-free initialisation at Construct
// (StableCosseratRodsSolver.cpp:208).  EnableHairHairColl turns on hair-hair collision with the reference solver's barrier
// (2 (1 - 0.05) CurveRadius), step limit and velocity radius (StableCosseratRodsSolver.cpp:176-186).
// Strands with fewer than 4 vertices are skipped, as there (StableCosseratRodsSolver.cpp:134-136).
// Construct first subdivides the Hair (SubdivCoeff, default 3) and resamples its strands to
// ResampleLen (EnableResample, default on) on the GPU, as the reference solver does; BuildDescriptor
// (and the driver's dry run) describes the Hair as it is.
class StableCosseratRodsB200Solver : public Solver {
   public:
    explicit StableCosseratRodsB200Solver(std::shared_ptr<Hair> hair) : Solver(std::move(hair)) {}
    ~StableCosseratRodsB200Solver() override;

    void SetBody(const BodySDF& body) { body_ = body; has_body_ = true; }
    void SetBodyTransform(const float rotation_xyzw[4], const float translate[3]);

    // Fills the C-ABI descriptor from the settings file and the Hair, without touching a device.
    kami_vbd_desc BuildDescriptor(const std::string& settingJsonPath);

    void Construct(const std::string& settingJsonPath = "") override;
    void SolveNextStep(float dt) override;
    void UploadHair() override;
    void DownloadHair() override;
    std::string GetInfoString() override;

    // the SDF solver's strain limiting as the settings set it (UseStrainLimiting, StrainError)
    bool strain_limiting() const { return strain_limiting_; }
    float strain_error() const { return strain_error_; }

    // the C-ABI handle, for calls beyond the Solver interface (runs what is held back first)
    kami_vbd_handle handle() {
        if (handle_) Flush();
        return handle_;
    }

   private:
    kami_vbd_handle handle_ = nullptr;
    BodySDF body_;
    bool has_body_ = false;
    bool enable_sdf_ = true;
    float sdf_threshold_ = 0.015f;
    bool strain_limiting_ = false;
    float strain_error_ = 0.1f;
    // strain limiting runs inside the SDF solver's step, so only with EnableSDF
    bool limits_strain() const { return strain_limiting_ && enable_sdf_; }
    void StepAndLimit(bool upload);
    std::string settings_dump_;
    std::vector<int> strand_refs_;      // Hair strand of each simulated strand
    std::vector<int32_t> strand_begin_;
    std::vector<float> packed_pos_, packed_vel_;
    kami_vbd_sdf_desc sdf_desc_{};
    // Frames over the Hair.  Construct page-locks the Hair's position and velocity arrays
    // (kami_host_register); they must then not be reallocated until the solver is destroyed.  The
    // last SolveNextStep before a DownloadHair, and an UploadHair before a SolveNextStep, are held
    // back and run as one kami_vbd_step_hair call (upload, step and download in one launch), or, with
    // strain limiting, as upload, step, strain limiting and download; any other call runs what is
    // held back first, so errors of a held-back step surface at that call.
    bool pinned_ = false;
    bool pending_upload_ = false, pending_step_ = false;
    float pending_dt_ = 0.f;
    void Flush();
    void ReleasePins();
    void check(kami_status st, const char* what);
    // SubdivCoeff (DivideHair) and EnableResample / ResampleLen on the Hair, as Construct and
    // BuildYarnBallHair do them (StableCosseratRodsSolver.cpp:40, :141-163)
    void Preprocess(const std::string& settingJsonPath);
};

}  // namespace kami
