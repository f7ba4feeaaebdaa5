// StableCosseratRodsB200Solver.cpp -- the Solver plugin on the C ABI (see kami_plugin.h).
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "json_lite.h"
#include "kami_plugin.h"

namespace kami {

namespace {

std::string read_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open settings file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

}  // namespace

StableCosseratRodsB200Solver::~StableCosseratRodsB200Solver() {
    try {
        Flush();
    } catch (...) {  // a destructor does not throw; the held-back step's error is dropped with the solver
    }
    ReleasePins();
    if (handle_) kami_vbd_destroy(handle_);
}

void StableCosseratRodsB200Solver::ReleasePins() {
    if (pinned_) {
        kami_host_unregister(hair_->positions.data());
        kami_host_unregister(hair_->velocities.data());
    }
    pinned_ = false;
}

// A held-back step followed by the SDF solver's strain limiting (SDFBodyCollisionSolver::SolveNextStep,
// SDFBodyCollisionSolver.cpp:182-187): upload, step and strain limiting as three calls.
void StableCosseratRodsB200Solver::StepAndLimit(bool upload) {
    if (upload)
        check(kami_vbd_upload_hair(handle_, hair_->positions.data(), hair_->velocities.data(), KAMI_MEMORY_HOST),
              "UploadHair");
    check(kami_vbd_step(handle_, pending_dt_, nullptr), "SolveNextStep");
    check(kami_vbd_strain_limit(handle_, strain_error_, nullptr), "SolveNextStep (strain limiting)");
}

// Runs what UploadHair / SolveNextStep held back, without a download.
void StableCosseratRodsB200Solver::Flush() {
    const float* x = pending_upload_ ? hair_->positions.data() : nullptr;
    const float* v = pending_upload_ ? hair_->velocities.data() : nullptr;
    if (pending_step_) {
        const bool up = pending_upload_;
        pending_step_ = pending_upload_ = false;
        if (limits_strain())
            StepAndLimit(up);
        else
            check(kami_vbd_step_hair(handle_, pending_dt_, x, v, nullptr, nullptr), "SolveNextStep");
    } else if (pending_upload_) {
        pending_upload_ = false;
        check(kami_vbd_upload_hair(handle_, x, v, KAMI_MEMORY_HOST), "UploadHair");
    }
}

void StableCosseratRodsB200Solver::check(kami_status st, const char* what) {
    if (st != KAMI_OK) throw std::runtime_error(std::string(what) + ": " + kami_vbd_last_error_string());
}

void StableCosseratRodsB200Solver::SetBodyTransform(const float rotation_xyzw[4], const float translate[3]) {
    if (!handle_) return;
    Flush();  // a held-back step runs with the transform it was given
    check(kami_vbd_set_body_transform(handle_, rotation_xyzw, translate), "SetBodyTransform");
}

// StableCosseratRodsSolver::LoadSettingJsonContent + BuildYarnBallHair (StableCosseratRodsSolver.cpp:76-212).
kami_vbd_desc StableCosseratRodsB200Solver::BuildDescriptor(const std::string& settingJsonPath) {
    kami_vbd_desc d;
    check(kami_vbd_desc_init(&d), "kami_vbd_desc_init");
    // reference solver defaults (JsonParams(), StableCosseratRodsSolver.h:86-111) beyond the C-ABI ones
    bool use_young = true;
    float curve_radius = 4e-5f;
    d.num_itr = 8;
    d.wind_peak = 40.f;
    d.gravity[0] = 0.f;
    d.gravity[1] = -9.8f;  // MetaData default (YBSimulator.cu:84)
    d.gravity[2] = 0.f;
    enable_sdf_ = true;
    sdf_threshold_ = 0.015f;
    std::map<std::string, JsonValue> j;
    if (!settingJsonPath.empty()) {
        settings_dump_ = read_file(settingJsonPath);
        j = parse_json_object(settings_dump_);
    }
    auto num = [&](const char* k, float& dst) {
        auto it = j.find(k);
        if (it != j.end() && it->second.kind == JsonValue::Number) dst = (float)it->second.number;
    };
    auto boolean = [&](const char* k, bool& dst) {
        auto it = j.find(k);
        if (it != j.end() && it->second.kind == JsonValue::Bool) dst = it->second.boolean;
    };
    // What this solver does not build is refused rather than ignored: a YarnBall JSON scene
    // (YBJsonPath, the reference's buildFromJSON route, StableCosseratRodsSolver.cpp:42-46: explicit
    // pins, glued endpoints and their connection springs, jsonBuilder.cpp:83-85).
    auto yb = j.find("YBJsonPath");
    if (yb != j.end() && yb->second.kind == JsonValue::String && !yb->second.text.empty() &&
        std::ifstream(yb->second.text).good())
        throw std::runtime_error("YBJsonPath: YarnBall JSON scenes (buildFromJSON, glued endpoints) are not supported");
    // The SDF solver's strain limiting and its tolerance (SDFBodyCollisionSolver.cpp:36-37, defaults
    // SDFBodyCollisionSolver.h:26-27), read from this settings file: the reference's SDF solver reads
    // them from its own settings file, which StableCosseratRodsSolver never passes it (its enabling
    // call, StableCosseratRodsSolver.cpp:60, is commented out).  Runs after each step when EnableSDF.
    strain_limiting_ = false;
    strain_error_ = 0.1f;
    boolean("UseStrainLimiting", strain_limiting_);
    num("StrainError", strain_error_);
    if (!(strain_error_ >= 0.f) || !std::isfinite(strain_error_))
        throw std::runtime_error("StrainError must be finite and >= 0");
    float num_itr = (float)d.num_itr, sag_free = 0.f;
    bool hair_hair = false;
    num("NumItr", num_itr);
    num("YoungsModule", d.young);
    num("StiffnessDeviationCoeff", d.deviation);
    num("StretchK", d.k_stretch);
    num("BendK", d.k_bend);
    num("CurveRadius", curve_radius);
    num("Density", d.density);
    num("VelocityDecay", d.velocity_decay);
    num("ExternalForceMultiplier", d.external_force_multiplier);
    num("WindPeak", d.wind_peak);
    num("WindYFreq", d.wind_y_freq);
    num("WindZFreq", d.wind_z_freq);
    num("WindTimeFreq", d.wind_time_freq);
    num("WindSharpness", d.wind_sharpness);
    num("SagFreeItr", sag_free);
    num("MaxTimeStep", d.max_h);
    num("SDFThreshold", sdf_threshold_);
    boolean("UseYoungsModule", use_young);
    boolean("EnableSDF", enable_sdf_);
    boolean("EnableHairHairColl", hair_hair);
    auto g = j.find("Gravity");
    if (g != j.end() && g->second.kind == JsonValue::Array && g->second.array.size() == 3)
        for (int a = 0; a < 3; a++) d.gravity[a] = (float)g->second.array[a];
    auto sch = j.find("Schedule");
    if (sch != j.end() && sch->second.kind == JsonValue::String) {
        if (sch->second.text == "jacobi") d.schedule = KAMI_SCHEDULE_JACOBI;
        else if (sch->second.text == "colour2") d.schedule = KAMI_SCHEDULE_COLOUR2;
        else throw std::runtime_error("Schedule must be \"colour2\" or \"jacobi\"");
    }
    auto frm = j.find("Form");
    if (frm != j.end() && frm->second.kind == JsonValue::String) {
        if (frm->second.text == "fused") d.form = KAMI_FORM_FUSED;
        else if (frm->second.text == "sweep") d.form = KAMI_FORM_SWEEP;
        else if (frm->second.text == "auto") d.form = KAMI_FORM_AUTO;
        else throw std::runtime_error("Form must be \"auto\", \"fused\" or \"sweep\"");
    }
    d.num_itr = (int32_t)num_itr;
    d.radius = 0.05f * curve_radius;  // StableCosseratRodsSolver.cpp:177-179
    // hair-hair collision: barrier, step limit and velocity radius as the reference solver sets them
    // (StableCosseratRodsSolver.cpp:180-186); it runs on the sweep form
    d.sag_free_itr = sag_free > 0 ? (int32_t)sag_free : 0;  // StableCosseratRodsSolver.cpp:208
    d.hair_hair = hair_hair ? 1 : 0;
    d.barrier_thickness = 2.f * (1.f - 0.05f) * curve_radius;
    d.step_limit = hair_hair ? 1 : 0;
    d.velocity_radius = 1;
    d.stiffness_mode = use_young ? KAMI_STIFFNESS_YOUNG : KAMI_STIFFNESS_K;
    d.pin_roots = 1;

    // the Hair's strands with >= 4 vertices, packed (StableCosseratRodsSolver.cpp:127-173)
    Hair& hair = *hair_;
    strand_refs_.clear();
    strand_begin_.assign(1, 0);
    packed_pos_.clear();
    for (uint32_t s = 0; s < hair.num_strands; s++) {
        const uint32_t n = hair.strand_vert_count[s];
        if (n < 4) continue;
        strand_refs_.push_back((int)s);
        for (uint32_t v = 0; v < n; v++) packed_pos_.insert(packed_pos_.end(), hair.pos(s, v), hair.pos(s, v) + 3);
        strand_begin_.push_back(strand_begin_.back() + (int32_t)n);
    }
    packed_vel_.assign(packed_pos_.size(), 0.f);
    d.num_strands = (int32_t)strand_refs_.size();
    d.strand_begin = strand_begin_.data();
    d.positions = packed_pos_.data();
    d.velocities = nullptr;
    d.sdf = nullptr;
    if (enable_sdf_ && has_body_) {
        sdf_desc_ = kami_vbd_sdf_desc{};
        for (int a = 0; a < 3; a++) {
            sdf_desc_.dims[a] = body_.dims[a];
            sdf_desc_.grid_min[a] = body_.grid_min[a];
            sdf_desc_.grid_max[a] = body_.grid_max[a];
        }
        sdf_desc_.threshold = sdf_threshold_;
        sdf_desc_.phi = body_.phi.data();
        sdf_desc_.grad = body_.grad.data();
        d.sdf = &sdf_desc_;
    }
    return d;
}

void StableCosseratRodsB200Solver::Preprocess(const std::string& settingJsonPath) {
    // JsonParams defaults (StableCosseratRodsSolver.h:86-111)
    float subdiv = 3.f, resample_len = 1e-3f;
    bool resample = true;
    if (!settingJsonPath.empty()) {
        auto j = parse_json_object(read_file(settingJsonPath));
        auto it = j.find("SubdivCoeff");
        if (it != j.end() && it->second.kind == JsonValue::Number) subdiv = (float)it->second.number;
        it = j.find("ResampleLen");
        if (it != j.end() && it->second.kind == JsonValue::Number) resample_len = (float)it->second.number;
        it = j.find("EnableResample");
        if (it != j.end() && it->second.kind == JsonValue::Bool) resample = it->second.boolean;
    }
    Hair& hair = *hair_;
    std::vector<int32_t> counts(hair.strand_vert_count.begin(), hair.strand_vert_count.end());
    const int32_t mul = (int32_t)subdiv;
    if (mul > 1) {  // Construct: DivideHair when SubdivCoeff > 1 (StableCosseratRodsSolver.cpp:40)
        const uint32_t out_verts = (hair.max_verts - 1) * (uint32_t)mul + 1;
        std::vector<int32_t> oc(hair.num_strands);
        std::vector<float> ox((size_t)hair.num_strands * out_verts * 3, 0.f), ov(ox.size(), 0.f);
        check(kami_hair_subdivide((int32_t)hair.num_strands, counts.data(), (int32_t)hair.max_verts, hair.positions.data(),
                                  hair.velocities.data(), mul, oc.data(), ox.data(), ov.data(), -1),
              "Construct (SubdivCoeff)");
        hair.max_verts = out_verts;
        hair.positions.swap(ox);
        hair.velocities.swap(ov);
        counts.swap(oc);
    }
    if (resample) {
        check(kami_hair_resample((int32_t)hair.num_strands, counts.data(), (int32_t)hair.max_verts, hair.positions.data(),
                                 resample_len, -1),
              "Construct (EnableResample)");
    }
    hair.strand_vert_count.assign(counts.begin(), counts.end());
}

void StableCosseratRodsB200Solver::Construct(const std::string& settingJsonPath) {
    if (handle_) Flush();
    ReleasePins();  // Preprocess may reallocate the Hair's arrays
    Preprocess(settingJsonPath);
    kami_vbd_desc d = BuildDescriptor(settingJsonPath);
    if (d.num_strands == 0) throw std::runtime_error("the Hair has no strand with at least 4 vertices");
    if (handle_) kami_vbd_destroy(handle_);
    handle_ = nullptr;
    check(kami_vbd_create(&d, &handle_), "Construct");
    // the Hair's padded arrays are read and written in place, through the strandRefs mapping
    check(kami_vbd_set_hair_layout(handle_, (int32_t)hair_->num_strands, (int32_t)hair_->max_verts, strand_refs_.data()),
          "Construct");
    // page-locked Hair arrays let a frame read and write them from the kernel (kami_vbd_step_hair)
    const size_t bytes = sizeof(float) * hair_->positions.size();
    if (bytes > 0 && hair_->velocities.size() == hair_->positions.size()) {
        const bool px = kami_host_register(hair_->positions.data(), bytes) == KAMI_OK;
        const bool pv = px && kami_host_register(hair_->velocities.data(), bytes) == KAMI_OK;
        if (px && !pv) kami_host_unregister(hair_->positions.data());
        pinned_ = px && pv;  // otherwise the frames copy the arrays
    }
}

// Sim::advance + the SDF pass (StableCosseratRodsSolver.cpp:216-234).  Held back until the next
// call, so that a DownloadHair right after it makes one kernel launch of the step and the download.
void StableCosseratRodsB200Solver::SolveNextStep(float dt) {
    if (!handle_) throw std::runtime_error("SolveNextStep before Construct");
    if (pending_step_) Flush();
    pending_step_ = true;
    pending_dt_ = dt;
}

// Sim -> Hair (StableCosseratRodsSolver.cpp:258-277): with a held-back step, the step and the
// download in one call; else one gather on the GPU into the padded arrays
void StableCosseratRodsB200Solver::DownloadHair() {
    if (pending_step_ && !limits_strain()) {
        const bool up = pending_upload_;
        pending_step_ = pending_upload_ = false;
        check(kami_vbd_step_hair(handle_, pending_dt_, up ? hair_->positions.data() : nullptr,
                                 up ? hair_->velocities.data() : nullptr, hair_->positions.data(),
                                 hair_->velocities.data()),
              "SolveNextStep + DownloadHair");
        return;
    }
    Flush();
    check(kami_vbd_download_hair(handle_, hair_->positions.data(), hair_->velocities.data(), KAMI_MEMORY_HOST),
          "DownloadHair");
}

// Hair -> Sim (StableCosseratRodsSolver.cpp:238-256): held back until the next step or download
void StableCosseratRodsB200Solver::UploadHair() {
    if (!handle_) throw std::runtime_error("UploadHair before Construct");
    Flush();
    pending_upload_ = true;
}

std::string StableCosseratRodsB200Solver::GetInfoString() {
    std::stringstream ss;
    ss << "Solver: Stable Cosserat Rods (B200, " << kami_vbd_version() << ")\n";
    ss << "Simulated strands: " << strand_refs_.size() << "\n";
    ss << "Json:\n" << settings_dump_;
    return ss.str();
}

}  // namespace kami
