// solver_driver.cpp -- runs StableCosseratRodsB200Solver the way KamiSimulator drives a solver
// (Construct, then per frame SolveNextStep + DownloadHair), for the tests.
//
//   kami_solver_driver settings.json hair.bin steps dt out.bin [sdf.bin]
//   kami_solver_driver --dry-run settings.json hair.bin        (prints the descriptor, no device)
//
// hair.bin: uint32 strands, uint32 max_verts, uint32 counts[strands], float positions[strands][max_verts][3],
//           or a USC-HairSalon .data file (read into a Hair of 100 vertices per strand, as
//           ImportUSCHairSalonToHair does, importers/USCHairsalonImporter.cpp:56-80)
// out.bin:  float positions[strands][max_verts][3], float velocities[...], or a .data file of the
//           final positions (ExportHairAsUSCHairsalon, exporters/USCHairsalonExporter.cpp:20-26)
// sdf.bin:  int32 dims[3], float min[3], float max[3], float phi[n], float grad[3n]
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>

#include "kami_plugin.h"

using namespace kami;

static bool is_usc(const char* path) {
    const size_t n = std::strlen(path);
    return n > 5 && std::strcmp(path + n - 5, ".data") == 0;
}

static std::shared_ptr<Hair> read_hair(const char* path) {
    if (is_usc(path)) {
        int32_t ns = 0, mx = 0;
        int64_t nv = 0;
        if (kami_usc_info(path, &ns, &nv, &mx) != KAMI_OK) throw std::runtime_error(kami_vbd_last_error_string());
        auto h = std::make_shared<Hair>();
        h->num_strands = (uint32_t)ns;
        h->max_verts = 100;
        std::vector<int32_t> counts(ns);
        h->positions.assign((size_t)ns * h->max_verts * 3, 0.f);
        if (kami_usc_read(path, (int32_t)h->max_verts, counts.data(), h->positions.data()) != KAMI_OK)
            throw std::runtime_error(kami_vbd_last_error_string());
        h->strand_vert_count.assign(counts.begin(), counts.end());
        h->velocities.assign(h->positions.size(), 0.f);
        return h;
    }
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open hair file");
    auto h = std::make_shared<Hair>();
    f.read((char*)&h->num_strands, 4);
    f.read((char*)&h->max_verts, 4);
    h->strand_vert_count.resize(h->num_strands);
    f.read((char*)h->strand_vert_count.data(), 4 * h->num_strands);
    h->positions.resize((size_t)h->num_strands * h->max_verts * 3);
    f.read((char*)h->positions.data(), 4 * h->positions.size());
    h->velocities.assign(h->positions.size(), 0.f);
    if (!f) throw std::runtime_error("short hair file");
    return h;
}

int main(int argc, char** argv) {
    try {
        if (argc >= 4 && std::strcmp(argv[1], "--dry-run") == 0) {
            auto hair = read_hair(argv[3]);
            StableCosseratRodsB200Solver s(hair);
            kami_vbd_desc d = s.BuildDescriptor(argv[2]);
            std::printf("{\"num_strands\": %d, \"num_vertices\": %d, \"radius\": %.9g, \"density\": %.9g, "
                        "\"num_itr\": %d, \"young\": %.9g, \"deviation\": %.9g, \"stiffness_mode\": %d, "
                        "\"velocity_decay\": %.9g, \"wind_peak\": %.9g, \"max_h\": %.9g, \"schedule\": %d, "
                        "\"form\": %d, \"gravity\": [%.9g, %.9g, %.9g], \"hair_hair\": %d, "
                        "\"barrier_thickness\": %.9g, \"step_limit\": %d, \"sag_free_itr\": %d, "
                        "\"strain_limiting\": %d, \"strain_error\": %.9g}\n",
                        d.num_strands, d.strand_begin[d.num_strands], d.radius, d.density, d.num_itr, d.young,
                        d.deviation, d.stiffness_mode, d.velocity_decay, d.wind_peak, d.max_h, d.schedule, d.form,
                        d.gravity[0], d.gravity[1], d.gravity[2], d.hair_hair, d.barrier_thickness, d.step_limit,
                        d.sag_free_itr, s.strain_limiting() ? 1 : 0, s.strain_error());
            return 0;
        }
        if (argc < 6) {
            std::fprintf(stderr, "usage: %s settings.json hair.bin steps dt out.bin [sdf.bin]\n", argv[0]);
            return 2;
        }
        auto hair = read_hair(argv[2]);
        const int steps = std::atoi(argv[3]);
        const float dt = (float)std::atof(argv[4]);
        StableCosseratRodsB200Solver s(hair);
        if (argc >= 7) {
            std::ifstream f(argv[6], std::ios::binary);
            BodySDF b;
            f.read((char*)b.dims, 12);
            f.read((char*)b.grid_min, 12);
            f.read((char*)b.grid_max, 12);
            const size_t n = (size_t)b.dims[0] * b.dims[1] * b.dims[2];
            b.phi.resize(n);
            b.grad.resize(3 * n);
            f.read((char*)b.phi.data(), 4 * n);
            f.read((char*)b.grad.data(), 12 * n);
            if (!f) throw std::runtime_error("short sdf file");
            s.SetBody(b);
        }
        s.Construct(argv[1]);
        for (int i = 0; i < steps; i++) {
            s.SolveNextStep(dt);
            s.DownloadHair();
        }
        if (is_usc(argv[5])) {
            std::vector<int32_t> counts(hair->strand_vert_count.begin(), hair->strand_vert_count.end());
            if (kami_usc_write(argv[5], (int32_t)hair->num_strands, counts.data(), (int32_t)hair->max_verts,
                               hair->positions.data()) != KAMI_OK)
                throw std::runtime_error(kami_vbd_last_error_string());
        } else {
            std::ofstream o(argv[5], std::ios::binary);
            o.write((const char*)hair->positions.data(), 4 * hair->positions.size());
            o.write((const char*)hair->velocities.data(), 4 * hair->velocities.size());
        }
        std::cout << s.GetInfoString().substr(0, 80) << std::endl;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
