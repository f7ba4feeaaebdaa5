// kami_io.cpp -- USC-HairSalon .data files, the hair format KamiSimulator reads and writes
// (importers/USCHairsalonImporter.cpp:56-80, exporters/USCHairsalonExporter.cpp:6-18):
// a little-endian uint32 strand count, then for each strand a uint32 vertex count followed by
// that many float (x, y, z) triples.
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "kami_vbd.h"
#include "vbd_host.h"

namespace {

struct FileCloser {
    void operator()(FILE* f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<FILE, FileCloser>;

kami_status io_fail(const std::string& msg) {
    kami::set_last_error(msg.c_str());
    return KAMI_ERR_IO;
}

// Reads the strand table (and, when xyz is given, the vertices) of a .data file.  max_verts > 0
// writes xyz padded to [strand][max_verts]; max_verts == 0 writes it packed in strand order.
kami_status read_usc(const char* path, std::vector<uint32_t>& counts, int32_t max_verts, float* xyz) {
    if (!path) return io_fail("null path");
    File f(std::fopen(path, "rb"));
    if (!f) return io_fail(std::string("cannot open ") + path);
    std::fseek(f.get(), 0, SEEK_END);
    const long size = std::ftell(f.get());
    std::fseek(f.get(), 0, SEEK_SET);
    uint32_t ns = 0;
    if (std::fread(&ns, 4, 1, f.get()) != 1) return io_fail(std::string(path) + ": no strand count");
    if ((int64_t)ns * 4 > (int64_t)size) return io_fail(std::string(path) + ": strand count exceeds the file");
    counts.assign(ns, 0);
    int64_t packed = 0;
    std::vector<float> buf;
    for (uint32_t s = 0; s < ns; s++) {
        uint32_t n = 0;
        if (std::fread(&n, 4, 1, f.get()) != 1)
            return io_fail(std::string(path) + ": truncated at strand " + std::to_string(s));
        const long here = std::ftell(f.get());
        if ((int64_t)n * 12 > (int64_t)(size - here))
            return io_fail(std::string(path) + ": strand " + std::to_string(s) + " runs past the end of the file");
        counts[s] = n;
        if (xyz) {
            if (max_verts > 0 && (int64_t)n > max_verts)
                return io_fail(std::string(path) + ": strand " + std::to_string(s) + " has " + std::to_string(n) +
                               " vertices, more than max_verts");
            float* dst = max_verts > 0 ? xyz + (int64_t)s * max_verts * 3 : xyz + packed * 3;
            if (n > 0 && std::fread(dst, 12, n, f.get()) != n)
                return io_fail(std::string(path) + ": truncated in strand " + std::to_string(s));
        } else if (n > 0 && std::fseek(f.get(), (long)n * 12, SEEK_CUR) != 0) {
            return io_fail(std::string(path) + ": truncated in strand " + std::to_string(s));
        }
        packed += n;
    }
    return KAMI_OK;
}

}  // namespace

extern "C" {

kami_status kami_usc_info(const char* path, int32_t* num_strands, int64_t* num_vertices, int32_t* max_strand_verts) {
    std::vector<uint32_t> counts;
    kami_status st = read_usc(path, counts, 0, nullptr);
    if (st != KAMI_OK) return st;
    int64_t nv = 0;
    uint32_t mx = 0;
    for (uint32_t c : counts) {
        nv += c;
        mx = c > mx ? c : mx;
    }
    if (counts.size() > (size_t)INT32_MAX) return io_fail("too many strands");
    if (num_strands) *num_strands = (int32_t)counts.size();
    if (num_vertices) *num_vertices = nv;
    if (max_strand_verts) *max_strand_verts = (int32_t)mx;
    return KAMI_OK;
}

kami_status kami_usc_read(const char* path, int32_t max_verts, int32_t* strand_vert_count, float* xyz) {
    if (!strand_vert_count || !xyz) {
        kami::set_last_error("null output array");
        return KAMI_ERR_INVALID_ARGUMENT;
    }
    if (max_verts < 0) {
        kami::set_last_error("max_verts must be >= 0");
        return KAMI_ERR_INVALID_ARGUMENT;
    }
    std::vector<uint32_t> counts;
    kami_status st = read_usc(path, counts, max_verts, xyz);
    if (st != KAMI_OK) return st;
    for (size_t s = 0; s < counts.size(); s++) strand_vert_count[s] = (int32_t)counts[s];
    return KAMI_OK;
}

kami_status kami_usc_write(const char* path, int32_t num_strands, const int32_t* strand_vert_count, int32_t max_verts,
                           const float* xyz) {
    if (!path || !strand_vert_count || (!xyz && num_strands > 0) || num_strands < 0 || max_verts < 0) {
        kami::set_last_error("bad arguments to kami_usc_write");
        return KAMI_ERR_INVALID_ARGUMENT;
    }
    for (int32_t s = 0; s < num_strands; s++)
        if (strand_vert_count[s] < 0 || (max_verts > 0 && strand_vert_count[s] > max_verts)) {
            kami::set_last_error("a strand vertex count is negative or exceeds max_verts");
            return KAMI_ERR_INVALID_ARGUMENT;
        }
    File f(std::fopen(path, "wb"));
    if (!f) return io_fail(std::string("cannot create ") + path);
    const uint32_t ns = (uint32_t)num_strands;
    bool ok = std::fwrite(&ns, 4, 1, f.get()) == 1;
    int64_t packed = 0;
    for (int32_t s = 0; s < num_strands && ok; s++) {
        const uint32_t n = (uint32_t)strand_vert_count[s];
        const float* src = max_verts > 0 ? xyz + (int64_t)s * max_verts * 3 : xyz + packed * 3;
        ok = std::fwrite(&n, 4, 1, f.get()) == 1 && (n == 0 || std::fwrite(src, 12, n, f.get()) == n);
        packed += n;
    }
    if (!ok || std::fflush(f.get()) != 0) return io_fail(std::string("cannot write ") + path);
    return KAMI_OK;
}

}  // extern "C"
