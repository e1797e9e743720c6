// scene_io.h — host-only snapshot file format and scene builders.
#pragma once

#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/wcsph.h"

namespace wcsph_host {

constexpr uint32_t kSnapshotVersion = 1;  // Snapshot::VERSION (snapshot.cuh:19)
constexpr size_t kAppNameMax = 64;        // Snapshot::APP_NAME_MAX (snapshot.cuh:20)

struct Status {
    int code = WCSPH_OK;
    std::string message;
    bool ok() const { return code == WCSPH_OK; }
};

Status snapshot_read_header(const std::string& path, std::string* app_name, uint32_t* fluid_n,
                            std::ifstream* keep_open = nullptr);
Status snapshot_read(const std::string& path, const std::string& app_name, uint32_t fluid_n, float* pos, float* vel);
Status snapshot_write(const std::string& path, const std::string& app_name, uint32_t fluid_n, const float* pos,
                      const float* vel);

void make_lattice(const float origin[3], const uint32_t dims[3], float r, float jitter, uint64_t seed, float* out);
void make_velocities(uint32_t n, float sigma, uint64_t seed, float* out);
uint32_t sample_box_walls(const float mn[3], const float mx[3], float spacing, float* out);
uint32_t sample_triangles(const float* verts, uint32_t ntri, float voxel, float* out);
std::vector<float> icosphere_triangles(const float center[3], float radius, int level);
// Triangles (9 floats each) of the first shape of a Wavefront .obj file,
// optionally normalised, then transformed by a column-major model matrix
// (NULL = identity). Fills *status on failure and returns no triangles.
std::vector<float> load_obj_triangles(const std::string& path, bool normalize, const float* model, Status* status);

}  // namespace wcsph_host
