// Wavefront OBJ ingest for the scene loader (WavefrontObjMesh,
// src/mesh/WavefrontObjMesh.cpp:10-152): the same result as the reference's
// line-by-line reader -- positions transformed by toWorld, normals by the
// inverse transpose and normalised, quads split (v1,v2,v3) (v4,v1,v3),
// vertices de-duplicated on their (position, texcoord, normal) index triple
// in order of first use -- parsed in parallel over line-aligned chunks of the
// file held in memory.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hikari {

struct ObjMesh {
    std::vector<float> pos;      // 3 per vertex, world space
    std::vector<float> nrm;      // 3 per vertex, or empty
    std::vector<float> uv;       // 2 per vertex, or empty
    std::vector<uint32_t> idx;   // 3 per triangle
};

// M: toWorld row-major 4x4; Minv its inverse (normals use its transpose).
// Throws std::runtime_error with the reference's messages on malformed input.
ObjMesh load_obj(const std::string &path, const float *M, const float *Minv, int threads = 0);

// Inverse of a row-major 4x4 (Gauss-Jordan in double); false when singular.
bool invert4(const float *m, float *out);

}  // namespace hikari
