// Scene ingest internals: OBJ/MTL meshes and the XML element tree.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace nomad {
namespace ingest {

// Material as encodeMaterial lays it out (Scene/Material.h:11-44), 20 floats, with the
// defaults of Material's member initialisers.
struct Mat {
  float v[20];
  Mat();
  float *diffuse() { return v + 0; }
  float &opacity() { return v[3]; }
  float *specular() { return v + 4; }
  float &shininess() { return v[7]; }
  float *emission() { return v + 8; }
  float &emission_power() { return v[11]; }
  float *transmission() { return v + 12; }
  float &ior() { return v[15]; }
  float &roughness() { return v[19]; }
};

// One OBJ file after parsing and triangulation, as the reference's CachedMesh holds it
// (Scene/SceneLoader.cpp:216-224): every `v` position, the triangles that index existing
// positions, per-triangle texture coordinates and material index (-1 none), and the converted
// materials of the MTL libraries.
struct Mesh {
  std::vector<float> vertices;     // 3 per position
  std::vector<uint32_t> tris;      // 3 per triangle
  std::vector<float> uvs;          // 6 per triangle
  std::vector<int32_t> triMat;     // 1 per triangle
  std::vector<Mat> materials;
  bool ok = false;                 // false: the file could not be read or parsed (no triangles)
  uint32_t invalidTris = 0;        // triangles dropped for out-of-range vertex indices
  std::string message;             // why `ok` is false
};

// Reads `path` with MTL libraries searched in `mtlDir` (the OBJ's directory with a trailing
// separator, or empty).
void load_obj(const std::string &path, const std::string &mtlDir, Mesh &out);

// tinyobjloader's decimal parser (tryParseDouble, vendored tiny_obj_loader.h:897-1028).
bool parse_obj_double(const char *s, const char *end, double *out);

// ---- XML ----

struct XmlAttr {
  std::string name, value;
};

struct XmlElem {
  std::string name;
  std::vector<XmlAttr> attrs;
  std::vector<XmlElem> children;
  const char *attr(const char *n) const;  // first attribute of that name, or null
};

// Parses a whole document; returns false with `err` set when it is not well formed. Top-level
// elements go to `roots` in document order.
bool parse_xml(const std::string &text, std::vector<XmlElem> &roots, std::string &err);

}  // namespace ingest
}  // namespace nomad
