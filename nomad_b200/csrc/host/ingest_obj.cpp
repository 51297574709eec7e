// OBJ / MTL reading for scene ingest.
//
// The reference reads meshes with the vendored tinyobjloader 2.0 (Nomad Path Tracer/
// tiny_obj_loader.h, called from Scene/SceneLoader.cpp:228-341 with triangulation on) and then
// keeps only the triangles whose vertex indices exist. This file restates the parts of that
// pipeline that decide the triangles, their texture coordinates and their materials, line for
// line in behaviour:
//   - line splitting on \n, \r\n and \r (safeGetline, tiny_obj_loader.h:767-799);
//   - the decimal parser tryParseDouble (:897-1028): digits accumulated in a double, fraction
//     digits scaled by 10^-k, the exponent applied as ldexp(m * 5^e, e); a token that does not
//     parse leaves the field's default;
//   - index fixing (fixIndex :819-852): 1-based, negative = relative to the elements read so far,
//     a zero or out-of-range relative vertex index fails the whole file;
//   - faces flushed to the output at `usemtl` changes, `g`, `o` and end of file with the material
//     current then (:2833-2861, :2931-3004, :3096-3102), so triangles keep file order;
//   - triangulation (exportGroupsToShape :1482-2004): quads split on the shorter diagonal,
//     larger polygons ear-clipped in the plane of the two dominant axes of the first
//     non-degenerate corner, with the point-in-triangle test of W. R. Franklin's pnpoly;
//   - MTL parsing (LoadMtl :2069-2468) of the fields the reference's material conversion reads,
//     first definition of a name wins, the last material always kept;
//   - the reference's material conversion (MaterialUtils::ConvertTinyMaterial,
//     Scene/MaterialUtils.cpp:144-190) with no texture decoded.
// Arithmetic is FP32 where tinyobjloader uses real_t = float, each operation rounded
// separately (the library is built without contraction), so the triangulation decisions match.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <limits>
#include <map>
#include <set>
#include <sstream>

#include "ingest.h"

namespace nomad {
namespace ingest {

Mat::Mat() {
  const float d[20] = {0.8f, 0.8f, 0.8f, 1.0f,   0.04f, 0.04f, 0.04f, 32.0f, 0.0f,  0.0f,
                       0.0f, 0.0f, 0.0f, 0.0f,   0.0f,  1.0f,  -1.0f, -1.0f, -1.0f, 0.5f};
  std::memcpy(v, d, sizeof(d));
}

namespace {

inline bool is_space(char c) { return c == ' ' || c == '\t'; }
inline bool is_digit(char c) { return static_cast<unsigned>(c - '0') < 10u; }
inline bool is_newline(char c) { return c == '\r' || c == '\n' || c == '\0'; }

float luminance(const float *c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; }
float clamp01(float x) { return std::clamp(x, 0.0f, 1.0f); }

// parseReal: skip blanks, parse up to the next blank, keep `def` when it does not parse.
float parse_real(const char **t, double def = 0.0) {
  *t += std::strspn(*t, " \t");
  const char *end = *t + std::strcspn(*t, " \t\r");
  double val = def;
  parse_obj_double(*t, end, &val);
  *t = end;
  return static_cast<float>(val);
}

int parse_int(const char **t) {
  *t += std::strspn(*t, " \t");
  const int i = std::atoi(*t);
  *t += std::strcspn(*t, " \t\r");
  return i;
}

std::string parse_string(const char **t) {
  *t += std::strspn(*t, " \t");
  const size_t e = std::strcspn(*t, " \t\r");
  std::string s(*t, *t + e);
  *t += e;
  return s;
}

struct VIdx {
  int v = -1, vt = -1, vn = -1;
};

bool fix_index(int idx, int n, int *ret, bool allowZero) {
  if (idx > 0) {
    *ret = idx - 1;
    return true;
  }
  if (idx == 0) {
    *ret = -1;
    return allowZero;
  }
  *ret = n + idx;
  return *ret >= 0;
}

// i, i/j, i//k, i/j/k
bool parse_triple(const char **t, int vsize, int vnsize, int vtsize, VIdx *out) {
  VIdx vi;
  if (!fix_index(std::atoi(*t), vsize, &vi.v, false)) return false;
  *t += std::strcspn(*t, "/ \t\r");
  if ((*t)[0] != '/') {
    *out = vi;
    return true;
  }
  ++*t;
  if ((*t)[0] == '/') {
    ++*t;
    if (!fix_index(std::atoi(*t), vnsize, &vi.vn, true)) return false;
    *t += std::strcspn(*t, "/ \t\r");
    *out = vi;
    return true;
  }
  if (!fix_index(std::atoi(*t), vtsize, &vi.vt, true)) return false;
  *t += std::strcspn(*t, "/ \t\r");
  if ((*t)[0] != '/') {
    *out = vi;
    return true;
  }
  ++*t;
  if (!fix_index(std::atoi(*t), vnsize, &vi.vn, true)) return false;
  *t += std::strcspn(*t, "/ \t\r");
  *out = vi;
  return true;
}

// Point in triangle, W. Randolph Franklin's crossing test.
bool pnpoly3(const float *vx, const float *vy, float tx, float ty) {
  bool c = false;
  for (int i = 0, j = 2; i < 3; j = i++) {
    if (((vy[i] > ty) != (vy[j] > ty)) && (tx < (vx[j] - vx[i]) * (ty - vy[i]) / (vy[j] - vy[i]) + vx[i]))
      c = !c;
  }
  return c;
}

// The text of a file split into lines the way safeGetline does: "\n", "\r\n" and "\r" end a
// line; a last line without an ending still counts.
template <class F>
void for_each_line(const std::string &text, F &&fn) {
  std::string line;
  size_t i = 0, n = text.size();
  while (i < n) {
    size_t j = i;
    while (j < n && text[j] != '\n' && text[j] != '\r') ++j;
    line.assign(text, i, j - i);
    if (j < n && text[j] == '\r' && j + 1 < n && text[j + 1] == '\n') ++j;
    i = j + 1;
    if (!fn(line)) return;
  }
}

bool read_file(const std::string &path, std::string &out) {
  std::ifstream f(path.c_str(), std::ios::binary);
  if (!f) return false;
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

// The MTL fields the material conversion reads (tinyobj::material_t subset).
struct MtlMat {
  std::string name;
  float diffuse[3], specular[3], transmittance[3], emission[3];
  float shininess, ior, dissolve, roughness;
  void init() {
    name.clear();
    for (int i = 0; i < 3; ++i) diffuse[i] = specular[i] = transmittance[i] = emission[i] = 0.0f;
    shininess = 1.0f;
    ior = 1.0f;
    dissolve = 1.0f;
    roughness = 0.0f;
  }
};

void parse3(const char **t, float *o) {
  o[0] = parse_real(t);
  o[1] = parse_real(t);
  o[2] = parse_real(t);
}

void load_mtl(const std::string &text, std::map<std::string, int> &map, std::vector<MtlMat> &mats) {
  MtlMat m;
  m.init();
  bool hasD = false, hasKd = false;
  for_each_line(text, [&](std::string &line) {
    if (!line.empty()) {
      const size_t last = line.find_last_not_of(" \t");
      line.resize(last == std::string::npos ? 0 : last + 1);
    }
    if (line.empty()) return true;
    const char *t = line.c_str();
    t += std::strspn(t, " \t");
    if (t[0] == '\0' || t[0] == '#') return true;
    if (std::strncmp(t, "newmtl", 6) == 0 && is_space(t[6])) {
      if (!m.name.empty()) {
        map.insert(std::make_pair(m.name, static_cast<int>(mats.size())));
        mats.push_back(m);
      }
      m.init();
      hasD = hasKd = false;
      t += 7;
      m.name = parse_string(&t);
      return true;
    }
    if (t[0] == 'K' && t[1] == 'a' && is_space(t[2])) return true;
    if (t[0] == 'K' && t[1] == 'd' && is_space(t[2])) {
      t += 2;
      parse3(&t, m.diffuse);
      hasKd = true;
      return true;
    }
    if (t[0] == 'K' && t[1] == 's' && is_space(t[2])) {
      t += 2;
      parse3(&t, m.specular);
      return true;
    }
    if ((t[0] == 'K' && t[1] == 't' && is_space(t[2])) || (t[0] == 'T' && t[1] == 'f' && is_space(t[2]))) {
      t += 2;
      parse3(&t, m.transmittance);
      return true;
    }
    if (t[0] == 'N' && t[1] == 'i' && is_space(t[2])) {
      t += 2;
      m.ior = parse_real(&t);
      return true;
    }
    if (t[0] == 'K' && t[1] == 'e' && is_space(t[2])) {
      t += 2;
      parse3(&t, m.emission);
      return true;
    }
    if (t[0] == 'N' && t[1] == 's' && is_space(t[2])) {
      t += 2;
      m.shininess = parse_real(&t);
      return true;
    }
    if (std::strncmp(t, "illum", 5) == 0 && is_space(t[5])) return true;
    if (t[0] == 'd' && is_space(t[1])) {
      t += 1;
      m.dissolve = parse_real(&t);
      hasD = true;
      return true;
    }
    if (t[0] == 'T' && t[1] == 'r' && is_space(t[2])) {
      t += 2;
      if (!hasD) m.dissolve = 1.0f - parse_real(&t);
      return true;
    }
    if (t[0] == 'P' && t[1] == 'r' && is_space(t[2])) {
      t += 2;
      m.roughness = parse_real(&t);
      return true;
    }
    // Pm Ps Pc Pcr aniso anisor map_Ka: not read by the conversion
    if (std::strncmp(t, "map_Kd", 6) == 0 && is_space(t[6])) {
      if (!hasKd) m.diffuse[0] = m.diffuse[1] = m.diffuse[2] = 0.6f;
      return true;
    }
    return true;  // other texture maps and unknown parameters
  });
  map.insert(std::make_pair(m.name, static_cast<int>(mats.size())));
  mats.push_back(m);
}

// MaterialFileReader: the base directory may list several directories separated by ':'.
bool read_mtl(const std::string &baseDir, const std::string &id, std::map<std::string, int> &map,
              std::vector<MtlMat> &mats) {
  std::string text;
  if (!baseDir.empty()) {
    std::istringstream f(baseDir);
    std::string dir;
    while (std::getline(f, dir, ':')) {
      std::string p = dir.empty() ? id : (dir.back() != '/' ? dir + "/" + id : dir + id);
      if (read_file(p, text)) {
        load_mtl(text, map, mats);
        return true;
      }
    }
    return false;
  }
  if (!read_file(id, text)) return false;
  load_mtl(text, map, mats);
  return true;
}

// SplitString(s, ' ', '\\'): backslash escapes the next character; the last token is always kept.
std::vector<std::string> split_names(const std::string &s) {
  std::vector<std::string> out;
  std::string tok;
  bool esc = false;
  for (char ch : s) {
    if (esc) {
      esc = false;
    } else if (ch == '\\') {
      esc = true;
      continue;
    } else if (ch == ' ') {
      if (!tok.empty()) out.push_back(tok);
      tok.clear();
      continue;
    }
    tok += ch;
  }
  out.push_back(tok);
  return out;
}

Mat convert(const MtlMat &s) {
  Mat m;
  for (int i = 0; i < 3; ++i) {
    m.diffuse()[i] = s.diffuse[i];
    m.specular()[i] = s.specular[i];
    m.transmission()[i] = s.transmittance[i];
    m.emission()[i] = s.emission[i];
  }
  m.emission_power() = luminance(m.emission()) > 0.0f ? 1.0f : 0.0f;
  m.shininess() = s.shininess;
  m.ior() = s.ior != 0.0f ? s.ior : 1.0f;
  m.opacity() = clamp01(s.dissolve);
  float r;
  if (s.roughness > 0.0f)
    r = clamp01(s.roughness);
  else if (m.shininess() <= 0.0f)
    r = 1.0f;
  else
    r = clamp01(std::sqrt(2.0f / (m.shininess() + 2.0f)));
  m.roughness() = r;
  if (luminance(m.transmission()) <= 0.0f && m.opacity() < 1.0f) {
    const float tr = 1.0f - m.opacity();
    m.transmission()[0] = m.transmission()[1] = m.transmission()[2] = tr;
  }
  return m;  // texture indices stay -1: no image is decoded
}

struct Corner {
  VIdx i;
};

struct Parser {
  std::vector<float> v;   // positions
  std::vector<float> vt;  // texture coordinates
  size_t vnCount = 0;
  std::vector<std::vector<VIdx>> faces;  // pending faces
  int material = -1;
  // output triangles: corners and material
  std::vector<VIdx> triCorners;
  std::vector<int32_t> triMaterial;

  void emit(const VIdx &a, const VIdx &b, const VIdx &c) {
    triCorners.push_back(a);
    triCorners.push_back(b);
    triCorners.push_back(c);
    triMaterial.push_back(material);
  }

  void flush() {
    for (const auto &face : faces) triangulate(face);
    faces.clear();
  }

  void triangulate(const std::vector<VIdx> &face) {
    const size_t n = face.size();
    if (n < 3) return;
    if (n == 3) {
      emit(face[0], face[1], face[2]);
      return;
    }
    const size_t vs = v.size();
    if (n == 4) {
      const size_t i0 = face[0].v, i1 = face[1].v, i2 = face[2].v, i3 = face[3].v;
      if (3 * i0 + 2 >= vs || 3 * i1 + 2 >= vs || 3 * i2 + 2 >= vs || 3 * i3 + 2 >= vs) return;
      const float e02x = v[i2 * 3] - v[i0 * 3], e02y = v[i2 * 3 + 1] - v[i0 * 3 + 1],
                  e02z = v[i2 * 3 + 2] - v[i0 * 3 + 2];
      const float e13x = v[i3 * 3] - v[i1 * 3], e13y = v[i3 * 3 + 1] - v[i1 * 3 + 1],
                  e13z = v[i3 * 3 + 2] - v[i1 * 3 + 2];
      const float s02 = e02x * e02x + e02y * e02y + e02z * e02z;
      const float s13 = e13x * e13x + e13y * e13y + e13z * e13z;
      if (s02 < s13) {
        emit(face[0], face[1], face[2]);
        emit(face[0], face[2], face[3]);
      } else {
        emit(face[0], face[1], face[3]);
        emit(face[1], face[2], face[3]);
      }
      return;
    }
    // Projection plane: the two dominant axes of the first corner with a non-degenerate cross
    // product.
    size_t axes[2] = {1, 2};
    for (size_t k = 0; k < n; ++k) {
      const size_t a = face[k % n].v, b = face[(k + 1) % n].v, c = face[(k + 2) % n].v;
      if (3 * a + 2 >= vs || 3 * b + 2 >= vs || 3 * c + 2 >= vs) continue;
      const float e0x = v[b * 3] - v[a * 3], e0y = v[b * 3 + 1] - v[a * 3 + 1], e0z = v[b * 3 + 2] - v[a * 3 + 2];
      const float e1x = v[c * 3] - v[b * 3], e1y = v[c * 3 + 1] - v[b * 3 + 1], e1z = v[c * 3 + 2] - v[b * 3 + 2];
      const float cx = std::fabs(e0y * e1z - e0z * e1y);
      const float cy = std::fabs(e0z * e1x - e0x * e1z);
      const float cz = std::fabs(e0x * e1y - e0y * e1x);
      const float eps = std::numeric_limits<float>::epsilon();
      if (cx > eps || cy > eps || cz > eps) {
        if (!(cx > cy && cx > cz)) {
          axes[0] = 0;
          if (cz > cx && cz > cy) axes[1] = 1;
        }
        break;
      }
    }
    std::vector<VIdx> rem = face;
    size_t guess = 0, iterations = n, previous = n;
    VIdx ind[3];
    float vx[3], vy[3];
    while (rem.size() > 3 && iterations > 0) {
      const size_t np = rem.size();
      if (guess >= np) guess -= np;
      if (previous != np) {
        previous = np;
        iterations = np;
      } else {
        --iterations;
      }
      for (size_t k = 0; k < 3; ++k) {
        ind[k] = rem[(guess + k) % np];
        const size_t vi = ind[k].v;
        if (vi * 3 + axes[0] >= vs || vi * 3 + axes[1] >= vs) {
          vx[k] = vy[k] = 0.0f;
        } else {
          vx[k] = v[vi * 3 + axes[0]];
          vy[k] = v[vi * 3 + axes[1]];
        }
      }
      const float e0x = vx[1] - vx[0], e0y = vy[1] - vy[0], e1x = vx[2] - vx[1], e1y = vy[2] - vy[1];
      const float cross = e0x * e1y - e0y * e1x;
      const float area = (vx[0] * vy[1] - vy[0] * vx[1]) * 0.5f;
      if (cross * area < 0.0f) {
        ++guess;
        continue;
      }
      bool overlap = false;
      for (size_t o = 3; o < np; ++o) {
        const size_t ovi = rem[(guess + o) % np].v;
        if (ovi * 3 + axes[0] >= vs || ovi * 3 + axes[1] >= vs) continue;
        if (pnpoly3(vx, vy, v[ovi * 3 + axes[0]], v[ovi * 3 + axes[1]])) {
          overlap = true;
          break;
        }
      }
      if (overlap) {
        ++guess;
        continue;
      }
      emit(ind[0], ind[1], ind[2]);
      rem.erase(rem.begin() + static_cast<std::ptrdiff_t>((guess + 1) % np));
    }
    if (rem.size() == 3) emit(rem[0], rem[1], rem[2]);
  }
};

}  // namespace

bool parse_obj_double(const char *s, const char *end, double *result) {
  if (s >= end) return false;
  double mantissa = 0.0;
  int exponent = 0;
  char sign = '+', expSign = '+';
  const char *c = s;
  int read = 0;
  bool more = false, leadingDot = false;
  if (*c == '+' || *c == '-') {
    sign = *c;
    ++c;
    if (c != end && *c == '.') leadingDot = true;
  } else if (is_digit(*c)) {
  } else if (*c == '.') {
    leadingDot = true;
  } else {
    return false;
  }
  more = (c != end);
  if (!leadingDot) {
    while (more && is_digit(*c)) {
      mantissa *= 10;
      mantissa += static_cast<int>(*c - '0');
      ++c;
      ++read;
      more = (c != end);
    }
    if (read == 0) return false;
  }
  if (more) {
    bool expPart = false;
    if (*c == '.') {
      ++c;
      read = 1;
      more = (c != end);
      static const double kTenths[] = {1.0, 0.1, 0.01, 0.001, 0.0001, 0.00001, 0.000001, 0.0000001};
      while (more && is_digit(*c)) {
        mantissa += static_cast<int>(*c - '0') * (read < 8 ? kTenths[read] : std::pow(10.0, -read));
        ++read;
        ++c;
        more = (c != end);
      }
      expPart = more;
    } else if (*c == 'e' || *c == 'E') {
      expPart = true;
    }
    if (expPart && (*c == 'e' || *c == 'E')) {
      ++c;
      more = (c != end);
      if (more && (*c == '+' || *c == '-')) {
        expSign = *c;
        ++c;
      } else if (is_digit(*c)) {
      } else {
        return false;
      }
      read = 0;
      more = (c != end);
      while (more && is_digit(*c)) {
        if (exponent > 2147483647 / 10) return false;
        exponent *= 10;
        exponent += static_cast<int>(*c - '0');
        ++c;
        ++read;
        more = (c != end);
      }
      exponent *= (expSign == '+' ? 1 : -1);
      if (read == 0) return false;
    }
  }
  *result = (sign == '+' ? 1 : -1) * (exponent ? std::ldexp(mantissa * std::pow(5.0, exponent), exponent) : mantissa);
  return true;
}

void load_obj(const std::string &path, const std::string &mtlDir, Mesh &out) {
  out = Mesh();
  std::string text;
  if (!read_file(path, text)) {
    out.message = "cannot open file [" + path + "]";
    return;
  }
  Parser P;
  std::map<std::string, int> matMap;
  std::vector<MtlMat> mats;
  std::set<std::string> mtlFiles;
  bool failed = false;
  std::string baseDir = mtlDir;
  if (!baseDir.empty() && baseDir.back() != '/') baseDir += '/';

  for_each_line(text, [&](const std::string &line) {
    if (line.empty()) return true;
    const char *t = line.c_str();
    t += std::strspn(t, " \t");
    if (t[0] == '\0' || t[0] == '#') return true;
    const int vsize = static_cast<int>(P.v.size() / 3), vnsize = static_cast<int>(P.vnCount),
              vtsize = static_cast<int>(P.vt.size() / 2);
    if (t[0] == 'v' && is_space(t[1])) {
      t += 2;
      const float x = parse_real(&t), y = parse_real(&t), z = parse_real(&t);
      P.v.push_back(x);
      P.v.push_back(y);
      P.v.push_back(z);
      return true;
    }
    if (t[0] == 'v' && t[1] == 'n' && is_space(t[2])) {
      ++P.vnCount;
      return true;
    }
    if (t[0] == 'v' && t[1] == 't' && is_space(t[2])) {
      t += 3;
      const float x = parse_real(&t), y = parse_real(&t);
      P.vt.push_back(x);
      P.vt.push_back(y);
      return true;
    }
    if (t[0] == 'v' && t[1] == 'w' && is_space(t[2])) {
      t += 3;
      parse_int(&t);
      while (!is_newline(t[0]) && t[0] != '#') {
        const float j = parse_real(&t, -1.0);
        parse_real(&t, 0.0);
        if (j < 0.0f) {
          failed = true;
          out.message = "negative joint id in a `vw` line";
          return false;
        }
        t += std::strspn(t, " \t\r");
      }
      return true;
    }
    const bool isL = t[0] == 'l' && is_space(t[1]), isP = t[0] == 'p' && is_space(t[1]),
               isF = t[0] == 'f' && is_space(t[1]);
    if (isL || isP || isF) {
      t += 2;
      if (isF) t += std::strspn(t, " \t");
      std::vector<VIdx> face;
      while (!is_newline(t[0]) && t[0] != '#') {
        VIdx vi;
        if (!parse_triple(&t, vsize, vnsize, vtsize, &vi)) {
          failed = true;
          out.message = "bad index in an `" + std::string(1, isF ? 'f' : (isL ? 'l' : 'p')) + "` line";
          return false;
        }
        if (isF) face.push_back(vi);
        t += std::strspn(t, " \t\r");
      }
      if (isF) P.faces.push_back(std::move(face));
      return true;
    }
    if (std::strncmp(t, "usemtl", 6) == 0) {
      t += 6;
      const std::string name = parse_string(&t);
      auto it = matMap.find(name);
      const int id = it != matMap.end() ? it->second : -1;
      if (id != P.material) {
        P.flush();
        P.material = id;
      }
      return true;
    }
    if (std::strncmp(t, "mtllib", 6) == 0 && is_space(t[6])) {
      t += 7;
      for (const std::string &f : split_names(std::string(t))) {
        if (mtlFiles.count(f)) continue;
        if (read_mtl(baseDir, f, matMap, mats)) {
          mtlFiles.insert(f);
          break;
        }
      }
      return true;
    }
    if ((t[0] == 'g' || t[0] == 'o') && is_space(t[1])) {
      P.flush();
      return true;
    }
    return true;  // s, t and anything else do not change the triangles
  });
  if (failed) return;  // the reference keeps nothing of a file that fails to parse
  P.flush();

  out.vertices.swap(P.v);
  out.materials.reserve(mats.size());
  for (const MtlMat &m : mats) out.materials.push_back(convert(m));
  const size_t nv = out.vertices.size() / 3, ntri = P.triMaterial.size();
  out.tris.reserve(ntri * 3);
  out.uvs.reserve(ntri * 6);
  out.triMat.reserve(ntri);
  for (size_t f = 0; f < ntri; ++f) {
    const VIdx *c = &P.triCorners[3 * f];
    if (static_cast<size_t>(c[0].v) >= nv || static_cast<size_t>(c[1].v) >= nv ||
        static_cast<size_t>(c[2].v) >= nv) {
      ++out.invalidTris;
      continue;
    }
    for (int k = 0; k < 3; ++k) out.tris.push_back(static_cast<uint32_t>(c[k].v));
    for (int k = 0; k < 3; ++k) {
      const int ti = c[k].vt;
      if (ti >= 0 && static_cast<size_t>(ti * 2 + 1) < P.vt.size()) {
        out.uvs.push_back(P.vt[ti * 2]);
        out.uvs.push_back(P.vt[ti * 2 + 1]);
      } else {
        out.uvs.push_back(0.0f);
        out.uvs.push_back(0.0f);
      }
    }
    const int m = P.triMaterial[f];
    out.triMat.push_back(m >= 0 && static_cast<size_t>(m) < out.materials.size() ? m : -1);
  }
  out.ok = true;
}

}  // namespace ingest
}  // namespace nomad
