// ORACLE glue — test infrastructure only. Runs the reference's own scene pipeline
// (Scene::addObjectSilent, Scene::buildBVH and the create*Buffer packers, compiled here from
// the reference sources SceneBVH.cpp and Scene.cpp) on a scene description and hands the
// packed arrays back, so tests can compare this repository's builder against it.
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "Scene.h"
#include "SceneLoader.h"

namespace NomadPathTracer {
// The XML loader is not part of the checked path; Scene::clear() only calls ClearCache.
bool SceneLoader::LoadSceneFromXML(const std::string &, Scene *) { return false; }
void SceneLoader::ClearCache() {}
}  // namespace NomadPathTracer

using namespace NomadPathTracer;

namespace {
struct RefScene {
  std::vector<float> bvh, tlas, prims, mats;
  std::vector<int32_t> idx, roots;
};

simd::float3 f3(const float *p) { return simd::make_float3(p[0], p[1], p[2]); }
}  // namespace

extern "C" int ref_build_scene(uint32_t primCount, const int32_t *type, const float *geom,
                               const float *mat, uint32_t objCount, const uint32_t *first,
                               const uint32_t *count, void **out) {
  if (!out) return 1;
  Scene *scene = new Scene();
  for (uint32_t o = 0; o < objCount; ++o) {
    std::vector<Primitive> prims;
    prims.reserve(count[o]);
    for (uint32_t k = 0; k < count[o]; ++k) {
      uint32_t i = first[o] + k;
      alignas(Primitive) unsigned char storage[sizeof(Primitive)];
      std::memset(storage, 0, sizeof(storage));
      Primitive &p = *reinterpret_cast<Primitive *>(storage);
      const float *g = geom + 15ull * i;
      const float *m = mat + 20ull * i;
      Material mm;
      mm.diffuseColor = f3(m + 0);
      mm.opacity = m[3];
      mm.specularColor = f3(m + 4);
      mm.shininess = m[7];
      mm.emissionColor = f3(m + 8);
      mm.emissionPower = m[11];
      mm.transmissionColor = f3(m + 12);
      mm.indexOfRefraction = m[15];
      mm.diffuseTextureIndex = static_cast<int>(m[16]);
      mm.specularTextureIndex = static_cast<int>(m[17]);
      mm.normalTextureIndex = static_cast<int>(m[18]);
      mm.roughness = m[19];
      p.material = mm;
      p.type = static_cast<PrimitiveType>(type[i]);
      if (type[i] == 0) {
        p.sphere.center = f3(g);
        p.sphere.radius = g[3];
        p.sphere.supportsNormalMap = 0;
      } else if (type[i] == 2) {
        p.rectangle.center = f3(g);
        p.rectangle.u = f3(g + 3);
        p.rectangle.v = f3(g + 6);
        p.rectangle.tangent = simd::make_float3(1.0f, 0.0f, 0.0f);
        p.rectangle.bitangent = simd::make_float3(0.0f, 1.0f, 0.0f);
        p.rectangle.normal = simd::make_float3(0.0f, 0.0f, 1.0f);
        p.rectangle.supportsNormalMap = false;
      } else {
        p.triangle.v0 = f3(g);
        p.triangle.v1 = f3(g + 3);
        p.triangle.v2 = f3(g + 6);
        p.triangle.uv0 = simd::make_float2(g[9], g[10]);
        p.triangle.uv1 = simd::make_float2(g[11], g[12]);
        p.triangle.uv2 = simd::make_float2(g[13], g[14]);
        p.triangle.tangent = simd::make_float3(1.0f, 0.0f, 0.0f);
        p.triangle.bitangent = simd::make_float3(0.0f, 1.0f, 0.0f);
        p.triangle.normal = simd::make_float3(0.0f, 0.0f, 1.0f);
      }
      prims.push_back(p);
    }
    scene->addObjectSilent(prims);
  }
  scene->buildBVH();
  RefScene *r = new RefScene();
  size_t nb = scene->getBVHNodeCount();
  simd::float4 *b = scene->createBVHBuffer();
  for (size_t i = 0; i < 2 * nb; ++i) r->bvh.insert(r->bvh.end(), {b[i].x, b[i].y, b[i].z, b[i].w});
  delete[] b;
  size_t nt = 0;
  simd::float4 *t = scene->createTLASBuffer(nt);
  for (size_t i = 0; i < 2 * nt; ++i) r->tlas.insert(r->tlas.end(), {t[i].x, t[i].y, t[i].z, t[i].w});
  delete[] t;
  simd::float4 *pr = scene->createTransformsBuffer();
  for (size_t i = 0; i < 7ull * primCount; ++i)
    r->prims.insert(r->prims.end(), {pr[i].x, pr[i].y, pr[i].z, pr[i].w});
  delete[] pr;
  simd::float4 *ma = scene->createMaterialsBuffer();
  for (size_t i = 0; i < 5ull * primCount; ++i)
    r->mats.insert(r->mats.end(), {ma[i].x, ma[i].y, ma[i].z, ma[i].w});
  delete[] ma;
  int *ix = scene->createPrimitiveIndexBuffer();
  r->idx.assign(ix, ix + primCount);
  delete[] ix;
  for (const auto &obj : scene->getObjects()) r->roots.push_back(obj.blasRootIndex);
  delete scene;
  *out = r;
  return 0;
}

extern "C" void ref_scene_counts(void *h, uint32_t *out) {
  RefScene *r = static_cast<RefScene *>(h);
  out[0] = static_cast<uint32_t>(r->bvh.size() / 8);
  out[1] = static_cast<uint32_t>(r->tlas.size() / 8);
  out[2] = static_cast<uint32_t>(r->idx.size());
  out[3] = static_cast<uint32_t>(r->roots.size());
}

extern "C" void ref_scene_arrays(void *h, float *bvh, float *tlas, float *prims, float *mats,
                                 int32_t *idx, int32_t *roots) {
  RefScene *r = static_cast<RefScene *>(h);
  std::memcpy(bvh, r->bvh.data(), r->bvh.size() * 4);
  std::memcpy(tlas, r->tlas.data(), r->tlas.size() * 4);
  std::memcpy(prims, r->prims.data(), r->prims.size() * 4);
  std::memcpy(mats, r->mats.data(), r->mats.size() * 4);
  std::memcpy(idx, r->idx.data(), r->idx.size() * 4);
  std::memcpy(roots, r->roots.data(), r->roots.size() * 4);
}

extern "C" void ref_scene_free(void *h) { delete static_cast<RefScene *>(h); }
