// ORACLE -- test infrastructure only. Not part of the product library.
//
// extern "C" surface of the CPU oracle, loaded by tests/ (and by bench.py's
// CPU-baseline leg) through ctypes. It takes the same descriptor structs as
// the product ABI (include/mini_raytrace.h) so a test builds one scene and
// hands it to both sides.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "oracle_trace.hpp"

using namespace orc;

namespace {

struct OracleScene {
    Scene scene;
    std::unique_ptr<Packed> packed;
    Globals globals{};
    int bruteForce = 0;  // 1: brute force with the reference test, 2: with the watertight test
    bool allLeafInstances = false;  // Tracer::allLeafInstances
};

template <class Fn>
void parallelFor(uint32_t n, int threads, Fn fn) {
    if (threads <= 1 || n < 2) {
        for (uint32_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    const uint32_t chunk = 16;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            for (;;) {
                const uint32_t b = next.fetch_add(chunk);
                if (b >= n) break;
                const uint32_t e = std::min(n, b + chunk);
                for (uint32_t i = b; i < e; ++i) fn(i);
            }
        });
    for (auto& th : pool) th.join();
}

struct RayIn {
    float o[3];
    float tMax;
    float d[3];
    float pad;
};
struct HitOut {  // same layout as mrtxHit
    float t;
    uint32_t instance, prim, hit;
    float u, v;
    uint32_t pad[2];
};

}  // namespace

extern "C" {

void* orc_create() { return new OracleScene(); }
void orc_destroy(void* s) { delete static_cast<OracleScene*>(s); }

uint32_t orc_add_mesh(void* s, const mrtMeshDesc* d) { return static_cast<OracleScene*>(s)->scene.addMesh(*d); }
uint32_t orc_add_instance(void* s, uint32_t mesh, const float* xf, uint32_t mat) {
    return static_cast<OracleScene*>(s)->scene.addInstance(mesh, xf, mat);
}
uint32_t orc_add_material(void* s, const mrtMaterialDesc* d) {
    return static_cast<OracleScene*>(s)->scene.addMaterial(*d);
}
uint32_t orc_add_texture(void* s, const mrtTextureDesc* d) {
    return static_cast<OracleScene*>(s)->scene.addTexture(*d);
}
void orc_remove_texture(void* s, uint32_t id) { static_cast<OracleScene*>(s)->scene.removeTexture(id); }
uint32_t orc_add_light(void* s, const mrtLightDesc* d) { return static_cast<OracleScene*>(s)->scene.addLight(*d); }
void orc_set_environment(void* s, const mrtTextureDesc* d, float rot, float inten) {
    static_cast<OracleScene*>(s)->scene.setEnvironment(d, rot, inten);
}
void orc_set_camera(void* s, const mrtCameraDesc* d) {
    auto* o = static_cast<OracleScene*>(s);
    o->scene.cam = *d;
    o->scene.useCameraEx = false;
}
void orc_set_camera_ex(void* s, const mrtCameraDescEx* d) {
    auto* o = static_cast<OracleScene*>(s);
    o->scene.camEx = *d;
    o->scene.useCameraEx = true;
}
void orc_set_settings(void* s, const mrtRenderSettings* d) {
    Settings& st = static_cast<OracleScene*>(s)->scene.settings;
    st.width = d->width;
    st.height = d->height;
    st.maxBounces = d->maxBounces;
    st.sppLimit = d->sppLimit;
    st.exposureEV = d->exposureEV;
    st.fireflyClamp = d->fireflyClamp;
    st.tonemap = d->tonemap;
}

// Diagnostic switch: closest-hit rays of orc_render_f32_sum64 test every
// triangle instead of walking the BVH.
void orc_set_bruteforce(void* s, int mode) { static_cast<OracleScene*>(s)->bruteForce = mode; }

// 1: walk every instance of a TLAS leaf; 0 (default): only its first, as the
// reference shaders do (intersect.glsl:116-121, 150-152).
void orc_set_all_leaf_instances(void* s, int on) { static_cast<OracleScene*>(s)->allLeafInstances = on != 0; }

// After orc_commit: how many instances the reference traversal never enters
// (those after the first of a multi-instance TLAS leaf, Bvh.cpp:104).
uint32_t orc_unwalked_instances(void* s) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return 0;
    const Packed& P = *o->packed;
    uint32_t n = 0;
    for (size_t i = P.tlasRoot; i < P.nodes.size(); ++i) {
        const uint32_t count = P.nodes[i].packed >> 2;
        if (count > 1) n += count - 1;
    }
    return n;
}

// Pack the scene (BVH builds, CDF). Returns the number of BVH nodes.
uint32_t orc_commit(void* s) {
    auto* o = static_cast<OracleScene*>(s);
    o->packed = std::make_unique<Packed>(pack(o->scene));
    o->globals = makeGlobals(o->scene, *o->packed);
    return uint32_t(o->packed->nodes.size());
}

// Reference-order FP32 accumulation (pathtrace.comp:227-228) of frames
// [frame0, frame0 + nframes) over pixels `pixels` (NULL = all, row-major).
// accum holds 4 floats per listed pixel; frame 0 overwrites, others add.
// rayCounts (may be NULL) receives closest-hit and shadow ray totals.
int orc_render_f32(void* s, const uint32_t* pixels, uint32_t npix, uint32_t frame0, uint32_t nframes,
                   float* accum, int threads) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return -1;
    const Globals& g = o->globals;
    const uint32_t total = pixels ? npix : g.width * g.height;
    Tracer<float> tr{*o->packed, g};
    tr.allLeafInstances = o->allLeafInstances;
    tr.bruteForce = o->bruteForce != 0;
    tr.watertight = o->bruteForce == 2;
    parallelFor(total, threads, [&](uint32_t i) {
        const uint32_t p = pixels ? pixels[i] : i;
        const uint32_t px = p % g.width, py = p / g.width;
        float* a = accum + size_t(i) * 4;
        for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
            const V3<float> L = tr.tracePath(px, py, f);
            if (f == 0) {
                a[0] = 0.0f; a[1] = 0.0f; a[2] = 0.0f; a[3] = 0.0f;
            }
            a[0] = a[0] + L.x;
            a[1] = a[1] + L.y;
            a[2] = a[2] + L.z;
            a[3] = a[3] + 1.0f;
        }
    });
    return 0;
}

// FP32 paths (as orc_render_f32) summed in double in sample order:
// sums[3*i..] += double(L). This is the accumulation the GPU engine keeps, so
// its FP64 buffer can be compared bit for bit.
int orc_render_f32_sum64(void* s, const uint32_t* pixels, uint32_t npix, uint32_t frame0, uint32_t nframes,
                         double* sums, int threads) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return -1;
    const Globals& g = o->globals;
    const uint32_t total = pixels ? npix : g.width * g.height;
    Tracer<float> tr{*o->packed, g};
    tr.allLeafInstances = o->allLeafInstances;
    tr.bruteForce = o->bruteForce != 0;
    tr.watertight = o->bruteForce == 2;
    parallelFor(total, threads, [&](uint32_t i) {
        const uint32_t p = pixels ? pixels[i] : i;
        const uint32_t px = p % g.width, py = p / g.width;
        double* a = sums + size_t(i) * 3;
        for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
            const V3<float> L = tr.tracePath(px, py, f);
            a[0] += double(L.x);
            a[1] += double(L.y);
            a[2] += double(L.z);
        }
    });
    return 0;
}

// FP64 evaluation of the same sample streams; sums[3*i..] += L for each
// frame index in [frame0, frame0 + nframes).
int orc_render_f64(void* s, const uint32_t* pixels, uint32_t npix, uint32_t frame0, uint32_t nframes,
                   double* sums, int threads) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return -1;
    const Globals& g = o->globals;
    const uint32_t total = pixels ? npix : g.width * g.height;
    Tracer<double> tr{*o->packed, g};
    tr.allLeafInstances = o->allLeafInstances;
    tr.bruteForce = o->bruteForce != 0;
    tr.watertight = o->bruteForce == 2;
    parallelFor(total, threads, [&](uint32_t i) {
        const uint32_t p = pixels ? pixels[i] : i;
        const uint32_t px = p % g.width, py = p / g.width;
        double* a = sums + size_t(i) * 3;
        for (uint32_t f = frame0; f < frame0 + nframes; ++f) {
            const V3<double> L = tr.tracePath(px, py, f);
            a[0] += L.x;
            a[1] += L.y;
            a[2] += L.z;
        }
    });
    return 0;
}

// Closest hit through the reference BVH2 traversal (intersect.glsl:88-125).
int orc_trace(void* s, const RayIn* rays, uint32_t n, HitOut* out, int threads) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return -1;
    const Packed& P = *o->packed;
    Tracer<float> tr{P, o->globals};
    tr.allLeafInstances = o->allLeafInstances;
    parallelFor(n, threads, [&](uint32_t i) {
        Ray<float> r;
        r.origin = V3f(rays[i].o[0], rays[i].o[1], rays[i].o[2]);
        r.dir = V3f(rays[i].d[0], rays[i].d[1], rays[i].d[2]);
        r.tMax = rays[i].tMax;
        const Hit<float> h = tr.traceRay(r);
        HitOut& ho = out[i];
        std::memset(&ho, 0, sizeof(ho));
        ho.hit = h.hit ? 1u : 0u;
        if (h.hit) {
            ho.t = h.t;
            ho.instance = P.instances[h.inst].userId;
            ho.prim = P.tris[size_t(h.tri) * 4 + 3];
            ho.u = h.bary.x;
            ho.v = h.bary.y;
        }
    });
    return 0;
}

int orc_trace_shadow(void* s, const RayIn* rays, uint32_t n, uint32_t* occluded, int threads) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return -1;
    Tracer<float> tr{*o->packed, o->globals};
    tr.allLeafInstances = o->allLeafInstances;
    parallelFor(n, threads, [&](uint32_t i) {
        Ray<float> r;
        r.origin = V3f(rays[i].o[0], rays[i].o[1], rays[i].o[2]);
        r.dir = V3f(rays[i].d[0], rays[i].d[1], rays[i].d[2]);
        r.tMax = rays[i].tMax;
        occluded[i] = tr.traceShadowRay(r) ? 1u : 0u;
    });
    return 0;
}

// Brute force over every instance (id order) and every triangle (original
// index order), Moeller-Trumbore in object space, keeping the first triangle
// with the strictly smallest t (the brute-force oracle of reference
// tests/bvh_tests.cpp:145-151, extended to instances). Also reports the
// second-smallest t among all accepted hits (t2, +inf when none) and the
// smallest barycentric of the winning hit (minBary), which define the
// "non-degenerate" rays of the parity gate.
int orc_trace_bruteforce(void* s, const RayIn* rays, uint32_t n, HitOut* out, float* t2, float* minBary,
                         int threads) {
    auto* o = static_cast<OracleScene*>(s);
    if (!o->packed) return -1;
    const Scene& sc = o->scene;
    parallelFor(n, threads, [&](uint32_t i) {
        const V3f org(rays[i].o[0], rays[i].o[1], rays[i].o[2]);
        const V3f dir(rays[i].d[0], rays[i].d[1], rays[i].d[2]);
        float best = rays[i].tMax, second = INFINITY;
        HitOut h{};
        for (auto& [iid, in] : sc.instances) {
            auto mit = sc.meshes.find(in.mesh);
            if (mit == sc.meshes.end()) continue;
            const MeshData& m = mit->second;
            const M4<float> w2o = inverse(in.objectToWorld);
            const V3f oo = w2o.mulPoint(org);
            const V3f dd = w2o.mulDir(dir);
            const size_t nt = m.indices.size() / 3;
            for (size_t t = 0; t < nt; ++t) {
                const V3f v0 = m.positions[m.indices[t * 3]].xyz();
                const V3f e1 = m.positions[m.indices[t * 3 + 1]].xyz() - v0;
                const V3f e2 = m.positions[m.indices[t * 3 + 2]].xyz() - v0;
                const V3f p = cross(dd, e2);
                const float det = dot(e1, p);
                if (std::fabs(det) < 1e-12f) continue;
                const float invDet = 1.0f / det;
                const V3f sv = oo - v0;
                const float u = dot(sv, p) * invDet;
                if (u < 0.0f || u > 1.0f) continue;
                const V3f q = cross(sv, e1);
                const float v = dot(dd, q) * invDet;
                if (v < 0.0f || u + v > 1.0f) continue;
                const float tt = dot(e2, q) * invDet;
                if (!(tt > 1e-4f && tt < rays[i].tMax)) continue;
                if (tt < best) {
                    if (h.hit) second = std::min(second, best);
                    best = tt;
                    h.hit = 1;
                    h.t = tt;
                    h.instance = iid;
                    h.prim = uint32_t(t);
                    h.u = u;
                    h.v = v;
                } else {
                    second = std::min(second, tt);
                }
            }
        }
        out[i] = h;
        t2[i] = second;
        minBary[i] = h.hit ? std::min(std::min(h.u, h.v), 1.0f - h.u - h.v) : 0.0f;
    });
    return 0;
}

// Standalone reference BVH2 build over AABBs (6 floats each: lo xyz, hi xyz).
// nodesOut holds 2 * n nodes of 32 bytes; returns the node count.
uint32_t orc_bvh_build(const float* aabbs, uint32_t n, uint32_t maxLeaf, BvhNode* nodesOut,
                       uint32_t* primOrderOut) {
    std::vector<Aabb> b(n);
    for (uint32_t i = 0; i < n; ++i) {
        b[i].lo = V3f(aabbs[i * 6], aabbs[i * 6 + 1], aabbs[i * 6 + 2]);
        b[i].hi = V3f(aabbs[i * 6 + 3], aabbs[i * 6 + 4], aabbs[i * 6 + 5]);
    }
    const BvhBuild r = buildBvh(b, maxLeaf);
    std::memcpy(nodesOut, r.nodes.data(), r.nodes.size() * sizeof(BvhNode));
    std::memcpy(primOrderOut, r.primOrder.data(), r.primOrder.size() * 4);
    return uint32_t(r.nodes.size());
}

// Environment CDF (Renderer.cpp:620-655). cdfOut holds w*h + h floats.
float orc_env_cdf(const float* rgba, uint32_t w, uint32_t h, float* cdfOut) {
    std::vector<float> cdf;
    const float integral = buildEnvCdf(rgba, w, h, cdf);
    std::memcpy(cdfOut, cdf.data(), cdf.size() * 4);
    return integral;
}

// RGBA32F readback from an FP32 accumulation (Renderer.cpp:900-908).
void orc_readback_f32(const float* accum, uint32_t npix, uint32_t frameIndex, float* out) {
    const float inv = frameIndex > 0 ? 1.0f / float(frameIndex) : 0.0f;
    for (uint32_t i = 0; i < npix; ++i) {
        out[i * 4 + 0] = accum[i * 4 + 0] * inv;
        out[i * 4 + 1] = accum[i * 4 + 1] * inv;
        out[i * 4 + 2] = accum[i * 4 + 2] * inv;
        out[i * 4 + 3] = 1.0f;
    }
}

// RGBA8 resolve (resolve.comp:24-56) of an accumulation with count in .a.
void orc_resolve_rgba8(const float* accum, uint32_t npix, float exposureEV, uint32_t tonemap, uint8_t* out) {
    const float exposure = std::exp2(exposureEV);
    for (uint32_t i = 0; i < npix; ++i) {
        const float* a = accum + size_t(i) * 4;
        for (int c = 0; c < 3; ++c) {
            float v = a[3] > 0.0f ? a[c] / a[3] : 0.0f;
            v *= exposure;
            if (tonemap == 1) v = acesTonemap1(v);
            v = linearToSrgb1(clampv(v, 0.0f, 1e4f));
            out[i * 4 + c] = toUnorm8(v);
        }
        out[i * 4 + 3] = 255;
    }
}

// pcg4d on a batch of states (random.glsl:6-12), for the RNG pin.
void orc_pcg4d(const uint32_t* in, uint32_t n, uint32_t* out) {
    for (uint32_t i = 0; i < n; ++i) {
        const U4 v = pcg4d(U4{in[i * 4], in[i * 4 + 1], in[i * 4 + 2], in[i * 4 + 3]});
        out[i * 4] = v.x;
        out[i * 4 + 1] = v.y;
        out[i * 4 + 2] = v.z;
        out[i * 4 + 3] = v.w;
    }
}

// Derived attributes of one mesh as the oracle's scene store computes them
// (normals when none are given, tangents when uvs are given; Scene.cpp:13-92
// restated): normalsOut and tangentsOut receive 4 floats per vertex. Returns
// the number of tangents written.
int orc_mesh_attributes(const float* positions, uint32_t vertexCount, const uint32_t* indices, uint32_t indexCount,
                        const float* uvs, float* normalsOut, float* tangentsOut) {
    mrtMeshDesc d{};
    d.structSize = sizeof(d);
    d.vertexCount = vertexCount;
    d.indexCount = indexCount;
    d.positions = positions;
    d.uvs = uvs;
    d.indices = indices;
    const MeshData m = copyMesh(d);
    for (uint32_t i = 0; i < vertexCount; ++i) {
        const V4<float>& n = m.normals[i];
        normalsOut[4 * i] = n.x, normalsOut[4 * i + 1] = n.y, normalsOut[4 * i + 2] = n.z, normalsOut[4 * i + 3] = n.w;
    }
    if (tangentsOut)
        for (size_t i = 0; i < m.tangents.size(); ++i) {
            const V4<float>& t = m.tangents[i];
            tangentsOut[4 * i] = t.x, tangentsOut[4 * i + 1] = t.y, tangentsOut[4 * i + 2] = t.z;
            tangentsOut[4 * i + 3] = t.w;
        }
    return int(m.tangents.size());
}

// Kahan's a * b - c * d in single precision, as the watertight test's edge
// fallback evaluates it (4 floats per entry in, 1 out).
void orc_diff_of_products(const float* abcd, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i)
        out[i] = Tracer<float>::diffOfProducts(abcd[4 * i], abcd[4 * i + 1], abcd[4 * i + 2], abcd[4 * i + 3]);
}

// Scene statistics after orc_commit: nodes, triangles, instances, tlasRoot,
// max BLAS depth (root = 1).
void orc_stats(void* s, uint32_t* out5) {
    auto* o = static_cast<OracleScene*>(s);
    std::memset(out5, 0, 5 * 4);
    if (!o->packed) return;
    const Packed& P = *o->packed;
    out5[0] = uint32_t(P.nodes.size());
    out5[1] = uint32_t(P.tris.size() / 4);
    out5[2] = uint32_t(P.instances.size());
    out5[3] = P.tlasRoot;
    uint32_t maxDepth = 0;
    for (const auto& in : P.instances) {
        std::vector<std::pair<uint32_t, uint32_t>> st{{in.blasRoot, 1}};
        while (!st.empty()) {
            auto [nid, dep] = st.back();
            st.pop_back();
            maxDepth = std::max(maxDepth, dep);
            const BvhNode& n = P.nodes[nid];
            if ((n.packed >> 2) == 0) {
                st.push_back({n.leftOrPrim, dep + 1});
                st.push_back({n.leftOrPrim + 1, dep + 1});
            }
        }
    }
    out5[4] = maxDepth;
}

}  // extern "C"
