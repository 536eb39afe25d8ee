// Shading for sm_100a: pcg4d RNG, texture lookups, the "Disney-lite" BSDF,
// light sampling and surface reconstruction. Each function restates the
// reference shader function named beside it with the same operation order.
// This code is compiled without multiply-add contraction (-fmad=false) and
// takes sin/cos/atan2/acos from detmath.h, so every sample evaluates the same
// IEEE single-precision operations as the CPU evaluation of the shaders.
#pragma once

#include "../common/detmath.h"
#include "../common/device_types.h"
#include "vec.cuh"

#define MRT_PI 3.14159265358979323846f
#define MRT_TWO_PI 6.28318530717958647692f
#define MRT_INV_PI 0.31830988618379067154f

// ---- RNG: pcg4d (random.glsl:6-31) ------------------------------------------
struct Rng {
    uint32_t x, y, z, w;
};
MRT_DEV uint4 pcg4d(uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    x = x * 1664525u + 1013904223u;
    y = y * 1664525u + 1013904223u;
    z = z * 1664525u + 1013904223u;
    w = w * 1664525u + 1013904223u;
    x += y * w; y += z * x; z += x * y; w += y * z;
    x ^= x >> 16; y ^= y >> 16; z ^= z >> 16; w ^= w >> 16;
    x += y * w; y += z * x; z += x * y; w += y * z;
    return make_uint4(x, y, z, w);
}
// float(u) rounds to nearest (a draw may be exactly 1.0, as in the shader).
MRT_DEV float unitf(uint32_t u) { return __uint2float_rn(u) * (1.0f / 4294967296.0f); }
MRT_DEV float rng1(Rng& r) {
    r.w++;
    return unitf(pcg4d(r.x, r.y, r.z, r.w).x);
}
MRT_DEV float2 rng2(Rng& r) {
    r.w++;
    const uint4 v = pcg4d(r.x, r.y, r.z, r.w);
    return make_float2(unitf(v.x), unitf(v.y));
}

// ---- common.glsl:94-100 Duff et al. ONB ------------------------------------------
MRT_DEV void buildOnb(float3 n, float3& t, float3& b) {
    const float s = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (s + n.z);
    const float c = n.x * n.y * a;
    t = f3(1.0f + s * n.x * n.x * a, s * c, -s * n.x);
    b = f3(c, s + n.y * n.y * a, -n.y);
}

// ---- textures: bilinear, LOD 0, REPEAT in u and v -----------------------------------
// An 8-bit channel k decodes to k / 255; sRGB textures then go through
// c <= 0.04045 ? c / 12.92 : ((c + 0.055) / 1.055)^2.4, which is looked up
// in the 256-entry table the engine builds on the host (srgbLut).
MRT_DEV float4 texelFetch(const MrtTexture& t, const float* __restrict__ srgbLut, uint32_t x, uint32_t y) {
    const size_t i = size_t(y) * t.width + x;
    if (t.format == MRT_DTEX_RGBA32F) return ldg4(reinterpret_cast<const float4*>(t.texels) + i);
    const uint32_t p = __ldg(reinterpret_cast<const uint32_t*>(t.texels) + i);
    if (t.format == MRT_DTEX_RGBA8_SRGB)
        return make_float4(__ldg(srgbLut + (p & 255u)), __ldg(srgbLut + ((p >> 8) & 255u)),
                           __ldg(srgbLut + ((p >> 16) & 255u)), float(p >> 24) / 255.0f);
    return make_float4(float(p & 255u) / 255.0f, float((p >> 8) & 255u) / 255.0f, float((p >> 16) & 255u) / 255.0f,
                       float(p >> 24) / 255.0f);
}
// floor(f) mod n for an integral f (REPEAT addressing): a 32-bit remainder
// while f fits an int; beyond that fmodf, whose result is exact, gives the
// same residue.
MRT_DEV uint32_t wrapIndex(float f, uint32_t n) {
    const int m = fabsf(f) < 2147483648.0f ? int(f) % int(n) : int(fmodf(f, float(n)));
    return uint32_t(m < 0 ? m + int(n) : m);
}
MRT_DEV float4 sampleBilinear(const MrtTexture& t, const float* __restrict__ srgbLut, float u, float v) {
    if (t.texels == nullptr) return make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    const float fx = u * float(t.width) - 0.5f, fy = v * float(t.height) - 0.5f;
    const float x0f = floorf(fx), y0f = floorf(fy);
    const float ax = fx - x0f, ay = fy - y0f;
    const uint32_t x0 = wrapIndex(x0f, t.width), x1 = x0 + 1 == t.width ? 0 : x0 + 1;
    const uint32_t y0 = wrapIndex(y0f, t.height), y1 = y0 + 1 == t.height ? 0 : y0 + 1;
    const float4 t00 = texelFetch(t, srgbLut, x0, y0), t10 = texelFetch(t, srgbLut, x1, y0);
    const float4 t01 = texelFetch(t, srgbLut, x0, y1), t11 = texelFetch(t, srgbLut, x1, y1);
    const float w00 = (1.0f - ax) * (1.0f - ay), w10 = ax * (1.0f - ay), w01 = (1.0f - ax) * ay, w11 = ax * ay;
    return make_float4(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
                       w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
                       w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z,
                       w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w);
}
// RGBA32F environment, bilinear REPEAT
MRT_DEV float3 envFetch(const MrtFrameParams& P, float u, float v) {
    const uint32_t w = P.envW ? P.envW : 1, h = P.envH ? P.envH : 1;
    const float fx = u * float(w) - 0.5f, fy = v * float(h) - 0.5f;
    const float x0f = floorf(fx), y0f = floorf(fy);
    const float ax = fx - x0f, ay = fy - y0f;
    const uint32_t x0 = wrapIndex(x0f, w), x1 = x0 + 1 == w ? 0 : x0 + 1;
    const uint32_t y0 = wrapIndex(y0f, h), y1 = y0 + 1 == h ? 0 : y0 + 1;
    const float4 t00 = ldg4(P.envTexels + size_t(y0) * w + x0), t10 = ldg4(P.envTexels + size_t(y0) * w + x1);
    const float4 t01 = ldg4(P.envTexels + size_t(y1) * w + x0), t11 = ldg4(P.envTexels + size_t(y1) * w + x1);
    const float w00 = (1.0f - ax) * (1.0f - ay), w10 = ax * (1.0f - ay), w01 = (1.0f - ax) * ay, w11 = ax * ay;
    return f3(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x, w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
              w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z);
}

// ---- bsdf.glsl ----------------------------------------------------------------
struct Bsdf {
    float3 baseColor;
    float roughness, metallic, transmission, ior;
    bool entering;
};
MRT_DEV float ggxD(float3 h, float alpha) {  // bsdf.glsl:29-34
    const float a2 = alpha * alpha;
    const float c2 = h.z * h.z;
    const float d = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / mmax(MRT_PI * d * d, 1e-12f);
}
MRT_DEV float ggxLambda(float3 w, float alpha) {  // bsdf.glsl:36-40
    const float c2 = w.z * w.z;
    const float t2 = mmax(1.0f - c2, 0.0f) / mmax(c2, 1e-12f);
    return 0.5f * (sqrtf(1.0f + alpha * alpha * t2) - 1.0f);
}
MRT_DEV float ggxG1(float3 w, float alpha) { return 1.0f / (1.0f + ggxLambda(w, alpha)); }
MRT_DEV float ggxG2(float3 wo, float3 wi, float alpha) {
    return 1.0f / (1.0f + ggxLambda(wo, alpha) + ggxLambda(wi, alpha));
}
MRT_DEV float3 sampleGgxVndf(float3 wo, float alpha, float2 u) {  // bsdf.glsl:48-61 (Heitz 2018)
    const float3 vh = normalize(f3(alpha * wo.x, alpha * wo.y, wo.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const float3 T1 = lensq > 0.0f ? f3(-vh.y, vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : f3(1.0f, 0.0f, 0.0f);
    const float3 T2 = cross(vh, T1);
    const float r = sqrtf(u.x);
    float sphi, cphi;
    detm::sincos(MRT_TWO_PI * u.y, &sphi, &cphi);
    const float t1 = r * cphi;
    float t2 = r * sphi;
    const float s = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - s) * sqrtf(mmax(1.0f - t1 * t1, 0.0f)) + s * t2;
    const float3 nh = t1 * T1 + t2 * T2 + sqrtf(mmax(1.0f - t1 * t1 - t2 * t2, 0.0f)) * vh;
    return normalize(f3(alpha * nh.x, alpha * nh.y, mmax(nh.z, 1e-6f)));
}
MRT_DEV float3 fresnelSchlick(float3 f0, float cosTheta) {  // bsdf.glsl:63-67
    const float m = clampf(1.0f - cosTheta, 0.0f, 1.0f);
    const float m2 = m * m;
    return f0 + (f3(1.0f) - f0) * (m2 * m2 * m);
}
MRT_DEV float fresnelDielectric(float cosI, float eta) {  // bsdf.glsl:69-77
    cosI = clampf(cosI, 0.0f, 1.0f);
    const float sin2T = (1.0f - cosI * cosI) / (eta * eta);
    if (sin2T >= 1.0f) return 1.0f;
    const float cosT = sqrtf(1.0f - sin2T);
    const float rs = (cosI - eta * cosT) / (cosI + eta * cosT);
    const float rp = (eta * cosI - cosT) / (eta * cosI + cosT);
    return 0.5f * (rs * rs + rp * rp);
}
MRT_DEV void lobeWeights(const Bsdf& m, float3 wo, float& wDiff, float& wSpec, float& wTrans) {  // bsdf.glsl:87-95
    const float3 f0 = mix3(f3(0.04f), m.baseColor, m.metallic);
    wSpec = luminance(fresnelSchlick(f0, fabsf(wo.z)));
    wDiff = (1.0f - m.metallic) * (1.0f - m.transmission) * luminance(m.baseColor);
    wTrans = (1.0f - m.metallic) * m.transmission;
    float total = wDiff + wSpec + wTrans;
    if (total < 1e-7f) {
        wDiff = 1.0f;
        wSpec = 0.0f;
        wTrans = 0.0f;
        total = 1.0f;
    }
    wDiff /= total;
    wSpec /= total;
    wTrans /= total;
}
MRT_DEV void bsdfEval(const Bsdf& m, float3 wo, float3 wi, float3& f, float& pdf) {  // bsdf.glsl:100-144
    f = f3(0.0f);
    pdf = 0.0f;
    const float alpha = mmax(m.roughness * m.roughness, 1e-3f);
    float wDiff, wSpec, wTrans;
    lobeWeights(m, wo, wDiff, wSpec, wTrans);
    const float eta = m.entering ? m.ior : 1.0f / m.ior;
    if (wi.z > 0.0f) {
        if (wDiff > 0.0f) {
            const float3 fd = (1.0f - m.metallic) * (1.0f - m.transmission) * m.baseColor * MRT_INV_PI;
            f += fd;
            pdf += wDiff * wi.z * MRT_INV_PI;
        }
        const float3 h = normalize(wo + wi);
        const float d = ggxD(h, alpha);
        const float g2 = ggxG2(wo, wi, alpha);
        const float3 f0 = mix3(f3(0.04f), m.baseColor, m.metallic);
        const float3 F = fresnelSchlick(f0, dot(wo, h));
        f += d * g2 * F / mmax(4.0f * wo.z * wi.z, 1e-7f);
        pdf += wSpec * ggxG1(wo, alpha) * d / mmax(4.0f * wo.z, 1e-7f);
    } else if (wTrans > 0.0f) {
        float3 h = normalize(wo + wi * eta);
        if (h.z < 0.0f) h = -h;
        const float woH = dot(wo, h);
        const float wiH = dot(wi, h);
        if (woH * wiH < 0.0f) {
            const float F = fresnelDielectric(fabsf(woH), eta);
            const float d = ggxD(h, alpha);
            const float g2 = ggxG2(wo, f3(wi.x, wi.y, -wi.z), alpha);
            float denom = woH + eta * wiH;
            denom = mmax(denom * denom, 1e-7f);
            const float jac = eta * eta * fabsf(wiH) / denom;
            f += m.baseColor * (1.0f - F) * d * g2 * fabsf(woH) * jac / mmax(fabsf(wo.z * wi.z), 1e-7f) *
                 (1.0f - m.metallic) * m.transmission;
            pdf += wTrans * (1.0f - F) * ggxG1(wo, alpha) * d * fabsf(woH) / mmax(wo.z, 1e-7f) * jac;
        }
    }
}
struct BsdfSample {
    float3 wi, f;
    float pdf;
    bool valid;
};
MRT_DEV BsdfSample bsdfSample(const Bsdf& m, float3 wo, Rng& rng) {  // bsdf.glsl:147-192
    BsdfSample s;
    s.valid = false;
    const float alpha = mmax(m.roughness * m.roughness, 1e-3f);
    float wDiff, wSpec, wTrans;
    lobeWeights(m, wo, wDiff, wSpec, wTrans);
    const float eta = m.entering ? m.ior : 1.0f / m.ior;
    const float pick = rng1(rng);
    float3 wi;
    if (pick < wDiff) {  // cosine hemisphere (bsdf.glsl:79-84)
        const float2 u = rng2(rng);
        const float r = sqrtf(u.x);
        float sphi, cphi;
        detm::sincos(MRT_TWO_PI * u.y, &sphi, &cphi);
        wi = f3(r * cphi, r * sphi, sqrtf(mmax(1.0f - u.x, 0.0f)));
    } else if (pick < wDiff + wSpec) {
        const float3 h = sampleGgxVndf(wo, alpha, rng2(rng));
        wi = reflect(-wo, h);
        if (wi.z <= 0.0f) return s;
    } else {
        const float3 h = sampleGgxVndf(wo, alpha, rng2(rng));
        const float woH = dot(wo, h);
        const float F = fresnelDielectric(fabsf(woH), eta);
        if (rng1(rng) < F) {
            wi = reflect(-wo, h);
            if (wi.z <= 0.0f) return s;
        } else {
            wi = refract(-wo, h, 1.0f / eta);
            if (wi.z >= 0.0f || length(wi) < 1e-6f) return s;
            wi = normalize(wi);
        }
    }
    float3 f;
    float pdf;
    bsdfEval(m, wo, wi, f, pdf);
    if (pdf < 1e-9f) return s;
    s.wi = wi;
    s.f = f;
    s.pdf = pdf;
    s.valid = true;
    return s;
}

// ---- lights.glsl --------------------------------------------------------------------
MRT_DEV float2 dirToEquirect(const MrtFrameParams& P, float3 d) {  // lights.glsl:11-15
    const float phi = detm::atan2(d.z, d.x) - P.envRotation;
    const float theta = detm::acos(clampf(d.y, -1.0f, 1.0f));
    return make_float2(fractf(phi / MRT_TWO_PI + 1.0f), theta / MRT_PI);
}
MRT_DEV float3 equirectToDir(const MrtFrameParams& P, float2 uv) {  // lights.glsl:17-22
    const float phi = uv.x * MRT_TWO_PI + P.envRotation;
    const float theta = uv.y * MRT_PI;
    float st, ct, sp, cp;
    detm::sincos(theta, &st, &ct);
    detm::sincos(phi, &sp, &cp);
    return f3(st * cp, ct, st * sp);
}
MRT_DEV bool hasEnv(const MrtFrameParams& P) { return (P.flags & MRT_FLAG_HAS_ENV) != 0u; }
MRT_DEV float3 envRadiance(const MrtFrameParams& P, float3 dir) {  // lights.glsl:24-27
    if (!hasEnv(P)) return f3(0.0f);
    const float2 uv = dirToEquirect(P, dir);
    return envFetch(P, uv.x, uv.y) * P.envIntensity;
}
MRT_DEV float envPdf(const MrtFrameParams& P, float3 dir) {  // lights.glsl:30-34
    if (!hasEnv(P)) return 0.0f;
    const float2 uv = dirToEquirect(P, dir);
    return luminance(envFetch(P, uv.x, uv.y)) / P.envIntegral;
}
MRT_DEV uint32_t searchCdf(const float* __restrict__ cdf, uint32_t base, uint32_t count, float u) {  // lights.glsl:37-45
    uint32_t lo = 0, hi = count - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(cdf + base + mid) < u) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
struct LightSample {
    float3 wi, radiance;
    float pdf, dist;
    bool delta, valid;
};
MRT_DEV LightSample sampleOneLight(const MrtFrameParams& P, float3 p, Rng& rng) {  // lights.glsl:70-134
    LightSample ls;
    ls.valid = false;
    if (P.lightCount == 0) return ls;
    const uint32_t idx = min(uint32_t(rng1(rng) * float(P.lightCount)), P.lightCount - 1);
    const float pickPdf = 1.0f / float(P.lightCount);
    const MrtLight& l = P.lights[idx];
    if (l.type == MRT_DLIGHT_ENV) {  // lights.glsl:48-58 sampleEnv
        const uint32_t w = P.envW, h = P.envH;
        if (w == 0 || h == 0) return ls;
        const uint32_t row = searchCdf(P.envCdf, w * h, h, rng1(rng));
        const uint32_t col = searchCdf(P.envCdf, row * w, w, rng1(rng));
        const float2 uv = make_float2((float(col) + 0.5f) / float(w), (float(row) + 0.5f) / float(h));
        const float3 dir = equirectToDir(P, uv);
        const float3 rad = envFetch(P, uv.x, uv.y) * P.envIntensity;
        const float pdf = envPdf(P, dir);
        if (!(pdf > 1e-9f)) return ls;
        ls.wi = dir;
        ls.radiance = rad;
        ls.pdf = pdf * pickPdf;
        ls.dist = 1e30f;
        ls.delta = false;
        ls.valid = true;
    } else if (l.type == MRT_DLIGHT_SUN) {
        const float cosMax = l.p0[3];
        const float2 u = rng2(rng);
        const float cosT = mixf(1.0f, cosMax, u.x);
        const float sinT = sqrtf(mmax(1.0f - cosT * cosT, 0.0f));
        float sphi, cphi;
        detm::sincos(MRT_TWO_PI * u.y, &sphi, &cphi);
        float3 t, b;
        const float3 n = f3p(l.p0);
        buildOnb(n, t, b);
        ls.wi = normalize(t * (sinT * cphi) + b * (sinT * sphi) + n * cosT);
        ls.radiance = f3p(l.p1);
        const float conePdf = 1.0f / (MRT_TWO_PI * mmax(1.0f - cosMax, 1e-7f));
        ls.pdf = conePdf * pickPdf;
        ls.dist = 1e30f;
        ls.delta = true;
        ls.valid = true;
    } else if (l.type == MRT_DLIGHT_POINT) {
        const float3 d = f3p(l.p0) - p;
        const float d2 = mmax(dot(d, d), 1e-8f);
        ls.dist = sqrtf(d2);
        ls.wi = d / ls.dist;
        ls.radiance = f3p(l.p1) / d2;
        ls.pdf = pickPdf;
        ls.delta = true;
        ls.valid = true;
    } else {
        const float2 u = rng2(rng);
        const float3 q = f3p(l.p0) + f3p(l.p1) * u.x + f3p(l.p2) * u.y;
        const float3 d = q - p;
        const float d2 = mmax(dot(d, d), 1e-8f);
        ls.dist = sqrtf(d2);
        ls.wi = d / ls.dist;
        const float3 n = normalize(cross(f3p(l.p1), f3p(l.p2)));
        float cosL = dot(n, -ls.wi);
        if (l.p3[3] > 0.5f) cosL = fabsf(cosL);
        if (cosL < 1e-6f) return ls;
        const float area = mmax(l.p0[3], 1e-8f);
        ls.radiance = f3p(l.p3);
        ls.pdf = (d2 / (cosL * area)) * pickPdf;
        ls.delta = true;
        ls.valid = true;
    }
    return ls;
}
MRT_DEV float envPickPdf(const MrtFrameParams& P) {  // lights.glsl:137-140
    return (hasEnv(P) && P.lightCount > 0) ? 1.0f / float(P.lightCount) : 0.0f;
}
MRT_DEV float balanceHeuristic(float a, float b) { return a / mmax(a + b, 1e-12f); }  // pathtrace.comp:96-98
