// Device-side kernel library of the B200 wavefront path tracer.
//
// Per-sample arithmetic of Colvillea's header-only kernel library
// (include/colvillea/libkernel/...), written for sm_100a: the same FP32
// operations in the same order as the reference, so that results match its
// source evaluated in IEEE FP32 (the library is compiled with -fmad=false and
// IEEE division/sqrt; the reference's own GPU build used --use_fast_math,
// CMakeLists.txt:118).  Transcendentals (sinf, cosf, tanf, atan2f, acosf) are
// CUDA's.
//
// Behaviour the reference delegates to OWL (vector math), OptiX (triangle
// test, barycentrics) and the CUDA texture unit is defined here:
//   normalize(v) = v * (1/sqrt(dot(v,v))), dot left to right (OWL v1.1.6);
//   watertight ray-triangle test (Woop, Benthin, Wald, JCGT 2013);
//   FP32 bilinear RGBA32F lookup with wrap addressing.
#pragma once

#include <cstdint>
#include <cfloat>

namespace clb
{
constexpr float kPiF   = 3.14159265358979323846f;  // M_PIf, math.h:15
constexpr float kInvPi = 0.318309886183790671538f; // M_1_PIf, math.h:21
constexpr double kPiD  = 3.14159265358979323846;   // M_PI, warp.h:38,43
constexpr float kRayEps = 0.001f;                   // kRayTOffsetEpsilon, config.h:11

// ---------------------------------------------------------------------------
// Vector type with explicit, ordered operations.
// ---------------------------------------------------------------------------
struct f3
{
    float x, y, z;
};
struct f2
{
    float x, y;
};

__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ f3 normalize(f3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ bool nonzero(f3 v) { return v.x > 0.0f || v.y > 0.0f || v.z > 0.0f; }
__device__ __forceinline__ float comp(f3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// ---------------------------------------------------------------------------
// Sampler (libkernel/base/sampler.h:16-78): pcg4d hash of
// (px, py, frame, counter); each draw increments the counter first.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pcg4d(uint32_t& x, uint32_t& y, uint32_t& z, uint32_t& w)
{
    x = x * 1664525u + 1013904223u;
    y = y * 1664525u + 1013904223u;
    z = z * 1664525u + 1013904223u;
    w = w * 1664525u + 1013904223u;
    x += y * w;
    y += z * x;
    z += x * y;
    w += y * z;
    x ^= x >> 16u;
    y ^= y >> 16u;
    z ^= z >> 16u;
    w ^= w >> 16u;
    x += y * w;
    y += z * x;
    z += x * y;
    w += y * z;
}
__device__ __forceinline__ float uintToFloat(uint32_t x) { return __uint_as_float(0x3f800000u | (x >> 9)) - 1.0f; }

struct Rng
{
    uint32_t px, py, frame, ctr;
    __device__ __forceinline__ float next1D()
    {
        ++ctr;
        uint32_t x = px, y = py, z = frame, w = ctr;
        pcg4d(x, y, z, w);
        return uintToFloat(x);
    }
    __device__ __forceinline__ f2 next2D()
    {
        float a = next1D();
        float b = next1D();
        return {a, b};
    }
};

// ---------------------------------------------------------------------------
// Frame (libkernel/base/frame.h:24-130).
// ---------------------------------------------------------------------------
struct Frame
{
    f3 s, t, n;
    __device__ __forceinline__ f3 toLocal(f3 v) const { return {dot(v, t), dot(v, s), dot(v, n)}; }
    __device__ __forceinline__ f3 toWorld(f3 v) const
    {
        return {v.x * t.x + v.y * s.x + v.z * n.x, v.x * t.y + v.y * s.y + v.z * n.y, v.x * t.z + v.y * s.z + v.z * n.z};
    }
};
__device__ __forceinline__ float sinThetaL(f3 v)
{
    float tmp = 1.0f - v.z * v.z;
    return tmp <= 0.0f ? 0.0f : sqrtf(tmp);
}
__device__ __forceinline__ float tanThetaL(f3 v) { return sinThetaL(v) / v.z; }

// makeFrame (libkernel/base/math.h:33-48).
__device__ __forceinline__ void makeFrame(f3 a, f3* b, f3* c)
{
    if (fabsf(a.x) > fabsf(a.y))
    {
        float invLen = 1.0f / sqrtf(a.x * a.x + a.z * a.z);
        *c           = {a.z * invLen, 0.0f, -a.x * invLen};
    }
    else
    {
        float invLen = 1.0f / sqrtf(a.y * a.y + a.z * a.z);
        *c           = {0.0f, a.z * invLen, -a.y * invLen};
    }
    *b = cross(*c, a);
}

// hypot2 (math.h:55-73).
__device__ __forceinline__ float hypot2(float a, float b)
{
    float r;
    if (fabsf(a) > fabsf(b))
    {
        r = b / a;
        r = fabsf(a) * sqrtf(1.0f + r * r);
    }
    else if (b != 0.0f)
    {
        r = a / b;
        r = fabsf(b) * sqrtf(1.0f + r * r);
    }
    else
        r = 0.0f;
    return r;
}

// ---------------------------------------------------------------------------
// Warps (libkernel/base/warp.h:25-64).  The concentric-disk angle is a double
// expression in the reference (M_PI), evaluated in double here too.
// ---------------------------------------------------------------------------
__device__ __forceinline__ f2 concentricDisk(f2 s)
{
    float r1 = 2.0f * s.x - 1.0f;
    float r2 = 2.0f * s.y - 1.0f;
    float phi, r;
    if (r1 == 0.0f && r2 == 0.0f)
    {
        r = phi = 0.0f;
    }
    else if (r1 * r1 > r2 * r2)
    {
        r   = r1;
        phi = float((kPiD / 4.0) * double(r2 / r1));
    }
    else
    {
        r   = r2;
        phi = float((kPiD / 2.0) - double(r1 / r2) * (kPiD / 4.0));
    }
    float c = cosf(phi), sn = sinf(phi);
    return {r * c, r * sn};
}
__device__ __forceinline__ f3 cosineHemisphere(f2 s)
{
    f2    p = concentricDisk(s);
    float z = sqrtf(1.0f - p.x * p.x - p.y * p.y);
    return {p.x, p.y, z};
}
__device__ __forceinline__ float cosineHemispherePdf(f3 v) { return v.z * kInvPi; }
__device__ __forceinline__ float misBalanced(float a, float b) { return a / (a + b); } // warp.h:86-89

// ---------------------------------------------------------------------------
// Fresnel, reflect, refract (libkernel/base/math.h:172-329).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fresnelConductor1(float cosI, float c2, float s2, float s4, float eta, float k)
{
    float temp1 = eta * eta - k * k - s2;
    float a2pb2 = sqrtf(temp1 * temp1 + k * k * eta * eta * 4.0f);
    float a     = sqrtf((a2pb2 + temp1) * 0.5f);
    float term1 = a2pb2 + c2;
    float term2 = a * (2.0f * cosI);
    float Rs2   = (term1 - term2) / (term1 + term2);
    float term3 = a2pb2 * c2 + s4;
    float term4 = term2 * s2;
    float Rp2   = Rs2 * (term3 - term4) / (term3 + term4);
    return 0.5f * (Rp2 + Rs2);
}
__device__ __forceinline__ f3 fresnelConductor(float cosI, f3 eta, f3 k)
{
    float c2 = cosI * cosI, s2 = 1.0f - c2, s4 = s2 * s2;
    return {fresnelConductor1(cosI, c2, s2, s4, eta.x, k.x), fresnelConductor1(cosI, c2, s2, s4, eta.y, k.y),
            fresnelConductor1(cosI, c2, s2, s4, eta.z, k.z)};
}

__device__ __forceinline__ float fresnelDielectric(float cosThetaI_, float eta)
{
    if (eta == 1.0f) return 0.0f;
    float scale = (cosThetaI_ > 0.0f) ? 1.0f / eta : eta;
    float cosThetaTSqr = 1.0f - (1.0f - cosThetaI_ * cosThetaI_) * (scale * scale);
    if (cosThetaTSqr <= 0.0f) return 1.0f;
    float cosThetaI = fabsf(cosThetaI_);
    float cosThetaT = sqrtf(cosThetaTSqr);
    float Rs        = (cosThetaI - eta * cosThetaT) / (cosThetaI + eta * cosThetaT);
    float Rp        = (eta * cosThetaI - cosThetaT) / (eta * cosThetaI + cosThetaT);
    return 0.5f * (Rs * Rs + Rp * Rp);
}

__device__ __forceinline__ float fresnelDielectricExt(float cosThetaI_, float* cosThetaT_, float eta)
{
    if (eta == 1.0f)
    {
        *cosThetaT_ = -cosThetaI_;
        return 0.0f;
    }
    float scale = (cosThetaI_ > 0.0f) ? 1.0f / eta : eta;
    float cosThetaTSqr = 1.0f - (1.0f - cosThetaI_ * cosThetaI_) * (scale * scale);
    if (cosThetaTSqr <= 0.0f)
    {
        *cosThetaT_ = 0.0f;
        return 1.0f;
    }
    float cosThetaI = fabsf(cosThetaI_);
    float cosThetaT = sqrtf(cosThetaTSqr);
    float Rs        = (cosThetaI - eta * cosThetaT) / (cosThetaI + eta * cosThetaT);
    float Rp        = (eta * cosThetaI - cosThetaT) / (eta * cosThetaI + cosThetaT);
    *cosThetaT_     = (cosThetaI_ > 0.0f) ? -cosThetaT : cosThetaT;
    return 0.5f * (Rs * Rs + Rp * Rp);
}

__device__ __forceinline__ f3 reflect(f3 wo, f3 n)
{
    float d = 2.0f * dot(wo, n);
    return {-wo.x + d * n.x, -wo.y + d * n.y, -wo.z + d * n.z};
}
// ---------------------------------------------------------------------------
// Normal-mapped shading frame (Material::getShadingFrame,
// libkernel/base/material.h:128-287).
// ---------------------------------------------------------------------------
constexpr float kUpliftEps = 1.1f; // float(kNormalmapAutoAdapationUpliftEpsilon()), config.h:9

// fixNormalPerturbingShadingFrame (material.h:238-285): IRay's pull-up of a
// perturbed normal whose mirror direction of wo falls below the surface.
__device__ __forceinline__ void fixNormalPerturbing(f3 wo, Frame* fr, f3 ng)
{
    if (dot(wo, ng) < 0.0f)
    {
        fr->n = fr->n * -1.0f;
        ng    = ng * -1.0f;
    }
    if (dot(wo, ng) > 0.0f)
    {
        f3 r = reflect(wo, fr->n);
        if (dot(r, ng) <= 0.0f)
        {
            float a  = fabsf(dot(r, ng));
            float b  = dot(fr->n, ng);
            f3    up = (a / b) * fr->n;
            up       = up * kUpliftEps;
            fr->n    = normalize(normalize(r + up) + wo);
            fr->t    = normalize(fr->t - dot(fr->t, fr->n) * fr->n);
            fr->s    = normalize(cross(fr->n, fr->t));
            if (dot(fr->n, ng) < 0.0f)
            {
                fr->n = fr->n * -1.0f;
                fr->t = fr->t * -1.0f;
            }
        }
    }
}

// getShadingFrameImpl with a normal-map texel (material.h:164-221): the
// texel's rgb * 2 - 1, normalised, taken from the tangent frame
// {dpdv, dpdu, nb} to world; dpdu re-orthogonalised; everything flipped to
// nb's side.  pullUp: reflection-only materials (diffuse, metal) also get
// fixNormalPerturbing against nb (material.h:136-146).
__device__ __forceinline__ Frame normalMappedFrame(f3 wo, f3 dpdu, f3 dpdv, f3 nb, f3 texel, bool pullUp)
{
    f3 m = texel * 2.0f;
    m    = {m.x - 1.0f, m.y - 1.0f, m.z - 1.0f};
    m    = normalize(m);
    m    = Frame{dpdv, dpdu, nb}.toWorld(m);
    f3 du = dpdu - m * dot(dpdu, m);
    du    = normalize(du);
    f3 dv = normalize(cross(m, du));
    if (dot(m, nb) < 0.0f)
    {
        m  = m * -1.0f;
        du = du * -1.0f;
    }
    Frame fr{dv, du, m};
    if (pullUp) fixNormalPerturbing(wo, &fr, nb);
    return fr;
}

__device__ __forceinline__ f3 refract(f3 wi, f3 n, float eta, float cosThetaT)
{
    if (cosThetaT < 0.0f) eta = 1.0f / eta;
    float ne = -eta;
    float c  = eta * dot(wi, n) + cosThetaT;
    return {ne * wi.x + c * n.x, ne * wi.y + c * n.y, ne * wi.z + c * n.z};
}

// ---------------------------------------------------------------------------
// GGX (libkernel/base/microfacet.h:21-140).
// ---------------------------------------------------------------------------
struct GGX
{
    float alpha;
    __device__ __forceinline__ explicit GGX(float a) { alpha = fmaxf(a, 1e-4f); }
    __device__ __forceinline__ float smithG1(f3 v, f3 m) const
    {
        if (dot(v, m) * v.z <= 0.0f) return 0.0f;
        float tt = fabsf(tanThetaL(v));
        if (tt == 0.0f) return 1.0f;
        float root = alpha * tt;
        return 2.0f / (1.0f + hypot2(1.0f, root));
    }
    __device__ __forceinline__ float G(f3 wi, f3 wo, f3 m) const { return smithG1(wi, m) * smithG1(wo, m); }
    __device__ __forceinline__ float D(f3 m) const
    {
        if (m.z <= 0.0f) return 0.0f;
        float cosTheta2        = m.z * m.z;
        float beckmannExponent = (m.x * m.x + m.y * m.y) / (alpha * alpha * cosTheta2);
        float root             = (1.0f + beckmannExponent) * cosTheta2;
        return 1.0f / (kPiF * alpha * alpha * root * root);
    }
    __device__ __forceinline__ f3 sampleAll(f2 u, float* pdf) const
    {
        float alphaSqr   = alpha * alpha;
        float sinPhiM    = sinf((2.0f * kPiF) * u.y);
        float cosPhiM    = cosf((2.0f * kPiF) * u.y);
        float tanThetaM2 = alphaSqr * u.x / (1.0f - u.x);
        float cosThetaM  = 1.0f / sqrtf(1.0f + tanThetaM2);
        float temp       = 1.0f + tanThetaM2 / alphaSqr;
        *pdf             = kInvPi / (alphaSqr * cosThetaM * cosThetaM * cosThetaM * temp * temp);
        if (*pdf < 1e-20f) *pdf = 0.0f;
        float sinThetaM = sqrtf(fmaxf(0.0f, 1.0f - cosThetaM * cosThetaM));
        return {sinThetaM * cosPhiM, sinThetaM * sinPhiM, cosThetaM};
    }
    __device__ __forceinline__ float pdfAll(f3 m) const { return D(m) * m.z; }
};

// ---------------------------------------------------------------------------
// BSDFs (libkernel/bsdfs/*.h, tagged union libkernel/base/bsdf.h:36-107).
// ---------------------------------------------------------------------------
enum : uint32_t
{
    kDiffuse    = 0,
    kConductor  = 1,
    kDielectric = 2
};

struct Bsdf
{
    uint32_t type;
    f3       r;      // reflectance / specular reflectance
    float    alpha;  // GGX alpha
    float    etaInt; // dielectric interior IOR (exterior 1, roughdielectric.h:261)
    f3       eta, k; // conductor complex IOR
};

__device__ __forceinline__ f3 bsdfEval(const Bsdf& b, f3 wo, f3 wi)
{
    const f3 zero{0.0f, 0.0f, 0.0f};
    if (b.type == kDiffuse)
    {
        // smoothdiffuse.h:32-44
        if (wo.z <= 0.0f || wi.z <= 0.0f) return zero;
        return b.r * kInvPi;
    }
    if (b.type == kConductor)
    {
        // roughconductor.h:40-70
        if (wo.z <= 0.0f || wi.z <= 0.0f) return zero;
        f3  h = normalize(wo + wi);
        GGX dist(b.alpha);
        float D = dist.D(h);
        if (D == 0.0f) return zero;
        f3    F   = fresnelConductor(dot(wo, h), b.eta, b.k) * b.r;
        float G   = dist.G(wo, wi, h);
        float den = 4.0f * wo.z * wi.z;
        return {F.x * D * G / den, F.y * D * G / den, F.z * D * G / den};
    }
    // roughdielectric.h:37-103 (local wi/wo swap, :40-41)
    const f3 wI = wo, wO = wi;
    if (wI.z == 0.0f) return zero;
    bool refl = wI.z * wO.z > 0.0f;
    f3   H;
    if (refl)
        H = normalize(wO + wI);
    else
    {
        float eta = wI.z > 0.0f ? b.etaInt / 1.0f : 1.0f / b.etaInt;
        H         = normalize(wI + wO * eta);
    }
    H = H * (H.z > 0.0f ? 1.0f : -1.0f);
    GGX   distr(b.alpha);
    float D = distr.D(H);
    if (D == 0.0f) return zero;
    float F = fresnelDielectric(dot(wI, H), b.etaInt / 1.0f);
    float G = distr.G(wI, wO, H);
    float v;
    if (refl)
        v = F * D * G / (4.0f * fabsf(wI.z) * fabsf(wO.z));
    else
    {
        float eta       = wI.z > 0.0f ? b.etaInt / 1.0f : 1.0f / b.etaInt;
        float sqrtDenom = dot(wI, H) + eta * dot(wO, H);
        v = fabsf((1.0f - F) * D * G * dot(wI, H) * dot(wO, H) / (sqrtDenom * sqrtDenom * fabsf(wI.z) * fabsf(wO.z)));
    }
    return {v, v, v};
}

// `compat`: the reference's pdf functions (Q1 pdfAll(wo) for the conductor,
// Q2 cos(wo) for the diffuse lobe, Q3 an extra cos(H) for the dielectric).
__device__ __forceinline__ float bsdfPdf(const Bsdf& b, f3 wo, f3 wi, bool compat)
{
    if (b.type == kDiffuse)
    {
        if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f; // smoothdiffuse.h:46-57
        return cosineHemispherePdf(compat ? wo : wi);
    }
    if (b.type == kConductor)
    {
        if (wo.z <= 0.0f || wi.z <= 0.0f) return 0.0f; // roughconductor.h:72-90
        f3  h = normalize(wo + wi);
        GGX dist(b.alpha);
        return dist.pdfAll(compat ? wo : h) / (4.0f * fabsf(dot(wo, h)));
    }
    // roughdielectric.h:105-156
    const f3 wI = wo, wO = wi;
    bool     refl = wI.z * wO.z > 0.0f;
    f3       H;
    float    dwh_dwo;
    if (refl)
    {
        H       = normalize(wO + wI);
        dwh_dwo = 1.0f / (4.0f * dot(wO, H));
    }
    else
    {
        float eta       = wI.z > 0.0f ? b.etaInt / 1.0f : 1.0f / b.etaInt;
        H               = normalize(wI + wO * eta);
        float sqrtDenom = dot(wI, H) + eta * dot(wO, H);
        dwh_dwo         = (eta * eta * dot(wO, H)) / (sqrtDenom * sqrtDenom);
    }
    H = H * (H.z < 0.0f ? -1.0f : 1.0f);
    GGX   sd(b.alpha);
    float prob = compat ? sd.pdfAll(H) * H.z : sd.pdfAll(H);
    float F    = fresnelDielectric(dot(wI, H), b.etaInt / 1.0f);
    prob       = prob * (refl ? F : (1.0f - F));
    return fabsf(prob * dwh_dwo);
}

// BSDF::sample (bsdf.h:81-96); callers initialise *pdf to 0
// (raygeneration.cu:397), as the diffuse lobe leaves it untouched on the back.
__device__ __forceinline__ f3 bsdfSample(const Bsdf& b, f3 wo, f2 u, f3* wi, float* pdf)
{
    const f3 zero{0.0f, 0.0f, 0.0f};
    if (b.type == kDiffuse)
    {
        // smoothdiffuse.h:59-79
        if (wo.z <= 0.0f) return zero;
        *wi  = cosineHemisphere(u);
        *pdf = cosineHemispherePdf(*wi);
        return b.r * kInvPi;
    }
    if (b.type == kConductor)
    {
        // roughconductor.h:92-137
        if (wo.z <= 0.0f) return zero;
        GGX dist(b.alpha);
        f3  m = dist.sampleAll(u, pdf);
        if (*pdf == 0.0f) return zero;
        *wi = reflect(wo, m);
        if (wi->z <= 0.0f) return zero;
        *pdf    = *pdf / (4.0f * dot(wo, m));
        float D = dist.D(m);
        if (D == 0.0f) return zero;
        f3    F   = fresnelConductor(dot(wo, m), b.eta, b.k) * b.r;
        float G   = dist.G(wo, *wi, m);
        float den = 4.0f * wo.z * wi->z;
        return {F.x * D * G / den, F.y * D * G / den, F.z * D * G / den};
    }
    // roughdielectric.h:158-251
    const f3 wI = wo;
    GGX      distr(b.alpha);
    float    mpdf = 0.0f;
    f3       m    = distr.sampleAll(u, &mpdf);
    if (mpdf == 0.0f) return zero;
    *pdf            = mpdf;
    float cosThetaT = 0.0f;
    float F         = fresnelDielectricExt(dot(wI, m), &cosThetaT, b.etaInt / 1.0f);
    bool  sampleR   = true;
    if (u.x > F)
    {
        sampleR = false;
        *pdf    = *pdf * (1.0f - F);
    }
    else
        *pdf = *pdf * F;
    float D = distr.D(m);
    if (sampleR)
    {
        *wi = reflect(wI, m);
        if (wI.z * wi->z <= 0.0f) return zero;
        float G   = distr.G(*wi, wI, m);
        float dwh = fabsf(1.0f / (4.0f * dot(*wi, m)));
        *pdf      = *pdf * dwh;
        float v   = fabsf(F * D * G / (4.0f * wi->z * wI.z));
        return {v, v, v};
    }
    if (cosThetaT == 0.0f) return zero;
    *wi = refract(wI, m, b.etaInt / 1.0f, cosThetaT);
    if (wi->z * wI.z >= 0.0f) return zero;
    float G         = distr.G(*wi, wI, m);
    float eta       = wI.z > 0.0f ? b.etaInt / 1.0f : 1.0f / b.etaInt;
    float sqrtDenom = dot(wI, m) + eta * dot(*wi, m);
    float dwh       = fabsf(dot(*wi, m) * eta * eta / (sqrtDenom * sqrtDenom));
    *pdf            = *pdf * dwh;
    float v = fabsf((1.0f - F) * D * G * dot(wI, m) * dot(*wi, m) / (sqrtDenom * sqrtDenom * fabsf(wI.z) * fabsf(wi->z)));
    return {v, v, v};
}

// ---------------------------------------------------------------------------
// Texture: RGBA32F, wrap, bilinear, normalised coordinates
// (libkernel/textures/imagetex2d.h:34-37, src/core/nodes/textures/imagetex2d.cpp:51-65).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int wrapIndex(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__device__ __forceinline__ f3 texBilinear(const float4* __restrict__ tex, int w, int h, float u, float v)
{
    u        = u - floorf(u);
    v        = v - floorf(v);
    float x  = u * float(w) - 0.5f;
    float y  = v * float(h) - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    float ax = x - fx, ay = y - fy;
    int   ix = int(fx), iy = int(fy);
    int   x0 = wrapIndex(ix, w), x1 = wrapIndex(ix + 1, w);
    int   y0 = wrapIndex(iy, h), y1 = wrapIndex(iy + 1, h);
    float4 t00 = __ldg(tex + size_t(y0) * w + x0);
    float4 t10 = __ldg(tex + size_t(y0) * w + x1);
    float4 t01 = __ldg(tex + size_t(y1) * w + x0);
    float4 t11 = __ldg(tex + size_t(y1) * w + x1);
    float  bx = 1.0f - ax, by = 1.0f - ay;
    f3     out;
    {
        float top = t00.x * bx + t10.x * ax, bot = t01.x * bx + t11.x * ax;
        out.x     = top * by + bot * ay;
    }
    {
        float top = t00.y * bx + t10.y * ax, bot = t01.y * bx + t11.y * ax;
        out.y     = top * by + bot * ay;
    }
    {
        float top = t00.z * bx + t10.z * ax, bot = t01.z * bx + t11.z * ax;
        out.z     = top * by + bot * ay;
    }
    return out;
}

// ---------------------------------------------------------------------------
// HDRI dome (libkernel/emitters/hdridome.h).
// ---------------------------------------------------------------------------
struct DomeView
{
    const float4* __restrict__ tex;
    const float* __restrict__ pU;   // pUcondV_c, (w+1)*h
    const float* __restrict__ cdfU; // CDFpUcondV, (w+1)*h
    const float* __restrict__ pV;   // pV_c, h+1
    const float* __restrict__ cdfV; // CDFpV, h+1
    const uint2* __restrict__ aliasRow; // h entries {prob bits, alias row}
    const uint2* __restrict__ aliasCol; // w*h entries {prob bits, alias column}
    int w, h;
};

__device__ __forceinline__ uint32_t upperBound(const float* a, uint32_t begin, uint32_t end, float value)
{
    while (begin < end)
    {
        uint32_t middle = begin + (end - begin) / 2;
        if (__ldg(a + middle) <= value)
            begin = middle + 1;
        else
            end = middle;
    }
    return begin;
}

// Distribution1D::sample1D (hdridome.h:30-60).
__device__ __forceinline__ float sample1D(const float* f, const float* cdf, uint32_t N, float c, float u,
                                          uint32_t cdfOffset, float* pdf, uint32_t* sampledOffset)
{
    if (c == 0.0f) return 0.0f;
    uint32_t off = upperBound(cdf, cdfOffset, cdfOffset + N + 1, u) - 1;
    off          = off < cdfOffset ? cdfOffset : (off > cdfOffset + N - 1 ? cdfOffset + N - 1 : off);
    *pdf         = __ldg(f + off) / c;
    float c0 = __ldg(cdf + off), c1 = __ldg(cdf + off + 1);
    float du = u - c0;
    if (c1 - c0 != 0.0f) du = du / (c1 - c0);
    off            = off - cdfOffset;
    *sampledOffset = off;
    return (float(off) + du) / float(N);
}

// Distribution2D::sample2D (hdridome.h:95-123).
__device__ __forceinline__ f2 domeSample2DCdf(const DomeView& d, f2 r, float* pdf)
{
    float    px = 0.0f, py = 0.0f;
    uint32_t off = 0;
    f2       pt{0.0f, 0.0f};
    pt.y         = sample1D(d.pV, d.cdfV, uint32_t(d.h), __ldg(d.pV + d.h), r.y, 0, &py, &off);
    uint32_t W1  = uint32_t(d.w) + 1;
    pt.x = sample1D(d.pU, d.cdfU, uint32_t(d.w), __ldg(d.pU + size_t(off) * W1 + d.w), r.x, off * W1, &px, &off);
    *pdf = px * py;
    return pt;
}

// Distribution2D::pdf2D (hdridome.h:125-135).
__device__ __forceinline__ float domePdf2D(const DomeView& d, f2 s)
{
    if (s.x < 0.0f || s.y < 0.0f) return 0.0f;
    uint32_t tu = uint32_t(float(d.w) * s.x);
    uint32_t tv = uint32_t(float(d.h) * s.y);
    tu          = tu > uint32_t(d.w) - 1 ? uint32_t(d.w) - 1 : tu;
    tv          = tv > uint32_t(d.h) - 1 ? uint32_t(d.h) - 1 : tv;
    return __ldg(d.pU + size_t(tv) * (d.w + 1) + tu) / __ldg(d.pV + d.h);
}

// Two-level alias sampling over the same piecewise-constant density:
// rows by the marginal alias table, then columns by the row's alias table
// (Walker/Vose tables built in FP64 by the dome preprocessing).  Each level
// uses one uniform number: its integer part picks the bucket, its fraction is
// the coin and, rescaled, the continuous offset inside the chosen cell.  The
// returned pdf is the CDF sampler's (f/c, same table), so MIS weights agree.
__device__ __forceinline__ f2 domeSample2DAlias(const DomeView& d, f2 r, float* pdf)
{
    float    yv = r.y * float(d.h);
    uint32_t i  = min(uint32_t(yv), uint32_t(d.h) - 1);
    float    fr = yv - float(i);
    uint2    e  = __ldg(d.aliasRow + i);
    float    p  = __uint_as_float(e.x);
    uint32_t row;
    float    dv;
    if (fr < p)
    {
        row = i;
        dv  = fr / p;
    }
    else
    {
        row = e.y;
        dv  = (fr - p) / (1.0f - p);
    }
    float    xv = r.x * float(d.w);
    uint32_t j  = min(uint32_t(xv), uint32_t(d.w) - 1);
    float    fc = xv - float(j);
    uint2    g  = __ldg(d.aliasCol + size_t(row) * d.w + j);
    float    q  = __uint_as_float(g.x);
    uint32_t col;
    float    du;
    if (fc < q)
    {
        col = j;
        du  = fc / q;
    }
    else
    {
        col = g.y;
        du  = (fc - q) / (1.0f - q);
    }
    du = fminf(du, 0.99999994f);
    dv = fminf(dv, 0.99999994f);
    f2 uv{(float(col) + du) / float(d.w), (float(row) + dv) / float(d.h)};
    *pdf = __ldg(d.pU + size_t(row) * (d.w + 1) + col) / __ldg(d.pV + d.h);
    return uv;
}

// acos argument of a direction's y.  `clampY` keeps directions whose y
// rounded past +-1 (toWorld of a near-vertical local direction) on the
// sphere; the reference passes y unclamped (acos gives NaN there), which the
// compat estimator reproduces.
__device__ __forceinline__ float cosY(float y, bool clampY) { return clampY ? fminf(fmaxf(y, -1.0f), 1.0f) : y; }

// directionToUVCoords (hdridome.h:472-476).
__device__ __forceinline__ f2 dirToUV(f3 dir, bool clampY = false)
{
    return {atan2f(dir.x, dir.z) * -kInvPi * 0.5f + 0.5f, acosf(cosY(dir.y, clampY)) * kInvPi};
}

// evalEnvironment (hdridome.h:291-297).
__device__ __forceinline__ f3 domeEval(const DomeView& d, f3 dir, bool clampY = false)
{
    f2 uv = dirToUV(dir, clampY);
    return texBilinear(d.tex, d.w, d.h, uv.x, uv.y);
}

// pdfDirect (hdridome.h:248-279), importance sampling on.
__device__ __forceinline__ float domePdf(const DomeView& d, f3 dir, bool clampY = false)
{
    float phi      = atan2f(dir.x, dir.z);
    float theta    = acosf(cosY(dir.y, clampY));
    float sinTheta = sinf(theta);
    if (sinTheta == 0.0f) return 0.0f;
    f2 uv{phi * -kInvPi * 0.5f + 0.5f, theta * kInvPi};
    return domePdf2D(d, uv) / (2.0f * kPiF * kPiF * sinTheta);
}

// sampleDirect (hdridome.h:186-228).
__device__ __forceinline__ f3 domeSample(const DomeView& d, f2 u, bool alias, f3* dir, float* pdf)
{
    f2    uv       = alias ? domeSample2DAlias(d, u, pdf) : domeSample2DCdf(d, u, pdf);
    float theta    = kPiF * uv.y;
    float phi      = -2.0f * kPiF * (uv.x - 0.5f);
    float sinTheta = sinf(theta), cosTheta = cosf(theta);
    float sinPhi = sinf(phi), cosPhi = cosf(phi);
    if (sinTheta == 0.0f)
    {
        *pdf = 0.0f;
        return {0.0f, 0.0f, 0.0f};
    }
    *dir = {sinTheta * sinPhi, cosTheta, sinTheta * cosPhi}; // warp.h:16-22
    *pdf = *pdf / (2.0f * kPiF * kPiF * sinTheta);
    return texBilinear(d.tex, d.w, d.h, uv.x, uv.y);
}

// ---------------------------------------------------------------------------
// Directional emitter (libkernel/emitters/directional.h:30-66).
// ---------------------------------------------------------------------------
struct DirectionalLight
{
    f3    intensity, direction;
    float angularRadius;
};

__device__ __forceinline__ f3 directionalSample(const DirectionalLight& e, f2 u, f3* dir, float* pdf)
{
    f3    rev  = -e.direction;
    f2    disk = concentricDisk(u);
    float tr   = tanf(e.angularRadius);
    disk       = {disk.x * tr, disk.y * tr};
    f3 ax, ay;
    makeFrame(rev, &ax, &ay);
    f3 d           = rev + ax * disk.x;
    d              = d + ay * disk.y;
    *dir           = normalize(d);
    float tanTheta = sqrtf(disk.x * disk.x + disk.y * disk.y);
    float cosTheta = 1.0f / sqrtf(1.0f + tanTheta * tanTheta);
    float tanR     = tanf(e.angularRadius);
    *pdf           = kInvPi / (tanR * tanR * cosTheta * cosTheta * cosTheta);
    return e.intensity;
}

// ---------------------------------------------------------------------------
// Watertight ray-triangle test (Woop, Benthin and Wald, JCGT 2013).
// ---------------------------------------------------------------------------
struct RayPre
{
    f3    o;
    int   kx, ky, kz;
    float Sx, Sy, Sz;
};

__device__ __forceinline__ RayPre rayPrepare(f3 o, f3 d)
{
    RayPre r;
    r.o      = o;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    r.kz     = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    r.kx     = r.kz + 1 == 3 ? 0 : r.kz + 1;
    r.ky     = r.kx + 1 == 3 ? 0 : r.kx + 1;
    float dz = comp(d, r.kz);
    if (dz < 0.0f)
    {
        int t = r.kx;
        r.kx  = r.ky;
        r.ky  = t;
    }
    r.Sx = comp(d, r.kx) / dz;
    r.Sy = comp(d, r.ky) / dz;
    r.Sz = 1.0f / dz;
    return r;
}

// True with t, b1, b2 when the ray crosses the triangle's plane inside the
// triangle (edges inclusive, det != 0); the t-range test is the caller's.
__device__ __forceinline__ bool intersectTri(const RayPre& r, f3 v0, f3 v1, f3 v2, float* t, float* b1, float* b2)
{
    f3    A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
    float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    float Ax = comp(A, r.kx) - r.Sx * Akz, Ay = comp(A, r.ky) - r.Sy * Akz;
    float Bx = comp(B, r.kx) - r.Sx * Bkz, By = comp(B, r.ky) - r.Sy * Bkz;
    float Cx = comp(C, r.kx) - r.Sx * Ckz, Cy = comp(C, r.ky) - r.Sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f)
    {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float Az = r.Sz * Akz, Bz = r.Sz * Bkz, Cz = r.Sz * Ckz;
    float T   = U * Az + V * Bz + W * Cz;
    float rcp = 1.0f / det;
    *t        = T * rcp;
    *b1       = V * rcp;
    *b2       = W * rcp;
    return true;
}

} // namespace clb
