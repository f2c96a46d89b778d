// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's per-sample arithmetic for the wavefront
// path-tracing hot path (Colvillea, include/colvillea/libkernel/...).  Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may call it,
// and only as the checker.  The product (colvillea_b200) never links it.
//
// Every function cites the reference file:line it restates.  The arithmetic
// is written out in the reference's evaluation order, in the scalar type T:
// T = float reproduces the reference's FP32 numbers (build with
// -ffp-contract=off, no fast-math); T = double gives the FP64 evaluation of
// the same formulas, used to classify ulp outliers.
//
// Pinning: this restatement is checked against the reference's own headers
// compiled on the host (oracle/_ref/libclref.so, built by oracle/ref/Makefile)
// through golden vectors committed under tests/golden/.
//
// Third-party arithmetic the reference leaves to OWL v1.1.6 (owl::common vector
// math, absent from the reference tree) is restated from OWL's published
// definitions: dot left to right, normalize(v) = v * (1/sqrt(dot(v,v))).
// Behaviour the reference leaves to OptiX 7 (ray-triangle test, barycentrics)
// and to the CUDA texture unit (bilinear RGBA32F lookup) is defined here and
// in the product identically (watertight test of Woop, Benthin and Wald 2013;
// FP32 bilinear filter with wrap addressing).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc
{
// ---------------------------------------------------------------------------
// Scalars.  The reference's float code calls the float overloads of sin, cos,
// tan, atan2, acos and sqrt; glibc's are used here.
// ---------------------------------------------------------------------------
constexpr float kPiF   = 3.14159265358979323846f; // M_PIf, math.h:15
constexpr float kInvPi = 0.318309886183790671538f; // M_1_PIf, math.h:21
constexpr double kPiD  = 3.14159265358979323846;  // M_PI (warp.h:38,43)

template <class T> struct V2
{
    T x, y;
};
template <class T> struct V3
{
    T x, y, z;
    T&       operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
};

template <class T> inline V3<T> mk(T a, T b, T c) { return V3<T>{a, b, c}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline T     dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline V3<T> normalize(V3<T> a) { return a * (T(1) / std::sqrt(dot(a, a))); }
template <class T> inline bool  nonzero(V3<T> v) { return v.x > T(0) || v.y > T(0) || v.z > T(0); }

inline float f_from_bits(uint32_t u)
{
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t bits_from_f(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// ---------------------------------------------------------------------------
// Sampler: pcg4d (sampler.h:16-36), uintToFloat (:39-42), rand (:51-55).
// ---------------------------------------------------------------------------
inline void pcg4d(uint32_t v[4])
{
    for (int i = 0; i < 4; ++i) v[i] = v[i] * 1664525u + 1013904223u;
    v[0] += v[1] * v[3];
    v[1] += v[2] * v[0];
    v[2] += v[0] * v[1];
    v[3] += v[1] * v[2];
    for (int i = 0; i < 4; ++i) v[i] ^= v[i] >> 16u;
    v[0] += v[1] * v[3];
    v[1] += v[2] * v[0];
    v[2] += v[0] * v[1];
    v[3] += v[1] * v[2];
}
inline float uint_to_float(uint32_t x) { return f_from_bits(0x3f800000u | (x >> 9)) - 1.0f; }

// State (px, py, frame, counter), initRNG (sampler.h:45-48); each draw
// increments the counter first, then hashes (sampler.h:51-55).
struct Rng
{
    uint32_t px, py, frame, ctr;
    float    next1D()
    {
        ++ctr;
        uint32_t v[4] = {px, py, frame, ctr};
        pcg4d(v);
        return uint_to_float(v[0]);
    }
    V2<float> next2D()
    {
        float a = next1D();
        float b = next1D();
        return {a, b};
    }
};

// ---------------------------------------------------------------------------
// Frame (frame.h:24-130): local basis (t, s, n) = (x, y, z).
// ---------------------------------------------------------------------------
template <class T> struct Frame
{
    V3<T> s, t, n;
    V3<T> toLocal(V3<T> v) const { return {dot(v, t), dot(v, s), dot(v, n)}; }
    V3<T> toWorld(V3<T> v) const
    {
        return {v.x * t.x + v.y * s.x + v.z * n.x, v.x * t.y + v.y * s.y + v.z * n.y, v.x * t.z + v.y * s.z + v.z * n.z};
    }
};
template <class T> inline T cosTheta(V3<T> v) { return v.z; }
template <class T> inline T sinTheta(V3<T> v)
{
    T tmp = T(1) - v.z * v.z;
    return tmp <= T(0) ? T(0) : std::sqrt(tmp);
}
template <class T> inline T tanTheta(V3<T> v) { return sinTheta(v) / cosTheta(v); }

// makeFrame (math.h:33-48).
template <class T> inline void makeFrame(V3<T> a, V3<T>* b, V3<T>* c)
{
    if (std::abs(a.x) > std::abs(a.y))
    {
        T invLen = T(1) / std::sqrt(a.x * a.x + a.z * a.z);
        *c       = {a.z * invLen, T(0), -a.x * invLen};
    }
    else
    {
        T invLen = T(1) / std::sqrt(a.y * a.y + a.z * a.z);
        *c       = {T(0), a.z * invLen, -a.y * invLen};
    }
    *b = cross(*c, a);
}

// hypot2 (math.h:55-73).
template <class T> inline T hypot2(T a, T b)
{
    T r;
    if (std::abs(a) > std::abs(b))
    {
        r = b / a;
        r = std::abs(a) * std::sqrt(T(1) + r * r);
    }
    else if (b != T(0))
    {
        r = a / b;
        r = std::abs(b) * std::sqrt(T(1) + r * r);
    }
    else
        r = T(0);
    return r;
}

// ---------------------------------------------------------------------------
// Warps (warp.h:25-64).  The concentric-disk angle is evaluated in double in
// the reference (M_PI is a double constant, warp.h:38,43).
// ---------------------------------------------------------------------------
template <class T> inline V2<T> concentricDisk(V2<T> s)
{
    T r1 = T(2) * s.x - T(1);
    T r2 = T(2) * s.y - T(1);
    T phi, r;
    if (r1 == 0 && r2 == 0)
    {
        r = phi = 0;
    }
    else if (r1 * r1 > r2 * r2)
    {
        r   = r1;
        phi = T((kPiD / 4.0) * double(r2 / r1));
    }
    else
    {
        r   = r2;
        phi = T((kPiD / 2.0) - double(r1 / r2) * (kPiD / 4.0));
    }
    T c = std::cos(phi), sn = std::sin(phi);
    return {r * c, r * sn};
}
template <class T> inline V3<T> cosineHemisphere(V2<T> s)
{
    V2<T> p = concentricDisk(s);
    T     z = std::sqrt(T(1) - p.x * p.x - p.y * p.y);
    return {p.x, p.y, z};
}
template <class T> inline T cosineHemispherePdf(V3<T> v) { return v.z * T(kInvPi); }

// Balance heuristic (warp.h:86-89).
template <class T> inline T misBalanced(T a, T b) { return a / (a + b); }

// ---------------------------------------------------------------------------
// Fresnel, reflect, refract (math.h:172-329).
// ---------------------------------------------------------------------------
template <class T> inline V3<T> fresnelConductor(T cosThetaI, V3<T> eta, V3<T> k)
{
    T     c2 = cosThetaI * cosThetaI, s2 = T(1) - c2, s4 = s2 * s2;
    V3<T> temp1, a2pb2, a, term1, term2, Rs2, term3, term4, Rp2, out;
    for (int i = 0; i < 3; ++i)
    {
        temp1[i] = eta[i] * eta[i] - k[i] * k[i] - s2;
        a2pb2[i] = std::sqrt(temp1[i] * temp1[i] + k[i] * k[i] * eta[i] * eta[i] * T(4));
        a[i]     = std::sqrt((a2pb2[i] + temp1[i]) * T(0.5));
        term1[i] = a2pb2[i] + c2;
        term2[i] = a[i] * (T(2) * cosThetaI);
        Rs2[i]   = (term1[i] - term2[i]) / (term1[i] + term2[i]);
        term3[i] = a2pb2[i] * c2 + s4;
        term4[i] = term2[i] * s2;
        Rp2[i]   = Rs2[i] * (term3[i] - term4[i]) / (term3[i] + term4[i]);
        out[i]   = T(0.5) * (Rp2[i] + Rs2[i]);
    }
    return out;
}

template <class T> inline T fresnelDielectric(T cosThetaI_, T eta)
{
    if (eta == T(1)) return T(0);
    T scale = (cosThetaI_ > 0) ? T(1) / eta : eta, cosThetaTSqr = T(1) - (T(1) - cosThetaI_ * cosThetaI_) * (scale * scale);
    if (cosThetaTSqr <= T(0)) return T(1);
    T cosThetaI = std::abs(cosThetaI_);
    T cosThetaT = std::sqrt(cosThetaTSqr);
    T Rs        = (cosThetaI - eta * cosThetaT) / (cosThetaI + eta * cosThetaT);
    T Rp        = (eta * cosThetaI - cosThetaT) / (eta * cosThetaI + cosThetaT);
    return T(0.5) * (Rs * Rs + Rp * Rp);
}

template <class T> inline T fresnelDielectricExt(T cosThetaI_, T* cosThetaT_, T eta)
{
    if (eta == T(1))
    {
        *cosThetaT_ = -cosThetaI_;
        return T(0);
    }
    T scale = (cosThetaI_ > 0) ? T(1) / eta : eta, cosThetaTSqr = T(1) - (T(1) - cosThetaI_ * cosThetaI_) * (scale * scale);
    if (cosThetaTSqr <= T(0))
    {
        *cosThetaT_ = T(0);
        return T(1);
    }
    T cosThetaI = std::abs(cosThetaI_);
    T cosThetaT = std::sqrt(cosThetaTSqr);
    T Rs        = (cosThetaI - eta * cosThetaT) / (cosThetaI + eta * cosThetaT);
    T Rp        = (eta * cosThetaI - cosThetaT) / (eta * cosThetaI + cosThetaT);
    *cosThetaT_ = (cosThetaI_ > 0) ? -cosThetaT : cosThetaT;
    return T(0.5) * (Rs * Rs + Rp * Rp);
}

template <class T> inline V3<T> reflect(V3<T> wo, V3<T> n)
{
    T d = T(2) * dot(wo, n);
    return {-wo.x + d * n.x, -wo.y + d * n.y, -wo.z + d * n.z};
}
// ---------------------------------------------------------------------------
// Normal-mapped shading frame (Material::getShadingFrame, material.h:128-287).
// ---------------------------------------------------------------------------
constexpr float kUpliftEps = 1.1f; // float(kNormalmapAutoAdapationUpliftEpsilon()), config.h:9

// fixNormalPerturbingShadingFrame (material.h:238-285).
template <class T> inline void fixNormalPerturbing(V3<T> wo, Frame<T>* fr, V3<T> ng)
{
    if (dot(wo, ng) < T(0))
    {
        fr->n = fr->n * T(-1);
        ng    = ng * T(-1);
    }
    if (dot(wo, ng) > T(0))
    {
        V3<T> r = reflect(wo, fr->n);
        if (dot(r, ng) <= T(0))
        {
            T     a  = std::abs(dot(r, ng));
            T     b  = dot(fr->n, ng);
            V3<T> up = (a / b) * fr->n;     // a / b * shFrame.n * eps
            up       = up * T(kUpliftEps);
            fr->n    = normalize(normalize(r + up) + wo);
            fr->t    = normalize(fr->t - dot(fr->t, fr->n) * fr->n);
            fr->s    = normalize(cross(fr->n, fr->t));
            if (dot(fr->n, ng) < T(0))
            {
                fr->n = fr->n * T(-1);
                fr->t = fr->t * T(-1);
            }
        }
    }
}

// getShadingFrameImpl with a normal map (material.h:164-221): nb is the
// normal of the unmodified tangent frame {dpdv, dpdu, nb}.
template <class T> inline Frame<T> normalMappedFrame(V3<T> wo, V3<T> dpdu, V3<T> dpdv, V3<T> nb, V3<T> texel, bool pullUp)
{
    V3<T> m = texel * T(2);
    m       = {m.x - T(1), m.y - T(1), m.z - T(1)};
    m       = normalize(m);
    m       = Frame<T>{dpdv, dpdu, nb}.toWorld(m);
    V3<T> du = dpdu - m * dot(dpdu, m);
    du       = normalize(du);
    V3<T> dv = normalize(cross(m, du));
    if (dot(m, nb) < T(0))
    {
        m  = m * T(-1);
        du = du * T(-1);
    }
    Frame<T> fr{dv, du, m};
    if (pullUp) fixNormalPerturbing(wo, &fr, nb);
    return fr;
}

template <class T> inline V3<T> refract(V3<T> wi, V3<T> n, T eta, T cosThetaT)
{
    if (cosThetaT < T(0)) eta = T(1) / eta;
    T ne = -eta;
    T c  = eta * dot(wi, n) + cosThetaT;
    return {ne * wi.x + c * n.x, ne * wi.y + c * n.y, ne * wi.z + c * n.z};
}

// ---------------------------------------------------------------------------
// GGX microfacet distribution (microfacet.h:21-140).
// ---------------------------------------------------------------------------
template <class T> struct GGX
{
    T alpha;
    explicit GGX(T a) { alpha = std::fmax(a, T(1e-4f)); }
    T smithG1(V3<T> v, V3<T> m) const
    {
        if (dot(v, m) * cosTheta(v) <= T(0)) return T(0);
        T tt = std::abs(tanTheta(v));
        if (tt == T(0)) return T(1);
        T root = alpha * tt;
        return T(2) / (T(1) + hypot2(T(1), root));
    }
    T G(V3<T> wi, V3<T> wo, V3<T> m) const { return smithG1(wi, m) * smithG1(wo, m); }
    T D(V3<T> m) const
    {
        if (cosTheta(m) <= T(0)) return T(0);
        T cosTheta2        = m.z * m.z;
        T beckmannExponent = (m.x * m.x + m.y * m.y) / (alpha * alpha * cosTheta2);
        T root             = (T(1) + beckmannExponent) * cosTheta2;
        return T(1) / (T(kPiF) * alpha * alpha * root * root);
    }
    V3<T> sampleAll(V2<T> u, T* pdf) const
    {
        T alphaSqr   = alpha * alpha;
        T sinPhiM    = std::sin(T(2.0f * kPiF) * u.y);
        T cosPhiM    = std::cos(T(2.0f * kPiF) * u.y);
        T tanThetaM2 = alphaSqr * u.x / (T(1) - u.x);
        T cosThetaM  = T(1) / std::sqrt(T(1) + tanThetaM2);
        T temp       = T(1) + tanThetaM2 / alphaSqr;
        *pdf         = T(kInvPi) / (alphaSqr * cosThetaM * cosThetaM * cosThetaM * temp * temp);
        if (*pdf < T(1e-20f)) *pdf = T(0);
        T sinThetaM = std::sqrt(std::fmax(T(0), T(1) - cosThetaM * cosThetaM));
        return {sinThetaM * cosPhiM, sinThetaM * sinPhiM, cosThetaM};
    }
    T pdfAll(V3<T> m) const { return D(m) * cosTheta(m); }
};

// ---------------------------------------------------------------------------
// BSDFs (bsdfs/smoothdiffuse.h, roughconductor.h, roughdielectric.h).
// `compat` reproduces the reference's pdf functions exactly (quirks Q1-Q3);
// without it the pdfs are the densities the sample() routines draw from.
// ---------------------------------------------------------------------------
enum BsdfType : uint32_t
{
    kDiffuse    = 0,
    kConductor  = 1,
    kDielectric = 2
};

template <class T> struct Bsdf
{
    uint32_t type;
    V3<T>    r;     // reflectance (diffuse) / specular reflectance (conductor)
    T        alpha; // GGX alpha (after the roughness^2 remap of metal.h:52 / glass.h:26)
    T        etaInt;
    V3<T>    eta, k;
    T        etaExt = T(1); // roughdielectric.h:261
};

template <class T> inline V3<T> bsdfEval(const Bsdf<T>& b, V3<T> wo, V3<T> wi)
{
    const V3<T> zero{0, 0, 0};
    if (b.type == kDiffuse)
    {
        // smoothdiffuse.h:32-44
        if (cosTheta(wo) <= T(0) || cosTheta(wi) <= T(0)) return zero;
        return b.r * T(kInvPi);
    }
    if (b.type == kConductor)
    {
        // roughconductor.h:40-70
        if (cosTheta(wo) <= T(0) || cosTheta(wi) <= T(0)) return zero;
        V3<T>  h = normalize(wo + wi);
        GGX<T> dist(b.alpha);
        T      D = dist.D(h);
        if (D == T(0)) return zero;
        V3<T> F = fresnelConductor(dot(wo, h), b.eta, b.k) * b.r;
        T     G = dist.G(wo, wi, h);
        T     den = T(4) * cosTheta(wo) * cosTheta(wi);
        return {F.x * D * G / den, F.y * D * G / den, F.z * D * G / den};
    }
    // roughdielectric.h:37-103 (wi/wo swapped locally, :40-41)
    const V3<T>& wI = wo;
    const V3<T>& wO = wi;
    if (cosTheta(wI) == T(0)) return zero;
    bool  refl = cosTheta(wI) * cosTheta(wO) > 0;
    V3<T> H;
    if (refl)
        H = normalize(wO + wI);
    else
    {
        T eta = cosTheta(wI) > 0 ? b.etaInt / b.etaExt : b.etaExt / b.etaInt;
        H     = normalize(wI + wO * eta);
    }
    H = H * (cosTheta(H) > T(0) ? T(1) : T(-1));
    GGX<T> distr(b.alpha);
    T      D = distr.D(H);
    if (D == T(0)) return zero;
    T F = fresnelDielectric(dot(wI, H), b.etaInt / b.etaExt);
    T G = distr.G(wI, wO, H);
    T v;
    if (refl)
        v = F * D * G / (T(4) * std::abs(cosTheta(wI)) * std::abs(cosTheta(wO)));
    else
    {
        T eta       = cosTheta(wI) > T(0) ? b.etaInt / b.etaExt : b.etaExt / b.etaInt;
        T sqrtDenom = dot(wI, H) + eta * dot(wO, H);
        v = std::abs((T(1) - F) * D * G * dot(wI, H) * dot(wO, H) /
                     (sqrtDenom * sqrtDenom * std::abs(cosTheta(wI)) * std::abs(cosTheta(wO))));
    }
    return {v, v, v};
}

template <class T> inline T bsdfPdf(const Bsdf<T>& b, V3<T> wo, V3<T> wi, bool compat)
{
    if (b.type == kDiffuse)
    {
        // smoothdiffuse.h:46-57 (Q2: the reference uses cos(wo))
        if (cosTheta(wo) <= T(0) || cosTheta(wi) <= T(0)) return T(0);
        return cosineHemispherePdf(compat ? wo : wi);
    }
    if (b.type == kConductor)
    {
        // roughconductor.h:72-90 (Q1: the reference evaluates pdfAll(wo))
        if (cosTheta(wo) <= T(0) || cosTheta(wi) <= T(0)) return T(0);
        V3<T>  h = normalize(wo + wi);
        GGX<T> dist(b.alpha);
        return dist.pdfAll(compat ? wo : h) / (T(4) * std::abs(dot(wo, h)));
    }
    // roughdielectric.h:105-156 (Q3: the reference multiplies by an extra cos(H))
    const V3<T>& wI   = wo;
    const V3<T>& wO   = wi;
    bool         refl = cosTheta(wI) * cosTheta(wO) > 0;
    V3<T>        H;
    T            dwh_dwo;
    if (refl)
    {
        H       = normalize(wO + wI);
        dwh_dwo = T(1) / (T(4) * dot(wO, H));
    }
    else
    {
        T eta       = cosTheta(wI) > 0 ? b.etaInt / b.etaExt : b.etaExt / b.etaInt;
        H           = normalize(wI + wO * eta);
        T sqrtDenom = dot(wI, H) + eta * dot(wO, H);
        dwh_dwo     = (eta * eta * dot(wO, H)) / (sqrtDenom * sqrtDenom);
    }
    H = H * (cosTheta(H) < T(0) ? T(-1) : T(1));
    GGX<T> sd(b.alpha);
    T      prob = compat ? sd.pdfAll(H) * cosTheta(H) : sd.pdfAll(H);
    T      F    = fresnelDielectric(dot(wI, H), b.etaInt / b.etaExt);
    prob        = prob * (refl ? F : (T(1) - F));
    return std::abs(prob * dwh_dwo);
}

// BSDF::sample.  *wi and *pdf are written exactly where the reference writes
// them; callers initialise *pdf to 0 (raygeneration.cu:397).
template <class T> inline V3<T> bsdfSample(const Bsdf<T>& b, V3<T> wo, V2<T> u, V3<T>* wi, T* pdf)
{
    const V3<T> zero{0, 0, 0};
    if (b.type == kDiffuse)
    {
        // smoothdiffuse.h:59-79
        if (cosTheta(wo) <= T(0)) return zero;
        *wi  = cosineHemisphere(u);
        *pdf = cosineHemispherePdf(*wi);
        return b.r * T(kInvPi);
    }
    if (b.type == kConductor)
    {
        // roughconductor.h:92-137
        if (cosTheta(wo) <= T(0)) return zero;
        GGX<T> dist(b.alpha);
        V3<T>  m = dist.sampleAll(u, pdf);
        if (*pdf == T(0)) return zero;
        *wi = reflect(wo, m);
        if (cosTheta(*wi) <= T(0)) return zero;
        *pdf = *pdf / (T(4) * dot(wo, m));
        T D  = dist.D(m);
        if (D == T(0)) return zero;
        V3<T> F   = fresnelConductor(dot(wo, m), b.eta, b.k) * b.r;
        T     G   = dist.G(wo, *wi, m);
        T     den = T(4) * cosTheta(wo) * cosTheta(*wi);
        return {F.x * D * G / den, F.y * D * G / den, F.z * D * G / den};
    }
    // roughdielectric.h:158-251
    const V3<T> wI = wo;
    GGX<T>      distr(b.alpha);
    T           mpdf = T(0);
    V3<T>       m    = distr.sampleAll(u, &mpdf);
    if (mpdf == T(0)) return zero;
    *pdf         = mpdf;
    T cosThetaT  = T(0);
    T F          = fresnelDielectricExt(dot(wI, m), &cosThetaT, b.etaInt / b.etaExt);
    bool sampleR = true;
    if (u.x > F)
    {
        sampleR = false;
        *pdf    = *pdf * (T(1) - F);
    }
    else
        *pdf = *pdf * F;
    T D = distr.D(m);
    if (sampleR)
    {
        *wi = reflect(wI, m);
        if (cosTheta(wI) * cosTheta(*wi) <= T(0)) return zero;
        T G   = distr.G(*wi, wI, m);
        T dwh = std::abs(T(1) / (T(4) * dot(*wi, m)));
        *pdf  = *pdf * dwh;
        T v   = std::abs(F * D * G / (T(4) * cosTheta(*wi) * cosTheta(wI)));
        return {v, v, v};
    }
    if (cosThetaT == T(0)) return zero;
    *wi = refract(wI, m, b.etaInt / b.etaExt, cosThetaT);
    if (cosTheta(*wi) * cosTheta(wI) >= T(0)) return zero;
    T G         = distr.G(*wi, wI, m);
    T eta       = cosTheta(wI) > T(0) ? b.etaInt / b.etaExt : b.etaExt / b.etaInt;
    T sqrtDenom = dot(wI, m) + eta * dot(*wi, m);
    T dwh       = std::abs(dot(*wi, m) * eta * eta / (sqrtDenom * sqrtDenom));
    *pdf        = *pdf * dwh;
    T v         = std::abs((T(1) - F) * D * G * dot(wI, m) * dot(*wi, m) /
                           (sqrtDenom * sqrtDenom * std::abs(cosTheta(wI)) * std::abs(cosTheta(*wi))));
    return {v, v, v};
}

} // namespace orc
