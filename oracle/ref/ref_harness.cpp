// oracle/_ref harness: the reference's own header-only kernel code, compiled
// on the host from its sources, exposed as plain C batch functions.
//
// TEST INFRASTRUCTURE ONLY.  This file includes the reference's headers in
// place (include/colvillea/libkernel/...), through the owl::common shim in
// ref/shim, and is built by oracle/ref/Makefile into oracle/_ref/libclref.so.
// Nothing of the product links it; the golden-vector generator
// (tests/golden/gen_golden.py) calls it to pin the oracle's restatement.
//
// Compiled: g++ -O2 -ffp-contract=off (IEEE FP32, no contraction), so that
// the numbers are those of the reference source evaluated in plain FP32.
// `uintToFloat` (sampler.h:39-42) is CL_GPU-only and needs
// `__uint_as_float`; the host definition below is the bit cast it names.

#include <cstdint>
#include <cstring>

static inline float __uint_as_float(unsigned int x)
{
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

#include <libkernel/base/sampler.h>
#include <libkernel/base/math.h>
#include <libkernel/base/frame.h>
#include <libkernel/base/warp.h>
#include <libkernel/base/microfacet.h>
#include <libkernel/base/bsdf.h>

using namespace colvillea::kernel;

namespace
{
// Per-item BSDF parameters, 11 floats:
//   [0..2] reflectance (diffuse) / specular reflectance (conductor)
//   [3]    alpha (GGX, conductor and dielectric)
//   [4]    interior IOR (dielectric)
//   [5..7] eta (conductor), [8..10] k (conductor)
BSDF makeBSDF(int type, const float* p)
{
    vec3f r{p[0], p[1], p[2]};
    vec3f eta{p[5], p[6], p[7]};
    vec3f k{p[8], p[9], p[10]};
    switch (type)
    {
        case 0: return BSDF{SmoothDiffuse{r}};
        case 1: return BSDF{RoughConductor{r, p[3], eta, k}};
        default: return BSDF{RoughDielectric{p[3], p[4]}};
    }
}
inline vec3f ld3(const float* p) { return vec3f{p[0], p[1], p[2]}; }
inline void  st3(float* p, const vec3f& v)
{
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}
} // namespace

extern "C" {

// pcg4d (sampler.h:16-36) on n 4-lane states.
void ref_pcg4d(const uint32_t* in, uint32_t* out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        vec4ui v{in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]};
        vec4ui r = pcg4d(v);
        out[4 * i]     = r.x;
        out[4 * i + 1] = r.y;
        out[4 * i + 2] = r.z;
        out[4 * i + 3] = r.w;
    }
}

// The first `m` draws of Sampler::next1D (sampler.h:51-55,74-77) from
// initSamplerSeed(px,py,frame) (sampler.h:64-67), for n seeds.
void ref_sampler_sequence(const uint32_t* pxpyframe, int n, int m, float* out)
{
    for (int i = 0; i < n; ++i)
    {
        vec4ui s = Sampler::initSamplerSeed(vec2ui{pxpyframe[3 * i], pxpyframe[3 * i + 1]}, pxpyframe[3 * i + 2]);
        for (int j = 0; j < m; ++j) out[i * m + j] = Sampler::next1D(s);
    }
}

void ref_bsdf_eval(int type, const float* params, const float* wo, const float* wi, float* out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        BSDF               b = makeBSDF(type, params + 11 * i);
        BSDFSamplingRecord rec;
        rec.woLocal = ld3(wo + 3 * i);
        rec.wiLocal = ld3(wi + 3 * i);
        st3(out + 3 * i, b.eval(rec));
    }
}

void ref_bsdf_pdf(int type, const float* params, const float* wo, const float* wi, float* out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        BSDF               b = makeBSDF(type, params + 11 * i);
        BSDFSamplingRecord rec;
        rec.woLocal = ld3(wo + 3 * i);
        rec.wiLocal = ld3(wi + 3 * i);
        out[i]      = b.pdf(rec);
    }
}

// BSDF::sample (bsdf.h:81-96): writes wi (3), pdf (1), value (3) per item.
// The pdf slot starts at 0 for every item (the integrator's initial value,
// raygeneration.cu:397), since SmoothDiffuse::sample leaves it untouched on
// the back side.
void ref_bsdf_sample(int type, const float* params, const float* wo, const float* u2, float* wi_out, float* pdf_out,
                     float* val_out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        BSDF               b = makeBSDF(type, params + 11 * i);
        BSDFSamplingRecord rec;
        rec.woLocal = ld3(wo + 3 * i);
        float pdf   = 0.0f;
        vec3f v     = b.sample(&rec, &pdf, vec2f{u2[2 * i], u2[2 * i + 1]});
        st3(wi_out + 3 * i, rec.wiLocal);
        pdf_out[i] = pdf;
        st3(val_out + 3 * i, v);
    }
}

// GGX: D, smithG1, G, pdfAll (microfacet.h:40-134).
void ref_ggx_eval(const float* alpha, const float* m, const float* wi, const float* wo, float* D, float* G1wi,
                  float* G, float* pdfAll, int n)
{
    for (int i = 0; i < n; ++i)
    {
        MicrofacetDistribution d{alpha[i]};
        vec3f                  mm = ld3(m + 3 * i), a = ld3(wi + 3 * i), b = ld3(wo + 3 * i);
        D[i]      = d.D(mm);
        G1wi[i]   = d.smithG1(a, mm);
        G[i]      = d.G(a, b, mm);
        pdfAll[i] = d.pdfAll(mm);
    }
}

// GGX sampleAll (microfacet.h:92-121).
void ref_ggx_sample(const float* alpha, const float* u2, float* m_out, float* pdf_out, int n)
{
    for (int i = 0; i < n; ++i)
    {
        MicrofacetDistribution d{alpha[i]};
        float                  pdf = 0.0f;
        st3(m_out + 3 * i, d.sampleAll(vec2f{u2[2 * i], u2[2 * i + 1]}, &pdf));
        pdf_out[i] = pdf;
    }
}

// fresnelConductor (math.h:172-193).
void ref_fresnel_conductor(const float* cosi, const float* eta, const float* k, float* out, int n)
{
    for (int i = 0; i < n; ++i) st3(out + 3 * i, fresnelConductor(cosi[i], ld3(eta + 3 * i), ld3(k + 3 * i)));
}

// fresnelDielectricExt (math.h:255-287).
void ref_fresnel_dielectric(const float* cosi, const float* eta, float* F, float* cost, int n)
{
    for (int i = 0; i < n; ++i)
    {
        float ct = 0.0f;
        F[i]     = fresnelDielectricExt(cosi[i], &ct, eta[i]);
        cost[i]  = ct;
    }
}

// warp (warp.h:25-64) and makeFrame (math.h:33-48).
void ref_warp(const float* u2, float* disk2, float* hemi3, int n)
{
    for (int i = 0; i < n; ++i)
    {
        vec2f s{u2[2 * i], u2[2 * i + 1]};
        vec2f d          = warp::squareToUniformConcentricDisk(s);
        disk2[2 * i]     = d.x;
        disk2[2 * i + 1] = d.y;
        st3(hemi3 + 3 * i, warp::squareToCosineHemisphere(s));
    }
}

void ref_make_frame(const float* a, float* b, float* c, int n)
{
    for (int i = 0; i < n; ++i)
    {
        vec3f bb, cc;
        makeFrame(ld3(a + 3 * i), &bb, &cc);
        st3(b + 3 * i, bb);
        st3(c + 3 * i, cc);
    }
}

// Frame::toLocal / toWorld (frame.h:47-63) with frame (s, t, n) per item.
void ref_frame(const float* s, const float* t, const float* nrm, const float* v, float* local, float* world, int n)
{
    for (int i = 0; i < n; ++i)
    {
        Frame f{ld3(s + 3 * i), ld3(t + 3 * i), ld3(nrm + 3 * i)};
        st3(local + 3 * i, f.toLocal(ld3(v + 3 * i)));
        st3(world + 3 * i, f.toWorld(ld3(v + 3 * i)));
    }
}

} // extern "C"
