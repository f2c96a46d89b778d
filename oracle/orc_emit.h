// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's emitters (directional cone light, HDRI
// dome with its 2-D piecewise-constant CDF sampler), the RGBA32F bilinear
// texture lookup, the triangle hit-attribute computation and the ray-triangle
// test.  See orc_core.h for the rules this restatement follows.
#pragma once

#include <cstring>

#include "orc_core.h"

#include <vector>

namespace orc
{
// ---------------------------------------------------------------------------
// Texture lookup: tex2D<float4> on an RGBA32F array with wrap addressing,
// linear filtering and normalised coordinates (imagetex2d.h:34-37, texture
// description imagetex2d.cpp:51-65).  The hardware filter is replaced by
// this FP32 definition, used identically on the GPU.
// ---------------------------------------------------------------------------
inline int wrapIndex(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

inline V3<float> texBilinear(const float* rgba, int w, int h, float u, float v)
{
    u       = u - std::floor(u);
    v       = v - std::floor(v);
    float x = u * float(w) - 0.5f;
    float y = v * float(h) - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    float ax = x - fx, ay = y - fy;
    int   ix = int(fx), iy = int(fy);
    int   x0 = wrapIndex(ix, w), x1 = wrapIndex(ix + 1, w);
    int   y0 = wrapIndex(iy, h), y1 = wrapIndex(iy + 1, h);
    const float* t00 = rgba + 4 * (size_t(y0) * w + x0);
    const float* t10 = rgba + 4 * (size_t(y0) * w + x1);
    const float* t01 = rgba + 4 * (size_t(y1) * w + x0);
    const float* t11 = rgba + 4 * (size_t(y1) * w + x1);
    float bx = 1.0f - ax, by = 1.0f - ay;
    V3<float> out;
    for (int c = 0; c < 3; ++c)
    {
        float top = t00[c] * bx + t10[c] * ax;
        float bot = t01[c] * bx + t11[c] * ax;
        out[c]    = top * by + bot * ay;
    }
    return out;
}

// ---------------------------------------------------------------------------
// Material image textures (ImageTexture2D, imagetex2d.cpp:8-68): texture
// objects with linear filtering, wrap addressing and normalised coordinates,
// read through the GPU's texture unit (the reference's path and the
// product's).  The unit's filter as measured on B200
// (tests/golden/texture_unit.npz):
//   x = frac(u) * w - 0.5 in FP32, texel floor(x) (wrapped);
//   a = frac(x) in 1/256 steps, rounded half up (b likewise for y);
//   texel weights (256-a)(256-b), a(256-b), (256-a)b, ab in 1/65536 steps,
//   rounded to 1/256 steps: half up for the first and last, half down for
//   the middle two (they sum to 256);
//   RGBA32F: sum of weight * texel;
//   RGBA8: S = sum of weight * byte, result round(S * 257/256) / 65535
//   (16-bit UNORM).
// The unit computes x at a slightly different precision: where frac(x) * 256
// is within about 1e-3 of a half step, a (or b) can differ by one step
// (about 0.1% of lookups).  sRGB textures are not reproduced: the unit's
// decode and blend are quantised differently; this model decodes each texel
// with the IEC 61966-2-1 curve and blends in double (measured absolute
// difference at most 0.007 on [0, 1]).
// ---------------------------------------------------------------------------
struct Texture
{
    int         format; // 0 RGBA8, 1 RGBA32F
    int         w, h, srgb;
    const void* texels;
};
struct F4
{
    float v[4];
};

inline int weight8(float f)
{
    float s = f * 256.0f, fl = std::floor(s);
    return int(fl) + (s - fl >= 0.5f ? 1 : 0);
}

inline F4 texUnit(const Texture& t, float u, float v)
{
    float x = (u - std::floor(u)) * float(t.w) - 0.5f;
    float y = (v - std::floor(v)) * float(t.h) - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    int   a = weight8(x - fx), b = weight8(y - fy);
    int   x0 = wrapIndex(int(fx), t.w), x1 = wrapIndex(int(fx) + 1, t.w);
    int   y0 = wrapIndex(int(fy), t.h), y1 = wrapIndex(int(fy) + 1, t.h);
    // products in 1/65536 steps -> 1/256 steps (p + 128) >> 8 half up, (p + 127) >> 8 half down
    int    wt[4] = {((256 - a) * (256 - b) + 128) >> 8, (a * (256 - b) + 127) >> 8, ((256 - a) * b + 127) >> 8,
                    (a * b + 128) >> 8};
    size_t idx[4] = {size_t(y0) * t.w + x0, size_t(y0) * t.w + x1, size_t(y1) * t.w + x0, size_t(y1) * t.w + x1};
    F4     out;
    for (int c = 0; c < 4; ++c)
    {
        if (t.format == 1)
        {
            const float* p = static_cast<const float*>(t.texels);
            double       s = 0.0;
            for (int k = 0; k < 4; ++k) s += double(wt[k]) * double(p[4 * idx[k] + c]);
            out.v[c] = float(s / 256.0);
        }
        else
        {
            const uint8_t* p = static_cast<const uint8_t*>(t.texels);
            if (t.srgb && c < 3)
            {
                double s = 0.0;
                for (int k = 0; k < 4; ++k)
                {
                    double e = double(p[4 * idx[k] + c]) / 255.0;
                    s += double(wt[k]) * (e <= 0.04045 ? e / 12.92 : std::pow((e + 0.055) / 1.055, 2.4));
                }
                out.v[c] = float(s / 256.0);
            }
            else
            {
                long S = 0;
                for (int k = 0; k < 4; ++k) S += long(wt[k]) * long(p[4 * idx[k] + c]);
                out.v[c] = float(double((S * 257 + 128) >> 8) / 65535.0);
            }
        }
    }
    return out;
}

// linearToLuminance (math.h:155-158): evaluated in double, returned as float.
inline float luminance(V3<float> c) { return float(double(c.x) * 0.212671 + double(c.y) * 0.71516 + double(c.z) * 0.072169); }

// ---------------------------------------------------------------------------
// HDRI dome (emitters/hdridome.h).  Tables laid out as the reference:
// pUcondV_c and CDFpUcondV (w+1)*h, pV_c and CDFpV h+1.
// ---------------------------------------------------------------------------
struct Dome
{
    int          w = 0, h = 0;
    const float* texels = nullptr; // RGBA32F, w*h
    const float* pUcondV_c = nullptr;
    const float* cdfU      = nullptr;
    const float* pV_c      = nullptr;
    const float* cdfV      = nullptr;
    // Alias tables of the B200 build (not in the reference): {prob bits,
    // alias} per row (h entries) and per column of each row (w*h entries).
    const uint32_t* aliasRow = nullptr;
    const uint32_t* aliasCol = nullptr;
};

// Preprocessing, FP32, in the reference's order: prefiltering
// (hdridome.h:311-324), preprocessPCondV (:333-385), preprocessPV (:387-432).
inline void buildDomeTables(const float* texels, int w, int h, std::vector<float>& pU, std::vector<float>& cU,
                            std::vector<float>& pV, std::vector<float>& cV)
{
    const int W1 = w + 1;
    pU.assign(size_t(W1) * h, 0.0f);
    cU.assign(size_t(W1) * h, 0.0f);
    pV.assign(h + 1, 0.0f);
    cV.assign(h + 1, 0.0f);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            float u        = (float(x) + 0.5f) / float(w);
            float v        = (float(y) + 0.5f) / float(h);
            float sinTheta = std::sin(kPiF * (float(y) + 0.5f) / float(h));
            pU[size_t(y) * W1 + x] = sinTheta * luminance(texBilinear(texels, w, h, u, v));
        }
    for (int y = 0; y < h; ++y)
    {
        float* p = &pU[size_t(y) * W1];
        float* c = &cU[size_t(y) * W1];
        c[0]     = 0.0f;
        for (int i = 1; i < w + 1; ++i) c[i] = c[i - 1] + p[i - 1] / float(w);
        float csum = c[w];
        p[w]       = csum;
        if (csum <= 0.0f)
        {
            for (int i = 0; i < w; ++i)
            {
                p[i] = 0.0f;
                c[i] = float(i) / float(w);
            }
            c[w] = 1.0f;
            p[w] = 0.0f;
        }
        else
            for (int i = 0; i < w + 1; ++i) c[i] = c[i] / csum;
        pV[y] = csum;
    }
    // preprocessPV: every job j in [0, h] reads pV[0..h-1] only.
    std::vector<float> cdfOut(h + 1), pvOut(pV);
    for (int j = 0; j <= h; ++j)
    {
        float sum = 0.0f, c = 0.0f;
        for (int i = 1; i <= h; ++i)
        {
            if (i <= j) sum += pV[i - 1];
            c += pV[i - 1];
        }
        cdfOut[j] = sum / float(h);
        c         = c / float(h);
        if (j == h) pvOut[h] = c;
        if (c <= 0.0f)
        {
            pvOut[j]  = 0.0f;
            cdfOut[j] = float(j) / float(h);
        }
        else
            cdfOut[j] = cdfOut[j] / c;
    }
    pV = pvOut;
    cV = cdfOut;
}

// upper_bound (math.h:84-96) over [begin, end).
inline uint32_t upperBound(const float* a, uint32_t begin, uint32_t end, float value)
{
    while (begin < end)
    {
        uint32_t middle = begin + (end - begin) / 2;
        if (a[middle] <= value)
            begin = middle + 1;
        else
            end = middle;
    }
    return begin;
}

// Distribution1D::sample1D (hdridome.h:30-60).
inline float sample1D(const float* f, const float* cdf, uint32_t N, float c, float u, uint32_t cdfOffset, float* pdf,
                      uint32_t* sampledOffset)
{
    if (c == 0.0f) return 0.0f;
    uint32_t off = upperBound(cdf, cdfOffset, cdfOffset + N + 1, u);
    off          = off - 1;
    off          = off < cdfOffset ? cdfOffset : (off > cdfOffset + N - 1 ? cdfOffset + N - 1 : off);
    *pdf         = f[off] / c;
    float du     = u - cdf[off];
    if (cdf[off + 1] - cdf[off] != 0.0f) du = du / (cdf[off + 1] - cdf[off]);
    off            = off - cdfOffset;
    *sampledOffset = off;
    return (float(off) + du) / float(N);
}

// Distribution2D::sample2D (hdridome.h:95-123).
inline V2<float> sample2D(const Dome& d, V2<float> r, float* pdf)
{
    float    px = 0.0f, py = 0.0f;
    uint32_t off = 0;
    V2<float> pt{0.0f, 0.0f};
    pt.y = sample1D(d.pV_c, d.cdfV, uint32_t(d.h), d.pV_c[d.h], r.y, 0, &py, &off);
    uint32_t W1 = uint32_t(d.w) + 1;
    pt.x        = sample1D(d.pUcondV_c, d.cdfU, uint32_t(d.w), d.pUcondV_c[size_t(off) * W1 + d.w], r.x, off * W1, &px, &off);
    *pdf        = px * py;
    return pt;
}

// Distribution2D::pdf2D (hdridome.h:125-135).
inline float pdf2D(const Dome& d, V2<float> s)
{
    if (s.x < 0.f || s.y < 0.f) return 0.0f;
    uint32_t tu = uint32_t(float(d.w) * s.x);
    uint32_t tv = uint32_t(float(d.h) * s.y);
    tu          = tu > uint32_t(d.w) - 1 ? uint32_t(d.w) - 1 : tu;
    tv          = tv > uint32_t(d.h) - 1 ? uint32_t(d.h) - 1 : tv;
    return d.pUcondV_c[size_t(tv) * (d.w + 1) + tu] / d.pV_c[d.h];
}

// Two-level alias sampling over the same density (the GPU's dome sampler,
// not in the reference; restated here from colvillea_b200's device code, so
// that same-seed renders with alias sampling can be compared).  Rows by the
// marginal table, then columns by the row's table; each level takes one
// uniform: integer part = bucket, fraction = coin and, rescaled, the offset
// inside the chosen cell.  pdf is the CDF sampler's (same table values).
inline float bitsToFloat(uint32_t b)
{
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
inline V2<float> sample2DAlias(const Dome& d, V2<float> r, float* pdf)
{
    float    yv = r.y * float(d.h);
    uint32_t i  = std::min(uint32_t(yv), uint32_t(d.h) - 1);
    float    fr = yv - float(i);
    float    p  = bitsToFloat(d.aliasRow[2 * size_t(i)]);
    uint32_t row;
    float    dv;
    if (fr < p)
    {
        row = i;
        dv  = fr / p;
    }
    else
    {
        row = d.aliasRow[2 * size_t(i) + 1];
        dv  = (fr - p) / (1.0f - p);
    }
    float    xv = r.x * float(d.w);
    uint32_t j  = std::min(uint32_t(xv), uint32_t(d.w) - 1);
    float    fc = xv - float(j);
    size_t   e  = size_t(row) * d.w + j;
    float    q  = bitsToFloat(d.aliasCol[2 * e]);
    uint32_t col;
    float    du;
    if (fc < q)
    {
        col = j;
        du  = fc / q;
    }
    else
    {
        col = d.aliasCol[2 * e + 1];
        du  = (fc - q) / (1.0f - q);
    }
    du = std::fmin(du, 0.99999994f);
    dv = std::fmin(dv, 0.99999994f);
    V2<float> uv{(float(col) + du) / float(d.w), (float(row) + dv) / float(d.h)};
    *pdf = d.pUcondV_c[size_t(row) * (d.w + 1) + col] / d.pV_c[d.h];
    return uv;
}

// acos argument of a direction's y: `clampY` (corrected estimator) keeps
// directions whose y rounded past +-1 on the sphere; the reference passes y
// unclamped (NaN there), reproduced by the compat estimator.
inline float cosY(float y, bool clampY) { return clampY ? std::fmin(std::fmax(y, -1.0f), 1.0f) : y; }

// directionToUVCoords (hdridome.h:472-476).
inline V2<float> dirToUV(V3<float> dir, bool clampY = false)
{
    return {std::atan2(dir.x, dir.z) * -kInvPi * 0.5f + 0.5f, std::acos(cosY(dir.y, clampY)) * kInvPi};
}

// evalEnvironment (hdridome.h:291-297).
inline V3<float> domeEval(const Dome& d, V3<float> dir, bool clampY = false)
{
    V2<float> uv = dirToUV(dir, clampY);
    return texBilinear(d.texels, d.w, d.h, uv.x, uv.y);
}

// HDRIDome::pdfDirect (hdridome.h:248-279), IMPORTANCE_SAMPLING on (Q11).
inline float domePdf(const Dome& d, V3<float> dir, bool clampY = false)
{
    float phi      = std::atan2(dir.x, dir.z);
    float theta    = std::acos(cosY(dir.y, clampY));
    float sinTheta = std::sin(theta);
    if (sinTheta == 0.0f) return 0.0f;
    V2<float> uv{phi * -kInvPi * 0.5f + 0.5f, theta * kInvPi};
    return pdf2D(d, uv) / (2.0f * kPiF * kPiF * sinTheta);
}

// HDRIDome::sampleDirect (hdridome.h:186-228).
inline V3<float> domeSample(const Dome& d, V2<float> u, V3<float>* dir, float* pdf, bool alias = false)
{
    V2<float> uv       = alias ? sample2DAlias(d, u, pdf) : sample2D(d, u, pdf);
    float     theta    = kPiF * uv.y;
    float     phi      = -2 * kPiF * (uv.x - 0.5f);
    float     sinTheta = std::sin(theta), cosTheta = std::cos(theta);
    float     sinPhi = std::sin(phi), cosPhi = std::cos(phi);
    if (sinTheta == 0.0f)
    {
        *pdf = 0.0f;
        return {0.0f, 0.0f, 0.0f};
    }
    *dir = {sinTheta * sinPhi, cosTheta, sinTheta * cosPhi}; // warp.h:16-22
    *pdf = *pdf / (2.0f * kPiF * kPiF * sinTheta);
    return texBilinear(d.texels, d.w, d.h, uv.x, uv.y);
}

// ---------------------------------------------------------------------------
// Directional emitter (emitters/directional.h:30-66).
// ---------------------------------------------------------------------------
struct Directional
{
    V3<float> intensity, direction;
    float     angularRadius;
};

inline V3<float> directionalSample(const Directional& e, V2<float> u, V3<float>* dir, float* pdf)
{
    V3<float> rev  = -e.direction;
    V2<float> disk = concentricDisk(u);
    float     tr   = std::tan(e.angularRadius);
    disk           = {disk.x * tr, disk.y * tr};
    V3<float> ax, ay;
    makeFrame(rev, &ax, &ay);
    V3<float> d       = rev + ax * disk.x;
    d                 = d + ay * disk.y;
    *dir              = normalize(d);
    float tanTheta    = std::sqrt(disk.x * disk.x + disk.y * disk.y);
    float cosTheta    = 1.0f / std::sqrt(1.0f + tanTheta * tanTheta);
    float tanR        = std::tan(e.angularRadius);
    *pdf              = kInvPi / (tanR * tanR * cosTheta * cosTheta * cosTheta);
    return e.intensity;
}

// ---------------------------------------------------------------------------
// Ray-triangle test.  Watertight algorithm of Woop, Benthin and Wald (JCGT
// 2013): shear into a ray-aligned frame, signed edge functions with a
// double-precision re-evaluation when an edge function is exactly 0.
// Replaces OptiX's built-in triangle test (optix.cu:64-74); the product's
// traversal kernels evaluate the identical FP32 sequence.
// ---------------------------------------------------------------------------
struct RayPre
{
    V3<float> o;
    int       kx, ky, kz;
    float     Sx, Sy, Sz;
};

inline RayPre rayPrepare(V3<float> o, V3<float> d)
{
    RayPre r;
    r.o      = o;
    float ax = std::abs(d.x), ay = std::abs(d.y), az = std::abs(d.z);
    r.kz     = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    r.kx     = r.kz + 1 == 3 ? 0 : r.kz + 1;
    r.ky     = r.kx + 1 == 3 ? 0 : r.kx + 1;
    if (d[r.kz] < 0.0f) std::swap(r.kx, r.ky);
    r.Sx = d[r.kx] / d[r.kz];
    r.Sy = d[r.ky] / d[r.kz];
    r.Sz = 1.0f / d[r.kz];
    return r;
}

// Returns true with t, b1, b2 when the ray plane-crosses inside the
// triangle (edges inclusive) with det != 0; the t-range test is the caller's.
inline bool intersectTri(const RayPre& r, V3<float> v0, V3<float> v1, V3<float> v2, float* t, float* b1, float* b2)
{
    V3<float> A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
    float     Ax = A[r.kx] - r.Sx * A[r.kz], Ay = A[r.ky] - r.Sy * A[r.kz];
    float     Bx = B[r.kx] - r.Sx * B[r.kz], By = B[r.ky] - r.Sy * B[r.kz];
    float     Cx = C[r.kx] - r.Sx * C[r.kz], Cy = C[r.ky] - r.Sy * C[r.kz];
    float     U = Cx * By - Cy * Bx;
    float     V = Ax * Cy - Ay * Cx;
    float     W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f)
    {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float Az = r.Sz * A[r.kz], Bz = r.Sz * B[r.kz], Cz = r.Sz * C[r.kz];
    float T  = U * Az + V * Bz + W * Cz;
    float rcp = 1.0f / det;
    *t        = T * rcp;
    *b1       = V * rcp;
    *b2       = W * rcp;
    return true;
}

// ---------------------------------------------------------------------------
// Hit attributes (closest-hit program, optix.cu:137-227).
// ---------------------------------------------------------------------------
struct MeshView
{
    const float*    pos;  // 3 per vertex
    const float*    nrm;  // 3 per vertex or null
    const float*    tan;  // 3 per vertex (required, optix.cu:187-188)
    const float*    uv;   // 2 per vertex or null
    const uint32_t* idx;  // 3 per triangle (global vertex ids)
};

struct HitAttr
{
    V3<float> p, ng, ns, dpdu, dpdv;
    V2<float> uv;
};

inline V3<float> ld3(const float* p, uint32_t i) { return {p[3 * size_t(i)], p[3 * size_t(i) + 1], p[3 * size_t(i) + 2]}; }

inline HitAttr hitAttributes(const MeshView& m, uint32_t prim, float b1, float b2)
{
    uint32_t  i0 = m.idx[3 * size_t(prim)], i1 = m.idx[3 * size_t(prim) + 1], i2 = m.idx[3 * size_t(prim) + 2];
    V3<float> p0 = ld3(m.pos, i0), p1 = ld3(m.pos, i1), p2 = ld3(m.pos, i2);
    float     b0 = 1.0f - b1 - b2;
    HitAttr   a;
    a.p = b0 * p0 + b1 * p1;
    a.p = a.p + b2 * p2;
    if (m.uv)
    {
        const float* u = m.uv;
        a.uv = {b0 * u[2 * i0] + b1 * u[2 * i1] + b2 * u[2 * i2], b0 * u[2 * i0 + 1] + b1 * u[2 * i1 + 1] + b2 * u[2 * i2 + 1]};
    }
    else
        a.uv = {b0, b1};
    V3<float> Ng = normalize(cross(p1 - p0, p2 - p0));
    V3<float> Ns;
    if (m.nrm)
    {
        V3<float> n = b0 * ld3(m.nrm, i0) + b1 * ld3(m.nrm, i1);
        n           = n + b2 * ld3(m.nrm, i2);
        Ns          = normalize(n);
    }
    else
        Ns = normalize(Ng);
    if (dot(Ns, Ns) == 0.0f) Ns = Ng;
    if (dot(Ng, Ns) < 0.0f) Ng = -Ng;
    V3<float> t    = b0 * ld3(m.tan, i0) + b1 * ld3(m.tan, i1);
    t              = t + b2 * ld3(m.tan, i2);
    V3<float> dpdu = normalize(t);
    V3<float> dpdv{0.0f, 0.0f, 0.0f};
    if (dot(dpdu, dpdu) > 0.0f)
    {
        dpdv = cross(Ns, dpdu);
        if (dot(dpdv, dpdv) > 0.0f)
        {
            dpdv = normalize(dpdv);
            dpdu = cross(dpdv, Ns);
        }
        else
            makeFrame(Ns, &dpdu, &dpdv);
    }
    else
        makeFrame(Ns, &dpdu, &dpdv);
    a.ng   = Ng;
    a.ns   = Ns;
    a.dpdu = dpdu;
    a.dpdv = dpdv;
    return a;
}

} // namespace orc
