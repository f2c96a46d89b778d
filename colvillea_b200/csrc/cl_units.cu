// Batch entry points over the device functions of cl_device.cuh, for parity
// tests against the CPU oracle: the same inlined code the integrator kernels
// run, one item per thread, host buffers in and out.
#include "cl_device.cuh"
#include "cl_internal.h"
#include "cl_mlp_tc.cuh"
#include "cl_texture.h"

#include <vector>

namespace clb
{
namespace
{
__device__ __forceinline__ f3 g3(const float* p, uint32_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void s3(float* p, uint32_t i, f3 v)
{
    p[3 * i]     = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ Bsdf bsdfParams(uint32_t type, const float* p)
{
    Bsdf b;
    b.type   = type;
    b.r      = {p[0], p[1], p[2]};
    b.alpha  = p[3];
    b.etaInt = p[4];
    b.eta    = {p[5], p[6], p[7]};
    b.k      = {p[8], p[9], p[10]};
    return b;
}

__global__ void kBsdfEval(uint32_t type, const float* params, const float* wo, const float* wi, float* out, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    s3(out, i, bsdfEval(bsdfParams(type, params + 11 * size_t(i)), g3(wo, i), g3(wi, i)));
}
__global__ void kBsdfPdf(uint32_t type, const float* params, const float* wo, const float* wi, float* out, uint32_t n,
                         bool compat)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = bsdfPdf(bsdfParams(type, params + 11 * size_t(i)), g3(wo, i), g3(wi, i), compat);
}
__global__ void kBsdfSample(uint32_t type, const float* params, const float* wo, const float* u2, float* wi, float* pdf,
                            float* val, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3    w{0.0f, 0.0f, 0.0f};
    float p = 0.0f;
    f3    v = bsdfSample(bsdfParams(type, params + 11 * size_t(i)), g3(wo, i), f2{u2[2 * i], u2[2 * i + 1]}, &w, &p);
    s3(wi, i, w);
    pdf[i] = p;
    s3(val, i, v);
}
__global__ void kGgxEval(const float* alpha, const float* m, const float* wi, const float* wo, float* D, float* G1,
                         float* G, float* pa, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    GGX d(alpha[i]);
    f3  mm = g3(m, i), a = g3(wi, i), b = g3(wo, i);
    D[i]  = d.D(mm);
    G1[i] = d.smithG1(a, mm);
    G[i]  = d.G(a, b, mm);
    pa[i] = d.pdfAll(mm);
}
__global__ void kGgxSample(const float* alpha, const float* u2, float* m, float* pdf, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    GGX   d(alpha[i]);
    float p = 0.0f;
    s3(m, i, d.sampleAll(f2{u2[2 * i], u2[2 * i + 1]}, &p));
    pdf[i] = p;
}
__global__ void kFresnelCond(const float* c, const float* eta, const float* k, float* out, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    s3(out, i, fresnelConductor(c[i], g3(eta, i), g3(k, i)));
}
__global__ void kFresnelDiel(const float* c, const float* eta, float* F, float* ct, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float t = 0.0f;
    F[i]    = fresnelDielectricExt(c[i], &t, eta[i]);
    ct[i]   = t;
}
__global__ void kWarp(const float* u2, float* disk, float* hemi, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f2 s{u2[2 * i], u2[2 * i + 1]};
    f2 d            = concentricDisk(s);
    disk[2 * i]     = d.x;
    disk[2 * i + 1] = d.y;
    s3(hemi, i, cosineHemisphere(s));
}
__global__ void kMakeFrame(const float* a, float* b, float* c, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3 bb, cc;
    makeFrame(g3(a, i), &bb, &cc);
    s3(b, i, bb);
    s3(c, i, cc);
}
__global__ void kFrame(const float* s, const float* t, const float* nn, const float* v, float* loc, float* wld, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Frame f{g3(s, i), g3(t, i), g3(nn, i)};
    s3(loc, i, f.toLocal(g3(v, i)));
    s3(wld, i, f.toWorld(g3(v, i)));
}
__global__ void kPcg(const uint32_t* in, uint32_t* out, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x = in[4 * i], y = in[4 * i + 1], z = in[4 * i + 2], w = in[4 * i + 3];
    pcg4d(x, y, z, w);
    out[4 * i]     = x;
    out[4 * i + 1] = y;
    out[4 * i + 2] = z;
    out[4 * i + 3] = w;
}
__global__ void kSeq(const uint32_t* s, uint32_t n, uint32_t m, float* out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Rng r{s[3 * i], s[3 * i + 1], s[3 * i + 2], 0u};
    for (uint32_t j = 0; j < m; ++j) out[size_t(i) * m + j] = r.next1D();
}
__global__ void kDomeSample(DomeView d, const float* u2, float* dir, float* pdf, float* val, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3    dd{0.0f, 0.0f, 0.0f};
    float p = 0.0f;
    f3    v = domeSample(d, f2{u2[2 * i], u2[2 * i + 1]}, false, &dd, &p);
    s3(dir, i, dd);
    pdf[i] = p;
    s3(val, i, v);
}
__global__ void kDomePdfEval(DomeView d, const float* dirs, float* pdf, float* val, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3 dd  = g3(dirs, i);
    pdf[i] = domePdf(d, dd);
    s3(val, i, domeEval(d, dd));
}
__global__ void kDirectional(DirectionalLight e, const float* u2, float* dir, float* pdf, float* val, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3    dd{0.0f, 0.0f, 0.0f};
    float p = 0.0f;
    f3    v = directionalSample(e, f2{u2[2 * i], u2[2 * i + 1]}, &dd, &p);
    s3(dir, i, dd);
    pdf[i] = p;
    s3(val, i, v);
}

// Device staging for a batch call: inputs copied in, outputs copied back.
struct Batch
{
    std::vector<DevBuf*>            bufs;
    std::vector<std::pair<void*, DevBuf*>> outs;
    std::string*                    err;
    explicit Batch(std::string* e) : err(e) {}
    ~Batch()
    {
        for (auto* b : bufs) delete b;
    }
    template <class T> cl_status in(const T* host, size_t count, T** dev)
    {
        auto* b = new DevBuf();
        bufs.push_back(b);
        CL_TRY(b->alloc(count * sizeof(T), err));
        CL_CUDA(cudaMemcpy(b->p, host, count * sizeof(T), cudaMemcpyHostToDevice), err);
        *dev = b->as<T>();
        return CL_OK;
    }
    template <class T> cl_status out(T* host, size_t count, T** dev)
    {
        auto* b = new DevBuf();
        bufs.push_back(b);
        CL_TRY(b->alloc(count * sizeof(T), err));
        CL_CUDA(cudaMemset(b->p, 0, count * sizeof(T)), err);
        outs.push_back({host, b});
        b->bytes = count * sizeof(T);
        *dev     = b->as<T>();
        return CL_OK;
    }
    cl_status finish()
    {
        CL_CUDA(cudaGetLastError(), err);
        CL_CUDA(cudaDeviceSynchronize(), err);
        for (auto& o : outs) CL_CUDA(cudaMemcpy(o.first, o.second->p, o.second->bytes, cudaMemcpyDeviceToHost), err);
        return CL_OK;
    }
};

inline uint32_t grid(uint32_t n) { return (n + 127) / 128; }

// The tensor-core kernels' bounded mbarrier wait on a barrier that nothing
// arrives at: out[0] = 1 when the wait returned false (ran out), out[1..2] =
// the nanoseconds waited.
__global__ void kMbarTimeout(uint32_t* out)
{
    __shared__ __align__(8) unsigned long long bar;
    const uint32_t                             a = guide::smemAddr(&bar);
    guide::mbarInit(a, 1u);
    const uint64_t t0 = guide::globalTimerNs();
    const bool     ok = guide::mbarWait(a, 0u);
    const uint64_t dt = guide::globalTimerNs() - t0;
    out[0]            = ok ? 0u : 1u;
    out[1]            = uint32_t(dt);
    out[2]            = uint32_t(dt >> 32);
}

} // namespace

#define CL_REQ(cond)                                                                                                   \
    do                                                                                                                 \
    {                                                                                                                  \
        if (!(cond))                                                                                                   \
        {                                                                                                              \
            *err = "invalid argument: " #cond;                                                                         \
            return CL_ERR_INVALID_ARG;                                                                                 \
        }                                                                                                              \
    } while (0)

cl_status unitBsdfEval(uint32_t type, const float* params, const float* wo, const float* wi, float* value, uint32_t n,
                       std::string* err)
{
    CL_REQ(type <= 2u && params && wo && wi && value);
    if (!n) return CL_OK;
    Batch  b(err);
    float *p, *a, *c, *o;
    CL_TRY(b.in(params, 11 * size_t(n), &p));
    CL_TRY(b.in(wo, 3 * size_t(n), &a));
    CL_TRY(b.in(wi, 3 * size_t(n), &c));
    CL_TRY(b.out(value, 3 * size_t(n), &o));
    kBsdfEval<<<grid(n), 128>>>(type, p, a, c, o, n);
    return b.finish();
}

cl_status unitBsdfPdf(uint32_t type, const float* params, const float* wo, const float* wi, float* pdf, uint32_t n,
                      uint32_t compat, std::string* err)
{
    CL_REQ(type <= 2u && params && wo && wi && pdf);
    if (!n) return CL_OK;
    Batch  b(err);
    float *p, *a, *c, *o;
    CL_TRY(b.in(params, 11 * size_t(n), &p));
    CL_TRY(b.in(wo, 3 * size_t(n), &a));
    CL_TRY(b.in(wi, 3 * size_t(n), &c));
    CL_TRY(b.out(pdf, size_t(n), &o));
    kBsdfPdf<<<grid(n), 128>>>(type, p, a, c, o, n, compat != 0);
    return b.finish();
}

cl_status unitBsdfSample(uint32_t type, const float* params, const float* wo, const float* u2, float* wi, float* pdf,
                         float* value, uint32_t n, std::string* err)
{
    CL_REQ(type <= 2u && params && wo && u2 && wi && pdf && value);
    if (!n) return CL_OK;
    Batch  b(err);
    float *p, *a, *u, *w, *q, *v;
    CL_TRY(b.in(params, 11 * size_t(n), &p));
    CL_TRY(b.in(wo, 3 * size_t(n), &a));
    CL_TRY(b.in(u2, 2 * size_t(n), &u));
    CL_TRY(b.out(wi, 3 * size_t(n), &w));
    CL_TRY(b.out(pdf, size_t(n), &q));
    CL_TRY(b.out(value, 3 * size_t(n), &v));
    kBsdfSample<<<grid(n), 128>>>(type, p, a, u, w, q, v, n);
    return b.finish();
}

cl_status unitGgxEval(const float* alpha, const float* m, const float* wi, const float* wo, float* D, float* G1,
                      float* G, float* pa, uint32_t n, std::string* err)
{
    CL_REQ(alpha && m && wi && wo && D && G1 && G && pa);
    if (!n) return CL_OK;
    Batch  b(err);
    float *al, *mm, *a, *c, *d, *g1, *g, *p;
    CL_TRY(b.in(alpha, n, &al));
    CL_TRY(b.in(m, 3 * size_t(n), &mm));
    CL_TRY(b.in(wi, 3 * size_t(n), &a));
    CL_TRY(b.in(wo, 3 * size_t(n), &c));
    CL_TRY(b.out(D, n, &d));
    CL_TRY(b.out(G1, n, &g1));
    CL_TRY(b.out(G, n, &g));
    CL_TRY(b.out(pa, n, &p));
    kGgxEval<<<grid(n), 128>>>(al, mm, a, c, d, g1, g, p, n);
    return b.finish();
}

cl_status unitGgxSample(const float* alpha, const float* u2, float* m, float* pdf, uint32_t n, std::string* err)
{
    CL_REQ(alpha && u2 && m && pdf);
    if (!n) return CL_OK;
    Batch  b(err);
    float *al, *u, *mm, *p;
    CL_TRY(b.in(alpha, n, &al));
    CL_TRY(b.in(u2, 2 * size_t(n), &u));
    CL_TRY(b.out(m, 3 * size_t(n), &mm));
    CL_TRY(b.out(pdf, n, &p));
    kGgxSample<<<grid(n), 128>>>(al, u, mm, p, n);
    return b.finish();
}

cl_status unitFresnelConductor(const float* c, const float* eta, const float* k, float* out, uint32_t n, std::string* err)
{
    CL_REQ(c && eta && k && out);
    if (!n) return CL_OK;
    Batch  b(err);
    float *cc, *e, *kk, *o;
    CL_TRY(b.in(c, n, &cc));
    CL_TRY(b.in(eta, 3 * size_t(n), &e));
    CL_TRY(b.in(k, 3 * size_t(n), &kk));
    CL_TRY(b.out(out, 3 * size_t(n), &o));
    kFresnelCond<<<grid(n), 128>>>(cc, e, kk, o, n);
    return b.finish();
}

cl_status unitFresnelDielectric(const float* c, const float* eta, float* F, float* ct, uint32_t n, std::string* err)
{
    CL_REQ(c && eta && F && ct);
    if (!n) return CL_OK;
    Batch  b(err);
    float *cc, *e, *f, *t;
    CL_TRY(b.in(c, n, &cc));
    CL_TRY(b.in(eta, n, &e));
    CL_TRY(b.out(F, n, &f));
    CL_TRY(b.out(ct, n, &t));
    kFresnelDiel<<<grid(n), 128>>>(cc, e, f, t, n);
    return b.finish();
}

cl_status unitWarp(const float* u2, float* disk, float* hemi, uint32_t n, std::string* err)
{
    CL_REQ(u2 && disk && hemi);
    if (!n) return CL_OK;
    Batch  b(err);
    float *u, *d, *h;
    CL_TRY(b.in(u2, 2 * size_t(n), &u));
    CL_TRY(b.out(disk, 2 * size_t(n), &d));
    CL_TRY(b.out(hemi, 3 * size_t(n), &h));
    kWarp<<<grid(n), 128>>>(u, d, h, n);
    return b.finish();
}

cl_status unitMakeFrame(const float* a, float* bb, float* cc, uint32_t n, std::string* err)
{
    CL_REQ(a && bb && cc);
    if (!n) return CL_OK;
    Batch  b(err);
    float *x, *y, *z;
    CL_TRY(b.in(a, 3 * size_t(n), &x));
    CL_TRY(b.out(bb, 3 * size_t(n), &y));
    CL_TRY(b.out(cc, 3 * size_t(n), &z));
    kMakeFrame<<<grid(n), 128>>>(x, y, z, n);
    return b.finish();
}

cl_status unitFrame(const float* s, const float* t, const float* nn, const float* v, float* loc, float* wld, uint32_t n,
                    std::string* err)
{
    CL_REQ(s && t && nn && v && loc && wld);
    if (!n) return CL_OK;
    Batch  b(err);
    float *a, *c, *d, *e, *f, *g;
    CL_TRY(b.in(s, 3 * size_t(n), &a));
    CL_TRY(b.in(t, 3 * size_t(n), &c));
    CL_TRY(b.in(nn, 3 * size_t(n), &d));
    CL_TRY(b.in(v, 3 * size_t(n), &e));
    CL_TRY(b.out(loc, 3 * size_t(n), &f));
    CL_TRY(b.out(wld, 3 * size_t(n), &g));
    kFrame<<<grid(n), 128>>>(a, c, d, e, f, g, n);
    return b.finish();
}

// in: 16 floats per item {wo, dpdu, dpdv, nb, texel rgb, pullUp}; out: 9 {s, t, n}.
__global__ void kNormalFrame(const float* in, float* out, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = in + 16 * size_t(i);
    f3    wo{p[0], p[1], p[2]}, du{p[3], p[4], p[5]}, dv{p[6], p[7], p[8]}, nb{p[9], p[10], p[11]};
    f3    tx{p[12], p[13], p[14]};
    Frame f = normalMappedFrame(wo, du, dv, nb, tx, p[15] != 0.0f);
    float* o = out + 9 * size_t(i);
    o[0] = f.s.x; o[1] = f.s.y; o[2] = f.s.z;
    o[3] = f.t.x; o[4] = f.t.y; o[5] = f.t.z;
    o[6] = f.n.x; o[7] = f.n.y; o[8] = f.n.z;
}

__global__ void kTexLookup(const unsigned long long* tex, const float* uv, float4* out, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = tex2D<float4>(cudaTextureObject_t(tex[0]), uv[2 * size_t(i)], uv[2 * size_t(i) + 1]);
}

cl_status unitNormalFrame(const float* in, float* out, uint32_t n, std::string* err)
{
    CL_REQ(in && out);
    if (!n) return CL_OK;
    Batch  b(err);
    float *x, *y;
    CL_TRY(b.in(in, 16 * size_t(n), &x));
    CL_TRY(b.out(out, 9 * size_t(n), &y));
    kNormalFrame<<<grid(n), 128>>>(x, y, n);
    return b.finish();
}

cl_status unitTcWaitTimeout(uint64_t* waitedNs, std::string* err)
{
    CL_REQ(waitedNs);
    Batch     b(err);
    uint32_t  h[3] = {0u, 0u, 0u};
    uint32_t* d;
    CL_TRY(b.out(h, 3, &d));
    kMbarTimeout<<<1, 1>>>(d);
    CL_TRY(b.finish());
    *waitedNs = uint64_t(h[1]) | (uint64_t(h[2]) << 32);
    if (h[0])
    {
        *err = "tensor-core wait ran out (expected: nothing arrives at the barrier)";
        return CL_ERR_TIMEOUT;
    }
    return CL_OK;
}

cl_status unitBinaryVersion(int32_t* binaryVersion, int32_t* ptxVersion, std::string* err)
{
    CL_REQ(binaryVersion && ptxVersion);
    cudaFuncAttributes a{};
    CL_CUDA(cudaFuncGetAttributes(&a, kMbarTimeout), err);
    *binaryVersion = a.binaryVersion;
    *ptxVersion    = a.ptxVersion;
    return CL_OK;
}

cl_status unitTextureLookup(const cl_texture_desc* t, const float* uv, float* rgba, uint32_t n, std::string* err)
{
    CL_REQ(t && uv && rgba);
    if (!n) return CL_OK;
    TextureSet ts;
    CL_TRY(ts.build(t, 1, nullptr, err));
    Batch  b(err);
    float *u, *o;
    CL_TRY(b.in(uv, 2 * size_t(n), &u));
    CL_TRY(b.out(rgba, 4 * size_t(n), &o));
    kTexLookup<<<grid(n), 128>>>(ts.device(), u, reinterpret_cast<float4*>(o), n);
    return b.finish();
}

cl_status unitPcg(const uint32_t* in, uint32_t* out, uint32_t n, std::string* err)
{
    CL_REQ(in && out);
    if (!n) return CL_OK;
    Batch     b(err);
    uint32_t *i, *o;
    CL_TRY(b.in(in, 4 * size_t(n), &i));
    CL_TRY(b.out(out, 4 * size_t(n), &o));
    kPcg<<<grid(n), 128>>>(i, o, n);
    return b.finish();
}

cl_status unitSeq(const uint32_t* s, uint32_t n, uint32_t m, float* out, std::string* err)
{
    CL_REQ(s && out && m <= 4096u);
    if (!n || !m) return CL_OK;
    Batch     b(err);
    uint32_t* i;
    float*    o;
    CL_TRY(b.in(s, 3 * size_t(n), &i));
    CL_TRY(b.out(out, size_t(n) * m, &o));
    kSeq<<<grid(n), 128>>>(i, n, m, o);
    return b.finish();
}

cl_status unitDomeSample(const float* texels, uint32_t w, uint32_t h, const float* pU, const float* cU, const float* pV,
                         const float* cV, const float* u2, float* dir, float* pdf, float* val, uint32_t n,
                         std::string* err)
{
    CL_REQ(texels && w && h && pU && cU && pV && cV && u2 && dir && pdf && val);
    if (!n) return CL_OK;
    Batch  b(err);
    float *t, *a, *c, *d, *e, *u, *o1, *o2, *o3;
    CL_TRY(b.in(texels, 4 * size_t(w) * h, &t));
    CL_TRY(b.in(pU, size_t(w + 1) * h, &a));
    CL_TRY(b.in(cU, size_t(w + 1) * h, &c));
    CL_TRY(b.in(pV, size_t(h + 1), &d));
    CL_TRY(b.in(cV, size_t(h + 1), &e));
    CL_TRY(b.in(u2, 2 * size_t(n), &u));
    CL_TRY(b.out(dir, 3 * size_t(n), &o1));
    CL_TRY(b.out(pdf, n, &o2));
    CL_TRY(b.out(val, 3 * size_t(n), &o3));
    DomeView dv{};
    dv.tex  = reinterpret_cast<const float4*>(t);
    dv.pU   = a;
    dv.cdfU = c;
    dv.pV   = d;
    dv.cdfV = e;
    dv.w    = int(w);
    dv.h    = int(h);
    kDomeSample<<<grid(n), 128>>>(dv, u, o1, o2, o3, n);
    return b.finish();
}

cl_status unitDomePdfEval(const float* texels, uint32_t w, uint32_t h, const float* pU, const float* pV,
                          const float* dirs, float* pdf, float* val, uint32_t n, std::string* err)
{
    CL_REQ(texels && w && h && pU && pV && dirs && pdf && val);
    if (!n) return CL_OK;
    Batch  b(err);
    float *t, *a, *d, *x, *o2, *o3;
    CL_TRY(b.in(texels, 4 * size_t(w) * h, &t));
    CL_TRY(b.in(pU, size_t(w + 1) * h, &a));
    CL_TRY(b.in(pV, size_t(h + 1), &d));
    CL_TRY(b.in(dirs, 3 * size_t(n), &x));
    CL_TRY(b.out(pdf, n, &o2));
    CL_TRY(b.out(val, 3 * size_t(n), &o3));
    DomeView dv{};
    dv.tex = reinterpret_cast<const float4*>(t);
    dv.pU  = a;
    dv.pV  = d;
    dv.w   = int(w);
    dv.h   = int(h);
    kDomePdfEval<<<grid(n), 128>>>(dv, x, o2, o3, n);
    return b.finish();
}

cl_status unitDirectional(const float* p7, const float* u2, float* dir, float* pdf, float* val, uint32_t n,
                          std::string* err)
{
    CL_REQ(p7 && u2 && dir && pdf && val);
    if (!n) return CL_OK;
    Batch  b(err);
    float *u, *o1, *o2, *o3;
    CL_TRY(b.in(u2, 2 * size_t(n), &u));
    CL_TRY(b.out(dir, 3 * size_t(n), &o1));
    CL_TRY(b.out(pdf, n, &o2));
    CL_TRY(b.out(val, 3 * size_t(n), &o3));
    DirectionalLight e{{p7[0], p7[1], p7[2]}, {p7[3], p7[4], p7[5]}, p7[6]};
    kDirectional<<<grid(n), 128>>>(e, u, o1, o2, o3, n);
    return b.finish();
}

} // namespace clb
