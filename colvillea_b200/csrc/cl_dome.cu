// HDRI dome preprocessing on the device, in FP64.
//
// Replaces the reference's FP32 preprocessing kernels (prefiltering,
// preprocessPCondV, preprocessPV: libkernel/emitters/hdridome.h:311-432,
// src/kernel/emitters/hdridome.cu:15-51, launched by
// src/core/devices/cudadevice.h:155-177).  Outputs:
//   * the reference's tables (same layout and meaning, hdridome.h:494-510),
//     rounded to FP32 from FP64 sums: pUcondV_c and CDFpUcondV ((w+1)*h),
//     pV_c and CDFpV (h+1).  They serve the CDF sampler and every pdf lookup;
//   * alias tables for O(1) sampling of the same density: per row over
//     columns (w*h entries) and over rows (h entries), Vose's method in FP64.
// One block per row (kDomeRowTables) and one for the marginal
// (kDomeMarginalTable) with the row in shared memory: rows of up to 16,384
// texels.  Wider rows take the one-thread-per-row kernels over global
// scratch (kDomeWeights, kDomeRows, kDomeMarginal).
// Texel weights are sin(theta_v) * luminance(texel) at texel centres
// (hdridome.h:319-323, luminance weights math.h:155-158).
#include "cl_dome.h"

namespace clb
{
namespace
{
__global__ void kDomeWeights(const float4* __restrict__ tex, int w, int h, double* __restrict__ wgt)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    int v = blockIdx.y;
    if (u >= w || v >= h) return;
    float4 t     = tex[size_t(v) * w + u];
    double lum   = double(t.x) * 0.212671 + double(t.y) * 0.71516 + double(t.z) * 0.072169;
    double sinth = sin(3.14159265358979323846 * (double(v) + 0.5) / double(h));
    wgt[size_t(v) * w + u] = sinth * lum;
}

// Vose alias construction over n weights (FP64); prob/alias as uint2 {float
// bits, index}.  `small` and `large` are scratch index lists of n entries.
__device__ void voseBuild(const double* wgt, int n, double total, uint2* out, uint32_t* small, uint32_t* large,
                          double* q)
{
    if (!(total > 0.0))
    {
        for (int i = 0; i < n; ++i) out[i] = make_uint2(__float_as_uint(1.0f), uint32_t(i));
        return;
    }
    int ns = 0, nl = 0;
    for (int i = 0; i < n; ++i)
    {
        q[i] = wgt[i] * double(n) / total;
        if (q[i] < 1.0)
            small[ns++] = uint32_t(i);
        else
            large[nl++] = uint32_t(i);
    }
    while (ns > 0 && nl > 0)
    {
        uint32_t l = small[--ns];
        uint32_t g = large[--nl];
        out[l]     = make_uint2(__float_as_uint(float(q[l])), g);
        q[g]       = (q[g] + q[l]) - 1.0;
        if (q[g] < 1.0)
            small[ns++] = g;
        else
            large[nl++] = g;
    }
    while (nl > 0)
    {
        uint32_t g = large[--nl];
        out[g]     = make_uint2(__float_as_uint(1.0f), g);
    }
    while (ns > 0)
    {
        uint32_t l = small[--ns];
        out[l]     = make_uint2(__float_as_uint(1.0f), l);
    }
}

// Rows wider than the shared-memory path takes: one thread per row, FP64 row
// sums, CDF row, alias row.
__global__ void kDomeRows(const double* __restrict__ wgt, int w, int h, float* __restrict__ pU, float* __restrict__ cU,
                          double* __restrict__ rowC, uint2* __restrict__ aliasCol, uint32_t* scratchIdx,
                          double* scratchQ)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= h) return;
    const double* f   = wgt + size_t(v) * w;
    float*        p   = pU + size_t(v) * (w + 1);
    float*        c   = cU + size_t(v) * (w + 1);
    double        sum = 0.0;
    for (int i = 0; i < w; ++i) sum += f[i];
    double cv = sum / double(w);
    rowC[v]   = cv;
    if (cv > 0.0)
    {
        double acc = 0.0;
        c[0]       = 0.0f;
        for (int i = 0; i < w; ++i)
        {
            p[i] = float(f[i]);
            acc += f[i];
            c[i + 1] = float(acc / sum);
        }
        c[w] = 1.0f;
        p[w] = float(cv);
    }
    else
    {
        for (int i = 0; i < w; ++i)
        {
            p[i] = 0.0f;
            c[i] = float(i) / float(w);
        }
        c[w] = 1.0f;
        p[w] = 0.0f;
    }
    voseBuild(f, w, sum, aliasCol + size_t(v) * w, scratchIdx + size_t(v) * 2 * w, scratchIdx + size_t(v) * 2 * w + w,
              scratchQ + size_t(v) * w);
}

// Marginal over more rows than the shared-memory path takes: one thread.
__global__ void kDomeMarginal(const double* __restrict__ rowC, int h, float* __restrict__ pV, float* __restrict__ cV,
                              uint2* __restrict__ aliasRow, uint32_t* scratchIdx, double* scratchQ)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double sum = 0.0;
    for (int v = 0; v < h; ++v) sum += rowC[v];
    double c = sum / double(h);
    if (c > 0.0)
    {
        double acc = 0.0;
        cV[0]      = 0.0f;
        for (int v = 0; v < h; ++v)
        {
            pV[v] = float(rowC[v]);
            acc += rowC[v];
            cV[v + 1] = float(acc / sum);
        }
        cV[h] = 1.0f;
        pV[h] = float(c);
    }
    else
    {
        for (int v = 0; v <= h; ++v)
        {
            pV[v] = 0.0f;
            cV[v] = float(v) / float(h);
        }
    }
    voseBuild(rowC, h, sum, aliasRow, scratchIdx, scratchIdx + h, scratchQ);
}

// ---------------------------------------------------------------------------
// One table per block, in shared memory: the path for rows whose table fits
// in 227 KB (16,384 texels; the kernels above serve wider ones).
// ---------------------------------------------------------------------------
constexpr int kDomeThreads = 256;

// Shared memory of one n-entry table: q (double, n) | chunk totals (double,
// T+1) | small counts (uint32, T+1) | Vose work list (uint32, n).
size_t domeTableSmem(int n)
{
    return size_t(n) * 12 + size_t(kDomeThreads + 1) * 12;
}

// The table of the n FP64 weights in q[0, n):
//   * total: thread t sums its chunk [t*k, t*k+k) in order, thread 0 adds the
//     chunk totals in order; CDF entry i+1 is (offset of the chunk + prefix
//     within the chunk) / total, so the CDF is non-decreasing and its last
//     prefix equals the total exactly;
//   * p[0, n) = float(weights), p[n] = float(total / n), c[0] = 0, c[n] = 1
//     (all-zero weights: p = 0, c[i] = i / n), as kDomeRows/kDomeMarginal;
//   * the alias table by Vose's method on q = w * n / total, with the small
//     and large work lists in index order (one shared list: small from the
//     front, large from the back).  Thread 0 pairs them.  Both lists are
//     stacks, so an entry that changes list is the next one popped from the
//     other; the loop keeps it in registers, reads the initial lists from
//     their tops down, and writes the same table as voseBuild.
// Returns the total to every thread.
__device__ double domeTable(double* q, int n, float* __restrict__ p, float* __restrict__ c, uint2* __restrict__ alias)
{
    double*   part = q + n;
    uint32_t* cnt  = reinterpret_cast<uint32_t*>(part + kDomeThreads + 1);
    uint32_t* list = cnt + kDomeThreads + 1;
    const int t    = threadIdx.x;
    const int k    = (n + kDomeThreads - 1) / kDomeThreads;
    const int b    = min(n, t * k);
    const int e    = min(n, b + k);

    double loc = 0.0;
    for (int i = b; i < e; ++i) loc += q[i];
    part[t] = loc;
    __syncthreads();
    if (t == 0)
    {
        double off = 0.0;
        for (int j = 0; j < kDomeThreads; ++j)
        {
            double x = part[j];
            part[j]  = off;
            off += x;
        }
        part[kDomeThreads] = off;
    }
    __syncthreads();
    const double sum = part[kDomeThreads];
    const double off = part[t];
    const double cv  = sum / double(n);
    if (cv > 0.0)
    {
        double acc = 0.0;
        for (int i = b; i < e; ++i)
        {
            p[i] = float(q[i]);
            acc += q[i];
            if (i + 1 < n) c[i + 1] = float((off + acc) / sum);
        }
        if (t == 0)
        {
            c[0] = 0.0f;
            c[n] = 1.0f;
            p[n] = float(cv);
        }
    }
    else
    {
        for (int i = b; i < e; ++i)
        {
            p[i] = 0.0f;
            c[i] = float(i) / float(n);
        }
        if (t == 0)
        {
            c[n] = 1.0f;
            p[n] = 0.0f;
        }
    }
    if (!(sum > 0.0))
    {
        for (int i = b; i < e; ++i) alias[i] = make_uint2(__float_as_uint(1.0f), uint32_t(i));
        return sum;
    }

    uint32_t nsLoc = 0;
    for (int i = b; i < e; ++i)
    {
        q[i] = q[i] * double(n) / sum;
        nsLoc += q[i] < 1.0 ? 1u : 0u;
    }
    cnt[t] = nsLoc;
    __syncthreads();
    if (t == 0)
    {
        uint32_t o = 0;
        for (int j = 0; j < kDomeThreads; ++j)
        {
            uint32_t x = cnt[j];
            cnt[j]     = o;
            o += x;
        }
        cnt[kDomeThreads] = o;
    }
    __syncthreads();
    {
        uint32_t si = cnt[t], li = uint32_t(b) - cnt[t];
        for (int i = b; i < e; ++i)
        {
            if (q[i] < 1.0)
                list[si++] = uint32_t(i);
            else
                list[n - 1 - int(li++)] = uint32_t(i);
        }
    }
    __syncthreads();
    if (t != 0) return sum;

    int ns = int(cnt[kDomeThreads]), nl = n - ns;
    if (ns > 0 && nl > 0)
    {
        uint32_t l  = list[--ns];
        double   ql = q[l];
        uint32_t g  = list[n - nl];
        --nl;
        double   qg  = q[g];
        // Next entries of the two initial lists, read one step ahead.
        uint32_t sN  = ns > 0 ? list[ns - 1] : 0u;
        double   sNq = ns > 0 ? q[sN] : 0.0;
        uint32_t lN  = nl > 0 ? list[n - nl] : 0u;
        double   lNq = nl > 0 ? q[lN] : 0.0;
        for (;;)
        {
            alias[l] = make_uint2(__float_as_uint(float(ql)), g);
            qg       = (qg + ql) - 1.0;
            if (qg < 1.0)
            {
                // g turns small and is paired next.
                if (nl == 0)
                {
                    alias[g] = make_uint2(__float_as_uint(1.0f), g);
                    break;
                }
                l  = g;
                ql = qg;
                g  = lN;
                qg = lNq;
                --nl;
                if (nl > 0)
                {
                    lN  = list[n - nl];
                    lNq = q[lN];
                }
            }
            else
            {
                // g stays large and stays the top of the large list.
                if (ns == 0)
                {
                    alias[g] = make_uint2(__float_as_uint(1.0f), g);
                    break;
                }
                l  = sN;
                ql = sNq;
                --ns;
                if (ns > 0)
                {
                    sN  = list[ns - 1];
                    sNq = q[sN];
                }
            }
        }
    }
    for (int i = 0; i < ns; ++i) alias[list[i]] = make_uint2(__float_as_uint(1.0f), list[i]);
    for (int j = 0; j < nl; ++j) alias[list[n - 1 - j]] = make_uint2(__float_as_uint(1.0f), list[n - 1 - j]);
    return sum;
}

// Block v: the texel weights of row v (as kDomeWeights) into shared memory,
// then the row's tables.
__global__ void __launch_bounds__(kDomeThreads) kDomeRowTables(const float4* __restrict__ tex, int w, int h,
                                                               float* __restrict__ pU, float* __restrict__ cU,
                                                               double* __restrict__ rowC, uint2* __restrict__ aliasCol)
{
    extern __shared__ __align__(16) unsigned char domeSmem[];
    double*      q     = reinterpret_cast<double*>(domeSmem);
    const int    v     = blockIdx.x;
    const double sinth = sin(3.14159265358979323846 * (double(v) + 0.5) / double(h));
    for (int u = threadIdx.x; u < w; u += kDomeThreads)
    {
        float4 t   = tex[size_t(v) * w + u];
        double lum = double(t.x) * 0.212671 + double(t.y) * 0.71516 + double(t.z) * 0.072169;
        q[u]       = sinth * lum;
    }
    __syncthreads();
    double sum = domeTable(q, w, pU + size_t(v) * (w + 1), cU + size_t(v) * (w + 1), aliasCol + size_t(v) * w);
    if (threadIdx.x == 0) rowC[v] = sum / double(w);
}

// One block: the marginal over the row integrals.
__global__ void __launch_bounds__(kDomeThreads) kDomeMarginalTable(const double* __restrict__ rowC, int h,
                                                                   float* __restrict__ pV, float* __restrict__ cV,
                                                                   uint2* __restrict__ aliasRow)
{
    extern __shared__ __align__(16) unsigned char domeSmem[];
    double* q = reinterpret_cast<double*>(domeSmem);
    for (int v = threadIdx.x; v < h; v += kDomeThreads) q[v] = rowC[v];
    __syncthreads();
    domeTable(q, h, pV, cV, aliasRow);
}

// Largest table the shared-memory kernels take (227 KB per block).
constexpr size_t kDomeSmemMax = 227u * 1024u;

} // namespace

cl_status launchDomeBuild(const float4* dTex, int w, int h, cudaStream_t st, const DomeScratch& s, float* pU, float* cU,
                          float* pV, float* cV, uint2* aliasRow, uint2* aliasCol, std::string* err)
{
    // Rows: one block per row in shared memory when the row fits, else one
    // thread per row over the global scratch.
    const size_t smemW = domeTableSmem(w), smemH = domeTableSmem(h);
    if (smemW <= kDomeSmemMax)
    {
        if (smemW > 48u * 1024u)
            CL_CUDA(cudaFuncSetAttribute(kDomeRowTables, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemW)), err);
        kDomeRowTables<<<h, kDomeThreads, smemW, st>>>(dTex, w, h, pU, cU, s.rowC, aliasCol);
    }
    else
    {
        dim3 g((w + 127) / 128, h);
        kDomeWeights<<<g, 128, 0, st>>>(dTex, w, h, s.weights);
        kDomeRows<<<(h + 63) / 64, 64, 0, st>>>(s.weights, w, h, pU, cU, s.rowC, aliasCol, s.idx, s.q);
    }
    if (smemH <= kDomeSmemMax)
    {
        if (smemH > 48u * 1024u)
            CL_CUDA(cudaFuncSetAttribute(kDomeMarginalTable, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemH)),
                    err);
        kDomeMarginalTable<<<1, kDomeThreads, smemH, st>>>(s.rowC, h, pV, cV, aliasRow);
    }
    else
    {
        kDomeMarginal<<<1, 32, 0, st>>>(s.rowC, h, pV, cV, aliasRow, s.idx, s.q);
    }
    CL_CUDA(cudaGetLastError(), err);
    return CL_OK;
}

cl_status buildDome(const float* hostTexels, int w, int h, cudaStream_t st, DomeTables* out, std::string* err)
{
    if (w <= 0 || h <= 0 || !hostTexels)
    {
        *err = "dome: invalid texture";
        return CL_ERR_INVALID_ARG;
    }
    out->w = w;
    out->h = h;
    size_t n = size_t(w) * h;
    CL_TRY(out->tex.alloc(n * 16, err));
    CL_TRY(out->pU.alloc(size_t(w + 1) * h * 4, err));
    CL_TRY(out->cU.alloc(size_t(w + 1) * h * 4, err));
    CL_TRY(out->pV.alloc(size_t(h + 1) * 4, err));
    CL_TRY(out->cV.alloc(size_t(h + 1) * 4, err));
    CL_TRY(out->aliasRow.alloc(size_t(h) * 8, err));
    CL_TRY(out->aliasCol.alloc(n * 8, err));
    DevBuf weights, rowC, idx, q;
    CL_TRY(weights.alloc(n * 8, err));
    CL_TRY(rowC.alloc(size_t(h) * 8, err));
    CL_TRY(idx.alloc(n * 2 * 4 + size_t(h) * 2 * 4, err));
    CL_TRY(q.alloc(n * 8 + size_t(h) * 8, err));
    CL_CUDA(cudaMemcpyAsync(out->tex.p, hostTexels, n * 16, cudaMemcpyHostToDevice, st), err);
    DomeScratch s{weights.as<double>(), rowC.as<double>(), idx.u(), q.as<double>()};
    CL_TRY(launchDomeBuild(out->tex.as<float4>(), w, h, st, s, out->pU.f(), out->cU.f(), out->pV.f(), out->cV.f(),
                           out->aliasRow.as<uint2>(), out->aliasCol.as<uint2>(), err));
    CL_CUDA(cudaStreamSynchronize(st), err);
    return CL_OK;
}

} // namespace clb

// ---------------------------------------------------------------------------
// Allocation-free variant of the dome build (cl_dome_build_tables_noalloc).
//
// For callers that cannot allocate device memory: hosts whose allocator owns
// all device memory (a pool reserved at start-up), and render callbacks that
// must not allocate.
// The scratch of launchDomeBuild comes from one static device array instead
// of cudaMalloc.  In host code `gDomeScratch` names a host-side stand-in, not
// the device array, so its device address is resolved once per device with
// cudaGetSymbolAddress (with that device current) and passed to the kernels.
// ---------------------------------------------------------------------------
#include <mutex>

namespace clb
{
namespace
{
constexpr size_t kNoAllocTexels = size_t(CL_DOME_NOALLOC_MAX_TEXELS);
constexpr size_t kNoAllocRows   = size_t(CL_DOME_NOALLOC_MAX_ROWS);
// Layout: weights (double, texels) | q (double, texels + rows) |
//         rowC (double, rows) | idx (uint32, 2 texels + 2 rows).
constexpr size_t kOffQ     = 8 * kNoAllocTexels;
constexpr size_t kOffRowC  = kOffQ + 8 * (kNoAllocTexels + kNoAllocRows);
constexpr size_t kOffIdx   = kOffRowC + 8 * kNoAllocRows;
constexpr size_t kScratchB = kOffIdx + 4 * (2 * kNoAllocTexels + 2 * kNoAllocRows);
static_assert(kScratchB == size_t(CL_DOME_NOALLOC_SCRATCH_BYTES), "scratch size mismatch");

static __device__ __align__(256) unsigned char gDomeScratch[kScratchB];

constexpr int kMaxDevices = 64;
std::mutex    gScratchMutex;
// Per device: the context the address was resolved in, and the address.  A
// device address of a module variable belongs to one CUDA context, so a
// caller that makes another context current on the same device (a context
// created with the driver API, or the primary context re-created after
// cudaDeviceReset) gets the address resolved again in that context.
void*          gScratchCtx[kMaxDevices]  = {};
unsigned char* gScratchAddr[kMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry point (no link to the
// driver library); null when the driver does not provide it.
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctxGetCurrentFn()
{
    static CtxGetCurrentFn fn = [] {
        void*                           p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
        {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    return fn;
}

// Device address of gDomeScratch in the current device's current context
// (resolved on the first call per device and context).
cl_status scratchAddress(unsigned char** out, std::string* err)
{
    int dev = 0;
    CL_CUDA(cudaGetDevice(&dev), err);
    if (dev < 0 || dev >= kMaxDevices)
    {
        *err = "device index out of range";
        return CL_ERR_INVALID_ARG;
    }
    void*           ctx = nullptr;
    CtxGetCurrentFn get = ctxGetCurrentFn();
    if (get && get(&ctx) != 0) ctx = nullptr;
    std::lock_guard<std::mutex> lock(gScratchMutex);
    if (!gScratchAddr[dev] || gScratchCtx[dev] != ctx)
    {
        void*       p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, gDomeScratch);
        if (e != cudaSuccess || !p)
        {
            *err = std::string("cudaGetSymbolAddress(dome scratch): ") + cudaGetErrorString(e);
            cudaGetLastError();
            return CL_ERR_CUDA;
        }
        // The lookup makes the device's primary context current when no
        // context was: record the context it resolved the address in.
        if (get && get(&ctx) != 0) ctx = nullptr;
        gScratchAddr[dev] = static_cast<unsigned char*>(p);
        gScratchCtx[dev]  = ctx;
    }
    *out = gScratchAddr[dev];
    return CL_OK;
}

cl_status domeNoAlloc(const float* texels, uint32_t w, uint32_t h, float* pU, float* cU, float* pV, float* cV,
                      uint32_t* aliasRow, uint32_t* aliasCol, void* stream, std::string* err)
{
    if (!texels || !pU || !cU || !pV || !cV || !aliasRow || !aliasCol)
    {
        *err = "cl_dome_build_tables_noalloc: null buffer";
        return CL_ERR_INVALID_ARG;
    }
    if (w == 0 || h == 0)
    {
        *err = "cl_dome_build_tables_noalloc: empty texture";
        return CL_ERR_INVALID_ARG;
    }
    if (size_t(w) * h > kNoAllocTexels || h > kNoAllocRows)
    {
        *err = "cl_dome_build_tables_noalloc: " + std::to_string(w) + "x" + std::to_string(h) +
               " exceeds the static scratch (at most " + std::to_string(kNoAllocTexels) + " texels and " +
               std::to_string(kNoAllocRows) + " rows); use cl_build_emitters";
        return CL_ERR_INVALID_ARG;
    }
    if ((reinterpret_cast<uintptr_t>(texels) & 15u) || (reinterpret_cast<uintptr_t>(aliasRow) & 7u) ||
        (reinterpret_cast<uintptr_t>(aliasCol) & 7u))
    {
        *err = "cl_dome_build_tables_noalloc: texels must be 16-byte and alias tables 8-byte aligned";
        return CL_ERR_INVALID_ARG;
    }
    unsigned char* base = nullptr;
    CL_TRY(scratchAddress(&base, err));
    DomeScratch s{reinterpret_cast<double*>(base), reinterpret_cast<double*>(base + kOffRowC),
                  reinterpret_cast<uint32_t*>(base + kOffIdx), reinterpret_cast<double*>(base + kOffQ)};
    return launchDomeBuild(reinterpret_cast<const float4*>(texels), int(w), int(h), static_cast<cudaStream_t>(stream),
                           s, pU, cU, pV, cV, reinterpret_cast<uint2*>(aliasRow), reinterpret_cast<uint2*>(aliasCol),
                           err);
}
} // namespace
} // namespace clb

extern "C" cl_status cl_dome_build_tables_noalloc(const float* texels, uint32_t width, uint32_t height,
                                                  float* pUcondV_c, float* cdfU, float* pV_c, float* cdfV,
                                                  uint32_t* alias_row, uint32_t* alias_col, void* stream)
{
    std::string err;
    cl_status   s = clb::domeNoAlloc(texels, width, height, pUcondV_c, cdfU, pV_c, cdfV, alias_row, alias_col, stream,
                                     &err);
    if (s != CL_OK) clb::setLastError(err);
    return s;
}
