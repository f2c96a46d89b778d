// HDRI dome tables on the device (built in FP64 by cl_dome.cu).
#pragma once

#include "cl_device.cuh"
#include "cl_internal.h"

namespace clb
{
struct DomeTables
{
    DevBuf tex;      // float4 w*h
    DevBuf pU, cU;   // float (w+1)*h
    DevBuf pV, cV;   // float h+1
    DevBuf aliasRow; // uint2 h
    DevBuf aliasCol; // uint2 w*h
    int    w = 0, h = 0;

    DomeView view() const
    {
        DomeView d;
        d.tex      = tex.as<const float4>();
        d.pU       = pU.f();
        d.cdfU     = cU.f();
        d.pV       = pV.f();
        d.cdfV     = cV.f();
        d.aliasRow = aliasRow.as<const uint2>();
        d.aliasCol = aliasCol.as<const uint2>();
        d.w        = w;
        d.h        = h;
        return d;
    }
};

// Scratch of the build: FP64 texel weights (w*h), FP64 row integrals (h),
// Vose work lists (2*w*h + 2*h indices) and FP64 scaled weights (w*h + h).
struct DomeScratch
{
    double*   weights;
    double*   rowC;
    uint32_t* idx;
    double*   q;
};

cl_status launchDomeBuild(const float4* dTex, int w, int h, cudaStream_t st, const DomeScratch& s, float* pU, float* cU,
                          float* pV, float* cV, uint2* aliasRow, uint2* aliasCol, std::string* err);

cl_status buildDome(const float* hostTexels, int w, int h, cudaStream_t st, DomeTables* out, std::string* err);

} // namespace clb
