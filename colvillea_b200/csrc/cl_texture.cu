// Image textures (see cl_texture.h).
#include "cl_texture.h"

namespace clb
{
void TextureSet::release()
{
    for (cudaTextureObject_t t : objs_) cudaDestroyTextureObject(t);
    for (cudaArray_t a : arrays_) cudaFreeArray(a);
    objs_.clear();
    arrays_.clear();
    dev_.release();
}

cl_status TextureSet::build(const cl_texture_desc* d, uint32_t n, cudaStream_t st, std::string* err)
{
    release();
    if (n && !d)
    {
        *err = "textures is null";
        return CL_ERR_INVALID_ARG;
    }
    for (uint32_t i = 0; i < n; ++i)
    {
        const cl_texture_desc& t = d[i];
        std::string            tag = "texture " + std::to_string(i) + ": ";
        if (t.format > CL_TEXTURE_RGBA32F || !t.texels || t.width == 0 || t.height == 0 || t.width > 65536u ||
            t.height > 65536u || (t.srgb && t.format != CL_TEXTURE_RGBA8))
        {
            *err = tag + "needs RGBA8 or RGBA32F texels, a size in 1..65536 and sRGB only for RGBA8";
            return CL_ERR_INVALID_ARG;
        }
    }
    for (uint32_t i = 0; i < n; ++i)
    {
        const cl_texture_desc& t  = d[i];
        bool                   u8 = t.format == CL_TEXTURE_RGBA8;
        // imagetex2d.cpp:13-25: uchar4 or float4 channels.
        cudaChannelFormatDesc cd = u8 ? cudaCreateChannelDesc<uchar4>() : cudaCreateChannelDesc<float4>();
        cudaArray_t           arr = nullptr;
        cudaError_t           e   = cudaMallocArray(&arr, &cd, t.width, t.height);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            release();
            *err = "cudaMallocArray: " + std::string(cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? CL_ERR_OOM : CL_ERR_CUDA;
        }
        arrays_.push_back(arr);
        size_t row = size_t(t.width) * (u8 ? 4 : 16);
        e          = cudaMemcpy2DToArrayAsync(arr, 0, 0, t.texels, row, row, t.height, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
        {
            release();
            *err = "texture upload: " + std::string(cudaGetErrorString(e));
            return CL_ERR_CUDA;
        }
        // imagetex2d.cpp:44-64: wrap, linear, normalised coordinates, no mip maps.
        cudaResourceDesc rd{};
        rd.resType         = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td{};
        td.addressMode[0]   = cudaAddressModeWrap;
        td.addressMode[1]   = cudaAddressModeWrap;
        td.filterMode       = cudaFilterModeLinear;
        td.readMode         = u8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
        td.normalizedCoords = 1;
        td.maxAnisotropy    = 1;
        td.sRGB             = t.srgb ? 1 : 0;
        cudaTextureObject_t obj = 0;
        e                       = cudaCreateTextureObject(&obj, &rd, &td, nullptr);
        if (e != cudaSuccess)
        {
            release();
            *err = "cudaCreateTextureObject: " + std::string(cudaGetErrorString(e));
            return CL_ERR_CUDA;
        }
        objs_.push_back(obj);
    }
    if (n)
    {
        static_assert(sizeof(cudaTextureObject_t) == sizeof(unsigned long long), "texture object size");
        cl_status s = dev_.alloc(size_t(n) * 8, err);
        cudaError_t e = s == CL_OK ? cudaMemcpyAsync(dev_.p, objs_.data(), size_t(n) * 8, cudaMemcpyHostToDevice, st)
                                   : cudaSuccess;
        if (s == CL_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (s != CL_OK || e != cudaSuccess)
        {
            release();
            if (s == CL_OK) *err = "texture object upload: " + std::string(cudaGetErrorString(e));
            return s != CL_OK ? s : CL_ERR_CUDA;
        }
    }
    return CL_OK;
}

} // namespace clb
