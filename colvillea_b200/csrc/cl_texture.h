// Image textures: CUDA arrays read through texture objects (the reference's
// ImageTexture2D, src/core/nodes/textures/imagetex2d.cpp:8-68).
#pragma once

#include "cl_internal.h"

#include <vector>

namespace clb
{
class TextureSet
{
public:
    TextureSet() = default;
    TextureSet(const TextureSet&) = delete;
    TextureSet& operator=(const TextureSet&) = delete;
    ~TextureSet() { release(); }

    // Replaces the set; on error the set is left empty.
    cl_status build(const cl_texture_desc* d, uint32_t n, cudaStream_t st, std::string* err);
    void      release();

    uint32_t size() const { return uint32_t(objs_.size()); }
    // Device array of cudaTextureObject_t, one per texture (null when empty).
    const unsigned long long* device() const { return dev_.as<const unsigned long long>(); }

private:
    std::vector<cudaArray_t>         arrays_;
    std::vector<cudaTextureObject_t> objs_;
    DevBuf                           dev_;
};

} // namespace clb
