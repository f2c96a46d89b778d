// C ABI (include/colvillea_b200.h) over the C++ integrator.  Every entry
// point returns a status and records a message for cl_last_error; no entry
// point throws or exits (the reference exits on CUDA errors,
// src/core/devices/cudacommon.h:13-26).
#include "cl_integrator.h"

#include <atomic>

#include <cstring>
#include <memory>
#include <new>

// A guiding network: standalone (own network and stream) or the network of
// an integrator (borrowed, on the integrator's stream).
struct cl_guide
{
    clb::GuideNet*                 net = nullptr;
    std::unique_ptr<clb::GuideNet> own;
    cudaStream_t                   stream = nullptr;
    ~cl_guide()
    {
        own.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

// A radiance-cache network: standalone or an integrator's (borrowed).
struct cl_cache
{
    clb::CacheNet*                 net = nullptr;
    std::unique_ptr<clb::CacheNet> own;
    cudaStream_t                   stream = nullptr;
    ~cl_cache()
    {
        own.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

struct cl_integrator
{
    clb::Integrator impl;
    cl_cache        cacheView; // borrowed view of impl's radiance cache
    cl_guide        guideView; // borrowed view of impl's network
    cl_integrator(cl_integrator_type t, uint32_t w, uint32_t h, const cl_render_config& c) : impl(t, w, h, c) {}
};

namespace clb
{
static thread_local std::string gLastError;
void setLastError(const std::string& msg) { gLastError = msg; }

double& allocMs()
{
    static thread_local double ms = 0.0;
    return ms;
}

static std::atomic<bool> gTcSuspect{false};
bool tcSuspect() { return gTcSuspect.load(); }
void markTcSuspect() { gTcSuspect.store(true); }
cl_status refuseIfTcSuspect(std::string* err)
{
    if (!gTcSuspect.load()) return CL_OK;
    *err = "a tensor-core wait ran out earlier in this process; the CUDA context is suspect and network kernels "
           "are refused (restart the process)";
    return CL_ERR_STATE;
}

cl_status unitBsdfEval(uint32_t, const float*, const float*, const float*, float*, uint32_t, std::string*);
cl_status unitBsdfPdf(uint32_t, const float*, const float*, const float*, float*, uint32_t, uint32_t, std::string*);
cl_status unitBsdfSample(uint32_t, const float*, const float*, const float*, float*, float*, float*, uint32_t,
                         std::string*);
cl_status unitGgxEval(const float*, const float*, const float*, const float*, float*, float*, float*, float*, uint32_t,
                      std::string*);
cl_status unitGgxSample(const float*, const float*, float*, float*, uint32_t, std::string*);
cl_status unitFresnelConductor(const float*, const float*, const float*, float*, uint32_t, std::string*);
cl_status unitFresnelDielectric(const float*, const float*, float*, float*, uint32_t, std::string*);
cl_status unitWarp(const float*, float*, float*, uint32_t, std::string*);
cl_status unitMakeFrame(const float*, float*, float*, uint32_t, std::string*);
cl_status unitFrame(const float*, const float*, const float*, const float*, float*, float*, uint32_t, std::string*);
cl_status unitPcg(const uint32_t*, uint32_t*, uint32_t, std::string*);
cl_status unitNormalFrame(const float*, float*, uint32_t, std::string*);
cl_status unitTcWaitTimeout(uint64_t*, std::string*);
cl_status unitBinaryVersion(int32_t*, int32_t*, std::string*);
cl_status unitTextureLookup(const cl_texture_desc*, const float*, float*, uint32_t, std::string*);
cl_status unitSeq(const uint32_t*, uint32_t, uint32_t, float*, std::string*);
cl_status unitDomeSample(const float*, uint32_t, uint32_t, const float*, const float*, const float*, const float*,
                         const float*, float*, float*, float*, uint32_t, std::string*);
cl_status unitDomePdfEval(const float*, uint32_t, uint32_t, const float*, const float*, const float*, float*, float*,
                          uint32_t, std::string*);
cl_status unitDirectional(const float*, const float*, float*, float*, float*, uint32_t, std::string*);
} // namespace clb

namespace
{
template <class F> cl_status guarded(F&& f)
{
    std::string err;
    cl_status   s;
    try
    {
        s = f(&err);
    }
    catch (const std::bad_alloc&)
    {
        err = "host allocation failed";
        s   = CL_ERR_OOM;
    }
    catch (const std::exception& e)
    {
        err = e.what();
        s   = CL_ERR_STATE;
    }
    if (s != CL_OK)
        clb::setLastError(err.empty() ? std::string("error ") + std::to_string(s) : err);
    return s;
}

#define CL_NEED(ptr)                                                                                                   \
    do                                                                                                                 \
    {                                                                                                                  \
        if (!(ptr))                                                                                                    \
        {                                                                                                              \
            clb::setLastError(#ptr " is null");                                                                        \
            return CL_ERR_INVALID_ARG;                                                                                 \
        }                                                                                                              \
    } while (0)
} // namespace

extern "C" {

cl_status cl_integrator_create(cl_integrator_type type, uint32_t width, uint32_t height, const cl_render_config* config,
                               cl_integrator** out)
{
    CL_NEED(out);
    *out = nullptr;
    if (type != CL_INTEGRATOR_PATH_TRACING && type != CL_INTEGRATOR_DIRECT_LIGHTING)
    {
        clb::setLastError("unknown integrator type");
        return CL_ERR_INVALID_ARG;
    }
    cl_render_config cfg{5u, 0u, CL_COMPAT_ALL, 0u};
    if (config) cfg = *config;
    return guarded([&](std::string* err) -> cl_status {
        auto* it = new cl_integrator(type, width, height, cfg);
        cl_status s = it->impl.init(err);
        if (s != CL_OK)
        {
            delete it;
            return s;
        }
        *out = it;
        return CL_OK;
    });
}

cl_status cl_integrator_destroy(cl_integrator* it)
{
    delete it;
    return CL_OK;
}

cl_status cl_build_meshes(cl_integrator* it, const cl_mesh_desc* meshes, uint32_t count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.buildMeshes(meshes, count, e); });
}

cl_status cl_build_instances(cl_integrator* it, const cl_instance_desc* instances, uint32_t count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.buildInstances(instances, count, e); });
}

cl_status cl_update_mesh_vertices(cl_integrator* it, uint32_t mesh_id, const float* positions, const float* normals,
                                  const float* tangents, uint32_t num_vertices, cl_bvh_update mode)
{
    CL_NEED(it);
    return guarded([&](std::string* e) {
        return it->impl.updateMeshVertices(mesh_id, positions, normals, tangents, num_vertices, uint32_t(mode), e);
    });
}

cl_status cl_get_bvh(cl_integrator* it, void* nodes, size_t node_bytes, void* triangles, size_t triangle_bytes)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.getBvh(nodes, node_bytes, triangles, triangle_bytes, e); });
}

cl_status cl_build_textures(cl_integrator* it, const cl_texture_desc* textures, uint32_t count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.buildTextures(textures, count, e); });
}

cl_status cl_build_materials(cl_integrator* it, const cl_material_desc* materials, uint32_t count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.buildMaterials(materials, count, e); });
}

cl_status cl_build_emitters(cl_integrator* it, const cl_emitter_desc* emitters, uint32_t count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.buildEmitters(emitters, count, e); });
}

cl_status cl_update_camera(cl_integrator* it, const cl_camera* camera)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.updateCamera(camera, e); });
}

cl_status cl_render(cl_integrator* it, uint32_t spp)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.render(spp, e); });
}

cl_status cl_readback_film(cl_integrator* it, float* rgba, size_t bytes)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.readbackFilm(rgba, bytes, e); });
}

cl_status cl_readback_film_async(cl_integrator* it, float* rgba, size_t bytes)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.readbackFilmAsync(rgba, bytes, e); });
}

cl_status cl_readback_wait(cl_integrator* it)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.readbackWait(e); });
}

cl_status cl_readback_film_stats(cl_integrator* it, double* sum, double* sumsq, size_t count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.readbackFilmStats(sum, sumsq, count, e); });
}

cl_status cl_resize(cl_integrator* it, uint32_t width, uint32_t height)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.resize(width, height, e); });
}

cl_status cl_get_film_size(cl_integrator* it, uint32_t* width, uint32_t* height)
{
    CL_NEED(it);
    CL_NEED(width);
    CL_NEED(height);
    *width  = it->impl.width();
    *height = it->impl.height();
    return CL_OK;
}

cl_status cl_reset_iteration(cl_integrator* it)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.resetIteration(e); });
}

cl_status cl_set_iteration(cl_integrator* it, uint32_t iteration)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.setIteration(iteration, e); });
}

cl_status cl_get_stats(cl_integrator* it, cl_stats* stats)
{
    CL_NEED(it);
    CL_NEED(stats);
    it->impl.stats(stats);
    return CL_OK;
}

cl_status cl_last_error(char* buffer, size_t size)
{
    CL_NEED(buffer);
    if (size == 0) return CL_ERR_INVALID_ARG;
    const std::string& s = clb::gLastError;
    size_t             n = std::min(size - 1, s.size());
    memcpy(buffer, s.data(), n);
    buffer[n] = '\0';
    return CL_OK;
}

cl_status cl_trace_rays(cl_integrator* it, const float* rays, uint32_t count, float* t, uint32_t* prim, float* b1,
                        float* b2)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.traceRays(rays, count, t, prim, b1, b2, e); });
}

cl_status cl_occluded_rays(cl_integrator* it, const float* rays, uint32_t count, uint8_t* occluded)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.occludedRays(rays, count, occluded, e); });
}

cl_status cl_trace_stats(cl_integrator* it, const float* rays, uint32_t count, uint64_t* nodes, uint64_t* triangles)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.traceStats(rays, count, nodes, triangles, e); });
}

cl_status cl_get_dome_tables(cl_integrator* it, float* pU, float* cU, float* pV, float* cV)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.domeTables(pU, cU, pV, cV, e); });
}

cl_status cl_get_wave_rays(cl_integrator* it, uint64_t* rays, uint32_t capacity, uint32_t* count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.waveRays(rays, capacity, count, e); });
}

cl_status cl_integrator_guide_probe(cl_integrator* it, uint32_t capacity, float* rows, uint32_t* count)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.guideProbe(capacity, rows, count, e); });
}

cl_status cl_get_dome_alias_tables(cl_integrator* it, uint32_t* alias_row, uint32_t* alias_col)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.domeAliasTables(alias_row, alias_col, e); });
}

cl_status cl_dome_alias_sample(cl_integrator* it, const float* u2, float* dir, float* pdf, float* value, uint32_t count)
{
    CL_NEED(it);
    CL_NEED(u2);
    CL_NEED(dir);
    CL_NEED(pdf);
    CL_NEED(value);
    return guarded([&](std::string* e) { return it->impl.domeAliasSample(u2, dir, pdf, value, count, e); });
}

cl_status cl_unit_bsdf_eval(uint32_t type, const float* params, const float* wo, const float* wi, float* value,
                            uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitBsdfEval(type, params, wo, wi, value, count, e); });
}

cl_status cl_unit_bsdf_pdf(uint32_t type, const float* params, const float* wo, const float* wi, float* pdf,
                           uint32_t count, uint32_t compat)
{
    return guarded([&](std::string* e) { return clb::unitBsdfPdf(type, params, wo, wi, pdf, count, compat, e); });
}

cl_status cl_unit_bsdf_sample(uint32_t type, const float* params, const float* wo, const float* u2, float* wi,
                              float* pdf, float* value, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitBsdfSample(type, params, wo, u2, wi, pdf, value, count, e); });
}

cl_status cl_unit_ggx_eval(const float* alpha, const float* m, const float* wi, const float* wo, float* D, float* G1wi,
                           float* G, float* pdfAll, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitGgxEval(alpha, m, wi, wo, D, G1wi, G, pdfAll, count, e); });
}

cl_status cl_unit_ggx_sample(const float* alpha, const float* u2, float* m, float* pdf, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitGgxSample(alpha, u2, m, pdf, count, e); });
}

cl_status cl_unit_fresnel_conductor(const float* cos_i, const float* eta, const float* k, float* out, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitFresnelConductor(cos_i, eta, k, out, count, e); });
}

cl_status cl_unit_fresnel_dielectric(const float* cos_i, const float* eta, float* F, float* cos_t, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitFresnelDielectric(cos_i, eta, F, cos_t, count, e); });
}

cl_status cl_unit_warp(const float* u2, float* disk, float* hemisphere, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitWarp(u2, disk, hemisphere, count, e); });
}

cl_status cl_unit_make_frame(const float* a, float* b, float* c, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitMakeFrame(a, b, c, count, e); });
}

cl_status cl_unit_frame(const float* s, const float* t, const float* n, const float* v, float* local, float* world,
                        uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitFrame(s, t, n, v, local, world, count, e); });
}

cl_status cl_unit_normal_frame(const float* in, float* frame, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitNormalFrame(in, frame, count, e); });
}

cl_status cl_unit_tc_wait_timeout(uint64_t* waited_ns)
{
    return guarded([&](std::string* e) { return clb::unitTcWaitTimeout(waited_ns, e); });
}

cl_status cl_unit_binary_version(int32_t* binary_version, int32_t* ptx_version)
{
    return guarded([&](std::string* e) { return clb::unitBinaryVersion(binary_version, ptx_version, e); });
}

cl_status cl_unit_texture_lookup(const cl_texture_desc* texture, const float* uv, float* rgba, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitTextureLookup(texture, uv, rgba, count, e); });
}

cl_status cl_unit_pcg4d(const uint32_t* in, uint32_t* out, uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitPcg(in, out, count, e); });
}

cl_status cl_unit_sampler_sequence(const uint32_t* px_py_frame, uint32_t count, uint32_t draws, float* out)
{
    return guarded([&](std::string* e) { return clb::unitSeq(px_py_frame, count, draws, out, e); });
}

cl_status cl_unit_dome_sample(const float* texels, uint32_t w, uint32_t h, const float* pUcondV_c, const float* cdfU,
                              const float* pV_c, const float* cdfV, const float* u2, float* dir, float* pdf,
                              float* value, uint32_t count)
{
    return guarded([&](std::string* e) {
        return clb::unitDomeSample(texels, w, h, pUcondV_c, cdfU, pV_c, cdfV, u2, dir, pdf, value, count, e);
    });
}

cl_status cl_unit_dome_pdf_eval(const float* texels, uint32_t w, uint32_t h, const float* pUcondV_c, const float* pV_c,
                                const float* dirs, float* pdf, float* value, uint32_t count)
{
    return guarded(
        [&](std::string* e) { return clb::unitDomePdfEval(texels, w, h, pUcondV_c, pV_c, dirs, pdf, value, count, e); });
}

cl_status cl_unit_directional_sample(const float* params7, const float* u2, float* dir, float* pdf, float* value,
                                     uint32_t count)
{
    return guarded([&](std::string* e) { return clb::unitDirectional(params7, u2, dir, pdf, value, count, e); });
}

// ---- Neural path guiding ----
void cl_guide_default_config(cl_guide_config* config)
{
    if (config) clb::guideDefaultConfig(config);
}

cl_status cl_guide_default_resolutions(float n_min, float n_max, uint32_t* resolutions16)
{
    CL_NEED(resolutions16);
    cl_status s = clb::guideResolutions(n_min, n_max, resolutions16);
    if (s != CL_OK) clb::setLastError("n_min/n_max out of range");
    return s;
}

cl_status cl_guide_create(const cl_guide_config* config, cl_guide** out)
{
    CL_NEED(config);
    CL_NEED(out);
    *out = nullptr;
    return guarded([&](std::string* e) -> cl_status {
        std::unique_ptr<cl_guide> g(new cl_guide());
        if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess)
        {
            g->stream = nullptr;
            cudaGetLastError();
            *e = "cudaStreamCreate failed";
            return CL_ERR_CUDA;
        }
        g->own.reset(new clb::GuideNet(*config));
        g->net = g->own.get();
        CL_TRY(g->net->init(g->stream, e));
        *out = g.release();
        return CL_OK;
    });
}

cl_status cl_guide_destroy(cl_guide* guide)
{
    if (guide && !guide->own)
    {
        clb::setLastError("an integrator's network is destroyed with the integrator");
        return CL_ERR_INVALID_ARG;
    }
    delete guide;
    return CL_OK;
}

cl_status cl_guide_param_count(const cl_guide* guide, uint64_t* count)
{
    CL_NEED(guide);
    CL_NEED(count);
    *count = guide->net->paramCount();
    return CL_OK;
}

cl_status cl_guide_get_resolutions(const cl_guide* guide, uint32_t* resolutions16)
{
    CL_NEED(guide);
    CL_NEED(resolutions16);
    for (int l = 0; l < CL_GUIDE_LEVELS; ++l) resolutions16[l] = guide->net->resolutions()[l];
    return CL_OK;
}

cl_status cl_guide_set_params(cl_guide* guide, const float* params, uint64_t count)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { return guide->net->setParams(params, count, e); });
}

cl_status cl_guide_get_params(const cl_guide* guide, float* params, uint64_t count)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { return guide->net->getParams(params, count, e); });
}

cl_status cl_guide_forward(cl_guide* guide, const float* in9, uint32_t count, float* out48)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return guide->net->forward(in9, count, out48, e); });
}

cl_status cl_guide_gradient(cl_guide* guide, const float* rec14, uint32_t count, double* loss, float* grad)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return guide->net->gradient(rec14, count, loss, grad, e); });
}

cl_status cl_guide_train_step(cl_guide* guide, const float* rec14, uint32_t count, double* loss)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return guide->net->trainStepHost(rec14, count, loss, e); });
}

cl_status cl_guide_sample(cl_guide* guide, const float* in9, const float* u3, uint32_t count, float* dir3, float* pdf)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return guide->net->sample(in9, u3, count, dir3, pdf, e); });
}

cl_status cl_guide_pdf(cl_guide* guide, const float* in9, const float* dir3, uint32_t count, float* pdf)
{
    CL_NEED(guide);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return guide->net->pdf(in9, dir3, count, pdf, e); });
}

cl_status cl_integrator_set_guiding(cl_integrator* it, const cl_guide_config* config)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.setGuiding(config, e); });
}

cl_status cl_integrator_get_guide(cl_integrator* it, cl_guide** guide)
{
    CL_NEED(it);
    CL_NEED(guide);
    clb::GuideNet* net = it->impl.guideNet();
    if (!net)
    {
        *guide = nullptr;
        return CL_OK;
    }
    it->guideView.net    = net;
    it->guideView.stream = nullptr;
    *guide               = &it->guideView;
    return CL_OK;
}

cl_status cl_integrator_guide_stats(cl_integrator* it, cl_guide_stats* stats)
{
    CL_NEED(it);
    CL_NEED(stats);
    return guarded([&](std::string* e) { return it->impl.guideStats(stats, e); });
}

// ---- Neural radiance cache ----
void cl_radiance_cache_default_config(cl_radiance_cache_config* config)
{
    if (!config) return;
    std::memset(config, 0, sizeof(*config));
    clb::guideDefaultConfig(&config->network);
    config->network.train_spp  = 0;
    config->network.class_mask = 0;
    config->prefix_bounces      = 2;
    config->train_log2_fraction = 4;
    config->train_spp           = 32;
}

cl_status cl_cache_create(const cl_guide_config* network, cl_cache** out)
{
    CL_NEED(network);
    CL_NEED(out);
    *out = nullptr;
    return guarded([&](std::string* e) -> cl_status {
        std::unique_ptr<cl_cache> c(new cl_cache());
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        {
            c->stream = nullptr;
            cudaGetLastError();
            *e = "cudaStreamCreate failed";
            return CL_ERR_CUDA;
        }
        c->own.reset(new clb::CacheNet(*network));
        c->net = c->own.get();
        CL_TRY(c->net->init(c->stream, e));
        *out = c.release();
        return CL_OK;
    });
}

cl_status cl_cache_destroy(cl_cache* cache)
{
    if (cache && !cache->own)
    {
        clb::setLastError("an integrator's radiance cache is destroyed with the integrator");
        return CL_ERR_INVALID_ARG;
    }
    delete cache;
    return CL_OK;
}

cl_status cl_cache_param_count(const cl_cache* cache, uint64_t* count)
{
    CL_NEED(cache);
    CL_NEED(count);
    *count = cache->net->paramCount();
    return CL_OK;
}

cl_status cl_cache_get_resolutions(const cl_cache* cache, uint32_t* resolutions16)
{
    CL_NEED(cache);
    CL_NEED(resolutions16);
    for (int l = 0; l < CL_GUIDE_LEVELS; ++l) resolutions16[l] = cache->net->resolutions()[l];
    return CL_OK;
}

cl_status cl_cache_set_params(cl_cache* cache, const float* params, uint64_t count)
{
    CL_NEED(cache);
    return guarded([&](std::string* e) { return cache->net->setParams(params, count, e); });
}

cl_status cl_cache_get_params(const cl_cache* cache, float* params, uint64_t count)
{
    CL_NEED(cache);
    return guarded([&](std::string* e) { return cache->net->getParams(params, count, e); });
}

cl_status cl_cache_forward(cl_cache* cache, const float* in9, uint32_t count, float* out16)
{
    CL_NEED(cache);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return cache->net->forward(in9, count, out16, e); });
}

cl_status cl_cache_gradient(cl_cache* cache, const float* rec12, uint32_t count, double* loss, float* grad)
{
    CL_NEED(cache);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return cache->net->gradient(rec12, count, loss, grad, e); });
}

cl_status cl_cache_train_step(cl_cache* cache, const float* rec12, uint32_t count, double* loss)
{
    CL_NEED(cache);
    return guarded([&](std::string* e) { CL_TRY(clb::refuseIfTcSuspect(e)); return cache->net->trainStepHost(rec12, count, loss, e); });
}

cl_status cl_integrator_set_radiance_cache(cl_integrator* it, const cl_radiance_cache_config* config)
{
    CL_NEED(it);
    return guarded([&](std::string* e) { return it->impl.setRadianceCache(config, e); });
}

cl_status cl_integrator_get_cache(cl_integrator* it, cl_cache** cache)
{
    CL_NEED(it);
    CL_NEED(cache);
    clb::CacheNet* net = it->impl.cacheNet();
    if (!net)
    {
        *cache = nullptr;
        return CL_OK;
    }
    it->cacheView.net    = net;
    it->cacheView.stream = nullptr;
    *cache               = &it->cacheView;
    return CL_OK;
}

cl_status cl_integrator_cache_stats(cl_integrator* it, cl_guide_stats* stats)
{
    CL_NEED(it);
    CL_NEED(stats);
    return guarded([&](std::string* e) { return it->impl.cacheStats(stats, e); });
}

} // extern "C"
