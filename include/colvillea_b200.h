/*
 * colvillea_b200 — C ABI of the B200 (sm_100a) wavefront path tracer.
 *
 * This is the drop-in boundary for Colvillea's integrator layer.  It replaces
 * the C++ interface `colvillea::core::Integrator`
 * (include/colvillea/librender/integrator.h:34-103) and its factory
 * `Integrator::createIntegrator` (src/core/librender/integrator.cpp:10-22),
 * implemented in the reference by WavefrontPathTracingIntegrator
 * (src/core/integrators/path.{h,cpp}) and WavefrontDirectLightingIntegrator
 * (src/core/integrators/direct.{h,cpp}) on top of OptiX/OWL.
 *
 * Conventions
 *   - Every call returns cl_status (CL_OK == 0).  Nothing calls exit(); the
 *     reference's CHECK_CUDA_CALL -> exit(-1) (src/core/devices/cudacommon.h:13-26)
 *     becomes an error code plus a message from cl_last_error().
 *   - Inputs are caller-owned host arrays, copied during the call
 *     (as the reference copies build* inputs, src/core/integrators/path.cpp:53-82).
 *   - One host thread per integrator; calls are blocking, like the
 *     reference's synchronous launches (src/core/devices/cudadevice.h:185-219).
 *     Each integrator owns one CUDA stream on the current device.
 *   - No torch or CUDA types appear in this header: plain pointers and sizes.
 */
#ifndef COLVILLEA_B200_H
#define COLVILLEA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t cl_status;
enum
{
    CL_OK                 = 0,
    CL_ERR_CUDA           = 1, /* a CUDA runtime call failed */
    CL_ERR_OOM            = 2, /* device allocation failed */
    CL_ERR_QUEUE_OVERFLOW = 3, /* a work queue would have overflowed; items were dropped */
    CL_ERR_TIMEOUT        = 4, /* a bounded device-side wait ran out (see below) */
    CL_ERR_INVALID_ARG    = 5, /* bad argument (null, size, index out of range) */
    CL_ERR_STATE          = 6  /* call out of order (e.g. render before the scene is built) */
};
/* CL_ERR_TIMEOUT from a render or a network call means a tensor-core kernel
 * stopped waiting for its own matrix operations after about one second and
 * released its tensor memory while an operation may still have been in
 * flight.  Treat the CUDA context as suspect and restart the process; the
 * integrator refuses further renders with a network (CL_ERR_STATE).  The test
 * entry point cl_unit_tc_wait_timeout issues no tensor-core operation and
 * leaves the context usable. */

/* IntegratorType (include/colvillea/librender/integrator.h:22-32). */
typedef enum
{
    CL_INTEGRATOR_DIRECT_LIGHTING = 1, /* WavefrontDirectLighting */
    CL_INTEGRATOR_PATH_TRACING    = 2  /* WavefrontPathTracing */
} cl_integrator_type;

/* Render configuration flags. */
enum
{
    /* Reproduce the reference's pdf functions as written, which differ from
     * the densities their sample functions draw from: RoughConductor::pdf
     * returns pdfAll(wo) (roughconductor.h), SmoothDiffuse::pdf cos(wo) / pi
     * (smoothdiffuse.h) and RoughDielectric::pdf carries an extra cos(H)
     * factor (roughdielectric.h). */
    CL_COMPAT_PDF = 1u << 0,
    /* Path tracing: shading frame normal = geometric normal, as the reference's
     * swapped getShadingFrame arguments (raygeneration.cu:324-330). */
    CL_COMPAT_FRAME = 1u << 1,
    /* The reference's MIS / escaped-ray bookkeeping: emitter value scaled by
     * the emitter count with the unscaled pdf in the weight, indirect rays only
     * where the dome pdf is non-zero, and the BSDF weight applied twice to
     * escaped indirect rays (raygeneration.cu:357,417,429-452,131). */
    CL_COMPAT_ESCAPE = 1u << 2,
    CL_COMPAT_ALL    = (1u << 0) | (1u << 1) | (1u << 2),
    /* Sample the HDRI dome with the FP64-built alias tables instead of the
     * reference's CDF binary search (same pdf values). */
    CL_DOME_ALIAS = 1u << 4,
    /* Keep an FP64 per-pixel film (sum and sum of squares of per-sample path
     * radiance) next to the FP32 film. */
    CL_FILM_FP64 = 1u << 5,
    /* Time each wavefront stage with CUDA events (cl_get_stats). */
    CL_PROFILE_STAGES = 1u << 6,
    /* Count BVH nodes visited and triangles tested by the traversal kernels
     * of each render (cl_get_stats); slower, for roofline accounting. */
    CL_TRACE_STATS = 1u << 7,
    /* Two-level scene: one 8-wide BVH per mesh in object space and one over
     * the instances' world boxes; rays enter an instance's tree mapped to
     * object space (instancing without flattening; no counterpart in the
     * reference, whose TLAS has no transforms, optix.cu:115).  Without it the
     * instances are flattened into one world-space tree. */
    CL_TWO_LEVEL = 1u << 8
};

typedef struct
{
    uint32_t max_depth;      /* ray segments per path (reference: 5, path.cpp:135) */
    uint32_t rr_start_depth; /* Russian roulette from this path depth on; 0 = off */
    uint32_t flags;          /* CL_COMPAT_*, CL_DOME_ALIAS, CL_FILM_FP64, CL_PROFILE_STAGES, CL_TRACE_STATS,
                                CL_TWO_LEVEL */
    uint32_t path_slots;     /* paths in flight; 0 = automatic (2^21); at most 2^28 - 1 */
} cl_render_config;

/* A triangle mesh (TriMesh, include/colvillea/libkernel/shapes/trimesh.h:16-32).
 * positions/normals/tangents: 3 floats per vertex; uvs: 2 floats per vertex;
 * indices: 3 uint32 per triangle.  Tangents are required (optix.cu:187-188);
 * normals and uvs may be null (Ns = Ng, uv = barycentrics, optix.cu:146-172). */
typedef struct
{
    const float*    positions;
    const float*    normals;
    const float*    tangents;
    const float*    uvs;
    uint32_t        num_vertices;
    const uint32_t* indices;
    uint32_t        num_triangles;
} cl_mesh_desc;

/* An entity: mesh instance + material (kernel::Entity, libkernel/base/entity.h:24-31,
 * with a row-major 3x4 object-to-world transform; the reference has none). */
typedef struct
{
    uint32_t mesh_id;
    uint32_t material_index;
    float    transform[12];
} cl_instance_desc;

/* Material (MaterialType, libkernel/base/material.h:24-37) in the reference's
 * units: Diffuse{reflectance}; Metal{specular reflectance, roughness, eta, k};
 * Glass{roughness, interior IOR}.  GGX alpha = roughness^2 (metal.h:52, glass.h:26). */
enum
{
    CL_MATERIAL_DIFFUSE = 0,
    CL_MATERIAL_METAL   = 1,
    CL_MATERIAL_GLASS   = 2
};
typedef struct
{
    uint32_t type;
    float    reflectance[3];
    float    roughness;
    float    interior_ior;
    float    eta[3];
    float    k[3];
    /* Textures: 1-based indices into the last cl_build_textures, 0 = none.
     * A texture replaces the constant (DiffuseMtl/MetalMtl::getBSDF,
     * libkernel/materials/diffusemtl.h:20-29, metal.h:37-55):
     *   reflectance_texture  rgb: diffuse reflectance or metal specular
     *                        reflectance (not glass);
     *   roughness_texture    red channel: metal roughness, squared to the GGX
     *                        alpha like the constant (metal only);
     *   normal_texture       tangent-space normal map, n = rgb * 2 - 1, any
     *                        type (Material::setNormalmap, material.h:91). */
    uint32_t reflectance_texture;
    uint32_t roughness_texture;
    uint32_t normal_texture;
} cl_material_desc;

/* Image textures (the reference's ImageTexture2D,
 * src/core/nodes/textures/imagetex2d.cpp:8-68): each one a CUDA array read
 * through a texture object with bilinear filtering, wrap addressing in u and
 * v, normalised coordinates and no mip maps.  RGBA8 texels are read as
 * normalised floats, decoded from sRGB to linear by the texture unit before
 * filtering when `srgb` is set; RGBA32F texels as floats.  Lookups use the
 * hit's uv (interpolated vertex uvs, or the barycentrics (b0, b1) for meshes
 * without uvs, optix.cu:164); texel row 0 is v = 0. */
enum
{
    CL_TEXTURE_RGBA8   = 0,
    CL_TEXTURE_RGBA32F = 1
};
typedef struct
{
    uint32_t    format; /* CL_TEXTURE_* */
    uint32_t    width;
    uint32_t    height;
    uint32_t    srgb;   /* RGBA8 only */
    const void* texels; /* width*height texels, 4 channels, rows of width */
} cl_texture_desc;

/* Emitter (EmitterType, libkernel/base/emitter.h:16-26).  Directional:
 * intensity, direction (from the light), angular radius (directional.h:19-22).
 * Dome: RGBA32F texels (width*height*4 floats, row-major, v down from +Y). */
enum
{
    CL_EMITTER_DIRECTIONAL = 0,
    CL_EMITTER_HDRI_DOME   = 1
};
typedef struct
{
    uint32_t     type;
    float        intensity[3];
    float        direction[3];
    float        angular_radius;
    const float* texels;
    uint32_t     width;
    uint32_t     height;
} cl_emitter_desc;

/* Camera (include/colvillea/librender/nodebase/camera.h:8-27). */
typedef struct
{
    float pos[3];
    float d00[3];
    float ddu[3];
    float ddv[3];
} cl_camera;

typedef struct
{
    uint64_t paths;          /* camera paths completed, all renders */
    uint64_t rays_closest;   /* closest-hit segments traced */
    uint64_t rays_shadow;    /* shadow rays traced */
    uint32_t iteration;      /* progressive frame index (path.cpp:220) */
    uint32_t spp;            /* samples accumulated in the film */
    uint32_t bvh_nodes;      /* 8-wide BVH nodes */
    uint32_t bvh_depth;      /* 8-wide BVH depth */
    uint32_t triangles;
    uint32_t waves;          /* wavefront iterations in the last render */
    float    ms_bvh_build;
    float    ms_dome_build;
    float    ms_last_render; /* device time of the last cl_render */
    float    ms_trace;       /* last render, CL_PROFILE_STAGES: the closest-hit traversal kernel */
    float    ms_shade;       /* ... shading-class queues and shading kernels */
    float    ms_shadow;      /* ... shadow kernels */
    uint32_t launches;       /* last render: closest-hit kernel launches */
    uint32_t pad;
    uint64_t trace_nodes;    /* last render, CL_TRACE_STATS: closest-hit nodes visited */
    uint64_t trace_tris;     /* ... closest-hit triangles tested */
    uint64_t shadow_nodes;   /* ... shadow-ray nodes visited */
    uint64_t shadow_tris;    /* ... shadow-ray triangles tested */
    uint64_t last_rays_closest; /* last render: closest-hit segments */
    uint64_t last_rays_shadow;  /* last render: shadow rays */
    float    ms_bvh_update;     /* last cl_update_mesh_vertices: device time of the refit and/or rebuild */
    float    ms_bvh_refit;      /* ... of its refit alone (0: none) */
    uint32_t bvh_refits;        /* refits since the integrator was created */
    uint32_t bvh_rebuilds;      /* rebuilds after vertex updates */
    double   bvh_sah;           /* surface-area cost of the current tree (root = 1) */
    double   bvh_sah_build;     /* ... right after its last full build */
    float    ms_bvh_build_wall; /* last full build: host wall time (allocations, launches and waits) */
    float    ms_bvh_build_alloc; /* ... of which in device allocation */
} cl_stats;

typedef struct cl_integrator cl_integrator;

/* Integrator::createIntegrator (src/core/librender/integrator.cpp:10-22). */
cl_status cl_integrator_create(cl_integrator_type type, uint32_t width, uint32_t height,
                               const cl_render_config* config, cl_integrator** out);
cl_status cl_integrator_destroy(cl_integrator* integrator);

/* Integrator::buildBLAS (integrator.h:47). */
cl_status cl_build_meshes(cl_integrator* integrator, const cl_mesh_desc* meshes, uint32_t count);
/* Integrator::buildTLAS + buildGeometryEntities (integrator.h:49-54): builds the
 * 8-wide BVH on the device over all instances. */
cl_status cl_build_instances(cl_integrator* integrator, const cl_instance_desc* instances, uint32_t count);
/* Shape edit: new vertex positions (and optionally normals and tangents) for
 * mesh `mesh_id` of the last cl_build_meshes, same vertex count, same
 * triangles.  The reference's TriangleMesh::updateVertices
 * (include/colvillea/nodes/shapes/trianglemesh.h:111-118, marks ShapeEdited)
 * followed by RenderEngine::compileAccelStructs
 * (src/core/librender/renderengine.cpp:65-77), which rebuilds the BLAS and
 * calls resetIterationIndex.  Every instance of the mesh is re-flattened
 * with its transform; then the BVH is
 *   CL_BVH_UPDATE_REFIT    refitted: same tree, boxes recomputed bottom-up
 *                          on the device (exact boxes, requantised);
 *   CL_BVH_UPDATE_REBUILD  rebuilt from scratch, as the reference does;
 *   CL_BVH_UPDATE_AUTO     refitted, then rebuilt if the refitted tree's
 *                          surface-area cost exceeds 1.5x the cost right
 *                          after its last build (cl_stats.bvh_sah*).
 * The progressive iteration restarts (film cleared).  Positions must be
 * finite.  Normals/tangents null: kept. */
typedef enum
{
    CL_BVH_UPDATE_AUTO    = 0,
    CL_BVH_UPDATE_REFIT   = 1,
    CL_BVH_UPDATE_REBUILD = 2
} cl_bvh_update;
cl_status cl_update_mesh_vertices(cl_integrator* integrator, uint32_t mesh_id, const float* positions,
                                  const float* normals, const float* tangents, uint32_t num_vertices,
                                  cl_bvh_update mode);
/* The built 8-wide BVH for inspection: nodes (bvh_nodes * 80 bytes, layout
 * of cl_bvh.cuh: 5 x uint4 per node) and leaf triangles (triangles * 48
 * bytes: 3 float4 each, {v0.xyz, prim id bits} {v1.xyz, 0} {v2.xyz, 0}).
 * Either pointer may be null.  No counterpart in the reference. */
cl_status cl_get_bvh(cl_integrator* integrator, void* nodes, size_t node_bytes, void* triangles,
                     size_t triangle_bytes);
/* Textures created by the scene before materials refer to them
 * (Scene::createTexture, scene.h:151-160; compiled with the materials,
 * RenderEngine::compileMaterials).  Replaces all textures; materials keep
 * their indices. */
cl_status cl_build_textures(cl_integrator* integrator, const cl_texture_desc* textures, uint32_t count);
/* Integrator::buildMaterials (integrator.h:52). */
cl_status cl_build_materials(cl_integrator* integrator, const cl_material_desc* materials, uint32_t count);
/* Integrator::buildEmitters (integrator.h:56-58): the last dome in the list is
 * the environment; its sampling tables are built on the device in FP64. */
cl_status cl_build_emitters(cl_integrator* integrator, const cl_emitter_desc* emitters, uint32_t count);
/* Integrator::updateCamera (integrator.h:80): resets accumulation on change
 * (src/core/integrators/path.h:73-80). */
cl_status cl_update_camera(cl_integrator* integrator, const cl_camera* camera);
/* Integrator::render (integrator.h:61): `spp` progressive iterations.  Within
 * one call the paths of the next iteration start in the slots that finished
 * paths free, so several iterations per call keep the device busy where one
 * per call ends with small draining waves (config 2: 350 Mpaths/s at 1 spp
 * per call, 400 at 64). */
cl_status cl_render(cl_integrator* integrator, uint32_t spp);
/* Integrator::readbackFramebuffer (integrator.h:72): linear HDR mean radiance,
 * RGBA32F, width*height*4 floats (alpha = 1). */
cl_status cl_readback_film(cl_integrator* integrator, float* rgba, size_t bytes);
/* The same readback, returning once it is queued: the mean is staged on the
 * device and copied into `rgba` on a copy stream, so that the copy overlaps
 * the next cl_render.  `rgba` must stay valid (and is best page-locked) until
 * cl_readback_wait returns; a later readback of either kind waits for this
 * one's copy before reusing the staging buffer.  No counterpart in the
 * reference. */
cl_status cl_readback_film_async(cl_integrator* integrator, float* rgba, size_t bytes);
cl_status cl_readback_wait(cl_integrator* integrator);
/* FP64 film (CL_FILM_FP64): per-pixel sum and sum of squares, 3 doubles each. */
cl_status cl_readback_film_stats(cl_integrator* integrator, double* sum, double* sumsq, size_t count);
/* Integrator::resize / getFilmSize / resetIterationIndex (integrator.h:64,74,76). */
cl_status cl_resize(cl_integrator* integrator, uint32_t width, uint32_t height);
cl_status cl_get_film_size(cl_integrator* integrator, uint32_t* width, uint32_t* height);
cl_status cl_reset_iteration(cl_integrator* integrator);
/* Like cl_reset_iteration, but the next render continues from progressive
 * frame `iteration` (the sampler's frame key): independent render seeds for
 * the same scene.  No counterpart in the reference. */
cl_status cl_set_iteration(cl_integrator* integrator, uint32_t iteration);
cl_status cl_get_stats(cl_integrator* integrator, cl_stats* stats);
/* Profiling (CL_PROFILE_STAGES; no counterpart in the reference): the
 * closest-hit rays traced by each wave of the last render, in launch order
 * (the units of each closest-hit kernel launch).  Writes up to `capacity`
 * counts; *count = the number of waves. */
cl_status cl_get_wave_rays(cl_integrator* integrator, uint64_t* rays, uint32_t capacity, uint32_t* count);
/* Last error message of the calling thread. */
cl_status cl_last_error(char* buffer, size_t size);

/* ---- Ray queries on a built scene (OptiX trace replacement, optix.cu:38-110).
 * rays: 8 floats each {o.xyz, tmin, d.xyz, tmax}.  Closest hit in (tmin, tmax);
 * miss: prim = 0xffffffff.  prim is the triangle's global id in instance order. */
cl_status cl_trace_rays(cl_integrator* integrator, const float* rays, uint32_t count, float* t, uint32_t* prim,
                        float* b1, float* b2);
cl_status cl_occluded_rays(cl_integrator* integrator, const float* rays, uint32_t count, uint8_t* occluded);
/* Traversal statistics over the given rays: wide nodes visited and triangles
 * tested, summed (closest-hit kernel). */
cl_status cl_trace_stats(cl_integrator* integrator, const float* rays, uint32_t count, uint64_t* nodes,
                         uint64_t* triangles);
/* The dome's sampling tables as used by the device (reference layout,
 * hdridome.h:494-510): pUcondV_c and CDFpUcondV (w+1)*h, pV_c and CDFpV h+1. */
cl_status cl_get_dome_tables(cl_integrator* integrator, float* pUcondV_c, float* cdfU, float* pV_c, float* cdfV);
/* The dome's alias tables (CL_DOME_ALIAS sampling; no counterpart in the
 * reference): alias_row 2*h uint32 {prob bits, row}, alias_col 2*w*h uint32
 * {prob bits, column}.  Either pointer may be NULL. */
cl_status cl_get_dome_alias_tables(cl_integrator* integrator, uint32_t* alias_row, uint32_t* alias_col);

/* ---- Device functions on batches (the exact device code the integrator runs).
 * BSDF params: 11 floats per item {r.xyz, alpha, interior IOR, eta.xyz, k.xyz};
 * type: CL_MATERIAL_* (BSDFType, libkernel/base/bsdf.h:17-30). */
cl_status cl_unit_bsdf_eval(uint32_t type, const float* params, const float* wo, const float* wi, float* value,
                            uint32_t count);
cl_status cl_unit_bsdf_pdf(uint32_t type, const float* params, const float* wo, const float* wi, float* pdf,
                           uint32_t count, uint32_t compat);
cl_status cl_unit_bsdf_sample(uint32_t type, const float* params, const float* wo, const float* u2, float* wi,
                              float* pdf, float* value, uint32_t count);
cl_status cl_unit_ggx_eval(const float* alpha, const float* m, const float* wi, const float* wo, float* D, float* G1wi,
                           float* G, float* pdfAll, uint32_t count);
cl_status cl_unit_ggx_sample(const float* alpha, const float* u2, float* m, float* pdf, uint32_t count);
cl_status cl_unit_fresnel_conductor(const float* cos_i, const float* eta, const float* k, float* out, uint32_t count);
cl_status cl_unit_fresnel_dielectric(const float* cos_i, const float* eta, float* F, float* cos_t, uint32_t count);
cl_status cl_unit_warp(const float* u2, float* disk, float* hemisphere, uint32_t count);
cl_status cl_unit_make_frame(const float* a, float* b, float* c, uint32_t count);
cl_status cl_unit_frame(const float* s, const float* t, const float* n, const float* v, float* local, float* world,
                        uint32_t count);
/* Normal-mapped shading frame (Material::getShadingFrameImpl with a normal
 * map, material.h:164-221, and fixNormalPerturbingShadingFrame,
 * material.h:238-285): per item 16 floats {wo, dpdu, dpdv, base normal,
 * normal-map texel rgb, pull-up (0 or 1)}; out 9 floats {s, t, n}. */
cl_status cl_unit_normal_frame(const float* in, float* frame, uint32_t count);
/* The bounded wait of the tensor-core network kernels (an mbarrier wait of at
 * most about one second) on a barrier that nothing arrives at: returns
 * CL_ERR_TIMEOUT with the time waited, and the context stays usable.  No
 * counterpart in the reference; it tests the failure path without a fault. */
cl_status cl_unit_tc_wait_timeout(uint64_t* waited_ns);
/* Target of the library's device code as the CUDA runtime reports it for one
 * of its kernels (cudaFuncGetAttributes: binaryVersion 100 = sm_100a SASS).
 * No counterpart in the reference. */
cl_status cl_unit_binary_version(int32_t* binary_version, int32_t* ptx_version);
/* Lookups in one texture set up like the integrator's: uv pairs in, RGBA out. */
cl_status cl_unit_texture_lookup(const cl_texture_desc* texture, const float* uv, float* rgba, uint32_t count);
cl_status cl_unit_pcg4d(const uint32_t* in, uint32_t* out, uint32_t count);
cl_status cl_unit_sampler_sequence(const uint32_t* px_py_frame, uint32_t count, uint32_t draws, float* out);
/* HDRI dome against caller tables (reference layout): CDF sampling, pdf, eval. */
cl_status cl_unit_dome_sample(const float* texels, uint32_t w, uint32_t h, const float* pUcondV_c, const float* cdfU,
                              const float* pV_c, const float* cdfV, const float* u2, float* dir, float* pdf,
                              float* value, uint32_t count);
cl_status cl_unit_dome_pdf_eval(const float* texels, uint32_t w, uint32_t h, const float* pUcondV_c,
                                const float* pV_c, const float* dirs, float* pdf, float* value, uint32_t count);
/* Directional emitter: params {intensity.xyz, direction.xyz, angular radius}. */
cl_status cl_unit_directional_sample(const float* params7, const float* u2, float* dir, float* pdf, float* value,
                                     uint32_t count);
/* Alias-table dome sampling on the integrator's dome (CL_DOME_ALIAS path). */
cl_status cl_dome_alias_sample(cl_integrator* integrator, const float* u2, float* dir, float* pdf, float* value,
                               uint32_t count);

/* ---- Allocation-free dome preprocessing.
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory: hosts whose allocator owns all device memory (a pool reserved at
 * start-up and handed out to the renderer, where a cudaMalloc would bypass
 * the pool's accounting or fail once the pool holds the memory), and host
 * applications whose render callbacks must not allocate.  The caller passes
 * device buffers for the input and every output;
 * the function allocates nothing.  Its FP64 scratch (texel weights, row
 * integrals, alias work lists) lives in one static device array of
 * CL_DOME_NOALLOC_SCRATCH_BYTES (about 12 MiB) that every GPU loading the
 * library holds until the process exits; it limits the dome to
 * CL_DOME_NOALLOC_MAX_TEXELS texels (e.g. 1024x512) and
 * CL_DOME_NOALLOC_MAX_ROWS rows, larger sizes return CL_ERR_INVALID_ARG.
 *   texels     device, RGBA32F, width*height*4 floats, 16-byte aligned
 *   pUcondV_c, cdfU  device, (width+1)*height floats each
 *   pV_c, cdfV       device, height+1 floats each
 *   alias_row  device, 2*height uint32 {prob bits, row}, 8-byte aligned
 *   alias_col  device, 2*width*height uint32 {prob bits, column}, 8-byte aligned
 *   stream     cudaStream_t to run on (null: the legacy default stream)
 * Results equal the tables cl_build_emitters builds for the same texels.
 * The call is asynchronous on `stream`.  Its first call on a device resolves
 * the scratch array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture begins.  The
 * address is kept per device and per CUDA context: a caller that switches to
 * another context on the same device (one made with the driver API, or the
 * primary context re-created after cudaDeviceReset) gets it resolved again on
 * its first call in that context, which then also belongs before a capture.  All calls
 * on a device share the one scratch array (each call overwrites every scratch
 * value it reads, so nothing needs clearing), so calls whose work overlaps on
 * the GPU (different streams, or threads) race: serialise them. */
enum
{
    CL_DOME_NOALLOC_MAX_TEXELS = 1 << 19,
    CL_DOME_NOALLOC_MAX_ROWS   = 4096
};
#define CL_DOME_NOALLOC_SCRATCH_BYTES                                                                              \
    (8u * CL_DOME_NOALLOC_MAX_TEXELS + 8u * (CL_DOME_NOALLOC_MAX_TEXELS + CL_DOME_NOALLOC_MAX_ROWS) +              \
     8u * CL_DOME_NOALLOC_MAX_ROWS + 4u * (2u * CL_DOME_NOALLOC_MAX_TEXELS + 2u * CL_DOME_NOALLOC_MAX_ROWS))
cl_status cl_dome_build_tables_noalloc(const float* texels, uint32_t width, uint32_t height, float* pUcondV_c,
                                       float* cdfU, float* pV_c, float* cdfV, uint32_t* alias_row,
                                       uint32_t* alias_col, void* stream);

/* ---- Scene ingestion and film output.
 * Replace the reference's asset delegates: MeshImporter::loadMeshes (assimp,
 * src/delegate/meshimporter.cpp:41-120, flags Triangulate | GenSmoothNormals |
 * GenUVCoords | FlipUVs | CalcTangentSpace) and
 * ImageUtils::loadImageFromDiskRadianceHDR (stb_image,
 * src/delegate/imageutil.cpp:98-139).  Host-side parsing; no device work.
 *
 * OBJ: one mesh per `o`/`g`/`usemtl` group with faces; polygons are
 * triangulated as fans; vertices are unified per (v, vt, vn) triple; normals
 * come from vn when every corner has one, else smooth normals (area-weighted
 * face normals summed per position); uvs come from vt with v flipped (1 - v)
 * when every corner has one, else none; tangents are dP/du from the uvs,
 * summed per vertex and orthogonalised against the normal (without uvs: any
 * perpendicular, since cl_build_meshes requires tangents).  The returned
 * descriptors point into the cl_obj and stay valid until cl_obj_free; pass
 * them to cl_build_meshes directly.
 * HDR: Radiance RGBE ("#?RADIANCE", FORMAT=32-bit_rle_rgbe, "-Y h +X w",
 * flat or new-style run-length scanlines), decoded as byte * 2^(e - 136),
 * into RGBA32F rows top to bottom with alpha 1 (the dome texel layout);
 * free with cl_image_free.
 * PFM: RGB float32, rows stored bottom up (written from RGBA rows top to
 * bottom, e.g. cl_readback_film's); read back into RGBA32F. */
typedef struct cl_obj cl_obj;
cl_status cl_obj_load(const char* path, cl_obj** out);
cl_status cl_obj_mesh_count(const cl_obj* obj, uint32_t* count);
cl_status cl_obj_get_mesh(const cl_obj* obj, uint32_t index, cl_mesh_desc* mesh);
cl_status cl_obj_free(cl_obj* obj);
cl_status cl_image_load_hdr(const char* path, float** rgba, uint32_t* width, uint32_t* height);
cl_status cl_image_free(float* rgba);
cl_status cl_image_write_pfm(const char* path, const float* rgba, uint32_t width, uint32_t height);
cl_status cl_image_read_pfm(const char* path, float** rgba, uint32_t* width, uint32_t* height);

/* ---- Neural path guiding.
 * No counterpart in the reference (its path tracer samples the BSDF only).
 * A guiding network maps (position, shading normal, outgoing direction) to a
 * mixture of CL_GUIDE_LOBES von Mises-Fisher lobes over incident directions:
 *   position: multiresolution hash grid, CL_GUIDE_LEVELS levels x 2 features,
 *             2^log2_table bf16 entries per level, trilinear interpolation;
 *   normal, outgoing direction: one-blob encoding of (theta/pi, phi/2pi+1/2),
 *             16 Gaussian bins per scalar;
 *   MLP 96 -> 64 -> 64 -> 64 -> 64 -> 48, ReLU, no biases, BF16 operands
 *             and FP32 accumulation on the tensor cores;
 *   head: outputs 5k..5k+4 = (mu_xyz, log kappa, weight logit) of lobe k;
 *             mu normalised, kappa = exp(clamp(., -5, 7)), softmax weights.
 * Training minimises the KL divergence to the product f |cos| L_i with
 * Adam: loss = -sum_s (w_s / sum w) log p(omega_s), w_s = the luminance of
 * f |cos| L_i / p_sample of the recorded direction.
 * Parameters (flat FP32, the layout of cl_guide_get_params): the hash table
 * [level][entry][feature], then W0 (64x96), W1..W3 (64x64), W4 (48x64),
 * each row-major [out][in].
 * With learn_selection, output 40 gives the probability of sampling the
 * network, a = 0.05 + 0.9 sigmoid(o40), and the loss uses the density the
 * tracer samples from, p = (1 - a) p_bsdf + a p_guide.
 * Record layouts of the host entry points:
 *   in9:   position in [0,1]^3 (scene box), shading normal, outgoing dir;
 *   rec14: in9, then the sampled direction omega (3), the weight w and the
 *          BSDF pdf of omega (used with learn_selection). */
enum
{
    CL_GUIDE_LEVELS  = 16,
    CL_GUIDE_OUTPUTS = 48,
    CL_GUIDE_LOBES   = 8
};
typedef struct cl_guide cl_guide;
typedef struct cl_guide_config
{
    uint32_t log2_table;                   /* entries per level: 2^log2_table, 8..24 (19) */
    uint32_t resolutions[CL_GUIDE_LEVELS]; /* per-level grid resolution; all 0: from n_min, n_max */
    float    n_min, n_max;                 /* coarsest and finest resolution (16, 1024) */
    float    learning_rate;                /* Adam (1e-2) */
    float    beta1, beta2, epsilon;        /* (0.9, 0.99, 1e-10) */
    float    bsdf_fraction;                /* one-sample MIS: probability of BSDF sampling, [0, 1] (0.5) */
    uint32_t batch;                        /* training samples per step (2^18) */
    uint32_t train_spp;                    /* one training step after each of the first train_spp spp (32) */
    uint32_t class_mask;                   /* guided BSDFs: bit 0 diffuse, 1 conductor, 2 dielectric (7) */
    uint32_t seed;                         /* parameter initialisation */
    uint32_t learn_selection;              /* 1: the probability of sampling the network is learned (head
                                              output 40) and training minimises -log of the whole one-sample
                                              MIS density; 0: it is 1 - bsdf_fraction and training minimises
                                              -log of the network's mixture (0) */
    float    weight_clamp;                 /* training weights above weight_clamp x the batch mean are
                                              clamped to it (robust fit to heavy-tailed records); 0 = off */
    uint32_t min_depth;                    /* guided vertices: path depth >= min_depth (1 = every vertex,
                                              the camera ray's hit included; 2 = indirect vertices only);
                                              shallower vertices sample the BSDF alone and are neither
                                              inferred nor recorded (0 or 1: every vertex) */
    float    min_alpha;                    /* guided conductor and dielectric vertices: GGX alpha (after
                                              textures) >= min_alpha; smoother ones sample the BSDF alone
                                              and are not recorded; diffuse vertices are not affected
                                              (0 = every vertex of the guided classes) */
} cl_guide_config;

typedef struct cl_guide_stats
{
    uint64_t steps;            /* training steps taken */
    uint64_t samples_trained;  /* training samples consumed */
    uint64_t records_last;     /* records collected during the last training spp */
    uint64_t inferred;         /* network evaluations by the integrator */
    double   last_loss;        /* loss of the last step */
    float    ms_train;         /* device time of training so far */
    float    ms_infer;         /* last render with CL_PROFILE_STAGES: device time of inference */
} cl_guide_stats;

void      cl_guide_default_config(cl_guide_config* config);
/* Level resolutions floor(n_min * b^l), b = (n_max / n_min)^(1/15) (host only). */
cl_status cl_guide_default_resolutions(float n_min, float n_max, uint32_t* resolutions16);
cl_status cl_guide_create(const cl_guide_config* config, cl_guide** out);
cl_status cl_guide_destroy(cl_guide* guide);
cl_status cl_guide_param_count(const cl_guide* guide, uint64_t* count);
cl_status cl_guide_get_resolutions(const cl_guide* guide, uint32_t* resolutions16);
/* Replaces all parameters and resets Adam's moments and step count. */
cl_status cl_guide_set_params(cl_guide* guide, const float* params, uint64_t count);
cl_status cl_guide_get_params(const cl_guide* guide, float* params, uint64_t count);
/* Raw head outputs (count x 48). */
cl_status cl_guide_forward(cl_guide* guide, const float* in9, uint32_t count, float* out48);
/* Loss and gradient (param_count floats) of one batch, parameters unchanged. */
cl_status cl_guide_gradient(cl_guide* guide, const float* rec14, uint32_t count, double* loss, float* grad);
/* One Adam step on one batch. */
cl_status cl_guide_train_step(cl_guide* guide, const float* rec14, uint32_t count, double* loss);
/* Sampling and pdf of the network's vMF mixture alone (u3: lobe, then the
 * two direction uniforms). */
cl_status cl_guide_sample(cl_guide* guide, const float* in9, const float* u3, uint32_t count, float* dir3,
                          float* pdf);
cl_status cl_guide_pdf(cl_guide* guide, const float* in9, const float* dir3, uint32_t count, float* pdf);

/* Guided path tracing: the path tracer samples each vertex of a guided class
 * from the one-sample MIS mixture bsdf_fraction * BSDF + (1 - bsdf_fraction)
 * * network, trains the network online on the paths it traces, and keeps an
 * unbiased estimator.  Needs CL_INTEGRATOR_PATH_TRACING and the corrected estimator
 * (no CL_COMPAT_* flag).  NULL switches guiding off.  Resets the iteration. */
cl_status cl_integrator_set_guiding(cl_integrator* integrator, const cl_guide_config* config);
/* The integrator's network (owned by the integrator), or NULL when off. */
cl_status cl_integrator_get_guide(cl_integrator* integrator, cl_guide** guide);
cl_status cl_integrator_guide_stats(cl_integrator* integrator, cl_guide_stats* stats);
/* Test probe of the integrator's fused guide inference (no counterpart in the
 * reference): traces the camera rays of the next frame and runs the guide's
 * inference on their hits exactly as a render does, without shading them (the
 * film and the iteration index are unchanged).  For the first `capacity`
 * guided rows it returns 52 floats each: in9 (the network input, as for
 * cl_guide_forward), the ray index as uint32 bits (0xffffffff: not inferred),
 * then 8 x {mu.xyz, kappa} and the 8 lobe weights (which sum to the
 * probability of sampling the network), 2 unused.  *count = rows written. */
cl_status cl_integrator_guide_probe(cl_integrator* integrator, uint32_t capacity, float* rows, uint32_t* count);

/* ---- Neural radiance cache.
 * No counterpart in the reference.  A second hash-grid network, 96 -> 64 ->
 * 64 -> 16 (ReLU; outputs 0-2: RGB), predicts the outgoing radiance at a
 * path vertex from (position, shading normal, outgoing direction), with the
 * same encoding as the guiding network.  Path tracing with the cache: a
 * path is shaded normally for `prefix_bounces` vertices and terminates into
 * the cache at the next one (its radiance is throughput x prediction; no
 * emitter sample there).  One path in 2^train_log2_fraction (by a hash of
 * the path index) is a training path: it is traced to max_depth, and each of
 * its vertices k yields the record (x_k, n_k, wo_k) -> (L - L_k) / T_k, the
 * radiance the path gathered from k on divided by the throughput that
 * reached k.  Training minimises the relative L2 loss (o - y)^2 / (o^2 +
 * 0.01) with Adam, one step on up to `network.batch` records after each of
 * the first train_spp samples per pixel (0: after every sample).  The cache
 * trades bias for shorter paths.
 * Host record layout of the cache's own entry points:
 *   rec12: in9 (as for the guiding network), then the target RGB. */
typedef struct cl_cache cl_cache;
typedef struct cl_radiance_cache_config
{
    cl_guide_config network;       /* hash grid, Adam and batch (the guiding-only fields are ignored) */
    uint32_t        prefix_bounces; /* shaded vertices before the cache terminates a path (2) */
    uint32_t        train_log2_fraction; /* 1 / 2^k of the paths are training paths (4) */
    uint32_t        train_spp;      /* training steps after the first train_spp spp; 0 = after every spp (32) */
} cl_radiance_cache_config;

void      cl_radiance_cache_default_config(cl_radiance_cache_config* config);
cl_status cl_cache_create(const cl_guide_config* network, cl_cache** out);
cl_status cl_cache_destroy(cl_cache* cache);
cl_status cl_cache_param_count(const cl_cache* cache, uint64_t* count);
cl_status cl_cache_get_resolutions(const cl_cache* cache, uint32_t* resolutions16);
cl_status cl_cache_set_params(cl_cache* cache, const float* params, uint64_t count);
cl_status cl_cache_get_params(const cl_cache* cache, float* params, uint64_t count);
/* Raw outputs (count x 16; RGB in 0-2). */
cl_status cl_cache_forward(cl_cache* cache, const float* in9, uint32_t count, float* out16);
cl_status cl_cache_gradient(cl_cache* cache, const float* rec12, uint32_t count, double* loss, float* grad);
cl_status cl_cache_train_step(cl_cache* cache, const float* rec12, uint32_t count, double* loss);
/* Path tracing with the radiance cache (CL_INTEGRATOR_PATH_TRACING, no
 * CL_COMPAT_* flag); NULL switches it off.  Combines with guiding.  Resets
 * the iteration. */
cl_status cl_integrator_set_radiance_cache(cl_integrator* integrator, const cl_radiance_cache_config* config);
cl_status cl_integrator_get_cache(cl_integrator* integrator, cl_cache** cache);
/* steps, samples_trained, records_last, inferred (cache queries), last_loss, ms_train. */
cl_status cl_integrator_cache_stats(cl_integrator* integrator, cl_guide_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* COLVILLEA_B200_H */
