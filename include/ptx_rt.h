/* ptx_rt.h — C ABI of the B200 transport loop for PathTracerGLSL scenes.
 *
 * This library replaces the WebGL executor of a CompiledRenderer
 * (reference: src/engine/RenderExecutor.ts:27-230, driven by src/engine/Engine.ts:83-438).
 * The host compiles a SceneDescription + RenderStrategy into a packed scene (the
 * counterpart of CompiledScene.sceneData, src/compiler/types.ts:1154-1164, executed by
 * src/app/sceneData.ts:27) and a program description (the estimator/measurement knobs of
 * ProgramDescription, src/compiler/plan/types.ts:39-112), then renders frames and reads
 * exports exactly where the reference calls Engine.renderFrame / Engine.readExport.
 *
 * Conventions (mirroring the reference's engine contract):
 *   - every entry point returns an int status: 0 = OK, negative = error class (PTR_E_*);
 *     ptr_last_error(ctx) returns the message of the last failure on that context;
 *   - the host owns every array it passes; upload copies them (registerDataTexture);
 *   - calls on one context are not re-entrant (one host thread per context, like the
 *     reference's single JS main thread); rendering is asynchronous on the context's
 *     stream and ptr_sync / ptr_read_export synchronise.
 *   - images are row-major with row 0 at the BOTTOM (gl_FragCoord convention), RGB.
 */
#ifndef PTX_RT_H
#define PTX_RT_H

#ifndef __CUDACC_RTC__   /* the runtime-compiled kernels (ptr_specialize) define these themselves */
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PTR_ABI_VERSION 4

/* ---- status codes ------------------------------------------------------------- */
#define PTR_OK 0
#define PTR_E_INVALID -1     /* bad argument / malformed scene (Validator-class error)  */
#define PTR_E_CUDA -2        /* CUDA runtime/driver error                                */
#define PTR_E_NOMEM -3       /* device allocation failed                                 */
#define PTR_E_TIMEOUT -4     /* ptr_sync timed out (work still in flight)                */
#define PTR_E_DEVICE -5      /* a kernel reported an error flag (budget / bounds guard)  */
#define PTR_E_UNSUPPORTED -6 /* feature not available in this build                      */

/* ---- shapes (one region = one scene object, reference region index order) --------- */
/* Shape occupants: src/components/geometry/{plane,sphere,quad,box}, meshes
 * src/components/intersection/mesh, instanced batches src/components/intersection/instancing. */
#define PTR_SHAPE_PLANE 0     /* p: normal.xyz, offset            (plane.glsl)            */
#define PTR_SHAPE_SPHERE 1    /* p: center.xyz, radius            (sphere.glsl)           */
#define PTR_SHAPE_QUAD 2      /* p: corner, edge1, edge2, normal  (quad.glsl)  thin       */
#define PTR_SHAPE_BOX 3       /* p: center.xyz, halfSize.xyz      (box.glsl)              */
#define PTR_SHAPE_MESH 4      /* ref = mesh index; thin (v0 meshes are open surfaces)     */
#define PTR_SHAPE_INSTANCES 5 /* ref = batch index (placements of one prototype)          */

typedef struct ptr_region {
    int32_t shape;     /* PTR_SHAPE_*                                                    */
    int32_t material;  /* material_of(region); -1 = none                                 */
    int32_t thin;      /* 1 = zero-thickness owner (scene_region_thin)                   */
    int32_t ref;       /* mesh / batch index for PTR_SHAPE_MESH / PTR_SHAPE_INSTANCES     */
    float ior;         /* ior_of(region)                                                 */
    float p[15];       /* shape parameters, layout per PTR_SHAPE_*                       */
} ptr_region;          /* 80 bytes */

/* ---- materials (src/components/materials, volume_scattering, transport/volume) ---- */
#define PTR_MAT_LAMBERT 0
#define PTR_MAT_DIELECTRIC 1
#define PTR_MAT_GGX 2
#define PTR_MAT_MIRROR 3   /* one delta lobe, Schlick F0 (materials/mirror/mirror.glsl)       */
#define PTR_MAT_NONE 4 /* null interface: a medium boundary with no optical surface */
#define PTR_MAT_ROUGH_DIELECTRIC 5 /* two-lobe microfacet dielectric (rough_dielectric.glsl) */

#define PTR_MATF_EMISSIVE 1
#define PTR_MATF_MEDIUM 2       /* material_has_medium                               */
#define PTR_MATF_SCATTERING 4   /* medium with sigma_s > 0 (HG phase)                */

typedef struct ptr_material {
    int32_t model;          /* PTR_MAT_*                                                  */
    int32_t flags;          /* PTR_MATF_*                                                 */
    int32_t field_a;        /* heterogeneous medium: 1 + the word offset of sigma_a's
                               program in field_code; 0 = the constant sigma_a below      */
    int32_t field_s;        /* likewise sigma_s                                           */
    float albedo[4];        /* lambert albedo (rgb)                                       */
    float emission[4];      /* emitted radiance (rgb)                                     */
    float transmittance[4]; /* dielectric interface tint                                  */
    float f0[4];            /* ggx / mirror normal-incidence reflectance                  */
    float sigma_a[4];       /* medium absorption (rgb)                                    */
    float sigma_s[4];       /* medium scattering (rgb)                                    */
    float alpha;            /* ggx alpha = max(1e-3, roughness^2)  (ggx.glsl:7-9)          */
    float phase_g;          /* HG asymmetry                                               */
    float majorant;         /* heterogeneous medium: the density ceiling sigma_bar; the
                               rendered medium is the field scaled so max sigma_t <= it   */
    float pad3;
} ptr_material;             /* 128 bytes */

/* ---- heterogeneous media: coefficient fields ----------------------------------------
 * A medium coefficient given as a GLSL expression of the position p (the reference's
 * {kind: 'glsl', source, params} coefficients, delta_tracking.glsl) travels as a stack
 * program: uint32 opcodes, CONST followed by three float bit patterns, SWZ by a component
 * index.  Every slot holds three floats (scalars broadcast); the host validates each
 * program (known opcodes, stack within PTR_FIELD_MAX_STACK, END inside the table). */
#define PTR_FIELD_MAX_STACK 16
enum {
    PTR_FOP_END, PTR_FOP_CONST, PTR_FOP_P, PTR_FOP_SWZ, PTR_FOP_ADD, PTR_FOP_SUB, PTR_FOP_MUL, PTR_FOP_DIV,
    PTR_FOP_NEG, PTR_FOP_EXP, PTR_FOP_LOG, PTR_FOP_SIN, PTR_FOP_COS, PTR_FOP_SQRT, PTR_FOP_ABS, PTR_FOP_FLOOR,
    PTR_FOP_FRACT, PTR_FOP_POW, PTR_FOP_MIN, PTR_FOP_MAX, PTR_FOP_MOD, PTR_FOP_STEP, PTR_FOP_CLAMP, PTR_FOP_MIX,
    PTR_FOP_SMOOTHSTEP, PTR_FOP_DOT, PTR_FOP_LENGTH, PTR_FOP_VEC3, PTR_FOP_COUNT
};

/* ---- lights (src/components/lights/{quad,sphere,point,mesh}) ---------------------------- */
#define PTR_LIGHT_QUAD 0   /* p: corner(3) edge1(3) edge2(3) normal(3) area(1) */
#define PTR_LIGHT_SPHERE 1 /* p: center(3) radius(1)                            */
#define PTR_LIGHT_POINT 2  /* p: position(3)     radiance = intensity (W/sr)    */
#define PTR_LIGHT_MESH 3   /* p: mesh index(1, as float) .. world area(p[12]); one-sided    
                      emission from the cross(b-a, c-a) side; only from an emissive
                      mesh object (lights/mesh/mesh.ts), region = that object     */

typedef struct ptr_light {
    int32_t kind;
    int32_t region;        /* the hittable region desugared from this light; -1 for delta
                              lights and for instance lights (their batch's light_base)   */
    float select_pdf;      /* selection probability among finite lights (power CDF)       */
    float select_cdf;      /* cumulative probability up to and including this light       */
    float radiance[4];
    float p[16];
} ptr_light;               /* 96 bytes */

/* ---- environment (src/components/env; features/environment.ts) --------------------- */
#define PTR_ENV_NONE 0
#define PTR_ENV_CONSTANT 1
#define PTR_ENV_IMAGE 2 /* equirect table + 2-level CDF (importance.ts, sampler_cdf.glsl) */

typedef struct ptr_env {
    int32_t kind;
    int32_t sample_as_light;  /* joins NEE/MIS                                          */
    int32_t width, height;    /* equirect table size                                    */
    float color[4];           /* constant radiance                                      */
    float intensity;          /* live multiplier (u_envIntensity)                       */
    float select_prob;        /* P(sample env) in two-stage NEE (u_envSelectProb)       */
    float rotation;           /* azimuth rotation, radians (u_envRotation)              */
    float pad;
    const float* radiance;    /* width*height*4 RGBA32F, row 0 = v=0 (+Y pole)          */
    const float* marginal;    /* height floats: cumulative CDF over rows                 */
    const float* conditional; /* height*width floats: cumulative CDF within each row     */
} ptr_env;

/* ---- triangle meshes, BVH / CWBVH (src/components/accel, intersection/mesh) --------- */
typedef struct ptr_mesh_desc {
    int32_t n_vertices, n_triangles;
    const float* positions;    /* 3*V, object-local                                       */
    const uint32_t* indices;   /* 3*T                                                     */
    const float* tri_alpha;    /* optional per-triangle GGX alpha (T), NULL = material's  */
} ptr_mesh_desc;

typedef struct ptr_batch_desc {
    int32_t prototype_shape;   /* PTR_SHAPE_SPHERE or PTR_SHAPE_MESH                     */
    int32_t prototype_ref;     /* mesh index for mesh prototypes                          */
    int32_t n_instances;
    int32_t light_base;        /* light-tree selection: instance i (placement order) is light
                                  light_base + i (a sphere light row); -1 = not lights     */
    float proto[4];            /* sphere prototype: center.xyz, radius                   */
    const float* placements;   /* 8*N: quaternion xyzw (world->local rigid), ts = (t_rigid.xyz, s) */
} ptr_batch_desc;

/* ---- spectral colour model (src/components/color/spectral, sensor/cie1931) ----------
 * The host lifts every constant RGB colour of the scene once (the table lookup of
 * lookup.glsl:15-36 over the shipped Jakob-Hanika atlas); the device evaluates
 *   value(lambda) = scale * base(lambda) * (d65 ? D65(lambda) : 1)
 * with base = 1 (PTR_SPEC_GREY: exact greys bypass the table), the bounded sigmoid
 * clamp(0.5 + 0.5 p / sqrt(1 + p^2), 0, 1), p = (c0 t + c1) t + c2, t = (lambda - 360) / 470
 * (PTR_SPEC_LIFTED), or Planck relative to 550 nm with c0 = kelvin and c1 = the unit-Y
 * normalization (PTR_SPEC_BLACKBODY, blackbody.glsl:4-10). */
#define PTR_COLOR_RGB 0
#define PTR_COLOR_SPECTRAL 1
#define PTR_WAVELENGTHS_VISIBLE 0   /* sech^2 density (visible.glsl:3-13)  */
#define PTR_WAVELENGTHS_UNIFORM 1   /* uniform density (uniform.glsl:1-2)  */
#define PTR_SPEC_GREY 0
#define PTR_SPEC_LIFTED 1
#define PTR_SPEC_BLACKBODY 2

typedef struct ptr_spectrum {
    int32_t kind;              /* PTR_SPEC_*                                              */
    int32_t d65;               /* 1: multiply by the D65 curve (emission lift)            */
    float scale;
    float c[3];
    int32_t pad[2];
} ptr_spectrum;                /* 32 bytes */

typedef struct ptr_spectral_material {
    ptr_spectrum albedo, emission, transmittance, f0, sigma_a, sigma_s;
} ptr_spectral_material;       /* 192 bytes; lifts of the ptr_material colours */

typedef struct ptr_spectral_desc {
    const ptr_spectral_material* materials;  /* n_materials                                */
    const ptr_spectrum* lights;              /* n_lights: the lights' radiance / intensity  */
    ptr_spectrum env;                        /* constant environment colour                 */
    const float* curves;                     /* 95 x 4: CIE 1931 x, y, z and D65 at 5 nm from 360 nm */
    float xyz_to_rgb[9];                     /* row-major, XYZ -> linear sRGB               */
    float cie_y_integral;                    /* int ybar d lambda                           */
} ptr_spectral_desc;

typedef struct ptr_scene_desc {
    int32_t abi_version;       /* PTR_ABI_VERSION                                         */
    int32_t n_regions;
    const ptr_region* regions;
    int32_t n_materials;
    const ptr_material* materials;
    int32_t n_lights;
    const ptr_light* lights;
    int32_t ambient_material;  /* material_of(-1); -1 = vacuum                             */
    ptr_env env;
    int32_t n_meshes;
    const ptr_mesh_desc* meshes;
    int32_t n_batches;
    const ptr_batch_desc* batches;
    const ptr_spectral_desc* spectral;  /* NULL: the scene renders in RGB only             */
    /* light tree (estimator.lightSelection 'bvh'; accel/light_tree/light_tree.ts), from
     * ptr_build_light_tree over all n_lights; NULL = the power CDF selects.  Nodes: 8 floats
     * (min.xyz, phi, max.xyz, link), preorder, left child = node + 1, link >= 0 the right
     * child, link < 0 a leaf of light -link - 1.  Trails: 2 words per light. */
    int32_t n_tree_nodes;      /* 2 n_lights - 1, or 0                                    */
    const float* light_tree;
    const uint32_t* light_trails;
    int32_t n_field_code;      /* words of the heterogeneous media's field programs       */
    const uint32_t* field_code;
} ptr_scene_desc;

/* ---- program (strategy) ---------------------------------------------------------- */
#define PTR_DIRECT_NONE 0
#define PTR_DIRECT_NEE 1
#define PTR_DIRECT_MIS 2
#define PTR_ACCEL_BVH 0   /* binary SAH BVH (bvh.ts)                   */
#define PTR_ACCEL_CWBVH 1 /* compressed wide BVH (cwbvh.ts)            */
/* estimator.mediumLightSampling: 'vertex' (NEE at medium scattering vertices) or
 * 'equiangular' (one Kulla-Fajardo estimate per medium segment,
 * transport/techniques/equiangular/equiangular.glsl:18-57).  The reference pins it to
 * delta lights and plain NEE; PTR_EQUIANGULAR_AREA is this library's extension that also
 * admits quad and sphere lights (a uniform point on the light's area, then the
 * equiangular distance towards it). */
#define PTR_EQUIANGULAR_OFF 0
#define PTR_EQUIANGULAR_DELTA 1
#define PTR_EQUIANGULAR_AREA 2

typedef struct ptr_program_desc {
    int32_t abi_version;
    int32_t max_bounces;        /* measurement.maxBounces                             */
    int32_t max_null_crossings; /* measurement.maxNullCrossings (default 32)          */
    int32_t direct;             /* estimator.directLighting                           */
    int32_t rr_start;           /* russianRoulette.startDepth, -1 = off               */
    float rr_max_survival;      /* russianRoulette.maxSurvival (0.95)                 */
    int32_t scattering;         /* measurement.scattering: 1 full, 0 ignored           */
    int32_t accel;              /* PTR_ACCEL_*  (meshTraversal / instanceAccel)        */
    int32_t equiangular;        /* PTR_EQUIANGULAR_*  (mediumLightSampling)            */
    int32_t color;              /* PTR_COLOR_*  (measurement.color)                    */
    int32_t wavelengths;        /* PTR_WAVELENGTHS_*  (estimator.wavelengths)          */
    float lambda_min;           /* sampled range, nm (the reference's 360..830)        */
    float lambda_max;
    int32_t instance_accel;     /* PTR_ACCEL_* of instanced batches' TLAS (estimator.instanceAccel:
                                   'tlas' binary, 'cwbvh' wide; intersection/index.ts:68-159) */
    int32_t light_tree;         /* estimator.lightSelection 'bvh': the scene's light tree
                                   selects (stochastic descent, trail-replayed pmf)      */
    int32_t aovs;               /* measurement.aovs (components/aov): PTR_AOV_* bits; each
                                   is read with ptr_read_export("albedo" / "normal")     */
} ptr_program_desc;
/* First-hit pictures (denoiser guides): at the first non-null surface a path reaches
 * before any scattering event, the material's albedo fact clamped to [0, 1] (lambert
 * albedo, dielectrics' transmittance, GGX / mirror f0) times the path's throughput, and
 * the shading normal faced toward the arriving ray times the throughput's channel mean;
 * 0 otherwise.  RGB programs only. */
#define PTR_AOV_ALBEDO 1
#define PTR_AOV_NORMAL 2

/* The per-frame builtins + camera uniforms (Engine.ts:231-258, camera.ts:69-160). */
typedef struct ptr_camera {
    float position[3];
    float forward[3];
    float right[3];
    float up[3];
    float tan_fov;              /* tan(fov/2) */
    float aspect;               /* width/height */
} ptr_camera;

typedef struct ptr_frame {
    int32_t width, height;      /* the film rendered by this call (a tile's size)     */
    int32_t first_sample;       /* engine.sampleCount of the first sample             */
    int32_t spp;                /* samples per pixel rendered by this call            */
    uint32_t reset_salt;        /* engine.resetSalt                                   */
    int32_t pixel_offset[2];    /* engine.pixelOffset (tiled renders)                 */
    int32_t accumulate;         /* 0 = clear the film first, 1 = add to it            */
    ptr_camera camera;
    int32_t image_size[2];      /* engine.imageSize: the full image the camera maps film
                                   points through (pinhole.glsl:6); 0, 0 = width, height.
                                   A tile of a larger image (TiledRenderer.ts:63-117)
                                   passes the full size here and its own size above.  */
} ptr_frame;

typedef struct ptr_counters {
    uint64_t paths;             /* camera paths traced                                */
    uint64_t closest_queries;   /* closest-hit ray queries                            */
    uint64_t shadow_queries;    /* shadow (any-hit / transmittance) queries           */
    uint64_t nodes_visited;     /* mesh BLAS nodes popped (counting pass only)         */
    uint64_t prims_tested;      /* triangles tested (counting pass only)               */
    uint64_t tlas_nodes;        /* instance TLAS nodes popped (counting pass only)     */
    uint64_t instances;         /* instances entered (counting pass only)              */
    uint64_t shadow_work[4];    /* the same four tallies for the shadow queries        */
    uint32_t error_flags;       /* device-side guard flags (stack / budget)            */
    uint32_t pad;
} ptr_counters;

typedef struct ptr_ctx ptr_ctx;
typedef struct ptr_scene ptr_scene;
typedef struct ptr_program ptr_program;

/* Context: one CUDA device + stream.  (Engine constructor, Engine.ts:83) */
int ptr_create(int device_ordinal, ptr_ctx** out);
int ptr_destroy(ptr_ctx* ctx);
const char* ptr_last_error(const ptr_ctx* ctx);
int ptr_abi_version(void);

/* Scene data upload, once per scene (Engine.registerDataTexture, Engine.ts:438;
 * sceneData.ts:27).  Builds the BVH/CWBVH of every mesh on the host and copies all
 * arrays to device memory. */
int ptr_upload_scene(ptr_ctx* ctx, const ptr_scene_desc* desc, ptr_scene** out);
int ptr_free_scene(ptr_scene* scene);

/* ---- scene data in the reference's packed channel format (rail v2) ----------------------
 * The reference's App packs a scene's array data into RGBA32F channels, one texel = 4
 * floats, each tenant at the base texel the ledger assigns (planDataLayout,
 * src/components/data/ledger.ts:121; writers src/components/data/pack.ts; executed by
 * packSceneData, src/app/sceneData.ts:27):
 *   vertices  one vec3 texel per vertex (mesh geometry; mesh-light world positions)
 *   indices   one texel per triangle: its three vertex ids as exact floats, in BVH leaf order
 *   nodes     two texels per binary BVH node: (min.xyz, A) (max.xyz, B), A >= 1 a leaf of A
 *             items from offset B, A < 0 an internal node (axis -A-1, right child B)
 *   records   instance placements in TLAS leaf order (frame tier: two texels, q_inv and
 *             (t_rigid, s); params tier: one texel, the folded (centre, radius)), mesh-light
 *             area CDFs (.x per texel)
 * ptr_upload_scene_rails takes those channels as the App packed them (host memory, row-major
 * texels, copied to the device once each) and uses the reference's mesh BVHs, instance
 * TLASes and placement records in place: no re-packing and no host BVH build.  The
 * scene description still carries the regions, materials, lights and environment, and its
 * mesh and batch entries their roles (mesh positions/indices and batch placements may be
 * NULL): mesh i and batch i of the description take rail slot i.  The compressed wide
 * BVH of each mesh (meshTraversal 'cwbvh') and the wide twin of each TLAS are built from
 * the rail data (the mesh's on the device).  Hit ids: a rail triangle or instance is its
 * caller's index when tri_order / inst_order give it (buildBVH's and the TLAS build's leaf
 * permutations), else its leaf index.  A mesh light samples its triangles by the rail's
 * CDF, in leaf order as the reference does.  Every base, count, index, node link and
 * permutation is checked before anything runs (PTR_E_INVALID). */
typedef struct ptr_rail_mesh {         /* one geometry slot (ledger MeshSlot)            */
    int64_t vbase, tbase, nbase;       /* vertices / indices / nodes base texels          */
    int32_t vertex_count, tri_count;
    int32_t node_count, pad;           /* BVH nodes (2 texels each)                       */
    const uint32_t* tri_order;         /* caller index of each leaf triangle, or NULL     */
    const float* tri_alpha;            /* per-triangle GGX alpha by caller index, or NULL */
} ptr_rail_mesh;
typedef struct ptr_rail_batch {        /* one instance batch (ledger BatchSlot)           */
    int64_t placements_base, tlas_base;   /* records / nodes base texels                  */
    int32_t instance_count, node_count;
    int32_t placement_texels, pad;     /* 2: frame tier (mesh prototypes), 1: params tier (spheres) */
    const uint32_t* inst_order;        /* caller index of each leaf placement, or NULL   */
} ptr_rail_batch;
typedef struct ptr_rail_mesh_light {   /* a samplable mesh emitter (ledger MeshLightSlot) */
    int32_t mesh, pad;
    int64_t wpos_base, cdf_base;       /* vertices / records base texels                  */
} ptr_rail_mesh_light;
typedef struct ptr_rails {
    const float* vertices; int64_t vertices_texels;
    const float* indices;  int64_t indices_texels;
    const float* nodes;    int64_t nodes_texels;
    const float* records;  int64_t records_texels;
    int32_t n_meshes, n_batches, n_mesh_lights, pad;
    const ptr_rail_mesh* meshes;
    const ptr_rail_batch* batches;
    const ptr_rail_mesh_light* mesh_lights;
} ptr_rails;
int ptr_upload_scene_rails(ptr_ctx* ctx, const ptr_scene_desc* desc, const ptr_rails* rails, ptr_scene** out);

/* Program per scene x strategy (Engine.loadRenderer, Engine.ts:147). */
int ptr_compile(ptr_ctx* ctx, const ptr_program_desc* desc, ptr_program** out);
int ptr_free_program(ptr_program* prog);

/* Render frame.spp samples per pixel into the program's film, asynchronously
 * (Engine.renderFrame, Engine.ts:190-204; one call may fold many frames). */
int ptr_render(ptr_program* prog, ptr_scene* scene, const ptr_frame* frame);

/* Batched rendering: many scenes x programs x frames of uneven size in ONE wavefront —
 * the jobs' paths share one path pool and every wave is one CUDA graph of the
 * generate / closest / shade / shadow / film kernels over the concatenated job space,
 * with per-job scene, program and frame tables (paths of shallow jobs retire early;
 * compaction keeps the queues dense).  Each job accumulates into its own program's film
 * (read it with ptr_read_export).  All jobs must share directLighting.  Synchronises.
 * No counterpart in the reference (one fragment draw per renderer and frame). */
typedef struct ptr_batch_job {
    ptr_program* prog;
    ptr_scene* scene;
    ptr_frame frame;
} ptr_batch_job;
int ptr_render_batch(ptr_ctx* ctx, const ptr_batch_job* jobs, int n_jobs);
/* Counters of the last batched render (paths, closest and shadow queries). */
int ptr_get_batch_counters(ptr_ctx* ctx, ptr_counters* out);
/* Instrument the next ptr_render_batch (PTR_PROFILE_TIMING: CUDA events around every
 * launch, no graph) and read the per-kernel-class times like ptr_get_profile. */
int ptr_profile_batch_next(ptr_ctx* ctx, int mode);
int ptr_get_batch_profile(ptr_ctx* ctx, float* ms_out, int* launches_out, int n);

/* Test hook: render like ptr_render (film included) and also copy every sample's radiance
 * to host_out, laid out [sample][row][column][rgb] (n >= width*height*spp*3 floats).
 * The per-sample values are what the reference's accumulation folds in (accumulation.ts:14-51). */
int ptr_render_samples(ptr_program* prog, ptr_scene* scene, const ptr_frame* frame, float* host_out, size_t n);

/* Nearest-hit queries on an uploaded scene: rays are n x (origin.xyz, direction.xyz);
 * per ray returns the region (-1 = miss), the instance (its index among the batch's
 * placements; 0 for other regions), the ORIGINAL triangle index of a mesh hit (-1
 * otherwise) and t (1000 = MAX_DIST on a miss).  accel selects the mesh BLAS walk
 * (PTR_ACCEL_BVH / PTR_ACCEL_CWBVH).  The scene_intersect traversal of the reference
 * (features/intersection.ts:1665-1713) without the region probe.  Hits at equal t go to
 * the lower region, then the lower instance, then the lower triangle index, whatever
 * order the walk visits them in. */
int ptr_trace_closest(ptr_ctx* ctx, ptr_scene* scene, int accel, const float* rays, int n,
                      int* region, int* element, int* prim, float* t);

/* Host builders on their own (no GPU): the binary SAH BVH of the reference's
 * buildBVHNodesFlat (src/components/accel/bvh/bvh.ts:344-383; 8 floats per node) and the
 * compressed wide BVH of buildCWBVH (src/components/accel/cwbvh/cwbvh.ts:80-372; 20 u32
 * per node) over n boxes of 6 doubles (min.xyz, max.xyz).  order_out[i] = item index of
 * leaf slot i.  Pass nodes_out = NULL to query node_count first. */
int ptr_build_bvh(const double* boxes, int n, int leaf_size, int always_split,
                  float* nodes_out, int nodes_cap, uint32_t* order_out, int* node_count, int* max_depth);
int ptr_build_cwbvh(const double* boxes, int n, double c_prim,
                    uint32_t* nodes_out, int nodes_cap, uint32_t* order_out, int* node_count, int* max_depth);
/* The light tree of buildLightTree (src/components/accel/light_tree/light_tree.ts:44-72)
 * over n lights: boxes 6 doubles each (min.xyz, max.xyz; degenerate boxes allowed),
 * powers > 0.  Writes 2n - 1 nodes (8 floats each, the ptr_scene_desc.light_tree layout)
 * and 2 trail words per light (root-to-leaf decisions, LSB first, levels 0-23 and 24-47).
 * Returns the tree's depth (<= 47), or PTR_E_INVALID. */
int ptr_build_light_tree(const double* boxes, const double* powers, int32_t n, float* nodes_out,
                         uint32_t* trails_out);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own work
 * (timing events, cache flushes) with the library's launches. */
int ptr_get_stream(ptr_ctx* ctx, void** stream);

/* Allocation-free rendering.  No counterpart in the reference (its WebGL engine owns all
 * GPU memory); added for callers that cannot allocate device memory themselves: hosts
 * that give the whole GPU to their own memory pool, plugin hosts that forbid driver
 * allocations in their frame loop, or loops that cannot take the device-wide stall an
 * allocation may cause.  It renders frame->spp samples per pixel of an ANALYTIC scene
 * (no meshes, no instanced batches, no image environment) given as host tables like
 * ptr_upload_scene, on `stream` (a cudaStream_t, NULL = the legacy default stream), and
 * accumulates into the caller's device film buffers sum_dev / sumsq_dev (3 doubles per
 * pixel each; cleared first unless frame->accumulate).  It calls no cudaMalloc, cudaFree
 * or other allocating routine: the scene tables and the path pool live in one fixed
 * array inside the library, about 15 MB on every GPU that loads the library, held until
 * the process exits, for at most 65536 paths in flight (larger frames run in waves) and
 * at most 256 regions, materials and lights (more returns PTR_E_INVALID).
 * The first call on each device looks the array's device address up (with that device
 * current); make that first call before any stream capture.  The address is kept for
 * the life of the process, so resetting a device (cudaDeviceReset) after its first call
 * is not supported.  Every call shares the array: calls that overlap on the GPU race.
 * The scene tables pass the same checks as ptr_upload_scene's, and only quad, sphere and
 * point lights are accepted.  The current device must be set by the caller.  Returns a
 * PTR_E_* status (messages go to stderr; there is no context). */
int ptr_render_noalloc(const ptr_scene_desc* scene, const ptr_program_desc* prog, const ptr_frame* frame,
                       double* sum_dev, double* sumsq_dev, void* stream);

/* ---- adjoint (path replay backpropagation) ----------------------------------------
 * No counterpart in the reference (it renders only).  Parameters are per material,
 * PTR_GRAD_SLOTS each, in material-table order; a slot that a material's model does not
 * use receives 0.  The IOR gradient holds the interface terms (Fresnel lobe choice and
 * the eta^2 radiance factor), not the refracted direction's own dependence on the IOR.
 * Media must be grey (sigma_a, sigma_s equal in r, g, b); the medium's parameters are
 * sigma_t = sigma_a + sigma_s and the single-scattering albedo sigma_s / sigma_t. */
#define PTR_GRAD_SLOTS 8
#define PTR_GRAD_COLOR_R 0         /* the model's colour r, g, b: slots 0, 1, 2 -
                                      Lambert albedo, GGX / mirror F0, dielectric
                                      transmittance                                   */
#define PTR_GRAD_ALBEDO_R PTR_GRAD_COLOR_R
#define PTR_GRAD_ALPHA 3           /* GGX alpha (materials without per-triangle alpha) */
#define PTR_GRAD_IOR 4             /* dielectric IOR (interface terms)               */
#define PTR_GRAD_SIGMA_T 5         /* grey homogeneous medium sigma_t               */
#define PTR_GRAD_MEDIUM_ALBEDO 6   /* its single-scattering albedo                  */
#define PTR_GRAD_HG_G 7            /* its HG asymmetry g                            */

/* Gradient of a loss with respect to the scene's material parameters: renders
 * frame->spp samples per pixel of the frame twice on the same random numbers — the
 * forward walk, then its replay, which scatters dL_dimage[pixel] * d(sample)/d(theta) / spp
 * into float64 accumulators — and writes grads[PTR_GRAD_SLOTS * material + slot]
 * (n >= PTR_GRAD_SLOTS * n_materials doubles, host memory).  dL_dimage is host memory,
 * 3 floats per pixel (row 0 at the bottom), typically 2 (I - target) / n for an L2 loss on
 * an image I rendered with ptr_render.  The program's film is left untouched.  Synchronises.
 * Returns PTR_E_INVALID, before any device work, for spectral programs, chromatic or
 * heterogeneous media, equiangular or light-tree programs, programs with AOVs and more
 * than 512 materials.  The program keeps a log of the forward walk's
 * closest hits and shadow-query results for its replay (64 bytes per path and walk
 * iteration, at most 4 GiB of device memory, freed with the program). */
int ptr_backward(ptr_program* prog, ptr_scene* scene, const ptr_frame* frame, const float* dL_dimage,
                 double* grads, size_t n);

/* Live parameters (ptr_set_params of the engine contract; UniformBinding.compute,
 * src/compiler/types.ts:793-812, evaluated on the host): replace the uploaded material
 * table and, when regions is not NULL, the regions' IOR values.  Shapes and counts must
 * equal the uploaded scene's (PTR_E_INVALID otherwise).  Ordered on the context's stream. */
int ptr_update_params(ptr_scene* scene, const ptr_material* materials, int n_materials,
                      const ptr_region* regions, int n_regions);

/* ---- per-scene kernels (replaces the reference's per scene x strategy code generation:
 * Generate emits GLSL for each scene x strategy, src/compiler/generate/Generator.ts:10-91,
 * compiled by the WebGL driver in RenderExecutor.ts:86-107).
 * Compiles the program's closest-hit, shading and shadow kernels for this scene with NVRTC
 * (sm_100a): material models, light kinds, environment kind and region shapes the scene
 * lacks fold away, and with at most 16 regions the region loops unroll into one arm per
 * region with its intersection routine fixed, like the reference's generated arms (in
 * place of the region BVH, which returns the same hits).  Later ptr_render calls of the
 * program with this scene use them (samples are bit-identical to the generic kernels), and
 * so does ptr_backward's forward walk; its replay kernels (shading and shadow with the
 * adjoint terms) are compiled for the same census at the first ptr_backward that follows.
 * The counting passes keep the generic kernels (a batch takes ptr_specialize_batch).
 * Modules are cached per occupant census for the process.
 * seconds_out (may be NULL): compile time (0 for a cached module).  scene = NULL returns
 * the program to the generic kernels.  PTR_E_UNSUPPORTED when NVRTC cannot be loaded. */
int ptr_specialize(ptr_program* prog, ptr_scene* scene, double* seconds_out);

/* The batched kernels of ptr_render_batch compiled for a job mix (no counterpart in the
 * reference, which draws one scene per frame): the union of the jobs' occupant censuses
 * (material models, light kinds, environment kinds, region shapes; no region unrolling),
 * compiled with NVRTC like ptr_specialize.  Later ptr_render_batch calls on the context
 * whose jobs have the same union census use them; samples are identical to the generic
 * batched kernels.  The jobs' frames are not read.  seconds_out as for ptr_specialize. */
int ptr_specialize_batch(ptr_ctx* ctx, const ptr_batch_job* jobs, int n_jobs, double* seconds_out);

/* ---- where mesh BVHs are built (no counterpart in the reference, which builds on the host:
 * buildBVHCore / buildCWBVH, src/components/accel/bvh/bvh.ts:132-343 and
 * src/components/accel/cwbvh/cwbvh.ts:80-372).  PTR_BUILD_HOST (the default): the
 * reference's binned-SAH binary BVH (leaf 2) and its SAH collapse to the compressed wide
 * BVH, on the host.  PTR_BUILD_DEVICE: a linear BVH over Morton codes (Karras 2012) and a
 * greedy eight-wide collapse with the same quantized 80-byte nodes, on the GPU, from the
 * mesh's vertex and index arrays.  Hits are the same either way (exact nearest hits with
 * one tie rule); node counts and traversal cost differ.  Applies to later
 * ptr_upload_scene calls on the context. */
#define PTR_BUILD_HOST 0
#define PTR_BUILD_DEVICE 1
int ptr_set_accel_build(ptr_ctx* ctx, int where);

/* ---- launch tuning (no counterpart in the reference: WebGL draws one fragment per pixel) ----
 * capacity: paths in flight per wave (0 = the default 2^24); block: threads per block of the
 * wavefront kernels (128 or 256; the grid keeps 2048 resident threads per SM);
 * sort_buckets: the occupant-sorted shading queue — 1 = off, 8 = live paths grouped by the
 * material model they shade, 16 = by model and whether the segment starts in a medium;
 * ray_sort: the ray-coherence order of the traversal queues.  Every knob changes the order
 * of work only: each path's samples are bit-identical under any tuning.
 * Applies to every later ptr_render / ptr_render_batch / ptr_backward on the context.
 * pathtracerglsl_b200.autotune picks and records these per workload. */
typedef struct ptr_tuning {
    int32_t capacity;
    int32_t block;
    int32_t sort_buckets;
    int32_t ray_sort;          /* 1: closest-hit and shadow queues grouped by (direction octant,
                                  origin octant) before each traversal; 0: off               */
} ptr_tuning;
int ptr_set_tuning(ptr_ctx* ctx, const ptr_tuning* t);
int ptr_get_tuning(ptr_ctx* ctx, ptr_tuning* out);

/* Wait for the context's stream, at most timeout_ms (<0 = no limit). */
int ptr_sync(ptr_ctx* ctx, int timeout_ms);

/* Read an export into host memory (Engine.readExport, Engine.ts:351).
 * name: "radiance" (mean, 3 floats/pixel), "variance" (per-pixel sample variance of
 * the mean's samples, 3 floats/pixel), "samples" (1 float/pixel: sample count).
 * n = number of floats in dst. */
int ptr_read_export(ptr_program* prog, const char* name, float* dst, size_t n);

/* Same, but the destination is device memory (no synchronisation). */
int ptr_read_export_device(ptr_program* prog, const char* name, float* dst_device, size_t n);

/* Device work counters of the last ptr_render on this program (synchronises). */
int ptr_get_counters(ptr_program* prog, ptr_counters* out);

/* Instrument the next ptr_render (mode bits): PTR_PROFILE_TIMING runs it without the
 * CUDA graph with a pair of CUDA events around each kernel class's launches of every
 * walk iteration on the context's stream — ptr_get_profile then returns, per kernel
 * class k (0 generate, 1 closest-hit, 2 shade, 3 shadow, 4 film, 5 queue sorts), the
 * summed device time ms_out[k] and the number of kernel launches launches_out[k]
 * (n <= PTR_PROFILE_CLASSES entries); PTR_PROFILE_WORK runs the traversal kernels'
 * counting variants, which tally nodes, triangles, TLAS nodes and instances into
 * ptr_counters. */
#define PTR_PROFILE_TIMING 1
#define PTR_PROFILE_WORK 2
#define PTR_PROFILE_CLASSES 6
int ptr_profile_next(ptr_program* prog, int enable);
int ptr_get_profile(ptr_program* prog, float* ms_out, int* launches_out, int n);

#ifdef __cplusplus
}
#endif
#endif /* PTX_RT_H */
