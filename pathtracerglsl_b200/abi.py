"""ctypes mirror of ``include/ptx_rt.h`` (the C ABI of the transport loop).

Every structure here has the exact layout of its C counterpart; ``tests/`` checks
the sizes against the header.  Both the CUDA engine and the oracle bindings build
their descriptors from these types, so the two consume byte-identical scenes.
"""
import ctypes as C

ABI_VERSION = 4
FIELD_MAX_STACK = 16

PTR_OK = 0
PTR_E_INVALID = -1
PTR_E_CUDA = -2
PTR_E_NOMEM = -3
PTR_E_TIMEOUT = -4
PTR_E_DEVICE = -5
PTR_E_UNSUPPORTED = -6

SHAPE_PLANE, SHAPE_SPHERE, SHAPE_QUAD, SHAPE_BOX, SHAPE_MESH, SHAPE_INSTANCES = range(6)
MAT_LAMBERT, MAT_DIELECTRIC, MAT_GGX, MAT_MIRROR, MAT_NONE, MAT_ROUGH_DIELECTRIC = range(6)
MATF_EMISSIVE, MATF_MEDIUM, MATF_SCATTERING = 1, 2, 4
LIGHT_QUAD, LIGHT_SPHERE, LIGHT_POINT, LIGHT_MESH = range(4)
ENV_NONE, ENV_CONSTANT, ENV_IMAGE = range(3)
DIRECT_NONE, DIRECT_NEE, DIRECT_MIS = range(3)
ACCEL_BVH, ACCEL_CWBVH = range(2)
BUILD_HOST, BUILD_DEVICE = range(2)
EQUIANGULAR_OFF, EQUIANGULAR_DELTA, EQUIANGULAR_AREA = range(3)
# adjoint parameter slots per material (include/ptx_rt.h PTR_GRAD_*)
GRAD_SLOTS = 8
# slots 0-2: the model's colour (Lambert albedo, GGX / mirror F0, dielectric transmittance)
GRAD_COLOR_R, GRAD_COLOR_G, GRAD_COLOR_B, GRAD_ALPHA, GRAD_IOR, GRAD_SIGMA_T, GRAD_MEDIUM_ALBEDO, GRAD_HG_G = range(8)
GRAD_ALBEDO_R, GRAD_ALBEDO_G, GRAD_ALBEDO_B = GRAD_COLOR_R, GRAD_COLOR_G, GRAD_COLOR_B
GRAD_NAMES = ("color.r", "color.g", "color.b", "alpha", "ior", "sigma_t", "medium_albedo", "g")

F4 = C.c_float * 4


class Region(C.Structure):
    _fields_ = [("shape", C.c_int32), ("material", C.c_int32), ("thin", C.c_int32),
                ("ref", C.c_int32), ("ior", C.c_float), ("p", C.c_float * 15)]


class Material(C.Structure):
    _fields_ = [("model", C.c_int32), ("flags", C.c_int32), ("field_a", C.c_int32), ("field_s", C.c_int32),
                ("albedo", F4), ("emission", F4), ("transmittance", F4), ("f0", F4),
                ("sigma_a", F4), ("sigma_s", F4), ("alpha", C.c_float), ("phase_g", C.c_float),
                ("majorant", C.c_float), ("pad3", C.c_float)]


class Light(C.Structure):
    _fields_ = [("kind", C.c_int32), ("region", C.c_int32), ("select_pdf", C.c_float),
                ("select_cdf", C.c_float), ("radiance", F4), ("p", C.c_float * 16)]


class Env(C.Structure):
    _fields_ = [("kind", C.c_int32), ("sample_as_light", C.c_int32), ("width", C.c_int32),
                ("height", C.c_int32), ("color", F4), ("intensity", C.c_float),
                ("select_prob", C.c_float), ("rotation", C.c_float), ("pad", C.c_float),
                ("radiance", C.POINTER(C.c_float)), ("marginal", C.POINTER(C.c_float)),
                ("conditional", C.POINTER(C.c_float))]


class MeshDesc(C.Structure):
    _fields_ = [("n_vertices", C.c_int32), ("n_triangles", C.c_int32),
                ("positions", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_uint32)),
                ("tri_alpha", C.POINTER(C.c_float))]


class BatchDesc(C.Structure):
    _fields_ = [("prototype_shape", C.c_int32), ("prototype_ref", C.c_int32),
                ("n_instances", C.c_int32), ("light_base", C.c_int32), ("proto", F4),
                ("placements", C.POINTER(C.c_float))]


class RailMesh(C.Structure):
    _fields_ = [("vbase", C.c_int64), ("tbase", C.c_int64), ("nbase", C.c_int64),
                ("vertex_count", C.c_int32), ("tri_count", C.c_int32), ("node_count", C.c_int32), ("pad", C.c_int32),
                ("tri_order", C.POINTER(C.c_uint32)), ("tri_alpha", C.POINTER(C.c_float))]


class RailBatch(C.Structure):
    _fields_ = [("placements_base", C.c_int64), ("tlas_base", C.c_int64),
                ("instance_count", C.c_int32), ("node_count", C.c_int32),
                ("placement_texels", C.c_int32), ("pad", C.c_int32),
                ("inst_order", C.POINTER(C.c_uint32))]


class RailMeshLight(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("pad", C.c_int32), ("wpos_base", C.c_int64), ("cdf_base", C.c_int64)]


class Rails(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("vertices_texels", C.c_int64),
                ("indices", C.POINTER(C.c_float)), ("indices_texels", C.c_int64),
                ("nodes", C.POINTER(C.c_float)), ("nodes_texels", C.c_int64),
                ("records", C.POINTER(C.c_float)), ("records_texels", C.c_int64),
                ("n_meshes", C.c_int32), ("n_batches", C.c_int32), ("n_mesh_lights", C.c_int32), ("pad", C.c_int32),
                ("meshes", C.POINTER(RailMesh)), ("batches", C.POINTER(RailBatch)),
                ("mesh_lights", C.POINTER(RailMeshLight))]


COLOR_RGB, COLOR_SPECTRAL = range(2)
WAVELENGTHS_VISIBLE, WAVELENGTHS_UNIFORM = range(2)
SPEC_GREY, SPEC_LIFTED, SPEC_BLACKBODY = range(3)


class Spectrum(C.Structure):
    _fields_ = [("kind", C.c_int32), ("d65", C.c_int32), ("scale", C.c_float), ("c", C.c_float * 3),
                ("pad", C.c_int32 * 2)]


class SpectralMaterial(C.Structure):
    _fields_ = [("albedo", Spectrum), ("emission", Spectrum), ("transmittance", Spectrum), ("f0", Spectrum),
                ("sigma_a", Spectrum), ("sigma_s", Spectrum)]


class SpectralDesc(C.Structure):
    _fields_ = [("materials", C.POINTER(SpectralMaterial)), ("lights", C.POINTER(Spectrum)), ("env", Spectrum),
                ("curves", C.POINTER(C.c_float)), ("xyz_to_rgb", C.c_float * 9), ("cie_y_integral", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("n_regions", C.c_int32), ("regions", C.POINTER(Region)),
                ("n_materials", C.c_int32), ("materials", C.POINTER(Material)),
                ("n_lights", C.c_int32), ("lights", C.POINTER(Light)),
                ("ambient_material", C.c_int32), ("env", Env),
                ("n_meshes", C.c_int32), ("meshes", C.POINTER(MeshDesc)),
                ("n_batches", C.c_int32), ("batches", C.POINTER(BatchDesc)),
                ("spectral", C.POINTER(SpectralDesc)),
                ("n_tree_nodes", C.c_int32), ("light_tree", C.POINTER(C.c_float)),
                ("light_trails", C.POINTER(C.c_uint32)),
                ("n_field_code", C.c_int32), ("field_code", C.POINTER(C.c_uint32))]


class ProgramDesc(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("max_bounces", C.c_int32),
                ("max_null_crossings", C.c_int32), ("direct", C.c_int32), ("rr_start", C.c_int32),
                ("rr_max_survival", C.c_float), ("scattering", C.c_int32), ("accel", C.c_int32),
                ("equiangular", C.c_int32), ("color", C.c_int32), ("wavelengths", C.c_int32),
                ("lambda_min", C.c_float), ("lambda_max", C.c_float), ("instance_accel", C.c_int32),
                ("light_tree", C.c_int32), ("aovs", C.c_int32)]

AOV_ALBEDO, AOV_NORMAL = 1, 2


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("tan_fov", C.c_float), ("aspect", C.c_float)]


class Frame(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("first_sample", C.c_int32),
                ("spp", C.c_int32), ("reset_salt", C.c_uint32), ("pixel_offset", C.c_int32 * 2),
                ("accumulate", C.c_int32), ("camera", Camera), ("image_size", C.c_int32 * 2)]


class BatchJob(C.Structure):
    _fields_ = [("prog", C.c_void_p), ("scene", C.c_void_p), ("frame", Frame)]


class Counters(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("closest_queries", C.c_uint64), ("shadow_queries", C.c_uint64),
                ("nodes_visited", C.c_uint64), ("prims_tested", C.c_uint64), ("tlas_nodes", C.c_uint64),
                ("instances", C.c_uint64), ("shadow_work", C.c_uint64 * 4),
                ("error_flags", C.c_uint32), ("pad", C.c_uint32)]


PROFILE_TIMING, PROFILE_WORK = 1, 2
PROFILE_CLASSES = 6


class Tuning(C.Structure):
    _fields_ = [("capacity", C.c_int32), ("block", C.c_int32), ("sort_buckets", C.c_int32), ("ray_sort", C.c_int32)]


# Sizes the header documents (checked by the CPU tests).
EXPECTED_SIZES = {"Region": 80, "Material": 128, "Light": 96, "Spectrum": 32, "SpectralMaterial": 192,
                  "ProgramDesc": 64, "RailMesh": 56, "RailBatch": 40, "RailMeshLight": 24, "Rails": 104}
