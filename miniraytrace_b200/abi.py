"""ctypes mirror of include/mini_raytrace.h and include/mrt_ext.h.

Field order, types and enum values are those of the C header, which are in
turn those of the reference ABI (capi/include/mini_raytrace.h:28-181).
"""
from __future__ import annotations

import ctypes as C

# mrtResult (reference mini_raytrace.h:28-37)
MRT_SUCCESS = 0
MRT_ERROR_UNKNOWN = 1
MRT_ERROR_VULKAN_INIT = 2
MRT_ERROR_OUT_OF_MEMORY = 3
MRT_ERROR_INVALID_ARGUMENT = 4
MRT_ERROR_INVALID_HANDLE = 5
MRT_ERROR_SHADER_LOAD = 6
MRT_ERROR_DEVICE_LOST = 7

MRT_INVALID_ID = 0

MRT_PIXEL_RGBA8_SRGB = 0
MRT_PIXEL_RGBA32F_LINEAR = 1

MRT_TEX_RGBA8_SRGB = 0
MRT_TEX_RGBA8_UNORM = 1
MRT_TEX_RGBA32F = 2

MRT_LIGHT_SUN = 0
MRT_LIGHT_POINT = 1
MRT_LIGHT_RECT = 2

MRT_TONEMAP_LINEAR = 0
MRT_TONEMAP_ACES = 1

MRT_CAMERA_PERSPECTIVE = 0
MRT_CAMERA_ORTHOGRAPHIC = 1

F3 = C.c_float * 3


class _Sized(C.Structure):
    """A struct whose first field is structSize, pre-filled with sizeof()."""

    def __init__(self, **kw):
        super().__init__()
        self.structSize = C.sizeof(self)
        for k, v in kw.items():
            setattr(self, k, v)


class EngineDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("enableValidation", C.c_int32), ("width", C.c_uint32),
                ("height", C.c_uint32), ("gpuIndex1", C.c_uint32)]


class MeshDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("vertexCount", C.c_uint32), ("indexCount", C.c_uint32),
                ("positions", C.c_void_p), ("normals", C.c_void_p), ("uvs", C.c_void_p),
                ("indices", C.c_void_p)]


class MaterialDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("baseColor", F3), ("opacity", C.c_float), ("roughness", C.c_float),
                ("metallic", C.c_float), ("transmission", C.c_float), ("ior", C.c_float), ("emission", F3),
                ("baseColorTex", C.c_uint32), ("roughnessTex", C.c_uint32), ("metallicTex", C.c_uint32),
                ("normalTex", C.c_uint32), ("emissionTex", C.c_uint32)]


class TextureDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("width", C.c_uint32), ("height", C.c_uint32),
                ("format", C.c_int32), ("pixels", C.c_void_p), ("generateMips", C.c_int32)]


class LightDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("type", C.c_int32), ("direction", F3), ("position", F3),
                ("radiance", F3), ("angularRadius", C.c_float), ("corner", F3), ("edge0", F3), ("edge1", F3),
                ("twoSided", C.c_int32)]


class CameraDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("position", F3), ("target", F3), ("up", F3), ("fovYDeg", C.c_float)]


class CameraDescEx(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("projection", C.c_int32), ("position", F3), ("forward", F3),
                ("up", F3), ("left", C.c_float), ("right", C.c_float), ("bottom", C.c_float), ("top", C.c_float)]


class RenderSettings(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("width", C.c_uint32), ("height", C.c_uint32),
                ("maxBounces", C.c_uint32), ("sppLimit", C.c_uint32), ("exposureEV", C.c_float),
                ("fireflyClamp", C.c_float), ("tonemap", C.c_int32), ("denoise", C.c_int32)]


class FrameInfo(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("spp", C.c_uint32), ("converged", C.c_int32),
                ("denoised", C.c_int32), ("frameMs", C.c_float)]


class RadianceCacheDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("enabled", C.c_int32), ("trainingPaths", C.c_uint32),
                ("stepsPerSample", C.c_uint32), ("learningRate", C.c_float), ("seed", C.c_uint32),
                ("boundsLo", C.c_float * 3), ("boundsHi", C.c_float * 3), ("samplesPerUpdate", C.c_uint32),
                ("trainingVertices", C.c_uint32)]


class DenoiserDesc(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("enabled", C.c_int32), ("iterations", C.c_uint32),
                ("guideSamples", C.c_uint32), ("minSpp", C.c_uint32), ("sigmaColor", C.c_float),
                ("normalPower", C.c_float), ("sigmaAlbedo", C.c_float), ("sigmaDepth", C.c_float)]


class CommitStats(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("blasRebuilt", C.c_uint32), ("tlasRebuilt", C.c_int32),
                ("commitMs", C.c_float)]


# ---- extensions (include/mrt_ext.h) -----------------------------------------

class Ray(C.Structure):
    _fields_ = [("origin", F3), ("tMax", C.c_float), ("dir", F3), ("pad", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("instance", C.c_uint32), ("prim", C.c_uint32), ("hit", C.c_uint32),
                ("u", C.c_float), ("v", C.c_float), ("pad", C.c_uint32 * 2)]


class Stats(_Sized):
    _fields_ = [("structSize", C.c_size_t), ("lastRenderMs", C.c_float), ("lastRenderSpp", C.c_uint32),
                ("commitBvhMs", C.c_float), ("commitEnvCdfMs", C.c_float), ("commitUploadMs", C.c_float),
                ("commitTotalMs", C.c_float), ("bvhNodes", C.c_uint32), ("triangles", C.c_uint32),
                ("instances", C.c_uint32), ("kernelLaunches", C.c_uint32), ("deviceBytes", C.c_uint64),
                ("raysClosest", C.c_uint64), ("raysShadow", C.c_uint64), ("nodeFetches", C.c_uint64),
                ("triTests", C.c_uint64), ("surfaceHits", C.c_uint64), ("commitH2DBytes", C.c_uint64),
                ("shadowNodeFetches", C.c_uint64), ("shadowTriTests", C.c_uint64), ("nodeBytes", C.c_uint32),
                ("triBytes", C.c_uint32), ("extendMs", C.c_float), ("shadeMs", C.c_float), ("shadowMs", C.c_float),
                ("otherMs", C.c_float), ("extendLaunches", C.c_uint32), ("cacheQueryMs", C.c_float),
                ("cacheTrainMs", C.c_float), ("cacheQueries", C.c_uint64), ("cacheRecords", C.c_uint64),
                ("cacheSteps", C.c_uint32), ("batchJobs", C.c_uint32), ("commitDeviceBlas", C.c_uint32),
                ("commitDeviceTlas", C.c_uint32)]


LOG_FN = C.CFUNCTYPE(None, C.c_int, C.c_char_p, C.c_void_p)

# numpy dtypes matching mrtxRay / mrtxHit (32 bytes each)
RAY_DTYPE = [("origin", "<f4", 3), ("tMax", "<f4"), ("dir", "<f4", 3), ("pad", "<f4")]
HIT_DTYPE = [("t", "<f4"), ("instance", "<u4"), ("prim", "<u4"), ("hit", "<u4"), ("u", "<f4"), ("v", "<f4"),
             ("pad", "<u4", 2)]

# (name, restype, argtypes) for every exported function
FUNCTIONS = [
    ("mrtCreateEngine", C.c_int, [C.POINTER(EngineDesc), C.POINTER(C.c_void_p)]),
    ("mrtDestroyEngine", None, [C.c_void_p]),
    ("mrtAddMesh", C.c_uint32, [C.c_void_p, C.POINTER(MeshDesc)]),
    ("mrtUpdateMesh", None, [C.c_void_p, C.c_uint32, C.POINTER(MeshDesc)]),
    ("mrtRemoveMesh", None, [C.c_void_p, C.c_uint32]),
    ("mrtAddInstance", C.c_uint32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    ("mrtSetInstanceTransform", None, [C.c_void_p, C.c_uint32, C.c_void_p]),
    ("mrtRemoveInstance", None, [C.c_void_p, C.c_uint32]),
    ("mrtAddMaterial", C.c_uint32, [C.c_void_p, C.POINTER(MaterialDesc)]),
    ("mrtUpdateMaterial", None, [C.c_void_p, C.c_uint32, C.POINTER(MaterialDesc)]),
    ("mrtRemoveMaterial", None, [C.c_void_p, C.c_uint32]),
    ("mrtAddTexture", C.c_uint32, [C.c_void_p, C.POINTER(TextureDesc)]),
    ("mrtRemoveTexture", None, [C.c_void_p, C.c_uint32]),
    ("mrtAddLight", C.c_uint32, [C.c_void_p, C.POINTER(LightDesc)]),
    ("mrtUpdateLight", None, [C.c_void_p, C.c_uint32, C.POINTER(LightDesc)]),
    ("mrtRemoveLight", None, [C.c_void_p, C.c_uint32]),
    ("mrtSetEnvironment", None, [C.c_void_p, C.POINTER(TextureDesc), C.c_float, C.c_float]),
    ("mrtSetCamera", None, [C.c_void_p, C.POINTER(CameraDesc)]),
    ("mrtSetCameraEx", None, [C.c_void_p, C.POINTER(CameraDescEx)]),
    ("mrtCommitScene", C.c_int, [C.c_void_p, C.POINTER(CommitStats)]),
    ("mrtSetRenderSettings", C.c_int, [C.c_void_p, C.POINTER(RenderSettings)]),
    ("mrtRenderFrame", C.c_int, [C.c_void_p, C.POINTER(FrameInfo)]),
    ("mrtReadFramebuffer", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    ("mrtResetAccumulation", None, [C.c_void_p]),
    ("mrtSetLogCallback", None, [LOG_FN, C.c_void_p]),
    ("mrtResultToString", C.c_char_p, [C.c_int]),
    ("mrtGetLastErrorMessage", C.c_char_p, []),
    ("mrtxRenderFrames", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(FrameInfo)]),
    ("mrtxTraceRays", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("mrtxTraceShadowRays", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("mrtxReadAccumulation", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32)]),
    ("mrtxGetStats", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("mrtxMeasureL2Bandwidth", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("mrtxBuildEnvCdf", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                  C.POINTER(C.c_float)]),
    ("mrtxSetSampleStream", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    ("mrtxSetTraversalBudget", C.c_int, [C.c_void_p, C.c_uint32]),
    ("mrtxSetBvhBuildThresholds", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    ("mrtxTraceRaysWavefront", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("mrtxSetRadianceCacheAveraging", C.c_int, [C.c_void_p, C.c_float]),
    ("mrtxSetRadianceCacheSchedule", C.c_int, [C.c_void_p, C.c_float, C.c_float]),
    ("mrtxRadianceCacheGradients", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                             C.c_void_p]),
    ("mrtxInjectAllocationFailure", C.c_int, [C.c_int32]),
    ("mrtxCopyAccumulationDevice", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int32]),
    ("mrtxBuildWideBvh", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                   C.POINTER(C.c_uint32)]),
    ("mrtxSetRadianceCache", C.c_int, [C.c_void_p, C.POINTER(RadianceCacheDesc)]),
    ("mrtxSetDenoiser", C.c_int, [C.c_void_p, C.POINTER(DenoiserDesc)]),
    ("mrtxReadDenoised", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    ("mrtxReadDenoiserGuides", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]),
    ("mrtxRadianceCacheQuery", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("mrtxRadianceCacheTrain", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                         C.POINTER(C.c_float)]),
    ("mrtxRadianceCacheParams", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mrtxRenderBatch", C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_uint32), C.c_uint32,
                                  C.POINTER(FrameInfo)]),
    ("mrtxBuildMeshBvh", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32)]),
    ("mrtxBuildEnvCdfNoAlloc", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
]

# radiance cache sizes (floats)
CACHE_GRID_FLOATS = 16 * (1 << 19) * 2
CACHE_MLP_FLOATS = 6 * 64 * 64

# mrtxBuildMeshBvh builders
MRTX_BVH_HOST_SAH, MRTX_BVH_HOST_LBVH, MRTX_BVH_DEVICE_LBVH = 0, 1, 2

# mrtxBuildEnvCdfNoAlloc's height limit (MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT)
ENV_CDF_NOALLOC_MAX_HEIGHT = 8192

# numpy dtype of one 80-byte MrtWideNode
WIDE_NODE_DTYPE = [("p", "<f4", 3), ("e", "u1", 3), ("imask", "u1"), ("childBase", "<u4"), ("primBase", "<u4"),
                   ("meta", "u1", 8), ("qlo", "u1", (3, 8)), ("qhi", "u1", (3, 8))]
