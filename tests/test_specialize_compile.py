"""The per-scene kernels' sources compile with NVRTC for sm_100a (no GPU needed).

ptr_specialize compiles k_closest, k_shade and k_shadow from the device headers at run
time; this guards those headers on the CPU for the occupant censuses of the workloads
(the same options ptr_specialize passes: the masks, the unrolled region shapes, the
fixed-width-type prelude).  The GPU tests check that the compiled kernels render the
generic kernels' samples.  Skipped where NVRTC is absent.
"""
import ctypes as C
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRELUDE = (b"typedef signed char int8_t; typedef unsigned char uint8_t; typedef short int16_t;\n"
           b"typedef unsigned short uint16_t; typedef int int32_t; typedef unsigned int uint32_t;\n"
           b"typedef long long int64_t; typedef unsigned long long uint64_t;\n"
           b"#include \"wavefront.cuh\"\n")


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            return C.CDLL(name)
        except OSError:
            continue
    pytest.skip("NVRTC not available")


def _code(shapes):
    return sum(s << (4 * k) for k, s in enumerate(shapes))


# (material models, light kinds, environment kinds, region shapes in order, colour, direct, media)
CENSUS = {
    "cornell": (0b11, 0b1, 0b1, [2, 2, 2, 2, 2, 1, 1, 2], "ptx::f3", 2, "false"),
    "cornell-rough": (0b101001, 0b1, 0b1, [2, 2, 2, 2, 2, 1, 1, 2], "ptx::f3", 2, "false"),
    "mesh": (0b101, 0b0, 0b100, [0, 5], "ptx::f3", 2, "false"),
    "cornell-mesh-light": (0b11, 0b1000, 0b1, [2, 2, 2, 2, 2, 1, 1, 4], "ptx::f3", 2, "false"),
    "fog-mesh-light": (0b10001, 0b1011, 0b1, [0, 0, 1, 4], "ptx::f3", 1, "true"),
    "many-lights-no-tree": (0b100101, 0b1011, 0b1, [2, 2, 2, 2, 2, 1, 1, 5, 5, 4, 2], "ptx::f3", 2, "false", 0),
    "media-spectral": (0b10011, 0b11, 0b1, [0, 1, 1, 1, 2, 2, 2, 2], "ptx::s4", 1, "true"),
    "many-regions": (0b1, 0b1, 0b10, [2] * 16, "ptx::f3", 2, "false"),
}


@pytest.mark.parametrize("case", sorted(CENSUS))
def test_specialised_kernels_compile(case):
    lib = _nvrtc()
    mats, lights, envs, shapes, col, direct, media, *tree = CENSUS[case]
    names = [b"ptx::k_closest<false, false>",
             f"ptx::k_shade<{col}, {direct}, {media}, false, false>".encode(),
             f"ptx::k_shadow<{col}, {media}, false, false, false>".encode()]
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-fmad=false", b"-default-device",
            ("-I" + os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device")).encode(),
            ("-I" + os.path.join(ROOT, "include")).encode(),
            f"-DPTR_SPEC_MATS={mats}u".encode(), f"-DPTR_SPEC_LIGHTS={lights}u".encode(),
            f"-DPTR_SPEC_ENVS={envs}u".encode(),
            f"-DPTR_SPEC_SHAPES={sum(1 << s for s in set(shapes))}u".encode(),
            f"-DPTR_SPEC_NREGIONS={len(shapes)}".encode(), f"-DPTR_SPEC_SHAPE_CODE={_code(shapes)}ull".encode(),
            f"-DPTR_SPEC_TREE={tree[0] if tree else 1}".encode()]
    prog = C.c_void_p()
    assert lib.nvrtcCreateProgram(C.byref(prog), PRELUDE, b"ptr_specialize.cu", 0, None, None) == 0
    try:
        for n in names:
            assert lib.nvrtcAddNameExpression(prog, n) == 0
        arr = (C.c_char_p * len(opts))(*opts)
        rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
        size = C.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, C.byref(size))
        log = C.create_string_buffer(size.value)
        lib.nvrtcGetProgramLog(prog, log)
        assert rc == 0, log.value.decode(errors="replace")[:4000]
        cubin = C.c_size_t()
        assert lib.nvrtcGetCUBINSize(prog, C.byref(cubin)) == 0 and cubin.value > 0
        for n in names:
            low = C.c_char_p()
            assert lib.nvrtcGetLoweredName(prog, n, C.byref(low)) == 0 and low.value
    finally:
        lib.nvrtcDestroyProgram(C.byref(prog))


@pytest.mark.parametrize("media", ["false", "true"])
def test_batched_kernels_compile(media):
    """ptr_specialize_batch's union census of the uneven Cornell-style mix (Lambert,
    dielectric and GGX; quad lights; quads and spheres; no region unrolling), BATCH = true."""
    lib = _nvrtc()
    names = [b"ptx::k_closest<false, true>", f"ptx::k_shade<ptx::f3, 2, {media}, true, false>".encode(),
             f"ptx::k_shadow<ptx::f3, {media}, false, true, false>".encode()]
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-fmad=false", b"-default-device",
            ("-I" + os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device")).encode(),
            ("-I" + os.path.join(ROOT, "include")).encode(),
            b"-DPTR_SPEC_MATS=7u", b"-DPTR_SPEC_LIGHTS=1u", b"-DPTR_SPEC_ENVS=1u",
            f"-DPTR_SPEC_SHAPES={(1 << 1) | (1 << 2)}u".encode(), b"-DPTR_SPEC_NREGIONS=0",
            b"-DPTR_SPEC_SHAPE_CODE=0ull", b"-DPTR_SPEC_TREE=0"]
    prog = C.c_void_p()
    assert lib.nvrtcCreateProgram(C.byref(prog), PRELUDE, b"ptr_specialize.cu", 0, None, None) == 0
    try:
        for n in names:
            assert lib.nvrtcAddNameExpression(prog, n) == 0
        arr = (C.c_char_p * len(opts))(*opts)
        rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
        size = C.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, C.byref(size))
        log = C.create_string_buffer(size.value)
        lib.nvrtcGetProgramLog(prog, log)
        assert rc == 0, log.value.decode(errors="replace")[:4000]
        for n in names:
            low = C.c_char_p()
            assert lib.nvrtcGetLoweredName(prog, n, C.byref(low)) == 0 and low.value
    finally:
        lib.nvrtcDestroyProgram(C.byref(prog))


def test_wide_math_kernels_compile():
    """The per-scene kernels with PTR_WIDE_MATH (double-rounded float transcendentals, the
    parity build of tests/test_gpu_math_parity.py)."""
    lib = _nvrtc()
    names = [b"ptx::k_closest<false, false>", b"ptx::k_shade<ptx::f3, 2, true, false, false>",
             b"ptx::k_shadow<ptx::f3, true, false, false, false>"]
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-fmad=false", b"-default-device", b"-DPTR_WIDE_MATH",
            ("-I" + os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device")).encode(),
            ("-I" + os.path.join(ROOT, "include")).encode()]
    prog = C.c_void_p()
    assert lib.nvrtcCreateProgram(C.byref(prog), PRELUDE, b"ptr_specialize.cu", 0, None, None) == 0
    try:
        for n in names:
            assert lib.nvrtcAddNameExpression(prog, n) == 0
        arr = (C.c_char_p * len(opts))(*opts)
        rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
        size = C.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, C.byref(size))
        log = C.create_string_buffer(size.value)
        lib.nvrtcGetProgramLog(prog, log)
        assert rc == 0, log.value.decode(errors="replace")[:4000]
    finally:
        lib.nvrtcDestroyProgram(C.byref(prog))


@pytest.mark.parametrize("media", ["false", "true"])
def test_replay_kernels_compile(media):
    """The adjoint replay's kernels (ADJ = true) for the inverse-rendering scene's census:
    Lambert, dielectric, GGX and the null interface; one quad light; quads and spheres; 70
    regions (too many to unroll)."""
    lib = _nvrtc()
    names = [b"ptx::k_closest<false, false>", f"ptx::k_shade<ptx::f3, 2, {media}, false, true>".encode(),
             f"ptx::k_shadow<ptx::f3, {media}, false, false, true>".encode()]
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-fmad=false", b"-default-device",
            ("-I" + os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device")).encode(),
            ("-I" + os.path.join(ROOT, "include")).encode(),
            b"-DPTR_SPEC_MATS=23u", b"-DPTR_SPEC_LIGHTS=1u", b"-DPTR_SPEC_ENVS=1u",
            f"-DPTR_SPEC_SHAPES={(1 << 1) | (1 << 2)}u".encode(), b"-DPTR_SPEC_NREGIONS=0",
            b"-DPTR_SPEC_SHAPE_CODE=0ull", b"-DPTR_SPEC_TREE=0"]
    prog = C.c_void_p()
    assert lib.nvrtcCreateProgram(C.byref(prog), PRELUDE, b"ptr_specialize.cu", 0, None, None) == 0
    try:
        for n in names:
            assert lib.nvrtcAddNameExpression(prog, n) == 0
        arr = (C.c_char_p * len(opts))(*opts)
        rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
        size = C.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, C.byref(size))
        log = C.create_string_buffer(size.value)
        lib.nvrtcGetProgramLog(prog, log)
        assert rc == 0, log.value.decode(errors="replace")[:4000]
        for n in names:
            low = C.c_char_p()
            assert lib.nvrtcGetLoweredName(prog, n, C.byref(low)) == 0 and low.value
    finally:
        lib.nvrtcDestroyProgram(C.byref(prog))
