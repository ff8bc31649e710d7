"""CudaEngine — the executor a CompiledRenderer runs on, over the C ABI.

Mirrors the reference's Engine surface (``src/engine/Engine.ts:83-438``):

* ``register_scene``  ~ ``registerDataTexture`` for the whole scene-data plan (:438)
* ``load_renderer`` / ``select_renderer`` (:147-186)
* ``render_frame``    ~ ``renderFrame`` (:190-204): sampleCount advances per sample,
  resetSalt decorrelates accumulation resets; ``spp`` folds several frames per call
* ``read_export``     ~ ``readExport`` (:351): linear HDR radiance / variance
* ``reset`` / ``pin_reset_salt`` ~ accumulation reset and the witness salt pin

Errors from the library raise ``EngineError`` carrying ``ptr_last_error``.
"""
import ctypes as C

import numpy as np

from . import abi
from ._native import load


class EngineError(RuntimeError):
    def __init__(self, code, message):
        self.code = code
        super().__init__(f"ptx_rt error {code}: {message}")


# Tile offsets are multiples of this (src/app/tiling.ts: TILE_ALIGN); the default tile
# edge of a production render (src/app/TiledRenderer.ts: DEFAULT_TILE_SIZE).
TILE_ALIGN = 64
DEFAULT_TILE_SIZE = 1024


def plan_tiles(width, height, tile_size):
    """``planTiles`` (src/app/tiling.ts:43-63): cover a width x height image with tiles of
    the requested size rounded up to TILE_ALIGN, anchored at the lower-left corner (engine
    coordinates, y from the bottom), listed top row first and left to right; the last
    column and the top row are cut to the image."""
    for name, v in (("width", width), ("height", height), ("tileSize", tile_size)):
        if not isinstance(v, int) or v < 1:
            raise ValueError(f"planTiles: {name} must be a positive integer (got {v})")
    size = -(-tile_size // TILE_ALIGN) * TILE_ALIGN
    cols, rows = -(-width // size), -(-height // size)
    tiles = []
    for row in range(rows):
        y = (rows - 1 - row) * size
        for col in range(cols):
            x = col * size
            tiles.append({"col": col, "row": row, "x": x, "y": y,
                          "width": min(size, width - x), "height": min(size, height - y)})
    return {"cols": cols, "rows": rows, "size": size, "tiles": tiles}


def _source_revision():
    """The source revision of this package (git HEAD), or 'unknown' outside a checkout."""
    import os
    import subprocess
    try:
        out = subprocess.run(["git", "rev-parse", "--short", "HEAD"], capture_output=True, text=True, timeout=5,
                             cwd=os.path.dirname(os.path.abspath(__file__)))
        return out.stdout.strip() or "unknown" if out.returncode == 0 else "unknown"
    except (OSError, subprocess.SubprocessError):
        return "unknown"


class CudaEngine:
    def __init__(self, device=0):
        self.lib = load()
        self.ctx = C.c_void_p()
        rc = self.lib.ptr_create(device, C.byref(self.ctx))
        if rc != abi.PTR_OK:
            raise EngineError(rc, f"cannot create a context on CUDA device {device}")
        self.scene = None
        self._scene_data = None
        self.programs = {}
        self.renderers = {}
        self.current = None
        self.sample_count = 0
        self.reset_salt = 0
        self._pinned_salt = None
        self.width = self.height = 0
        self.params = {}
        self._batches = []

    # -- errors ---------------------------------------------------------------------
    def _check(self, rc):
        if rc != abi.PTR_OK:
            msg = self.lib.ptr_last_error(self.ctx)
            raise EngineError(rc, msg.decode() if msg else "")
        return rc

    # -- scene data --------------------------------------------------------------------
    def set_accel_build(self, where):
        """Where later register_scene calls build mesh BVHs: 'host' (the reference's SAH
        builders restated, the default) or 'device' (linear BVH + wide collapse on the GPU)."""
        code = {"host": abi.BUILD_HOST, "device": abi.BUILD_DEVICE}[where]
        self._check(self.lib.ptr_set_accel_build(self.ctx, code))

    def register_scene(self, packed):
        """Upload a packed scene (host arrays are copied; the host keeps ownership)."""
        if self.scene is not None:
            self.lib.ptr_free_scene(self.scene)
            self.scene = None
        desc = packed.desc()
        h = C.c_void_p()
        self._check(self.lib.ptr_upload_scene(self.ctx, C.byref(desc), C.byref(h)))
        self.scene = h
        self._scene_data = packed
        self.reset()

    def register_scene_rails(self, packed, rails, with_orders=True, bare=True):
        """Upload a packed scene whose array data comes as the reference's packed channels
        (``rails.pack``: rail v2) through ptr_upload_scene_rails.  bare: the description's
        mesh positions/indices and batch placements are left NULL, so everything of the
        meshes and batches comes from the rails.  with_orders: pass the leaf permutations
        (hit ids are the caller's), else hit ids are leaf indices."""
        if self.scene is not None:
            self.lib.ptr_free_scene(self.scene)
            self.scene = None
        desc = packed.desc()
        if bare:
            for i in range(desc.n_meshes):
                desc.meshes[i].positions = None
                desc.meshes[i].indices = None
                desc.meshes[i].tri_alpha = None
            for i in range(desc.n_batches):
                desc.batches[i].placements = None
        st = rails.struct(with_orders)
        h = C.c_void_p()
        self._check(self.lib.ptr_upload_scene_rails(self.ctx, C.byref(desc), C.byref(st), C.byref(h)))
        self.scene = h
        self._scene_data = packed
        self.reset()

    # -- renderers ----------------------------------------------------------------------
    def load_renderer(self, renderer):
        h = C.c_void_p()
        self._check(self.lib.ptr_compile(self.ctx, C.byref(renderer.program), C.byref(h)))
        if renderer.id in self.programs:
            self.lib.ptr_free_program(self.programs[renderer.id])
        self.programs[renderer.id] = h
        self.renderers[renderer.id] = renderer
        if self.current is None:
            self.current = renderer.id
        return renderer.id

    def select_renderer(self, rid):
        if rid not in self.programs:
            raise KeyError(f"renderer {rid!r} not loaded")
        self.current = rid
        self.reset()

    def set_parameter(self, path, value):
        """Live parameter (camera.* re-evaluates the camera uniforms; a triggersReset
        parameter resets accumulation)."""
        self.params[path] = value
        self.reset()

    # -- accumulation ---------------------------------------------------------------------
    def pin_reset_salt(self, salt):
        self._pinned_salt = salt
        self.reset_salt = salt

    def reset(self):
        self.sample_count = 0
        if self._pinned_salt is None:
            self.reset_salt += 1
        else:
            self.reset_salt = self._pinned_salt

    def _frame(self, width, height, spp, accumulate, image=None):
        """A ptr_frame of this engine's state; ``image`` = the full image's (width, height)
        when the frame is one tile of it (engine.imageSize)."""
        r = self.renderers[self.current]
        fr = abi.Frame()
        fr.width, fr.height = width, height
        fr.first_sample = self.sample_count
        fr.spp = spp
        fr.reset_salt = self.reset_salt & 0xFFFFFFFF
        fr.accumulate = 1 if accumulate else 0
        iw, ih = image or (width, height)
        fr.camera = r.camera(self.params, iw, ih)
        fr.image_size = (C.c_int32 * 2)(iw, ih)
        return fr

    def render_frame(self, width, height, spp=1, sync=False):
        """Render ``spp`` more samples per pixel into the current renderer's film."""
        if self.scene is None or self.current is None:
            raise EngineError(abi.PTR_E_INVALID, "no scene registered or no renderer loaded")
        if (width, height) != (self.width, self.height):
            self.width, self.height = width, height
            self.reset()
        fr = self._frame(width, height, spp, accumulate=self.sample_count > 0)
        self._check(self.lib.ptr_render(self.programs[self.current], self.scene, C.byref(fr)))
        self.sample_count += spp
        if sync:
            self.sync()
        return self.sample_count

    def render_samples(self, width, height, spp):
        """Render and also return every sample's radiance, shape (spp, H, W, 3)."""
        self.width, self.height = width, height
        fr = self._frame(width, height, spp, accumulate=self.sample_count > 0)
        out = np.zeros((spp, height, width, 3), np.float32)
        self._check(self.lib.ptr_render_samples(self.programs[self.current], self.scene, C.byref(fr),
                                                out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        self.sample_count += spp
        return out

    def stream_handle(self):
        """The context's cudaStream_t as an integer (e.g. for torch.cuda.ExternalStream)."""
        h = C.c_void_p()
        self._check(self.lib.ptr_get_stream(self.ctx, C.byref(h)))
        return h.value or 0

    def sync(self, timeout_ms=-1):
        self._check(self.lib.ptr_sync(self.ctx, timeout_ms))

    def read_export(self, name="radiance", out=None):
        """Linear HDR export as (H, W, 3) float32, row 0 = bottom (gl_FragCoord order)."""
        if out is None:
            out = np.empty((self.height, self.width, 3), np.float32)
        self._check(self.lib.ptr_read_export(self.programs[self.current], name.encode(),
                                             out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    # -- production outputs ------------------------------------------------------------------
    def render_tiled(self, width, height, spp, tile_size=None, pictures=("radiance",), scene_id=None):
        """A tiled production render (TiledRenderer.render, src/app/TiledRenderer.ts:63-143):
        the image is covered by tiles of ``tile_size`` rounded up to TILE_ALIGN
        (``plan_tiles``), each rendered at ``spp`` from a fresh accumulation with its
        pixel offset and the full image size, under one reset salt for the whole job (a
        salt the caller pinned is kept).  Every pixel therefore computes exactly what it
        would in one full-size render.  Returns ``(images, stamps)``: per picture a
        (height, width, 3) float32 array, row 0 = bottom, and its reproducibility stamp
        with the full image's resolution and spp."""
        if self.scene is None or self.current is None:
            raise EngineError(abi.PTR_E_INVALID, "no scene registered or no renderer loaded")
        if not isinstance(spp, int) or spp < 1:
            raise ValueError(f"Tiled render: spp must be a positive integer (got {spp})")
        plan = plan_tiles(width, height, tile_size or DEFAULT_TILE_SIZE)
        pinned = self._pinned_salt
        self.pin_reset_salt(pinned if pinned is not None else self.reset_salt + 1)
        images = {p: np.zeros((height, width, 3), np.float32) for p in pictures}
        stamps = {}
        try:
            for t in plan["tiles"]:
                self.render_tile(t["x"], t["y"], t["width"], t["height"], width, height, spp)
                for p in pictures:
                    images[p][t["y"]:t["y"] + t["height"], t["x"]:t["x"] + t["width"]] = self.read_export(p)
            for p in pictures:
                stamps[p] = self.render_stamp(p, scene_id=scene_id, resolution=(width, height), spp=spp)
        finally:
            if pinned is None:
                self._pinned_salt = None
            else:
                self.pin_reset_salt(pinned)
        return images, stamps

    def render_tile(self, x, y, tile_width, tile_height, width, height, spp, accumulate=False):
        """Render ``spp`` samples per pixel of the tile at (x, y) (y from the bottom) of a
        width x height image into the current renderer's film (engine.pixelOffset +
        engine.imageSize): from a fresh accumulation, or with ``accumulate`` onto the
        samples already folded for the same tile.  The film then holds the tile's pixels."""
        if self.scene is None or self.current is None:
            raise EngineError(abi.PTR_E_INVALID, "no scene registered or no renderer loaded")
        if not accumulate or (self.width, self.height) != (tile_width, tile_height):
            self.width, self.height = tile_width, tile_height
            self.reset()
        fr = self._frame(tile_width, tile_height, spp, accumulate=self.sample_count > 0, image=(width, height))
        fr.pixel_offset = (C.c_int32 * 2)(x, y)
        self._check(self.lib.ptr_render(self.programs[self.current], self.scene, C.byref(fr)))
        self.sample_count += spp

    def render_stamp(self, picture="radiance", scene_id=None, resolution=None, spp=None):
        """The reproducibility stamp of a saved picture (App.buildRenderStamp,
        src/app/App.ts:821-842; the RenderStamp of src/app/utils/file-export.ts:13-24):
        the picture, the scene id, the active strategy, its resolved measurement, the live
        parameters, the sample count, the resolution, the reset salt, the source revision
        ('unknown' when there is none) and a UTC date; plus this library's ABI version.
        A tiled render passes the full image's resolution and spp."""
        import datetime
        r = self.renderers.get(self.current)
        return {
            "picture": picture,
            "scene": scene_id or "unknown",
            "strategy": r.strategy if r is not None else None,
            "measurement": r.measurement if r is not None else None,
            "parameters": dict(self.params),
            "spp": int(self.sample_count if spp is None else spp),
            "resolution": list(resolution or (self.width, self.height)),
            "resetSalt": int(self.reset_salt),
            "git": _source_revision(),
            "date": datetime.datetime.now(datetime.timezone.utc).isoformat(),
            "abi": int(self.lib.ptr_abi_version()),
        }

    # -- differentiation ---------------------------------------------------------------------
    def backward(self, dl_dimage, width, height, spp, first_sample=0, salt=None):
        """Path-replay adjoint: gradient of a loss whose derivative with respect to the
        current renderer's image is ``dl_dimage`` ((H, W, 3), row 0 = bottom), estimated
        from ``spp`` samples per pixel.  Returns an (n_materials, GRAD_SLOTS) float64 array
        (slots: abi.GRAD_NAMES).  The film is left untouched."""
        n_mat = len(self._scene_data.materials)
        dl = np.ascontiguousarray(dl_dimage, dtype=np.float32)
        if dl.shape != (height, width, 3):
            raise ValueError(f"dl_dimage must have shape {(height, width, 3)}")
        r = self.renderers[self.current]
        fr = abi.Frame()
        fr.width, fr.height, fr.spp = width, height, spp
        fr.first_sample = first_sample
        fr.reset_salt = (self.reset_salt if salt is None else salt) & 0xFFFFFFFF
        fr.camera = r.camera(self.params, width, height)
        g = np.zeros((n_mat, abi.GRAD_SLOTS), np.float64)
        self._check(self.lib.ptr_backward(self.programs[self.current], self.scene, C.byref(fr),
                                          dl.ctypes.data_as(C.POINTER(C.c_float)),
                                          g.ctypes.data_as(C.POINTER(C.c_double)), g.size))
        return g

    def update_params(self, packed):
        """Push a packed scene's (edited) material table and region IORs to the device
        (the live-parameter path; shapes must be unchanged)."""
        self._check(self.lib.ptr_update_params(
            self.scene, packed.materials.ctypes.data_as(C.POINTER(abi.Material)), len(packed.materials),
            packed.regions.ctypes.data_as(C.POINTER(abi.Region)), len(packed.regions)))
        self._scene_data = packed
        self.reset()

    # -- launch tuning ---------------------------------------------------------------------
    def specialize(self, enable=True):
        """Compile the current renderer's kernels for the registered scene (ptr_specialize:
        NVRTC, per scene x strategy, cached per occupant census); later renders of this
        pair use them.  enable=False returns to the generic kernels.  Returns the compile
        seconds (0 when the module was cached)."""
        secs = C.c_double(0.0)
        self._check(self.lib.ptr_specialize(self.programs[self.current], self.scene if enable else None,
                                            C.byref(secs)))
        return secs.value

    def set_tuning(self, capacity=0, block=256, sort_buckets=1, ray_sort=0):
        """Pool capacity (0 = default), block size (128/256), occupant-sort buckets (1 = off)
        and the ray-coherence queue order (0/1) of every later render on this context
        (ptr_set_tuning)."""
        t = abi.Tuning(int(capacity), int(block), int(sort_buckets), int(ray_sort))
        self._check(self.lib.ptr_set_tuning(self.ctx, C.byref(t)))

    def get_tuning(self):
        t = abi.Tuning()
        self._check(self.lib.ptr_get_tuning(self.ctx, C.byref(t)))
        return {"capacity": t.capacity, "block": t.block, "sort_buckets": t.sort_buckets, "ray_sort": t.ray_sort}

    KERNEL_CLASSES = ("generate", "closest", "shade", "shadow", "film", "sort")

    def profile_render(self, width, height, spp, mode=abi.PROFILE_TIMING):
        """Render once instrumented: PROFILE_TIMING (CUDA events around every launch; per
        kernel class returns (summed device ms, launch count)) and/or PROFILE_WORK (the
        traversal tallies, read with counters())."""
        self._check(self.lib.ptr_profile_next(self.programs[self.current], mode))
        self.render_frame(width, height, spp, sync=True)
        nc = len(self.KERNEL_CLASSES)
        ms = (C.c_float * nc)()
        n = (C.c_int * nc)()
        self._check(self.lib.ptr_get_profile(self.programs[self.current], ms, n, nc))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    def counters(self):
        c = abi.Counters()
        self._check(self.lib.ptr_get_counters(self.programs[self.current], C.byref(c)))
        return {"paths": c.paths, "closest_queries": c.closest_queries, "shadow_queries": c.shadow_queries,
                "blas_nodes": c.nodes_visited, "triangles": c.prims_tested, "tlas_nodes": c.tlas_nodes,
                "instances": c.instances, "shadow_blas_nodes": c.shadow_work[0], "shadow_triangles": c.shadow_work[1],
                "shadow_tlas_nodes": c.shadow_work[2], "shadow_instances": c.shadow_work[3],
                "error_flags": c.error_flags}

    def batch(self, items):
        """A ``Batch`` of (renderer, packed scene) jobs on this engine's context."""
        b = Batch(self, items)
        self._batches.append(b)
        return b

    def close(self):
        for b in self._batches:
            b.close()
        self._batches.clear()
        for h in self.programs.values():
            self.lib.ptr_free_program(h)
        self.programs.clear()
        if self.scene is not None:
            self.lib.ptr_free_scene(self.scene)
            self.scene = None
        if self.ctx:
            self.lib.ptr_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many (renderer, scene) jobs rendered together: ``render`` draws every job's frame
    in ONE batched wavefront (``ptr_render_batch``: one path pool, one CUDA graph per
    wave over all jobs); ``render_plain`` draws the same frames one job per launch
    (``ptr_render``).  Each job keeps its own film, read with ``read_export(j)``.
    No counterpart in the reference, which draws one renderer per frame."""

    def __init__(self, engine, items):
        self.engine = engine
        self.lib = engine.lib
        self.scenes, self.programs, self.renderers, self.sizes = [], [], [], []
        self._packed = []
        try:
            for renderer, packed in items:
                desc = packed.desc()
                h = C.c_void_p()
                engine._check(self.lib.ptr_upload_scene(engine.ctx, C.byref(desc), C.byref(h)))
                self.scenes.append(h)
                self._packed.append(packed)
                p = C.c_void_p()
                engine._check(self.lib.ptr_compile(engine.ctx, C.byref(renderer.program), C.byref(p)))
                self.programs.append(p)
                self.renderers.append(renderer)
                self.sizes.append((0, 0))
        except Exception:
            self.close()
            raise

    def __len__(self):
        return len(self.programs)

    def _jobs(self, frames):
        """frames: per job (width, height, spp[, first_sample[, salt[, params]]])."""
        if len(frames) != len(self.programs):
            raise ValueError("one frame per job")
        arr = (abi.BatchJob * len(frames))()
        for j, f in enumerate(frames):
            w, h, spp = f[:3]
            first = f[3] if len(f) > 3 else 0
            salt = f[4] if len(f) > 4 else 0
            params = f[5] if len(f) > 5 else {}
            J = arr[j]
            J.prog = self.programs[j].value
            J.scene = self.scenes[j].value
            J.frame.width, J.frame.height, J.frame.spp = w, h, spp
            J.frame.first_sample = first
            J.frame.reset_salt = salt & 0xFFFFFFFF
            J.frame.accumulate = 1 if first > 0 else 0
            J.frame.camera = self.renderers[j].camera(params, w, h)
            self.sizes[j] = (w, h)
        return arr

    def render(self, frames):
        arr = self._jobs(frames)
        self.engine._check(self.lib.ptr_render_batch(self.engine.ctx, arr, len(arr)))

    def profile(self, frames):
        """Render batched once with CUDA events around each kernel class's launches; per
        kernel class (summed device ms, kernel launches)."""
        self.engine._check(self.lib.ptr_profile_batch_next(self.engine.ctx, abi.PROFILE_TIMING))
        self.render(frames)
        nc = len(CudaEngine.KERNEL_CLASSES)
        ms = (C.c_float * nc)()
        n = (C.c_int * nc)()
        self.engine._check(self.lib.ptr_get_batch_profile(self.engine.ctx, ms, n, nc))
        return {k: (ms[i], n[i]) for i, k in enumerate(CudaEngine.KERNEL_CLASSES)}

    def render_plain(self, frames, sync=True):
        """The same frames one job per launch, each job's whole spp budget in one
        ptr_render."""
        arr = self._jobs(frames)
        for j in range(len(arr)):
            self.engine._check(self.lib.ptr_render(self.programs[j], self.scenes[j], C.byref(arr[j].frame)))
        if sync:
            self.engine.sync()

    def render_progressive(self, frames, sync=True):
        """The reference's own plain schedule: one scene per frame and one sample per pixel
        per frame (Engine.renderFrame, src/engine/Engine.ts:190-204), i.e. spp ptr_render
        calls of 1 spp per job, each accumulating into the job's film."""
        arr = self._jobs(frames)
        for j in range(len(arr)):
            fr = abi.Frame()
            C.pointer(fr)[0] = arr[j].frame
            spp = fr.spp
            for k in range(spp):
                fr.spp = 1
                fr.first_sample = arr[j].frame.first_sample + k
                fr.accumulate = 1 if (k > 0 or arr[j].frame.accumulate) else 0
                self.engine._check(self.lib.ptr_render(self.programs[j], self.scenes[j], C.byref(fr)))
        if sync:
            self.engine.sync()

    def specialize_off(self):
        """Return every job's plain renders to the generic kernels (the batched kernels of
        the mix stay compiled)."""
        secs = C.c_double()
        for p in self.programs:
            self.engine._check(self.lib.ptr_specialize(p, None, C.byref(secs)))

    def specialize(self, plain=False):
        """Compile the batched kernels for this mix's occupant census (ptr_specialize_batch);
        with plain=True also each job's own per-scene kernels for render_plain /
        render_progressive (ptr_specialize).  Returns the compile seconds."""
        sizes = list(self.sizes)
        arr = self._jobs([(1, 1, 1)] * len(self.programs))
        self.sizes = sizes
        secs = C.c_double()
        self.engine._check(self.lib.ptr_specialize_batch(self.engine.ctx, arr, len(arr), C.byref(secs)))
        total = secs.value
        if plain:
            for j in range(len(arr)):
                self.engine._check(self.lib.ptr_specialize(self.programs[j], self.scenes[j], C.byref(secs)))
                total += secs.value
        return total

    def read_export(self, j, name="radiance"):
        w, h = self.sizes[j]
        out = np.empty((h, w, 3), np.float32)
        self.engine._check(self.lib.ptr_read_export(self.programs[j], name.encode(),
                                                    out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def counters(self):
        c = abi.Counters()
        self.engine._check(self.lib.ptr_get_batch_counters(self.engine.ctx, C.byref(c)))
        return {"paths": c.paths, "closest_queries": c.closest_queries, "shadow_queries": c.shadow_queries}

    def close(self):
        for p in self.programs:
            self.lib.ptr_free_program(p)
        for h in self.scenes:
            self.lib.ptr_free_scene(h)
        self.programs, self.scenes = [], []


def render(scene, strategy, width, height, spp, params=None, salt=0, device=0, engine=None):
    """Compile, upload and render one scene x strategy; returns (mean, variance, engine)."""
    from .compiler import Compiler
    renderer, packed = Compiler().compile(scene, strategy, params)
    eng = engine or CudaEngine(device)
    eng.register_scene(packed)
    eng.load_renderer(renderer)
    eng.select_renderer(renderer.id)
    eng.params = dict(params or {})
    eng.pin_reset_salt(salt)
    eng.render_frame(width, height, spp)
    mean = eng.read_export("radiance")
    var = eng.read_export("variance")
    return mean, var, eng
