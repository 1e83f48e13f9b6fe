"""The add-on's render session and F12 loop over the CUDA ``lucidrenderer`` module.

Lucid's Blender add-on drives the C++ core through ``RenderSession``
(LucidRenderer/render_session.py:61-674), which ``engine.py`` (F12 renders)
and ``viewport.py`` (the async viewport) call.  This module keeps that
surface — the same classes, method names, defaults and failure behaviour
(methods return False / None / "{}" instead of raising) — minus the parts
that need Blender itself (``sync_scene`` over a depsgraph, the scene cache).

What changes is the data path the callers see:

* images are float32 numpy arrays, rendered straight into the array
  (``Renderer.render_tile_numpy``) instead of Python float lists;
* the F12 loop (engine.py:401-447) adds each iteration's sample sum into a
  numpy buffer reused between iterations, instead of the per-float Python
  loop over an ``array('f')`` (engine.py:437-443), and builds Blender's
  display rectangle in one vector operation (engine.py:575-599).  Both give
  the same float32 values as the list code: a float32 sum computed in double
  and stored as float32 rounds to the float32 sum, and the display scale is
  applied in double as Python does.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass
from typing import Any, Callable, List, Optional, Tuple

import numpy as np

import lucidrenderer


# ---------------------------------------------------------------------------
# State records (LucidRenderer/state.py:44-119)
# ---------------------------------------------------------------------------

@dataclass(frozen=True)
class CameraParams:
    """Camera: position, view direction, up vector (both normalised), fov in degrees."""
    pos: Tuple[float, float, float]
    dir: Tuple[float, float, float]
    up: Tuple[float, float, float]
    fov: float


@dataclass(frozen=True)
class RenderParams:
    """One render call (state.py:74-95): same fields and defaults."""
    width: int
    height: int
    samples: int = 1
    max_bounces: int = 8
    algorithm: str = "nee"
    debug_mode: Optional[str] = None
    sample_offset: int = 0
    backend: str = "cpu"


@dataclass
class RenderResult:
    """A render call's output (state.py:102-119); ``pixels`` is a float32
    array of width * height * 4 values (RGBA sums over the call's samples,
    bottom row first)."""
    pixels: Any
    width: int
    height: int
    samples: int = 1
    cancelled: bool = False
    job_id: int = 0


# Debug-mode names the add-on passes, upper or lower case
# (render_session.py:549-555).
_DEBUG_MODES = {
    "NORMAL": "normal", "ALBEDO": "albedo", "EMISSION": "emission",
    "normal": "normal", "albedo": "albedo", "emission": "emission",
    "volume": "volume",
}


class RenderSession:
    """One render engine instance's renderer (render_session.py:61-674).

    Every backend value renders on the GPU: the CUDA module has no CPU path,
    so ``backend`` only selects between the two method names the reference
    calls (``render_tile`` and ``render_tile_gpu`` run the same code here).
    """

    _session_counter: int = 0

    def __init__(self):
        RenderSession._session_counter += 1
        self._session_id = RenderSession._session_counter
        self._renderer: Any = lucidrenderer.Renderer()
        self._executor: Optional[ThreadPoolExecutor] = ThreadPoolExecutor(max_workers=1)
        self._scene_hash: Optional[str] = None
        self._job_id = 0
        self._diagnostics_enabled = False

    @property
    def session_id(self) -> int:
        return self._session_id

    @property
    def is_available(self) -> bool:
        return self._renderer is not None

    @property
    def renderer(self) -> Any:
        """The underlying ``lucidrenderer.Renderer``."""
        return self._renderer

    def shutdown(self) -> None:
        """Joins the async worker, cancels any render and drops the renderer
        (render_session.py:128-154)."""
        if self._renderer is not None:
            self._renderer.render_stop_async()
            self._renderer.cancel()
        if self._executor is not None:
            self._executor.shutdown(wait=False)
            self._executor = None
        self._renderer = None
        self._scene_hash = None

    # -- scene ---------------------------------------------------------------

    def load_scene_if_changed(self, scene_hash: str, json_str: str) -> bool:
        """Loads the scene unless ``scene_hash`` is the loaded one
        (render_session.py:158-186); sets the object names from the meshes."""
        if not self.is_available:
            return False
        if scene_hash == self._scene_hash:
            return True
        if self._renderer.load_scene_json(json_str):
            self._scene_hash = scene_hash
            self._set_object_names_from_json(json_str)
            return True
        return False

    def _set_object_names_from_json(self, json_str: str) -> None:
        try:
            meshes = json.loads(json_str).get("meshes", [])
            self._renderer.set_object_names([m.get("name", f"Object_{i}") for i, m in enumerate(meshes)])
        except Exception:
            pass

    def load_scene_json(self, json_str: str) -> bool:
        """Loads a scene keyed by the MD5 of its text (render_session.py:204-214)."""
        return self.load_scene_if_changed(hashlib.md5(json_str.encode()).hexdigest(), json_str)

    def load_scene_file(self, scene_file: str) -> bool:
        try:
            with open(scene_file, "r") as f:
                json_str = f.read()
        except OSError:
            return False
        return self.load_scene_json(json_str)

    def invalidate_scene(self) -> None:
        self._scene_hash = None

    # -- camera and algorithm -------------------------------------------------

    def set_camera(self, camera: CameraParams) -> None:
        if not self.is_available:
            return
        self._renderer.set_camera(*camera.pos, *camera.dir, *camera.up, camera.fov)

    def set_camera_from_dict(self, cam_params: dict) -> None:
        if not self.is_available:
            return
        pos, dir_, up = cam_params["pos"], cam_params["dir"], cam_params["up"]
        self._renderer.set_camera(pos[0], pos[1], pos[2], dir_[0], dir_[1], dir_[2], up[0], up[1], up[2],
                                  cam_params["fov"])

    def set_algorithm(self, algorithm: str) -> None:
        if not self.is_available:
            return
        self._renderer.set_algorithm(algorithm)

    # -- async accumulator (render_session.py:313-371) --------------------------

    def start_render_async(self, width: int, height: int, max_depth: int) -> bool:
        if not self.is_available:
            return False
        self._renderer.render_start_async(width, height, max_depth)
        return self._renderer.is_render_async_running()

    def poll_render_async(self):
        """(samples, RGBA float32 array averaged over the samples); samples == 0
        means no snapshot yet."""
        if not self.is_available:
            return 0, np.zeros(0, np.float32)
        return self._renderer.render_poll_async()

    def stop_render_async(self) -> None:
        if self.is_available:
            self._renderer.render_stop_async()

    def reset_render_async(self, width: int, height: int, max_depth: int) -> None:
        if self.is_available:
            self._renderer.render_reset_async(width, height, max_depth)

    def is_render_async_running(self) -> bool:
        return self.is_available and self._renderer.is_render_async_running()

    def snapshot_revision_async(self) -> int:
        return self._renderer.render_snapshot_revision_async() if self.is_available else 0

    # -- diagnostics (render_session.py:390-528) --------------------------------

    def enable_diagnostics(self, preset: str = "standard") -> bool:
        if not self.is_available:
            return False
        try:
            if preset == "minimal":
                config = lucidrenderer.PathRecordingConfig.minimal()
            elif preset == "detailed":
                config = lucidrenderer.PathRecordingConfig.detailed()
            else:
                config = lucidrenderer.PathRecordingConfig.standard()
            self._renderer.enable_diagnostics(config)
            self._diagnostics_enabled = True
            return True
        except Exception:
            return False

    def disable_diagnostics(self) -> None:
        if not self.is_available:
            return
        try:
            self._renderer.disable_diagnostics()
            self._diagnostics_enabled = False
        except Exception:
            pass

    def is_diagnostics_enabled(self) -> bool:
        return self._diagnostics_enabled and self.is_available

    def _diag(self, name: str, *args, default=None):
        if not self.is_available or not self._diagnostics_enabled:
            return default
        try:
            return getattr(self._renderer, name)(*args)
        except Exception:
            return default

    def get_diagnostic_stats(self):
        return self._diag("get_diagnostic_stats")

    def get_diagnostic_variance_map(self):
        return self._diag("get_diagnostic_variance_map")

    def get_pixel_diagnostic(self, x: int, y: int):
        return self._diag("get_pixel_diagnostic", x, y)

    def get_top_variance_groups(self, count: int = 10):
        return self._diag("get_top_variance_groups", count)

    def export_diagnostic_json(self) -> str:
        return self._diag("export_diagnostic_json", default="{}")

    def clear_diagnostics(self) -> None:
        if not self.is_available:
            return
        try:
            self._renderer.clear_diagnostics()
        except Exception:
            pass

    # -- rendering (render_session.py:530-649) ------------------------------------

    def render_tile(self, params: RenderParams, out: Optional[np.ndarray] = None) -> RenderResult:
        """Renders the full frame ``params`` describes; ``out`` (float32,
        width * height * 4 values) receives the pixels when given."""
        if not self.is_available:
            return RenderResult(pixels=np.zeros(0, np.float32), width=params.width, height=params.height,
                                cancelled=True)
        r = self._renderer
        r.set_algorithm(params.algorithm)
        w, h = params.width, params.height
        if params.debug_mode:
            mode = _DEBUG_MODES.get(params.debug_mode, "normal")
            call = r.render_debug_gpu if params.backend == "gpu" else r.render_debug
            pixels = np.asarray(call(0, 0, w, h, w, h, mode), dtype=np.float32)
            if out is not None:
                out.reshape(-1)[:] = pixels
                pixels = out
        else:
            pixels = r.render_tile_numpy(0, 0, w, h, w, h, params.samples, params.sample_offset,
                                         params.max_bounces, out)
        self._job_id += 1
        return RenderResult(pixels=pixels.reshape(-1), width=w, height=h, samples=params.samples,
                            cancelled=r.is_cancelled(), job_id=self._job_id)

    def render_tile_async(self, params: RenderParams, scene_file: str, camera: CameraParams) -> Optional[Future]:
        """Loads ``scene_file``, sets the camera and renders on the session's
        worker thread (render_session.py:610-649)."""
        if not self.is_available or self._executor is None:
            return None

        def task() -> RenderResult:
            if not self.load_scene_file(scene_file):
                return RenderResult(pixels=np.zeros(0, np.float32), width=params.width, height=params.height,
                                    cancelled=True)
            self.set_camera(camera)
            return self.render_tile(params)

        return self._executor.submit(task)

    def cancel(self) -> None:
        if self._renderer is not None:
            self._renderer.cancel()

    def is_cancelled(self) -> bool:
        return self._renderer.is_cancelled() if self._renderer is not None else False

    def reset_cancel(self) -> None:
        if self._renderer is not None:
            self._renderer.reset_cancel()

    def __repr__(self) -> str:
        return f"<RenderSession #{self._session_id} ({'available' if self.is_available else 'unavailable'})>"


# ---------------------------------------------------------------------------
# The F12 loop (LucidRenderer/engine.py:401-447, 558-599)
# ---------------------------------------------------------------------------

def compute_sample_iterations(target_samples: int) -> List[int]:
    """The F12 sample schedule (engine.py:558-573): one call up to 16
    samples, else 4, 8, 16, 32, then 64 per call until the target."""
    if target_samples <= 16:
        return [target_samples]
    iterations = []
    remaining, batch = target_samples, 4
    while remaining > 0:
        n = min(batch, remaining)
        iterations.append(n)
        remaining -= n
        batch = min(batch * 2, 64)
    return iterations


# Host threads for the F12 loop's per-iteration array work: numpy releases
# the GIL inside its loops, so contiguous chunks of a 1080p frame (8.3 M
# floats) convert in parallel (62 ms -> 12 ms per iteration on 8 cores).
_CHUNK = 1 << 18
_host_pool: Optional[ThreadPoolExecutor] = None


def _pool() -> ThreadPoolExecutor:
    global _host_pool
    if _host_pool is None:
        _host_pool = ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1)), thread_name_prefix="lucid-f12")
    return _host_pool


def _chunked(n: int, fn) -> None:
    if n <= _CHUNK:
        fn(0, n)
        return
    for f in [_pool().submit(fn, s, min(s + _CHUNK, n)) for s in range(0, n, _CHUNK)]:
        f.result()


def display_pixels(accumulated: np.ndarray, total_samples: int, out: Optional[np.ndarray] = None) -> np.ndarray:
    """Blender's Combined-pass rectangle from the accumulated sums
    (engine.py:575-599): RGB times 1 / total_samples (in double, then
    float32 as Blender stores it), alpha 1; shape (pixels, 4).  Every
    channel is scaled in double over contiguous chunks on the host threads
    and alpha set afterwards, which gives the same float32 values as the
    reference's per-value loop.  `out` (float32, pixels * 4) is filled and
    returned instead of a new array when given."""
    acc = np.ascontiguousarray(accumulated, dtype=np.float32).reshape(-1)
    rect = np.empty_like(acc) if out is None else out.reshape(-1)
    inv = 1.0 / total_samples

    def part(s, e):
        np.copyto(rect[s:e], np.multiply(acc[s:e], inv, dtype=np.float64), casting="same_kind")

    _chunked(acc.size, part)
    rect = rect.reshape(-1, 4)
    rect[:, 3] = 1.0
    return rect


@dataclass
class F12Result:
    """What the F12 loop leaves: the RGBA sums (float32, width * height * 4,
    alpha summing to the number of iterations as in the reference), the
    samples taken and whether the loop stopped early."""
    accumulated: Optional[np.ndarray]
    total_samples: int
    iterations: List[int]
    cancelled: bool
    render_s: float
    host_s: float


def render_f12(session: RenderSession, width: int, height: int, target_samples: int, max_bounces: int = 8,
               algorithm: str = "nee", backend: str = "gpu",
               test_break: Optional[Callable[[], bool]] = None,
               on_progress: Optional[Callable[[float, int, int, float], None]] = None,
               on_result: Optional[Callable[[np.ndarray, int], None]] = None) -> F12Result:
    """The add-on's progressive F12 render (engine.py:401-447).

    Calls ``session.render_tile`` once per entry of
    ``compute_sample_iterations(target_samples)`` with the running sample
    offset, adds each call's sums into one float32 buffer and hands the
    display rectangle to ``on_result`` after every iteration (Blender's
    ``begin_result`` / ``end_result``).  ``test_break`` is polled before each
    iteration and cancels the session when it returns True;
    ``on_progress(progress, samples_done, samples_total, eta_s)`` mirrors
    the status line the add-on updates.
    """
    iterations = compute_sample_iterations(target_samples)
    max_samples = sum(iterations)
    accumulated = None
    # the first iteration renders straight into the sums, later ones into
    # `scratch`; the display rectangle handed to on_result is one buffer
    # refilled every iteration (Blender copies it at once: foreach_set)
    acc_buf = np.empty(width * height * 4, np.float32)
    scratch = np.empty(width * height * 4, np.float32)
    shown = np.empty(width * height * 4, np.float32) if on_result is not None else None
    total = 0
    cancelled = False
    render_s = host_s = 0.0
    start = time.perf_counter()
    for n in iterations:
        if test_break is not None and test_break():
            session.cancel()
            cancelled = True
            break
        if on_progress is not None:
            progress = total / max_samples
            elapsed = time.perf_counter() - start
            eta = (elapsed / max(progress, 0.001)) * (1 - progress) if progress > 0 else 0.0
            on_progress(progress, total, max_samples, eta)
        params = RenderParams(width=width, height=height, samples=n, sample_offset=total,
                              max_bounces=max_bounces, algorithm=algorithm, backend=backend)
        t0 = time.perf_counter()
        result = session.render_tile(params, out=acc_buf if accumulated is None else scratch)
        t1 = time.perf_counter()
        render_s += t1 - t0
        if result.cancelled:
            cancelled = True
            break
        if accumulated is None:
            accumulated = acc_buf
        else:
            _chunked(accumulated.size, lambda s, e: np.add(accumulated[s:e], scratch[s:e], out=accumulated[s:e]))
        total += n
        if on_result is not None:
            on_result(display_pixels(accumulated, total, out=shown), total)
        host_s += time.perf_counter() - t1
    return F12Result(accumulated=accumulated, total_samples=total, iterations=iterations, cancelled=cancelled,
                     render_s=render_s, host_s=host_s)
