"""Headless ray-marched viewer.

The reference viewer (th/*/render_gl.py ``GLRenderer`` on
visualization/gl_backend.py ``GLBackend``) builds an RGBA volume from the
simulation's density and field in CUDA, uploads it as a 3-D texture and
ray-marches it in an OpenGL fragment shader.  ``HeadlessRenderer`` keeps the
viewer's controls, camera and defaults and computes the same frame with two
library calls into plain device buffers, no window or graphics API:

* ``sky_build_rgba_volume`` -- the extrema and the (Z, Y, X, 4) FP32 volume;
* ``sky_render_volume``     -- the ray-march into a (height, width, 4) FP32
  RGBA image, row 0 at the top.

``save_screenshot`` writes the RGB bytes the reference reads back with
glReadPixels (GL_RGB, GL_UNSIGNED_BYTE, flipped to top-first) as a PNG.
"""
from __future__ import annotations

import os
from datetime import datetime

import numpy as np

from .. import _lib

DISPLAY_ENERGY_SINGLE = 1
DISPLAY_BARYON = 2
DISPLAY_TITLES = {DISPLAY_ENERGY_SINGLE: "Energy density", DISPLAY_BARYON: "Baryon density"}


def advance_solver(sim, steps_per_frame: int, state: dict) -> None:
    """The viewer's solver advance (th/nuclear_skyrme/render_gl.py:944-973): the first call
    takes the energy from ``observables()``; with Newton flow on, ``steps_per_frame`` calls of
    ``sim.step`` update ``state["energy"]``, ``state["error"]`` and ``state["epochs"]``."""
    if state.get("energy") is None:
        state["energy"] = float(sim.observables()["energy"])
    if sim.rp.newtonflow:
        for _ in range(int(steps_per_frame)):
            state["energy"], state["error"] = sim.step(state["energy"])
            state["epochs"] += 1


def hud_text(sim, state: dict, running: bool = True):
    """The viewer's two HUD lines (render_gl.py:1055-1069): time and epochs with the error,
    then energy, baryon number and the run state."""
    epochs = int(state.get("epochs", 0))
    top = f"t={epochs * float(sim.p_f_h[7]):.3f} ({epochs} epochs)"
    if state.get("error") is not None:
        top += f", err={float(state['error']):.3e}"
    parts = []
    if state.get("energy") is not None:
        parts.append(f"E={float(state['energy']):.6f}")
    if state.get("baryon") is not None:
        parts.append(f"B={float(state['baryon']):.6f}")
    parts.append("running" if running else "paused")
    return top, ", ".join(parts)


def viewer_loop(sim, renderer, density_for_mode, *, steps_per_frame: int = 5, frames: int = 1,
                output_dir: str | None = "screenshots", display_mode: int = DISPLAY_ENERGY_SINGLE):
    """The reference's run_viewer loop (render_gl.py:1001-1075) without a window: per frame,
    advance the solver, read the observables, fill the density of the display mode, draw, and
    (when output_dir is given) save a screenshot.  Returns (state, screenshot paths)."""
    renderer.bind_sim(sim)
    renderer.set_display_mode(display_mode)
    state = {"energy": None, "error": None, "epochs": 0, "baryon": None}
    paths = []
    for _ in range(int(frames)):
        advance_solver(sim, steps_per_frame, state)
        obs = sim.observables()
        state["energy"] = float(obs["energy"])
        if "skyrmion_number" in obs:
            state["baryon"] = float(obs["skyrmion_number"])
        density_for_mode(sim, renderer.display_mode)
        top, bottom = hud_text(sim, state)
        renderer.set_hud_text(top=top, bottom=bottom)
        renderer.render(density_flat=sim.en, field_flat=sim.Field)
        if output_dir is not None:
            paths.append(renderer.save_screenshot(output_dir))
    return state, paths


def inv_view_rows(view_rotation=(0.0, 0.0, 0.0), view_translation=(0.0, 0.0, -4.0)) -> np.ndarray:
    """Rows 0..2 (float32, shape (3, 4)) of R @ T(-t) with R = R_x(-rx) R_y(-ry), the shader's
    inverse view (gl_backend.py:1166-1228): columns 0..2 rotate the eye ray, column 3 is its origin."""
    ax = np.deg2rad(-float(view_rotation[0]))
    ay = np.deg2rad(-float(view_rotation[1]))
    rx = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(ax), -np.sin(ax)], [0.0, np.sin(ax), np.cos(ax)]], np.float32)
    ry = np.array([[np.cos(ay), 0.0, np.sin(ay)], [0.0, 1.0, 0.0], [-np.sin(ay), 0.0, np.cos(ay)]], np.float32)
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = rx @ ry
    t = np.eye(4, dtype=np.float32)
    t[:3, 3] = -np.asarray(view_translation, np.float32)
    return np.ascontiguousarray((m @ t)[:3], np.float32)


class HeadlessRenderer:
    """Off-screen counterpart of the reference ``GLRenderer(width, height, depth)``.

    ``bind_sim(sim)`` sizes the volume from the simulation's lattice and sets the box
    aspect from its extents; ``render(density_flat=sim.en, field_flat=sim.Field)`` draws
    one frame into ``self.image`` (CUDA tensor (height, width, 4), FP32).  The display
    mode picks the colouring: DISPLAY_BARYON uses the pion vector's colour, the other
    modes the transfer table (the reference's color_mode 1 / 0).  ``titles`` lists the
    display modes; the theories' render_headless modules add their third mode.
    """

    titles = DISPLAY_TITLES

    def __init__(self, width: int, height: int, depth: int = 1, title: str = "skyrmion_solver (headless)",
                 device=None) -> None:
        if int(width) < 1 or int(height) < 1:
            raise ValueError("width and height must be >= 1")
        self.width = int(width)
        self.height = int(height)
        self.depth = int(depth)
        self.title = title
        self._device = device
        self.display_mode = DISPLAY_ENERGY_SINGLE
        self.view_rotation = np.array([0.0, 0.0, 0.0], dtype=np.float32)
        self.view_translation = np.array([0.0, 0.0, -4.0], dtype=np.float32)
        self.zoom = 5.5
        self.brightness = 6.0
        self.levelset = 0.2
        self.transfer_scale = 4.0
        self.opacity_scale = 1.0
        self.max_steps = 2500
        self.tstep = 0.002
        self.density_min = 0.0
        self.density_max = 1.0  # the volume's channel 0 is already normalised to [0, 1]
        self.box_scale = np.array([1.0, 1.0, 1.0], dtype=np.float32)
        self._sim = None
        self._dims = None
        self.volume = None
        self.image = None
        self._scratch = None
        self.hud_top_text = ""
        self.hud_bottom_text = ""

    # -- binding and controls -------------------------------------------------
    def bind_params(self, p_i, p_f, device=None) -> None:
        """Attach a lattice by its packed parameters alone (e.g. a resident engine instance,
        whose FP64 field and density come from ``Engine.view``)."""
        class _Lattice:
            pass
        lat = _Lattice()
        lat.p_i_h = np.asarray(p_i, np.int32)
        lat.p_f_h = np.asarray(p_f, np.float64)
        if device is not None:
            self._device = device
        self.bind_sim(lat)

    def bind_sim(self, sim) -> None:
        """Attach a simulation: device buffers for its lattice (on the device of its field) and
        the box aspect of its domain."""
        import torch
        self._sim = sim
        if self._device is not None:
            dev = torch.device("cuda", int(self._device))
        else:
            fld = getattr(sim, "Field", None)
            dev = fld.device if isinstance(fld, torch.Tensor) and fld.is_cuda else \
                torch.device("cuda", torch.cuda.current_device())
        X, Y, Z = (int(v) for v in np.asarray(sim.p_i_h)[:3])
        if self._dims != (X, Y, Z) or self.volume is None or self.volume.device != dev:
            self.volume = torch.empty((Z, Y, X, 4), dtype=torch.float32, device=dev)
            self.image = torch.empty((self.height, self.width, 4), dtype=torch.float32, device=dev)
            self._scratch = torch.empty(int(_lib.load().sky_volume_scratch_size()), dtype=torch.float64, device=dev)
            self._dims = (X, Y, Z)
        self._sync_box_scale()

    def _sync_box_scale(self) -> None:
        """Box aspect from the domain extents p_f[0..2] (render_gl.py:389-414)."""
        if self._sim is None:
            return
        size = np.asarray(self._sim.p_f_h, np.float64)[:3]
        scale = max(float(size.max()), 1.0e-8)
        self.set_render_params(box_scale=(size / scale).astype(np.float32))

    def set_display_mode(self, mode: int) -> None:
        if mode in self.titles:
            self.display_mode = mode

    def set_hud_text(self, *, top: str = "", bottom: str = "") -> None:
        self.hud_top_text = top
        self.hud_bottom_text = bottom

    def set_render_params(self, *, brightness=None, levelset=None, transfer_scale=None, opacity_scale=None,
                          max_steps=None, tstep=None, density_min=None, density_max=None, box_scale=None,
                          **_ignored) -> None:
        """The backend's set_render_params (gl_backend.py:1044-1124) for the keys the shader reads."""
        if brightness is not None:
            self.brightness = float(brightness)
        if levelset is not None:
            self.levelset = float(levelset)
        if transfer_scale is not None:
            self.transfer_scale = float(transfer_scale)
        if opacity_scale is not None:
            self.opacity_scale = float(opacity_scale)
        if max_steps is not None:
            self.max_steps = int(max_steps)
        if tstep is not None:
            self.tstep = float(tstep)
        if density_min is not None:
            self.density_min = float(density_min)
        if density_max is not None:
            self.density_max = float(density_max)
        if box_scale is not None:
            arr = np.asarray(box_scale, dtype=np.float32)
            if arr.shape != (3,):
                raise ValueError("box_scale must have shape (3,).")
            self.box_scale = np.maximum(arr, np.float32(1.0e-8))

    def set_camera_pose(self, *, view_rotation=None, view_translation=None, zoom=None) -> None:
        if view_rotation is not None:
            self.view_rotation = np.asarray(view_rotation, np.float32).copy()
        if view_translation is not None:
            self.view_translation = np.asarray(view_translation, np.float32).copy()
        if zoom is not None:
            self.zoom = float(zoom)

    def make_inv_view_rows(self):
        r = inv_view_rows(self.view_rotation, self.view_translation)
        return r[0].copy(), r[1].copy(), r[2].copy()

    @property
    def color_mode(self) -> int:
        """Pion-vector colouring for the baryon display, the transfer table otherwise (the
        viewers' _sync_render_params)."""
        return 1 if self.display_mode == DISPLAY_BARYON else 0

    def shader_params(self) -> np.ndarray:
        """The 23 floats of sky_render_volume: view rows, box, zoom, brightness, levelset,
        density min / max, transfer scale, opacity scale, tstep."""
        rows = inv_view_rows(self.view_rotation, self.view_translation)
        tail = [self.zoom, self.brightness, self.levelset, self.density_min, self.density_max,
                self.transfer_scale, self.opacity_scale, self.tstep]
        return np.ascontiguousarray(np.concatenate([rows.ravel(), self.box_scale, np.asarray(tail)]), np.float32)

    # -- frame ------------------------------------------------------------------
    def build_volume(self, density_flat, field_flat, stream=None):
        """Fill ``self.volume`` from the density (N FP64 values) and the field; returns it.
        Asynchronous: the density extrema stay on the device until ``extrema`` is read."""
        if self._sim is None:
            raise RuntimeError("bind_sim(sim) first")
        p_i, _ = _lib.host_params(self._sim.p_i_h)
        _lib.call("sky_build_rgba_volume", _lib.i32p(p_i), len(p_i), _lib.dptr(density_flat), _lib.dptr(field_flat),
                  _lib.dptr(self._scratch), self._scratch.numel(), _lib.dptr(self.volume, "float32"), None,
                  _lib.stream_ptr(stream))
        return self.volume

    @property
    def extrema(self):
        """(min, max) of the density of the last volume (the library leaves them in scratch[0:2])."""
        if self._scratch is None:
            return None
        mm = self._scratch[:2].cpu().numpy()
        return float(mm[0]), float(mm[1])

    def draw(self, stream=None):
        """Ray-march ``self.volume`` into ``self.image`` with the current controls; returns it."""
        if self.volume is None:
            raise RuntimeError("bind_sim(sim) first")
        X, Y, Z = self._dims
        prm = self.shader_params()
        _lib.call("sky_render_volume", _lib.dptr(self.volume, "float32"), X, Y, Z, _lib.f32p(prm), len(prm),
                  int(self.max_steps), int(self.color_mode), self.width, self.height,
                  _lib.dptr(self.image, "float32"), _lib.stream_ptr(stream))
        return self.image

    def render(self, *, density_flat, field_flat, stream=None):
        """One frame: the volume from (density_flat, field_flat), then the ray-march."""
        if self._sim is None:
            return None
        self.build_volume(density_flat, field_flat, stream)
        return self.draw(stream)

    def read_pixels(self) -> np.ndarray:
        """(height, width, 3) uint8, top row first: the RGB bytes of the frame."""
        rgb = self.image[..., :3].clamp(0.0, 1.0).mul(255.0).round().to("cpu").numpy()
        return rgb.astype(np.uint8)

    def save_screenshot(self, directory: str = "screenshots") -> str:
        from PIL import Image
        os.makedirs(directory, exist_ok=True)
        stamp = datetime.now().strftime("%Y%m%d_%H%M%S")
        path = os.path.join(directory, f"skyrmion_solver_{stamp}.png")
        Image.fromarray(self.read_pixels()).save(path)
        return path

    def close(self) -> None:
        self.volume = None
        self._sim = None
