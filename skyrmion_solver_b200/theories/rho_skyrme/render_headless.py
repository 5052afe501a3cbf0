"""Headless viewer of the rho-Skyrme model (th/rho_skyrme/render_gl.py without a window).

``run_viewer`` runs the viewer's loop for a number of frames and saves each frame
as a PNG; ``Renderer`` is the headless renderer with this theory's display modes.
"""
from __future__ import annotations

from ...visualization.headless import (DISPLAY_BARYON, DISPLAY_ENERGY_SINGLE, HeadlessRenderer,  # noqa: F401
                                       advance_solver, viewer_loop)

DISPLAY_RHO_MESON = 3

DISPLAY_TITLES = {
    DISPLAY_ENERGY_SINGLE: "Rho-Skyrme: Energy density",
    DISPLAY_BARYON: "Rho-Skyrme: Baryon density",
    DISPLAY_RHO_MESON: "Rho-Skyrme: Rho-meson density",
}


class Renderer(HeadlessRenderer):
    titles = DISPLAY_TITLES


def _compute_density_for_mode(sim, mode: int) -> None:
    """The density the display mode shows, in ``sim.en`` (render_gl.py _compute_density_for_mode)."""
    if mode == DISPLAY_RHO_MESON and hasattr(sim, "compute_rho_meson_density"):
        sim.compute_rho_meson_density()
        return
    if hasattr(sim, "compute_baryon_density"):
        sim.compute_baryon_density()


def run_viewer(sim, params=None, *, steps_per_frame: int = 5, frames: int = 1, output_dir: str | None = "screenshots",
               display_mode: int = DISPLAY_ENERGY_SINGLE, width: int = 1200, height: int = 900):
    """The viewer loop of run_viewer for ``frames`` frames; returns (state, screenshot paths)."""
    renderer = Renderer(width, height, int(sim.p_i_h[2]), title=DISPLAY_TITLES[DISPLAY_ENERGY_SINGLE])
    try:
        return viewer_loop(sim, renderer, _compute_density_for_mode, steps_per_frame=steps_per_frame,
                           frames=frames, output_dir=output_dir, display_mode=display_mode)
    finally:
        renderer.close()
