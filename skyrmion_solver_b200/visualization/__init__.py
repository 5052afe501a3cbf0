"""Headless counterpart of the reference viewer: volume builder and ray-march on the device."""
from .headless import (DISPLAY_BARYON, DISPLAY_ENERGY_SINGLE, DISPLAY_TITLES, HeadlessRenderer,  # noqa: F401
                       advance_solver, hud_text, inv_view_rows, viewer_loop)
