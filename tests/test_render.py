"""Headless viewer: the RGBA volume builder and the ray-march.

* The volume oracle against the reference's own kernels (tests/golden/volume.npz,
  made by make_golden_volume.py under Numba's CUDA simulator), and the device
  builder against both.
* The ray-march oracle against cases derived by hand from the shader, and the
  device ray-march against the oracle on the same volume.  The shader runs only
  through OpenGL, so the image itself is not pinned to the reference.

Image tolerance: the device and the oracle both compute in FP32 but round
differently (the device contracts multiply-adds), and the shader has hard
thresholds (box-edge test, alpha > 0.95, t > tfar), so a pixel whose ray
passes a threshold within rounding may take the other branch.  At most 1% of
the pixels may differ by more than 1e-3 in any channel, and the median pixel
difference must stay below 1e-5.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import render_oracle as R
from skyrmion_solver_b200 import _lib
from skyrmion_solver_b200.visualization import HeadlessRenderer, inv_view_rows

HERE = os.path.dirname(os.path.abspath(__file__))
VOLUME = os.path.join(HERE, "golden", "volume.npz")


def _gold():
    if not os.path.exists(VOLUME):
        pytest.skip("volume.npz not generated")
    return dict(np.load(VOLUME))


def _uniform(value, n=(1.0, 0.0, 0.0), dims=(6, 5, 4)):
    X, Y, Z = dims
    vol = np.empty((Z, Y, X, 4), np.float32)
    vol[..., 0] = value
    vol[..., 1:] = np.asarray(n, np.float32)
    return vol


# ---------------------------------------------------------------------------
# CPU: the oracle and the host logic
# ---------------------------------------------------------------------------
def test_volume_oracle_matches_the_reference_kernels():
    d = _gold()
    X, Y, Z = (int(v) for v in d["p_i"][:3])
    vol, vmin, vmax = R.rgba_volume(d["density"], np.load(os.path.join(HERE, "golden", "nuclear.npz"))["field0"],
                                    (X, Y, Z))
    assert vmin == d["dmin"] and vmax == d["dmax"]
    assert vol.dtype == np.float32 and vol.shape == d["volume"].shape == (Z, Y, X, 4)
    assert np.array_equal(vol, d["volume"])


def test_view_rows_match_the_oracle():
    for rot, tr in [((0, 0, 0), (0, 0, -4)), ((30, -45, 10), (0.3, -0.2, -3.5)), ((-90, 180, 0), (1, 2, 3))]:
        assert np.array_equal(inv_view_rows(rot, tr), R.inv_view_rows(rot, tr))
    rows = inv_view_rows()
    assert np.array_equal(rows[:, 3], [0.0, 0.0, 4.0])   # default eye at z = 4 looking down -z


def test_shader_params_layout_and_defaults():
    r = HeadlessRenderer(40, 30, 8)

    class _Sim:
        p_i_h = np.array([8, 6, 4], np.int32)
        p_f_h = np.array([2.0, 1.0, 0.5], np.float64)
    r._sim = _Sim()
    r._sync_box_scale()
    prm = r.shader_params()
    assert prm.dtype == np.float32 and prm.shape == (23,)
    assert np.array_equal(prm[:12], inv_view_rows().ravel())
    assert np.array_equal(prm[12:15], np.array([1.0, 0.5, 0.25], np.float32))
    assert np.allclose(prm[15:], [5.5, 6.0, 0.2, 0.0, 1.0, 4.0, 1.0, 0.002])
    assert r.color_mode == 0 and r.max_steps == 2500
    r.set_display_mode(2)
    assert r.color_mode == 1
    r.set_display_mode(99)                               # unknown modes are ignored
    assert r.color_mode == 1


def test_oracle_hand_cases():
    W, H = 33, 25                      # odd sizes: the centre pixel's ray is the view axis
    c = (H // 2, W // 2)
    rows = inv_view_rows()
    # norm 0.5 lands on transfer texel 4 exactly: opaque green, alpha 1 on the first sample
    img = R.render(_uniform(0.5), rows, width=W, height=H, color_mode=0)
    assert np.array_equal(img[c], [0.0, 1.0, 0.0, 1.0])
    # pion vector (1, 0, 0) has hue 0: red; input (0.45 - 0.2) * 4 = 1
    img = R.render(_uniform(0.45), rows, width=W, height=H, color_mode=1)
    assert np.allclose(img[c], [1.0, 0.0, 0.0, 1.0], atol=1e-6)
    # a camera well to the side misses the box: every pixel keeps the white clear colour
    img = R.render(_uniform(0.5), inv_view_rows((0, 0, 0), (5, 0, -4)), width=W, height=H)
    assert np.array_equal(img, np.ones_like(img))
    # constant per-sample opacity a and white colour (n = (0, 0, 1)): after n samples
    # alpha = 1 - (1 - a)^n and rgb = a * alpha; the axis ray crosses the box (t = 3..5) in ~1001 samples
    a = 1e-4
    img = R.render(_uniform(0.5, (0.0, 0.0, 1.0)), rows, width=W, height=H, color_mode=1, brightness=1.0,
                   levelset=0.0, transfer_scale=2 * a)
    alpha = img[c][3]
    n = np.log(1.0 - alpha) / np.log(1.0 - a)
    assert abs(n - 1001) < 1.5
    assert np.allclose(img[c][:3], a * alpha, rtol=1e-3)


def test_volume_and_render_reject_bad_arguments():
    lib = _lib.load()
    pi = np.array([8, 8, 8, 2, 3, 4, 512, 2048, 1, 1, 1], dtype=np.int32)
    dummy = ctypes.c_void_p(256)
    mm = np.zeros(2)
    n = lib.sky_volume_scratch_size()
    assert n > 0
    assert lib.sky_build_rgba_volume(_lib.i32p(pi), 11, None, dummy, dummy, n, dummy, _lib.f64p(mm), None) == 1
    assert lib.sky_build_rgba_volume(_lib.i32p(pi), 11, dummy, dummy, dummy, n, ctypes.c_void_p(260),
                                     _lib.f64p(mm), None) == 1            # volume not 16-byte aligned
    assert lib.sky_build_rgba_volume(_lib.i32p(pi), 11, dummy, dummy, dummy, n - 1, dummy, _lib.f64p(mm), None) == 5
    prm = np.zeros(23, np.float32)
    prm[12:15] = 1.0
    prm[22] = 0.002
    args = (dummy, 8, 8, 8, _lib.f32p(prm), 23)
    assert lib.sky_render_volume(*args, 100, 0, 0, 10, dummy, None) == 1    # empty image
    assert lib.sky_render_volume(*args, -1, 0, 10, 10, dummy, None) == 1    # negative step count
    assert lib.sky_render_volume(*args, 100, 0, 10, 10, None, None) == 1    # null image
    assert lib.sky_render_volume(dummy, 8, 8, 8, _lib.f32p(prm), 22, 100, 0, 10, 10, dummy, None) == 1
    bad = prm.copy()
    bad[22] = 0.0
    assert lib.sky_render_volume(dummy, 8, 8, 8, _lib.f32p(bad), 23, 100, 0, 10, 10, dummy, None) == 1
    bad = prm.copy()
    bad[13] = 0.0
    assert lib.sky_render_volume(dummy, 8, 8, 8, _lib.f32p(bad), 23, 100, 0, 10, 10, dummy, None) == 1


# ---------------------------------------------------------------------------
# GPU: the device path through the C ABI
# ---------------------------------------------------------------------------
def _image_close(got, want):
    diff = np.abs(got - want).max(axis=-1)
    return float((diff > 1e-3).mean()) <= 0.01 and float(np.median(diff)) <= 1e-5


def _draw(vol, rows, box=(1.0, 1.0, 1.0), zoom=5.5, brightness=6.0, levelset=0.2, dmin=0.0, dmax=1.0,
          transfer_scale=4.0, opacity_scale=1.0, tstep=0.002, max_steps=2500, color_mode=0, width=64, height=48):
    import torch
    Z, Y, X = vol.shape[:3]
    v = torch.from_numpy(np.ascontiguousarray(vol)).cuda()
    img = torch.empty((height, width, 4), dtype=torch.float32, device="cuda")
    prm = np.concatenate([np.asarray(rows, np.float32).ravel(), np.asarray(box, np.float32),
                          np.asarray([zoom, brightness, levelset, dmin, dmax, transfer_scale, opacity_scale, tstep],
                                     np.float32)]).astype(np.float32)
    _lib.call("sky_render_volume", _lib.dptr(v, "float32"), X, Y, Z, _lib.f32p(prm), len(prm), max_steps,
              color_mode, width, height, _lib.dptr(img, "float32"), _lib.stream_ptr())
    torch.cuda.synchronize()
    return img.cpu().numpy()


@pytest.mark.gpu
def test_device_volume_matches_the_reference_kernels():
    import torch
    from tests._gpu import dev
    d = _gold()
    X, Y, Z = (int(v) for v in d["p_i"][:3])
    field = np.load(os.path.join(HERE, "golden", "nuclear.npz"))["field0"]
    vol = torch.empty((Z, Y, X, 4), dtype=torch.float32, device="cuda")
    scratch = torch.empty(int(_lib.load().sky_volume_scratch_size()), dtype=torch.float64, device="cuda")
    mm = np.zeros(2)
    p_i = np.ascontiguousarray(d["p_i"], np.int32)
    dens_d, field_d = dev(d["density"]), dev(field)       # held: the call reads them on the device
    _lib.call("sky_build_rgba_volume", _lib.i32p(p_i), len(p_i), _lib.dptr(dens_d), _lib.dptr(field_d),
              _lib.dptr(scratch), scratch.numel(), _lib.dptr(vol, "float32"), _lib.f64p(mm), _lib.stream_ptr())
    assert mm[0] == d["dmin"] and mm[1] == d["dmax"]
    assert np.array_equal(vol.cpu().numpy(), d["volume"])


@pytest.mark.gpu
def test_device_volume_at_a_larger_lattice_matches_the_oracle():
    """Ragged tile edges (X, Z not multiples of 32) and more than one extrema block."""
    import torch
    from tests._gpu import dev
    X, Y, Z = 45, 38, 70
    rng = np.random.default_rng(5)
    dens = rng.standard_normal(X * Y * Z) * 3.0
    field = rng.standard_normal((4, X * Y * Z))
    field[1:, :50] = 0.0                                  # pion vector below the threshold: (0, 0, 1)
    pi = np.array([X, Y, Z, 2, 3, 4, X * Y * Z, 4 * X * Y * Z, 1, 1, 1], np.int32)
    vol = torch.empty((Z, Y, X, 4), dtype=torch.float32, device="cuda")
    scratch = torch.empty(int(_lib.load().sky_volume_scratch_size()), dtype=torch.float64, device="cuda")
    mm = np.zeros(2)
    dens_d, field_d = dev(dens), dev(field)
    _lib.call("sky_build_rgba_volume", _lib.i32p(pi), len(pi), _lib.dptr(dens_d), _lib.dptr(field_d),
              _lib.dptr(scratch), scratch.numel(), _lib.dptr(vol, "float32"), _lib.f64p(mm), _lib.stream_ptr())
    want, vmin, vmax = R.rgba_volume(dens, field, (X, Y, Z))
    assert mm[0] == vmin and mm[1] == vmax
    assert np.array_equal(vol.cpu().numpy(), want)
    # without a host pointer the call is asynchronous and leaves the extrema in scratch[0:2]
    vol.zero_()
    scratch.zero_()
    _lib.call("sky_build_rgba_volume", _lib.i32p(pi), len(pi), _lib.dptr(dens_d), _lib.dptr(field_d),
              _lib.dptr(scratch), scratch.numel(), _lib.dptr(vol, "float32"), None, _lib.stream_ptr())
    torch.cuda.synchronize()
    assert scratch[0].item() == vmin and scratch[1].item() == vmax
    assert np.array_equal(vol.cpu().numpy(), want)


@pytest.mark.gpu
def test_device_render_hand_cases():
    W, H = 33, 25
    c = (H // 2, W // 2)
    rows = inv_view_rows()
    assert np.array_equal(_draw(_uniform(0.5), rows, width=W, height=H)[c], [0.0, 1.0, 0.0, 1.0])
    img = _draw(_uniform(0.5), inv_view_rows((0, 0, 0), (5, 0, -4)), width=W, height=H)
    assert np.array_equal(img, np.ones_like(img))
    a = 1e-4
    img = _draw(_uniform(0.5, (0.0, 0.0, 1.0)), rows, width=W, height=H, color_mode=1, brightness=1.0,
                levelset=0.0, transfer_scale=2 * a)
    n = np.log(1.0 - img[c][3]) / np.log(1.0 - a)
    assert abs(n - 1001) < 1.5
    assert np.allclose(img[c][:3], a * img[c][3], rtol=1e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("color_mode", [0, 1])
@pytest.mark.parametrize("pose", [((0, 0, 0), (0, 0, -4), 5.5), ((25, -40, 0), (0.2, -0.1, -3.6), 4.0)])
def test_device_render_matches_the_oracle(color_mode, pose):
    from skyrmion_solver_b200 import initial as ini
    rot, tr, zoom = pose
    # a B = 2 rational map on an anisotropic box, with a smooth density concentrated on it
    dims = (40, 34, 28)
    h = (0.12, 0.14, 0.16)
    F = ini.normalise(ini.rational_map(dims, h, 2, ini.exp_profile(1.2), (0.0, 0.0, 0.0)))
    r2 = sum(((np.arange(n) - (n - 1) / 2.0) * s)[tuple(slice(None) if k == j else None for k in range(3))] ** 2
             for j, (n, s) in enumerate(zip(dims, h)))
    dens = np.exp(-r2 / 0.6) * (1.0 - F[0])
    vol, _, _ = R.rgba_volume(dens.ravel(), F.reshape(4, -1), dims)
    size = np.array([(n - 1) * s for n, s in zip(dims, h)])
    box = (size / size.max()).astype(np.float32)
    rows = inv_view_rows(rot, tr)
    kw = dict(box=box, zoom=zoom, color_mode=color_mode, width=64, height=48)
    got = _draw(vol, rows, **kw)
    want = R.render(vol, rows, **kw)
    assert (want != 1.0).any() and (want == 1.0).all(axis=-1).mean() < 0.9   # the soliton is in view
    assert _image_close(got, want)


@pytest.mark.gpu
def test_headless_renderer_frame_and_screenshot(tmp_path):
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation
    th = T.load_theory("Nuclear Skyrme model")
    params = th.params.default_params(xlen=32, ylen=32, zlen=32, lsx=0.2, lsy=0.2, lsz=0.2, time_step=0.04)
    sim = Simulation(params, th)
    sim.initialize({"mode": "rational_map", "baryon_number": 2})
    sim.compute_baryon_density()
    r = HeadlessRenderer(48, 36, 32)
    r.bind_sim(sim)
    img = r.render(density_flat=sim.en, field_flat=sim.Field)
    torch.cuda.synchronize()
    vol, vmin, vmax = R.rgba_volume(sim.en.cpu().numpy(), sim.Field.cpu().numpy(), (32, 32, 32))
    assert r.extrema == (vmin, vmax)
    assert np.array_equal(r.volume.cpu().numpy(), vol)
    want = R.render(vol, inv_view_rows(), box=r.box_scale, width=48, height=36)
    assert _image_close(img.cpu().numpy(), want)
    r.set_display_mode(2)
    img2 = r.draw().cpu().numpy()
    assert _image_close(img2, R.render(vol, inv_view_rows(), box=r.box_scale, color_mode=1, width=48, height=36))
    path = r.save_screenshot(str(tmp_path))
    from PIL import Image
    px = np.asarray(Image.open(path))
    assert px.shape == (36, 48, 3) and px.dtype == np.uint8
    assert np.array_equal(px, r.read_pixels())


# ---------------------------------------------------------------------------
# the viewer loop (render_gl.py advance_solver / run_viewer without a window)
# ---------------------------------------------------------------------------
class _FakeSim:
    """Records the calls the viewer loop makes; energy falls by 1 per step."""

    def __init__(self, newtonflow=True):
        self.rp = type("RP", (), {"newtonflow": newtonflow})()
        self.p_f_h = np.array([1.0, 1.0, 1.0, 0.1, 0.1, 0.1, 1e-3, 0.25])
        self.calls = []

    def observables(self):
        self.calls.append("observables")
        return {"energy": 10.0}

    def step(self, e):
        self.calls.append("step")
        return e - 1.0, 0.5


def test_advance_solver_follows_the_reference():
    from skyrmion_solver_b200.visualization import advance_solver, hud_text
    sim = _FakeSim()
    state = {"energy": None, "error": None, "epochs": 0, "baryon": None}
    advance_solver(sim, 3, state)
    assert sim.calls == ["observables", "step", "step", "step"]
    assert state == {"energy": 7.0, "error": 0.5, "epochs": 3, "baryon": None}
    advance_solver(sim, 2, state)
    assert state["epochs"] == 5 and state["energy"] == 5.0 and sim.calls.count("observables") == 1
    state["baryon"] = 1.0
    assert hud_text(sim, state) == ("t=1.250 (5 epochs), err=5.000e-01", "E=5.000000, B=1.000000, running")
    off = _FakeSim(newtonflow=False)                      # without Newton flow the viewer does not step
    st = {"energy": None, "error": None, "epochs": 0}
    advance_solver(off, 4, st)
    assert off.calls == ["observables"] and st["epochs"] == 0


def test_viewer_loop_host_logic():
    """Frame order of the loop with a recording renderer: advance, observables, density, HUD,
    draw, screenshot."""
    from skyrmion_solver_b200.visualization import viewer_loop
    from skyrmion_solver_b200.visualization.headless import HeadlessRenderer

    class _Rec(HeadlessRenderer):
        def bind_sim(self, sim):
            self._sim = sim
            sim.calls.append("bind")

        def render(self, *, density_flat, field_flat, stream=None):
            self._sim.calls.append(("render", self.hud_top_text, self.hud_bottom_text))

        def save_screenshot(self, directory="screenshots"):
            self._sim.calls.append("shot")
            return directory + "/frame.png"

    sim = _FakeSim()
    sim.en, sim.Field = "en", "field"
    state, paths = viewer_loop(sim, _Rec(8, 6), lambda s, m: s.calls.append(("density", m)), steps_per_frame=1,
                               frames=2, output_dir="out", display_mode=2)
    assert paths == ["out/frame.png"] * 2 and state["epochs"] == 2
    assert sim.calls == ["bind", "observables", "step", "observables", ("density", 2),
                         ("render", "t=0.250 (1 epochs), err=5.000e-01", "E=10.000000, running"), "shot",
                         "step", "observables", ("density", 2),
                         ("render", "t=0.500 (2 epochs), err=5.000e-01", "E=10.000000, running"), "shot"]


def test_theory_display_modes():
    from skyrmion_solver_b200 import theories as T
    for short, third in [("nuclear", None), ("berger", None), ("lightly_bound", None),
                         ("omega", "DISPLAY_OMEGA"), ("coulomb", "DISPLAY_COULOMB"), ("rho", "DISPLAY_RHO_MESON")]:
        m = T.by_short_name(short).render_headless
        r = m.Renderer(16, 12)
        assert r.color_mode == 0                          # energy display: transfer table
        r.set_display_mode(2)
        assert r.color_mode == 1                          # baryon display: pion colouring
        if third:
            r.set_display_mode(getattr(m, third))
            assert r.display_mode == 3 and r.color_mode == 0
        else:
            r.set_display_mode(3)
            assert r.display_mode == 2                    # not a mode of this theory


@pytest.mark.gpu
@pytest.mark.parametrize("short,mode", [("nuclear", 2), ("omega", 3), ("rho", 3)])
def test_headless_run_viewer(tmp_path, short, mode):
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation
    th = T.by_short_name(short)
    params = th.params.default_params(xlen=24, ylen=24, zlen=24, lsx=0.25, lsy=0.25, lsz=0.25)
    sim = Simulation(params, th)
    sim.initialize({"mode": "rational_map", "baryon_number": 2})
    e0 = float(sim.observables()["energy"])
    state, paths = th.render_headless.run_viewer(sim, params, steps_per_frame=2, frames=3, output_dir=str(tmp_path),
                                                 display_mode=mode, width=40, height=30)
    torch.cuda.synchronize()
    assert state["epochs"] == 6 and len(paths) == 3 and all(os.path.exists(p) for p in paths)
    assert state["energy"] < e0
    # the last frame shows the display mode's density, as left in sim.en
    want = {2: "compute_baryon_density", 3: ("compute_potential_density" if short == "omega"
                                             else "compute_rho_meson_density")}[mode]
    en = sim.en.clone()
    sim.en.zero_()                                        # the rho-meson kernel accumulates, as the reference's does
    getattr(sim, want)()
    torch.cuda.synchronize()
    assert torch.equal(en, sim.en)


@pytest.mark.gpu
def test_renderer_draws_a_resident_engine_instance():
    """Engine.view's FP64 buffers of a defect-corrected FP32 instance, drawn by a renderer bound
    to the instance's parameters: the volume equals the oracle's volume of those buffers."""
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200.theories._init_common import build_reference_field
    th = T.by_short_name("nuclear")
    p = th.params.default_params(xlen=36, ylen=30, zlen=33, lsx=0.2, lsy=0.2, lsz=0.2)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
    F = torch.empty(int(p_i[7]), dtype=torch.float64, device="cuda")
    build_reference_field("nuclear", p_i, p_f, {"mode": "rational_map", "baryon_number": 3}, F)
    with Engine(0) as eng:
        i = eng.add("nuclear", (p_i, p_f), F.cpu().numpy().reshape((4,) + tuple(int(v) for v in p_i[:3])),
                    None, precision="fp32d")
        eng.step(4)
        field, en = eng.view(i, "baryon")
        r = HeadlessRenderer(40, 30)
        r.bind_params(p_i, p_f)
        img = r.render(density_flat=en, field_flat=field)
        torch.cuda.synchronize()
        want, vmin, vmax = R.rgba_volume(en.cpu().numpy(), field.cpu().numpy(), tuple(int(v) for v in p_i[:3]))
        assert r.extrema == (vmin, vmax)
        assert np.array_equal(r.volume.cpu().numpy(), want)
        assert _image_close(img.cpu().numpy(), R.render(want, inv_view_rows(), box=r.box_scale, width=40, height=30))
