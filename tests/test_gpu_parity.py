"""Device parity against the reference built from its own sources (GPU).

Tolerances (FP32 device against the FP64 reference):
  random stream    bit-exact u32; the FP32 value is the reference double truncated
                   to 24 bits (exactly representable, never 1.0)
  camera rays      |d_gpu - d_ref| <= 4e-7 per component
  lobes / noise    relative 2e-4 (absolute 1e-5) on f, pdf, weights, directions
  ray queries      tests/test_gpu_ray_ids.py (ids, t, normals, near-ties)
  images           per-pixel two-sample z-scores; mean relative error <= 1%
"""

import numpy as np
import pytest

import albedo_b200 as ab
from oracle import reference as ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference library not built")]


def test_pixel_stream_is_bit_exact():
    for seed, (x, y), width in [(0, (0, 0), 320), (7, (319, 179), 320), (2**40 + 3, (17, 5), 960)]:
        u32 = np.zeros(200, np.uint32)
        real = np.zeros(200, np.float32)
        from ctypes import POINTER, c_float, c_uint32

        lib = ab._lib.library()
        status = lib.albedo_probe_pixel_stream(seed, x, y, width, 200, u32.ctypes.data_as(POINTER(c_uint32)),
                                               real.ctypes.data_as(POINTER(c_float)))
        assert status == 0
        expected = ref.pixel_stream(seed, x, y, width, 200)
        np.testing.assert_array_equal(u32.astype(np.float64) / 4294967296.0, expected)
        assert np.all(real.astype(np.float64) <= expected)
        assert np.all(expected - real.astype(np.float64) < 2.0 ** -24)
        assert np.all(real < 1.0)


def test_camera_rays_match(room_path):
    scene = ab.Scene.load(room_path)
    rng = np.random.default_rng(0)
    film = rng.uniform(0, 1, size=(4096, 2)).astype(np.float32)
    out = np.zeros((4096, 6), np.float32)
    from ctypes import POINTER, c_float

    lib = ab._lib.library()
    assert lib.albedo_probe_camera_rays(scene.handle, 320, 180, film.ctypes.data_as(POINTER(c_float)), 4096,
                                        out.ctypes.data_as(POINTER(c_float))) == 0
    expected = ref.RefScene(room_path).camera_rays(320, 180, film.astype(np.float64))
    np.testing.assert_allclose(out[:, :3], expected[:, :3], atol=1e-6)
    np.testing.assert_allclose(out[:, 3:], expected[:, 3:], atol=4e-7)


def _probe_eval(kind, params, wo_wi):
    from ctypes import POINTER, c_float

    lib = ab._lib.library()
    p = np.zeros(8, np.float32)
    p[:len(params)] = params
    x = np.ascontiguousarray(wo_wi, np.float32)
    f = np.zeros((len(x), 3), np.float32)
    pdf = np.zeros(len(x), np.float32)
    assert lib.albedo_probe_lobe_eval(kind, p.ctypes.data_as(POINTER(c_float)), x.ctypes.data_as(POINTER(c_float)),
                                      len(x), f.ctypes.data_as(POINTER(c_float)),
                                      pdf.ctypes.data_as(POINTER(c_float))) == 0
    return f, pdf


def _probe_sample(kind, params, inputs):
    from ctypes import POINTER, c_float, c_int32

    lib = ab._lib.library()
    p = np.zeros(8, np.float32)
    p[:len(params)] = params
    x = np.ascontiguousarray(inputs, np.float32)
    n = len(x)
    valid = np.zeros(n, np.int32)
    d = np.zeros((n, 3), np.float32)
    w = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    spec = np.zeros(n, np.int32)
    fp = POINTER(c_float)
    ip = POINTER(c_int32)
    assert lib.albedo_probe_lobe_sample(kind, p.ctypes.data_as(fp), x.ctypes.data_as(fp), n, valid.ctypes.data_as(ip),
                                        d.ctypes.data_as(fp), w.ctypes.data_as(fp), pdf.ctypes.data_as(fp),
                                        spec.ctypes.data_as(ip)) == 0
    return valid, d, w, pdf, spec


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


LOBES = [
    (0, [0.7, 0.5, 0.3]),                                    # Lambert
    (1, [0.156, 0.424, 1.383, 3.602, 2.472, 1.915, 0.0625]),  # rough gold, alpha = 0.25^2
    (1, [0.155, 0.117, 0.138, 4.83, 3.12, 2.15, 0.0]),        # silver mirror
    (2, [1.5, 0.2]),                                          # rough glass, alpha 0.2
    (2, [1.5, 0.0]),                                          # smooth glass
    (2, [1.0 / 1.5, 0.1]),                                    # leaving rough glass
]


@pytest.mark.parametrize("kind, params", LOBES)
def test_lobe_evaluate_and_pdf_match(kind, params):
    rng = np.random.default_rng(kind * 10 + len(params))
    wo = _unit(rng.normal(size=(20000, 3)))
    wo[:, 2] = np.abs(wo[:, 2])
    wi = _unit(rng.normal(size=(20000, 3)))
    x = np.concatenate([wo, wi], axis=1).astype(np.float32)
    f, pdf = _probe_eval(kind, params, x)
    rf, rpdf = ref.lobe_eval(kind, np.array(params, np.float32).astype(np.float64), x.astype(np.float64))
    # Grazing configurations amplify FP32 rounding; compare away from them.
    keep = (np.abs(x[:, 2]) > 0.02) & (np.abs(x[:, 5]) > 0.02)
    np.testing.assert_allclose(f[keep], rf[keep], rtol=2e-3, atol=1e-5)
    np.testing.assert_allclose(pdf[keep], rpdf[keep], rtol=2e-3, atol=1e-5)


@pytest.mark.parametrize("kind, params", LOBES)
def test_lobe_sample_matches(kind, params):
    rng = np.random.default_rng(100 + kind)
    wo = _unit(rng.normal(size=(20000, 3)))
    wo[:, 2] = np.abs(wo[:, 2]) + 0.05
    wo = _unit(wo)
    u = rng.uniform(0, 1, size=(20000, 3))
    x = np.concatenate([wo, u], axis=1).astype(np.float32)
    valid, d, w, pdf, spec = _probe_sample(kind, params, x)
    rvalid, rd, rw, rpdf, rspec = ref.lobe_sample(kind, np.array(params, np.float32).astype(np.float64),
                                                  x.astype(np.float64))
    agree = valid == rvalid
    assert agree.mean() > 0.999
    both = (valid == 1) & (rvalid == 1)
    # A reflect/refract choice can flip when u_choice sits within FP32 rounding of F.
    same_side = np.sign(d[:, 2]) == np.sign(rd[:, 2])
    assert same_side[both].mean() > 0.999
    sel = both & same_side
    np.testing.assert_allclose(d[sel], rd[sel], atol=2e-4)
    np.testing.assert_allclose(w[sel], rw[sel], rtol=2e-3, atol=1e-5)
    np.testing.assert_allclose(pdf[sel], rpdf[sel], rtol=5e-3, atol=1e-5)
    np.testing.assert_array_equal(spec[sel], rspec[sel])


def test_perlin_matches():
    from ctypes import POINTER, c_float

    rng = np.random.default_rng(9)
    pts = rng.uniform(-50, 50, size=(20000, 3)).astype(np.float32)
    noise = np.zeros(len(pts), np.float32)
    turb = np.zeros(len(pts), np.float32)
    lib = ab._lib.library()
    assert lib.albedo_probe_perlin(pts.ctypes.data_as(POINTER(c_float)), len(pts),
                                   noise.ctypes.data_as(POINTER(c_float)),
                                   turb.ctypes.data_as(POINTER(c_float))) == 0
    rn, rt = ref.perlin(pts.astype(np.float64))
    np.testing.assert_allclose(noise, rn, atol=2e-5)
    np.testing.assert_allclose(turb, rt, atol=5e-5)


def ulp_distance(ours_f32: np.ndarray, reference_f64: np.ndarray) -> np.ndarray:
    """Distance in FP32 ulps between a device float and the reference double rounded to FP32."""
    a = ours_f32.astype(np.float32).view(np.int32).astype(np.int64)
    b = reference_f64.astype(np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def random_rays(count, seed, low, high):
    rng = np.random.default_rng(seed)
    origin = rng.uniform(low, high, size=(count, 3))
    direction = _unit(rng.normal(size=(count, 3)))
    return np.concatenate([origin, direction], axis=1).astype(np.float32)


@pytest.mark.parametrize("which", ["room", "trefoil"])
def test_reference_box_counts_match_the_restatement(which, room_path, trefoil_path):
    """The counting traversal's estimate of the boxes the reference's binary
    traversal tests (one per node popped), and its primitive counts, against the
    FP64 restatement of that traversal on the same rays. The device tests each
    collapsed node's boxes when it reaches the node, the reference when it pops
    them (possibly after the range shrank), and FP32 boxes are rounded outward:
    both can only add work, so the device may count a few percent more."""
    from oracle import restatement

    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    rays = random_rays(50_000, 9, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    device = ab.trace_work_counts(scene, rays)
    theirs = restatement.intersect(scene, rays.astype(np.float64))["counts"].sum(axis=0)
    assert device["rays"] == len(rays)
    ratio = device["reference_boxes"] / theirs[0]
    assert 0.99 < ratio < 1.10, (ratio, device, theirs)
    for k, i in (("triangles", 1), ("spheres", 2), ("instances", 3)):
        if theirs[i] == 0:
            assert device[k] == 0, (k, device, theirs)
        else:
            assert 0.99 < device[k] / theirs[i] < 1.05, (k, device, theirs)


def test_occlusion_queries_match(room_path):
    scene = ab.Scene.load(room_path)
    rays = random_rays(50_000, 6, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    t_max = np.random.default_rng(7).uniform(0.1, 6.0, size=len(rays)).astype(np.float32)
    ours = scene.occluded(rays, t_max)
    theirs = ref.RefScene(room_path).occluded(rays.astype(np.float64), t_max.astype(np.float64))
    assert (ours != theirs).sum() <= 10


def _pixel_grid(width, height, count, seed):
    rng = np.random.default_rng(seed)
    xs = rng.integers(0, width, count)
    ys = rng.integers(0, height, count)
    return np.stack([xs, ys], axis=1).astype(np.int32)


@pytest.mark.parametrize("which, width, height, n, depth", [("room", 320, 180, 4, 8), ("trefoil", 960, 540, 4, 10)])
def test_images_match_reference_at_equal_spp(which, width, height, n, depth, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    pixels = _pixel_grid(width, height, 1500, 11)
    job = ab.RenderJob(width, height, samples_per_axis=n, max_depth=depth)
    acc, squares = ab.render_pixels(scene, job, pixels, with_squares=True)
    assert np.all(acc["count"] == n * n)
    rsum, rsq = ref.RefScene(path).render_pixels(width, height, n, pixels, max_depth=depth)
    samples = n * n
    ours = np.stack([acc["r"], acc["g"], acc["b"]], axis=1) / samples
    theirs = rsum / samples
    var_o = np.maximum(squares / samples - ours**2, 0)
    var_t = np.maximum(rsq / samples - theirs**2, 0)
    z = (ours - theirs) / np.sqrt((var_o + var_t) / samples + 1e-12)
    # Same random streams: paths mostly coincide, so |z| is far below 1 almost everywhere.
    assert np.mean(np.abs(z) > 4) < 0.005, np.mean(np.abs(z) > 4)
    rel = np.abs(ours.mean() - theirs.mean()) / theirs.mean()
    assert rel < 0.01, rel


def trace_modes(scene, rays, any_hit, persistent, t_max=float("inf")):
    from ctypes import POINTER, c_float, c_int32, c_uint32

    n = len(rays)
    rays = np.ascontiguousarray(rays, dtype=np.float32)
    out = {"hit": np.zeros(n, np.int32), "t": np.zeros(n, np.uint32), "object": np.zeros(n, np.uint32),
           "triangle": np.zeros(n, np.uint32)}
    lib = ab._lib.library()
    status = lib.albedo_probe_trace_modes(
        scene.handle, rays.ctypes.data_as(POINTER(c_float)), n, 0.0, t_max, int(any_hit), int(persistent),
        out["hit"].ctypes.data_as(POINTER(c_int32)), out["t"].ctypes.data_as(POINTER(c_uint32)),
        out["object"].ctypes.data_as(POINTER(c_uint32)), out["triangle"].ctypes.data_as(POINTER(c_uint32)))
    assert status == 0, ab._lib.library().albedo_last_error()
    return out


@pytest.mark.parametrize("which", ["room", "trefoil"])
@pytest.mark.parametrize("any_hit", [False, True])
@pytest.mark.parametrize("mode", [1, 2, 3])
def test_persistent_traversal_equals_the_per_thread_traversal(which, any_hit, mode, room_path, trefoil_path):
    """The wavefront's persistent kernels (warp fetch; a turn descends nodes then
    handles a leaf, mode 1, takes one step, mode 2, or traces the whole query out
    of line, mode 3; 4-byte stack entries that keep no entry distance) reach the
    leaves in the same order as the per-thread
    traversal the ray-query tests compare with the reference, and give the same
    hits: hit flags, FP32 t, object and triangle are identical bit for bit, for
    closest-hit and any-hit queries."""
    scene = ab.Scene.load(room_path if which == "room" else trefoil_path)
    rays = random_rays(100_000, 12, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    t_max = 3.0 if any_hit else float("inf")
    per_thread = trace_modes(scene, rays, any_hit, 0, t_max)
    persistent = trace_modes(scene, rays, any_hit, mode, t_max)
    assert 0.05 < per_thread["hit"].mean() < 1.0
    for key in ("hit", "t", "object", "triangle"):
        np.testing.assert_array_equal(persistent[key], per_thread[key], err_msg=key)


TEXTURES = """\
camera from 0 2.2 6.5  at 0 0.7 0  up 0 1 0  fov 45
material marble perlin low 0.2 0.15 0.1  high 0.9 0.85 0.8  scale 3  veins 5
material smoke perlin low 0.05 0.05 0.08  high 0.6 0.6 0.7  scale 8
material tiles checker even 0.8 0.8 0.8  odd 0.1 0.1 0.1  frequency 2
material gold conductor eta 0.156 0.424 1.383  k 3.602 2.472 1.915  roughness 0.25
material frosted dielectric ior 1.5 roughness 0.3
material veined mix first gold second marble scale 2 veins 6 threshold 0.45
material cloudy mix first frosted second smoke scale 4 threshold 0.6
sphere 0 -1000 0 radius 1000 material tiles
sphere -1.6 0.7 0 radius 0.7 material marble
sphere 0 0.7 -0.4 radius 0.7 material veined
sphere 1.6 0.7 0 radius 0.7 material cloudy
sphere 0.8 0.3 1.2 radius 0.3 material smoke
area_light 0 4 1 radius 0.8 radiance 6 6 5
point_light -2 3 3 intensity 2 2 2
sky nadir 0.1 0.12 0.15 zenith 0.3 0.35 0.45
"""


def test_textured_and_mixed_materials_match_reference_images(tmp_path):
    """Perlin textures (with and without veins), checker, and mix materials of a
    conductor or a rough dielectric with a Perlin-textured diffuse: the same
    per-pixel two-sample test against the reference at equal spp as the other
    image tests."""
    path = tmp_path / "textures.scene"
    path.write_text(TEXTURES)
    scene = ab.Scene.load(path)
    width, height, n, depth = 320, 180, 4, 8
    pixels = _pixel_grid(width, height, 1500, 21)
    acc, squares = ab.render_pixels(scene, ab.RenderJob(width, height, samples_per_axis=n, max_depth=depth), pixels,
                                    with_squares=True)
    rsum, rsq = ref.RefScene(path).render_pixels(width, height, n, pixels, max_depth=depth)
    samples = n * n
    ours = np.stack([acc["r"], acc["g"], acc["b"]], axis=1) / samples
    theirs = rsum / samples
    var_o = np.maximum(squares / samples - ours**2, 0)
    var_t = np.maximum(rsq / samples - theirs**2, 0)
    z = (ours - theirs) / np.sqrt((var_o + var_t) / samples + 1e-12)
    assert np.mean(np.abs(z) > 4) < 0.005, np.mean(np.abs(z) > 4)
    assert abs(ours.mean() - theirs.mean()) / theirs.mean() < 0.01


def test_textured_and_mixed_materials_same_in_both_forms(tmp_path):
    """The wavefront's per-class shade kernels (the mix class included) against
    the megakernel on the textured scene: identical sample counts, image sums
    within 1e-4, at most 0.5% of pixels beyond 1e-3 relative (the wavefront
    tests' tolerance)."""
    import torch

    path = tmp_path / "textures.scene"
    path.write_text(TEXTURES)
    scene = ab.Scene.load(path)
    images = []
    for method in (ab.MEGAKERNEL, ab.WAVEFRONT):
        job = ab.RenderJob(160, 90, samples_per_axis=4, seed=3, max_depth=8, method=method)
        acc = torch.zeros((160 * 90, 4), dtype=torch.float64, device="cuda")
        ab.render_device(scene, job, acc.data_ptr())
        torch.cuda.synchronize()
        scene.check()
        images.append(acc.cpu().numpy())
    mega, wave = images
    np.testing.assert_array_equal(np.ascontiguousarray(wave[:, 3]).view(np.int64),
                                  np.ascontiguousarray(mega[:, 3]).view(np.int64))
    assert abs(wave[:, :3].sum() - mega[:, :3].sum()) / mega[:, :3].sum() < 1e-4
    rel = np.abs(wave[:, :3] - mega[:, :3]) / np.maximum(np.abs(mega[:, :3]), 1e-3)
    assert np.mean(rel.max(axis=1) > 1e-3) < 0.005
