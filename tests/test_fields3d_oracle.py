"""Known answers of the oracle's macro-field sampler (render3d.ts:33-65, 159-230) on analytic fields.

The reference has no tests of these shaders; the checks here follow from the formulas: trilinear
interpolation reproduces a linear field exactly at the sample points used, the curl of a
solid-body rotation has magnitude 2|omega|, the slice quad's pixel centres are the cell centres when
the pixel counts equal the grid, and a tracer in a uniform flow moves by u * steps.
"""
import numpy as np

from oracle.oracle import advect, sample_slice


def field(W, H, D, fn):
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    ux, uy, uz = fn(x.astype(np.float64), y.astype(np.float64), z.astype(np.float64))
    mac = np.zeros((D, H, W, 4), dtype=np.float32)
    mac[..., 0], mac[..., 1], mac[..., 2], mac[..., 3] = ux, uy, uz, 1.0
    return mac.reshape(-1)


def test_uniform_flow_speed_slice_and_solid_marks():
    W, H, D = 12, 10, 8
    mac = field(W, H, D, lambda x, y, z: (0.08 + 0 * x, 0.06 + 0 * y, 0 * z))
    mac4 = mac.reshape(D, H, W, 4)
    mac4[4, 5, 6, 3] = 0.0  # one solid node
    out = sample_slice(mac, W, H, D, 2, 4 / 7, 0, 0.1, W, H)  # z = 4 exactly, pixel centres = cells
    speed = np.float32(np.sqrt(np.float32(0.08) ** 2 + np.float32(0.06) ** 2)) / np.float32(0.16)
    assert np.isnan(out[5, 6])
    rest = np.delete(out.reshape(-1), 5 * W + 6)
    np.testing.assert_allclose(rest, speed, rtol=1e-6)


def test_rotation_vorticity_is_twice_omega():
    W, H, D = 16, 16, 16
    om = 0.004
    cx = cy = 7.5
    mac = field(W, H, D, lambda x, y, z: (-om * (y - cy), om * (x - cx), 0 * z))
    out = sample_slice(mac, W, H, D, 2, 0.5, 1, 0.1, W, H)
    inner = out[2:-2, 2:-2]  # away from the clamped edges
    np.testing.assert_allclose(inner, 2 * om / (0.3 * 0.1), rtol=1e-4)


def test_slice_axes_sample_linear_field_exactly_at_cell_centres():
    W, H, D = 9, 7, 5
    mac = field(W, H, D, lambda x, y, z: (0.01 * x, 0 * y, 0 * z))
    for axis, (nu, nv) in ((0, (H, D)), (1, (W, D)), (2, (W, H))):
        out = sample_slice(mac, W, H, D, axis, 1.0, 0, 0.1, nu, nv)
        if axis == 0:
            np.testing.assert_allclose(out, 0.01 * (W - 1) / 0.16, rtol=1e-6)
        else:
            np.testing.assert_allclose(out, np.broadcast_to(0.01 * np.arange(W) / 0.16, (nv, W)), rtol=1e-5,
                                       atol=1e-7)


def test_tracers_uniform_flow_substeps_and_reseed():
    W, H, D = 20, 8, 8
    u = 0.1
    mac = field(W, H, D, lambda x, y, z: (u + 0 * x, 0 * y, 0 * z))
    seeds = np.array([[1, 3, 3, 0], [2, 4, 4, 0]], dtype=np.float32)
    parts = np.zeros((2, 8), dtype=np.float32)
    parts[0, :3] = (3.0, 3.0, 3.0)
    parts[1, :3] = (18.0, 4.0, 4.0)  # leaves the box within the frame: restarts at its seed
    out = advect(mac, W, H, D, seeds, parts, 30.0, u)  # travel 3 cells: 3 sub-steps
    np.testing.assert_allclose(out[0, :3], (6.0, 3.0, 3.0), rtol=1e-6)
    np.testing.assert_allclose(out[0, 4:7], (u, 0, 0), rtol=1e-6)
    np.testing.assert_array_equal(out[1, :3], seeds[1, :3])


def test_ppm_image_of_a_slice(tmp_path):
    from cells_b200.images import SOLID_GREY, colourise, write_ppm

    vals = np.array([[0.0, 0.5, np.nan], [1.0, 2.0, -1.0]], dtype=np.float32)
    rgb = colourise(vals)
    assert rgb.shape == (2, 3, 3) and rgb.dtype == np.uint8
    assert (rgb[0, 2] == SOLID_GREY).all()
    assert (rgb[1, 1] == rgb[1, 0]).all() and (rgb[1, 2] == rgb[0, 0]).all()  # clamped to [0, 1]
    p = tmp_path / "slice.ppm"
    write_ppm(str(p), vals)
    data = p.read_bytes()
    assert data.startswith(b"P6\n3 2\n255\n") and len(data) == len(b"P6\n3 2\n255\n") + 18
