"""CPU checks of the torch sequence renderer (benchmark input generation): its undeformed
frame is the numpy analytic rendering bit for bit, and its deformation moves speckles where
the scene's material-to-world map says (run on the CPU device)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from aldic_b200 import synth, synth_gpu  # noqa: E402


@pytest.fixture(scope="module")
def scene():
    return synth_gpu.stereo_sequence(frames=3, M=320, N=240, f=300.0, noise=0.0, device="cpu",
                                     plane_half=(900.0, 700.0))


def test_frame0_is_the_numpy_rendering(scene):
    rng = np.random.default_rng(4)
    mm = 1000.0 / 300.0
    sp = synth.make_speckles(rng, int(round(0.0153 * 1800 * 1400 / mm ** 2)), -900, 900, -700, 700, 2 * mm, 4 * mm,
                             60, 200)
    sp.a = sp.a * 200.0
    Xw = np.stack([sp.cx, sp.cy, np.full_like(sp.cx, 1000.0)], -1)
    for cam, imgs in ((scene.camL, scene.L), (scene.camR, scene.R)):
        u, v = cam.project(Xw)

        def to_mat(X, Y, cam=cam):
            W = synth._ray_plane(cam, X, Y, 1000.0)
            return W[:, 0], W[:, 1]

        ref = np.clip(np.rint(synth.render(320, 240, sp, (u + 1, v + 1), to_mat, 12)), 0, 65535)
        got = imgs[0].to(torch.int32).numpy().reshape(240, 320).T
        assert np.array_equal(got, ref)


def test_last_frame_follows_the_deformation(scene):
    # material points on the x axis of the plane: the last frame stretches them by `stretch`
    k = scene.params["frames"] - 1
    X = np.array([-300.0, 0.0, 300.0])
    Y = np.zeros(3)
    w0 = scene.material_to_world(X, Y, 0)
    wk = scene.material_to_world(X, Y, k)
    assert np.allclose(w0[:, 2], 1000.0)
    assert np.allclose(wk[:, 0], X * (1 + scene.params["stretch"]))
    u0, _ = scene.camL.project(w0)
    uk, _ = scene.camL.project(wk)
    # points move apart along x as the plane stretches
    assert (uk[2] - uk[0]) > (u0[2] - u0[0]) * 1.05
    # and the rendered frames differ from frame 0
    assert not torch.equal(scene.L[k], scene.L[0])
