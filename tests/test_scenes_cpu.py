"""Scene generation on the host: level-set files against the reference's own
DistrGen output, the seabed noise, and the oracle's wave paddle."""
import os

import numpy as np

from conftest import GOLDEN

LS = os.path.join(GOLDEN, "levelsets")


def test_levelset_files_give_the_reference_labels():
    """tests/golden/levelsets/ holds files written by the reference's
    DistrGen functions (make_levelset_golden.py): two level sets and the label
    file generate_combined_labels_simple made of them.  The reader plus the
    rule (SOLID where solid < 0, else FLUID where fluid < 0, else AIR) give
    that label file."""
    from fluidprjct_b200 import capi
    solid = capi.read_levelset_file(os.path.join(LS, "solid_init.txt"))
    fluid = capi.read_levelset_file(os.path.join(LS, "fluid_init_ball.txt"))
    assert solid.shape == fluid.shape == (32, 40)
    dims = np.zeros(3, np.int32)
    path = os.path.join(LS, "labels_simple.txt").encode()
    assert capi.lib().fp_read_label_file(path, 2, capi.ptr(dims), None) == 0
    lab = np.zeros(int(dims[0]) * int(dims[1]), np.uint8)
    capi.lib().fp_read_label_file(path, 2, capi.ptr(dims), capi.ptr(lab))
    lab = lab.reshape(int(dims[1]), int(dims[0]))
    rule = np.where(solid < 0, 0, np.where(fluid < 0, 1, 2)).astype(np.uint8)
    assert np.array_equal(rule, lab)
    assert set(np.unique(lab)) == {0, 1, 2}
    # the floor is at the bottom (j = 0), the ball above the water
    assert (lab[0] == 0).all() and (lab[-1] != 0).any()


def test_levelset_reader_rejects_bad_files(tmp_path):
    from fluidprjct_b200 import capi
    p = tmp_path / "bad.txt"
    p.write_text("S 3 2\n1 2 3\n4 5\n")
    dims = np.zeros(2, np.int32)
    assert capi.lib().fp_read_levelset_file(str(p).encode(), capi.ptr(dims), None) == capi.FP_ERR_IO


def test_value_noise_and_seabed():
    from fluidprjct_b200 import scenes
    n1 = scenes.value_noise_2d((48, 64), 4, 4)
    assert np.array_equal(n1, scenes.value_noise_2d((48, 64), 4, 4))
    assert not np.array_equal(n1, scenes.value_noise_2d((48, 64), 4, 5))
    assert 0.0 <= n1.min() and n1.max() <= 1.0 and n1.std() > 0.05
    lab = scenes.seabed(64, 32, 48, 1 / 32, level=0.45, water_xmin=0.2)
    D, H, W = lab.shape
    x = (np.arange(W) + 0.5) / 32
    assert not (lab[:, :, x < 0.2] == scenes.FLUID).any()
    # bed between 0.15 and 0.20 of height: rows below 0.15 are SOLID, above 0.2 not (inside the walls)
    y = (np.arange(H) + 0.5) / 32
    inner = lab[1:-1, :, 1:-1]
    assert (inner[:, y < 0.15, :] == scenes.SOLID).all()
    assert not (inner[:, (y > 0.2) & (y < H / 32 - 1 / 32), :] == scenes.SOLID).any()


def test_oracle_paddle_marks_and_moves(O):
    """The oracle's paddle: BODY where the cell centre has x < x_p(t), never
    over SOLID; x_p(t) = x0 + A sin(2 pi t / T) after each body phase."""
    from fluidprjct_b200 import scenes
    n, dx, dt = 24, 1 / 24, 0.01
    lab = scenes.box_3d(n, n, n, dx, 0.6, 0.5, 1.0, xmin=0.1)
    o = O.Sim3(n, n, n, dx, dt)
    o.set_labels(lab)
    o.set_paddle(0.15, 0.05, 0.5)
    o.phase(O.PH_LABEL)
    got = o.labels()
    x = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * np.float32(dx)
    behind = (x - np.float32(0.15)) <= 0
    assert ((got == 3) == (behind[None, None, :] & (lab != 0))).all()
    o.phase(O.PH_PRESSURE)
    o.phase(O.PH_BODY)
    st = o.body_state()
    t = float(np.float32(dt))
    w = 2 * np.pi / float(np.float32(0.5))
    assert np.isclose(st["pos"][0], float(np.float32(0.15)) + float(np.float32(0.05)) * np.sin(w * t), rtol=0, atol=1e-15)
    assert np.isclose(st["vel"][0], float(np.float32(0.05)) * w * np.cos(w * t), rtol=0, atol=1e-15)
    assert st["vel"][1] == st["vel"][2] == 0.0
