"""The numpy restatement of the bench scenes (oracle/scenes.py, used by the
reference arm so that it never loads this project's library) reproduces the
library's presets bit for bit: positions, velocities, wall particles and the
tilting-box schedule."""
import numpy as np
import pytest

import refpath
import scenes
import wcsph


@pytest.mark.parametrize("name", ["large_tilting", "dam_break"])
def test_numpy_scene_matches_the_library_preset(name):
    pre = wcsph.preset(name, seed=0)
    sc = scenes.scene(name, seed=0)
    assert sc.pos.tobytes() == pre.pos.tobytes()
    assert sc.vel.tobytes() == pre.vel.tobytes()
    if pre.bpos is None or len(pre.bpos) == 0:
        assert sc.bpos is None
    else:
        assert sc.bpos.tobytes() == pre.bpos.tobytes()
    assert sc.delta == pre.info.delta
    assert bool(sc.moving) == bool(pre.info.moving_box)
    assert sc.box0.tobytes() == refpath.box_floats(pre.box).tobytes()
    for k in (1, 2, 17, 999, 2000, 2500):
        assert sc.box_at(k).tobytes() == refpath.box_floats(pre.box_at(k)).tobytes(), k


def test_splitmix_stream_seeds():
    a = scenes.splitmix_uniform(5, 10)
    b = scenes.splitmix_uniform(5, 20)
    assert np.array_equal(a, b[:10]) and (a >= 0).all() and (a < 1).all()
    assert not np.array_equal(a, scenes.splitmix_uniform(6, 10))
