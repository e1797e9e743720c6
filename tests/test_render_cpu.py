"""The renderer's camera helper against the reference Camera conventions
(glm::perspective / glm::lookAt) and the CPU restatement of the particle
view on a hand-checkable scene. Runs on CPU."""
import numpy as np

import render_oracle
import wcsph


def _glm_perspective(fovy, aspect, zn, zf):
    t = np.tan(fovy / 2)
    m = np.zeros((4, 4))
    m[0, 0] = 1 / (aspect * t)
    m[1, 1] = 1 / t
    m[2, 2] = -(zf + zn) / (zf - zn)
    m[3, 2] = -1
    m[2, 3] = -2 * zf * zn / (zf - zn)
    return m


def test_camera_matches_glm_conventions():
    cam = wcsph.camera_look((0.3, -0.2, 2.5), np.radians(260.0), np.radians(10.0), 800, 600)
    P = np.array(cam.projection, np.float64).reshape(4, 4).T
    assert np.allclose(P, _glm_perspective(np.radians(45.0), 800 / 600, 0.1, 100.0), rtol=1e-6, atol=1e-7)
    V = np.array(cam.view, np.float64).reshape(4, 4).T
    # the view maps the eye to the origin and the front vector to -z
    eye = np.array([0.3, -0.2, 2.5])
    assert np.allclose(V @ np.append(eye, 1), [0, 0, 0, 1], atol=1e-6)
    yaw, pitch = np.radians(260.0), np.radians(10.0)
    front = np.array([np.cos(yaw) * np.cos(pitch), np.sin(pitch), np.sin(yaw) * np.cos(pitch)])
    assert np.allclose(V[:3, :3] @ front, [0, 0, -1], atol=1e-6)
    assert np.allclose(V[:3, :3] @ V[:3, :3].T, np.eye(3), atol=1e-6)


def test_oracle_single_sphere_known_answers():
    cam = wcsph.camera_look((0.0, 0.0, 2.5), np.radians(270.0), 0.0, 64, 64)
    pos = np.array([[0.0, 0.0, 0.0, 1.0]], np.float32)
    rgba, depth = render_oracle.render(pos, None, cam, 64, 64, radius=0.2)
    # centred sphere: the centre pixels face the camera (n.z ~ 1), fluid colour (0, 0.5, 1)
    c = rgba[31:33, 31:33, :3].astype(int)
    assert np.all(np.abs(c - [0, 128, 255]) <= 2)
    # disk radius in pixels = R / (d tan(fovy/2)) * H/2 with d the eye distance
    r_px = 0.2 / (2.5 * np.tan(np.radians(22.5))) * 32
    covered = (depth < 1.0).sum()
    assert abs(covered - np.pi * r_px ** 2) < 2 * np.pi * r_px + 4
    # the disk's centre is nearer than its rim, all inside (0, 1)
    assert 0 < depth[32, 32] < depth[32, 32 + int(r_px) - 1] < 1
    assert np.all(rgba[0, 0] == [0, 0, 0, 255])
