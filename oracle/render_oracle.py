"""CPU restatement of the reference's particle view — TEST INFRASTRUCTURE ONLY.

Follows shaders/instanced_ball.vert:20-32 (camera-facing quad of half-width
RADIUS: to_camera = normalize(eye - p), right = normalize(cross(up0, to_camera)),
up = cross(to_camera, right)) and shaders/instanced_ball.frag (billboard
coordinates c in the unit disk, n = (c, sqrt(1 - |c|^2)), depth of
center_view + n R through the projection mapped to [0, 1], colour base * n.z;
scalar fields shade grey, vector fields scale the base colour by dot(v, n);
optional [min, max] normalisation). GL interpolates the quad's billboard
coordinate perspective-correctly; here it is evaluated exactly by
intersecting each pixel centre's view ray with the quad's plane, in float64.
Nearest depth wins per pixel. Used by the tests to check the CUDA renderer.
"""
from __future__ import annotations

import numpy as np

FLUID = np.array([0.0, 0.5, 1.0])
BOUNDARY = np.array([1.0, 0.5, 0.0])


def _mat(m) -> np.ndarray:
    return np.array(list(m), np.float64).reshape(4, 4).T   # column-major -> matrix


def render(pos, bpos, cam, width, height, radius, show_boundary=False, scalar=None, vec=None,
           normalize=False, vmin=0.0, vmax=1.0, background=(0.0, 0.0, 0.0)):
    """-> (rgba uint8 [H, W, 4], depth float [H, W]); row 0 is the top row."""
    P, V = _mat(cam.projection), _mat(cam.view)
    VP = P @ V
    inv = np.linalg.inv(VP)
    eye = np.array(list(cam.eye), np.float64)
    depth = np.full((height, width), np.inf)
    col = np.zeros((height, width, 3))
    pts = [(np.asarray(p[:3], np.float64), False, i) for i, p in enumerate(pos)]
    if show_boundary and bpos is not None:
        pts += [(np.asarray(p[:3], np.float64), True, i) for i, p in enumerate(bpos)]
    R = float(radius)
    for p, is_b, i in pts:
        tc = eye - p
        tc = tc / np.linalg.norm(tc)
        right = np.cross([0.0, 1.0, 0.0], tc)
        right = right / np.linalg.norm(right)
        up = np.cross(tc, right)
        corners = [p + sx * R * right + sy * R * up for sx in (-1, 1) for sy in (-1, 1)]
        clip = [VP @ np.append(c, 1.0) for c in corners]
        if any(c[3] <= 1e-6 for c in clip):
            continue
        px = [(c[0] / c[3] * 0.5 + 0.5) * width for c in clip]
        py = [(c[1] / c[3] * 0.5 + 0.5) * height for c in clip]
        x0, x1 = max(0, int(np.ceil(min(px) - 0.5))), min(width - 1, int(np.floor(max(px) - 0.5)))
        y0, y1 = max(0, int(np.ceil(min(py) - 0.5))), min(height - 1, int(np.floor(max(py) - 0.5)))
        if x0 > x1 or y0 > y1:
            continue
        xs, ys = np.meshgrid(np.arange(x0, x1 + 1), np.arange(y0, y1 + 1))
        ndc = np.stack([(xs + 0.5) / width * 2 - 1, (ys + 0.5) / height * 2 - 1, np.ones_like(xs, float),
                        np.ones_like(xs, float)], -1)
        far = ndc @ inv.T
        d = far[..., :3] / far[..., 3:4] - eye
        t = ((p - eye) @ tc) / (d @ tc)
        h = eye + d * t[..., None] - p
        cx, cy = (h @ right) / R, (h @ up) / R
        nz2 = 1.0 - (cx * cx + cy * cy)
        ok = nz2 >= 0.0
        nz = np.sqrt(np.where(ok, nz2, 0.0))
        cv = (V @ np.append(p, 1.0))[:3]
        vp = cv + np.stack([cx, cy, nz], -1) * R
        cp = np.concatenate([vp, np.ones(vp.shape[:-1] + (1,))], -1) @ P.T
        dep = cp[..., 2] / cp[..., 3] * 0.5 + 0.5
        ok &= (dep >= 0.0) & (dep <= 1.0)
        base = np.broadcast_to(BOUNDARY if is_b else FLUID, cx.shape + (3,)).copy()
        if not is_b and scalar is not None:
            base = np.broadcast_to(float(scalar[i]), cx.shape + (3,)).copy()
        elif not is_b and vec is not None:
            nv = np.stack([cx, cy, nz], -1)
            base = FLUID * (nv @ np.asarray(vec[i][:3], np.float64))[..., None]
        if not is_b and (scalar is not None or vec is not None) and normalize:
            base = (base - vmin) / (vmax - vmin)
        c = base * nz[..., None]
        rows = height - 1 - ys
        cur = depth[rows, xs]
        win = ok & (dep < cur)
        depth[rows[win], xs[win]] = dep[win]
        col[rows[win], xs[win]] = c[win]
    rgba = np.zeros((height, width, 4), np.uint8)
    q = np.rint(np.clip(col, 0.0, 1.0) * 255.0).astype(np.uint8)
    empty = ~np.isfinite(depth)
    bg = np.rint(np.clip(np.asarray(background, float), 0.0, 1.0) * 255.0).astype(np.uint8)
    rgba[..., :3] = np.where(empty[..., None], bg, q)
    rgba[..., 3] = 255
    depth = np.where(empty, 1.0, depth)
    return rgba, depth
