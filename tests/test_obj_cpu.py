"""Wavefront .obj meshes in front of the boundary sampler (wcsph_load_obj):
the reference loads its obstacle meshes with Geometry::from_file and
Geometry::load_triangles (src/render/geometry.cpp:50-140, 185-207) and
voxelises them in generate_boundary_particles (boundary.cpp:8-35)."""
import numpy as np
import pytest

import wcsph

# a unit tetrahedron written with the four face-vertex forms and a relative
# index, followed by a second shape that the loader must ignore
TETRA = """# tetrahedron
v 0 0 0
v 1 0 0
v 0 1 0
v 0 0 1
o first
f 1 3 2
f 1/1 2/1 4/1
f 1//1 4//1 3//1
f 2/1/1 3/1/1 -1/1/1
o second
v 5 5 5
f 1 2 5
"""


def test_first_shape_triangles_in_file_order(tmp_path):
    p = tmp_path / "tetra.obj"
    p.write_text(TETRA)
    tris = wcsph.load_obj(p)
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    want = v[np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])]
    assert tris.shape == (4, 3, 3)
    assert np.array_equal(tris, want)


def test_normalise_and_model_transform(tmp_path):
    p = tmp_path / "tetra.obj"
    p.write_text(TETRA)
    tris = wcsph.load_obj(p, normalize=True)
    # bounding box [0, 1]^3 -> centred at the origin, largest side 1
    assert np.allclose(tris.reshape(-1, 3).min(0), -0.5) and np.allclose(tris.reshape(-1, 3).max(0), 0.5)
    model = np.eye(4, dtype=np.float32)
    model[3, :3] = (0.5, 0.5, 0.5)          # column-major: translation in the last column
    moved = wcsph.load_obj(p, normalize=True, model=model.reshape(-1))
    assert np.allclose(moved, tris + 0.5)


def test_faces_beyond_triangles_are_rejected_with_the_reference_message(tmp_path):
    p = tmp_path / "quad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    with pytest.raises(wcsph.WcsphError) as e:
        wcsph.load_obj(p)
    assert e.value.status == wcsph.ERR_INVALID_ARGUMENT
    assert e.value.message == f"In {p}: face 0 has 4 vertices (not a triangle)"
    with pytest.raises(wcsph.WcsphError) as e:
        wcsph.load_obj(tmp_path / "missing.obj")
    assert e.value.status == wcsph.ERR_IO


def test_mesh_round_trip_samples_like_the_triangle_soup(tmp_path):
    """A closed box mesh (12 triangles) written as .obj with exact float32
    digits loads back to the same triangles and the same boundary particles."""
    c = np.array([[x, y, z] for x in (0.2, 0.7) for y in (0.1, 0.45) for z in (0.3, 0.65)], np.float32)
    faces = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                      [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]])
    soup = c[faces]
    p = tmp_path / "box.obj"
    p.write_text("\n".join([f"v {x:.9g} {y:.9g} {z:.9g}" for x, y, z in c] +
                           [f"f {a + 1} {b + 1} {d + 1}" for a, b, d in faces]) + "\n")
    tris = wcsph.load_obj(p)
    assert np.array_equal(tris, soup)
    got = wcsph.sample_triangles(tris, 0.02)
    want = wcsph.sample_triangles(soup, 0.02)
    assert got.shape[0] > 0 and np.array_equal(got, want)
