"""The sort's compressed keys (radix_sort.cuh): with every cell coordinate
in [-2^B, 2^B), the Morton code of c + 2^B orders particles exactly as the
reference's 63-bit Morton code of c + 2^20, so the stable sort permutation
is the same. Checked on random cell sets (many duplicate cells, both signs,
several B) in Python integers. Runs on CPU."""
import numpy as np
import pytest


def interleave(v, bits):
    """x | y << 1 | z << 2 bit interleave of non-negative coordinates."""
    key = np.zeros(len(v), dtype=object)
    for b in range(bits):
        for a in range(3):
            key = key | (((v[:, a] >> b) & 1).astype(object) << (3 * b + a))
    return key


def full_key(c):
    return interleave((c + (1 << 20)) & ((1 << 21) - 1), 21)


def compressed_key(c):
    """Smallest B with all coordinates (and 0) in [-2^B, 2^B); keys of 3(B+1) bits."""
    lo, hi = min(0, int(c.min())), max(0, int(c.max()))
    B = 0
    while B < 20 and not (lo >= -(1 << B) and hi < (1 << B)):
        B += 1
    return interleave(c + (1 << B), B + 1), B


@pytest.mark.parametrize("B", [0, 1, 3, 6, 7, 10, 19])
@pytest.mark.parametrize("span", ["both", "positive", "negative"])
def test_compressed_keys_give_the_same_stable_order(B, span):
    rng = np.random.default_rng(B * 7 + len(span))
    lo, hi = {"both": (-(1 << B), (1 << B) - 1), "positive": (0, (1 << B) - 1),
              "negative": (-(1 << B), -1 if B else 0)}[span]
    c = rng.integers(lo, hi + 1, size=(3000, 3), dtype=np.int64)
    c[rng.integers(0, 3000, 300)] = c[rng.integers(0, 3000, 300)]   # duplicate cells
    f = full_key(c)
    k, b = compressed_key(c)
    assert b <= B
    assert np.array_equal(np.argsort(f, kind="stable"), np.argsort(k, kind="stable"))
    i, j = rng.integers(0, 3000, 2000), rng.integers(0, 3000, 2000)
    assert np.array_equal(f[i] < f[j], k[i] < k[j]) and np.array_equal(f[i] == f[j], k[i] == k[j])


def test_tilting_box_scene_sorts_in_three_digit_passes():
    # cells of the 2 x 1 x 1 box centred on the origin at h = 0.016: x in [-63, 62], y, z in [-32, 31]
    c = np.array([[-63, -32, -32], [62, 31, 31], [0, 0, 0]])
    _, B = compressed_key(c)
    assert (3 * (B + 1) + 7) // 8 == 3
