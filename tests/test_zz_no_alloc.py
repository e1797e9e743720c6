"""wcsph_sort_keys_static: the stable key sort for callers that cannot
allocate device memory while they run (a render or control loop that must
not take the device-wide synchronisation of cudaFree, or a host working in a
device-memory budget reserved up front). It must give, call after call, the
permutation the step's own sort gives for the same keys (integer work:
bit-exact), while every call reuses the one scratch block inside the library.

This file is collected last on purpose: it runs after every other test (and
passes alone as well). Torch only provides the caller's device buffers.
"""
import numpy as np
import pytest

import wcsph
from parity import dam_break_scene

pytestmark = pytest.mark.gpu


def _device_sort(torch, keys: np.ndarray, calls: int = 2) -> list[np.ndarray]:
    d_keys = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    stream = torch.cuda.current_stream()
    out = []
    for _ in range(calls):
        d_perm = torch.full((len(keys),), -1, dtype=torch.int32, device="cuda")
        wcsph.sort_keys_static(d_keys.data_ptr(), len(keys), d_perm.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        out.append(d_perm.cpu().numpy().view(np.uint32))
    return out


def test_static_sort_matches_the_step_permutation():
    torch = pytest.importorskip("torch")
    p, bx, pos, bpos = dam_break_scene(dims=(24, 24, 24))  # 13,824 particles + walls
    sim = wcsph.CUDASPHSimulator(p, pos, bx, boundary_pos=bpos)
    sim.update(1e-3)
    keys = sim.field("morton_keys")
    want = sim.field("permutation")
    sim.close()
    for got in _device_sort(torch, keys):   # two calls in a row share the scratch
        assert np.array_equal(got, want)


def test_static_sort_at_the_maximum_size_and_the_limit():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    n = wcsph.STATIC_SORT_MAX_KEYS
    # few distinct values in several digits, so that equal keys test stability
    keys = (rng.integers(0, 300, n).astype(np.uint64) << np.uint64(40)) | rng.integers(0, 7, n).astype(np.uint64)
    want = np.argsort(keys, kind="stable").astype(np.uint32)
    for got in _device_sort(torch, keys):
        assert np.array_equal(got, want)
    d = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    with pytest.raises(wcsph.WcsphError) as e:
        wcsph.sort_keys_static(d.data_ptr(), n + 1, d.data_ptr(), None)
    assert e.value.status == wcsph.ERR_INVALID_ARGUMENT and "exceeds the maximum" in e.value.message


def test_static_sort_allocates_no_device_memory():
    """The property the entry point exists for: after a first call (which may
    load the library's device image), repeated sorts at the maximum size leave
    the device's free memory unchanged."""
    torch = pytest.importorskip("torch")
    n = wcsph.STATIC_SORT_MAX_KEYS
    rng = np.random.default_rng(8)
    d_keys = torch.from_numpy(rng.integers(0, 1 << 62, n, dtype=np.int64)).cuda()
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    wcsph.sort_keys_static(d_keys.data_ptr(), n, d_perm.data_ptr(), stream)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(8):
        wcsph.sort_keys_static(d_keys.data_ptr(), n, d_perm.data_ptr(), stream)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    want = np.argsort(d_keys.cpu().numpy().view(np.uint64), kind="stable").astype(np.uint32)
    assert np.array_equal(d_perm.cpu().numpy().view(np.uint32), want)


def test_static_sort_marks_its_output_when_a_wait_runs_out():
    """A look-back wait that runs out (forced by the bounded stall hook; no
    fault, no hang) leaves every perm entry at STATIC_SORT_FAILED, and the next
    call, with the scratch cleared again, sorts correctly."""
    torch = pytest.importorskip("torch")
    n = wcsph.STATIC_SORT_MAX_KEYS
    keys = np.random.default_rng(9).integers(0, 1 << 40, n).astype(np.uint64)
    with wcsph.stall_sort():
        stalled = _device_sort(torch, keys, calls=1)[0]
    assert (stalled == np.uint32(wcsph.STATIC_SORT_FAILED)).all()
    want = np.argsort(keys, kind="stable").astype(np.uint32)
    for got in _device_sort(torch, keys):
        assert np.array_equal(got, want)
