"""The out-of-core planner (maxi_out_of_core_plan) on the CPU: slab depth,
repetitions per round (exchange rounds when R x radius halos leave no room)
and the resident bit-packed mask, for given device budgets.  No GPU needed:
the planner is host arithmetic."""
import ctypes

import pytest

from maxibone_b200 import _lib

GB = 10 ** 9


def plan(shape, kernel_size, reps, field="bf16", device_bytes=180 * GB, slab=0, flags=0):
    s, k, res = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    rc = _lib.lib().maxi_out_of_core_plan(*shape, slab, kernel_size, reps, _lib.FIELD_TYPES[field], flags,
                                          device_bytes, ctypes.byref(s), ctypes.byref(k), ctypes.byref(res))
    return rc, s.value, k.value, bool(res.value)


def test_full_size_out_of_core_volume_fits_deep_halos():
    # 3456 x 3456 x 4096 (z, y, x), sigma 8 (65 taps), R = 20, BF16: one round,
    # the mask resident bit-packed (6.1 GB), slabs of several hundred planes.
    rc, S, k, res = plan((3456, 3456, 4096), 65, 20)
    assert rc == 0 and k == 20 and res
    assert 512 <= S <= 3456


def test_large_r_times_radius_switches_to_exchange_rounds(monkeypatch):
    # R x radius = 6400 planes exceeds the volume: deep halos would make every
    # slab the whole volume, which does not fit; rounds of k < R do, on a host
    # that can pin the two FP32 copies of the field (8 bytes per voxel).
    monkeypatch.setenv("MAXIBONE_OOC_HOST_BUDGET", str(400 * GB))
    rc, S, k, res = plan((3456, 3456, 4096), 65, 200, field="f32")
    assert rc == 0 and 1 <= k < 200 and S >= 1


def test_exchange_rounds_need_the_host_memory(monkeypatch):
    # Without room for the host copies of the field the planner keeps deep
    # halos (when those fit) or reports the host limit instead of planning
    # rounds whose pinned allocations would fail.
    monkeypatch.setenv("MAXIBONE_OOC_HOST_BUDGET", str(100 * GB))
    rc, S, k, res = plan((3456, 3456, 4096), 65, 20)
    assert rc == 0 and k == 20
    rc, S, k, res = plan((3456, 3456, 4096), 65, 200, field="f32")
    assert rc == 3
    assert b"pinned host memory" in _lib.lib().maxi_last_error()
    monkeypatch.setenv("MAXIBONE_OOC_HOST_BUDGET", str(8 * 96 * 64 * 64))
    rc, S, k, _ = plan((96, 64, 64), 9, 12, field="f32", device_bytes=4 * 10 ** 6)
    assert rc == 0 and k < 12


def test_caller_slab_depth_is_an_upper_bound():
    rc, S, k, _ = plan((3456, 3456, 4096), 65, 20, slab=256)
    assert rc == 0 and S <= 256 and k >= 1


def test_whole_volume_in_one_slab_when_it_fits():
    rc, S, k, _ = plan((256, 256, 256), 65, 100, field="f32")
    assert rc == 0 and S == 256 and k == 100


def test_plane_not_whole_words_keeps_per_slab_masks():
    rc, S, k, res = plan((100, 33, 37), 9, 5, device_bytes=GB)
    assert rc == 0 and not res


def test_fp64_form_never_uses_exchange_rounds():
    rc, S, k, _ = plan((2048, 2048, 2048), 65, 100, field="f64", device_bytes=180 * GB)
    assert k == 100 or rc == 3


def test_no_slab_fits_is_an_out_of_memory_error():
    rc, S, k, _ = plan((64, 4096, 4096), 65, 10, field="f32", device_bytes=10 ** 6)
    assert rc == 3
    assert b"too large" in _lib.lib().maxi_last_error() or b"fits" in _lib.lib().maxi_last_error()


@pytest.mark.parametrize("budget", [4 * 10 ** 6, 6 * 10 ** 6, 40 * 10 ** 6])
def test_small_budgets_shrink_slabs_or_rounds(budget):
    rc, S, k, _ = plan((96, 64, 64), 9, 12, field="f32", device_bytes=budget)
    assert rc == 0 and 1 <= S <= 96 and 1 <= k <= 12
