"""Host-side failure handling that needs no GPU.

The reference's only runtime check is the NaN/Inf exit of IsConverged
(src/FFV/FFVILS.h:36-43); everything else (a block table BCMTools built
wrongly, a grid that is not 2:1 balanced) would show as wrong numbers or a
crash.  The library checks the grid description on the host before it
touches a device, so each malformed description below is reported as
FFVGPU_BAD_ARG with a message, here on a machine without a GPU.
"""
import ctypes

import numpy as np
import pytest

import ffvgpu


def explicit_desc(g, kind, ids):
    d = g.desc()
    d._kind_keep = np.ascontiguousarray(kind, np.int32)
    d._ids_keep = np.ascontiguousarray(ids, np.int32)
    d.neighbor_kind = d._kind_keep.ctypes.data
    d.neighbor_ids = d._ids_keep.ctypes.data
    return d


def create(d):
    h = ctypes.c_void_p()
    st = ffvgpu.lib().ffvgpu_pool_create(ctypes.byref(d), ctypes.byref(h))
    if st == ffvgpu.OK:
        ffvgpu.lib().ffvgpu_pool_destroy(h)
    return st, ffvgpu.lib().ffvgpu_last_error().decode()


@pytest.fixture(scope="module")
def grid():
    g = ffvgpu.SphereGrid(2)
    kind, ids = g.neighbors()
    return g, kind, ids


def first_face(kind, k):
    b, f = np.argwhere(kind == k)[0]
    return int(b), int(f)


def test_malformed_neighbour_kind_is_rejected(grid):
    g, kind, ids = grid
    k = kind.copy()
    k[3, 2] = 7
    st, msg = create(explicit_desc(g, k, ids))
    assert st == ffvgpu.BAD_ARG and "kind" in msg


def test_neighbour_id_out_of_range_is_rejected(grid):
    g, kind, ids = grid
    b, f = first_face(kind, ffvgpu.NB_SAME)
    i = ids.copy()
    i[b, f, 0] = g.nb + 5
    st, msg = create(explicit_desc(g, kind, i))
    assert st == ffvgpu.BAD_ARG and "out of range" in msg
    i[b, f, 0] = -1
    st, msg = create(explicit_desc(g, kind, i))
    assert st == ffvgpu.BAD_ARG and "out of range" in msg


def test_neighbour_on_the_wrong_level_is_rejected(grid):
    g, kind, ids = grid
    b, f = first_face(kind, ffvgpu.NB_COARSE)
    wrong = int(np.argwhere(g.level == g.level[b])[0][0])  # a block on b's own level
    i = ids.copy()
    i[b, f, 0] = wrong
    st, msg = create(explicit_desc(g, kind, i))
    assert st == ffvgpu.BAD_ARG and "level mismatch" in msg
    b, f = first_face(kind, ffvgpu.NB_FINE)
    i = ids.copy()
    i[b, f, 2] = b  # b is not one level finer than itself
    st, msg = create(explicit_desc(g, kind, i))
    assert st == ffvgpu.BAD_ARG and "level mismatch" in msg


def test_grid_that_is_not_2to1_balanced_is_rejected():
    # two root-level blocks and a level-2 block next to a level-0 one: the
    # coarse side would need a neighbour two levels finer
    d = ffvgpu.GridDesc()
    level = np.array([0, 2], np.int32)
    index = np.array([[0, 0, 0], [4, 0, 0]], np.int32).reshape(-1)
    d.num_blocks = 2
    d.cells = 16
    d.level = level.ctypes.data
    d.block_index = index.ctypes.data
    d.domain_origin = (0.0, 0.0, 0.0)
    d.root_length = 1.0
    d.root_grid = (2, 1, 1)
    d.bc_type = ffvgpu.P_BC_TYPE
    d.bc_value = ffvgpu.P_BC_VALUE
    kind = np.zeros((2, 6), np.int32)
    ids = np.zeros((2, 6, 4), np.int32)
    st = ffvgpu.lib().ffvgpu_grid_neighbors(ctypes.byref(d), kind.ctypes.data, ids.ctypes.data)
    assert st == ffvgpu.BAD_ARG
    assert "2:1" in ffvgpu.lib().ffvgpu_last_error().decode()
    st, msg = create(d)
    assert st == ffvgpu.BAD_ARG and "2:1" in msg


def test_block_outside_the_root_grid_is_rejected(grid):
    g, kind, ids = grid
    d = g.desc()
    idx = g.index.copy()
    idx[0] = (1 << int(g.level[0])) * np.array(g.params["root_grid"])  # one past the end
    keep = np.ascontiguousarray(idx.reshape(-1), np.int32)
    d.block_index = keep.ctypes.data
    st, msg = create(d)
    assert st == ffvgpu.BAD_ARG and "outside" in msg


def test_wait_limit_range_is_checked():
    L = ffvgpu.lib()
    assert L.ffvgpu_pool_set_wait_limit(None, 1.0) == ffvgpu.BAD_ARG


def test_serve_request_layout_matches_the_header():
    # ffvgpu_request: arrival_s, cancel_s, then the problem
    assert ffvgpu.Request.cancel_s.offset == 8
    assert ffvgpu.Request.problem.offset == 16


def test_closing_a_handle_twice_touches_no_library_call():
    """close() clears the handle in place, so a second close (or the __del__
    that runs at interpreter exit, when module globals may already be gone)
    does not call the library or build a new ctypes object."""
    for cls in (ffvgpu.Pool, ffvgpu.Batch, ffvgpu.Shard):
        obj = cls.__new__(cls)
        obj._h = ctypes.c_void_p()
        h = obj._h
        obj.close()
        obj.close()
        assert obj._h is h and h.value is None
