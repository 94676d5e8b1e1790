"""Uploads from pinned host memory, on the GPU.

A pinned host buffer is read by the pack kernel directly across the link (the
interior row by row and, for vector fields, the first guide layer); a
pageable buffer goes through a staging copy in device memory.  Both give the
same device fields, checked through downloads of the same pool state.
"""
import numpy as np
import pytest
import torch

import ffvgpu
from helpers import VC, assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [0, 2])
def test_pinned_upload_matches_staged_upload(level):
    g = ffvgpu.SphereGrid(level)
    P = ffvgpu.Pool(g.desc())   # pageable uploads (staging copy)
    Q = ffvgpu.Pool(g.desc())   # pinned uploads (read across the link)
    n = P.nb * (16 + 2 * VC) ** 3
    rng = np.random.default_rng(7 + level)
    for name in ("AP", "AW", "B", "X", "UX"):
        a = rng.standard_normal(n)
        P.upload(name, a, VC)
        t = torch.from_numpy(a.copy()).pin_memory()
        Q.upload_ptr(name, t.data_ptr(), VC)
        torch.cuda.synchronize()
        assert_bitwise(Q.download(name, VC), P.download(name, VC), name)
    # the solve sees the same system either way
    for name in ("AE", "AS", "AN", "AB", "AT"):
        a = np.full(n, 1.0 / 6.0)
        P.upload(name, a, VC)
        t = torch.from_numpy(a.copy()).pin_memory()
        Q.upload_ptr(name, t.data_ptr(), VC)
    ap = np.full(n, -1.0)
    P.upload("AP", ap, VC)
    t = torch.from_numpy(ap.copy()).pin_memory()
    Q.upload_ptr("AP", t.data_ptr(), VC)
    rp = P.solve_rbgs(1.2, 5, 0.0)
    rq = Q.solve_rbgs(1.2, 5, 0.0)
    assert_bitwise(rq["history"], rp["history"], "residual history")
    assert_bitwise(Q.download("X", VC), P.download("X", VC), "x")
    P.close()
    Q.close()


def test_pinned_upload_from_a_pointer_inside_a_buffer():
    """A pinned pointer 8 bytes into a buffer (off every 16-byte boundary) is
    read directly as well: the same field as the staged upload."""
    g = ffvgpu.SphereGrid(0)
    P = ffvgpu.Pool(g.desc())
    Q = ffvgpu.Pool(g.desc())
    n = P.nb * (16 + 2 * VC) ** 3
    a = np.random.default_rng(3).standard_normal(n)
    P.upload("B", a, VC)
    t = torch.zeros(n + 1, dtype=torch.float64).pin_memory()
    t[1:] = torch.from_numpy(a)
    Q.upload_ptr("B", t.data_ptr() + 8, VC)
    assert_bitwise(Q.download("B", VC), P.download("B", VC), "b")
    P.close()
    Q.close()


def test_pinned_instance_upload_matches_staged_upload():
    """The batch pool's per-instance upload takes the same two paths."""
    B = ffvgpu.Batch(600, 4)
    i = B.admit_sphere(ffvgpu.sphere_problem(1, seed=4))
    j = B.admit_sphere(ffvgpu.sphere_problem(1, seed=4))
    n = B.blocks(i) * (16 + 2 * VC) ** 3
    rng = np.random.default_rng(11)
    for name in ("B", "X"):
        a = rng.standard_normal(n)
        B.upload(i, name, a, VC)
        t = torch.from_numpy(a.copy()).pin_memory()
        B.upload_ptr(j, name, t.data_ptr(), VC)
        torch.cuda.synchronize()
        assert_bitwise(B.download(j, name, VC), B.download(i, name, VC), name)
    B.close()
