"""ffvgpu_dot_noalloc: the dot product that allocates nothing on the device.

It exists for callers that cannot call cudaMalloc (an application that gives
all device memory to its own allocator, or a loop that must not stall on the
synchronisation cudaMalloc/cudaFree bring): the caller passes device vectors
and a device result, and the partial sums live in a fixed array compiled
into the library.  Checked through the C ABI against the pool-based
ffvgpu_dot and against the CPU oracle's dot in the same fixed sum order, on
the same vectors (bit equality), on two calls in a row, since every call
reuses the same array.  This file is collected last so that a run stopping
at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import ffvgpu
import ffv_oracle as fo

pytestmark = pytest.mark.gpu


def colour_split_order():
    """perm[s] = natural index k*256 + j*16 + i of storage slot s of a block."""
    perm = np.empty(4096, np.int64)
    for k in range(16):
        for j in range(16):
            for i in range(16):
                c = (i + j + k) & 1
                s = c * 2048 + (k * 16 + j) * 8 + (i >> 1)
                perm[s] = k * 256 + j * 16 + i
    return perm


def test_dot_noalloc_matches_pool_dot_on_consecutive_calls():
    import torch
    torch.cuda.init()
    g = ffvgpu.SphereGrid(2)
    P = ffvgpu.Pool(g.desc())
    O = fo.Oracle.from_grid(g, vc=2, reduction=fo.RED_CANONICAL)
    rng = np.random.default_rng(2024)
    w = 20
    perm = colour_split_order()
    stream = torch.cuda.current_stream().cuda_stream
    L = ffvgpu.lib()
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):
        x = rng.standard_normal((g.nb, w, w, w))
        b = rng.standard_normal((g.nb, w, w, w)) * (call + 1)
        P.upload("X", x, 2)
        P.upload("B", b, 2)
        expected = P.dot("X", "B")
        O.field("X")[...] = x
        O.field("B")[...] = b
        assert O.dot("X", "B") == expected, call
        xi = x[:, 2:18, 2:18, 2:18].reshape(g.nb, 4096)[:, perm]
        bi = b[:, 2:18, 2:18, 2:18].reshape(g.nb, 4096)[:, perm]
        xd = torch.from_numpy(np.ascontiguousarray(xi)).cuda()
        bd = torch.from_numpy(np.ascontiguousarray(bi)).cuda()
        st = L.ffvgpu_dot_noalloc(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(bd.data_ptr()),
                                  g.nb, ctypes.c_void_p(result.data_ptr()),
                                  ctypes.c_void_p(stream))
        assert st == ffvgpu.OK, L.ffvgpu_last_error()
        torch.cuda.synchronize()
        got = float(result.item())
        assert got == expected, (call, got, expected)
    P.close()
    O.close()


def test_dot_noalloc_rejects_sizes_beyond_its_array():
    L = ffvgpu.lib()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = L.ffvgpu_dot_noalloc(dummy, dummy, 65537, dummy, None)
    assert st == ffvgpu.BAD_ARG
    assert b"num_blocks" in L.ffvgpu_last_error()
