"""Source checks of the device library that need no GPU.

A pool enqueues its work on a non-blocking stream, which does not wait for
the legacy default stream.  A plain cudaMemcpy from pageable host memory can
return before its data has reached the device, and cudaMemset on the legacy
stream is not ordered with the pool's stream either, so a kernel enqueued on
the pool's stream could read old contents.  Every copy and memset in the
library therefore goes through the pool's stream (cudaMemcpyAsync /
cudaMemsetAsync); this test keeps it that way.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ffv-hc_b200", "csrc")


def _sources():
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cpp", ".cu", ".h", ".cuh")):
            path = os.path.join(CSRC, name)
            with open(path) as f:
                yield name, f.read()


def test_no_copy_or_memset_on_the_legacy_stream():
    bad = []
    for name, text in _sources():
        for n, line in enumerate(text.splitlines(), 1):
            code = line.split("//")[0]
            if re.search(r"\bcudaMemcpy\s*\(|\bcudaMemset\s*\(", code):
                bad.append(f"{name}:{n}: {line.strip()}")
    assert not bad, "synchronous copies not ordered on the pool's stream:\n" + "\n".join(bad)
