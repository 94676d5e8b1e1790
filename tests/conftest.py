import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "ffv-hc_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    """make is idempotent: it rebuilds only what is older than its sources and
    headers, so the tests never run against a stale library.  Where the source
    tree travels without its build tools (a GPU host that runs the prebuilt
    libraries), a library that exists is used as it is."""
    for sub, lib in (("ffv-hc_b200", "libffvhc_b200.so"), ("oracle", "libffvoracle.so")):
        d = os.path.join(ROOT, sub)
        r = subprocess.run(["make", "-s", "-C", d], capture_output=True, text=True)
        if r.returncode != 0 and not os.path.exists(os.path.join(d, lib)):
            raise RuntimeError(f"building {sub} failed:\n{r.stdout}{r.stderr}")


_ensure_built()
