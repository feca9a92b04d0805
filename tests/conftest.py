"""pytest configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a B200 and call the CUDA library through its C ABI; everything else runs
on the CPU (oracle against golden vectors, ABI symbol checks, host-side logic, gloo ranks)."""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "polars-metal_b200", ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
