import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity against the CPU oracle")


def _ensure_built():
    from remobench_b200 import build
    libdir = os.path.join(ROOT, "remobench_b200", "lib")
    need = [os.path.join(libdir, n) for n in ("librb_synth.so", "librb_cuda.so")]
    if not all(os.path.exists(p) for p in need):
        build.build_all()
    from oracle import binding
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        binding.build()


_ensure_built()


@pytest.fixture(scope="session")
def c1_cloud():
    """Configuration 1 (2M points, 8 x 256K batches) and its box, generated once."""
    from remobench_b200 import synth
    cfg = synth.config(1)
    pts = synth.generate(cfg)
    bmin, bmax = synth.scene_box(cfg)
    return cfg, pts, bmin, bmax


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
