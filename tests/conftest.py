import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def lib():
    import bundling_thingy_b200 as bt

    if not os.path.exists(bt.library_path()):
        bt.build()
    return bt.library()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.lib()
    return O


def oracle_config(O, opts, threads=0):
    """Oracle configuration equivalent to library Options."""
    sx, sy = opts.resample_scale()
    return O.Config(
        width=opts.width,
        height=opts.height,
        radius=opts.neighbor_radius or 0,
        accumulate_density=opts.color_by == 0,
        resample_scale=(sx, sy),
        capacity=0xFFFFFFFF,
        sigma=float(np.float32(opts.blur_sigma)),
        shrink=float(np.float32(opts.blur_shrink)) if opts.blur_shrink else 1.0,
        threads=threads,
    )
