import glob
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(path):
    z = np.load(path, allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["kernel"] = str(d["kernel"])
    for k in ("M", "tol", "L"):
        d[k] = int(d[k])
    d["name"] = os.path.basename(path)[:-4]
    return d


@pytest.fixture(params=GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def golden(request):
    return load_golden(request.param)
