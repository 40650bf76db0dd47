import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
MESH_A = os.path.join(GOLDEN, "uns3dA.msh")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def mesh_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("meshes")


@pytest.fixture(scope="session")
def box_mesh(mesh_dir):
    """Factory: path of the seeded Kuhn-box mesh with n^3 nodes."""
    import kfun3d_b200 as kf
    cache = {}

    def make(n, seed=3, bump=0.1, jitter=0.2, permute=True):
        key = (n, seed, bump, jitter, permute)
        if key not in cache:
            p = os.path.join(str(mesh_dir), f"box{n}_s{seed}_b{bump}_j{jitter}_p{int(permute)}.msh")
            kf.generate_mesh(p, n, bump_height=bump, jitter=jitter, seed=seed, permute=permute)
            cache[key] = p
        return cache[key]
    return make


def seeded_state(q0, seed, amp=0.05):
    """Free stream plus a seeded U(-amp, amp) perturbation per component."""
    rng = np.random.default_rng(seed)
    return q0 + rng.uniform(-amp, amp, q0.shape)
