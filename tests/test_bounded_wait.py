"""Failure detection without a GPU fault: the device-side waits of the
library (the sync-free triangular sweep's row flags, the grid barriers of
the cooperative kernels) are bounded.  A wait on a flag that nothing sets
gives up after the poll limit and reports it, and the context stays usable:
the library's kernels run bit-identically afterwards."""
import numpy as np
import pytest

from conftest import MESH_A, seeded_state
import kfun3d_b200 as kf
from oracle import port

pytestmark = pytest.mark.gpu

KFUN3D_ERR_TIMEOUT = 8


def test_a_wait_nothing_ends_gives_up_and_the_context_survives():
    kf.set_abort_on_error(True)
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_aoa(3.0)
    assert kf.lib().kfun3d_check_bounded_wait() == KFUN3D_ERR_TIMEOUT
    m = kf.Mesh(MESH_A)
    q = seeded_state(m.view.q.copy(), 3)
    (_, r1) = m.flux(q)
    (_, r2) = port.flux(m.g, 3.0, q)
    assert np.array_equal(r1, r2)
    assert kf.lib().kfun3d_check_bounded_wait() == KFUN3D_ERR_TIMEOUT
    kf.clear_status()
