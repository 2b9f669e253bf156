"""The bounded device waits give up and report, without hanging the GPU.

The tensor-core transform kernel waits on mbarriers for its TMA copies and
its MMAs; every wait gives up after a fixed number of tries, sets the device
error flag, releases what it holds and returns, and the host turns the flag
into QS_ERR_TIMEOUT.  qs_selftest_wait_limit runs that wait routine on a
barrier that nothing completes (a flag nobody sets) for a few tries.
The call must report QS_ERR_TIMEOUT, clear the flag, and leave the handle
usable: a march on the same handle afterwards agrees with one on a fresh
handle (to FP32 rounding: the deposits add by atomics).
"""
import numpy as np
import pytest

from tertia_b200 import abi
from tertia_b200 import workload as wl
from gpu_helpers import cfg_for

pytestmark = pytest.mark.gpu


def test_wait_limit_runs_out_and_reports():
    from tertia_b200.mesh import Mesh
    cfg = cfg_for("fp32", n=32, layers=8)
    beam = wl.sample_beam(cfg, wl.BeamSpec(2000, nb_over_n0=0.1, seed=4))
    front = wl.front_plasma(cfg, seed=2)
    L = abi.load_library()
    with Mesh(cfg) as m, Mesh(cfg) as ref:
        for tries in (1, 64):
            assert L.qs_selftest_wait_limit(m._h, tries) == abi.QS_ERR_TIMEOUT
            assert "bounded device wait" in L.qs_last_error(m._h).decode()
        assert L.qs_selftest_wait_limit(m._h, 0) == abi.QS_ERR_INVALID
        for h in (m, ref):
            h.load_beam(beam)
            h.load_front_plasma(front)
            h.step()
        # FP32 deposits add by atomics, so two marches agree to rounding only
        scale = np.abs(ref.onaxis_ex()).max()
        assert scale > 0
        np.testing.assert_allclose(m.onaxis_ex(), ref.onaxis_ex(), rtol=0, atol=1e-6 * scale)
