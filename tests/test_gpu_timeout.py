"""The failure path of the tensor-core network kernels' bounded wait, tested
without a GPU fault: an mbarrier that nothing arrives at makes the wait (at
most about one second, on the device's global timer) run out; the entry point
returns CL_ERR_TIMEOUT with the time waited, and the context stays usable, as
a guided render right afterwards shows."""
import numpy as np
import pytest

import colvillea_b200 as cb
from colvillea_b200 import _native as N
from colvillea_b200 import scenes

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(native):
    status, waited = cb.tc_wait_timeout()
    assert status == N.CL_ERR_TIMEOUT
    assert 0.9 < waited < 5.0, waited
    it = cb.load_scene(scenes.config1(0, 64, 64), flags=cb.DOME_ALIAS)
    it.setGuiding(cb.GuideConfig(train_spp=2, batch=4096))
    it.render(4)
    img = it.readbackFramebuffer()
    gs = it.guideStats()
    it.close()
    assert np.isfinite(img).all() and img[..., :3].mean() > 0
    assert gs["inferred"] > 0
