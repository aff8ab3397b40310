"""Failure detection on the GPU without a fault: a bounded device-side wait that runs out.

Every pipeline wait of the tensor-core contractions is bounded; when one gives up, the kernel raises
the handle's error flag and returns, and the host reports LB_ERR_TIMEOUT at its next synchronisation.
The test makes such a wait run out on purpose, on a barrier that nothing arrives at, with a short
bound (a few thousand polls), then checks the status, the message, that the flag was cleared and
that the same handle still computes K correctly afterwards.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import rel_l2
from lionbolt_b200 import AngularClass, ScatteringOp, XSType
from lionbolt_b200 import _lib
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu


def test_pipeline_wait_timeout_is_reported_and_the_handle_stays_usable():
    m = M.box_mesh(3, 3, 3, (0, 0, 0), (1, 1, 1))
    k, w = P.quadrature(6, 12)
    sigt, sigs = np.array([0.5]), np.array([[0.45 * 0.8 ** l for l in range(6)]])
    K = ScatteringOp().Build(m, AngularClass(k=k, w=w), XSType(sigt, sigs))
    lib, h = K._h.lib, K._h.h
    assert lib.lb_probe_pipeline_timeout(h, 4096) == _lib.LB_ERR_TIMEOUT
    buf = ctypes.create_string_buffer(256)
    lib.lb_last_error(h, buf, 256)
    assert b"timed out" in buf.value
    # the flag was read and cleared: the next synchronisation is clean
    assert lib.lb_synchronize(h) == 0
    # the context and the handle still work
    o = O.Oracle(m)
    assert o.set_angular(k, w, 5) == 0
    o.set_xs(sigt, sigs)
    x = np.random.default_rng(3).normal(size=m.NENK * k.shape[0])
    ref = o.scatter_apply(x)
    out = x.copy()
    K.MatVec(out)
    assert rel_l2(out, ref) < 1e-5
