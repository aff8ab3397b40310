"""The allocation-free sweep entry point, checked against the regular one.

lb_transport_inv_noalloc serves callers that cannot allocate device memory when they solve (a host
framework that owns the device allocator, a Fortran runtime that passes only pre-allocated device
arrays, a loop that must not meet cudaMalloc's implicit synchronisation).  It takes a device vector
owned by the caller and keeps its dependency counters in a fixed file-scope device array.  This
file is collected last so that a run stopping at the first failure has already run every other
test; it passes alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2
from lionbolt_b200 import AngularClass, TransportOp, XSType
from lionbolt_b200 import _lib
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_noalloc_sweep_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    prob = P.config1_small(n=(6, 6, 12), G=1, Ng=6, Nc=12)
    m = prob.mesh
    T = TransportOp().Build(m, AngularClass(k=prob.k, w=prob.w), XSType(*prob.within_group(0)))
    lib, h = T._h.lib, T._h.h
    rng = np.random.default_rng(42)
    for call in range(2):
        q = rng.uniform(0.0, 1.0, size=m.NENK * prob.NI)
        ref = q.copy()
        T.MatInv(ref)                                            # regular entry point (host FP64 buffer)
        dev = torch.from_numpy(q.astype(np.float32)).to("cuda:0")   # caller-owned device vector
        torch.cuda.synchronize()
        st = lib.lb_transport_inv_noalloc(h, ctypes.c_void_p(dev.data_ptr()))
        assert st == 0, f"call {call}: status {st}"
        out = dev.cpu().numpy().astype(np.float64)
        assert rel_l2(out, ref) < TOL, f"call {call}"
    # a vector that is not 16-byte aligned is refused before anything is launched
    assert lib.lb_transport_inv_noalloc(h, ctypes.c_void_p(dev.data_ptr() + 4)) == _lib.LB_ERR_ARG
    buf = ctypes.create_string_buffer(256)
    lib.lb_last_error(h, buf, 256)
    assert b"aligned" in buf.value
