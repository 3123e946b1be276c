"""ocfd_show_flow_msg_noalloc: show_flow_msg on caller-owned device arrays with
no device allocation (GPU, through the C ABI).

It is meant for callers that cannot allocate device memory -- a host solver
whose device memory all belongs to its own pool allocator, or code that must not
trigger cudaFree's device-wide synchronisation while other streams run.  The
caller here owns its arrays as torch tensors.  Checked: two calls in a row give
identical results, both equal to ocfd_gpu_show_flow_msg on the same state within
rounding (the two sum in different orders); after the first call on the device
(which looks up the static array's address) the calls leave the device's free
memory and the torch allocator's statistics unchanged; a grid with more
k-planes than the static scratch holds is rejected.  This file is collected
last, so a run that stops at the first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from ocfd_b200 import _lib, cases
from ocfd_b200.params import SCHEME_OMP6
from ocfd_b200.solver import Solver

pytestmark = pytest.mark.gpu

OCFD_E_PARAM = -1
MAX_PLANES = 4096


def _call(L, p, f, prims, ajac, stream):
    E0 = np.zeros(3)
    ptrs = (C.c_void_p * 5)(*[q.data_ptr() for q in prims])
    rc = L.ocfd_show_flow_msg_noalloc(C.byref(p), C.c_void_p(f.data_ptr()), ptrs, C.c_void_p(ajac.data_ptr()),
                                      C.c_void_p(stream), E0.ctypes.data_as(C.POINTER(C.c_double)))
    return rc, E0


def _case(n, ny, nz):
    """State of a few Taylor-Green steps: the handle path's show_flow_msg and the
    same arrays copied to caller-owned device tensors."""
    import torch

    p = cases.tgv_params(n, scheme=SCHEME_OMP6, character=1, dt=0.002, ny=ny, nz=nz)
    s = Solver(p)
    s.init_mesh()
    s.init3d(cases.tgv_prims(s.p))
    s.step(3)
    ref = s.show_flow_msg()
    f_h, prims_h = s.download_state()
    ajac_h = s.download_metrics()[12]
    params = s.p
    s.close()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    f = torch.from_numpy(np.ascontiguousarray(f_h)).to(dev)
    prims = [torch.from_numpy(np.ascontiguousarray(q)).to(dev) for q in prims_h]
    ajac = torch.from_numpy(np.ascontiguousarray(ajac_h)).to(dev)
    torch.cuda.synchronize(dev)
    return params, ref, f, prims, ajac, torch.cuda.current_stream(dev).cuda_stream


@pytest.mark.parametrize("shape", [(32, 24, 20), (64, 64, 8)], ids=["box", "thin"])
def test_noalloc_show_flow_msg_matches_handle_entry_point(shape):
    import torch

    params, ref, f, prims, ajac, stream = _case(*shape)
    L = _lib.lib()
    # the first call on the device looks up the static array's address
    rc0, e0 = _call(L, params, f, prims, ajac, stream)
    assert rc0 == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    stats0 = {k: v for k, v in torch.cuda.memory_stats().items() if k.endswith(".allocated") or "reserved" in k}
    rc1, e1 = _call(L, params, f, prims, ajac, stream)
    rc2, e2 = _call(L, params, f, prims, ajac, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    stats1 = {k: v for k, v in torch.cuda.memory_stats().items() if k.endswith(".allocated") or "reserved" in k}
    assert rc1 == 0 and rc2 == 0
    assert free1 == free0, "the device's free memory changed across the calls"
    assert stats1 == stats0, "the torch allocator's statistics changed across the calls"
    np.testing.assert_array_equal(e1, e2)
    np.testing.assert_array_equal(e0, e1)
    np.testing.assert_allclose(e1, ref, rtol=1e-13, atol=0.0)

    big = type(params).from_buffer_copy(params)
    big.nz = MAX_PLANES + 1
    rc, _ = _call(L, big, f, prims, ajac, stream)
    assert rc == OCFD_E_PARAM
