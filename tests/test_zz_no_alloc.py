"""ocfd_show_flow_msg_noalloc: show_flow_msg on caller-owned device arrays with
no device allocation (GPU, through the C ABI).  The caller here owns its
arrays as torch tensors; the entry point itself allocates nothing.  Two calls
in a row give identical results, both equal to ocfd_gpu_show_flow_msg on the
same state within rounding (the two sum in different orders), and a grid with
more k-planes than the static scratch holds is rejected."""
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


def test_noalloc_show_flow_msg_matches_handle_entry_point():
    import torch

    p = cases.tgv_params(32, scheme=SCHEME_OMP6, character=1, dt=0.002, ny=24, nz=20)
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
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize(dev)

    L = _lib.lib()
    rc1, e1 = _call(L, params, f, prims, ajac, stream)
    rc2, e2 = _call(L, params, f, prims, ajac, stream)
    assert rc1 == 0 and rc2 == 0
    np.testing.assert_array_equal(e1, e2)
    np.testing.assert_allclose(e1, ref, rtol=1e-13, atol=0.0)

    big = type(params).from_buffer_copy(params)
    big.nz = MAX_PLANES + 1
    rc, _ = _call(L, big, f, prims, ajac, stream)
    assert rc == OCFD_E_PARAM
