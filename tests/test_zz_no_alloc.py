"""tm_anand_screen_noalloc: the Anand screening entry point that allocates no device memory.

It is meant for callers that cannot call cudaMalloc while they screen, such as a host
application whose allocator already owns the device memory or one that forbids
allocations (and the device synchronization they imply) after start-up. Its per-step
tables live in a fixed array of the library instead of fresh allocations. This test calls
it twice in a row through the C-ABI, with the strain table and the outputs in device
memory that the caller (torch) allocated, and checks both results against the regular
entry point tm_anand_screen at the tolerance of the other Anand tests (1e-8 relative).
Around the second call (the library is loaded and the array's address looked up by then) the
device's free memory, as cudaMemGetInfo reports it, must not change.
The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from tmsolve import _lib
from tmsolve.anand import cycle_history, cycling_temps, material, screen, synthetic_strain_table
from tmsolve.materials import SAC305, sac305_tables

pytestmark = pytest.mark.gpu


def test_noalloc_screen_matches_regular_entry_point_twice():
    import torch
    torch.cuda.init()
    Et, Ft = sac305_tables()
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3)
    temps = np.ascontiguousarray(cycling_temps(-40.0, 125.0))
    table, _, _ = synthetic_strain_table(200, temps, seed=7)
    ref_dW, ref_dE, ref_st = screen(SAC305, Et, Ft, temps, table, hist)
    assert np.all(np.isfinite(ref_dW)) and np.all(ref_dW > 0)

    L = _lib.load()
    m, keep = material(SAC305, Et, Ft)
    ns = table.shape[0]
    d_table = torch.from_numpy(np.ascontiguousarray(table).ravel()).cuda()
    t = np.ascontiguousarray(hist["t"], np.float64); T = np.ascontiguousarray(hist["T"], np.float64)
    cyc = np.ascontiguousarray(hist["cycle"], np.int32); ph = np.ascontiguousarray(hist["phase"], np.int32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        dW = torch.full((ns,), -1.0, dtype=torch.float64, device="cuda")
        dE = torch.full((ns,), -1.0, dtype=torch.float64, device="cuda")
        st = torch.full((ns,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rc = L.tm_anand_screen_noalloc(C.byref(m), ns, len(temps), vp(temps), C.c_void_p(d_table.data_ptr()), len(t), vp(t), vp(T),
                                      vp(cyc), vp(ph), int(hist["cycles"]), C.c_void_p(dW.data_ptr()), C.c_void_p(dE.data_ptr()),
                                      C.c_void_p(st.data_ptr()), C.c_void_p(stream))
        assert rc == _lib.TM_OK, _lib.last_error()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        if call == 1:
            assert free1 == free0, (free0, free1)
        assert np.allclose(dW.cpu().numpy(), ref_dW, rtol=1e-8, atol=0), call
        assert np.allclose(dE.cpu().numpy(), ref_dE, rtol=1e-8, atol=0), call
        assert np.allclose(st.cpu().numpy(), ref_st, rtol=1e-8, atol=0), call


def test_noalloc_rejects_oversized_history():
    import torch
    Et, Ft = sac305_tables()
    L = _lib.load()
    m, keep = material(SAC305, Et, Ft)
    n = 4097  # one above TM_NOALLOC_MAX_STEPS
    t = np.arange(n, dtype=np.float64); T = np.full(n, 25.0); cyc = np.ones(n, np.int32); ph = np.ones(n, np.int32)
    temps = np.array([-40.0, 25.0, 125.0])
    buf = torch.zeros(6 * 3, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = L.tm_anand_screen_noalloc(C.byref(m), 1, 3, vp(temps), C.c_void_p(buf.data_ptr()), n, vp(t), vp(T), vp(cyc), vp(ph), 1,
                                  C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.TM_BAD_INPUT
    assert "TM_NOALLOC_MAX_STEPS" in _lib.last_error()
