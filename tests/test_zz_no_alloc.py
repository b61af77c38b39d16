"""The allocation-free probability entry point.

dgq_calcProbOfAllZeroNoAlloc serves callers that cannot allocate GPU memory
while they call the library (hosts that own all device memory, such as a
caching allocator or a server with a fixed HBM budget; latency-bound loops
where cudaMalloc would synchronise the device): its scratch is a static
device array. This file is collected last so a failure here comes after
every other test. It checks, through the C ABI, that the entry point agrees
with the regular read-out (dgq_calcProbOfAllZero) on two calls in a row
(two different states, so stale scratch from the first call would show in
the second), that it rejects states larger than its scratch holds, and that
it rejects buffers that are not memory of the current device (a host query,
before any launch).
"""
import ctypes

import numpy as np
import pytest

from dgquest_b200 import circuits as C

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _probs_no_alloc(quest, q, torch):
    nb = ctypes.c_int(0)
    dstate = quest.dgq_getDeviceState(q, ctypes.byref(nb))
    out = torch.full((nb.value + 1,), -1.0, dtype=torch.float64, device="cuda")  # caller-owned output
    stream = quest.dgq_getStream(q)
    quest.dgq_sync(q)
    rc = quest.dgq_calcProbOfAllZeroNoAlloc(dstate, nb.value, out.data_ptr(), stream)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy(), nb.value


def test_no_alloc_matches_regular_readout_twice(quest, env):
    import torch
    # no swapGate here: the entry point reports address bits, the regular
    # read-out logical qubits, and a swap relabels one against the other
    kinds = [k for k in range(C.CY + 1) if k not in (C.SWAP, C.MEASURE)]
    states = [(22, C.random_layers(22, 8, C.config_seed(2, 71))), (17, C.mixed_ops(17, 300, 72, kinds=kinds))]
    for n, ops in states:
        q = quest.createQureg(n, env)
        C.replay(q, ops)
        got, nb = _probs_no_alloc(quest, q, torch)
        ref = quest.prob_all_zero(q)
        assert nb == n
        assert np.abs(got[:n] - ref).max() <= TOL
        assert abs(got[n] - 1.0) <= TOL
        quest.destroyQureg(q, env)


def test_no_alloc_rejects_oversized_state(quest, env):
    q = quest.createQureg(10, env)
    nb = ctypes.c_int(0)
    dstate = quest.dgq_getDeviceState(q, ctypes.byref(nb))
    with pytest.raises(quest.QuESTError) as ei:
        quest.dgq_calcProbOfAllZeroNoAlloc(dstate, 31, dstate, None)
    assert "1..30" in ei.value.message
    quest.destroyQureg(q, env)


def test_no_alloc_rejects_host_memory(quest, env):
    q = quest.createQureg(10, env)
    nb = ctypes.c_int(0)
    dstate = quest.dgq_getDeviceState(q, ctypes.byref(nb))
    host = np.zeros(nb.value + 1, dtype=np.float64)
    with pytest.raises(quest.QuESTError) as ei:
        quest.dgq_calcProbOfAllZeroNoAlloc(dstate, nb.value, host.ctypes.data, None)
    assert "current device" in ei.value.message or "not CUDA memory" in ei.value.message
    quest.destroyQureg(q, env)
