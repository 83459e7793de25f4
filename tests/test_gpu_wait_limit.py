"""Failure detection on the GPU without a fault: a wavefront wait whose
neighbour flag is never set gives up after its iteration limit, the frame
reports CVP9_JOB_TIMEOUT, and the context keeps working."""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import CVP9_OK, CudaBackend, Synth, cuda_lib, synth_config
from oracle.oracle_py import REFCPU, OracleStream

pytestmark = pytest.mark.gpu

JOB_TIMEOUT = 1 << 2


def test_neighbour_wait_gives_up_and_context_survives():
    lib = cuda_lib()
    lib.cuda_backend_selftest_wait_limit.argtypes = [C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]
    status, ms = C.c_uint32(), C.c_float()
    assert lib.cuda_backend_selftest_wait_limit(-1, C.byref(status), C.byref(ms)) == CVP9_OK
    assert status.value & JOB_TIMEOUT, hex(status.value)
    assert 0.0 < ms.value < 30000.0, ms.value
    # the same process then decodes normally
    syn = Synth(synth_config(1, 192, 128, seed=3))
    gpu, orc = CudaBackend(arith=REFCPU), OracleStream(REFCPU)
    for f in range(2):
        pf = syn.frame(f)
        want = orc.decode(pf)
        assert gpu.decode(pf, f) == CVP9_OK
        rc, got, _ = gpu.get_frame_array(wait=1)
        assert rc == CVP9_OK and np.array_equal(got, want)
    gpu.close()
