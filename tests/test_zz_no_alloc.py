"""hamlss_dot_noalloc: the dot product for callers that cannot let a library allocate
device memory (-m gpu).

Such callers (an application that has reserved the GPU's memory for its own pool, a
latency-critical loop where cudaMalloc / cudaFree would stall the device) get the same
kernel as hamlss_dot with its scratch in a fixed array inside the library.  The test calls
it through the C ABI twice in a row, on different inputs, and compares each result with
hamlss_dot's on the same inputs and with the oracle's sequential sum, within the bound
test_blas1 uses for the dot product (1e-13 of sum |x_i y_i|; hamlss_dot and the no-alloc
call use the same grid, so they agree bit for bit in practice).  The first call on the
device also performs the one-time look-up of the scratch address; later calls, on the
caller's stream or on a stream of its own, leave the device's free memory unchanged.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200 import _abi
from hsps_b200 import problems as P

pytestmark = pytest.mark.gpu


def test_dot_noalloc_matches_dot_twice(orc):
    need_gpu()
    import torch

    L = H.lib()
    ctx = H.Context.default()
    stream = torch.cuda.current_stream().cuda_stream
    for n, seeds in ((1_000_003, (31, 32)), (4_194_304, (33, 34))):
        a = P.rhs(n, seeds[0], -1, 1)
        b = P.rhs(n, seeds[1], -1, 1)
        da = torch.from_numpy(a).cuda()
        db = torch.from_numpy(b).cuda()
        torch.cuda.synchronize()
        want = C.c_double()
        assert L.hamlss_dot(ctx.h, n, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()),
                            C.byref(want)) == 0
        got = C.c_double()
        rc = L.hamlss_dot_noalloc(n, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()),
                                  C.byref(got), C.c_void_p(stream))
        assert rc == 0, L.hamlss_last_error()
        bound = 1e-13 * float(np.abs(a * b).sum())
        assert abs(got.value - want.value) <= bound, (n, got.value, want.value)
        seq = orc.dot(a, b)                      # the reference's sequential order
        assert abs(got.value - seq) <= bound, (n, got.value, seq)
        print(f"n={n}: noalloc {got.value!r} dot {want.value!r} oracle {seq!r} "
              f"identical={got.value == want.value}")


def test_dot_noalloc_allocates_nothing(orc):
    need_gpu()
    import torch

    L = H.lib()
    n = 2_000_000
    a = P.rhs(n, 41, -1, 1)
    b = P.rhs(n, 42, -1, 1)
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    side = torch.cuda.Stream()
    out = C.c_double()
    # first call: loads the kernel's module and looks up the scratch address
    assert L.hamlss_dot_noalloc(n, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()),
                                C.byref(out), None) == 0
    seen = []
    for _attempt in range(3):       # another process on the GPU may move the free figure
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        results = []
        for s in (torch.cuda.current_stream(), side, side):
            rc = L.hamlss_dot_noalloc(n, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()),
                                      C.byref(out), C.c_void_p(s.cuda_stream))
            assert rc == 0, L.hamlss_last_error()
            results.append(out.value)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        seen.append((free0, free1))
        if free1 == free0:
            break
    assert free1 == free0, seen
    assert results[0] == results[1] == results[2], results
    bound = 1e-13 * float(np.abs(a * b).sum())
    assert abs(results[0] - orc.dot(a, b)) <= bound


def test_dot_noalloc_arguments():
    need_gpu()
    L = H.lib()
    out = C.c_double(7.0)
    assert L.hamlss_dot_noalloc(0, None, None, C.byref(out), None) == 0 and out.value == 0.0
    assert L.hamlss_dot_noalloc(-1, None, None, C.byref(out), None) == _abi.ERR_INVALID
    assert b"bad arguments" in L.hamlss_last_error()
