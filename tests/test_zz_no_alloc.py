"""isw_dsum_static, the deterministic sum that allocates nothing (for callers that cannot allocate device memory at the
call: a host that reserved the device heap up front, or a plugin whose host owns it), called through the C ABI: its result equals
isw_dsum's bit for bit (the tolerance the sum tests use), on two calls in a row sharing its fixed scratch array; sizes
beyond the array are refused. This file sorts last so a run that stops at the first failure has run every other test."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_dsum_static_matches_dsum_twice():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from isw import _lib
    dev = torch.device('cuda:0')
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    for n in (2049, 1 << 20):                          # two calls in a row, the second reusing the array's contents
        i = np.arange(n, dtype=np.int64)
        x = torch.as_tensor(((i * 7919) % 10007 - 5003) / 997.0, device=dev)
        y = torch.as_tensor(((i * 104729) % 65521) / 4093.0, device=dev)
        want = ctypes.c_double()
        _lib.check(_lib.isw_dsum(x.data_ptr(), y.data_ptr(), n, ctypes.byref(want), stream))
        _lib.check(_lib.isw_dsum_static(x.data_ptr(), y.data_ptr(), n, out.data_ptr(), stream))
        torch.cuda.synchronize()
        assert float(out.item()) == want.value
    status = _lib.isw_dsum_static(x.data_ptr(), None, (1 << 27) + 1, out.data_ptr(), stream)
    assert status == _lib.ISW_EINVAL
    assert b'exceeds' in _lib.isw_last_error()
