"""The allocation-free fan entry point, iga_fan_run_device_noalloc, for callers
that cannot allocate device memory themselves (a fixed up-front device budget
with no cudaMalloc on the request path, or a host framework whose allocator owns
all device memory).  It must give the same arrivals as iga_fan_run_device
(the same kernel with a caller-provided workspace), call after call: the static
scratch it shares between calls is cleared by each call.

Collected last (file name) so that a run stopping at the first failure has run
everything else; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

import infraga_b200 as ig
from infraga_b200 import _lib, synth
from tests._cases import compare_arrivals, profile_path

pytestmark = pytest.mark.gpu


def _rows(n_arr, arr):
    return np.concatenate([arr[i, :n_arr[i]] for i in range(n_arr.size)])


def test_noalloc_entry_matches_device_entry_on_consecutive_calls():
    """Three calls in a row (the first a warm-up) against the workspace entry
    point, with the device's free memory unchanged over the last two."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    L = ig.lib()
    th, ph = synth.fan_angles(1, 45, 2, 0, 300, 60)
    atmo = ig.Atmosphere.load(profile_path(0))
    params = atmo.default_params(bounces=3, rng_max=1200.0)
    n, nb = th.size, params.bounces + 1
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    d_th = torch.tensor(th, dtype=torch.float64, device=dev)
    d_ph = torch.tensor(ph, dtype=torch.float64, device=dev)

    def outputs():
        return (torch.full((n, nb, 12), float("nan"), dtype=torch.float64, device=dev),
                torch.full((n,), -1, dtype=torch.int32, device=dev),
                torch.full((n,), -1, dtype=torch.int64, device=dev),
                torch.full((n,), -1, dtype=torch.int32, device=dev),
                torch.full((n, nb, ig._lib.AUX_COLS), float("nan"), dtype=torch.float64, device=dev))

    # reference: the existing device entry point with a caller workspace
    arr, cnt, steps, stat, aux = outputs()
    ws = torch.zeros(ig.fan_workspace_bytes(), dtype=torch.uint8, device=dev)
    ig.fan_run_device(atmo, params, d_th.data_ptr(), d_ph.data_ptr(), n, arr.data_ptr(), cnt.data_ptr(),
                      steps.data_ptr(), stat.data_ptr(), ws.data_ptr(), stream.cuda_stream, d_aux=aux.data_ptr())
    torch.cuda.synchronize()
    ref_cnt = cnt.cpu().numpy()
    ref_rows = _rows(ref_cnt, arr.cpu().numpy())
    ref_aux = _rows(ref_cnt, aux.cpu().numpy())
    ref_steps = steps.cpu().numpy()
    assert ref_rows.shape[0] > 0

    vp = ctypes.c_void_p
    # Output buffers are made up front so that torch's allocator does no work
    # between the memory readings below.  Call 0 is the warm-up: the first call
    # on a device is when the driver loads the library's device code and static
    # array.  Calls 1 and 2 must leave the device's free memory unchanged.
    bufs = [outputs() for _ in range(3)]
    torch.cuda.synchronize()
    free_after_warmup = None
    for call in range(3):
        arr, cnt, steps, stat, aux = bufs[call]
        if call == 1:
            free_after_warmup = torch.cuda.mem_get_info(dev)[0]
        rc = L.iga_fan_run_device_noalloc(atmo.handle, ctypes.byref(params), vp(d_th.data_ptr()),
                                          vp(d_ph.data_ptr()), n, vp(arr.data_ptr()), vp(cnt.data_ptr()),
                                          vp(steps.data_ptr()), vp(stat.data_ptr()), vp(aux.data_ptr()),
                                          vp(stream.cuda_stream))
        assert rc == _lib.IGA_OK, (call, _lib.strerror(rc), _lib.last_cuda_error())
        torch.cuda.synchronize()
        got_cnt = cnt.cpu().numpy()
        np.testing.assert_array_equal(got_cnt, ref_cnt)
        np.testing.assert_array_equal(steps.cpu().numpy(), ref_steps)
        ok, msg = compare_arrivals(_rows(got_cnt, arr.cpu().numpy()), ref_rows)
        assert ok, (call, msg)
        np.testing.assert_allclose(_rows(got_cnt, aux.cpu().numpy()), ref_aux, rtol=1e-12, atol=0)
    assert torch.cuda.mem_get_info(dev)[0] == free_after_warmup, "device memory changed across the no-alloc calls"

    # FP32C is refused (its absorption table would be allocated on first use)
    p32 = atmo.default_params(bounces=3, rng_max=1200.0, precision=ig.FP32C)
    rc = L.iga_fan_run_device_noalloc(atmo.handle, ctypes.byref(p32), vp(d_th.data_ptr()), vp(d_ph.data_ptr()), n,
                                      vp(arr.data_ptr()), vp(cnt.data_ptr()), vp(steps.data_ptr()), None, None,
                                      vp(stream.cuda_stream))
    assert rc == _lib.IGA_E_UNSUPPORTED
