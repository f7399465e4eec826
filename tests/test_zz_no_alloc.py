"""gem_ifft_run_noalloc, the inverse FFT that allocates nothing, against
gem_ifft_run_device on the same device buffers.

Both run the same table and transform kernels; the no-allocation entry point
takes its tables from a static device array instead of a context buffer, so
the series must agree within the inverse-FFT tests' tolerance (1e-7 relative
L2 per series).  Two calls in a row with different FFT lengths show that each
call rewrites the tables the previous one left in the shared array.  The file
is named to be collected last; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL_L2 = 1e-7


def _noalloc():
    from gemini_unified_b200.fk import lib
    f = lib().gem_ifft_run_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_longlong, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_char_p, ctypes.c_int]
    f.restype = ctypes.c_int
    return f


def test_noalloc_matches_ifft_run_device_on_two_calls(gpu):
    import torch
    from gemini_unified_b200.fk import FrequencyTime
    f = _noalloc()
    ft = FrequencyTime()
    stream = torch.cuda.current_stream()
    err = ctypes.create_string_buffer(256)
    # (nf1, nf2, df, nsamp, dt, series, leading dimension): the 8192-sample
    # series of the batched configuration, then the 2048-sample global one
    cases = [(2, 411, 1.0 / 2048, 8192, 0.25, 23, 420), (2, 52, 1.0 / 1024, 2048, 0.5, 37, 52)]
    free_after = []
    for i, (nf1, nf2, df, nsamp, dt, ntr, ld) in enumerate(cases):
        rng = np.random.default_rng(10 + i)
        sp = rng.standard_normal((ntr, ld)) + 1j * rng.standard_normal((ntr, ld))
        d_sp = torch.from_numpy(sp.view(np.float64).copy()).cuda()
        d_ref = torch.zeros((ntr, nsamp), dtype=torch.float32, device="cuda")
        d_out = torch.full((ntr, nsamp), float("nan"), dtype=torch.float32, device="cuda")
        sigma = 5 * df
        ft.run_device(nf1, nf2, df, sigma, ntr, d_sp.data_ptr(), ld, nsamp, dt, d_ref.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = f(nf1, nf2, df, sigma, ntr, d_sp.data_ptr(), ld, nsamp, dt, d_out.data_ptr(), stream.cuda_stream, err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        free_after.append((free_before, torch.cuda.mem_get_info()[0]))
        ref = d_ref.cpu().numpy().astype(np.float64)
        got = d_out.cpu().numpy().astype(np.float64)
        assert np.all(np.isfinite(got))
        rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rel.max() <= RTOL_L2
    # the second call (set-up already done) leaves the device's free memory unchanged
    assert free_after[1][0] == free_after[1][1]


def test_noalloc_rejects_fft_lengths_beyond_its_limit(gpu):
    """A 16384-sample transform is refused with GEM_ERROR and a message.  The
    8192-sample length limit is what keeps every call's tables inside the static
    array (a compile-time check in the library states that relation)."""
    import torch
    f = _noalloc()
    err = ctypes.create_string_buffer(256)
    d_sp = torch.zeros((1, 2 * 4200), dtype=torch.float64, device="cuda")
    d_ts = torch.zeros((1, 16384), dtype=torch.float32, device="cuda")
    rc = f(2, 4100, 1.0 / 16384, 0.0, 1, d_sp.data_ptr(), 4200, 16384, 1.0, d_ts.data_ptr(), None, err, 256)
    assert rc == 2
    assert b"8192" in err.value
