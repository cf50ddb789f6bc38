"""fmmgpu_direct_sum_noalloc: the direct sum on device buffers with module-scope scratch.

The file name puts it last in collection, so that in a full run it follows every other
test that used the library in the same process; it must pass alone as well.  The GPU
cases compare two calls in a row (fresh inputs each time) with the allocating entry
point, fmmgpu_direct_sum, bit for bit: both use the same kernels and source chunks.
"""
import ctypes as C

import numpy as np
import pytest

import fmm_b200 as F

SCRATCH = 16 << 20


def test_oversize_is_rejected_before_device_work():
    lib = F.lib()
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    # 70000 sources -> 128 chunks of partial sums, 32 bytes per (chunk, target)
    assert SCRATCH // (128 * 32) == 4096
    rc = lib.fmmgpu_direct_sum_noalloc(70000, fake, fake, 4097, fake, fake, None, 0, None)
    msg = lib.fmmgpu_last_error().decode()
    assert rc == 1 and str(SCRATCH) in msg and "at most 4096 targets" in msg, msg
    rc = lib.fmmgpu_direct_sum_noalloc(1000, fake, fake, 524289, fake, fake, None, 0, None)
    msg = lib.fmmgpu_last_error().decode()
    assert rc == 1 and "at most 524288 targets" in msg, msg
    rc = lib.fmmgpu_direct_sum_noalloc(10, None, None, 1, fake, fake, None, 0, None)
    assert rc == 1 and "null buffer" in lib.fmmgpu_last_error().decode()


@pytest.mark.gpu
@pytest.mark.parametrize("ns,nt", [(70000, 4096), (5000, 20000)])
def test_two_calls_match_the_allocating_entry_point(ns, nt):
    import torch

    lib = F.lib()
    rng = np.random.default_rng(ns + nt)
    stream = torch.cuda.Stream()
    for call, gradients in enumerate((True, False)):
        src = rng.uniform(-1, 1, (ns, 3))
        q = rng.normal(size=ns)
        tgt = np.concatenate([rng.uniform(-1.2, 1.2, (nt - 16, 3)), src[:16]])  # 16 coincide with sources
        want_phi, want_g = F.direct_sum(src, q, tgt, gradients=gradients)
        d_src, d_q, d_tgt = (torch.from_numpy(a).cuda() for a in (src, q, tgt))
        phi = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
        g = torch.full((nt, 3), float("nan"), dtype=torch.float64, device="cuda") if gradients else None
        torch.cuda.synchronize()
        rc = lib.fmmgpu_direct_sum_noalloc(ns, d_src.data_ptr(), d_q.data_ptr(), nt, d_tgt.data_ptr(),
                                           phi.data_ptr(), g.data_ptr() if gradients else None, 0,
                                           stream.cuda_stream)
        assert rc == 0, lib.fmmgpu_last_error()
        stream.synchronize()
        assert np.array_equal(phi.cpu().numpy(), want_phi), call
        if gradients:
            assert np.array_equal(g.cpu().numpy(), want_g), call
