"""The allocation-free scene build against the allocating one.

Callers that cannot allocate device memory themselves (a plugin inside a
runtime that owns the device's memory pool, a process with a fixed memory
budget) build scenes through ehss_scene_build_noalloc, whose workspace is one
fixed array inside the library.  This test calls it through the C ABI twice in
a row (the second call finds the first call's leftovers in that array) and
checks each scene, byte for byte, and the paths traced through it against the
scene built by ehss_scene_build with a caller-allocated workspace.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _zeroed_scene(torch, nbytes):
    buf = torch.zeros(nbytes + 256, dtype=torch.uint8, device='cuda')
    addr = (buf.data_ptr() + 255) & ~255
    return buf, addr, addr - buf.data_ptr()


def test_noalloc_build_matches_allocating_build():
    torch = pytest.importorskip('torch')
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ehss_b200 as eb
    from ehss_b200 import _lib, workloads as W
    from ehss_b200.device import stream_handle
    lib = _lib.load()
    stream = stream_handle()
    for call in range(2):
        # above 8192 atoms the keys go through the device-wide sort, whose counters also live in the
        # array; 20,000 atoms is the stated maximum
        for n, seed in ((650, 1 + call), (23, 7), (1, 3), (12000, 5), (20000, 8 + call)):
            c, r, _ = W.globule(n, seed)
            xyz = torch.from_numpy(np.ascontiguousarray(c)).cuda()
            rad = torch.from_numpy(np.ascontiguousarray(r)).cuda()
            sb, wb = ct.c_uint64(), ct.c_uint64()
            _lib.check(lib.ehss_scene_bytes(n, 4, ct.byref(sb), ct.byref(wb)))
            ref_buf, ref_addr, ref_off = _zeroed_scene(torch, sb.value)
            ws = torch.empty(wb.value + 256, dtype=torch.uint8, device='cuda')
            _lib.check(lib.ehss_scene_build(n, xyz.data_ptr(), rad.data_ptr(), 4, ref_addr, sb.value,
                                            (ws.data_ptr() + 255) & ~255, wb.value, stream))
            new_buf, new_addr, new_off = _zeroed_scene(torch, sb.value)
            _lib.check(lib.ehss_scene_build_noalloc(n, xyz.data_ptr(), rad.data_ptr(), 4, new_addr, sb.value, stream))
            torch.cuda.synchronize()
            a = ref_buf[ref_off:ref_off + sb.value].cpu().numpy()
            b = new_buf[new_off:new_off + sb.value].cpu().numpy()
            np.testing.assert_array_equal(a, b)
            # trace the same rays through both scenes
            o = torch.empty((1 << 10, 3), dtype=torch.float64, device='cuda')
            d = torch.empty_like(o)
            _lib.check(lib.ehss_source_rays(new_addr, 10, 99, 0, 1 << 10, o.data_ptr(), d.data_ptr(), stream))
            outs = []
            for addr in (ref_addr, new_addr):
                P, D = o.clone(), d.clone()
                last = torch.full((1 << 10,), -1, dtype=torch.int64, device='cuda')
                bounces = torch.zeros(1 << 10, dtype=torch.int64, device='cuda')
                esc = torch.zeros(1 << 10, dtype=torch.uint8, device='cuda')
                unres = torch.zeros_like(esc)
                _lib.check(lib.ehss_trace(addr, 1 << 10, 64, _lib.PREC_FP32, P.data_ptr(), D.data_ptr(),
                                          last.data_ptr(), bounces.data_ptr(), esc.data_ptr(), unres.data_ptr(),
                                          None, None, stream))
                outs.append([x.cpu().numpy() for x in (P, D, bounces, esc, unres)])
            for x, y in zip(*outs):
                np.testing.assert_array_equal(x, y)
    # beyond the stated maximum: a clear error, nothing launched
    n = 20001
    xyz = torch.zeros((n, 3), dtype=torch.float64, device='cuda')
    rad = torch.ones(n, dtype=torch.float64, device='cuda')
    rc = lib.ehss_scene_build_noalloc(n, xyz.data_ptr(), rad.data_ptr(), 4, xyz.data_ptr(), 1, stream)
    assert rc == _lib.ERR_VALUE
    assert b'20000' in lib.ehss_last_error()
