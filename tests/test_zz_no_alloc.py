"""granite_ccz4_constraint_norms_noalloc: constraint norms without allocation.

This entry point serves callers that cannot allocate device memory (code
inside another runtime's memory pool or a pre-sized arena, or code that must
not call cudaMalloc/cudaFree because they synchronise the device). It runs on
the caller's device buffer with a fixed scratch array inside the library.

Checked here through the C ABI against the context-based
granite_ccz4_constraint_norms on the same state, for two calls in a row (the
second on a different state, so stale partial sums from the first call would
show), that the second call leaves the device's free memory unchanged, plus
the rejection of a block beyond the fixed capacity. The file is
named to be collected last; it must also pass alone in a fresh process (the
first call does the per-device set-up).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import Geom

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the same scaled bound as the other parity tests; the reductions match


def _state(g: Geom, seed: int):
    o = oracle.Oracle()
    u = o.init_brill_lindquist(g, [1.0, 0.5], [[0.3, -0.2, 0.1], [-1.1, 0.4, 0.0]],
                               r_floor=0.5 * g.dx[0])
    return u + 1e-6 * oracle.hash_noise(g.shape, seed)


def _context_norms(gb, g: Geom, u):
    ev = gb.Evolver(gb.CCZ4Params())
    b = gb.GridBlock(0, 0, g.n, g.lo, g.hi)
    b.array[...] = u
    ev.add_block(b)
    ev.commit()
    ev.upload()
    h, m = ev.constraint_norms(0)
    ev.close()
    return h, m


def test_noalloc_norms_match_context_path():
    import torch

    import granite_b200 as gb

    lib = gb.load_library()
    fn = lib.granite_ccz4_constraint_norms_noalloc
    fn.argtypes = [C.POINTER(gb._BlockDesc), C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int

    g = Geom((40, 24, 20), (-4.0, -3.0, -2.5), (4.0, 3.0, 2.5))
    states = [_state(g, 1), _state(g, 2) * 1.0001]
    desc = gb.GridBlock(0, 0, g.n, g.lo, g.hi).desc()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    for call, u in enumerate(states):  # two calls in a row through the same static scratch
        u_dev = torch.from_numpy(u.reshape(-1).copy()).to("cuda:0")
        out.fill_(-1.0)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        rc = fn(C.byref(desc), C.c_void_p(u_dev.data_ptr()), C.c_void_p(out.data_ptr()),
                C.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        if call == 1:
            # after the first call has loaded the library's device data, a call
            # takes no device memory at all
            assert torch.cuda.mem_get_info(0)[0] == free_before
        h, m = out.cpu().numpy()
        h_ref, m_ref = _context_norms(gb, g, u)
        assert h_ref > 0 and m_ref > 0
        assert abs(h - h_ref) <= RTOL * h_ref, (h, h_ref)
        assert abs(m - m_ref) <= RTOL * m_ref, (m, m_ref)


def test_noalloc_rejects_blocks_beyond_capacity():
    import torch

    import granite_b200 as gb

    lib = gb.load_library()
    fn = lib.granite_ccz4_constraint_norms_noalloc
    fn.argtypes = [C.POINTER(gb._BlockDesc), C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    torch.cuda.set_device(0)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    # 1 x 2 x 80000 = 80,000 tiles > 65,536: refused before anything is launched
    big = gb._BlockDesc()
    for d, (n, hi) in enumerate(zip((32, 8, 80000), (1.0, 1.0, 100.0))):
        big.ncells[d] = n
        big.lo[d] = 0.0
        big.hi[d] = hi
    big.nghost = 4
    rc = fn(C.byref(big), C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert rc == -8
    assert np.all(out.cpu().numpy() == 0.0)
