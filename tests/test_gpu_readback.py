"""Read-backs into page-locked blocks from the library's cache.

GpuRun.dft() returns large DFT sums in blocks from vgpu_host_alloc, which
the device writes directly; a read into ordinary pageable memory goes
through the staged copy.  Both must give the same values, and a freed block
must serve the next request of its size."""
import ctypes as C

import numpy as np
import pytest

import vulture_b200 as vb
from vulture_b200 import _native as N
from vulture_b200 import meshgen
from vulture_b200.solver import _result_array
from helpers import stage_text

pytestmark = pytest.mark.gpu


def test_dft_read_pinned_equals_pageable():
    text = meshgen.graded_upml(nt=100, dims=(80, 72, 32), plane=64, nfreq=40, npml=4, ntd=2)
    m = vb.Mesh(stage_text(text, "readback.mesh"))
    g = vb.GpuRun(m, "fp32").run()
    re, im = g.dft()
    shape = (m.num_fd, 6, m.num_freq)
    assert re.nbytes >= (4 << 20)   # large enough for a page-locked block
    pr, pi = np.empty(shape), np.empty(shape)
    N.check_gpu(N.lib().vgpu_read_dft(g._e, pr.ctypes.data, pi.ctypes.data))
    big_r, big_i = _result_array(shape), _result_array(shape)
    N.check_gpu(N.lib().vgpu_read_dft(g._e, big_r.ctypes.data, big_i.ctypes.data))
    assert np.array_equal(re, pr) and np.array_equal(im, pi)
    assert np.array_equal(big_r, pr) and np.array_equal(big_i, pi)
    g.close()


def test_host_blocks_are_cached():
    L = N.lib()
    n = (13 << 20) + 4096   # a size no other test asks for: the cache holds none like it
    a = L.vgpu_host_alloc(n)
    assert a
    C.memset(a, 7, n)
    L.vgpu_host_free(a)
    b = L.vgpu_host_alloc(n)
    assert b == a
    L.vgpu_host_free(b)
    arr = _result_array((n // 8,))
    assert arr.nbytes == n and arr.ctypes.data == a
    arr[:] = 1.5
    assert float(arr.sum()) == 1.5 * (n // 8)
