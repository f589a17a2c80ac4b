"""The allocation-free colouring entry point (b2dev_colour_noalloc).

Some callers cannot allocate device memory: code recorded into a CUDA graph
while a stream is being captured, solvers embedded in an application whose
device memory belongs to its own allocator or pool, and real-time loops where
cudaMalloc would stall the device. For them the library offers one entry
point whose scratch is a fixed array compiled into the library. These tests
call it through the C ABI, twice in a row on different graphs so the second
call starts from the first call's leftovers in the shared scratch, and check
that the colours are exactly those of the allocating path for the same seed.
This file sorts last so a failure here comes after every other test has run;
it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from solfec_b200 import LOCDYN, scenes
from solfec_b200._lib import last_error, lib

pytestmark = pytest.mark.gpu

SEED = 0xC0FFEE
MAX_ROWS = 1 << 20


def colours_allocating(ld):
    ldy = LOCDYN()
    ldy.set_colour_seed(SEED)
    ldy.set(ld)
    col = ldy.colours()
    ldy.close()
    return col


def colours_noalloc(ld, torch):
    dev = torch.device('cuda', 0)
    adjptr = torch.from_numpy(np.ascontiguousarray(ld.adjptr, np.int32)).to(dev)
    adjcol = torch.from_numpy(np.ascontiguousarray(ld.adjcol, np.int32)).to(dev)
    colour = torch.full((ld.n,), 12345, dtype=torch.int32, device=dev)  # stale values the call must overwrite
    info = torch.full((4,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    rc = lib().b2dev_colour_noalloc(0, C.c_void_p(stream.cuda_stream), ld.n, C.c_void_p(adjptr.data_ptr()),
                                    C.c_void_p(adjcol.data_ptr()), SEED, C.c_void_p(colour.data_ptr()),
                                    C.c_void_p(info.data_ptr()))
    assert rc == 0, last_error()
    stream.synchronize()
    return colour.cpu().numpy(), info.cpu().numpy()


def test_colour_noalloc_matches_allocating_path_twice():
    torch = pytest.importorskip('torch')
    graphs = [O.assemble(scenes.spheres_lattice()), O.assemble(scenes.hexahedra_lattice(nx=24, ny=24, nz=4))]
    for ld in graphs:  # two calls in a row, different sizes
        expected = colours_allocating(ld)
        col, info = colours_noalloc(ld, torch)
        assert info[0] == 0 and info[1] == 0, info          # no timeout, no colour overflow
        assert info[2] == expected.max() + 1, info          # number of colours
        assert np.array_equal(col, expected)
        rows = np.repeat(np.arange(ld.n), np.diff(ld.adjptr))
        assert not np.any(col[rows] == col[ld.adjcol])      # a proper colouring


def test_colour_noalloc_rejects_oversize():
    pytest.importorskip('torch')
    rc = lib().b2dev_colour_noalloc(0, None, MAX_ROWS + 1, None, None, SEED, None, None)
    assert rc != 0
    assert 'exceed' in last_error()
