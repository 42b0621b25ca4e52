"""The allocation-free space-charge kick, sb2_sc3d_apply_noalloc.

Some callers own all device memory themselves and cannot let a library call
cudaMalloc/cudaFree (a framework with its own pool, a caller with a fixed
memory budget).  For them the library offers the kick of sb2_sc3d_apply with
every workspace in one fixed device array.  This file checks, through the C
ABI, that it gives the same kick as the allocating entry point -- on two
calls in a row, the second with a different grid and a fixed domain, so the
shared array's leftovers from the first call must not leak into the second
-- that a call leaves the device's free memory unchanged (it allocates
nothing), and that grids beyond its fixed workspace are refused.

It sits in a file of its own that pytest collects last; it passes alone in a
fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from helpers import MP, SIG_C0, gaussian_bunch, rel_l2

pytestmark = pytest.mark.gpu

TS = 1.25 / (0.96 * 299792458.0)  # one 1.25 m step at 2.5 GeV


def _allocating_kick(syn, parts, opts):
    ref = syn.Reference_particle(1, syn.Four_momentum(MP, MP + 2.5))
    b = syn.Bunch(ref, parts.shape[0], 1e11)
    b.set_particles(parts)
    syn.Space_charge_3d_open_hockney(opts).apply(b, TS)
    return b.get_particles()[0]


def _caller_arrays(syn, parts):
    """Device arrays that the caller owns (here: a bunch created by this
    test), filled with `parts`."""
    ref = syn.Reference_particle(1, syn.Four_momentum(MP, MP + 2.5))
    b = syn.Bunch(ref, parts.shape[0], 1e11)
    b.set_particles(parts)
    return b


def _noalloc_call(syn, b, n, opts):
    dparts, stride, dmasks, _ = b.device_arrays()
    syn.check(syn.lib().sb2_sc3d_apply_noalloc(ctypes.byref(opts._o), dparts, stride, dmasks, n, n, 1e11, 1, MP,
                                               MP + 2.5, 0, TS, None))


def _noalloc_kick(syn, parts, opts):
    """Kick particles held in caller-owned device memory through the C ABI."""
    b = _caller_arrays(syn, parts)
    _noalloc_call(syn, b, parts.shape[0], opts)
    return b.get_particles()[0]


def _same_kick(before, a, b):
    for j in (0, 2, 4, 6):
        assert np.array_equal(a[:, j], b[:, j]), j
    for j in (1, 3, 5):
        # only the deposit's summation order differs between the two runs
        assert rel_l2(b[:, j] - before[:, j], a[:, j] - before[:, j]) <= 1e-9, j


def test_noalloc_kick_matches_allocating_entry(syn):
    # first call: adaptive domain, 32 x 32 x 64 grid
    p1 = gaussian_bunch(100000, SIG_C0, 51)
    o1 = syn.Space_charge_3d_open_hockney_options(32, 32, 64)
    _same_kick(p1, _allocating_kick(syn, p1, o1), _noalloc_kick(syn, p1, o1))
    # second call in a row: another bunch, another grid, fixed domain
    p2 = gaussian_bunch(60000, [2e-3, 1e-4, 1e-3, 1e-4, 0.2, 1e-4], 52)
    o2 = syn.Space_charge_3d_open_hockney_options(16, 32, 32)
    o2.green_fn = syn.green_fn_t.pointlike
    o2.set_fixed_domain([0.0, 0.0, 0.0], [1.6e-2, 8e-3, 1.6])
    _same_kick(p2, _allocating_kick(syn, p2, o2), _noalloc_kick(syn, p2, o2))


def test_noalloc_call_leaves_device_memory_unchanged(syn):
    """After a first call (which resolves the workspace's address), another
    call on the same arrays changes the device's free memory by nothing: no
    workspace is allocated or freed behind the caller's back."""
    import torch
    p = gaussian_bunch(50000, SIG_C0, 54)
    o = syn.Space_charge_3d_open_hockney_options(32, 32, 64)
    b = _caller_arrays(syn, p)
    _noalloc_call(syn, b, p.shape[0], o)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _noalloc_call(syn, b, p.shape[0], o)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_grids_beyond_workspace(syn):
    p = gaussian_bunch(1000, SIG_C0, 53)
    o = syn.Space_charge_3d_open_hockney_options(64, 64, 128)
    with pytest.raises(syn.SB2Error, match="fixed workspace"):
        _noalloc_kick(syn, p, o)
