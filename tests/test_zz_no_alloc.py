"""pscfg_propagate_noalloc: the propagation entry point that allocates no
device memory, for hosts whose device memory is entirely managed by their own
pool and which cannot let a library call cudaMalloc behind their back.

Its output must match the allocating entry point pscfg_propagate (the same
step_exp kernels with scratch from cudaMalloc) to the 1e-12 relative
tolerance used by the other FP64 propagator tests, on two calls in a row
(the second call reuses the scratch array the first one left behind).
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from pscf_b200.engine import Engine, FP64, load_library
from tests.cases import diblock, rel_err, smooth_field

pytestmark = pytest.mark.gpu


def _noalloc(lib, system, ksq_dev, w_dev, q_dev, out_dev, b, ds, nsteps, stream):
    n = (C.c_int * 3)(*system.n)
    return lib.pscfg_propagate_noalloc(system.dim, n, C.c_void_p(ksq_dev.data_ptr()), C.c_void_p(w_dev.data_ptr()),
                                       b, ds, C.c_void_p(q_dev.data_ptr()), C.c_void_p(out_dev.data_ptr()),
                                       nsteps, C.c_void_p(stream))


@pytest.mark.parametrize("dim,ngrid,crystal,cell", [(3, [16, 16, 16], "cubic", [3.9]),
                                                    (3, [20, 12, 14], "orthorhombic", [2.0, 2.5, 3.0]),
                                                    (2, [24, 24], "hexagonal", [1.9]),
                                                    (1, [27], "lamellar", [1.4])])
def test_noalloc_matches_allocating_entry_point_twice(dim, ngrid, crystal, cell):
    import torch
    dev = torch.device("cuda", 0)
    s = diblock(dim, ngrid, crystal, cell)
    e = Engine([s], FP64)
    lib = load_library()
    ksq = torch.from_numpy(e.ksq(0)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for call, (seed, b, ds, nsteps) in enumerate([(11, 1.0, 0.01, 3), (23, 1.3, 0.005, 2)]):
        w = 7.5 + smooth_field(s, seed, 3.0)
        q0 = 1.0 + 0.3 * smooth_field(s, seed + 1, 1.0)
        ref = e.propagate(0, w, b, ds, q0, nsteps)
        w_dev = torch.from_numpy(w).to(dev)
        q_dev = torch.from_numpy(q0).to(dev)
        out = torch.full_like(q_dev, float("nan"))
        rc = _noalloc(lib, s, ksq, w_dev, q_dev, out, b, ds, nsteps, stream.cuda_stream)
        assert rc == 0, lib.pscfg_last_error(None)
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert rel_err(got, ref) < 1e-12, (call, rel_err(got, ref))


def test_noalloc_allocates_nothing_aliases_and_streams():
    """A second call leaves the free device memory unchanged; q_in may be
    q_out; work goes on the caller's (non-default) stream."""
    import torch
    dev = torch.device("cuda", 0)
    s = diblock(3, [16, 16, 16], "cubic", [3.9])
    e = Engine([s], FP64)
    lib = load_library()
    ksq = torch.from_numpy(e.ksq(0)).to(dev)
    w = 7.5 + smooth_field(s, 31, 3.0)
    q0 = 1.0 + 0.3 * smooth_field(s, 32, 1.0)
    ref = e.propagate(0, w, 1.0, 0.01, q0, 4)
    w_dev = torch.from_numpy(w).to(dev)
    side = torch.cuda.Stream(dev)
    for nsteps, expect in ((4, ref), (1, e.propagate(0, w, 1.0, 0.01, q0, 1))):
        q = torch.from_numpy(q0).to(dev)          # in place: q_in == q_out
        torch.cuda.synchronize(dev)
        free0 = torch.cuda.mem_get_info(dev)[0]
        with torch.cuda.stream(side):
            rc = _noalloc(lib, s, ksq, w_dev, q, q, 1.0, 0.01, nsteps, side.cuda_stream)
        assert rc == 0, lib.pscfg_last_error(None)
        side.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free0
        assert rel_err(q.cpu().numpy(), expect) < 1e-12, (nsteps, rel_err(q.cpu().numpy(), expect))


def test_noalloc_rejects_planes_over_shared_memory():
    import torch
    dev = torch.device("cuda", 0)
    lib = load_library()
    n = (C.c_int * 3)(128, 128, 1)            # 16384 points, but the 2-D plane step needs > 227 KB
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    rc = lib.pscfg_propagate_noalloc(2, n, p, p, 1.0, 0.01, p, p, 1, None)
    assert rc != 0
    assert b"no-allocation limit" in lib.pscfg_last_error(None)


def test_noalloc_rejects_grids_over_the_limit():
    import torch
    dev = torch.device("cuda", 0)
    lib = load_library()
    n = (C.c_int * 3)(48, 48, 48)             # 110592 points > PSCFG_NOALLOC_MAX_NR
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    rc = lib.pscfg_propagate_noalloc(3, n, p, p, 1.0, 0.01, p, p, 1, None)
    assert rc != 0
    assert b"limit" in lib.pscfg_last_error(None)
