"""GPU test of zl_moments_noalloc, the entry point that allocates nothing.

Callers that cannot call cudaMalloc (a device-synchronizing allocation is not allowed in
their loop, or their device memory belongs to another allocator) hand it their own device
arrays; its block partials live in a static device array.  The test calls it through the C
ABI on device buffers the test itself owns and checks it against zl_conservation on the
same state, on two calls in a row (the shared static array keeps the previous call's data).
"""
import ctypes

import numpy as np
import pytest

from fixtures import load_lbm, solver_config

pytestmark = pytest.mark.gpu

zl = pytest.importorskip("zllbm_b200")


def _moments_noalloc(lib, lattice, f_dev, n, out_dev, stream=None):
    return lib.zl_moments_noalloc(lattice, ctypes.c_void_p(f_dev.data_ptr()), n,
                                  ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_void_p(stream) if stream else None)


@pytest.mark.parametrize("name", ["tgv3d_mrt", "cavity2d_srt"])
def test_noalloc_moments_match_conservation(name):
    import torch
    meta, codes, f0, _ = load_lbm(name)
    cfg = solver_config(meta, zl.STORAGE_F64)
    lattice = cfg.lattice
    dims = cfg.dims
    with zl.Context(cfg) as ctx:
        ctx.set_level_nodes(0, codes)
        ctx.set_populations(0, codes, f0)
        ctx.advance(7)
        expected = ctx.conservation(0)
        f = ctx.get_populations(0, codes)
    # the reference stores duplicated periodic planes; the context counts each node once
    from oracle.port import morton_decode
    idx = morton_decode(codes, dims) - 1
    keep = np.ones(len(codes), dtype=bool)
    for a, kind in enumerate(meta["bc_kind"][: 2 * dims : 2]):
        if kind == zl.BC_PERIODIC:
            keep &= idx[:, a] < meta["n"][a] - 1
    f_dev = torch.from_numpy(np.ascontiguousarray(f[keep])).cuda()
    out_dev = torch.full((4,), np.nan, dtype=torch.float64, device="cuda")
    lib = zl.load_library()
    for call in range(2):
        out_dev.fill_(np.nan)
        torch.cuda.synchronize()
        assert _moments_noalloc(lib, lattice, f_dev, int(keep.sum()), out_dev) == 0
        torch.cuda.synchronize()
        got = out_dev.cpu().numpy()[: dims + 1]
        assert abs(got[0] - expected[0]) <= 1e-12 * abs(expected[0]), (call, got, expected)
        assert np.allclose(got[1:], expected[1:], rtol=1e-10, atol=1e-12), (call, got, expected)


def test_noalloc_rejects_oversized_and_bad_arguments():
    import torch
    lib = zl.load_library()
    f_dev = torch.zeros(19, dtype=torch.float64, device="cuda")
    out_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert _moments_noalloc(lib, zl.D3Q19, f_dev, 16_777_217, out_dev) == -7
    assert _moments_noalloc(lib, 7, f_dev, 1, out_dev) == -1
    assert lib.zl_moments_noalloc(zl.D3Q19, None, 1, ctypes.c_void_p(out_dev.data_ptr()), None) == -1
