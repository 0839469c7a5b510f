"""CPU tests of the C ABI library: it loads, exports every declared symbol, validates arguments."""
import ctypes

import numpy as np
import pytest

import zllbm_b200 as zl


def test_library_exports_every_header_symbol():
    lib = zl.load_library()
    names = zl.header_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name


def test_abi_version():
    assert zl.load_library().zl_abi_version() == 1


@pytest.mark.parametrize("mutate", [
    lambda c: setattr(c, "lattice", 5),
    lambda c: setattr(c, "collision", 7),
    lambda c: setattr(c, "storage", 9),
    lambda c: setattr(c, "max_level", 99),
    lambda c: setattr(c, "viscosity", 0.0),
])
def test_create_rejects_bad_config(mutate):
    cfg = zl.SolverConfig(domain_min=(1, 1, 1), domain_max=(8, 8, 8)).to_c()
    mutate(cfg)
    h = ctypes.c_void_p()
    assert zl.load_library().zl_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    assert not h.value


def test_create_rejects_unpaired_periodic_faces():
    cfg = zl.SolverConfig(domain_min=(1, 1, 1), domain_max=(8, 8, 8), bc_kind=(2, 1, 2, 2, 2, 2)).to_c()
    h = ctypes.c_void_p()
    assert zl.load_library().zl_create(ctypes.byref(cfg), ctypes.byref(h)) == -1


@pytest.mark.parametrize("dims", [2, 3])
def test_mrt_matrix_matches_reference_construction(dims, port):
    # host-side construction of M^-1 S M must equal the reference's (restated in the oracle) bit for bit
    lattice = zl.D2Q9 if dims == 2 else zl.D3Q19
    for tau in (0.503, 0.55, 1.268, 0.5024):
        assert np.array_equal(zl.mrt_matrix(lattice, tau), port.mrt_matrix(dims, tau))


def test_box_codes_helper():
    from oracle.port import morton_decode
    c = zl.box_codes(3, (1, 2, 3), (4, 5, 6))
    idx = morton_decode(c, 3)
    assert idx[0].tolist() == [1, 2, 3] and idx[1].tolist() == [2, 2, 3] and idx[-1].tolist() == [4, 5, 6]


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(zl, "_lib", None)
    with pytest.raises(RuntimeError, match="not built"):
        zl.load_library(str(tmp_path / "libzllbm_b200.so"))


def test_no_cpu_fallback_without_a_gpu():
    """With no CUDA device the solver refuses to start instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(zl.ZlError):
        zl.Context(zl.SolverConfig(domain_min=(1, 1, 1), domain_max=(8, 8, 8)))
