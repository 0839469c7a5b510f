"""CPU tests of the C ABI library: it loads, exports every declared symbol, validates arguments."""
import ctypes
import os

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
    assert zl.load_library().zl_abi_version() == zl.ABI_VERSION == 2


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


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++17")])
def test_header_is_plain_c_and_links(tmp_path, compiler, std):
    """The boundary a host binds: the header compiles as C99 and as C++, and a program linked
    against the library calls it (no device work: the ABI version and a rejected config)."""
    import shutil
    import subprocess
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.join(root, "zllbm_b200")
    src = tmp_path / ("probe.c" if compiler == "gcc" else "probe.cpp")
    src.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "zllbm_b200.h"\n'
        "int main(void) {\n"
        "    zl_config cfg;\n"
        "    zl_ctx* ctx = NULL;\n"
        "    memset(&cfg, 0, sizeof(cfg));\n"
        "    cfg.lattice = 5;\n"
        '    printf("%d %d %d\\n", zl_abi_version(), ZL_ABI_VERSION, zl_create(&cfg, &ctx) != ZL_OK && ctx == NULL);\n'
        "    return 0;\n}\n")
    exe = tmp_path / "probe"
    subprocess.run([compiler, std, "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(src), "-o", str(exe),
                    "-L", lib_dir, "-lzllbm_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out == ["2", "2", "1"]
