"""GPU parity of the multi-level (AMR) time step against the reference's own multi-level runs.

Fixtures come from the reference refining around its default shapes (GeometryInfoOrigin) with
NEQ inflow/outflow; every level's populations after a few background steps (sub-cycled
1:2[:4], coarse/fine explosion and coalescence every second fine sub-step) are compared.
"""
import glob
import json
import os

import numpy as np
import pytest

from fixtures import GOLDEN

AMR = sorted(os.path.basename(p)[4:-4] for p in glob.glob(os.path.join(GOLDEN, "amr_*.npz")))
FACES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
KINDS = {"bb": 1, "per": 2, "neq": 3}


def load_amr(name, prefix="amr"):
    z = np.load(os.path.join(GOLDEN, f"{prefix}_{name}.npz"))
    return json.loads(str(z["meta"])), z


def config(meta, storage):
    import zllbm_b200 as zl
    dims = meta["dims"]
    kinds, vels = [0] * 6, [(0.0, 0.0, 0.0)] * 6
    for b in meta["bc"]:
        parts = b.split(":")
        f = FACES.index(parts[0])
        kinds[f] = KINDS[parts[1]]
        if len(parts) > 2:
            v = [float(x) for x in parts[2].split(",")]
            vels[f] = tuple(v + [0.0] * (3 - len(v)))
    hi = [c + 1 for c in meta["n"]] + [0] * (3 - dims)
    cforce = [float(x) for x in meta["cforce"].split(",")] if "cforce" in meta else [0.0, 0.0, 0.0]
    return zl.SolverConfig(lattice=zl.D2Q9 if dims == 2 else zl.D3Q19,
                           collision=zl.MRT if meta["coll"] == "mrt" else zl.SRT, storage=storage,
                           max_level=meta["levels"], viscosity=meta["nu"], bc_kind=tuple(kinds),
                           bc_velocity=tuple(vels), domain_min=(1, 1, 1 if dims == 3 else 0), domain_max=tuple(hi),
                           forcing=1 if ("ib" in meta or "cforce" in meta) else 0,
                           constant_force=tuple(cforce + [0.0] * (3 - len(cforce))))


def test_amr_fixture_layers_are_consistent():
    for name in AMR:
        meta, z = load_amr(name)
        for lv in range(1, meta["levels"] + 1):
            assert np.isin(z[f"c2f_fine{lv}"], z[f"codes{lv}"]).all()
            assert np.isin(z[f"f2c_coarse{lv - 1}"], z[f"codes{lv - 1}"]).all()
            assert z[f"c2f_fine{lv}"].size > 0 and z[f"f2c_coarse{lv - 1}"].size > 0


def run(meta, z, storage, with_forces=False):
    import zllbm_b200 as zl
    levels = meta["levels"]
    with zl.Context(config(meta, storage)) as ctx:
        for lv in range(levels + 1):
            ctx.set_level_nodes(lv, z[f"codes{lv}"])
            ctx.set_populations(lv, z[f"codes{lv}"], z[f"f_before{lv}"])
        for lv in range(1, levels + 1):
            coarse_flags = z[f"flags{lv - 1}"]
            excluded = z[f"codes{lv - 1}"][(coarse_flags & 4) != 0]
            ctx.set_level_interface(lv, z[f"c2f_fine{lv}"], z[f"f2c_coarse{lv - 1}"], excluded)
        if "ib" in meta:
            v = z["vertices_before"]
            ctx.ib_set_vertices(levels, v[:, 0:3], v[:, 3:6], v[:, 6])
        ctx.advance(meta["steps"])
        pops = [ctx.get_populations(lv, z[f"codes{lv}"]) for lv in range(levels + 1)]
        forces = ctx.ib_get_forces(levels) if "ib" in meta else None
    return (pops, forces) if with_forces else pops


@pytest.mark.gpu
@pytest.mark.parametrize("name", AMR)
def test_amr_fp64_bit_exact_against_reference(name):
    """FP64: bit-exact, except immersed-boundary runs, whose node forces are sums over vertices
    in an order the reference takes from an unordered_map (tolerance 1e-12 relative)."""
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    got, forces = run(meta, z, zl.STORAGE_F64, with_forces=True)
    for lv, f in enumerate(got):
        ref = z[f"f_after{lv}"]
        if "ib" in meta:
            np.testing.assert_allclose(f, ref, rtol=1e-12, atol=1e-15, err_msg=f"level {lv}")
        else:
            assert np.array_equal(f, ref), (lv, float(np.abs(f - ref).max()))
    if "ib" in meta:
        vf, total = forces
        ref = z["vertices_after"][:, 7:10]
        np.testing.assert_allclose(vf, ref, rtol=1e-10, atol=1e-14)
        dims = meta["dims"]
        area = z["vertices_after"][:, 6]
        np.testing.assert_allclose(total[:dims], (ref * area[:, None]).sum(0)[:dims], rtol=1e-10, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("name", AMR)
def test_amr_fp32_against_reference(name):
    import zllbm_b200 as zl
    meta, z = load_amr(name)
    got = run(meta, z, zl.STORAGE_F32)
    for lv, f in enumerate(got):
        ref = z[f"f_after{lv}"]
        rel = np.abs(f - ref) / np.abs(ref)
        assert rel.max() <= 1e-5, (lv, float(rel.max()))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ib2d", "ib3d"])
def test_ib_step_from_taylor_green_matches_reference(name):
    """One immersed-boundary step of the reference from a Taylor-Green field (a circle in 2D, a
    sphere in 3D, four-point kernel, periodic box; tests/golden/ibpin_*.npz) through zl_advance in
    FP64: the vertex forces of the pass and the populations after the forced step equal the
    reference's (1e-12: node forces sum vertex shares in another order than the reference's
    unordered_map walk)."""
    import zllbm_b200 as zl
    meta, z = load_amr(name, prefix="ibpin")
    got, (vf, total) = run(meta, z, zl.STORAGE_F64, with_forces=True)
    ref_f = z["f_after0"]
    assert np.abs(ref_f - z["f_before0"]).max() > 1e-4  # the step changes the field
    np.testing.assert_allclose(got[0], ref_f, rtol=1e-12, atol=1e-15)
    ref = z["vertices_after"][:, 7:10]
    dims = meta["dims"]
    assert np.abs(ref[:, :dims]).max() > 1e-3  # non-zero forces
    np.testing.assert_allclose(vf, ref, rtol=1e-10, atol=1e-14)
    area = z["vertices_after"][:, 6]
    np.testing.assert_allclose(total[:dims], (ref * area[:, None]).sum(0)[:dims], rtol=1e-10, atol=1e-14)
