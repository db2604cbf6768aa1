"""C-ABI boundary checks that need no GPU: the library builds, loads, exports every function
the header declares, and its struct layouts match the ctypes mirrors."""

from __future__ import annotations

import ctypes as C

import pytest


@pytest.fixture(scope="module")
def L():
    from litter_physics_b200 import _lib

    _lib.build()
    return _lib


def test_library_exports_every_declared_symbol(L):
    names = L.declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L.lib(), n)]
    assert missing == []


def test_struct_layouts_match(L):
    from litter_physics_b200 import _abi

    sizes = L.struct_sizes()
    assert sizes == {
        "material": C.sizeof(_abi.Material),
        "fixture_spec": C.sizeof(_abi.FixtureSpec),
        "ledger": C.sizeof(_abi.Ledger),
        "counters": C.sizeof(_abi.Counters),
        "particles": C.sizeof(_abi.Particles),
        "pellet": C.sizeof(_abi.Pellet),
    }
    assert L.lib().lp_abi_version() == 1


def test_warm_table_constants_match_header(L):
    """The warm-start table's node layout in the C header equals the Python mirror, and its nodes
    cover every finite FP32 log(a)/8 the solver can form (a >= 1e-37)."""
    import re

    import numpy as np

    from litter_physics_b200 import _abi

    text = L.HEADER.read_text()
    defs = dict(re.findall(r"#define (LP_MLP_TAB_\w+) (.+)", text))
    assert int(defs["LP_MLP_TAB_N"]) == _abi.MLP_TAB_N
    nums = {k: [float(x) for x in re.findall(r"-?\d+\.\d+", v)] for k, v in defs.items()}
    lo = nums["LP_MLP_TAB_LO"][0]
    h = nums["LP_MLP_TAB_H"][0] / nums["LP_MLP_TAB_H"][1]  # written as a quotient
    assert lo == _abi.MLP_TAB_LO and h == _abi.MLP_TAB_H
    nodes = np.float32(lo) + np.arange(_abi.MLP_TAB_N, dtype=np.float32) * np.float32(h)
    assert np.array_equal(nodes.astype(np.float64), lo + np.arange(_abi.MLP_TAB_N) * h)  # exact in FP32
    assert nodes[0] < np.log(1e-37) / 8 and nodes[-1] > np.log(np.finfo(np.float32).max) / 8


def test_material_helpers_match_reference_formulas(L, oracle_mod):
    """constitutive.rs:146-243 on both sides of the boundary (host arithmetic only)."""
    lib = L.lib()
    for args in [(1000.0, 1e5, 0.3, 20.0, 5.0, 0.6), (1200.0, 56250.0, 0.40625, 50.0, 5.0, 0.5)]:
        a = lib.lp_material_paste_from_shear_rheology(*args)
        b = oracle_mod.material_paste_shear(*args)
        for f in ("shear_modulus", "lame_lambda", "bulk_modulus", "yield_stress", "consistency", "flow_index"):
            assert getattr(a, f) == getattr(b, f), f
        assert lib.lp_material_wave_speed(C.byref(a)) > 0
    liq = lib.lp_material_liquid(1000.0, 1e5, 0.2, 1e-3)
    assert liq.bulk_modulus == oracle_mod.material_liquid(1000.0, 1e5, 0.2, 1e-3).bulk_modulus
    assert lib.lp_material_diffusivity(C.byref(liq)) == pytest.approx(1e-6)


def test_hb_features_are_finite(L):
    out = (C.c_float * 6)()
    L.lib().lp_hb_features(100.0, 86.6, 11.4, 0.5, 2e4, 1e-4, out)
    assert all(abs(v) < 1e3 for v in out)


def test_compute_entry_points_fail_loudly_without_device(L):
    """No host fallback: without a CUDA device, creation returns LP_DEVICE."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from litter_physics_b200 import _abi, configs, sim

    with pytest.raises(sim.LPError) as e:
        sim.Simulation(configs.slump(16, (4, 4, 8)))
    assert e.value.status == _abi.LP_DEVICE


def test_export_into_caller_arrays_checks_every_field():
    """An export into a resident host particle set takes arrays of exactly the layout a fresh
    export allocates and refuses anything else before the library is called."""
    import numpy as np

    from litter_physics_b200 import _abi

    arrays, _ = _abi.particle_buffers(5)
    view = _abi.particle_out_view(arrays, 5)
    assert view.count == 5
    for name, bad in (("position", np.zeros((5, 3), np.float32)), ("deformation", np.zeros((5, 9))),
                      ("id", np.zeros(5, np.int64)), ("mass", np.zeros(10)[::2])):
        wrong = dict(arrays, **{name: bad})
        with pytest.raises(ValueError, match=name):
            _abi.particle_out_view(wrong, 5)
    missing = {k: v for k, v in arrays.items() if k != "velocity"}
    with pytest.raises(ValueError, match="velocity"):
        _abi.particle_out_view(missing, 5)
    frozen = dict(arrays)
    frozen["mass"] = arrays["mass"].copy()
    frozen["mass"].flags.writeable = False
    with pytest.raises(ValueError, match="mass"):
        _abi.particle_out_view(frozen, 5)
