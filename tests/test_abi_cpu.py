"""CPU-side checks of the product library: it loads, exports every symbol the public header
declares, and its host logic (config mapping, mesh generator) is consistent.  No compute calls."""
import ctypes
import os
import re

import numpy as np
import pytest

from ice_fem_2025a_b200 import abi, config as cf
from ice_fem_2025a_b200.meshgen import box_mesh, bezier_extraction_1d, open_uniform_knots

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "icefem_b200.h")).read()
    return sorted(set(re.findall(r"\bint\s+(ifem_[a-z_0-9]+)\s*\(", txt)))


def test_library_loads_and_exports_header_symbols(product_lib):
    names = _header_functions()
    assert len(names) >= len(abi.ABI_FUNCTIONS)
    for n in names:
        assert hasattr(product_lib, n), n
    assert product_lib.ifem_abi_version() == 1


def test_oracle_exports_same_abi(oracle_lib):
    for n in _header_functions():
        assert hasattr(oracle_lib, n.replace("ifem_", "oracle_", 1)), n


def test_struct_sizes_match_header():
    # reference sizes computed by the C compiler for the header structs
    import subprocess, tempfile
    src = r'''
#include <stdio.h>
#include "icefem_b200.h"
int main(){printf("%zu %zu %zu %zu %zu\n", sizeof(ifem_mesh_desc), sizeof(ifem_material), sizeof(ifem_options), sizeof(ifem_time), sizeof(ifem_stats));return 0;}
'''
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(td, "s")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(x) for x in out]
    assert sizes == [ctypes.sizeof(abi.MeshDesc), ctypes.sizeof(abi.Material), ctypes.sizeof(abi.Options),
                     ctypes.sizeof(abi.Time), ctypes.sizeof(abi.Stats)]


def test_bezier_extraction_reproduces_bsplines():
    from scipy.interpolate import BSpline
    kn = open_uniform_knots(6)
    C = bezier_extraction_1d(kn, 2)
    n = len(kn) - 3
    for e in range(6):
        for x in (0.0, 0.3, 0.77, 1.0 - 1e-12):
            xi = (e + x) / 6
            B = np.array([(1 - x) ** 2, 2 * x * (1 - x), x ** 2])
            full = np.nan_to_num(np.array([BSpline.basis_element(kn[i:i + 4], extrapolate=False)(xi) for i in range(n)]))
            assert np.allclose(full[e:e + 3], C[e] @ B, atol=1e-12)


def test_mesh_layout_matches_reference_generator():
    m = box_mesh((3, 2, 2), (3.0, 2.0, 2.0))
    nx, ny = 5, 4
    # element 0 local node (i,j,k) -> i + nx (j + ny k), x fastest
    e0 = m.elems[0]
    assert list(e0[:3]) == [0, 1, 2] and e0[3] == nx and e0[9] == nx * ny
    # element numbering x fastest
    assert m.elems[1][0] == 1 and m.elems[3][0] == nx
    full = m.elem_data()
    assert full.shape == (12, 27, 27)
    assert np.allclose(full.sum(axis=1).sum(axis=1), full.sum(axis=(1, 2)))


def test_config_mapping_reads_reference_keys():
    mesh, d, st = cf.config(2, scale=1 / 32)
    opts = cf.options_from_json(d)
    mat = cf.material_from_json(d, "Ice")
    assert opts.n_dofs == 4 and list(opts.dof_step)[:4] == [0, 0, 1, 2]
    assert opts.gravity == 1 and opts.viscous_heating == 1 and opts.thermal_model == 1
    assert mat.rheology == abi.RHEO["DamViscoElastic"] and mat.split == abi.SPLIT["VolStrains"]
    # Gc = 2 ft^2 l / E reproduces the requested fracture energy (IceMaterial.cpp:71-72)
    mesh0, d0, _ = cf.config(0, scale=0.125)
    m0 = cf.material_from_json(d0, "Ice")
    assert abs(2 * m0.ft0 ** 2 * m0.pf_l / m0.young - 1.0) < 1e-12
    with pytest.raises(ValueError):
        bad = dict(d0)
        bad["properties"] = {**d0["properties"], "Ice": {**d0["properties"]["Ice"],
                             "SolidProperties": {**d0["properties"]["Ice"]["SolidProperties"], "Rheology": "Bogus"}}}
        cf.material_from_json(bad, "Ice")
