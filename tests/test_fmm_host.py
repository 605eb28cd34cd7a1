"""Fast-multipole form, host side: the expansion primitives against a direct
kernel sum, and the support tree / near-far partition against the reference's
own makeSupportTree (fmm/support_tree.cpp) compiled into oracle/_ref."""
import ctypes as C

import numpy as np
import pytest

from hornsculpt_b200 import _lib, meshes
from oracle import oracle as O


def _tree(mesh, leaf, sep, ratio):
    lib = _lib.load()
    sizes = np.zeros(6, np.uintp)
    v = np.ascontiguousarray(mesh.vertices, np.float64)
    t = np.ascontiguousarray(mesh.triangles, np.uint32)
    _lib.check(lib.hs_bem_debug_fmm_tree(v.ctypes.data, mesh.vertex_count, t.ctypes.data, mesh.triangle_count, leaf,
                                         sep, ratio, sizes.ctypes.data, None, 0))
    total = int(sizes[2:].sum())
    links = np.zeros((max(total, 1), 2), np.uint32)
    _lib.check(lib.hs_bem_debug_fmm_tree(v.ctypes.data, mesh.vertex_count, t.ctypes.data, mesh.triangle_count, leaf,
                                         sep, ratio, sizes.ctypes.data, links.ctypes.data, total))
    return sizes.astype(np.int64), links[:total]


def test_expansion_primitives_against_direct_sum():
    err = C.c_double()
    _lib.check(_lib.load().hs_bem_debug_fmm_selftest(C.byref(err)))
    assert err.value < 1e-9


@pytest.mark.skipif(not O.reference_available(), reason="reference tree absent")
@pytest.mark.parametrize("case", ["icosphere3", "horn", "octa4"])
@pytest.mark.parametrize("leaf, sep", [(16, 1.5), (32, 2.0)])
def test_support_tree_matches_reference(case, leaf, sep):
    mesh = {"icosphere3": lambda: meshes.icosphere(3),
            "horn": lambda: meshes.exponential_horn(h=0.0128, seed=5),
            "octa4": lambda: meshes.octahedral_sphere(4)}[case]()
    mine, links = _tree(mesh, leaf, sep, 2.0)
    ref, ref_links = O.reference_support_tree(mesh, leaf, sep, 2.0)
    assert list(mine) == list(ref)
    assert np.array_equal(links, ref_links)
    assert mine[3] > 0  # the partition has far-field work


def test_invalid_tree_settings_are_rejected():
    mesh = meshes.icosphere(1)
    lib = _lib.load()
    sizes = np.zeros(6, np.uintp)
    v = np.ascontiguousarray(mesh.vertices, np.float64)
    t = np.ascontiguousarray(mesh.triangles, np.uint32)
    with pytest.raises(Exception, match="settings are invalid"):
        _lib.check(lib.hs_bem_debug_fmm_tree(v.ctypes.data, mesh.vertex_count, t.ctypes.data, mesh.triangle_count, 0,
                                             1.5, 2.0, sizes.ctypes.data, None, 0))


@pytest.mark.skipif(not O.reference_available(), reason="reference tree absent")
@pytest.mark.parametrize("case, leaf, sep, ratio", [
    ("revolved", 8, 1.5, 2.0), ("revolved", 64, 3.0, 1.0), ("ico4", 16, 1.5, 0.0),
    ("horn_coarse", 4, 1.8, 2.0), ("tetra", 4, 1.5, 2.0)])
def test_support_tree_matches_reference_more(case, leaf, sep, ratio):
    mesh = {"revolved": lambda: meshes.revolved_sphere(h=0.012, seed=2),
            "ico4": lambda: meshes.icosphere(4),
            "horn_coarse": lambda: meshes.exponential_horn(h=0.016, seed=1),
            "tetra": lambda: meshes.scalene_tetrahedron()}[case]()
    mine, links = _tree(mesh, leaf, sep, ratio)
    ref, ref_links = O.reference_support_tree(mesh, leaf, sep, ratio)
    assert list(mine) == list(ref)
    assert np.array_equal(links, ref_links)
