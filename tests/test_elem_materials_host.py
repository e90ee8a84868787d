"""Host side of per-element materials in the Python mirror (no GPU): the
element material lookup follows FemModel3d.getElementMaterial
(FemModel3d.java:608-614), the arrays handed to
b200fem_set_element_materials hold B200FEM_MAT_MODEL where an element keeps
the model's material, and a new mesh clears them."""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200.femmodel import (FemFactory, LinearMaterial, MooneyRivlinMaterial, NeoHookeanMaterial,
                                          StVenantKirchoffMaterial)


def test_element_material_lookup_and_arrays():
    fem = FemFactory.createTetGrid(None, 1.0, 0.4, 0.4, 2, 1, 1)
    fem.setMaterial(NeoHookeanMaterial(5e4, 0.4))
    E = fem.numElements()
    mr = MooneyRivlinMaterial(1e4, 2e3, 0, 0, 0, 1e5, 0.0, 1)
    lin = LinearMaterial(3e4, 0.3, True)
    fem.setElementMaterial(1, mr)
    fem.setElementMaterial(3, lin)
    assert fem.getElementMaterial(0) is fem.material
    assert fem.getElementMaterial(1) is mr and fem.getElementMaterial(3) is lin
    kinds, prm = fem._element_material_arrays()
    assert kinds.dtype == np.int32 and kinds.shape == (E,) and prm.shape == (E, 8)
    expect = np.full(E, L.MAT_MODEL)
    expect[1], expect[3] = L.MAT_MOONEYRIVLIN, L.MAT_LINEAR
    assert np.array_equal(kinds, expect)
    assert np.allclose(prm[1, : len(mr.params())], mr.params())
    assert np.allclose(prm[3, :3], lin.params()) and prm[3, 2] == 1
    assert not prm[0].any()
    fem.setElementMaterial(1, None)
    assert fem.getElementMaterial(1) is fem.material
    fem.setElementMaterials([StVenantKirchoffMaterial(4e4, 0.3)] * E)
    assert (fem._element_material_arrays()[0] == L.MAT_STVK).all()
    with pytest.raises(ValueError):
        fem.setElementMaterials([None] * (E + 1))
    fem.setElementMaterials(None)
    assert fem.elem_materials is None


def test_new_mesh_clears_element_materials():
    fem = FemFactory.createHexGrid(None, 1.0, 0.4, 0.4, 2, 1, 1)
    fem.setElementMaterial(0, NeoHookeanMaterial(1e4, 0.3))
    fem.setMesh(L.ELEM_HEX, fem.rest, fem.conn, fem.fixed)
    assert fem.elem_materials is None
