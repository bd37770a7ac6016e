"""CPU oracle over a membrane between two compartments (merged SSA units, no GPU).

Surface reactions with inner-volume reactants and outer-volume products, outer-volume
reactants and inner products, and a GHK current against the outer tet's concentration with
ion flux (sreac.cpp:305-520, ghkcurr.cpp:168-280): calcium only moves between the two
volumes, the buffer and the pumps, so its total is conserved while both directions of
transport run.
"""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from steps_b200.solver import flatten
from tests.outer_membrane import INITIAL, outer_mesh, outer_model


def _setup(seed=5, ghk=True, sdiff=False):
    mesh = outer_mesh()
    mdl = outer_model(ghk, sdiff)
    F = flatten(mdl, mesh)
    ora = Oracle(F, seed=seed)
    rng = np.random.default_rng(seed)
    comp = F["tet_comp"]
    ci, co = F["comp_index"]["cyto"], F["comp_index"]["ecs"]
    S = F["spec_index"]

    def place(n, tets):
        row = np.zeros(mesh.ntets, dtype=np.uint32)
        np.add.at(row, rng.choice(tets, size=n), 1)
        return row

    inner, outer = np.nonzero(comp == ci)[0], np.nonzero(comp == co)[0]
    ora.set_counts(S["Ca"], place(INITIAL["Ca_in"], inner) + place(INITIAL["Ca_out"], outer))
    ora.set_counts(S["B"], place(INITIAL["B"], inner))
    sf = F["surf"]
    M = len(sf["tris"])
    ss = sf["sspec_index"]
    for name in ("P", "Kc"):
        row = np.zeros(M, dtype=np.uint32)
        np.add.at(row, rng.integers(0, M, size=INITIAL[name]), 1)
        ora.set_tri_counts(ss[name], row)
    return mesh, F, ora


def _ca_total(F, ora):
    S, ss = F["spec_index"], F["surf"]["sspec_index"]
    return int(ora.get_counts(S["Ca"]).sum()) + int(ora.get_counts(S["CaB"]).sum()) + int(
        ora.get_tri_counts(ss["PCa"]).sum())


def test_outer_tets_are_recorded():
    mesh, F, _ = _setup()
    sf = F["surf"]
    outer = sf["tri_outer"]
    assert outer is not None and np.all(outer >= 0)
    comp = F["tet_comp"]
    assert np.all(comp[sf["tri_inner"]] == F["comp_index"]["cyto"])
    assert np.all(comp[outer] == F["comp_index"]["ecs"])
    assert [o is not None for o in sf["sreac_outer"]] == [True, False, False, False, True]


@pytest.mark.parametrize("sdiff", [False, True])
def test_calcium_conserved_across_the_membrane(sdiff):
    mesh, F, ora = _setup(sdiff=sdiff)
    S = F["spec_index"]
    total = _ca_total(F, ora)
    outer_tets = F["surf"]["tri_outer"]
    ca_out0 = int(ora.get_counts(S["Ca"])[np.unique(outer_tets)].sum())
    for k in range(1, 5):
        ora.run(k * 1.0e-3)
        assert _ca_total(F, ora) == total
    assert ora.surf_extent() > 0
    assert int(ora.get_counts(S["Ca"])[np.unique(outer_tets)].sum()) != ca_out0
