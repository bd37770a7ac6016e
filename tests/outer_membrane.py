"""A membrane between two compartments whose surface reactions and GHK current reach both
volumes: the model and mesh of the merged-SSA-unit tests.

The reference keeps a patch triangle and both of its tets in one rank's SSA
(src/steps/mpi/tetopsplit/sreac.cpp:200-300); with reactants or products in the outer
volume every tet linked through such triangles belongs to one SSA unit.  The box is cut at
its middle plane x = nx h / 2 into an inner and an outer compartment; the patch is the
triangles between them.
"""
import numpy as np

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W


def outer_model(ghk=True, sdiff=False):
    """Species, rules and reactions are created in name order, the order the reference's
    model keeps them in (std::map by name), so that the drop-in built from the reference's
    own model objects sees the same tables as the Python solver."""
    mdl = smodel.Model()
    b = smodel.Spec("B", mdl)
    ca = smodel.Spec("Ca", mdl, valence=2)
    cab = smodel.Spec("CaB", mdl)
    p = smodel.Spec("P", mdl)
    pc = smodel.Spec("PCa", mdl)
    ch = smodel.Chan("CaCh", mdl)
    kc = smodel.ChanState("Kc", mdl, ch)
    ko = smodel.ChanState("Ko", mdl, ch)
    vi = smodel.Volsys("vin", mdl)
    smodel.Diff("dB_i", vi, b, 5.0e-13)
    smodel.Diff("dCa_i", vi, ca, 2.0e-12)
    smodel.Reac("bind", vi, lhs=[ca, b], rhs=[cab], kcst=5.0e7)
    smodel.Reac("unbind", vi, lhs=[cab], rhs=[ca, b], kcst=40.0)
    vo = smodel.Volsys("vout", mdl)
    smodel.Diff("dCa_o", vo, ca, 1.0e-12)
    ss = smodel.Surfsys("ssys", mdl)
    # Open channels let outer Ca in (reactant in the outer volume); channels open and close;
    # the pump binds inner Ca and releases it to the outer side.
    smodel.SReac("back", ss, olhs=[ca], slhs=[ko], srhs=[ko], irhs=[ca], kcst=2.0e7)
    smodel.SReac("close", ss, slhs=[ko], srhs=[kc], kcst=90.0)
    smodel.SReac("open", ss, slhs=[kc], srhs=[ko], kcst=120.0)
    smodel.SReac("pin", ss, ilhs=[ca], slhs=[p], srhs=[pc], kcst=1.0e8)
    smodel.SReac("pout", ss, slhs=[pc], srhs=[p], orhs=[ca], kcst=60.0)
    if sdiff:
        smodel.Diff("dP", ss, p, 1.0e-13)
    if ghk:
        g = smodel.GHKcurr("ICa", ss, ko, ca, computeflux=True, virtual_oconc=-1.0)
        g.setPInfo(g=20e-12, V=-0.065, T=293.15, oconc=2e-3, iconc=1e-4)
    return mdl


def outer_split(mesh):
    """Inner tets (barycentre x below the middle plane), outer tets, and the triangles
    between the two halves."""
    xmid = 0.5 * (mesh.verts[:, 0].min() + mesh.verts[:, 0].max())
    inner = np.nonzero(mesh.tet_bary[:, 0] < xmid)[0]
    outer = np.nonzero(mesh.tet_bary[:, 0] >= xmid)[0]
    side = np.zeros(mesh.ntets, dtype=np.int8)
    side[outer] = 1
    tt = mesh.tri_tets
    both = (tt[:, 0] >= 0) & (tt[:, 1] >= 0)
    iface = np.nonzero(both & (side[np.maximum(tt[:, 0], 0)] != side[np.maximum(tt[:, 1], 0)]))[0]
    return inner, outer, iface


def outer_mesh(nx=6, ny=4, nz=4, h=W.H, replicas=None):
    """The box with compartments cyto (inner half) and ecs (outer half) and the patch memb
    between them; with replicas = n, n disjoint copies as batched realizations
    (mesh.offsets)."""
    base = sgeom.kuhn_box(nx, ny, nz, h)
    inner, outer, iface = outer_split(base)
    mesh = base
    if replicas is not None:
        mesh = sgeom.replicate(base, replicas)
        T, M = base.ntets, base.ntris
        inner = np.concatenate([inner + r * T for r in range(replicas)])
        outer = np.concatenate([outer + r * T for r in range(replicas)])
        iface = np.concatenate([iface + r * M for r in range(replicas)])
    ci = sgeom.TmComp("cyto", mesh, inner)
    ci.addVolsys("vin")
    co = sgeom.TmComp("ecs", mesh, outer)
    co.addVolsys("vout")
    patch = sgeom.TmPatch("memb", mesh, iface, ci, co)
    patch.addSurfsys("ssys")
    return mesh


INITIAL = {"Ca_in": 2000, "B": 3000, "Ca_out": 5000, "P": 600, "Kc": 300}


def calcium_total(counts_ca, counts_cab, tri_pc, tri_unused=None):
    """Ca in both volumes, bound to the buffer and held by the pumps."""
    return int(counts_ca.sum()) + int(counts_cab.sum()) + int(tri_pc.sum())
