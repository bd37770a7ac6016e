"""Kinetic model description for the solver boundary.

Mirrors the pieces of the reference's model layer that the operator-split path
consumes (src/steps/model/: model.hpp:53 Model, spec.hpp Spec, volsys.hpp Volsys,
reac.hpp Reac, diff.hpp Diff, surfsys.hpp Surfsys, sreac.hpp SReac,
vdepsreac.hpp VDepSReac, chan.hpp Chan, chanstate.hpp ChanState,
ohmiccurr.hpp OhmicCurr).  Names and argument meanings follow the reference's
Python API_1 (``steps.model``).
"""
from __future__ import annotations

import math


class Model:
    def __init__(self):
        self.specs = {}        # name -> Spec (volume and surface species alike)
        self.volsys = {}
        self.surfsys = {}
        self.chans = {}

    def getSpec(self, name):
        return self.specs[name]

    def getAllSpecs(self):
        return list(self.specs.values())


class Spec:
    def __init__(self, id, model, valence=0):
        if id in model.specs:
            raise ValueError(f"duplicate species '{id}'")
        self.id = id
        self.model = model
        self.valence = valence
        model.specs[id] = self

    def getID(self):
        return self.id

    def setValence(self, v):
        self.valence = int(v)

    def getValence(self):
        return self.valence


class Chan:
    def __init__(self, id, model):
        self.id = id
        self.model = model
        self.states = []
        model.chans[id] = self


class ChanState(Spec):
    """A channel state is a surface species (src/steps/model/chanstate.hpp)."""

    def __init__(self, id, model, chan):
        super().__init__(id, model)
        self.chan = chan
        chan.states.append(self)


class Volsys:
    def __init__(self, id, model):
        self.id = id
        self.model = model
        self.reacs = {}
        self.diffs = {}
        model.volsys[id] = self


class Surfsys:
    def __init__(self, id, model):
        self.id = id
        self.model = model
        self.sreacs = {}
        self.vdepsreacs = {}
        self.ohmiccurrs = {}
        self.ghkcurrs = {}
        self.diffs = {}
        model.surfsys[id] = self


def _ids(specs):
    return [s.id if isinstance(s, Spec) else str(s) for s in (specs or [])]


class Reac:
    """Volume reaction lhs -> rhs with constant kcst (order 0: M/s, 1: /s, 2: /(M s), ...)."""

    def __init__(self, id, volsys, lhs=None, rhs=None, kcst=0.0):
        self.id = id
        self.volsys = volsys
        self.lhs = _ids(lhs)
        self.rhs = _ids(rhs)
        self.kcst = float(kcst)
        if len(self.lhs) > 4:
            raise ValueError("reaction order above 4 is not supported")
        volsys.reacs[id] = self

    def getOrder(self):
        return len(self.lhs)


class Diff:
    """Volume (or surface) diffusion of one ligand with constant dcst (m^2/s)."""

    def __init__(self, id, sys, lig, dcst=0.0):
        self.id = id
        self.sys = sys
        self.lig = lig.id if isinstance(lig, Spec) else str(lig)
        self.dcst = float(dcst)
        sys.diffs[id] = self


class SReac:
    """Surface reaction: ilhs/olhs are volume reactants on the inner/outer side,
    slhs surface reactants; irhs/orhs/srhs the products (src/steps/model/sreac.hpp)."""

    def __init__(self, id, surfsys, ilhs=None, olhs=None, slhs=None, irhs=None, orhs=None,
                 srhs=None, kcst=0.0):
        self.id = id
        self.surfsys = surfsys
        self.ilhs, self.olhs, self.slhs = _ids(ilhs), _ids(olhs), _ids(slhs)
        self.irhs, self.orhs, self.srhs = _ids(irhs), _ids(orhs), _ids(srhs)
        self.kcst = float(kcst)
        surfsys.sreacs[id] = self


class VDepSReac(SReac):
    """Surface reaction whose constant k(V) is a function of membrane potential (V, volts).
    Like the reference (API_2 model.py:4896-4898) k is tabulated over [vmin, vmax] in steps of
    dv and linearly interpolated."""

    def __init__(self, id, surfsys, ilhs=None, olhs=None, slhs=None, irhs=None, orhs=None,
                 srhs=None, k=None, vrange=(-150.0e-3, 100.0e-3, 1.0e-4)):
        super().__init__(id, surfsys, ilhs, olhs, slhs, irhs, orhs, srhs, 0.0)
        del surfsys.sreacs[id]
        if k is None:
            raise ValueError("VDepSReac needs k(V)")
        self.kfunc = k
        self.vrange = tuple(float(x) for x in vrange)
        surfsys.vdepsreacs[id] = self


FARADAY = 96485.3399       # src/steps/math/constants.hpp:49
GAS_CONSTANT = 8.314472    # constants.hpp:53
E_CHARGE = 1.602176487e-19 # constants.hpp:57


def ghk_permeability(g, v, z, temp, iconc, oconc):
    """Single-channel permeability (m^3/s) giving conductance g (S) at potential v (V),
    temperature temp (K), inner/outer concentrations (M): the slope of the GHK current
    equation (the quantity src/steps/math/ghk.cpp:36-69 computes)."""
    b, c = iconc * 1000.0, oconc * 1000.0
    d = -z * FARADAY / (GAS_CONSTANT * temp)
    den = c * math.exp(2.0 * d * v) + ((b - c) * d * v - c - b) * math.exp(d * v) + b
    num = math.exp(2.0 * d * v) - 2.0 * math.exp(d * v) + 1.0
    a = g * (num / den) if (abs(num) > 2.220446049250313e-16 or abs(den) > 2.220446049250313e-16) else 2.0 * g / (c + b)
    return (a * GAS_CONSTANT * temp) / (z * z * FARADAY * FARADAY)


class GHKcurr:
    """GHK current through channel state chanstate of ion (src/steps/model/ghkcurr.hpp):
    per channel I = P z F nu (c_in - c_out e^-nu) / (1 - e^-nu), nu = z (V + vshift) F / (R T).
    computeflux moves the ions (one per z e of charge); virtual_oconc (M) fixes the outer
    concentration, and a negative virtual_oconc (the default) takes it from the triangle's
    outer tet, between which and the inner tet the ions then move."""

    def __init__(self, id, surfsys, chanstate, ion, computeflux=True, virtual_oconc=-1.0, vshift=0.0):
        self.id = id
        self.surfsys = surfsys
        self.chanstate = chanstate.id if isinstance(chanstate, Spec) else str(chanstate)
        self.ion = ion.id if isinstance(ion, Spec) else str(ion)
        self.valence = ion.valence if isinstance(ion, Spec) else 0
        self.computeflux = bool(computeflux)
        self.voconc = float(virtual_oconc)
        self.vshift = float(vshift)
        self.perm = None
        surfsys.ghkcurrs[id] = self

    def setP(self, p):
        if not (p > 0.0):
            raise ValueError("permeability must be positive")
        self.perm = float(p)

    def getP(self):
        return self.perm

    def setPInfo(self, g, V, T, oconc, iconc):
        if self.valence == 0:
            raise ValueError("the ion has no valence")
        self.perm = ghk_permeability(g, V, self.valence, T, iconc, oconc)


class OhmicCurr:
    """Ohmic current g * n_open * (V - erev) through channel state chanstate (per channel g, S)."""

    def __init__(self, id, surfsys, chanstate, g, erev):
        self.id = id
        self.surfsys = surfsys
        self.chanstate = chanstate.id if isinstance(chanstate, Spec) else str(chanstate)
        self.g = float(g)
        self.erev = float(erev)
        surfsys.ohmiccurrs[id] = self
