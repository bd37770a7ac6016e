// TetOpSplitB200 (steps::solver::API on the GPU solver); see tetopsplit_b200.hpp.
#include "tetopsplit_b200.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "geom/memb.hpp"
#include "geom/tetmesh.hpp"
#include "geom/tmcomp.hpp"
#include "geom/tmpatch.hpp"
#include "model/chanstate.hpp"
#include "model/model.hpp"
#include "model/vdepsreac.hpp"
#include "rng/rng.hpp"
#include "solver/compdef.hpp"
#include "solver/diffdef.hpp"
#include "solver/ghkcurrdef.hpp"
#include "solver/ohmiccurrdef.hpp"
#include "solver/patchdef.hpp"
#include "solver/reacdef.hpp"
#include "solver/specdef.hpp"
#include "solver/sreacdef.hpp"
#include "solver/statedef.hpp"
#include "solver/vdepsreacdef.hpp"
#include "util/error.hpp"

#include "steps_b200.h"

namespace steps::b200 {

namespace {

const double kAvogadro = 6.02214179e23;  // math/constants.hpp:45

// C ABI status -> the reference's exception classes (util/error.hpp:161-234).
void check(int st) {
    if (st == SG_OK) return;
    std::string msg = sg_last_error();
    switch (st) {
        case SG_EARG: ArgErrLog(msg);
        case SG_ENOTIMPL: NotImplErrLog(msg);
        default: ProgErrLog(msg);
    }
}

using V3 = std::array<double, 3>;
V3 sub(const V3& a, const V3& b) {
    return {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
}
V3 cross(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double norm(const V3& a) {
    return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}

// Face f of a tet is the face opposite its vertex f.
const int kFaceVerts[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};

}  // namespace

TetOpSplitB200::TetOpSplitB200(model::Model* m,
                               wm::Geom* g,
                               const rng::RNGptr& r,
                               int calcMembPot,
                               std::vector<int> const& /*tet_hosts*/,
                               const std::map<triangle_global_id, int>& /*tri_hosts*/,
                               std::vector<int> const& /*wm_hosts*/)
    : API(*m, *g, r)
    , efoption_(calcMembPot) {
    if (rng() == nullptr) ArgErrLog("No RNG provided to solver initializer function");
    if (dynamic_cast<tetmesh::Tetmesh*>(&geom()) == nullptr)
        ArgErrLog("Geometry description to TetOpSplitB200 is not a valid tetmesh::Tetmesh object.");
    check(sg_create(&h_, (uint64_t)rng()->seed(), 0));
    try {
        build_tables();
        check(sg_setup(h_));
        if (efoption_ != EF_NONE) build_efield(0);
    } catch (...) {
        sg_destroy(h_);
        h_ = nullptr;
        throw;
    }
}

TetOpSplitB200::~TetOpSplitB200() {
    if (h_) sg_destroy(h_);
}

// Statedef x Tetmesh -> the C ABI tables (the role of TetOpSplitP::_setup, TOS:479-1088).
void TetOpSplitB200::build_tables() {
    auto& sd = statedef();
    auto* mesh = dynamic_cast<tetmesh::Tetmesh*>(&geom());
    // Volume species: every species of the model that is not a channel state.
    std::vector<int> gspec;
    for (uint s = 0; s < sd.countSpecs(); ++s) {
        auto& sp = model()._getSpec(spec_global_id(s));
        if (dynamic_cast<model::ChanState*>(&sp) == nullptr) gspec.push_back((int)s);
    }
    std::vector<int> vol_of(sd.countSpecs(), -1);
    for (size_t i = 0; i < gspec.size(); ++i) vol_of[gspec[i]] = (int)i;
    if (gspec.empty()) gspec.push_back(-1);  // membrane-only model: one inert species
    nspec_ = (int)gspec.size();
    check(sg_set_nspecs(h_, nspec_));
    vol_spec_ = vol_of;

    // Per-tet geometry from the vertices (formulas of steps_b200/geom.py).
    ntets_ = (int)mesh->countTets();
    const int T = ntets_;
    std::vector<V3> bary(T);
    std::vector<double> area(4 * (size_t)T), dist(4 * (size_t)T, 0.0);
    std::vector<int32_t> neighb(4 * (size_t)T, -1);
    tet_vol_.assign(T, 0.0);
    std::map<std::array<uint32_t, 3>, std::pair<int, int>> faces;
    for (int t = 0; t < T; ++t) {
        const auto& tv = mesh->_getTet(tetrahedron_global_id(t));
        V3 p[4];
        for (int k = 0; k < 4; ++k) {
            const auto& q = mesh->_getVertex(tv[k]);
            p[k] = {q[0], q[1], q[2]};
        }
        const V3 e1 = sub(p[1], p[0]), e2 = sub(p[2], p[0]), e3 = sub(p[3], p[0]);
        const V3 c = cross(e2, e3);
        tet_vol_[t] = std::fabs(e1[0] * c[0] + e1[1] * c[1] + e1[2] * c[2]) / 6.0;
        for (int k = 0; k < 3; ++k) bary[t][k] = (((p[0][k] + p[1][k]) + p[2][k]) + p[3][k]) / 4.0;
        for (int f = 0; f < 4; ++f) {
            const V3& a = p[kFaceVerts[f][0]];
            const V3& b = p[kFaceVerts[f][1]];
            const V3& cc = p[kFaceVerts[f][2]];
            area[(size_t)t * 4 + f] = 0.5 * norm(cross(sub(b, a), sub(cc, a)));
            std::array<uint32_t, 3> key = {(uint32_t)tv[kFaceVerts[f][0]].get(), (uint32_t)tv[kFaceVerts[f][1]].get(),
                                           (uint32_t)tv[kFaceVerts[f][2]].get()};
            std::sort(key.begin(), key.end());
            auto it = faces.find(key);
            if (it == faces.end()) {
                faces.emplace(key, std::make_pair(t, f));
            } else {
                const int t2 = it->second.first, f2 = it->second.second;
                if (neighb[(size_t)t2 * 4 + f2] >= 0) ArgErrLog("a face is shared by more than two tetrahedra");
                neighb[(size_t)t * 4 + f] = t2;
                neighb[(size_t)t2 * 4 + f2] = t;
            }
        }
    }
    for (int t = 0; t < T; ++t)
        for (int f = 0; f < 4; ++f) {
            const int n = neighb[(size_t)t * 4 + f];
            if (n >= 0) dist[(size_t)t * 4 + f] = norm(sub(bary[n], bary[t]));
        }

    // Compartments in Statedef order; each tet belongs to at most one.
    const int C = (int)sd.countComps();
    tet_comp_.assign(T, -1);
    comp_vol_.assign(C, 0.0);
    for (int c = 0; c < C; ++c) {
        auto& cd = sd.compdef(comp_global_id(c));
        auto* tc = dynamic_cast<tetmesh::TmComp*>(&geom().getComp(cd.name()));
        if (tc == nullptr) ArgErrLog("compartment " + cd.name() + " is not a mesh compartment");
        for (const auto& t : tc->_getAllTetIndices()) {
            tet_comp_[t.get()] = c;
            comp_vol_[c] += tet_vol_[t.get()];
        }
    }
    std::vector<int32_t> tcomp(tet_comp_.begin(), tet_comp_.end());
    check(sg_set_mesh(h_, T, tet_vol_.data(), neighb.data(), area.data(), dist.data(), tcomp.data(),
                      std::max(C, 1)));

    // Reactions and diffusion rules per compartment, in the compartment's local order.
    const int S = nspec_;
    for (int c = 0; c < C; ++c) {
        auto& cd = sd.compdef(comp_global_id(c));
        for (uint l = 0; l < cd.countReacs(); ++l) {
            const auto rg = cd.reacL2G(reac_local_id(l));
            auto& rd = sd.reacdef(rg);
            std::vector<uint32_t> lhs(S, 0);
            std::vector<int32_t> upd(S, 0);
            for (uint s = 0; s < sd.countSpecs(); ++s) {
                const int v = vol_of[s];
                const uint ls = rd.lhs(spec_global_id(s));
                const int us = rd.upd(spec_global_id(s));
                if ((ls || us) && v < 0) ArgErrLog("reaction " + rd.name() + " involves a channel state");
                if (v >= 0) {
                    lhs[v] = ls;
                    upd[v] = us;
                }
            }
            int32_t idx = 0;
            check(sg_add_reac(h_, c, lhs.data(), upd.data(), rd.kcst(), &idx));
            reac_abi_[{c, (int)rg.get()}] = idx;
            reac_k_[{c, (int)rg.get()}] = rd.kcst();
            reac_active_[{c, (int)rg.get()}] = true;
        }
        for (uint l = 0; l < cd.countDiffs(); ++l) {
            auto& dd = sd.diffdef(cd.diffL2G(diff_local_id(l)));
            const int v = vol_of[dd.lig().get()];
            if (v < 0) ArgErrLog("diffusion of a channel state");
            int32_t idx = 0;
            check(sg_add_diff(h_, c, v, dd.dcst(), &idx));
        }
    }

    // Membrane triangles: the union of the patches with surface reactions or currents.
    const int P = (int)sd.countPatches();
    patch_area_.assign(P, 0.0);
    std::set<int> tris;
    std::vector<std::vector<int>> ptris(P);
    std::set<int> sspecs;
    for (int p = 0; p < P; ++p) {
        auto& pd = sd.patchdef(patch_global_id(p));
        auto* tp = dynamic_cast<tetmesh::TmPatch*>(&geom().getPatch(pd.name()));
        if (tp == nullptr) ArgErrLog("patch " + pd.name() + " is not a mesh patch");
        for (const auto& t : tp->_getAllTriIndices()) {
            ptris[p].push_back((int)t.get());
            patch_area_[p] += mesh->getTriArea(t);
        }
        if (pd.countSReacs() + pd.countVDepSReacs() + pd.countOhmicCurrs() + pd.countGHKcurrs() == 0) continue;
        if (pd.countSurfDiffs() > 0) NotImplErrLog("surface diffusion through TetOpSplitB200");
        for (int t : ptris[p]) tris.insert(t);
        for (uint l = 0; l < pd.countSpecs(); ++l) sspecs.insert((int)pd.specL2G(spec_local_id(l)).get());
    }
    if (tris.empty()) return;
    sspec_global_.assign(sspecs.begin(), sspecs.end());
    memb_tris_.assign(tris.begin(), tris.end());
    const int M = (int)memb_tris_.size();
    for (int i = 0; i < M; ++i) memb_index_[memb_tris_[i]] = i;
    tri_patch_.assign(M, -1);
    std::vector<int32_t> inner(M, -1), outer(M, -1), tpatch(M, -1);
    std::vector<double> tarea(M, 0.0);
    bool any_outer = false;
    for (int p = 0; p < P; ++p) {
        auto& pd = sd.patchdef(patch_global_id(p));
        if (pd.countSReacs() + pd.countVDepSReacs() + pd.countOhmicCurrs() + pd.countGHKcurrs() == 0) continue;
        auto& pt = geom().getPatch(pd.name());
        int ic = -1, oc = -2;
        for (int c = 0; c < C; ++c) {
            if (sd.compdef(comp_global_id(c)).name() == pt.getIComp().getID()) ic = c;
            if (pt.getOComp() != nullptr && sd.compdef(comp_global_id(c)).name() == pt.getOComp()->getID()) oc = c;
        }
        for (int t : ptris[p]) {
            const int m = memb_index_[t];
            if (tpatch[m] >= 0) ArgErrLog("a triangle belongs to two patches");
            tpatch[m] = p;
            const auto& tt = mesh->_getTriTetNeighb(triangle_global_id(t));
            int in = -1;
            for (const auto& x : tt)
                if (x.valid() && tet_comp_[x.get()] == ic) in = (int)x.get();
            if (in < 0) ArgErrLog("a patch triangle has no tet in the patch's inner compartment");
            inner[m] = in;
            // Tri::oTet: the other tet, when it lies in the patch's outer compartment.
            for (const auto& x : tt)
                if (x.valid() && (int)x.get() != in && tet_comp_[x.get()] == oc) {
                    outer[m] = (int)x.get();
                    any_outer = true;
                }
            tarea[m] = mesh->getTriArea(triangle_global_id(t));
        }
    }
    tri_patch_.assign(tpatch.begin(), tpatch.end());
    const int SS = (int)sspec_global_.size();
    check(sg_set_surface(h_, SS, M, inner.data(), tpatch.data(), tarea.data(), P));
    if (any_outer) check(sg_set_tri_outer(h_, outer.data()));
    std::vector<uint32_t> ol;
    std::vector<int32_t> ou;
    bool has_outer = false;
    auto rows = [&](auto& r, std::vector<uint32_t>& sl, std::vector<uint32_t>& il, std::vector<int32_t>& su,
                    std::vector<int32_t>& iu) {
        sl.assign(SS, 0);
        su.assign(SS, 0);
        il.assign(S, 0);
        iu.assign(S, 0);
        ol.assign(S, 0);
        ou.assign(S, 0);
        has_outer = false;
        for (uint s = 0; s < sd.countSpecs(); ++s) {
            const spec_global_id g(s);
            if (r.lhs_O(g) || r.upd_O(g)) {
                const int v = vol_of[s];
                if (v < 0) ArgErrLog("outer-volume term on a channel state");
                ol[v] = r.lhs_O(g);
                ou[v] = r.upd_O(g);
                has_outer = true;
            }
            if (r.lhs_S(g) || r.upd_S(g)) {
                const int k = surf_spec(g);
                sl[k] = r.lhs_S(g);
                su[k] = r.upd_S(g);
            }
            if (r.lhs_I(g) || r.upd_I(g)) {
                const int v = vol_of[s];
                if (v < 0) ArgErrLog("inner-volume term on a channel state");
                il[v] = r.lhs_I(g);
                iu[v] = r.upd_I(g);
            }
        }
    };
    for (int p = 0; p < P; ++p) {
        auto& pd = sd.patchdef(patch_global_id(p));
        std::vector<uint32_t> sl, il;
        std::vector<int32_t> su, iu;
        for (uint l = 0; l < pd.countSReacs(); ++l) {
            auto& r = sd.sreacdef(pd.sreacL2G(sreac_local_id(l)));
            rows(r, sl, il, su, iu);
            int32_t idx = 0;
            check(sg_add_sreac(h_, p, sl.data(), il.data(), su.data(), iu.data(), r.kcst(), &idx));
            if (has_outer) check(sg_set_sreac_outer(h_, idx, ol.data(), ou.data()));
        }
        for (uint l = 0; l < pd.countVDepSReacs(); ++l) {
            const auto g = pd.vdepsreacL2G(vdepsreac_local_id(l));
            auto& r = sd.vdepsreacdef(g);
            rows(r, sl, il, su, iu);
            auto& mv = model()._getVDepSReac(g);
            const auto& tab = mv._getK();
            int32_t idx = 0;
            check(sg_add_vdep_sreac(h_, p, sl.data(), il.data(), su.data(), iu.data(), mv._getVMin(), mv._getDV(),
                                    (int32_t)tab.size(), tab.data(), &idx));
            if (has_outer) check(sg_set_sreac_outer(h_, idx, ol.data(), ou.data()));
        }
        for (uint l = 0; l < pd.countOhmicCurrs(); ++l) {
            auto& oc = sd.ohmiccurrdef(pd.ohmiccurrL2G(ohmiccurr_local_id(l)));
            int32_t idx = 0;
            check(sg_add_ohmic(h_, p, surf_spec(oc.chanstate()), oc.getG(), oc.getERev(), &idx));
        }
        // GHKcurr (ghkcurr.cpp:168-280): voconc < 0 reads the triangle's outer tet.
        for (uint l = 0; l < pd.countGHKcurrs(); ++l) {
            auto& gd = pd.ghkcurrdef(ghkcurr_local_id(l));
            const int v = vol_of[gd.ion().get()];
            if (v < 0) ArgErrLog("GHK current of a channel state");
            int32_t idx = 0;
            check(sg_add_ghk(h_, p, surf_spec(gd.chanstate()), v, gd.valence(), gd.perm(), gd.vshift(), gd.voconc(),
                             gd.realflux() ? 1 : 0, &idx));
        }
    }
}

int TetOpSplitB200::surf_spec(spec_global_id s) const {
    auto it = std::lower_bound(sspec_global_.begin(), sspec_global_.end(), (int)s.get());
    if (it == sspec_global_.end() || *it != (int)s.get())
        ArgErrLog("species " + statedef().specdef(s).name() + " is not on a membrane patch");
    return (int)(it - sspec_global_.begin());
}

int TetOpSplitB200::memb_tri(triangle_global_id t) const {
    auto it = memb_index_.find((int)t.get());
    if (it == memb_index_.end()) ArgErrLog("triangle " + std::to_string(t.get()) + " is not a membrane triangle");
    return it->second;
}

// EField on the one membrane of the mesh (TOS:1092-1279 _setupEField).
void TetOpSplitB200::build_efield(int method) {
    auto* mesh = dynamic_cast<tetmesh::Tetmesh*>(&geom());
    if (mesh->_countMembs() != 1) ArgErrLog("the membrane potential needs exactly one Memb on the mesh");
    auto* memb = mesh->_getMemb(0);
    const auto& mt = memb->_getAllTriIndices();
    if (memb_tris_.size() != mt.size()) ArgErrLog("the membrane must consist of exactly the patches with surface systems");
    std::vector<int32_t> tri_verts;
    for (int t : memb_tris_) {
        const auto& v = mesh->_getTri(triangle_global_id(t));
        for (int k = 0; k < 3; ++k) tri_verts.push_back((int32_t)v[k].get());
    }
    const int NV = (int)mesh->countVertices();
    std::vector<double> verts(3 * (size_t)NV);
    for (int v = 0; v < NV; ++v) {
        const auto& q = mesh->_getVertex(vertex_id_t(v));
        for (int k = 0; k < 3; ++k) verts[(size_t)v * 3 + k] = q[k];
    }
    std::vector<int32_t> tv(4 * (size_t)ntets_);
    for (int t = 0; t < ntets_; ++t) {
        const auto& x = mesh->_getTet(tetrahedron_global_id(t));
        for (int k = 0; k < 4; ++k) tv[(size_t)t * 4 + k] = (int32_t)x[k].get();
    }
    vert_clamped_.assign(NV, false);
    check(sg_set_efield_mesh(h_, NV, verts.data(), tv.data(), (int32_t)memb_tris_.size(), tri_verts.data(), method));
}

// ---- information ----
std::string TetOpSplitB200::getSolverName() const {
    return "TetOpSplitB200";
}
std::string TetOpSplitB200::getSolverDesc() const {
    return "Operator-split spatial SSA on one GPU (per-tet SSA, binomial diffusion, PCG EField)";
}
std::string TetOpSplitB200::getSolverAuthors() const {
    return "steps-b200";
}
std::string TetOpSplitB200::getSolverEmail() const {
    return "";
}

// ---- control ----
void TetOpSplitB200::checkpoint(std::string const& file_name) {
    check(sg_checkpoint(h_, file_name.c_str()));
}
void TetOpSplitB200::restore(std::string const& file_name) {
    check(sg_restore(h_, file_name.c_str()));
}
void TetOpSplitB200::reset() {
    check(sg_reset(h_));
}
void TetOpSplitB200::run(double endtime) {
    check(sg_run(h_, endtime));
}
void TetOpSplitB200::advance(double adv) {
    check(sg_advance(h_, adv));
}
void TetOpSplitB200::step() {
    NotImplErrLog("step() is not available in an operator-split solver");
}
double TetOpSplitB200::getTime() const {
    double t = 0.0;
    check(sg_get_time(h_, &t));
    return t;
}
uint TetOpSplitB200::getNSteps() const {
    uint64_t n = 0;
    check(sg_get_nsteps(h_, &n));
    return (uint)n;
}
void TetOpSplitB200::setTemp(double t) {
    check(sg_set_temp(h_, t));
}
double TetOpSplitB200::getTemp() const {
    double t = 0.0;
    check(sg_get_temp(h_, &t));
    return t;
}
void TetOpSplitB200::setEfieldDT(double efdt) {
    check(sg_set_efield_dt(h_, efdt));
}
double TetOpSplitB200::getEfieldDT() const {
    double dt = 0.0;
    check(sg_get_efield_dt(h_, &dt));
    return dt;
}

void TetOpSplitB200::getBatchTetSpecCountsNP(const index_t* indices,
                                             size_t input_size,
                                             std::string const& s,
                                             double* counts,
                                             size_t output_size) const {
    if (input_size != output_size) ArgErrLog("Length of indices and counts must be the same.");
    const int v = vol_spec_.at(statedef().getSpecIdx(s).get());
    if (v < 0) ArgErrLog("species " + s + " is a channel state");
    std::vector<int32_t> idx(indices, indices + input_size);
    check(sg_get_batch_tet_counts(h_, v, idx.data(), (int32_t)idx.size(), counts));
}

// ---- compartments ----
double TetOpSplitB200::_getCompVol(comp_global_id cidx) const {
    return comp_vol_.at(cidx.get());
}
double TetOpSplitB200::_getCompSpecCount(comp_global_id cidx, spec_global_id sidx) const {
    double n = 0.0;
    check(sg_get_comp_count(h_, (int)cidx.get(), vol_spec_.at(sidx.get()), -1, &n));
    return n;
}
void TetOpSplitB200::_setCompSpecCount(comp_global_id cidx, spec_global_id sidx, double n) {
    check(sg_set_comp_count(h_, (int)cidx.get(), vol_spec_.at(sidx.get()), -1, n));
}
double TetOpSplitB200::_getCompSpecAmount(comp_global_id cidx, spec_global_id sidx) const {
    return _getCompSpecCount(cidx, sidx) / kAvogadro;
}
void TetOpSplitB200::_setCompSpecAmount(comp_global_id cidx, spec_global_id sidx, double a) {
    _setCompSpecCount(cidx, sidx, a * kAvogadro);
}
double TetOpSplitB200::_getCompSpecConc(comp_global_id cidx, spec_global_id sidx) const {
    return _getCompSpecCount(cidx, sidx) / (1.0e3 * _getCompVol(cidx) * kAvogadro);
}
void TetOpSplitB200::_setCompSpecConc(comp_global_id cidx, spec_global_id sidx, double c) {
    _setCompSpecCount(cidx, sidx, c * 1.0e3 * _getCompVol(cidx) * kAvogadro);
}
bool TetOpSplitB200::_getCompSpecClamped(comp_global_id, spec_global_id) const {
    NotImplErrLog("getCompSpecClamped");
}
void TetOpSplitB200::_setCompSpecClamped(comp_global_id cidx, spec_global_id sidx, bool b) {
    const int v = vol_spec_.at(sidx.get());
    for (int t = 0; t < ntets_; ++t)
        if (tet_comp_[t] == (int)cidx.get()) check(sg_set_tet_clamped(h_, t, v, b ? 1 : 0));
}
double TetOpSplitB200::_getCompReacK(comp_global_id cidx, reac_global_id ridx) const {
    return reac_k_.at({(int)cidx.get(), (int)ridx.get()});
}
void TetOpSplitB200::_setCompReacK(comp_global_id cidx, reac_global_id ridx, double kf) {
    const std::pair<int, int> key{(int)cidx.get(), (int)ridx.get()};
    reac_k_.at(key) = kf;
    if (reac_active_.at(key)) check(sg_set_reac_k(h_, reac_abi_.at(key), -1, kf));
}
bool TetOpSplitB200::_getCompReacActive(comp_global_id cidx, reac_global_id ridx) const {
    return reac_active_.at({(int)cidx.get(), (int)ridx.get()});
}
// An inactive reaction runs with constant 0 (its propensity vanishes), as TetOpSplitP's
// inactive kprocs report rate 0.
void TetOpSplitB200::_setCompReacActive(comp_global_id cidx, reac_global_id ridx, bool a) {
    const std::pair<int, int> key{(int)cidx.get(), (int)ridx.get()};
    reac_active_.at(key) = a;
    check(sg_set_reac_k(h_, reac_abi_.at(key), -1, a ? reac_k_.at(key) : 0.0));
}

// ---- patches ----
double TetOpSplitB200::_getPatchArea(patch_global_id pidx) const {
    return patch_area_.at(pidx.get());
}
double TetOpSplitB200::_getPatchSpecCount(patch_global_id pidx, spec_global_id sidx) const {
    double n = 0.0;
    check(sg_get_patch_count(h_, (int)pidx.get(), surf_spec(sidx), -1, &n));
    return n;
}
void TetOpSplitB200::_setPatchSpecCount(patch_global_id pidx, spec_global_id sidx, double n) {
    check(sg_set_patch_count(h_, (int)pidx.get(), surf_spec(sidx), -1, n));
}
double TetOpSplitB200::_getPatchSpecAmount(patch_global_id pidx, spec_global_id sidx) const {
    return _getPatchSpecCount(pidx, sidx) / kAvogadro;
}
void TetOpSplitB200::_setPatchSpecAmount(patch_global_id pidx, spec_global_id sidx, double a) {
    _setPatchSpecCount(pidx, sidx, a * kAvogadro);
}
bool TetOpSplitB200::_getPatchSpecClamped(patch_global_id, spec_global_id) const {
    NotImplErrLog("getPatchSpecClamped");
}
void TetOpSplitB200::_setPatchSpecClamped(patch_global_id, spec_global_id, bool) {
    NotImplErrLog("setPatchSpecClamped");
}
double TetOpSplitB200::_getPatchSReacK(patch_global_id, sreac_global_id) const {
    NotImplErrLog("getPatchSReacK");
}
void TetOpSplitB200::_setPatchSReacK(patch_global_id, sreac_global_id, double) {
    NotImplErrLog("setPatchSReacK");
}
bool TetOpSplitB200::_getPatchSReacActive(patch_global_id, sreac_global_id) const {
    NotImplErrLog("getPatchSReacActive");
}
void TetOpSplitB200::_setPatchSReacActive(patch_global_id, sreac_global_id, bool) {
    NotImplErrLog("setPatchSReacActive");
}

// ---- tetrahedrons ----
double TetOpSplitB200::_getTetVol(tetrahedron_global_id tidx) const {
    return tet_vol_.at(tidx.get());
}
double TetOpSplitB200::_getTetSpecCount(tetrahedron_global_id tidx, spec_global_id sidx) const {
    double n = 0.0;
    check(sg_get_tet_count(h_, (int)tidx.get(), vol_spec_.at(sidx.get()), &n));
    return n;
}
void TetOpSplitB200::_setTetSpecCount(tetrahedron_global_id tidx, spec_global_id sidx, double n) {
    check(sg_set_tet_count(h_, (int)tidx.get(), vol_spec_.at(sidx.get()), n));
}
double TetOpSplitB200::_getTetSpecAmount(tetrahedron_global_id tidx, spec_global_id sidx) const {
    return _getTetSpecCount(tidx, sidx) / kAvogadro;
}
void TetOpSplitB200::_setTetSpecAmount(tetrahedron_global_id tidx, spec_global_id sidx, double m) {
    _setTetSpecCount(tidx, sidx, m * kAvogadro);
}
double TetOpSplitB200::_getTetSpecConc(tetrahedron_global_id tidx, spec_global_id sidx) const {
    return _getTetSpecCount(tidx, sidx) / (1.0e3 * _getTetVol(tidx) * kAvogadro);
}
void TetOpSplitB200::_setTetSpecConc(tetrahedron_global_id tidx, spec_global_id sidx, double c) {
    _setTetSpecCount(tidx, sidx, c * 1.0e3 * _getTetVol(tidx) * kAvogadro);
}
void TetOpSplitB200::_setTetSpecClamped(tetrahedron_global_id tidx, spec_global_id sidx, bool buf) {
    check(sg_set_tet_clamped(h_, (int)tidx.get(), vol_spec_.at(sidx.get()), buf ? 1 : 0));
}

// ---- triangles ----
double TetOpSplitB200::_getTriArea(triangle_global_id tidx) const {
    return dynamic_cast<tetmesh::Tetmesh&>(geom()).getTriArea(tidx);
}
double TetOpSplitB200::_getTriSpecCount(triangle_global_id tidx, spec_global_id sidx) const {
    double n = 0.0;
    check(sg_get_tri_count(h_, memb_tri(tidx), surf_spec(sidx), &n));
    return n;
}
void TetOpSplitB200::_setTriSpecCount(triangle_global_id tidx, spec_global_id sidx, double n) {
    check(sg_set_tri_count(h_, memb_tri(tidx), surf_spec(sidx), n));
}
double TetOpSplitB200::_getTriV(triangle_global_id tidx) const {
    double v = 0.0;
    check(sg_get_tri_v(h_, memb_tri(tidx), &v));
    return v;
}
double TetOpSplitB200::_getTriOhmicI(triangle_global_id tidx) const {
    double a = 0.0;
    check(sg_get_tri_ohmic_i(h_, memb_tri(tidx), &a));
    return a;
}

// ---- vertices and membranes ----
double TetOpSplitB200::_getVertV(vertex_id_t vidx) const {
    double v = 0.0;
    check(sg_get_vert_v(h_, (int)vidx.get(), &v));
    return v;
}
void TetOpSplitB200::_setVertV(vertex_id_t vidx, double v) {
    check(sg_set_vert_v(h_, (int)vidx.get(), v));
}
bool TetOpSplitB200::_getVertVClamped(vertex_id_t vidx) const {
    if (efoption_ == EF_NONE) ProgErrLog("Method not available: this solver has no membrane potential");
    return vert_clamped_.at(vidx.get());
}
void TetOpSplitB200::_setVertVClamped(vertex_id_t vidx, bool cl) {
    check(sg_set_vert_v_clamped(h_, (int)vidx.get(), cl ? 1 : 0));
    vert_clamped_.at(vidx.get()) = cl;
}
void TetOpSplitB200::_setVertIClamp(vertex_id_t vidx, double i) {
    check(sg_set_vert_iclamp(h_, (int)vidx.get(), i));
}
void TetOpSplitB200::_setMembPotential(membrane_global_id, double v) {
    check(sg_set_memb_potential(h_, v));
}
void TetOpSplitB200::_setMembCapac(membrane_global_id, double cm) {
    check(sg_set_memb_capac(h_, cm));
}
void TetOpSplitB200::_setMembVolRes(membrane_global_id, double ro) {
    check(sg_set_memb_vol_res(h_, ro));
}
void TetOpSplitB200::_setMembRes(membrane_global_id, double ro, double vrev) {
    check(sg_set_memb_res(h_, ro, vrev));
}

}  // namespace steps::b200
