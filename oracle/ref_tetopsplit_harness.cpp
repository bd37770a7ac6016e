// TEST INFRASTRUCTURE ONLY — a C-callable driver of the reference solvers, built from the
// reference's own sources (oracle/build_ref_tetopsplit.py) against project-written
// stand-ins for MPI, easylogging++, Boost and METIS (oracle/ref_shim/).  It lets the
// tests and bench.py's CPU legs run the unmodified reference TetOpSplitP
// (src/steps/mpi/tetopsplit/tetopsplit.cpp) as `mpirun -n 1` runs it, and Tetexact
// (src/steps/tetexact/tetexact.cpp) as the exact-SSA cross-check, on the same mesh, model
// and seed as the GPU solver.  Nothing in the product links it.
//
// Model: one compartment holding every tet of a mesh given as vertex and tet arrays
// (geom/tetmesh.hpp:151), one volume system with the given species, reactions
// (model/reac.hpp:62) and diffusion rules (model/diff.hpp:52); RNG "r123" with the given
// seed and buffer (rng/create.cpp:44).  Optionally (ref_create_memb) a membrane model
// instead: every surface triangle a patch with a two-state channel (C <-> O by tabulated
// voltage-dependent reactions, model/vdepsreac.hpp:63), an ohmic current through O
// (model/ohmiccurr.hpp:57) and one Memb (geom/memb.hpp:63).
//
// Built with STEPS_WITH_B200_API, kind 2 is the drop-in TetOpSplitB200
// (steps_b200/steps_api/tetopsplit_b200.hpp) on the same reference objects.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "geom/tetmesh.hpp"
#include "geom/tmcomp.hpp"
#include "model/diff.hpp"
#include "model/model.hpp"
#include "model/reac.hpp"
#include "model/spec.hpp"
#include "model/volsys.hpp"
#include "mpi/tetopsplit/tetopsplit.hpp"
#include "rng/create.hpp"
#include "rng/rng.hpp"
#include "solver/api.hpp"
#include "tetexact/tetexact.hpp"
#include "geom/memb.hpp"
#include "geom/tmpatch.hpp"
#include "model/chan.hpp"
#include "model/chanstate.hpp"
#include "model/ohmiccurr.hpp"
#include "model/surfsys.hpp"
#include "model/vdepsreac.hpp"
#include "model/sreac.hpp"
#ifdef STEPS_WITH_B200_API
#include "steps_api/tetopsplit_b200.hpp"
#endif

namespace {

thread_local std::string g_err;

struct RefSim {
    std::unique_ptr<steps::model::Model> model;
    std::vector<steps::model::Spec*> specs;  // owned by the model
    std::unique_ptr<steps::tetmesh::Tetmesh> mesh;
    steps::tetmesh::TmComp* comp = nullptr;  // registered with (and unregistered from) mesh
    steps::tetmesh::TmComp* comp2 = nullptr; // outer compartment of ref_create_outer
    steps::tetmesh::TmPatch* patch = nullptr;
    steps::tetmesh::Memb* memb = nullptr;  // owned by the mesh
    bool has_chans = false;
    steps::rng::RNGptr rng;
    std::unique_ptr<steps::solver::API> solver;
    std::vector<std::string> spec_names;
    uint32_t ntets = 0;

    ~RefSim() {
        solver.reset();  // the solver refers to model, mesh and rng
        // The compartment unregisters itself from its mesh in its destructor, so it goes
        // while the mesh is whole (the base Geom destructor would reach it after the
        // Tetmesh part is gone).
        // The mesh owns the membrane (Tetmesh::~Tetmesh deletes it); patch and compartment
        // unregister themselves from the mesh in their destructors, so they go first.
        delete patch;
        delete comp;
        delete comp2;
        mesh.reset();
        // A model with an ohmic current on a channel state is released, not deleted: its
        // destructor deletes the channel state before the current and then throws from the
        // current's destructor.  Test processes are short-lived.
        if (has_chans)
            (void)model.release();
        else
            model.reset();
    }
};

std::string sname(int i) {
    return "S" + std::to_string(i);
}

}  // namespace

extern "C" {

const char* ref_last_error() {
    return g_err.c_str();
}

// kind: 0 = TetOpSplitP, 1 = Tetexact.  verts [nverts][3] (m), tets [ntets][4] vertex ids.
// dcst [nspec] (m^2/s; 0 = no diffusion rule), lhs / rhs [nreac][nspec] stoichiometries,
// kcst [nreac] in the reference's units (M^(1-order)/s).
void* ref_create(int kind, int nverts, const double* verts, int ntets, const int64_t* tets, int nspec,
                 const double* dcst, int nreac, const uint32_t* lhs, const uint32_t* rhs, const double* kcst,
                 uint64_t seed, int rng_buf) {
    try {
        auto s = std::make_unique<RefSim>();
        s->model = std::make_unique<steps::model::Model>();
        auto& mdl = *s->model;
        auto* vsys = new steps::model::Volsys("vsys", mdl);
        for (int i = 0; i < nspec; ++i) {
            s->spec_names.push_back(sname(i));
            s->specs.push_back(new steps::model::Spec(sname(i), mdl));
        }
        for (int q = 0; q < nreac; ++q) {
            std::vector<steps::model::Spec*> l, r;
            for (int i = 0; i < nspec; ++i) {
                for (uint32_t k = 0; k < lhs[(size_t)q * nspec + i]; ++k) l.push_back(s->specs[i]);
                for (uint32_t k = 0; k < rhs[(size_t)q * nspec + i]; ++k) r.push_back(s->specs[i]);
            }
            new steps::model::Reac("R" + std::to_string(q), *vsys, l, r, kcst[q]);
        }
        for (int i = 0; i < nspec; ++i)
            if (dcst[i] > 0.0) new steps::model::Diff("D" + std::to_string(i), *vsys, *s->specs[i], dcst[i]);

        std::vector<double> v(verts, verts + (size_t)nverts * 3);
        std::vector<steps::index_t> t((size_t)ntets * 4);
        for (size_t k = 0; k < t.size(); ++k) t[k] = (steps::index_t)tets[k];
        s->mesh = std::make_unique<steps::tetmesh::Tetmesh>(v, t);
        std::vector<steps::index_t> all(ntets);
        for (int k = 0; k < ntets; ++k) all[k] = (steps::index_t)k;
        s->comp = new steps::tetmesh::TmComp("comp", *s->mesh, all);
        s->comp->addVolsys("vsys");
        s->ntets = (uint32_t)ntets;

        s->rng = steps::rng::create("r123", (uint)rng_buf);
        s->rng->initialize((unsigned long)seed);
        if (kind == 0) {
            std::vector<int> tet_hosts((size_t)ntets, 0);
            s->solver = std::make_unique<steps::mpi::tetopsplit::TetOpSplitP>(
                s->model.get(), s->mesh.get(), s->rng, steps::solver::API::EF_NONE, tet_hosts);
        } else if (kind == 2) {
#ifdef STEPS_WITH_B200_API
            s->solver = std::make_unique<steps::b200::TetOpSplitB200>(s->model.get(), s->mesh.get(), s->rng,
                                                                       steps::solver::API::EF_NONE);
#else
            g_err = "built without the TetOpSplitB200 drop-in";
            return nullptr;
#endif
        } else {
            s->solver = std::make_unique<steps::tetexact::Tetexact>(s->model.get(), s->mesh.get(), s->rng,
                                                                     steps::solver::API::EF_NONE);
        }
        return s.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_destroy(void* h) {
    delete static_cast<RefSim*>(h);
}

int ref_set_comp_count(void* h, int spec, double n) {
    try {
        auto* s = static_cast<RefSim*>(h);
        s->solver->setCompSpecCount("comp", s->spec_names.at(spec), n);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// counts [ntets] for one species (as setTetSpecCount per tet).
int ref_set_tet_counts(void* h, int spec, const double* counts) {
    try {
        auto* s = static_cast<RefSim*>(h);
        const std::string& nm = s->spec_names.at(spec);
        for (uint32_t t = 0; t < s->ntets; ++t)
            s->solver->setTetSpecCount(steps::tetrahedron_global_id(t), nm, counts[t]);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ref_get_tet_counts(void* h, int spec, double* out) {
    try {
        auto* s = static_cast<RefSim*>(h);
        std::vector<steps::index_t> idx(s->ntets);
        for (uint32_t t = 0; t < s->ntets; ++t) idx[t] = t;
        s->solver->getBatchTetSpecCountsNP(idx.data(), idx.size(), s->spec_names.at(spec), out, idx.size());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ref_get_comp_count(void* h, int spec, double* out) {
    try {
        auto* s = static_cast<RefSim*>(h);
        *out = s->solver->getCompSpecCount("comp", s->spec_names.at(spec));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ref_run(void* h, double t_end) {
    try {
        static_cast<RefSim*>(h)->solver->run(t_end);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

double ref_get_time(void* h) {
    return static_cast<RefSim*>(h)->solver->getTime();
}

// The split window length (TetOpSplitP only; 0 for Tetexact).
double ref_upd_period(void* h) {
    auto* s = static_cast<RefSim*>(h);
    auto* p = dynamic_cast<steps::mpi::tetopsplit::TetOpSplitP*>(s->solver.get());
    return p ? p->getUpdPeriod() : 0.0;
}

uint64_t ref_nsteps(void* h) {
    auto* s = static_cast<RefSim*>(h);
    auto* p = dynamic_cast<steps::mpi::tetopsplit::TetOpSplitP*>(s->solver.get());
    return p ? (uint64_t)p->getNIteration() : (uint64_t)s->solver->getNSteps();
}

// Membrane model (see the header comment); kind 0 = TetOpSplitP, 2 = TetOpSplitB200, with
// the EField solver option efopt (api.hpp:61; 0 = none).  k tables at vmin + i dv (V), of
// the length the reference requires, floor((vmax - vmin) / dv) + 1 (model/vdepsreac.cpp).
void* ref_create_memb(int kind, int nverts, const double* verts, int ntets, const int64_t* tets, int ntab,
                      const double* kopen, const double* kclose, double vmin, double vmax, double dv, double g,
                      double erev, uint64_t seed, int efopt) {
    try {
        auto s = std::make_unique<RefSim>();
        s->model = std::make_unique<steps::model::Model>();
        auto& mdl = *s->model;
        new steps::model::Volsys("vsys", mdl);
        auto* ss = new steps::model::Surfsys("ssys", mdl);
        auto* ch = new steps::model::Chan("Ch", mdl);
        auto* c = new steps::model::ChanState("C", mdl, *ch);
        auto* o = new steps::model::ChanState("O", mdl, *ch);
        const int need = (int)std::floor((vmax - vmin) / dv) + 1;
        if (ntab != need) {
            g_err = "k(V) tables need floor((vmax - vmin) / dv) + 1 = " + std::to_string(need) + " entries";
            return nullptr;
        }
        std::vector<double> ko(kopen, kopen + ntab), kc(kclose, kclose + ntab);
        new steps::model::VDepSReac("open", *ss, {}, {}, {c}, {}, {o}, {}, ko, vmin, vmax, dv, (uint)ntab);
        new steps::model::VDepSReac("close", *ss, {}, {}, {o}, {}, {c}, {}, kc, vmin, vmax, dv, (uint)ntab);
        new steps::model::OhmicCurr("I", *ss, *o, erev, g);
        s->has_chans = true;
        s->spec_names = {"C", "O"};
        std::vector<double> v(verts, verts + (size_t)nverts * 3);
        std::vector<steps::index_t> t((size_t)ntets * 4);
        for (size_t k = 0; k < t.size(); ++k) t[k] = (steps::index_t)tets[k];
        s->mesh = std::make_unique<steps::tetmesh::Tetmesh>(v, t);
        std::vector<steps::index_t> all(ntets);
        for (int k = 0; k < ntets; ++k) all[k] = (steps::index_t)k;
        s->comp = new steps::tetmesh::TmComp("cyto", *s->mesh, all);
        s->comp->addVolsys("vsys");
        std::vector<steps::index_t> surf;
        for (const auto& x : s->mesh->getSurfTris()) surf.push_back((steps::index_t)x);
        s->patch = new steps::tetmesh::TmPatch("memb", *s->mesh, surf, *s->comp);
        s->patch->addSurfsys("ssys");
        s->memb = new steps::tetmesh::Memb("membrane", *s->mesh, {s->patch}, {});
        s->ntets = (uint32_t)ntets;
        s->rng = steps::rng::create("r123", 512u);
        s->rng->initialize((unsigned long)seed);
        if (kind == 0) {
            std::vector<int> tet_hosts((size_t)ntets, 0);
            std::map<steps::triangle_global_id, int> tri_hosts;
            for (auto x : surf) tri_hosts[steps::triangle_global_id(x)] = 0;
            s->solver = std::make_unique<steps::mpi::tetopsplit::TetOpSplitP>(s->model.get(), s->mesh.get(), s->rng,
                                                                              efopt, tet_hosts, tri_hosts);
        } else {
#ifdef STEPS_WITH_B200_API
            s->solver = std::make_unique<steps::b200::TetOpSplitB200>(s->model.get(), s->mesh.get(), s->rng, efopt);
#else
            g_err = "built without the TetOpSplitB200 drop-in";
            return nullptr;
#endif
        }
        return s.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// A membrane between two compartments (kind 0 TetOpSplitP, 1 Tetexact, 2 the drop-in):
// tets with is_outer[t] = 0 form "cyto" (volume system vin: Ca and B diffuse, Ca + B <->
// CaB), the others "ecs" (vout: Ca diffuses); the patch "memb" (inner cyto, outer ecs) is
// every triangle between the two, with surface system ssys: pump P binds inner Ca (pin) and
// releases it to the outer side (pout); channel Kc <-> Ko (open, close); open channels let
// outer Ca in (back: outer-volume reactant, inner product).  Constants as given.
void* ref_create_outer(int kind, int nverts, const double* verts, int ntets, const int64_t* tets,
                       const int32_t* is_outer, const double* k, uint64_t seed) {
    try {
        auto s = std::make_unique<RefSim>();
        s->model = std::make_unique<steps::model::Model>();
        auto& mdl = *s->model;
        auto* ca = new steps::model::Spec("Ca", mdl, 2);
        auto* b = new steps::model::Spec("B", mdl);
        auto* cab = new steps::model::Spec("CaB", mdl);
        auto* p = new steps::model::Spec("P", mdl);
        auto* pc = new steps::model::Spec("PCa", mdl);
        auto* ch = new steps::model::Chan("CaCh", mdl);
        auto* kc = new steps::model::ChanState("Kc", mdl, *ch);
        auto* ko = new steps::model::ChanState("Ko", mdl, *ch);
        auto* vin = new steps::model::Volsys("vin", mdl);
        auto* vout = new steps::model::Volsys("vout", mdl);
        new steps::model::Diff("dCa_i", *vin, *ca, k[0]);
        new steps::model::Diff("dB_i", *vin, *b, k[1]);
        new steps::model::Reac("bind", *vin, {ca, b}, {cab}, k[2]);
        new steps::model::Reac("unbind", *vin, {cab}, {ca, b}, k[3]);
        new steps::model::Diff("dCa_o", *vout, *ca, k[4]);
        auto* ss = new steps::model::Surfsys("ssys", mdl);
        // SReac(id, surfsys, olhs, ilhs, slhs, irhs, srhs, orhs, kcst) (model/sreac.hpp:67)
        new steps::model::SReac("pin", *ss, {}, {ca}, {p}, {}, {pc}, {}, k[5]);
        new steps::model::SReac("pout", *ss, {}, {}, {pc}, {}, {p}, {ca}, k[6]);
        new steps::model::SReac("open", *ss, {}, {}, {kc}, {}, {ko}, {}, k[7]);
        new steps::model::SReac("close", *ss, {}, {}, {ko}, {}, {kc}, {}, k[8]);
        new steps::model::SReac("back", *ss, {ca}, {}, {ko}, {ca}, {ko}, {}, k[9]);
        s->has_chans = true;
        std::vector<double> v(verts, verts + (size_t)nverts * 3);
        std::vector<steps::index_t> t((size_t)ntets * 4);
        for (size_t q = 0; q < t.size(); ++q) t[q] = (steps::index_t)tets[q];
        s->mesh = std::make_unique<steps::tetmesh::Tetmesh>(v, t);
        std::vector<steps::index_t> in, out;
        for (int q = 0; q < ntets; ++q) (is_outer[q] ? out : in).push_back((steps::index_t)q);
        s->comp = new steps::tetmesh::TmComp("cyto", *s->mesh, in);
        s->comp->addVolsys("vin");
        s->comp2 = new steps::tetmesh::TmComp("ecs", *s->mesh, out);
        s->comp2->addVolsys("vout");
        std::vector<steps::index_t> iface;
        const auto ntris = s->mesh->countTris();
        for (steps::index_t m = 0; m < ntris; ++m) {
            const auto& tt = s->mesh->_getTriTetNeighb(steps::triangle_global_id(m));
            if (!tt[0].valid() || !tt[1].valid()) continue;
            if ((is_outer[tt[0].get()] != 0) != (is_outer[tt[1].get()] != 0)) iface.push_back(m);
        }
        s->patch = new steps::tetmesh::TmPatch("memb", *s->mesh, iface, *s->comp, s->comp2);
        s->patch->addSurfsys("ssys");
        s->ntets = (uint32_t)ntets;
        s->rng = steps::rng::create("r123", 512u);
        s->rng->initialize((unsigned long)seed);
        if (kind == 0) {
            std::vector<int> tet_hosts((size_t)ntets, 0);
            std::map<steps::triangle_global_id, int> tri_hosts;
            for (auto x : iface) tri_hosts[steps::triangle_global_id(x)] = 0;
            s->solver = std::make_unique<steps::mpi::tetopsplit::TetOpSplitP>(
                s->model.get(), s->mesh.get(), s->rng, steps::solver::API::EF_NONE, tet_hosts, tri_hosts);
        } else if (kind == 2) {
#ifdef STEPS_WITH_B200_API
            s->solver = std::make_unique<steps::b200::TetOpSplitB200>(s->model.get(), s->mesh.get(), s->rng,
                                                                       steps::solver::API::EF_NONE);
#else
            g_err = "built without the TetOpSplitB200 drop-in";
            return nullptr;
#endif
        } else {
            s->solver = std::make_unique<steps::tetexact::Tetexact>(s->model.get(), s->mesh.get(), s->rng,
                                                                     steps::solver::API::EF_NONE);
        }
        return s.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

#define REF_TRY(body)                 \
    try {                             \
        body;                         \
        return 0;                     \
    } catch (const std::exception& e) { \
        g_err = e.what();             \
        return 1;                     \
    }

int ref_surf_tris(void* h, int64_t* out, int cap, int* n) {
    REF_TRY({
        auto* s = static_cast<RefSim*>(h);
        auto st = s->mesh->getSurfTris();
        *n = (int)st.size();
        for (int i = 0; i < *n && i < cap; ++i) out[i] = (int64_t)st[i];
    })
}
int ref_tri_verts(void* h, int64_t tri, int64_t* out) {
    REF_TRY({
        auto v = static_cast<RefSim*>(h)->mesh->getTri(steps::triangle_global_id((steps::index_t)tri));
        for (int k = 0; k < 3; ++k) out[k] = (int64_t)v[k];
    })
}
int ref_get_tet_count(void* h, int64_t tet, const char* spec, double* out) {
    REF_TRY(*out = static_cast<RefSim*>(h)->solver->getTetSpecCount(
                steps::tetrahedron_global_id((steps::index_t)tet), spec))
}
int ref_set_tet_count(void* h, int64_t tet, const char* spec, double n) {
    REF_TRY(static_cast<RefSim*>(h)->solver->setTetSpecCount(steps::tetrahedron_global_id((steps::index_t)tet),
                                                               spec, n))
}
int ref_get_tri_count(void* h, int64_t tri, const char* spec, double* out) {
    REF_TRY(*out = static_cast<RefSim*>(h)->solver->getTriSpecCount(
                steps::triangle_global_id((steps::index_t)tri), spec))
}
int ref_set_tri_count(void* h, int64_t tri, const char* spec, double n) {
    REF_TRY(static_cast<RefSim*>(h)->solver->setTriSpecCount(steps::triangle_global_id((steps::index_t)tri), spec,
                                                               n))
}
int ref_get_comp_count_named(void* h, const char* comp, const char* spec, double* out) {
    REF_TRY(*out = static_cast<RefSim*>(h)->solver->getCompSpecCount(comp, spec))
}
int ref_set_comp_count_named(void* h, const char* comp, const char* spec, double n) {
    REF_TRY(static_cast<RefSim*>(h)->solver->setCompSpecCount(comp, spec, n))
}
int ref_get_patch_count(void* h, const char* spec, double* out) {
    REF_TRY(*out = static_cast<RefSim*>(h)->solver->getPatchSpecCount("memb", spec))
}
int ref_set_patch_count(void* h, const char* spec, double n) {
    REF_TRY(static_cast<RefSim*>(h)->solver->setPatchSpecCount("memb", spec, n))
}
int ref_get_vert_v(void* h, int64_t v, double* out) {
    REF_TRY(*out = static_cast<RefSim*>(h)->solver->getVertV(steps::vertex_id_t((steps::index_t)v)))
}
int ref_set_vert_v(void* h, int64_t v, double x) {
    REF_TRY(static_cast<RefSim*>(h)->solver->setVertV(steps::vertex_id_t((steps::index_t)v), x))
}
int ref_set_vert_iclamp(void* h, int64_t v, double i) {
    REF_TRY(static_cast<RefSim*>(h)->solver->setVertIClamp(steps::vertex_id_t((steps::index_t)v), i))
}
int ref_set_memb(void* h, double v0, double cm, double ra, double ro, double vrev, double efdt) {
    REF_TRY({
        auto* sv = static_cast<RefSim*>(h)->solver.get();
        sv->setMembPotential("membrane", v0);
        sv->setMembCapac("membrane", cm);
        sv->setMembVolRes("membrane", ra);
        sv->setMembRes("membrane", ro, vrev);
        sv->setEfieldDT(efdt);
    })
}
int ref_solver_name(void* h, char* out, int cap) {
    REF_TRY({
        std::string n = static_cast<RefSim*>(h)->solver->getSolverName();
        std::snprintf(out, (size_t)cap, "%s", n.c_str());
    })
}

}  // extern "C"
