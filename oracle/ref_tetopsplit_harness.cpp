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
// seed and buffer (rng/create.cpp:44).
#include <cstdint>
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

namespace {

thread_local std::string g_err;

struct RefSim {
    std::unique_ptr<steps::model::Model> model;
    std::vector<steps::model::Spec*> specs;  // owned by the model
    std::unique_ptr<steps::tetmesh::Tetmesh> mesh;
    steps::tetmesh::TmComp* comp = nullptr;  // registered with (and unregistered from) mesh
    steps::rng::RNGptr rng;
    std::unique_ptr<steps::solver::API> solver;
    std::vector<std::string> spec_names;
    uint32_t ntets = 0;

    ~RefSim() {
        solver.reset();  // the solver refers to model, mesh and rng
        // The compartment unregisters itself from its mesh in its destructor, so it goes
        // while the mesh is whole (the base Geom destructor would reach it after the
        // Tetmesh part is gone).
        delete comp;
        mesh.reset();
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

}  // extern "C"
