// TetOpSplitB200: the reference's solver interface (steps::solver::API,
// src/steps/solver/api.hpp:58) implemented on the GPU solver of libsteps_b200.so.
//
// A STEPS build adds this class beside TetOpSplitP (src/steps/mpi/tetopsplit/
// tetopsplit.hpp:79) and binds it like _py_TetOpSplitP (pysteps/cysteps_mpi.pyx:74-80);
// the model, geometry and RNG objects are the reference's own.  The constructor
// flattens the reference Statedef (compartments, reactions, diffusion rules, patches,
// surface reactions, voltage-dependent reactions, ohmic currents) and the Tetmesh into
// the C ABI of include/steps_b200.h, then every API call below goes to the GPU.
//
// Per-tet geometry is derived here from the mesh vertices with the formulas of
// steps_b200/geom.py (face f opposite vertex f, volume |e1 . (e2 x e3)| / 6, face area
// |(b - a) x (c - a)| / 2, barycentre distances), so that the tables — and therefore the
// sample paths — equal those of the Python solver on the same mesh and model.
//
// Not bound through this class (they raise NotImplErr, as TetOpSplitP does for its own
// missing methods, TOS:1969-1973): diffusion boundaries, surface diffusion, GHK
// currents, outer-volume surface terms and the ~200 getters the reference also leaves to
// its base class.  Host lists (tet_hosts, tri_hosts, wm_hosts) are accepted and ignored:
// the mesh lives on one GPU.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "solver/api.hpp"

struct sg_solver;

namespace steps::b200 {

using namespace steps::solver;

class TetOpSplitB200: public solver::API {
  public:
    TetOpSplitB200(model::Model* m,
                   wm::Geom* g,
                   const rng::RNGptr& r,
                   int calcMembPot = EF_NONE,
                   std::vector<int> const& tet_hosts = {},
                   const std::map<triangle_global_id, int>& tri_hosts = {},
                   std::vector<int> const& wm_hosts = {});
    ~TetOpSplitB200() override;

    // ---- solver information (api.hpp:84-90) ----
    std::string getSolverName() const override;
    std::string getSolverDesc() const override;
    std::string getSolverAuthors() const override;
    std::string getSolverEmail() const override;

    // ---- simulation control (api.hpp:97-186) ----
    void checkpoint(std::string const& file_name) override;
    void restore(std::string const& file_name) override;
    void reset() override;
    void run(double endtime) override;
    void advance(double adv) override;
    void step() override;
    double getTime() const override;
    uint getNSteps() const override;
    void setTemp(double t) override;
    double getTemp() const override;
    void setEfieldDT(double efdt) override;
    double getEfieldDT() const override;

    // ---- batch recording (api.hpp:2014) ----
    void getBatchTetSpecCountsNP(const index_t* indices,
                                 size_t input_size,
                                 std::string const& s,
                                 double* counts,
                                 size_t output_size) const override;

    // The GPU solver handle (for callers that use the C ABI's extra controls).
    sg_solver* handle() const noexcept {
        return h_;
    }

  protected:
    // ---- compartments (api.hpp:2321-2370) ----
    double _getCompVol(comp_global_id cidx) const override;
    double _getCompSpecCount(comp_global_id cidx, spec_global_id sidx) const override;
    void _setCompSpecCount(comp_global_id cidx, spec_global_id sidx, double n) override;
    double _getCompSpecAmount(comp_global_id cidx, spec_global_id sidx) const override;
    void _setCompSpecAmount(comp_global_id cidx, spec_global_id sidx, double a) override;
    double _getCompSpecConc(comp_global_id cidx, spec_global_id sidx) const override;
    void _setCompSpecConc(comp_global_id cidx, spec_global_id sidx, double c) override;
    bool _getCompSpecClamped(comp_global_id cidx, spec_global_id sidx) const override;
    void _setCompSpecClamped(comp_global_id cidx, spec_global_id sidx, bool b) override;
    double _getCompReacK(comp_global_id cidx, reac_global_id ridx) const override;
    void _setCompReacK(comp_global_id cidx, reac_global_id ridx, double kf) override;
    bool _getCompReacActive(comp_global_id cidx, reac_global_id ridx) const override;
    void _setCompReacActive(comp_global_id cidx, reac_global_id ridx, bool a) override;

    // ---- patches (api.hpp:2631-2673) ----
    double _getPatchArea(patch_global_id pidx) const override;
    double _getPatchSpecCount(patch_global_id pidx, spec_global_id sidx) const override;
    void _setPatchSpecCount(patch_global_id pidx, spec_global_id sidx, double n) override;
    double _getPatchSpecAmount(patch_global_id pidx, spec_global_id sidx) const override;
    void _setPatchSpecAmount(patch_global_id pidx, spec_global_id sidx, double a) override;
    bool _getPatchSpecClamped(patch_global_id pidx, spec_global_id sidx) const override;
    void _setPatchSpecClamped(patch_global_id pidx, spec_global_id sidx, bool buf) override;
    double _getPatchSReacK(patch_global_id pidx, sreac_global_id sridx) const override;
    void _setPatchSReacK(patch_global_id pidx, sreac_global_id sridx, double kf) override;
    bool _getPatchSReacActive(patch_global_id pidx, sreac_global_id ridx) const override;
    void _setPatchSReacActive(patch_global_id pidx, sreac_global_id ridx, bool a) override;

    // ---- tetrahedrons (api.hpp:2570-2600) ----
    double _getTetVol(tetrahedron_global_id tidx) const override;
    double _getTetSpecCount(tetrahedron_global_id tidx, spec_global_id sidx) const override;
    void _setTetSpecCount(tetrahedron_global_id tidx, spec_global_id sidx, double n) override;
    double _getTetSpecAmount(tetrahedron_global_id tidx, spec_global_id sidx) const override;
    void _setTetSpecAmount(tetrahedron_global_id tidx, spec_global_id sidx, double m) override;
    double _getTetSpecConc(tetrahedron_global_id tidx, spec_global_id sidx) const override;
    void _setTetSpecConc(tetrahedron_global_id tidx, spec_global_id sidx, double c) override;
    void _setTetSpecClamped(tetrahedron_global_id tidx, spec_global_id sidx, bool buf) override;

    // ---- triangles (api.hpp:2790-2810) ----
    double _getTriArea(triangle_global_id tidx) const override;
    double _getTriSpecCount(triangle_global_id tidx, spec_global_id sidx) const override;
    void _setTriSpecCount(triangle_global_id tidx, spec_global_id sidx, double n) override;
    double _getTriV(triangle_global_id tidx) const override;
    double _getTriOhmicI(triangle_global_id tidx) const override;

    // ---- vertices and membranes (api.hpp:2870-2890) ----
    double _getVertV(vertex_id_t vidx) const override;
    void _setVertV(vertex_id_t vidx, double v) override;
    bool _getVertVClamped(vertex_id_t vidx) const override;
    void _setVertVClamped(vertex_id_t vidx, bool cl) override;
    void _setVertIClamp(vertex_id_t vidx, double i) override;
    void _setMembPotential(membrane_global_id midx, double v) override;
    void _setMembCapac(membrane_global_id midx, double cm) override;
    void _setMembVolRes(membrane_global_id midx, double ro) override;
    void _setMembRes(membrane_global_id midx, double ro, double vrev) override;

  private:
    void build_tables();
    void build_efield(int method);
    int memb_tri(triangle_global_id t) const;
    int surf_spec(spec_global_id s) const;

    sg_solver* h_ = nullptr;
    int efoption_ = EF_NONE;
    int nspec_ = 0;
    int ntets_ = 0;
    std::vector<double> tet_vol_;
    std::vector<int> tet_comp_;
    std::vector<double> comp_vol_;
    // Global reaction index -> ABI index per compartment, and whether it is active.
    std::map<std::pair<int, int>, int> reac_abi_;
    std::map<std::pair<int, int>, double> reac_k_;
    std::map<std::pair<int, int>, bool> reac_active_;
    std::vector<std::vector<uint32_t>> clamped_;  // [tet] species bits of clamped counts
    // Membrane triangles (the union of all patches with a surface system, sorted).
    std::vector<int> memb_tris_;
    std::map<int, int> memb_index_;
    std::vector<int> tri_patch_;
    std::vector<double> patch_area_;
    std::vector<int> vol_spec_;      // global species -> ABI volume species (-1: channel state)
    std::vector<int> sspec_global_;  // ABI surface species -> global species (sorted)
    std::vector<bool> vert_clamped_;
};

}  // namespace steps::b200
