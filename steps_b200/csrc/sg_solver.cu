// Host side of the B200 operator-split solver: owns the device state, flattens the
// model x mesh tables, runs the split-window loop and implements the
// get/set entry points of the reference solver API behind a C ABI.
//
// Replaces the implementation of steps::mpi::tetopsplit::TetOpSplitP
// (src/steps/mpi/tetopsplit/tetopsplit.hpp:79, tetopsplit.cpp "TOS").
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "sg_rng.cuh"
#include "sg_types.h"
#include "sg_window.cuh"
#include "sg_errors.h"
#include "sg_efield.h"
#include "../../include/steps_b200.h"

namespace sg {

static const double AVOGADRO = 6.02214179e23;  // src/steps/math/constants.hpp:45

// Membrane current per triangle over the EField step just taken (Tri::computeI,
// src/steps/mpi/tetopsplit/tri.cpp:664-694): sum over the patch's ohmic currents of
// g * (integral of the channel-state count / dt) * (V_tri - E_rev), in pA; the integrals
// restart at zero for the next step.
// out[i] = count of species row `row` in tet idx[i] (device-side gather for the batch
// getters, so a recording step moves only the selected tets).
__global__ void gather_counts_kernel(int n, const uint32_t* row, const int32_t* idx, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = (double)row[idx[i]];
}

// Membrane current of each triangle over the EField step just taken (tri.cpp:664-719):
// ohmic currents from the channel-state time integrals, plus the GHK charge the step's GHK
// events carried out (echarge e / dt).  Resets both accumulators.
__global__ void ohmic_current_kernel(int M, int nss, int noc, const sg_ohmic* oc, const int32_t* tri_patch,
                                     double* spec_int, const double* triV, double inv_dt, double* tri_I,
                                     double* tri_I_last, long long* echarge, double* tri_Ighk) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        const int p = tri_patch[m];
        double I = 0.0;
        for (int k = 0; k < noc; ++k) {
            if (oc[k].patch != p) continue;
            double nbar = spec_int[(size_t)oc[k].sspec * M + m] * inv_dt;
            I += (nbar * oc[k].g) * (triV[m] - oc[k].erev * 1.0e3);  // S * mV
        }
        I *= 1.0e9;  // S mV -> pA
        tri_I_last[m] = I;
        if (echarge) {
            const double ig = (double)echarge[m] * 1.602176487e-19 * inv_dt;  // A
            tri_Ighk[m] = ig;
            I += ig * 1.0e12;
            echarge[m] = 0;
        }
        tri_I[m] = I;
        for (int s = 0; s < nss; ++s) spec_int[(size_t)s * M + m] = 0.0;
    }
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        n = count;
        if (count) SG_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

struct Solver {
    int device = 0;
    uint64_t seed = 0;
    cudaStream_t stream = nullptr;
    int nsm = 148;

    // ---- model x mesh, host copies ----
    int ntets = 0, ncomp = 1, nspec = 0, nreal = 1;
    std::vector<double> vol, area, dist;        // [T], [T*4], [T*4]
    std::vector<int32_t> neighb, tet_comp;      // [T*4], [T]
    std::vector<int32_t> real_begin{0, 0};      // [nreal + 1]
    std::vector<sg_reac> reacs;                 // global reaction list, sorted by comp at setup
    std::vector<double> reac_kdef;              // model kcst per reaction
    std::vector<int32_t> reac_order_user;       // user reaction index -> sorted slot
    std::vector<double> dcst_def;               // [ncomp][S] model diffusion constants
    std::vector<int32_t> diff_comp, diff_spec;  // user diffusion rules
    std::vector<double> kcst;                   // [nreal][R] current constants
    std::vector<double> dcst;                   // [nreal][ncomp][S]
    std::vector<int32_t> comp_reac_begin;       // [ncomp + 1]
    std::vector<int32_t> diff_slot;             // [S]
    std::vector<float> geo;                     // [T*4]
    std::vector<int32_t> nbrp;                  // [T*4]
    std::vector<double> ivs;                    // [T]
    std::vector<uint32_t> clampm;               // [T]
    bool any_clamp = false;
    bool any_unassigned = false;
    int ndiff = 0;
    int diff_apply_threshold = 10;              // TOS:995; accepted, does not change the law
    bool is_setup = false;

    // ---- device state ----
    DevBuf<uint32_t> d_counts, d_outflow, d_clamp, d_status;
    DevBuf<unsigned int> d_work;  // [2][4] work counters of the split-window kernels
    DevBuf<int32_t> d_nbr, d_comp, d_crb, d_dslot, d_dspec;
    DevBuf<double> d_tdel;                      // [D][T] split mode only
    DevBuf<uint32_t> d_tmask;                   // [T] split mode only: species with a nonzero tdel
    // Diffusion boundaries.
    int nbnd = 0;
    std::vector<int32_t> face_bnd, bnd_comps;   // [T*4] boundary of each face or -1; [nbnd*2]
    std::vector<double> btab;                   // [nbnd][S][2] -1 closed, -2 own constant, >= 0 constant
    std::vector<uint8_t> bact;                  // [nbnd][S][2] direction open (side = source compartment)
    std::vector<double> bdcst;                  // [nbnd][S][2] direction constant, -1 = the source's own
    std::vector<uint32_t> bface;                // [T] bytes per face, 0xFF = none
    std::vector<int32_t> bnbr;                  // [T*4]
    std::vector<float> bcoef;                   // [T*4]
    DevBuf<uint32_t> d_bface;
    DevBuf<int32_t> d_bnbr, d_bcomps;
    DevBuf<float> d_bcoef;
    DevBuf<double> d_btab;
    bool split = false;                         // window as two kernels (reactions, diffusion)
    // Persistent form: all windows of a run() chunk in one cooperative launch
    // (persistent_window_kernel), tets per lane 1 or 2 (32 or 64 tets per work chunk).
    bool persist = false;
    int persist_tpl = 1;
    unsigned int persist_spin_limit = 1u << 22;  // polls (~100 ns each) before a wait gives up
    DevBuf<int32_t> d_pchunk;                   // [nreal + 1] first chunk of each realization
    DevBuf<unsigned int> d_pstate;              // done [nreal], ready [nreal], abort [1]
    DevBuf<unsigned long long> d_pnext;         // [1] next work item
    DevBuf<double> d_mode_tab;                  // [2][SG_MODE_TABLE]: 1/x, ln x! (persistent form)
    int pchunk_tpl = 0;                         // tets per lane d_pchunk was built for
    int pchunks = 0;
    DevBuf<float> d_geo;
    DevBuf<double> d_ivs, d_kcst, d_dcst;
    DevBuf<sg_reac> d_reacs;
    DevBuf<sg_real> d_reals;
    DevBuf<unsigned long long> d_totals, d_ext, d_ext_total, d_diff_total, d_launch;
    std::vector<sg_real> reals;                 // host mirror
    bool pending_host = false;
    uint64_t niteration = 0;
    uint64_t setup_calls = 0;                   // counter of the host placement stream
    int block = 128;
    int grid = 0;
    bool check = true;

    // ---- membrane triangles and surface reactions ----
    int nsspec = 0, ntris = 0, npatch = 0;
    std::vector<int32_t> tri_inner, tri_patch;      // [M]
    std::vector<double> tri_area;                   // [M] m^2
    std::vector<sg_sreac> sreacs;                   // grouped by patch at setup
    std::vector<double> skcst;
    std::vector<int32_t> sreac_order_user, patch_sb;
    std::vector<sg_vtab> vtabs;
    std::vector<double> vtab_vals;
    std::vector<sg_ohmic> ohmics;
    int max_sreac_per_patch = 0;
    bool surf_touches_volume = false;
    DevBuf<uint32_t> d_tri_counts;
    DevBuf<int32_t> d_tet_tris, d_tri_patch, d_psb;
    DevBuf<double> d_tri_area, d_skcst, d_vvals, d_spec_int, d_tri_Iohm;
    DevBuf<sg_sreac> d_sreacs;
    DevBuf<sg_vtab> d_vtabs;
    DevBuf<sg_ohmic> d_ohmics;
    DevBuf<unsigned long long> d_surf_ext;
    DevBuf<int32_t> d_memb_tets;                    // tets with membrane triangles
    int nmemb_tets = 0;
    // Surface diffusion (sdiff.cpp): edge neighbours, rules, device state.
    std::vector<int32_t> tri_nbr, tri_nbr_edge;     // [M*3] membrane neighbour across edge e, its edge
    std::vector<double> tri_len, tri_dist;          // [M*3] edge length, barycentre distance (m)
    std::vector<double> sdcst;                      // [npatch][SS] m^2/s, 0 = no rule
    std::vector<int32_t> sdiff_slot;                // [SS] compact index or -1
    std::vector<float> sgeo;                        // [M*4] c0, c1, 1, G (1/m^2)
    int nsdiff = 0;
    // GHK currents.
    std::vector<sg_ghk> ghks;
    double temp = 293.15;                           // K (API::setTemp)
    DevBuf<sg_ghk> d_ghks;
    DevBuf<long long> d_tri_echarge;
    DevBuf<double> d_tri_Ighk;
    DevBuf<uint32_t> d_tri_out;
    DevBuf<double> d_tri_occ, d_sdcst;
    DevBuf<int32_t> d_sdslot, d_sdspec, d_snbr, d_tri_inner;
    DevBuf<float> d_sgeo;
    bool has_surf() const { return ntris > 0 && nsspec > 0; }

    // Merged SSA units (triangles coupled to their outer tet, sreac.cpp:200-300).
    std::vector<int32_t> tri_outer;                 // [M] outer tet, -1 none (empty: not given)
    std::vector<int32_t> tet_unit_h;                // [T] unit of a merged tet, -1
    int nunits = 0, unit_rmax = 0;
    size_t unit_smem = 0;                           // shared bytes of the largest unit's tree and propensities
    DevBuf<int32_t> d_tri_outer, d_u_tet_begin, d_u_tets, d_u_tri_begin, d_u_tris, d_u_elem_base, d_u_tree_base,
        d_tet_unit, d_u_tet_adj, d_u_tri_side;
    DevBuf<double> d_u_prop, d_u_tree, d_u_socc, d_u_slast;

    // A patch couples its triangles' outer tets when a surface reaction counts or changes an
    // outer-volume species or a GHK current reads the outer tet's concentration.
    bool patch_coupled(int p) const {
        for (const auto& r : sreacs)
            if (r.patch == p && (r.vside != 0 || r.noupd > 0)) return true;
        for (const auto& g : ghks)
            if (g.patch == p && g.voconc < 0.0) return true;
        return false;
    }

    // Units: connected groups of tets linked by coupled triangles (union of inner and outer
    // tet), with every membrane triangle whose inner tet is in the group.  Elements in
    // canonical order: the unit's tets ascending, then its triangles ascending.
    void setup_units() {
        nunits = 0;
        tet_unit_h.assign(ntets, -1);
        std::vector<char> coupled(npatch, 0);
        bool any = false;
        for (int p = 0; p < npatch; ++p) {
            coupled[p] = patch_coupled(p) ? 1 : 0;
            any = any || coupled[p];
        }
        if (!any) return;
        if (tri_outer.size() != (size_t)ntris)
            throw ArgErr("surface reactions or GHK currents that reach the outer volume need the triangles' outer tets");
        std::vector<int32_t> par(ntets);
        for (int t = 0; t < ntets; ++t) par[t] = t;
        auto find = [&](int x) {
            while (par[x] != x) {
                par[x] = par[par[x]];
                x = par[x];
            }
            return x;
        };
        for (int m = 0; m < ntris; ++m) {
            if (!coupled[tri_patch[m]]) continue;
            const int o = tri_outer[m], i = tri_inner[m];
            if (o < 0) throw ArgErr("membrane triangle " + std::to_string(m) + " of a patch whose reactions reach the outer volume has no outer tet");
            if (realization_of(o) != realization_of(i)) throw ArgErr("a membrane triangle links tets of two realizations");
            const int a = find(i), b = find(o);
            if (a != b) par[a < b ? b : a] = a < b ? a : b;
        }
        std::vector<int32_t> size(ntets, 0), uid(ntets, -1);
        for (int t = 0; t < ntets; ++t) size[find(t)] += 1;
        for (int t = 0; t < ntets; ++t) {
            const int root = find(t);
            if (size[root] < 2) continue;
            if (uid[root] < 0) uid[root] = nunits++;
            tet_unit_h[t] = uid[root];
        }
        if (nunits == 0) return;
        std::vector<std::vector<int32_t>> ut(nunits), um(nunits);
        for (int t = 0; t < ntets; ++t)
            if (tet_unit_h[t] >= 0) ut[tet_unit_h[t]].push_back(t);
        for (int m = 0; m < ntris; ++m) {
            const int u = tet_unit_h[tri_inner[m]];
            if (u >= 0) um[u].push_back(m);
        }
        std::vector<int32_t> tb(nunits + 1, 0), mb(nunits + 1, 0), eb(nunits + 1, 0), trb(nunits + 1, 0);
        std::vector<int32_t> tets, tris;
        std::vector<int32_t> local(ntets, -1);
        for (int u = 0; u < nunits; ++u) {
            for (size_t k = 0; k < ut[u].size(); ++k) local[ut[u][k]] = (int32_t)k;
            tets.insert(tets.end(), ut[u].begin(), ut[u].end());
            tris.insert(tris.end(), um[u].begin(), um[u].end());
            const int E = (int)(ut[u].size() + um[u].size());
            int P = 1;
            while (P < E) P <<= 1;
            tb[u + 1] = tb[u] + (int)ut[u].size();
            mb[u + 1] = mb[u] + (int)um[u].size();
            eb[u + 1] = eb[u] + E;
            if ((long long)trb[u] + 2LL * P > 0x7FFFFFFFLL) throw ArgErr("merged SSA units too large");
            trb[u + 1] = trb[u] + 2 * P;
        }
        const int E = eb[nunits];
        std::vector<int32_t> adj((size_t)E * 4, -1), side((size_t)ntris * 2, -1);
        auto add_adj = [&](int e, int f) {
            for (int k = 0; k < 4; ++k) {
                int32_t& x = adj[(size_t)e * 4 + k];
                if (x == f) return;
                if (x < 0) {
                    x = f;
                    return;
                }
            }
            throw ArgErr("a tet borders more than four membrane triangles");
        };
        for (int u = 0; u < nunits; ++u) {
            const int nt = (int)ut[u].size();
            for (size_t j = 0; j < um[u].size(); ++j) {
                const int m = um[u][j];
                const int f = nt + (int)j;
                const int ei = local[tri_inner[m]];
                add_adj(eb[u] + ei, f);
                side[(size_t)m * 2] = ei;
                if (coupled[tri_patch[m]]) {
                    const int eo = local[tri_outer[m]];
                    add_adj(eb[u] + eo, f);
                    side[(size_t)m * 2 + 1] = eo;
                }
            }
        }
        unit_rmax = max_sreac_per_patch;
        for (int c = 0; c < ncomp; ++c) unit_rmax = std::max(unit_rmax, comp_reac_begin[c + 1] - comp_reac_begin[c]);
        unit_rmax = std::max(unit_rmax, 1);
        unit_smem = 0;
        for (int u = 0; u < nunits; ++u)
            unit_smem = std::max(unit_smem, ((size_t)(trb[u + 1] - trb[u]) + (size_t)(eb[u + 1] - eb[u]) * unit_rmax) * 8);
        if (tri_outer.size() == (size_t)ntris) {
            d_tri_outer.alloc(ntris);
            h2d(d_tri_outer.p, tri_outer.data(), tri_outer.size());
        }
        d_u_tet_begin.alloc(tb.size());
        d_u_tets.alloc(tets.size());
        d_u_tri_begin.alloc(mb.size());
        d_u_tris.alloc(std::max<size_t>(tris.size(), 1));
        d_u_elem_base.alloc(eb.size());
        d_u_tree_base.alloc(trb.size());
        d_tet_unit.alloc(ntets);
        d_u_tet_adj.alloc(adj.size());
        d_u_tri_side.alloc(side.size());
        d_u_prop.alloc((size_t)E * unit_rmax);
        d_u_tree.alloc((size_t)trb[nunits]);
        d_u_socc.alloc((size_t)nsspec * ntris);
        d_u_slast.alloc((size_t)nsspec * ntris);
        h2d(d_u_tet_begin.p, tb.data(), tb.size());
        h2d(d_u_tets.p, tets.data(), tets.size());
        h2d(d_u_tri_begin.p, mb.data(), mb.size());
        if (!tris.empty()) h2d(d_u_tris.p, tris.data(), tris.size());
        h2d(d_u_elem_base.p, eb.data(), eb.size());
        h2d(d_u_tree_base.p, trb.data(), trb.size());
        h2d(d_tet_unit.p, tet_unit_h.data(), tet_unit_h.size());
        h2d(d_u_tet_adj.p, adj.data(), adj.size());
        h2d(d_u_tri_side.p, side.data(), side.size());
        if (unit_smem <= kUnitSmemMax && unit_smem > 48 * 1024)
            SG_CUDA(cudaFuncSetAttribute(unit_ssa_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)unit_smem));
    }
    static constexpr size_t kUnitSmemMax = 200 * 1024;

    sg_unit_args unit_args() const {
        sg_unit_args u;
        std::memset(&u, 0, sizeof(u));
        if (nunits == 0) return u;
        u.tet_begin = d_u_tet_begin.p;
        u.tets = d_u_tets.p;
        u.tri_begin = d_u_tri_begin.p;
        u.tris = d_u_tris.p;
        u.elem_base = d_u_elem_base.p;
        u.tree_base = d_u_tree_base.p;
        u.tet_unit = d_tet_unit.p;
        u.tet_adj = d_u_tet_adj.p;
        u.tri_side = d_u_tri_side.p;
        u.prop = d_u_prop.p;
        u.tree = d_u_tree.p;
        u.socc = d_u_socc.p;
        u.slast = d_u_slast.p;
        u.nunits = nunits;
        u.rmax = unit_rmax;
        return u;
    }

    // Surface diffusion tables (sdiff.cpp:62-83): per triangle the edge coefficients
    // g_e = l_e / (A d_e) towards same-patch neighbours, G = sum g_e, and the conditional
    // selectors c0 = g0 / G, c1 = g1 / (g1 + g2); the scaled constant is D G.
    void setup_sdiff() {
        sdiff_slot.assign(nsspec, -1);
        nsdiff = 0;
        bool any = false;
        for (double d : sdcst)
            if (d > 0.0) any = true;
        if (!any) return;
        if (tri_nbr.size() != (size_t)ntris * 3) throw ArgErr("surface diffusion needs the triangle neighbours");
        std::vector<int32_t> sdspec;
        for (int s = 0; s < nsspec; ++s) {
            bool has = false;
            for (int p = 0; p < npatch; ++p)
                if (sdcst[(size_t)p * nsspec + s] > 0.0) has = true;
            if (has) {
                sdiff_slot[s] = (int32_t)sdspec.size();
                sdspec.push_back(s);
            }
        }
        nsdiff = (int)sdspec.size();
        sgeo.assign((size_t)ntris * 4, 0.0f);
        std::vector<int32_t> snbr((size_t)ntris * 4, -1);
        for (int m = 0; m < ntris; ++m) {
            double g[3] = {0.0, 0.0, 0.0};
            for (int e = 0; e < 3; ++e) {
                const int q = tri_nbr[(size_t)m * 3 + e];
                if (q < 0 || tri_patch[q] != tri_patch[m]) continue;
                const double d = tri_dist[(size_t)m * 3 + e];
                if (!(d > 0.0)) continue;
                g[e] = tri_len[(size_t)m * 3 + e] / (tri_area[m] * d);
                snbr[(size_t)m * 4 + e] = (q << 2) | tri_nbr_edge[(size_t)m * 3 + e];
            }
            const double G = g[0] + g[1] + g[2];
            const double r12 = g[1] + g[2];
            sgeo[(size_t)m * 4 + 0] = G > 0.0 ? (float)(g[0] / G) : 0.0f;
            sgeo[(size_t)m * 4 + 1] = r12 > 0.0 ? (float)(g[1] / r12) : 0.0f;
            sgeo[(size_t)m * 4 + 2] = 1.0f;
            sgeo[(size_t)m * 4 + 3] = (float)G;
        }
        d_tri_out.alloc((size_t)2 * nsdiff * ntris * 4);
        SG_CUDA(cudaMemsetAsync(d_tri_out.p, 0, d_tri_out.n * 4, stream));
        d_tri_occ.alloc((size_t)nsdiff * ntris);
        d_sdcst.alloc(sdcst.size());
        d_sdslot.alloc(nsspec);
        d_sdspec.alloc(nsdiff);
        d_snbr.alloc(snbr.size());
        d_sgeo.alloc(sgeo.size());
        if (!d_tri_inner.p) d_tri_inner.alloc(ntris);
        h2d(d_sdcst.p, sdcst.data(), sdcst.size());
        h2d(d_sdslot.p, sdiff_slot.data(), sdiff_slot.size());
        h2d(d_sdspec.p, sdspec.data(), sdspec.size());
        h2d(d_snbr.p, snbr.data(), snbr.size());
        h2d(d_sgeo.p, sgeo.data(), sgeo.size());
        h2d(d_tri_inner.p, tri_inner.data(), tri_inner.size());
    }

    void setup_surface() {
        if (!has_surf()) return;
        // Surface reactions grouped by patch.
        const int RS = (int)sreacs.size();
        std::vector<int32_t> order(RS);
        for (int i = 0; i < RS; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return sreacs[x].patch < sreacs[y].patch; });
        std::vector<sg_sreac> sorted(RS);
        std::vector<double> ks(RS);
        sreac_order_user.assign(RS, 0);
        for (int i = 0; i < RS; ++i) {
            sorted[i] = sreacs[order[i]];
            ks[i] = skcst[order[i]];
            sreac_order_user[order[i]] = i;
        }
        sreacs = sorted;
        skcst = ks;
        patch_sb.assign(npatch + 1, 0);
        for (auto& r : sreacs) patch_sb[r.patch + 1] += 1;
        for (int p = 0; p < npatch; ++p) patch_sb[p + 1] += patch_sb[p];
        max_sreac_per_patch = 1;
        for (int p = 0; p < npatch; ++p) {
            int ng = 0;
            for (const auto& g : ghks)
                if (g.patch == p) ++ng;
            max_sreac_per_patch = std::max(max_sreac_per_patch, patch_sb[p + 1] - patch_sb[p] + ng);
        }
        surf_touches_volume = false;
        for (auto& r : sreacs)
            if (r.niupd > 0 || r.noupd > 0) surf_touches_volume = true;
        for (auto& g : ghks)
            if (g.realflux) surf_touches_volume = true;
        if (!ghks.empty()) {
            d_ghks.alloc(ghks.size());
            h2d(d_ghks.p, ghks.data(), ghks.size());
            d_tri_echarge.alloc(ntris);
            d_tri_Ighk.alloc(ntris);
            SG_CUDA(cudaMemsetAsync(d_tri_echarge.p, 0, ntris * 8, stream));
            SG_CUDA(cudaMemsetAsync(d_tri_Ighk.p, 0, ntris * 8, stream));
        }
        // SSA units: each triangle joins the unit of its inner tet.
        std::vector<int32_t> tt((size_t)ntets * 4, -1);
        for (int m = 0; m < ntris; ++m) {
            int t = tri_inner[m];
            if (t < 0 || t >= ntets) throw ArgErr("membrane triangle without a valid inner tet");
            int slot = 0;
            while (slot < 4 && tt[(size_t)t * 4 + slot] >= 0) ++slot;
            if (slot == 4) throw ArgErr("a tet has more than four membrane triangles");
            tt[(size_t)t * 4 + slot] = m;
        }
        d_tri_counts.alloc((size_t)nsspec * ntris);
        d_tet_tris.alloc(tt.size());
        d_tri_patch.alloc(ntris);
        d_psb.alloc(npatch + 1);
        d_tri_area.alloc(ntris);
        d_skcst.alloc(std::max(RS, 1));
        d_vvals.alloc(std::max<size_t>(vtab_vals.size(), 1));
        d_spec_int.alloc((size_t)nsspec * ntris);
        d_tri_Iohm.alloc(ntris);
        d_sreacs.alloc(std::max(RS, 1));
        d_vtabs.alloc(std::max<size_t>(vtabs.size(), 1));
        d_ohmics.alloc(std::max<size_t>(ohmics.size(), 1));
        d_surf_ext.alloc(1);
        h2d(d_tet_tris.p, tt.data(), tt.size());
        if (!d_tri_inner.p) {
            d_tri_inner.alloc(ntris);
            h2d(d_tri_inner.p, tri_inner.data(), tri_inner.size());
        }
        setup_units();
        // Tets with membrane triangles and no merged unit, ascending: the SURF launch of a
        // split window.
        std::vector<int32_t> mt;
        for (int t = 0; t < ntets; ++t)
            if (tt[(size_t)t * 4] >= 0 && tet_unit_h[t] < 0) mt.push_back(t);
        nmemb_tets = (int)mt.size();
        d_memb_tets.alloc(std::max<size_t>(mt.size(), 1));
        if (!mt.empty()) h2d(d_memb_tets.p, mt.data(), mt.size());
        split = true;  // membrane models run the split window by default (see launch_window)
        setup_sdiff();
        h2d(d_tri_patch.p, tri_patch.data(), tri_patch.size());
        h2d(d_psb.p, patch_sb.data(), patch_sb.size());
        h2d(d_tri_area.p, tri_area.data(), tri_area.size());
        if (RS) h2d(d_skcst.p, skcst.data(), skcst.size());
        if (!vtab_vals.empty()) h2d(d_vvals.p, vtab_vals.data(), vtab_vals.size());
        if (RS) h2d(d_sreacs.p, sreacs.data(), sreacs.size());
        if (!vtabs.empty()) h2d(d_vtabs.p, vtabs.data(), vtabs.size());
        if (!ohmics.empty()) h2d(d_ohmics.p, ohmics.data(), ohmics.size());
    }

    void reset_surface() {
        if (!has_surf()) return;
        SG_CUDA(cudaMemsetAsync(d_tri_counts.p, 0, d_tri_counts.n * 4, stream));
        SG_CUDA(cudaMemsetAsync(d_spec_int.p, 0, d_spec_int.n * 8, stream));
        SG_CUDA(cudaMemsetAsync(d_tri_Iohm.p, 0, d_tri_Iohm.n * 8, stream));
        SG_CUDA(cudaMemsetAsync(d_surf_ext.p, 0, 8, stream));
    }

    sg_surf_args surf_args() {
        sg_surf_args s;
        std::memset(&s, 0, sizeof(s));
        if (!has_surf()) return s;
        s.tri_counts = d_tri_counts.p;
        s.tet_tris = d_tet_tris.p;
        s.tri_patch = d_tri_patch.p;
        s.tri_area = d_tri_area.p;
        s.tri_V = ef_on ? ef.tri_V : nullptr;
        s.sreacs = d_sreacs.p;
        s.patch_sreac_begin = d_psb.p;
        s.skcst = d_skcst.p;
        s.vtabs = d_vtabs.p;
        s.vtab_vals = d_vvals.p;
        s.spec_int = d_spec_int.p;
        if (!ghks.empty()) {
            s.ghks = d_ghks.p;
            s.nghk = (int)ghks.size();
            s.tri_echarge = d_tri_echarge.p;
        }
        s.temp = temp;
        s.tri_inner = d_tri_inner.p;
        s.tri_outer = d_tri_outer.p;
        if (nsdiff > 0) {
            s.tri_outflow = d_tri_out.p;
            s.tri_occ = d_tri_occ.p;
            s.sdiff_slot = d_sdslot.p;
            s.sdiff_spec = d_sdspec.p;
            s.sdcst = d_sdcst.p;
            s.snbr = d_snbr.p;
            s.sgeo = d_sgeo.p;
            s.nsdiff = nsdiff;
        }
        s.nsspec = nsspec;
        s.ntris = ntris;
        s.nsreac = (int)sreacs.size();
        s.max_sreac_per_patch = max_sreac_per_patch;
        return s;
    }

    // ---- EField (membrane potential) ----
    EFieldSystem ef;
    bool ef_on = false;
    double efdt = 1.0e-5;                       // s, TOS:938 default EField dt

    // ---- launch accounting and optional per-run CUDA-event timing ----
    uint64_t launches = 0;                      // kernels launched by this solver
    bool profiling = false;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    double prof_ms = 0.0;                       // device time of window launches
    uint64_t prof_windows = 0;

    Solver(uint64_t s, int dev) : device(dev), seed(s) {
        SG_CUDA(cudaSetDevice(device));
        SG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        SG_CUDA(cudaEventCreate(&ev_begin));
        SG_CUDA(cudaEventCreate(&ev_end));
        cudaDeviceProp prop;
        SG_CUDA(cudaGetDeviceProperties(&prop, device));
        nsm = prop.multiProcessorCount;
    }
    ~Solver() {
        drop_graph();
        if (ev_begin) cudaEventDestroy(ev_begin);
        if (ev_end) cudaEventDestroy(ev_end);
        if (stream) cudaStreamDestroy(stream);
    }

    void require_setup() const {
        if (!is_setup) throw ProgErr("solver tables are not set up (call sg_setup first)");
    }
    void require_not_setup() const {
        if (is_setup) throw ProgErr("model and mesh are fixed once sg_setup has been called");
    }
    void check_tet(int t) const {
        if (t < 0 || t >= ntets) throw ArgErr("tetrahedron index out of range: " + std::to_string(t));
    }
    void check_spec(int s) const {
        if (s < 0 || s >= nspec) throw ArgErr("species index out of range: " + std::to_string(s));
    }
    void check_comp(int c) const {
        if (c < 0 || c >= ncomp) throw ArgErr("compartment index out of range: " + std::to_string(c));
    }
    void check_real(int r) const {
        if (r < 0 || r >= nreal) throw ArgErr("realization index out of range: " + std::to_string(r));
    }

    template <typename T>
    void h2d(T* dst, const T* src, size_t n) {
        if (n) SG_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream));
    }
    template <typename T>
    void d2h(T* dst, const T* src, size_t n) {
        if (n) SG_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, stream));
    }
    void sync() { SG_CUDA(cudaStreamSynchronize(stream)); }

    int realization_of(int t) const {
        if (nreal == 1) return 0;
        auto it = std::upper_bound(real_begin.begin(), real_begin.end(), t);
        return (int)(it - real_begin.begin()) - 1;
    }

    // ------------------------------------------------------------------
    // Setup: flatten model x mesh into the device tables (TOS:479-1088,
    // diff.cpp:41-90 for the scaled diffusion constant and face selector,
    // reac.cpp:44-53 for the volume scaling of reaction constants).
    // ------------------------------------------------------------------
    void setup() {
        require_not_setup();
        if (ntets <= 0) throw ArgErr("mesh has no tetrahedra");
        if (nspec <= 0) throw ArgErr("model has no volume species");
        if ((int)real_begin.size() != nreal + 1 || real_begin[0] != 0 || real_begin[nreal] != ntets)
            throw ArgErr("realization tet offsets do not cover the mesh");
        for (int r = 0; r < nreal; ++r)
            if (real_begin[r + 1] < real_begin[r]) throw ArgErr("realization offsets decrease");

        // Reactions grouped by compartment (model order kept inside a compartment).
        const int R = (int)reacs.size();
        std::vector<int32_t> order(R);
        for (int i = 0; i < R; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return reacs[a].comp < reacs[b].comp; });
        std::vector<sg_reac> sorted(R);
        std::vector<double> ksorted(R);
        reac_order_user.assign(R, 0);
        for (int i = 0; i < R; ++i) {
            sorted[i] = reacs[order[i]];
            ksorted[i] = reac_kdef[order[i]];
            reac_order_user[order[i]] = i;
        }
        reacs = sorted;
        reac_kdef = ksorted;
        comp_reac_begin.assign(ncomp + 1, 0);
        for (int i = 0; i < R; ++i) comp_reac_begin[reacs[i].comp + 1] += 1;
        for (int c = 0; c < ncomp; ++c) comp_reac_begin[c + 1] += comp_reac_begin[c];

        // Diffusion: one compact slot per species that has a rule somewhere.
        diff_slot.assign(nspec, -1);
        ndiff = 0;
        for (size_t i = 0; i < diff_spec.size(); ++i)
            if (diff_slot[diff_spec[i]] < 0) diff_slot[diff_spec[i]] = ndiff++;

        build_geometry();

        // Per-realization parameter copies.
        kcst.assign((size_t)nreal * R, 0.0);
        dcst.assign((size_t)nreal * ncomp * nspec, 0.0);

        // Device buffers.
        d_counts.alloc((size_t)nspec * ntets);
        d_outflow.alloc((size_t)2 * std::max(ndiff, 1) * ntets * 4);
        SG_CUDA(cudaMemsetAsync(d_outflow.p, 0, d_outflow.n * 4, stream));
        d_nbr.alloc((size_t)ntets * 4);
        d_geo.alloc((size_t)ntets * 4);
        d_ivs.alloc(ntets);
        d_clamp.alloc(ntets);
        d_comp.alloc(ntets);
        d_reacs.alloc(std::max(R, 1));
        d_crb.alloc(ncomp + 1);
        d_dslot.alloc(nspec);
        d_kcst.alloc(std::max<size_t>(kcst.size(), 1));
        d_dcst.alloc(dcst.size());
        d_reals.alloc(nreal);
        d_totals.alloc((size_t)2 * nspec);
        d_ext.alloc((size_t)2 * std::max(R, 1));
        d_ext_total.alloc(std::max(R, 1));
        d_diff_total.alloc(1);
        d_launch.alloc(4);
        d_status.alloc(1);
        d_work.alloc(8);
        h2d(d_nbr.p, nbrp.data(), nbrp.size());
        h2d(d_geo.p, geo.data(), geo.size());
        h2d(d_ivs.p, ivs.data(), ivs.size());
        h2d(d_comp.p, tet_comp.data(), tet_comp.size());
        if (R) h2d(d_reacs.p, reacs.data(), reacs.size());
        h2d(d_crb.p, comp_reac_begin.data(), comp_reac_begin.size());
        h2d(d_dslot.p, diff_slot.data(), diff_slot.size());
        if (nbnd > 0) {
            bact.assign((size_t)nbnd * nspec * 2, 0);
            bdcst.assign((size_t)nbnd * nspec * 2, -1.0);
            btab.assign((size_t)nbnd * nspec * 2, -1.0);
            d_bface.alloc(bface.size());
            d_bnbr.alloc(bnbr.size());
            d_bcoef.alloc(bcoef.size());
            d_bcomps.alloc(bnd_comps.size());
            d_btab.alloc(btab.size());
            h2d(d_bface.p, bface.data(), bface.size());
            h2d(d_bnbr.p, bnbr.data(), bnbr.size());
            h2d(d_bcoef.p, bcoef.data(), bcoef.size());
            h2d(d_bcomps.p, bnd_comps.data(), bnd_comps.size());
            h2d(d_btab.p, btab.data(), btab.size());
        }
        {
            std::vector<int32_t> dspec(std::max(ndiff, 1), 0);
            for (int s = 0; s < nspec; ++s)
                if (diff_slot[s] >= 0) dspec[diff_slot[s]] = s;
            d_dspec.alloc(dspec.size());
            h2d(d_dspec.p, dspec.data(), dspec.size());
        }
        reals.assign(nreal, sg_real{});
        for (int r = 0; r < nreal; ++r) {
            reals[r].tet_begin = real_begin[r];
            reals[r].tet_end = real_begin[r + 1];
        }
        clampm.assign(ntets, 0u);
        is_setup = true;
        setup_surface();
        set_kernel_smem_limits();
        reset();
    }

    void build_geometry() {
        geo.assign((size_t)ntets * 4, 0.0f);
        nbrp.assign((size_t)ntets * 4, -1);
        ivs.assign(ntets, 0.0);
        any_unassigned = false;
        for (int t = 0; t < ntets; ++t) {
            int c = tet_comp[t];
            if (c < 0) any_unassigned = true;
            if (!(vol[t] > 0.0)) throw ArgErr("tetrahedron " + std::to_string(t) + " has no volume");
            ivs[t] = 1.0 / (1.0e3 * vol[t] * AVOGADRO);
            double g[4] = {0.0, 0.0, 0.0, 0.0};
            for (int f = 0; f < 4; ++f) {
                int n = neighb[(size_t)t * 4 + f];
                if (n < -1 || n >= ntets) throw ArgErr("neighbour index out of range");
                if (n < 0) continue;
                int rf = -1;
                for (int j = 0; j < 4; ++j)
                    if (neighb[(size_t)n * 4 + j] == t) rf = j;
                if (rf < 0) throw ArgErr("neighbour table is not symmetric at tet " + std::to_string(t));
                if (realization_of(t) != realization_of(n)) throw ArgErr("neighbour crosses realizations");
                double d = dist[(size_t)t * 4 + f];
                if (c >= 0 && d > 0.0 && tet_comp[n] == c) {
                    g[f] = area[(size_t)t * 4 + f] / (vol[t] * d);
                    nbrp[(size_t)t * 4 + f] = (n << 2) | rf;
                }
            }
            double G = g[0] + g[1] + g[2] + g[3];
            int lastf = -1;
            for (int f = 0; f < 4; ++f)
                if (g[f] > 0.0) lastf = f;
            double rem = G;
            for (int f = 0; f < 3; ++f) {
                double cf = 0.0;
                if (g[f] > 0.0) {
                    cf = (f == lastf) ? 1.0 : g[f] / rem;
                    if (cf > 1.0) cf = 1.0;
                    rem -= g[f];
                }
                geo[(size_t)t * 4 + f] = (float)cf;
            }
            geo[(size_t)t * 4 + 3] = (float)G;
        }
        build_boundaries();
    }

    // Boundary faces: the two tets of a face must be in the boundary's two compartments.
    void build_boundaries() {
        if (nbnd == 0) return;
        bface.assign(ntets, 0xFFFFFFFFu);
        bnbr.assign((size_t)ntets * 4, -1);
        bcoef.assign((size_t)ntets * 4, 0.0f);
        for (int t = 0; t < ntets; ++t)
            for (int f = 0; f < 4; ++f) {
                const int b = face_bnd[(size_t)t * 4 + f];
                if (b < 0) continue;
                if (b >= nbnd) throw ArgErr("diffusion boundary index out of range");
                const int n = neighb[(size_t)t * 4 + f];
                if (n < 0) throw ArgErr("diffusion boundary face without a second tet");
                const int ca = bnd_comps[(size_t)b * 2], cb = bnd_comps[(size_t)b * 2 + 1];
                const int c = tet_comp[t], cn = tet_comp[n];
                if (!((c == ca && cn == cb) || (c == cb && cn == ca)))
                    throw ArgErr("diffusion boundary face does not join the boundary's compartments");
                int rf = -1;
                for (int j = 0; j < 4; ++j)
                    if (neighb[(size_t)n * 4 + j] == t) rf = j;
                if (face_bnd[(size_t)n * 4 + rf] != b) throw ArgErr("diffusion boundary faces are not symmetric");
                bface[t] = (bface[t] & ~(0xFFu << (8 * f))) | ((uint32_t)b << (8 * f));
                bnbr[(size_t)t * 4 + f] = (n << 2) | rf;
                const double d = dist[(size_t)t * 4 + f];
                if (!(d > 0.0)) throw ArgErr("diffusion boundary face with zero distance");
            }
        // Face coefficients of every tet that has a boundary face (all its faces).
        for (int t = 0; t < ntets; ++t) {
            if (bface[t] == 0xFFFFFFFFu) continue;
            for (int f = 0; f < 4; ++f) {
                const int n = neighb[(size_t)t * 4 + f];
                const double d = dist[(size_t)t * 4 + f];
                if (n >= 0 && d > 0.0) bcoef[(size_t)t * 4 + f] = (float)(area[(size_t)t * 4 + f] / (vol[t] * d));
            }
        }
    }

    // setDiffBoundarySpecDiffusionActive / setDiffBoundarySpecDcst (TOS:2745-2800, 2865-2930).
    void check_bnd(int b, int s) const {
        if (b < 0 || b >= nbnd) throw ArgErr("diffusion boundary index out of range");
        check_spec(s);
        if (diff_slot[s] < 0) throw ArgErr("species has no diffusion rule");
    }
    void upload_btab() {
        for (size_t i = 0; i < btab.size(); ++i) btab[i] = bact[i] ? (bdcst[i] >= 0.0 ? bdcst[i] : -2.0) : -1.0;
        h2d(d_btab.p, btab.data(), btab.size());
        recompute_periods();
        upload_reals();
        sync();
    }
    void set_bnd_active(int b, int s, bool on) {
        require_setup();
        check_bnd(b, s);
        flush();
        for (int side = 0; side < 2; ++side) bact[((size_t)b * nspec + s) * 2 + side] = on ? 1 : 0;
        upload_btab();
    }
    bool get_bnd_active(int b, int s) const {
        check_bnd(b, s);
        return bact[((size_t)b * nspec + s) * 2] || bact[((size_t)b * nspec + s) * 2 + 1];
    }
    // direction_comp >= 0: only diffusion into that compartment takes dcst (and opens).
    void set_bnd_dcst(int b, int s, double d, int direction_comp) {
        require_setup();
        check_bnd(b, s);
        if (!(d >= 0.0)) throw ArgErr("diffusion constant must be non-negative");
        if (direction_comp >= 0 && direction_comp != bnd_comps[(size_t)b * 2] &&
            direction_comp != bnd_comps[(size_t)b * 2 + 1])
            throw ArgErr("direction compartment is not joined by this boundary");
        flush();
        for (int side = 0; side < 2; ++side) {
            const int src = bnd_comps[(size_t)b * 2 + side];
            if (direction_comp >= 0 && src == direction_comp) continue;
            bact[((size_t)b * nspec + s) * 2 + side] = 1;
            bdcst[((size_t)b * nspec + s) * 2 + side] = d;
        }
        upload_btab();
    }

    // Scaled diffusion constant of tet t for species s at constant D (TOS:5373 with the
    // boundary directions of diff.cpp:340-398).
    double tet_scaled_dcst(int t, int s, double D) const {
        if (nbnd == 0 || bface[t] == 0xFFFFFFFFu) return D * (double)geo[(size_t)t * 4 + 3];
        double tot = 0.0;
        for (int f = 0; f < 4; ++f) {
            const double cf = (double)bcoef[(size_t)t * 4 + f];
            if (nbrp[(size_t)t * 4 + f] >= 0) {
                tot += cf * D;
                continue;
            }
            const uint32_t b = (bface[t] >> (8 * f)) & 0xFFu;
            if (b == 0xFFu) continue;
            const int side = (tet_comp[t] == bnd_comps[(size_t)b * 2]) ? 0 : 1;
            const double v = btab[((size_t)b * nspec + s) * 2 + side];
            if (v < -1.5) tot += cf * D;
            else if (v >= 0.0) tot += cf * v;
        }
        return tot;
    }

    // Largest scaled diffusion constant per realization -> update period
    // (TOS:5373-5411 _computeUpdPeriod; the MPI max-reduction becomes a host max).
    void recompute_periods() {
        for (int r = 0; r < nreal; ++r) {
            double mx = 0.0;
            for (int t = real_begin[r]; t < real_begin[r + 1]; ++t) {
                int c = tet_comp[t];
                if (c < 0) continue;
                double G = (double)geo[(size_t)t * 4 + 3];
                for (int s = 0; s < nspec; ++s) {
                    if (diff_slot[s] < 0) continue;
                    const double D = dcst[((size_t)r * ncomp + c) * nspec + s];
                    double sd = (nbnd > 0) ? tet_scaled_dcst(t, s, D) : D * G;
                    if (sd > mx) mx = sd;
                }
            }
            // Surface diffusion rules count too (TOS:5373-5411 takes the max over both).
            for (int m = 0; nsdiff > 0 && m < ntris; ++m) {
                const int t = tri_inner[m];
                if (t < real_begin[r] || t >= real_begin[r + 1]) continue;
                const double G = (double)sgeo[(size_t)m * 4 + 3];
                for (int s = 0; s < nsspec; ++s) {
                    const double sd = sdcst[(size_t)tri_patch[m] * nsspec + s] * G;
                    if (sd > mx) mx = sd;
                }
            }
            reals[r].period = (mx > 0.0) ? 1.0 / mx : std::numeric_limits<double>::infinity();
        }
    }

    void upload_params() {
        h2d(d_kcst.p, kcst.data(), kcst.size());
        h2d(d_dcst.p, dcst.data(), dcst.size());
        recompute_periods();
        upload_reals();
    }
    void upload_reals() { h2d(d_reals.p, reals.data(), reals.size()); }
    void download_reals() {
        d2h(reals.data(), d_reals.p, reals.size());
        sync();
    }

    // Reference reset (TOS reset): counts to zero, time to zero, constants to the
    // model values, extents cleared, clamps released.
    void reset() {
        require_setup();
        SG_CUDA(cudaMemsetAsync(d_counts.p, 0, d_counts.n * 4, stream));
        SG_CUDA(cudaMemsetAsync(d_totals.p, 0, d_totals.n * 8, stream));
        SG_CUDA(cudaMemsetAsync(d_ext.p, 0, d_ext.n * 8, stream));
        SG_CUDA(cudaMemsetAsync(d_ext_total.p, 0, d_ext_total.n * 8, stream));
        SG_CUDA(cudaMemsetAsync(d_diff_total.p, 0, 8, stream));
        SG_CUDA(cudaMemsetAsync(d_launch.p, 0, 32, stream));
        SG_CUDA(cudaMemsetAsync(d_work.p, 0, 32, stream));
        SG_CUDA(cudaMemsetAsync(d_status.p, 0, 4, stream));
        const int R = (int)reacs.size();
        for (int r = 0; r < nreal; ++r)
            for (int i = 0; i < R; ++i) kcst[(size_t)r * R + i] = reac_kdef[i];
        for (int r = 0; r < nreal; ++r)
            for (int c = 0; c < ncomp; ++c)
                for (int s = 0; s < nspec; ++s)
                    dcst[((size_t)r * ncomp + c) * nspec + s] = dcst_def[(size_t)c * nspec + s];
        std::fill(clampm.begin(), clampm.end(), 0u);
        any_clamp = false;
        h2d(d_clamp.p, clampm.data(), clampm.size());
        for (auto& rl : reals) {
            rl.t = 0.0;
            rl.t_end = 0.0;
            rl.window = 0;
            rl.pending = 0;
        }
        pending_host = false;
        niteration = 0;
        reset_surface();
        upload_params();
        sync();
    }

    // ------------------------------------------------------------------
    // Split-window loop (TOS:1507-1527 run, TOS:1528-1839 _runWithoutEField).
    // ------------------------------------------------------------------
    static bool almost_equal(double x, double y) {  // src/steps/util/collections.hpp:144-148
        double d = std::fabs(x - y);
        return d <= std::numeric_limits<double>::epsilon() * std::fabs(x + y) * 4 ||
               d < std::numeric_limits<double>::min();
    }

    sg_window_args window_args() {
        sg_window_args a;
        std::memset(&a, 0, sizeof(a));
        a.counts = d_counts.p;
        a.outflow = d_outflow.p;
        a.nbr = d_nbr.p;
        a.geo = d_geo.p;
        a.ivs = d_ivs.p;
        a.comp = (ncomp > 1 || any_unassigned) ? d_comp.p : nullptr;
        a.clamp = any_clamp ? d_clamp.p : nullptr;
        a.reacs = d_reacs.p;
        a.comp_reac_begin = d_crb.p;
        a.kcst = d_kcst.p;
        a.dcst = d_dcst.p;
        a.diff_slot = d_dslot.p;
        a.reals = d_reals.p;
        a.totals = d_totals.p;
        a.ext = d_ext.p;
        a.ext_total = d_ext_total.p;
        a.diff_total = d_diff_total.p;
        a.launch_state = d_launch.p;
        a.status = d_status.p;
        a.surf = surf_args();
        a.units = unit_args();
        a.surf_ext = has_surf() ? d_surf_ext.p : nullptr;
        a.tdel = d_tdel.p;
        a.tmask = d_tmask.p;
        a.diff_spec = d_dspec.p;
        a.work = d_work.p;
        if (nbnd > 0) {
            a.bface = d_bface.p;
            a.bnbr = d_bnbr.p;
            a.bcoef = d_bcoef.p;
            a.bcomps = d_bcomps.p;
            a.btab = d_btab.p;
            a.nbnd = nbnd;
        }
        a.ntets = ntets;
        a.nspec = nspec;
        a.ndiff = ndiff;
        a.nreac = (int)reacs.size();
        a.ncomp = ncomp;
        a.nreal = nreal;
        a.seed = seed;
        ensure_mode_tables();
        a.mode_rcpl = d_mode_tab.p;
        a.mode_lnf = d_mode_tab.p + SG_MODE_TABLE;
        return a;
    }

    // Models with membrane triangles run the SURF kernel (block 128).
    int eff_block() const { return has_surf() ? 128 : block; }
    size_t window_smem() const {
        size_t b = smem_bytes(eff_block(), nspec, (int)reacs.size());
        if (has_surf()) b = ((b + 15) & ~(size_t)15) + surf_smem_bytes(128, nsspec, max_sreac_per_patch);
        return b;
    }
    int check_flag() const { return (check && !any_clamp && !(has_surf() && surf_touches_volume)) ? 1 : 0; }

    void set_kernel_smem_limits() {
        // Window kernels are occupancy-bound on shared memory: the largest carveout unless
        // the autotuner picked another.
        set_carveout(carveout);
        size_t sm = smem_bytes(256, nspec, (int)reacs.size());
        if (sm > 227 * 1024) throw NotImplErr("too many species for the shared-memory staging");
        if (sm > 48 * 1024) {
            SG_CUDA(cudaFuncSetAttribute(window_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            SG_CUDA(cudaFuncSetAttribute(window_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            SG_CUDA(cudaFuncSetAttribute(window_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            SG_CUDA(cudaFuncSetAttribute(window_kernel<64, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            SG_CUDA(cudaFuncSetAttribute(window_kernel<128, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            SG_CUDA(cudaFuncSetAttribute(window_kernel<256, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        }
        if (has_surf()) {
            size_t ss = window_smem();
            if (ss > 227 * 1024) throw NotImplErr("too many surface species or reactions for the shared-memory staging");
            if (ss > 48 * 1024) {
                SG_CUDA(cudaFuncSetAttribute(window_kernel<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)ss));
                SG_CUDA(cudaFuncSetAttribute(window_kernel<128, true, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
            }
        }
    }

    // grid > 0: that many blocks; 0: occupancy-sized (blocks stride over the tets);
    // -1: one tet per thread (the hardware schedules new blocks as old ones finish).
    int window_grid() {
        if (grid > 0) return grid;
        if (grid == -1) return (int)std::max(1L, ((long)ntets + eff_block() - 1) / eff_block());
        size_t sm = window_smem();
        int per_sm = 0;
        if (has_surf()) {
            SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<128, true>, 128, sm));
        } else {
            switch (block) {
                case 64: SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<64>, 64, sm)); break;
                case 128: SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<128>, 128, sm)); break;
                case 256: SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<256>, 256, sm)); break;
                default: throw ArgErr("block size must be 64, 128 or 256");
            }
        }
        if (per_sm < 1) per_sm = 1;
        long need = ((long)ntets + eff_block() - 1) / eff_block();
        long cap = (long)per_sm * nsm;
        return (int)std::max(1L, std::min(need, cap));
    }

    bool use_split() const { return split || nsdiff > 0 || nunits > 0; }
    // Kernels one window launch enqueues (launch_window).
    int kernels_per_window() const {
        if (!use_split()) return 1;
        if (!has_surf()) return 2;
        return 2 + (nmemb_tets > 0 ? 1 : 0) + (nunits > 0 ? 1 : 0) + (nsdiff > 0 ? 1 : 0);
    }
    void ensure_split_buffers() {
        if (!d_tdel.p && ndiff > 0) d_tdel.alloc((size_t)ndiff * ntets);
        if (!d_tmask.p && ndiff > 0) d_tmask.alloc((size_t)ntets);
    }

    // Grids of the dynamically scheduled split kernels: every block resident at once (warps
    // take their tets from a work counter), capped by the blocks the tets can fill.
    int occ_cache_key[3] = {-1, -1, -1};
    int occ_cache_val[3] = {0, 0, 0};
    int resident_blocks(int which, int blk, size_t smem) {
        const int key = blk * 1000003 + (int)smem;
        if (occ_cache_key[which] == key) return occ_cache_val[which];
        int per_sm = 0;
        if (which == 0) {
            switch (blk) {
                case 64: SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<64, false, true>, 64, smem)); break;
                case 128: SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<128, false, true>, 128, smem)); break;
                case 256: SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<256, false, true>, 256, smem)); break;
                default: throw ArgErr("block size must be 64, 128 or 256");
            }
        } else if (which == 1) {
            SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel<128, true, true>, 128, smem));
        } else {
            set_leave_carveout();
            SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, leave_kernel<256>, 256, 0));
        }
        occ_cache_key[which] = key;
        occ_cache_val[which] = std::max(per_sm, 1) * nsm;
        return occ_cache_val[which];
    }
    // The leave kernel's spilled values and the mode-search tables are served by L1, which
    // shares the SM's 256 KB with shared memory: ask for the smallest shared-memory carveout
    // that keeps the kernel's full occupancy (its blocks' static shared memory plus the
    // per-block reservation), leaving the rest to L1 (3% faster a window at 384k tets than
    // the default carveout).  Falls back to the largest carveout if the smaller one
    // would cost occupancy.
    bool leave_carveout_set = false;
    void set_leave_carveout() {
        if (leave_carveout_set) return;
        auto fn = leave_kernel<256>;
        int full = 0, smem_sm = 0, resv = 0, per = 0;
        SG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&full, fn, 256, 0));
        cudaFuncAttributes fa;
        SG_CUDA(cudaFuncGetAttributes(&fa, fn));
        SG_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
        SG_CUDA(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, device));
        const long need = (long)full * ((long)fa.sharedSizeBytes + resv);
        const int pct = (int)std::min(100L, std::max(1L, (need * 100 + smem_sm - 1) / std::max(smem_sm, 1)));
        SG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 256, 0));
        if (per < full) SG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        leave_carveout_set = true;
    }
    int split_ssa_grid(size_t smem, int ntodo) {
        const long need = ((long)ntodo + block - 1) / block;
        return (int)std::max(1L, std::min(need, (long)resident_blocks(0, block, smem)));
    }
    int surf_ssa_capacity(size_t smem) { return resident_blocks(1, 128, smem); }
    int leave_grid() {
        const long need = ((long)ntets + 255) / 256;
        return (int)std::max(1L, std::min(need, (long)resident_blocks(2, 256, 0)));
    }

    void launch_window(const sg_window_args& a, int g) {
        size_t sm = window_smem();
        int chk = check_flag();
        if (has_surf() && use_split()) {
            // Membrane models: the volume-only SSA for every other tet at the volume kernel's
            // occupancy, the SURF SSA over the membrane tet list, then the diffusion leave.
            if (ndiff > 0 && (!a.tdel || !a.tmask)) throw ProgErr("split window without its buffers");
            const size_t smv = smem_bytes(block, nspec, (int)reacs.size());
            const int gv = split_ssa_grid(smv, ntets);
            switch (block) {
                case 64: window_kernel<64, false, true><<<gv, 64, smv, stream>>>(a, chk); break;
                case 128: window_kernel<128, false, true><<<gv, 128, smv, stream>>>(a, chk); break;
                case 256: window_kernel<256, false, true><<<gv, 256, smv, stream>>>(a, chk); break;
                default: throw ArgErr("block size must be 64, 128 or 256");
            }
            SG_CUDA(cudaGetLastError());
            if (nmemb_tets > 0) {
                sg_window_args am = a;
                am.tet_list = d_memb_tets.p;
                am.nlist = nmemb_tets;
                const int gm = (int)std::min<long>(((long)nmemb_tets + 127) / 128, (long)surf_ssa_capacity(sm));
                window_kernel<128, true, true><<<gm, 128, sm, stream>>>(am, chk);
                SG_CUDA(cudaGetLastError());
            }
            if (nunits > 0) {
                // One warp per unit; the tree and the propensities in shared memory when the
                // largest unit's fit.
                const int gu = std::min(nunits, nsm * 32);
                if (unit_smem <= kUnitSmemMax) {
                    unit_ssa_kernel<true><<<gu, 32, unit_smem, stream>>>(a);
                } else {
                    unit_ssa_kernel<false><<<gu, 32, 0, stream>>>(a);
                }
                SG_CUDA(cudaGetLastError());
            }
            if (nsdiff > 0) {
                const long long sp = (long long)nsdiff * ntris;
                const int gsd = (int)std::max(1LL, std::min((sp + 255) / 256, (long long)nsm * 64));
                sdiffuse_kernel<256><<<gsd, 256, 0, stream>>>(a);
                SG_CUDA(cudaGetLastError());
            }
            leave_kernel<256><<<leave_grid(), 256, 0, stream>>>(a, chk);
        } else if (has_surf()) {
            window_kernel<128, true><<<g, 128, sm, stream>>>(a, chk);
        } else if (use_split()) {
            if (ndiff > 0 && (!a.tdel || !a.tmask)) throw ProgErr("split window without its buffers");
            const int gs = split_ssa_grid(sm, ntets);
            switch (block) {
                case 64: window_kernel<64, false, true><<<gs, 64, sm, stream>>>(a, chk); break;
                case 128: window_kernel<128, false, true><<<gs, 128, sm, stream>>>(a, chk); break;
                case 256: window_kernel<256, false, true><<<gs, 256, sm, stream>>>(a, chk); break;
                default: throw ArgErr("block size must be 64, 128 or 256");
            }
            SG_CUDA(cudaGetLastError());
            leave_kernel<256><<<leave_grid(), 256, 0, stream>>>(a, chk);
        } else {
            switch (block) {
                case 64: window_kernel<64><<<g, 64, sm, stream>>>(a, chk); break;
                case 128: window_kernel<128><<<g, 128, sm, stream>>>(a, chk); break;
                case 256: window_kernel<256><<<g, 256, sm, stream>>>(a, chk); break;
                default: throw ArgErr("block size must be 64, 128 or 256");
            }
        }
        SG_CUDA(cudaGetLastError());
    }

    // ---- persistent form ----
    // Models without membrane triangles whose realizations all take the same windows.
    bool persist_ok(const std::vector<uint64_t>& k, uint64_t n) const {
        if (has_surf() || nunits > 0) return false;
        for (uint64_t x : k)
            if (x != n) return false;
        return true;
    }
    // 1/x and ln x! of the binomial mode search, read through L1 by the leave and
    // persistent kernels.
    void ensure_mode_tables() {
        if (d_mode_tab.p) return;
        d_mode_tab.alloc((size_t)2 * SG_MODE_TABLE);
        mode_tables_kernel<<<4, 256, 0, stream>>>(d_mode_tab.p, d_mode_tab.p + SG_MODE_TABLE);
        SG_CUDA(cudaGetLastError());
    }
    void ensure_persist_tables() {
        if (pchunk_tpl == persist_tpl && d_pchunk.p) return;
        const int tpw = 32 * persist_tpl;
        std::vector<int32_t> cb(nreal + 1, 0);
        for (int r = 0; r < nreal; ++r) cb[r + 1] = cb[r] + (real_begin[r + 1] - real_begin[r] + tpw - 1) / tpw;
        d_pchunk.alloc(cb.size());
        h2d(d_pchunk.p, cb.data(), cb.size());
        if (!d_pstate.p) d_pstate.alloc((size_t)2 * nreal + 1);
        ensure_mode_tables();
        if (!d_pnext.p) d_pnext.alloc(1);
        pchunks = cb[nreal];
        pchunk_tpl = persist_tpl;
    }
    template <int B, int TPL>
    void persist_launch(sg_window_args a, sg_persist_args P, size_t sm) {
        auto fn = persistent_window_kernel<B, TPL>;
        if (sm > 48 * 1024) SG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int per_sm = 0;
        SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, B, sm));
        if (per_sm < 1) throw NotImplErr("the persistent window kernel does not fit an SM");
        const long need = ((long)P.nchunks * 32 + B - 1) / B;
        const int grid = (int)std::max(1L, std::min(need, (long)per_sm * nsm));
        a.mode_rcpl = d_mode_tab.p;
        a.mode_lnf = d_mode_tab.p + SG_MODE_TABLE;
        void* args[] = {&a, &P};
        SG_CUDA(cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(B), args, sm, stream));
    }
    // nwin windows of every realization in one launch; the next ordinary window launch skips
    // its conservation check (the persistent launch keeps no per-window totals).
    void launch_persistent(const sg_window_args& a, int nwin) {
        ensure_persist_tables();
        if (ndiff > 0 && (!a.tdel || !a.tmask)) throw ProgErr("persistent window without its buffers");
        SG_CUDA(cudaMemsetAsync(d_pstate.p, 0, d_pstate.n * sizeof(unsigned int), stream));
        SG_CUDA(cudaMemsetAsync(d_pnext.p, 0, sizeof(unsigned long long), stream));
        sg_persist_args P;
        std::memset(&P, 0, sizeof(P));
        P.chunk_begin = d_pchunk.p;
        P.done = d_pstate.p;
        P.ready = d_pstate.p + nreal;
        P.abort = d_pstate.p + 2 * nreal;
        P.next = d_pnext.p;
        P.spin_limit = persist_spin_limit;
        P.nchunks = pchunks;
        P.nwin = nwin;
        P.tpw = 32 * persist_tpl;
        const int B = block >= 256 ? 256 : 128;
        const size_t sm = smem_bytes(B, nspec, std::max((int)reacs.size(), 6));
        if (B == 256) {
            switch (persist_tpl) {
                case 8: persist_launch<256, 8>(a, P, sm); break;
                case 4: persist_launch<256, 4>(a, P, sm); break;
                case 2: persist_launch<256, 2>(a, P, sm); break;
                default: persist_launch<256, 1>(a, P, sm); break;
            }
        } else {
            switch (persist_tpl) {
                case 8: persist_launch<128, 8>(a, P, sm); break;
                case 4: persist_launch<128, 4>(a, P, sm); break;
                case 2: persist_launch<128, 2>(a, P, sm); break;
                default: persist_launch<128, 1>(a, P, sm); break;
            }
        }
        SG_CUDA(cudaGetLastError());
        SG_CUDA(cudaMemsetAsync(d_launch.p + 3, 0, sizeof(unsigned long long), stream));
    }

    // ---- CUDA graph of kGraphChunk window launches, rebuilt when the launch changes ----
    static constexpr int kGraphChunk = 16;
    bool use_graphs = true;
    cudaGraphExec_t graph_exec = nullptr;
    sg_window_args graph_args{};
    int graph_grid = -1, graph_block = -1, graph_check = -1, graph_split = -1;

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }

    cudaGraphExec_t window_graph(const sg_window_args& a, int g) {
        int chk = check_flag();
        if (graph_exec && g == graph_grid && block == graph_block && chk == graph_check &&
            (int)use_split() == graph_split && std::memcmp(&a, &graph_args, sizeof(a)) == 0)
            return graph_exec;
        drop_graph();
        cudaGraph_t graph = nullptr;
        SG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            for (int i = 0; i < kGraphChunk; ++i) launch_window(a, g);
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        SG_CUDA(cudaStreamEndCapture(stream, &graph));
        cudaError_t e = cudaGraphInstantiate(&graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        SG_CUDA(e);
        graph_args = a;
        graph_grid = g;
        graph_block = block;
        graph_check = chk;
        graph_split = (int)use_split();
        return graph_exec;
    }

    // Number of windows the device time recurrence takes to reach t_end.
    static uint64_t count_windows(double t, double t_end, double period) {
        uint64_t n = 0;
        while (t < t_end) {
            t = (t + period > t_end) ? t_end : t + period;
            n += 1;
        }
        return n;
    }

    double time() const { return reals.empty() ? 0.0 : reals[0].t; }

    void run(double endtime) {
        require_setup();
        double t = time();
        if (endtime < t) throw ArgErr("Endtime is before current simulation time");
        if (almost_equal(t, endtime)) {
            for (auto& rl : reals) rl.t = endtime;
            upload_reals();
            sync();
            return;
        }
        if (ef_on) {
            run_with_efield(endtime);
            return;
        }
        enqueue_windows(endtime);
        download_reals();
        check_status();
    }

    // TOS:1851-1952 _runWithEField: per EField step, the reaction-diffusion windows up to
    // min(t + efdt, endtime), then the membrane currents and the EField solve over the
    // step actually taken; the new triangle potentials feed the next windows.
    void run_with_efield(double endtime) {
        // Batched realizations share the EField steps: their vertex systems are disjoint
        // blocks of one system, so every realization must advance on the same windows.
        for (int r = 1; r < nreal; ++r)
            if (reals[r].t != reals[0].t || reals[r].period != reals[0].period)
                throw NotImplErr("EField with batched realizations of different times or update periods");
        while (time() < endtime) {
            double t0 = time();
            double t1 = std::min(t0 + efdt, endtime);
            if (almost_equal(t1, endtime)) t1 = endtime;
            if (almost_equal(t0, t1)) {
                for (auto& rl : reals) rl.t = t1;
                upload_reals();
                break;
            }
            enqueue_windows(t1);
            download_reals();
            check_status();
            double real_dt = time() - t0;
            // Membrane currents of the step from the channel-state time integrals.
            if (has_surf() && (!ohmics.empty() || !ghks.empty())) {
                int g = std::max(1, std::min((ntris + 255) / 256, nsm * 4));
                ohmic_current_kernel<<<g, 256, 0, stream>>>(ntris, nsspec, (int)ohmics.size(), d_ohmics.p,
                                                            d_tri_patch.p, d_spec_int.p, ef.tri_V, 1.0 / real_dt,
                                                            ef.tri_I, d_tri_Iohm.p, d_tri_echarge.p, d_tri_Ighk.p);
                SG_CUDA(cudaGetLastError());
                launches += 1;
            } else {
                SG_CUDA(cudaMemsetAsync(ef.tri_I, 0, std::max(ef.ntris, 1) * 8, stream));
                if (has_surf()) SG_CUDA(cudaMemsetAsync(d_spec_int.p, 0, d_spec_int.n * 8, stream));
            }
            ef.advance(real_dt * 1.0e3, stream);  // efield.cpp:229-234: s -> ms
        }
        sync();
    }

    void require_ef() const {
        if (!ef_on) throw ProgErr("Method not available: this solver has no membrane potential");
    }
    void check_vert(int v) const {
        if (v < 0 || v >= ef.nverts) throw ArgErr("vertex index out of range: " + std::to_string(v));
    }
    double get_vert_v(int v) {
        require_ef();
        check_vert(v);
        double x = 0.0;
        d2h(&x, ef.V + ef.vid(v), 1);
        sync();
        return x * 1.0e-3;  // mV -> V
    }
    void set_vert_v(int v, double volts) {
        require_ef();
        check_vert(v);
        double x = volts * 1.0e3;
        h2d(ef.V + ef.vid(v), &x, 1);
        sync();
    }
    double get_tri_v(int t) {
        require_ef();
        if (t < 0 || t >= ef.ntris) throw ArgErr("membrane triangle index out of range");
        double x = 0.0;
        d2h(&x, ef.tri_V + t, 1);
        sync();
        return x * 1.0e-3;
    }

    // ---- launch-shape autotuning ----
    // The sample path does not depend on the launch shape (every tet draws from its own
    // counter streams), so tuning runs real windows.  After one untimed window, each of a
    // fixed list of candidates is timed on one window in list order and on one more in
    // reverse order (a palindromic schedule, so that the drift of the per-window work as
    // the run evolves cancels to first order): block {64, 128, 256} x grid {occupancy-
    // sized, one tet per thread}; block 256, one tet per thread at a shared-memory carveout
    // of 75%; split windows at block 128 and 256; the persistent form at block 256 with 64,
    // 128 and 256 tets per work chunk (2, 4, 8 tets per lane), when every realization takes
    // the same windows.  The fastest is kept.
    static constexpr int kTuneWindows = 2;
    static constexpr int kTuneCands = 12;
    static constexpr uint64_t kPersistMaxWindows = 64;  // windows per persistent launch
    bool tune_pending = false;
    std::vector<float> tune_ms;
    int carveout = 100;  // preferred shared-memory carveout of the window kernels, percent

    void set_carveout(int pct) {
        carveout = pct;
        SG_CUDA(cudaFuncSetAttribute(window_kernel<64>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<128>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<256>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<64, false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<128, false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<256, false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<128, true>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        SG_CUDA(cudaFuncSetAttribute(window_kernel<128, true, true>, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    }

    uint64_t autotune(const sg_window_args& a, bool persist_allowed) {
        struct Cand {
            int block, grid, carve;
            bool split;
            int ptpl;  // > 0: persistent form with this many tets per lane
        };
        const Cand cands[kTuneCands] = {{64, 0, 100, false, 0},   {64, -1, 100, false, 0},
                                        {128, 0, 100, false, 0},  {128, -1, 100, false, 0},
                                        {256, 0, 100, false, 0},  {256, -1, 100, false, 0},
                                        {256, -1, 75, false, 0},  {128, -1, 100, true, 0},
                                        {256, -1, 100, true, 0},  {256, 0, 100, false, 2},
                                        {256, 0, 100, false, 4},  {256, 0, 100, false, 8}};
        tune_ms.assign(kTuneCands, 0.0f);
        cudaEvent_t e0, e1;
        SG_CUDA(cudaEventCreate(&e0));
        SG_CUDA(cudaEventCreate(&e1));
        ensure_split_buffers();
        const sg_window_args as = window_args();  // with the split buffers
        auto timed = [&](const Cand& c) {
            block = c.block;
            grid = c.grid;
            split = c.split;
            set_carveout(c.carve);
            const int g = window_grid();
            SG_CUDA(cudaEventRecord(e0, stream));
            if (c.ptpl > 0 && persist_allowed) {
                persist_tpl = c.ptpl;
                launch_persistent(as, 1);
            } else {
                launch_window(as, g);
            }
            SG_CUDA(cudaEventRecord(e1, stream));
            SG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            return ms;
        };
        timed(cands[5]);  // untimed: first-launch costs
        for (int i = 0; i < kTuneCands; ++i) tune_ms[i] += timed(cands[i]);
        for (int i = kTuneCands - 1; i >= 0; --i) tune_ms[i] += timed(cands[i]);
        int best = 0;
        for (int i = 1; i < kTuneCands; ++i)
            if (tune_ms[i] < tune_ms[best] && (cands[i].ptpl == 0 || persist_allowed)) best = i;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        block = cands[best].block;
        grid = cands[best].grid;
        split = cands[best].split;
        persist = cands[best].ptpl > 0;
        if (persist) persist_tpl = cands[best].ptpl;
        set_carveout(cands[best].carve);
        tune_pending = false;
        return (uint64_t)kTuneWindows * kTuneCands + 1;
    }

    // Enqueue every window up to endtime for all realizations (no host sync).
    uint64_t enqueue_windows(double endtime) {
        uint64_t n = 0;
        std::vector<uint64_t> k(nreal);
        for (int r = 0; r < nreal; ++r) {
            reals[r].t_end = endtime;
            k[r] = count_windows(reals[r].t, endtime, reals[r].period);
            n = std::max(n, k[r]);
        }
        upload_reals();
        if (n == 0) return 0;
        sg_window_args a = window_args();
        uint64_t done = 0;
        const bool pok = persist_ok(k, n);
        if (tune_pending && !has_surf() && n > (uint64_t)kTuneWindows * kTuneCands + 1) {
            done = autotune(a, pok);
            a = window_args();  // the tuner may have allocated the split buffers
        }
        if (use_split() || (persist && pok)) {
            ensure_split_buffers();
            a = window_args();
        }
        int g = window_grid();
        if (profiling) SG_CUDA(cudaEventRecord(ev_begin, stream));
        if (persist && pok) {
            // Persistent form: up to kPersistMaxWindows windows of every realization per launch.
            while (done < n) {
                const uint64_t nw = std::min(n - done, kPersistMaxWindows);
                launch_persistent(a, (int)nw);
                done += nw;
                launches += 1;
            }
        } else {
            // Windows advance their own time on the device, so a captured chunk of window
            // launches replays unchanged; the remainder is launched directly.
            if (use_graphs && n - done >= (uint64_t)kGraphChunk) {
                cudaGraphExec_t ge = window_graph(a, g);
                for (; done + kGraphChunk <= n; done += kGraphChunk) SG_CUDA(cudaGraphLaunch(ge, stream));
            }
            for (; done < n; ++done) launch_window(a, g);
            launches += n * (uint64_t)kernels_per_window();
        }
        if (profiling) {
            SG_CUDA(cudaEventRecord(ev_end, stream));
            SG_CUDA(cudaEventSynchronize(ev_end));
            float ms = 0.0f;
            SG_CUDA(cudaEventElapsedTime(&ms, ev_begin, ev_end));
            prof_ms += ms;
            prof_windows += n;
        }
        for (int r = 0; r < nreal; ++r) {
            reals[r].window += k[r];
            if (k[r]) reals[r].pending = 1;
            reals[r].t = endtime;
        }
        niteration += n;
        pending_host = true;
        return n;
    }

    void check_status() {
        uint32_t st = 0;
        d2h(&st, d_status.p, 1);
        sync();
        if (st) {
            SG_CUDA(cudaMemsetAsync(d_status.p, 0, 4, stream));
            sync();
            std::string m = "device status error:";
            if (st & SG_ERR_CONSERVATION) m += " molecule conservation violated;";
            if (st & SG_ERR_OVERFLOW) m += " count overflow;";
            if (st & SG_ERR_NEGATIVE) m += " negative count;";
            if (st & SG_ERR_TABLE) m += " table index out of range;";
            if (st & SG_ERR_CG) m += " EField CG did not converge;";
            if (st & SG_ERR_WAIT) m += " a persistent window launch gave up waiting on a realization;";
            throw DeviceErr(m);
        }
    }

    // Gather the pending inflow so that counts are complete (getters, setters).
    void flush() {
        if (!pending_host) return;
        sg_window_args a = window_args();
        int g = std::min((ntets + 255) / 256, nsm * 8);
        flush_kernel<<<std::max(g, 1), 256, 0, stream>>>(a);
        SG_CUDA(cudaGetLastError());
        if (nsdiff > 0) {
            const int gs = std::max(1, std::min((int)(((long long)nsdiff * ntris + 255) / 256), nsm * 8));
            sflush_kernel<<<gs, 256, 0, stream>>>(a);
            SG_CUDA(cudaGetLastError());
            launches += 1;
        }
        clear_pending_kernel<<<(nreal + 255) / 256, 256, 0, stream>>>(d_reals.p, nreal);
        SG_CUDA(cudaGetLastError());
        launches += 2;
        for (auto& rl : reals) rl.pending = 0;
        pending_host = false;
        sync();
        check_status();
    }

    // A host write to the counts breaks the window-to-window conservation link.
    void invalidate_check() {
        static const unsigned long long zero = 0ull;
        h2d(d_launch.p + 3, &zero, 1);
    }

    // ------------------------------------------------------------------
    // Host placement stream: one fresh Philox stream per setter call.
    // ------------------------------------------------------------------
    sg_stream setup_stream() {
        sg_stream st;
        sg_stream_init(&st, seed, 0u, (uint32_t)(setup_calls & 0xFFFFFFFFu), setup_calls >> 32,
                       SG_PURPOSE_SETUP);
        setup_calls += 1;
        return st;
    }

    // Stochastic rounding of a fractional count (TOS:3849-3890 _setTetSpecCount).
    static uint32_t round_count(double n, sg_stream* st) {
        if (!(n >= 0.0)) throw ArgErr("count must be non-negative");
        if (n > 4294967295.0)
            throw ArgErr("Can't set count greater than maximum unsigned integer (4294967295).");
        double ni = std::floor(n);
        double fr = n - ni;
        uint32_t c = (uint32_t)ni;
        if (fr > 0.0 && sg_u01_co(sg_next_u32(st)) < fr) c += 1;
        return c;
    }

    std::vector<uint32_t> row(int s) {
        std::vector<uint32_t> v(ntets);
        d2h(v.data(), d_counts.p + (size_t)s * ntets, ntets);
        sync();
        return v;
    }
    void put_row(int s, const std::vector<uint32_t>& v) {
        h2d(d_counts.p + (size_t)s * ntets, v.data(), (size_t)ntets);
        invalidate_check();
        sync();
    }

    double get_tet_count(int t, int s) {
        require_setup();
        check_tet(t);
        check_spec(s);
        flush();
        uint32_t c = 0;
        d2h(&c, d_counts.p + (size_t)s * ntets + t, 1);
        sync();
        return (double)c;
    }

    void set_tet_count(int t, int s, double n) {
        require_setup();
        check_tet(t);
        check_spec(s);
        if (tet_comp[t] < 0) throw ArgErr("Species undefined in tetrahedron.");
        flush();
        sg_stream st = setup_stream();
        uint32_t c = round_count(n, &st);
        h2d(d_counts.p + (size_t)s * ntets + t, &c, 1);
        invalidate_check();
        sync();
    }

    // Tets of compartment c (in realization r, or in all realizations when r < 0).
    std::vector<int> comp_tets(int c, int r) const {
        std::vector<int> v;
        int b = r < 0 ? 0 : real_begin[r], e = r < 0 ? ntets : real_begin[r + 1];
        for (int t = b; t < e; ++t)
            if (tet_comp[t] == c) v.push_back(t);
        return v;
    }

    double get_comp_count(int c, int s, int r) {
        require_setup();
        check_comp(c);
        check_spec(s);
        if (r >= 0) check_real(r);
        flush();
        std::vector<uint32_t> v = row(s);
        unsigned long long sum = 0;
        for (int t : comp_tets(c, r)) sum += v[t];
        return (double)sum;
    }

    // util::distribute_quantity (src/steps/util/distribute.hpp:102-193): volume-weighted
    // floor allocation, then the remainder placed by adjusted Pareto order sampling
    // (src/steps/math/sample.hpp:59-200) with the fractional parts as inclusion weights.
    void distribute(double x, const std::vector<int>& tets, std::vector<uint32_t>& v, sg_stream* st) {
        distribute_w(x, tets, vol, v, st);
    }

    // Same rule with weights w (tet volumes for compartments, triangle areas for patches).
    void distribute_w(double x, const std::vector<int>& tets, const std::vector<double>& vol,
                      std::vector<uint32_t>& v, sg_stream* st) {
        if (tets.empty()) return;
        if (x == 0.0) {
            for (int t : tets) v[t] = 0;
            return;
        }
        double total = 0.0;
        for (int t : tets) total += vol[t];
        if (!(total > 0.0)) throw ArgErr("cannot place molecules: the elements to fill have no volume (or area)");
        if (sg_u01_co(sg_next_u32(st)) < x - std::floor(x))
            x = 1.0 + std::floor(x);
        else
            x = std::floor(x);
        double xot = x / total;
        unsigned long long allocated = 0;
        std::vector<double> pi(tets.size());
        for (size_t i = 0; i < tets.size(); ++i) {
            double xi = xot * vol[tets[i]];
            double fl = std::floor(xi);
            pi[i] = xi - fl;
            v[tets[i]] = (uint32_t)fl;
            allocated += (unsigned long long)fl;
        }
        if ((double)allocated > x) throw ProgErr("placement: the rounded-down shares add up to more than the count placed");
        size_t rem = (size_t)(x - (double)allocated);
        if (rem == 0) return;
        // Adjusted Pareto order sampling: rank Q_i = q_i U_i / (1 - U_i), keep the rem smallest.
        double psum = 0.0;
        for (double p : pi) psum += p;
        double rescale = (double)rem / psum;
        double d = 0.0;
        for (double& p : pi) {
            p *= rescale;
            if (p > 1.0) p = 1.0;
            d += p * (1.0 - p);
        }
        double ood2 = (d == 0.0) ? 1.0 : 1.0 / (d * d);
        std::vector<std::pair<double, size_t>> keys;
        keys.reserve(tets.size());
        for (size_t i = 0; i < tets.size(); ++i) {
            double q = pi[i];
            if (q == 0.0) continue;
            double loga = q * (1.0 - q) * (q - 0.5) * ood2;
            double aa = 1.0 + loga + 0.5 * loga * loga;
            double qc = (1.0 - q) / q * aa;
            double u = sg_u01_co(sg_next_u32(st));
            keys.emplace_back(qc * u / (1.0 - u), i);
        }
        if (keys.size() < rem) rem = keys.size();
        if (rem == 0) return;
        std::nth_element(keys.begin(), keys.begin() + (rem - 1), keys.end());
        for (size_t j = 0; j < rem; ++j) v[tets[keys[j].second]] += 1;
    }

    void set_comp_count(int c, int s, double n, int r) {
        require_setup();
        check_comp(c);
        check_spec(s);
        if (r >= 0) check_real(r);
        if (!(n >= 0.0)) throw ArgErr("count must be non-negative");
        if (n > 4294967295.0) throw ArgErr("count exceeds the maximum unsigned integer");
        flush();
        std::vector<uint32_t> v = row(s);
        int rb = r < 0 ? 0 : r, re = r < 0 ? nreal : r + 1;
        for (int rr = rb; rr < re; ++rr) {
            sg_stream st = setup_stream();
            distribute(n, comp_tets(c, rr), v, &st);
        }
        put_row(s, v);
    }

    // getBatchTetSpecCountsNP (TOS:5715) without moving the whole row.
    DevBuf<int32_t> d_gidx;
    DevBuf<double> d_gout;
    void get_batch_tet_counts(int s, const int32_t* tets, int n, double* out) {
        require_setup();
        check_spec(s);
        if (n < 0) throw ArgErr("negative count of tets");
        if (n == 0) return;
        for (int i = 0; i < n; ++i) check_tet(tets[i]);
        flush();
        if (d_gidx.n < (size_t)n) {
            d_gidx.alloc(n);
            d_gout.alloc(n);
        }
        h2d(d_gidx.p, tets, (size_t)n);
        const int g = std::max(1, std::min((n + 255) / 256, nsm * 8));
        gather_counts_kernel<<<g, 256, 0, stream>>>(n, d_counts.p + (size_t)s * ntets, d_gidx.p, d_gout.p);
        SG_CUDA(cudaGetLastError());
        launches += 1;
        d2h(out, d_gout.p, (size_t)n);
        sync();
    }

    void get_spec_row(int s, uint32_t* out) {
        require_setup();
        check_spec(s);
        flush();
        d2h(out, d_counts.p + (size_t)s * ntets, ntets);
        sync();
    }

    void set_spec_row(int s, const uint32_t* in) {
        require_setup();
        check_spec(s);
        flush();
        h2d(d_counts.p + (size_t)s * ntets, in, (size_t)ntets);
        invalidate_check();
        sync();
    }

    void get_all_rows(uint32_t* out) {
        require_setup();
        flush();
        d2h(out, d_counts.p, (size_t)nspec * ntets);
        sync();
    }

    void set_all_rows(const uint32_t* in) {
        require_setup();
        flush();
        h2d(d_counts.p, in, (size_t)nspec * ntets);
        invalidate_check();
        sync();
    }

    void set_tet_clamped(int t, int s, bool on) {
        require_setup();
        check_tet(t);
        check_spec(s);
        flush();
        if (on)
            clampm[t] |= (1u << s);
        else
            clampm[t] &= ~(1u << s);
        any_clamp = false;
        for (uint32_t m : clampm)
            if (m) any_clamp = true;
        h2d(d_clamp.p + t, &clampm[t], 1);
        invalidate_check();
        sync();
    }

    void check_reac(int user_reac) const {
        if (user_reac < 0 || user_reac >= (int)reacs.size()) throw ArgErr("reaction index out of range");
    }

    void set_reac_k(int user_reac, int r, double k) {
        require_setup();
        check_reac(user_reac);
        if (r >= 0) check_real(r);
        if (!(k >= 0.0)) throw ArgErr("reaction constant must be non-negative");
        int slot = reac_order_user[user_reac];
        const int R = (int)reacs.size();
        int rb = r < 0 ? 0 : r, re = r < 0 ? nreal : r + 1;
        for (int rr = rb; rr < re; ++rr) kcst[(size_t)rr * R + slot] = k;
        h2d(d_kcst.p, kcst.data(), kcst.size());
        sync();
    }

    double get_reac_k(int user_reac, int r) const {
        check_reac(user_reac);
        if (r >= 0) check_real(r);
        return kcst[(size_t)std::max(r, 0) * reacs.size() + reac_order_user[user_reac]];
    }

    void set_diff_d(int c, int s, double d, int r) {
        require_setup();
        check_comp(c);
        check_spec(s);
        if (r >= 0) check_real(r);
        if (!(d >= 0.0)) throw ArgErr("diffusion constant must be non-negative");
        if (diff_slot[s] < 0) throw ArgErr("species has no diffusion rule");
        flush();
        int rb = r < 0 ? 0 : r, re = r < 0 ? nreal : r + 1;
        for (int rr = rb; rr < re; ++rr) dcst[((size_t)rr * ncomp + c) * nspec + s] = d;
        upload_params();
        sync();
    }

    // ---- membrane triangle counts (TOS:4831 getTriSpecCount, setTriSpecCount; patch
    //      counts distributed by triangle area as setPatchSpecCount) ----
    void check_tri(int m, int s) const {
        if (!has_surf()) throw ProgErr("no membrane triangles in this solver");
        if (m < 0 || m >= ntris) throw ArgErr("triangle index out of range: " + std::to_string(m));
        if (s < 0 || s >= nsspec) throw ArgErr("surface species index out of range: " + std::to_string(s));
    }
    double get_tri_count(int m, int s) {
        check_tri(m, s);
        flush();
        uint32_t c = 0;
        d2h(&c, d_tri_counts.p + (size_t)s * ntris + m, 1);
        sync();
        return (double)c;
    }
    void set_tri_count(int m, int s, double n) {
        check_tri(m, s);
        flush();
        sg_stream st = setup_stream();
        uint32_t c = round_count(n, &st);
        h2d(d_tri_counts.p + (size_t)s * ntris + m, &c, 1);
        sync();
    }
    // A triangle belongs to the realization of its inner tet; real = -1 selects all.
    bool tri_in(int m, int p, int real) const {
        if (tri_patch[m] != p) return false;
        if (real < 0) return true;
        return tri_inner[m] >= real_begin[real] && tri_inner[m] < real_begin[real + 1];
    }
    double get_patch_count(int p, int s, int real) {
        check_tri(0, s);
        if (real >= 0) check_real(real);
        flush();
        std::vector<uint32_t> v(ntris);
        d2h(v.data(), d_tri_counts.p + (size_t)s * ntris, ntris);
        sync();
        unsigned long long sum = 0;
        for (int m = 0; m < ntris; ++m)
            if (tri_in(m, p, real)) sum += v[m];
        return (double)sum;
    }
    void set_patch_count(int p, int s, int real, double n) {
        check_tri(0, s);
        if (p < 0 || p >= npatch) throw ArgErr("patch index out of range");
        if (real >= 0) check_real(real);
        flush();
        if (!(n >= 0.0) || n > 4294967295.0) throw ArgErr("count out of range");
        std::vector<uint32_t> v(ntris);
        d2h(v.data(), d_tri_counts.p + (size_t)s * ntris, ntris);
        sync();
        std::vector<int> tris;
        for (int m = 0; m < ntris; ++m)
            if (tri_in(m, p, real)) tris.push_back(m);
        sg_stream st = setup_stream();
        distribute_w(n, tris, tri_area, v, &st);
        h2d(d_tri_counts.p + (size_t)s * ntris, v.data(), (size_t)ntris);
        sync();
    }
    double get_tri_ghk_i(int m) {
        check_tri(m, 0);
        if (ghks.empty()) return 0.0;
        double x = 0.0;
        d2h(&x, d_tri_Ighk.p + m, 1);
        sync();
        return x;
    }
    double get_tri_ohmic_i(int m) {
        check_tri(m, 0);
        double x = 0.0;
        d2h(&x, d_tri_Iohm.p + m, 1);
        sync();
        return x * 1.0e-12;  // pA -> A
    }

    unsigned long long reac_extent(int user_reac) {
        require_setup();
        check_reac(user_reac);
        unsigned long long v = 0;
        d2h(&v, d_ext_total.p + reac_order_user[user_reac], 1);
        sync();
        return v;
    }
    unsigned long long diff_extent() {
        require_setup();
        unsigned long long v = 0;
        d2h(&v, d_diff_total.p, 1);
        sync();
        return v;
    }
    unsigned long long nsteps() {
        unsigned long long v = diff_extent();
        for (int i = 0; i < (int)reacs.size(); ++i) v += reac_extent(i);
        return v;
    }

    // ---- checkpoint / restore (TOS:217-451 checkpoint, restore) ----
    // Binary file: a header of sizes (checked on restore against this solver's mesh and
    // model), then every state array, each preceded by its element count and size.  The
    // pending inflow is applied first, so counts are complete.  Random streams are keyed by
    // (seed, realization, tet, window), so restoring the window indices and the seed makes
    // the continuation identical to the uninterrupted run.
    struct CkptHeader {
        char magic[8];
        uint32_t version;
        int32_t ntets, nspec, nreal, ncomp, nreac, ntris, nsspec, nverts, nsreac, nbnd;
        uint64_t seed, niteration, setup_calls;
        double efdt;
    };

    template <typename T>
    static void put(FILE* f, const T* p, size_t n) {
        uint64_t hd[2] = {(uint64_t)n, (uint64_t)sizeof(T)};
        if (std::fwrite(hd, sizeof(hd), 1, f) != 1 || (n && std::fwrite(p, sizeof(T), n, f) != n))
            throw ProgErr("checkpoint: write failed");
    }
    template <typename T>
    static void get(FILE* f, T* p, size_t n, const char* what) {
        uint64_t hd[2] = {0, 0};
        if (std::fread(hd, sizeof(hd), 1, f) != 1 || hd[0] != n || hd[1] != sizeof(T))
            throw ArgErr(std::string("checkpoint does not match this solver (") + what + ")");
        if (n && std::fread(p, sizeof(T), n, f) != n) throw ArgErr("checkpoint: truncated file");
    }
    template <typename T>
    void put_dev(FILE* f, const T* dp, size_t n) {
        std::vector<T> h(n);
        if (n) d2h(h.data(), dp, n);
        sync();
        put(f, h.data(), n);
    }
    template <typename T>
    void get_dev(FILE* f, T* dp, size_t n, const char* what) {
        std::vector<T> h(n);
        get(f, h.data(), n, what);
        if (n) h2d(dp, h.data(), n);
        sync();
    }

    CkptHeader ckpt_header() const {
        CkptHeader hd{};
        std::memcpy(hd.magic, "SGB2CKPT", 8);
        hd.version = 1;
        hd.ntets = ntets;
        hd.nspec = nspec;
        hd.nreal = nreal;
        hd.ncomp = ncomp;
        hd.nreac = (int32_t)reacs.size();
        hd.ntris = ntris;
        hd.nsspec = nsspec;
        hd.nverts = ef_on ? ef.nverts : 0;
        hd.nsreac = (int32_t)sreacs.size();
        hd.nbnd = nbnd;
        hd.seed = seed;
        hd.niteration = niteration;
        hd.setup_calls = setup_calls;
        hd.efdt = efdt;
        return hd;
    }

    void checkpoint(const std::string& path) {
        require_setup();
        flush();
        download_reals();
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) throw ArgErr("cannot open checkpoint file for writing: " + path);
        try {
            CkptHeader hd = ckpt_header();
            put(f, &hd, 1);
            put(f, reals.data(), reals.size());
            put(f, kcst.data(), kcst.size());
            put(f, dcst.data(), dcst.size());
            put(f, clampm.data(), clampm.size());
            put_dev(f, d_counts.p, d_counts.n);
            put_dev(f, d_totals.p, d_totals.n);
            put_dev(f, d_ext.p, d_ext.n);
            put_dev(f, d_ext_total.p, d_ext_total.n);
            put_dev(f, d_diff_total.p, d_diff_total.n);
            put_dev(f, d_launch.p, d_launch.n);
            if (nbnd > 0) {
                put(f, bact.data(), bact.size());
                put(f, bdcst.data(), bdcst.size());
            }
            if (has_surf()) {
                put(f, skcst.data(), skcst.size());
                put_dev(f, d_tri_counts.p, d_tri_counts.n);
                put_dev(f, d_spec_int.p, d_spec_int.n);
                put_dev(f, d_tri_Iohm.p, d_tri_Iohm.n);
                put_dev(f, d_surf_ext.p, d_surf_ext.n);
            }
            if (ef_on) {
                const int nv = ef.nverts;
                double mp[4] = {ef.cm, ef.sigma, ef.g_leak, ef.v_leak};
                put(f, mp, 4);
                put(f, ef.vclamped.data(), ef.vclamped.size());
                put(f, ef.vert_iclamp.data(), ef.vert_iclamp.size());
                put(f, ef.tri_iclamp.data(), ef.tri_iclamp.size());
                put_dev(f, ef.V, (size_t)nv);
                put_dev(f, ef.x, (size_t)nv);  // warm start of the next solve
                put_dev(f, ef.tri_V, (size_t)ef.ntris);
            }
        } catch (...) {
            std::fclose(f);
            throw;
        }
        if (std::fclose(f) != 0) throw ProgErr("checkpoint: close failed");
    }

    void restore(const std::string& path) {
        require_setup();
        flush();
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) throw ArgErr("cannot open checkpoint file: " + path);
        try {
            CkptHeader hd{};
            get(f, &hd, 1, "header");
            CkptHeader me = ckpt_header();
            if (std::memcmp(hd.magic, me.magic, 8) != 0 || hd.version != 1) throw ArgErr("not a checkpoint file");
            if (hd.ntets != me.ntets || hd.nspec != me.nspec || hd.nreal != me.nreal || hd.ncomp != me.ncomp ||
                hd.nreac != me.nreac || hd.ntris != me.ntris || hd.nsspec != me.nsspec || hd.nverts != me.nverts ||
                hd.nsreac != me.nsreac || hd.nbnd != me.nbnd)
                throw ArgErr("checkpoint was written by a solver with another mesh or model");
            get(f, reals.data(), reals.size(), "realizations");
            get(f, kcst.data(), kcst.size(), "reaction constants");
            get(f, dcst.data(), dcst.size(), "diffusion constants");
            get(f, clampm.data(), clampm.size(), "clamps");
            any_clamp = false;
            for (uint32_t m : clampm)
                if (m) any_clamp = true;
            h2d(d_clamp.p, clampm.data(), clampm.size());
            h2d(d_kcst.p, kcst.data(), kcst.size());
            h2d(d_dcst.p, dcst.data(), dcst.size());
            upload_reals();
            get_dev(f, d_counts.p, d_counts.n, "counts");
            get_dev(f, d_totals.p, d_totals.n, "totals");
            get_dev(f, d_ext.p, d_ext.n, "extents");
            get_dev(f, d_ext_total.p, d_ext_total.n, "extents");
            get_dev(f, d_diff_total.p, d_diff_total.n, "diffusion extent");
            get_dev(f, d_launch.p, d_launch.n, "launch state");
            // The counters of the next window's parity are zero between windows.
            SG_CUDA(cudaMemsetAsync(d_work.p, 0, 32, stream));
            if (nbnd > 0) {
                get(f, bact.data(), bact.size(), "diffusion boundaries");
                get(f, bdcst.data(), bdcst.size(), "diffusion boundary constants");
                for (size_t i = 0; i < btab.size(); ++i)
                    btab[i] = bact[i] ? (bdcst[i] >= 0.0 ? bdcst[i] : -2.0) : -1.0;
                h2d(d_btab.p, btab.data(), btab.size());
            }
            if (has_surf()) {
                get(f, skcst.data(), skcst.size(), "surface constants");
                h2d(d_skcst.p, skcst.data(), skcst.size());
                get_dev(f, d_tri_counts.p, d_tri_counts.n, "triangle counts");
                get_dev(f, d_spec_int.p, d_spec_int.n, "channel integrals");
                get_dev(f, d_tri_Iohm.p, d_tri_Iohm.n, "ohmic currents");
                get_dev(f, d_surf_ext.p, d_surf_ext.n, "surface extents");
            }
            if (ef_on) {
                const int nv = ef.nverts;
                double mp[4];
                get(f, mp, 4, "membrane");
                ef.cm = mp[0];
                ef.sigma = mp[1];
                ef.g_leak = mp[2];
                ef.v_leak = mp[3];
                get(f, ef.vclamped.data(), ef.vclamped.size(), "vertex clamps");
                get(f, ef.vert_iclamp.data(), ef.vert_iclamp.size(), "vertex current clamps");
                get(f, ef.tri_iclamp.data(), ef.tri_iclamp.size(), "triangle current clamps");
                get_dev(f, ef.V, (size_t)nv, "potentials");
                get_dev(f, ef.x, (size_t)nv, "EField warm start");
                get_dev(f, ef.tri_V, (size_t)ef.ntris, "triangle potentials");
                ef.dirty = true;
            }
            niteration = hd.niteration;
            setup_calls = hd.setup_calls;
            efdt = hd.efdt;
            pending_host = false;
        } catch (...) {
            std::fclose(f);
            throw;
        }
        std::fclose(f);
        drop_graph();
        sync();
    }
};

}  // namespace sg

// ===========================================================================
// C ABI.  Every entry point returns an sg_status; the message of the last
// failure on the calling thread is available from sg_last_error().
// ===========================================================================
using sg::Solver;

static thread_local std::string g_last_error;

void sg::set_last_error(const std::string& msg) { g_last_error = msg; }

template <typename F>
static int guarded(F&& f) {
    try {
        f();
        return SG_OK;
    } catch (const sg::ArgErr& e) {
        g_last_error = e.what();
        return SG_EARG;
    } catch (const sg::NotImplErr& e) {
        g_last_error = e.what();
        return SG_ENOTIMPL;
    } catch (const sg::CudaErr& e) {
        g_last_error = e.what();
        return SG_ECUDA;
    } catch (const sg::DeviceErr& e) {
        g_last_error = e.what();
        return SG_EDEVICE;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return SG_EPROG;
    }
}

static Solver* S(sg_solver* h) {
    if (!h) throw sg::ArgErr("null solver handle");
    return reinterpret_cast<Solver*>(h);
}

template <typename T>
static void need(T* p, const char* what) {
    if (!p) throw sg::ArgErr(std::string("null pointer: ") + what);
}

extern "C" {

const char* sg_last_error(void) { return g_last_error.c_str(); }

int sg_version(void) { return SG_ABI_VERSION; }

int sg_create(sg_solver** out, uint64_t seed, int device) {
    return guarded([&] {
        need(out, "out");
        *out = reinterpret_cast<sg_solver*>(new Solver(seed, device));
    });
}

int sg_destroy(sg_solver* h) {
    return guarded([&] { delete S(h); });
}

int sg_set_nspecs(sg_solver* h, int32_t nspec) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (nspec <= 0 || nspec > 32) throw sg::ArgErr("volume species count must be in 1..32");
        if (!s->reacs.empty() || !s->diff_spec.empty())
            throw sg::ProgErr("species count must be set before reactions and diffusions");
        s->nspec = nspec;
        s->dcst_def.assign((size_t)s->ncomp * nspec, 0.0);
    });
}

int sg_set_mesh(sg_solver* h, int32_t ntets, const double* vol, const int32_t* neighb,
                const double* area, const double* dist, const int32_t* tet_comp, int32_t ncomp) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        need(vol, "vol");
        need(neighb, "neighb");
        need(area, "area");
        need(dist, "dist");
        need(tet_comp, "tet_comp");
        if (ntets <= 0) throw sg::ArgErr("ntets must be positive");
        if (ntets >= (1 << 29)) throw sg::ArgErr("at most 2^29 - 1 tetrahedra per solver");
        if (ncomp <= 0) throw sg::ArgErr("at least one compartment is required");
        if (!s->reacs.empty() || !s->diff_spec.empty())
            throw sg::ProgErr("mesh must be set before reactions and diffusions");
        for (int32_t i = 0; i < ntets; ++i)
            if (tet_comp[i] < -1 || tet_comp[i] >= ncomp) throw sg::ArgErr("tet compartment index out of range");
        s->ntets = ntets;
        s->ncomp = ncomp;
        s->vol.assign(vol, vol + ntets);
        s->neighb.assign(neighb, neighb + (size_t)ntets * 4);
        s->area.assign(area, area + (size_t)ntets * 4);
        s->dist.assign(dist, dist + (size_t)ntets * 4);
        s->tet_comp.assign(tet_comp, tet_comp + ntets);
        s->real_begin = {0, ntets};
        s->nreal = 1;
        s->dcst_def.assign((size_t)ncomp * std::max(s->nspec, 0), 0.0);
    });
}

int sg_set_diff_boundaries(sg_solver* h, int32_t nbnd, const int32_t* face_bnd, const int32_t* bnd_comps) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->ntets <= 0) throw sg::ProgErr("set the mesh first");
        if (nbnd < 0 || nbnd > 254) throw sg::ArgErr("at most 254 diffusion boundaries");
        if (nbnd == 0) {
            s->nbnd = 0;
            return;
        }
        need(face_bnd, "face_bnd");
        need(bnd_comps, "bnd_comps");
        s->nbnd = nbnd;
        s->face_bnd.assign(face_bnd, face_bnd + (size_t)s->ntets * 4);
        s->bnd_comps.assign(bnd_comps, bnd_comps + (size_t)nbnd * 2);
        for (int32_t c : s->bnd_comps)
            if (c < 0 || c >= s->ncomp) throw sg::ArgErr("boundary compartment out of range");
    });
}

int sg_set_diff_boundary_active(sg_solver* h, int32_t bnd, int32_t spec, int32_t active) {
    return guarded([&] { S(h)->set_bnd_active(bnd, spec, active != 0); });
}

int sg_get_diff_boundary_active(sg_solver* h, int32_t bnd, int32_t spec, int32_t* active) {
    return guarded([&] {
        need(active, "active");
        *active = S(h)->get_bnd_active(bnd, spec) ? 1 : 0;
    });
}

int sg_set_diff_boundary_dcst(sg_solver* h, int32_t bnd, int32_t spec, double dcst, int32_t direction_comp) {
    return guarded([&] { S(h)->set_bnd_dcst(bnd, spec, dcst, direction_comp); });
}

int sg_add_reac(sg_solver* h, int32_t comp, const uint32_t* lhs, const int32_t* upd, double kcst,
                int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->nspec <= 0 || s->ntets <= 0) throw sg::ProgErr("set species count and mesh first");
        s->check_comp(comp);
        need(lhs, "lhs");
        need(upd, "upd");
        if (!(kcst >= 0.0)) throw sg::ArgErr("reaction constant must be non-negative");
        sg_reac r;
        std::memset(&r, 0, sizeof(r));
        r.comp = comp;
        for (int i = 0; i < s->nspec; ++i) {
            if (lhs[i] == 0) continue;
            if (lhs[i] > 4) throw sg::ArgErr("reactant stoichiometry above 4 is not supported");
            if (r.nlhs == SG_MAX_LHS) throw sg::ArgErr("more than 4 distinct reactants");
            r.lhs_spec[r.nlhs] = i;
            r.lhs_ord[r.nlhs] = (int32_t)lhs[i];
            r.nlhs += 1;
            r.order += (int32_t)lhs[i];
            r.lhs_mask |= 1u << i;
        }
        if (r.order > 4) throw sg::ArgErr("reaction order above 4 is not supported");
        for (int i = 0; i < s->nspec; ++i) {
            if (upd[i] == 0) continue;
            if (r.nupd == SG_MAX_UPD) throw sg::ArgErr("a reaction changes more than 8 species");
            r.upd_spec[r.nupd] = i;
            r.upd_delta[r.nupd] = upd[i];
            r.nupd += 1;
            r.upd_mask |= 1u << i;
        }
        r.fast = sg_reac_fast_code(&r);
        s->reacs.push_back(r);
        s->reac_kdef.push_back(kcst);
        if (out_idx) *out_idx = (int32_t)s->reacs.size() - 1;
    });
}

int sg_add_diff(sg_solver* h, int32_t comp, int32_t spec, double dcst, int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->nspec <= 0 || s->ntets <= 0) throw sg::ProgErr("set species count and mesh first");
        s->check_comp(comp);
        s->check_spec(spec);
        if (!(dcst >= 0.0)) throw sg::ArgErr("diffusion constant must be non-negative");
        for (size_t i = 0; i < s->diff_spec.size(); ++i)
            if (s->diff_spec[i] == spec && s->diff_comp[i] == comp)
                throw sg::ArgErr("duplicate diffusion rule for species in compartment");
        s->diff_comp.push_back(comp);
        s->diff_spec.push_back(spec);
        s->dcst_def[(size_t)comp * s->nspec + spec] = dcst;
        if (out_idx) *out_idx = (int32_t)s->diff_spec.size() - 1;
    });
}

int sg_set_realizations(sg_solver* h, int32_t nreal, const int32_t* tet_offsets) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        need(tet_offsets, "tet_offsets");
        if (nreal <= 0) throw sg::ArgErr("need nreal > 0");
        s->nreal = nreal;
        s->real_begin.assign(tet_offsets, tet_offsets + nreal + 1);
    });
}

int sg_setup(sg_solver* h) {
    return guarded([&] { S(h)->setup(); });
}

int sg_reset(sg_solver* h) {
    return guarded([&] { S(h)->reset(); });
}

int sg_run(sg_solver* h, double endtime) {
    return guarded([&] { S(h)->run(endtime); });
}

int sg_advance(sg_solver* h, double adv) {
    return guarded([&] {
        if (adv < 0.0) throw sg::ArgErr("Time to advance cannot be negative");
        Solver* s = S(h);
        s->run(s->time() + adv);
    });
}

int sg_get_time(sg_solver* h, double* t) {
    return guarded([&] {
        need(t, "t");
        *t = S(h)->time();
    });
}

int sg_get_update_period(sg_solver* h, int32_t real, double* period) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_setup();
        s->check_real(real);
        need(period, "period");
        *period = s->reals[real].period;
    });
}

int sg_get_tet_count(sg_solver* h, int32_t tet, int32_t spec, double* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->get_tet_count(tet, spec);
    });
}

int sg_set_tet_count(sg_solver* h, int32_t tet, int32_t spec, double n) {
    return guarded([&] { S(h)->set_tet_count(tet, spec, n); });
}

int sg_get_comp_count(sg_solver* h, int32_t comp, int32_t spec, int32_t real, double* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->get_comp_count(comp, spec, real);
    });
}

int sg_set_comp_count(sg_solver* h, int32_t comp, int32_t spec, int32_t real, double n) {
    return guarded([&] { S(h)->set_comp_count(comp, spec, n, real); });
}

int sg_get_spec_counts(sg_solver* h, int32_t spec, uint32_t* out) {
    return guarded([&] {
        need(out, "out");
        S(h)->get_spec_row(spec, out);
    });
}

int sg_get_batch_tet_counts(sg_solver* h, int32_t spec, const int32_t* tets, int32_t n, double* out) {
    return guarded([&] {
        if (n > 0) {
            need(tets, "tets");
            need(out, "out");
        }
        S(h)->get_batch_tet_counts(spec, tets, n, out);
    });
}

int sg_set_spec_counts(sg_solver* h, int32_t spec, const uint32_t* in) {
    return guarded([&] {
        need(in, "in");
        S(h)->set_spec_row(spec, in);
    });
}

int sg_get_all_counts(sg_solver* h, uint32_t* out) {
    return guarded([&] {
        need(out, "out");
        S(h)->get_all_rows(out);
    });
}

int sg_set_all_counts(sg_solver* h, const uint32_t* in) {
    return guarded([&] {
        need(in, "in");
        S(h)->set_all_rows(in);
    });
}

int sg_set_tet_clamped(sg_solver* h, int32_t tet, int32_t spec, int32_t clamped) {
    return guarded([&] { S(h)->set_tet_clamped(tet, spec, clamped != 0); });
}

int sg_set_reac_k(sg_solver* h, int32_t reac, int32_t real, double k) {
    return guarded([&] { S(h)->set_reac_k(reac, real, k); });
}

int sg_get_reac_k(sg_solver* h, int32_t reac, int32_t real, double* k) {
    return guarded([&] {
        need(k, "k");
        *k = S(h)->get_reac_k(reac, real);
    });
}

int sg_set_diff_d(sg_solver* h, int32_t comp, int32_t spec, int32_t real, double d) {
    return guarded([&] { S(h)->set_diff_d(comp, spec, d, real); });
}

int sg_set_diff_apply_threshold(sg_solver* h, int32_t threshold) {
    return guarded([&] {
        if (threshold < 0) throw sg::ArgErr("threshold must be non-negative");
        S(h)->diff_apply_threshold = threshold;
    });
}

int sg_get_reac_extent(sg_solver* h, int32_t reac, uint64_t* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->reac_extent(reac);
    });
}

int sg_get_diff_extent(sg_solver* h, uint64_t* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->diff_extent();
    });
}

int sg_checkpoint(sg_solver* h, const char* file_name) {
    return guarded([&] {
        need(file_name, "file_name");
        S(h)->checkpoint(file_name);
    });
}

int sg_restore(sg_solver* h, const char* file_name) {
    return guarded([&] {
        need(file_name, "file_name");
        S(h)->restore(file_name);
    });
}

int sg_get_nsteps(sg_solver* h, uint64_t* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->nsteps();
    });
}

int sg_get_niteration(sg_solver* h, uint64_t* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->niteration;
    });
}

int sg_set_launch(sg_solver* h, int32_t block, int32_t grid) {
    return guarded([&] {
        if (block != 64 && block != 128 && block != 256) throw sg::ArgErr("block must be 64, 128 or 256");
        if (grid < -1) throw sg::ArgErr("grid must be >= -1 (0 = occupancy-sized, -1 = one tet per thread)");
        S(h)->block = block;
        S(h)->grid = grid;
    });
}

int sg_get_launch(sg_solver* h, int32_t* block, int32_t* grid) {
    return guarded([&] {
        if (block) *block = S(h)->block;
        if (grid) *grid = S(h)->grid;
    });
}

int sg_set_split(sg_solver* h, int32_t on) {
    return guarded([&] { S(h)->split = on != 0; });
}

int sg_set_persistent(sg_solver* h, int32_t on, int32_t tets_per_lane) {
    return guarded([&] {
        if (tets_per_lane != 1 && tets_per_lane != 2 && tets_per_lane != 4 && tets_per_lane != 8)
            throw sg::ArgErr("tets per lane must be 1, 2, 4 or 8");
        Solver* s = S(h);
        s->persist = on != 0;
        s->persist_tpl = tets_per_lane;
    });
}

int sg_get_persistent(sg_solver* h, int32_t* on, int32_t* tets_per_lane) {
    return guarded([&] {
        need(on, "on");
        need(tets_per_lane, "tets_per_lane");
        *on = S(h)->persist ? 1 : 0;
        *tets_per_lane = S(h)->persist_tpl;
    });
}

int sg_set_window_wait_limit(sg_solver* h, uint32_t polls) {
    return guarded([&] { S(h)->persist_spin_limit = polls; });
}

int sg_get_split(sg_solver* h, int32_t* on) {
    return guarded([&] {
        need(on, "on");
        *on = S(h)->use_split() ? 1 : 0;
    });
}

int sg_get_carveout(sg_solver* h, int32_t* percent) {
    return guarded([&] {
        need(percent, "percent");
        *percent = S(h)->carveout;
    });
}

int sg_set_autotune(sg_solver* h, int32_t on) {
    return guarded([&] { S(h)->tune_pending = on != 0; });
}

int sg_get_autotune_ms(sg_solver* h, float* ms, int32_t cap, int32_t* count) {
    return guarded([&] {
        const auto& v = S(h)->tune_ms;
        if (count) *count = (int32_t)v.size();
        for (int i = 0; i < (int)v.size() && i < cap; ++i) ms[i] = v[i];
    });
}

int sg_set_graphs(sg_solver* h, int32_t on) {
    return guarded([&] {
        S(h)->use_graphs = on != 0;
        if (!on) S(h)->drop_graph();
    });
}

int sg_set_conservation_check(sg_solver* h, int32_t on) {
    return guarded([&] { S(h)->check = on != 0; });
}

int sg_set_surface(sg_solver* h, int32_t nsspec, int32_t ntris, const int32_t* tri_inner_tet,
                   const int32_t* tri_patch, const double* tri_area, int32_t npatch) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (nsspec <= 0 || nsspec > 32) throw sg::ArgErr("surface species count must be in 1..32");
        if (ntris <= 0 || npatch <= 0) throw sg::ArgErr("need membrane triangles and patches");
        need(tri_inner_tet, "tri_inner_tet");
        need(tri_patch, "tri_patch");
        need(tri_area, "tri_area");
        s->nsspec = nsspec;
        s->ntris = ntris;
        s->npatch = npatch;
        s->tri_inner.assign(tri_inner_tet, tri_inner_tet + ntris);
        s->tri_patch.assign(tri_patch, tri_patch + ntris);
        s->tri_area.assign(tri_area, tri_area + ntris);
        for (int32_t p : s->tri_patch)
            if (p < 0 || p >= npatch) throw sg::ArgErr("triangle patch index out of range");
        for (double a : s->tri_area)
            if (!(a > 0.0)) throw sg::ArgErr("triangle area must be positive");
    });
}

int sg_add_ghk(sg_solver* h, int32_t patch, int32_t sspec, int32_t ion, int32_t valence, double perm,
               double vshift, double voconc, int32_t realflux, int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->nsspec <= 0) throw sg::ProgErr("call sg_set_surface first");
        if (patch < 0 || patch >= s->npatch) throw sg::ArgErr("patch index out of range");
        if (sspec < 0 || sspec >= s->nsspec) throw sg::ArgErr("surface species index out of range");
        s->check_spec(ion);
        if (valence == 0) throw sg::ArgErr("GHK current of an ion without valence");
        if (!(perm > 0.0)) throw sg::ArgErr("GHK permeability must be positive (setP or setPInfo)");
        sg_ghk g{};
        g.patch = patch;
        g.sspec = sspec;
        g.ion = ion;
        g.valence = valence;
        g.perm = perm;
        g.vshift = vshift;
        g.voconc = voconc >= 0.0 ? voconc : -1.0;  // < 0: the outer tet's concentration
        g.realflux = realflux ? 1 : 0;
        s->ghks.push_back(g);
        if (out_idx) *out_idx = (int32_t)s->ghks.size() - 1;
    });
}

int sg_set_temp(sg_solver* h, double kelvin) {
    return guarded([&] {
        if (!(kelvin > 0.0)) throw sg::ArgErr("temperature must be positive");
        S(h)->temp = kelvin;
    });
}

int sg_get_temp(sg_solver* h, double* kelvin) {
    return guarded([&] {
        need(kelvin, "kelvin");
        *kelvin = S(h)->temp;
    });
}

int sg_get_tri_ghk_i(sg_solver* h, int32_t tri, double* amps) {
    return guarded([&] {
        need(amps, "amps");
        *amps = S(h)->get_tri_ghk_i(tri);
    });
}

int sg_set_tri_neighbours(sg_solver* h, const int32_t* nbr, const int32_t* nbr_edge, const double* len,
                          const double* dist) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->ntris <= 0) throw sg::ProgErr("call sg_set_surface first");
        need(nbr, "nbr");
        need(nbr_edge, "nbr_edge");
        need(len, "len");
        need(dist, "dist");
        const size_t n = (size_t)s->ntris * 3;
        s->tri_nbr.assign(nbr, nbr + n);
        s->tri_nbr_edge.assign(nbr_edge, nbr_edge + n);
        s->tri_len.assign(len, len + n);
        s->tri_dist.assign(dist, dist + n);
        for (size_t i = 0; i < n; ++i) {
            const int q = s->tri_nbr[i];
            if (q < -1 || q >= s->ntris) throw sg::ArgErr("triangle neighbour out of range");
            if (q >= 0 && (s->tri_nbr_edge[i] < 0 || s->tri_nbr_edge[i] > 2))
                throw sg::ArgErr("triangle neighbour edge out of range");
            if (q >= 0 && s->tri_nbr[(size_t)q * 3 + s->tri_nbr_edge[i]] != (int)(i / 3))
                throw sg::ArgErr("triangle neighbours are not reciprocal");
        }
    });
}

int sg_add_sdiff(sg_solver* h, int32_t patch, int32_t sspec, double dcst, int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->nsspec <= 0) throw sg::ProgErr("call sg_set_surface first");
        if (patch < 0 || patch >= s->npatch) throw sg::ArgErr("patch index out of range");
        if (sspec < 0 || sspec >= s->nsspec) throw sg::ArgErr("surface species index out of range");
        if (!(dcst >= 0.0)) throw sg::ArgErr("diffusion constant must be non-negative");
        s->sdcst.resize((size_t)s->npatch * s->nsspec, 0.0);
        s->sdcst[(size_t)patch * s->nsspec + sspec] = dcst;
        if (out_idx) *out_idx = patch * s->nsspec + sspec;
    });
}

static void build_sreac(Solver* s, int32_t patch, const uint32_t* slhs, const uint32_t* ilhs, const int32_t* supd,
                        const int32_t* iupd, sg_sreac& r) {
    s->require_not_setup();
    if (s->nsspec <= 0) throw sg::ProgErr("call sg_set_surface first");
    if (patch < 0 || patch >= s->npatch) throw sg::ArgErr("patch index out of range");
    need(slhs, "slhs");
    need(ilhs, "ilhs");
    need(supd, "supd");
    need(iupd, "iupd");
    std::memset(&r, 0, sizeof(r));
    r.patch = patch;
    r.vdep = -1;
    for (int i = 0; i < s->nsspec; ++i) {
        if (!slhs[i]) continue;
        if (slhs[i] > 4 || r.nslhs == SG_MAX_LHS) throw sg::ArgErr("surface reactant stoichiometry");
        r.slhs_spec[r.nslhs] = i;
        r.slhs_ord[r.nslhs++] = (int32_t)slhs[i];
        r.order += (int32_t)slhs[i];
    }
    for (int i = 0; i < s->nspec; ++i) {
        if (!ilhs[i]) continue;
        if (ilhs[i] > 4 || r.nilhs == SG_MAX_LHS) throw sg::ArgErr("volume reactant stoichiometry");
        r.ilhs_spec[r.nilhs] = i;
        r.ilhs_ord[r.nilhs++] = (int32_t)ilhs[i];
        r.order += (int32_t)ilhs[i];
    }
    if (r.order > 4) throw sg::ArgErr("reaction order above 4 is not supported");
    r.surf_surf = (r.nilhs == 0) ? 1 : 0;
    for (int i = 0; i < s->nsspec; ++i) {
        if (!supd[i]) continue;
        if (r.nsupd == SG_MAX_UPD) throw sg::ArgErr("too many changed surface species");
        r.supd_spec[r.nsupd] = i;
        r.supd_delta[r.nsupd++] = supd[i];
    }
    for (int i = 0; i < s->nspec; ++i) {
        if (!iupd[i]) continue;
        if (r.niupd == SG_MAX_UPD) throw sg::ArgErr("too many changed volume species");
        r.iupd_spec[r.niupd] = i;
        r.iupd_delta[r.niupd++] = iupd[i];
    }
}

int sg_add_sreac(sg_solver* h, int32_t patch, const uint32_t* slhs, const uint32_t* ilhs, const int32_t* supd,
                 const int32_t* iupd, double kcst, int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        sg_sreac r;
        build_sreac(s, patch, slhs, ilhs, supd, iupd, r);
        if (!(kcst >= 0.0)) throw sg::ArgErr("reaction constant must be non-negative");
        s->sreacs.push_back(r);
        s->skcst.push_back(kcst);
        if (out_idx) *out_idx = (int32_t)s->sreacs.size() - 1;
    });
}

int sg_add_vdep_sreac(sg_solver* h, int32_t patch, const uint32_t* slhs, const uint32_t* ilhs,
                      const int32_t* supd, const int32_t* iupd, double vmin, double dv, int32_t ntab,
                      const double* ktab, int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        sg_sreac r;
        build_sreac(s, patch, slhs, ilhs, supd, iupd, r);
        need(ktab, "ktab");
        if (ntab < 2 || !(dv > 0.0)) throw sg::ArgErr("k(V) table needs >= 2 points and dv > 0");
        for (int i = 0; i < ntab; ++i)
            if (!(ktab[i] >= 0.0)) throw sg::ArgErr("k(V) must be non-negative");
        sg_vtab vt;
        vt.vmin = vmin;
        vt.dv = dv;
        vt.off = (int32_t)s->vtab_vals.size();
        vt.n = ntab;
        s->vtab_vals.insert(s->vtab_vals.end(), ktab, ktab + ntab);
        r.vdep = (int32_t)s->vtabs.size();
        s->vtabs.push_back(vt);
        s->sreacs.push_back(r);
        s->skcst.push_back(0.0);
        if (out_idx) *out_idx = (int32_t)s->sreacs.size() - 1;
    });
}

int sg_set_tri_outer(sg_solver* h, const int32_t* tri_outer_tet) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (s->ntris <= 0) throw sg::ProgErr("call sg_set_surface first");
        need(tri_outer_tet, "tri_outer_tet");
        s->tri_outer.assign(tri_outer_tet, tri_outer_tet + s->ntris);
        for (int m = 0; m < s->ntris; ++m) {
            const int o = s->tri_outer[m];
            if (o < -1 || o >= s->ntets) throw sg::ArgErr("outer tet index out of range");
            if (o >= 0 && o == s->tri_inner[m]) throw sg::ArgErr("a triangle's outer tet equals its inner tet");
        }
    });
}

int sg_set_sreac_outer(sg_solver* h, int32_t sreac, const uint32_t* olhs, const int32_t* oupd) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (sreac < 0 || sreac >= (int32_t)s->sreacs.size()) throw sg::ArgErr("surface reaction index out of range");
        need(olhs, "olhs");
        need(oupd, "oupd");
        sg_sreac& r = s->sreacs[sreac];
        int n = 0, order = 0;
        for (int i = 0; i < s->nspec; ++i) {
            if (!olhs[i]) continue;
            if (olhs[i] > 4 || n == SG_MAX_LHS) throw sg::ArgErr("volume reactant stoichiometry");
            ++n;
            order += (int)olhs[i];
        }
        if (n > 0 && r.nilhs > 0)
            throw sg::ArgErr("a surface reaction has volume reactants on one side only (inner or outer)");
        if (n > 0) {
            r.nilhs = 0;
            for (int i = 0; i < s->nspec; ++i) {
                if (!olhs[i]) continue;
                r.ilhs_spec[r.nilhs] = i;
                r.ilhs_ord[r.nilhs++] = (int32_t)olhs[i];
            }
            r.order += order;
            if (r.order > 4) throw sg::ArgErr("reaction order above 4 is not supported");
            r.vside = 1;
            r.surf_surf = 0;
        }
        r.noupd = 0;
        for (int i = 0; i < s->nspec; ++i) {
            if (!oupd[i]) continue;
            if (r.noupd == SG_MAX_UPD) throw sg::ArgErr("too many changed volume species");
            r.oupd_spec[r.noupd] = i;
            r.oupd_delta[r.noupd++] = oupd[i];
        }
    });
}

int sg_add_ohmic(sg_solver* h, int32_t patch, int32_t sspec, double g, double erev, int32_t* out_idx) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_not_setup();
        if (patch < 0 || patch >= s->npatch) throw sg::ArgErr("patch index out of range");
        if (sspec < 0 || sspec >= s->nsspec) throw sg::ArgErr("surface species index out of range");
        if (!(g >= 0.0)) throw sg::ArgErr("conductance must be non-negative");
        s->ohmics.push_back(sg_ohmic{patch, sspec, g, erev});
        if (out_idx) *out_idx = (int32_t)s->ohmics.size() - 1;
    });
}

int sg_get_tri_count(sg_solver* h, int32_t tri, int32_t sspec, double* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->get_tri_count(tri, sspec);
    });
}

int sg_set_tri_count(sg_solver* h, int32_t tri, int32_t sspec, double n) {
    return guarded([&] { S(h)->set_tri_count(tri, sspec, n); });
}

int sg_get_patch_count(sg_solver* h, int32_t patch, int32_t sspec, int32_t real, double* n) {
    return guarded([&] {
        need(n, "n");
        *n = S(h)->get_patch_count(patch, sspec, real);
    });
}

int sg_set_patch_count(sg_solver* h, int32_t patch, int32_t sspec, int32_t real, double n) {
    return guarded([&] { S(h)->set_patch_count(patch, sspec, real, n); });
}

int sg_get_tri_ohmic_i(sg_solver* h, int32_t tri, double* amps) {
    return guarded([&] {
        need(amps, "amps");
        *amps = S(h)->get_tri_ohmic_i(tri);
    });
}

int sg_set_efield_mesh(sg_solver* h, int32_t nverts, const double* verts, const int32_t* tet_verts,
                       int32_t ntris, const int32_t* tri_verts, int32_t method) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_setup();
        if (s->has_surf() && ntris != s->ntris)
            throw sg::ArgErr("the EField membrane must be the surface triangles, in the same order");
        need(verts, "verts");
        need(tet_verts, "tet_verts");
        if (ntris > 0) need(tri_verts, "tri_verts");
        if (method != sg::EF_CG_FP64 && method != sg::EF_CG_MIXED) throw sg::ArgErr("unknown EField method");
        // Conducting volume: the tets of every compartment (efield.cpp:48 initMesh).
        std::vector<int32_t> tets;
        for (int t = 0; t < s->ntets; ++t)
            if (s->tet_comp[t] >= 0) tets.insert(tets.end(), tet_verts + (size_t)t * 4, tet_verts + (size_t)t * 4 + 4);
        std::vector<double> um((size_t)nverts * 3);
        for (size_t i = 0; i < um.size(); ++i) um[i] = verts[i] * 1.0e6;  // m -> um (efield units)
        s->ef.setup(nverts, um.data(), (int)(tets.size() / 4), tets.data(), ntris, tri_verts, s->stream, s->nsm);
        s->ef.method = method;
        s->ef_on = true;
        s->sync();
    });
}

int sg_set_efield_dt(sg_solver* h, double dt) {
    return guarded([&] {
        if (!(dt > 0.0)) throw sg::ArgErr("EField dt must be positive");
        S(h)->efdt = dt;
    });
}

int sg_get_efield_dt(sg_solver* h, double* dt) {
    return guarded([&] {
        need(dt, "dt");
        *dt = S(h)->efdt;
    });
}

int sg_set_efield_tolerance(sg_solver* h, double rel_tol, double inner_rel_tol, int32_t max_iter) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (!(rel_tol > 0.0) || !(inner_rel_tol > 0.0) || max_iter <= 0) throw sg::ArgErr("bad tolerance");
        s->ef.tol = rel_tol;
        s->ef.inner_tol = inner_rel_tol;
        s->ef.max_iter = max_iter;
    });
}

int sg_set_memb_potential(sg_solver* h, double v) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        s->ef.set_potential(v * 1.0e3, s->stream);
        s->sync();
    });
}

int sg_set_memb_capac(sg_solver* h, double cm) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (!(cm >= 0.0)) throw sg::ArgErr("capacitance must be non-negative");
        s->ef.cm = cm;  // F/m^2 == pF/um^2
        s->ef.dirty = true;
    });
}

int sg_set_memb_vol_res(sg_solver* h, double ra) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (!(ra > 0.0)) throw sg::ArgErr("resistivity must be positive");
        s->ef.sigma = 1.0 / (ra * 1.0e-3);  // ohm m -> nS/um  (efield.cpp:83-87)
        s->ef.dirty = true;
    });
}

int sg_set_memb_res(sg_solver* h, double ro, double vrev) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (!(ro > 0.0)) throw sg::ArgErr("membrane resistance must be positive");
        s->ef.g_leak = (1.0 / ro) * 1.0e-3;  // S/m^2 -> nS/um^2 (dVsolver.cpp:85)
        s->ef.v_leak = vrev * 1.0e3;
        s->ef.dirty = true;
    });
}

int sg_get_vert_v(sg_solver* h, int32_t v, double* volts) {
    return guarded([&] {
        need(volts, "volts");
        *volts = S(h)->get_vert_v(v);
    });
}

int sg_set_vert_v(sg_solver* h, int32_t v, double volts) {
    return guarded([&] { S(h)->set_vert_v(v, volts); });
}

int sg_get_tri_v(sg_solver* h, int32_t tri, double* volts) {
    return guarded([&] {
        need(volts, "volts");
        *volts = S(h)->get_tri_v(tri);
    });
}

int sg_set_vert_v_clamped(sg_solver* h, int32_t v, int32_t clamped) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        s->check_vert(v);
        s->ef.vclamped[s->ef.vid(v)] = clamped ? 1 : 0;
        s->ef.dirty = true;
    });
}

int sg_set_vert_iclamp(sg_solver* h, int32_t v, double amps) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        s->check_vert(v);
        s->ef.vert_iclamp[s->ef.vid(v)] = amps * 1.0e12;  // A -> pA, positive = into the cell (efield.cpp:214-225)
        s->ef.dirty = true;
    });
}

int sg_get_efield_stats(sg_solver* h, uint64_t* steps, uint64_t* iterations, double* solve_ms,
                        double* last_rel_residual) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (steps) *steps = s->ef.stats.steps;
        if (iterations) *iterations = s->ef.stats.iterations;
        if (solve_ms) *solve_ms = s->ef.stats.solve_ms;
        if (last_rel_residual) *last_rel_residual = s->ef.stats.last_rel_residual;
    });
}

int sg_set_efield_check(sg_solver* h, int32_t on, double rel_tol) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (on && !(rel_tol > 0.0)) throw sg::ArgErr("bad check tolerance");
        s->ef.check = on != 0;
        if (on) s->ef.check_tol = rel_tol;
    });
}

int sg_set_efield_persistent(sg_solver* h, int32_t on) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        s->ef.persistent = on != 0;
    });
}

int sg_set_efield_barrier_limit(sg_solver* h, uint32_t polls) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        s->ef.spin_limit = polls;
    });
}

int sg_set_efield_reliable_updates(sg_solver* h, int32_t on, double delta) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (on && !(delta > 0.0 && delta < 1.0)) throw sg::ArgErr("reliable-update factor must be in (0, 1)");
        s->ef.reliable = on != 0;
        if (on) s->ef.ru_delta = delta;
    });
}

int sg_get_efield_check(sg_solver* h, uint64_t* steps, double* max_rel, double* last_rel) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_ef();
        if (steps) *steps = s->ef.stats.check_steps;
        if (max_rel) *max_rel = s->ef.stats.check_max_rel;
        if (last_rel) *last_rel = s->ef.stats.check_last_rel;
    });
}

int sg_get_stream(sg_solver* h, void** stream) {
    return guarded([&] {
        need(stream, "stream");
        *stream = (void*)S(h)->stream;
    });
}

int sg_set_profiling(sg_solver* h, int32_t on) {
    return guarded([&] {
        Solver* s = S(h);
        s->profiling = on != 0;
        s->prof_ms = 0.0;
        s->prof_windows = 0;
    });
}

int sg_get_profile(sg_solver* h, double* window_ms, uint64_t* windows, uint64_t* launches) {
    return guarded([&] {
        Solver* s = S(h);
        if (window_ms) *window_ms = s->prof_ms;
        if (windows) *windows = s->prof_windows;
        if (launches) *launches = s->launches;
    });
}

int sg_get_status(sg_solver* h, uint32_t* status) {
    return guarded([&] {
        Solver* s = S(h);
        s->require_setup();
        need(status, "status");
        s->d2h(status, s->d_status.p, 1);
        s->sync();
    });
}

}  // extern "C"
