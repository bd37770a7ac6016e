// Device-side tables of the operator-split SSA step.  Plain structs shared by
// the host solver (which fills them) and the CUDA kernels (which read them).
//
// Layout in HBM (T = tets over all realizations, S = volume species,
// D = diffusing species, R = reactions):
//   counts   uint32  [S][T]        species-major, tet contiguous (coalesced)
//   outflow  uint4   [2][D][T]     per (diffusing species, tet): molecules leaving
//                                  through faces 0..3 in one window; double
//                                  buffered by window parity
//   nbr      int4    [T]           per face: (neighbour << 2) | face-of-neighbour,
//                                  or -1 when nothing diffuses through the face
//   geo      float4  [T]           (c0, c1, c2, G): conditional face selectors and
//                                  G = sum_f A_f / (V d_f)
//   ivs      double  [T]           1 / (1e3 V N_A): order scaling of reaction constants
#pragma once
#include <stdint.h>

#define SG_MAX_LHS 4   // distinct reactant species of one reaction
#define SG_MAX_UPD 8   // distinct species whose count a reaction changes

// One volume reaction, compacted from the dense lhs / upd rows of the reference
// Compdef (src/steps/solver/compdef.hpp:252-266).  Entries are in increasing
// species order.
typedef struct sg_reac {
    int32_t comp;                      // compartment the reaction lives in
    int32_t order;                     // sum of lhs stoichiometry
    int32_t nlhs;                      // number of distinct reactants
    int32_t nupd;                      // number of species changed
    int32_t lhs_spec[SG_MAX_LHS];      // reactant species (global volume index)
    int32_t lhs_ord[SG_MAX_LHS];       // its stoichiometry (1..4)
    int32_t upd_spec[SG_MAX_UPD];      // changed species
    int32_t upd_delta[SG_MAX_UPD];     // signed change
    uint32_t lhs_mask;                 // bit per reactant species (propensity dependencies)
    uint32_t upd_mask;                 // bit per changed species
    uint32_t fast;                     // propensity form: kind | first species << 8 | second << 16
} sg_reac;

// Propensity forms with a closed count product (order <= 2); everything else takes the
// general product.  The product of the counts is formed exactly in 64-bit integers and
// rounded once to double, which is the value the reference's double product gives
// (src/steps/mpi/tetopsplit/reac.cpp:184-232: the factors are exact, one rounding).
#define SG_RK_ZERO 0u                  // no reactant: h = 1
#define SG_RK_ONE 1u                   // A: h = c_A
#define SG_RK_PAIR 2u                  // A + B, A != B: h = c_A c_B
#define SG_RK_DIMER 3u                 // 2 A: h = c_A (c_A - 1)
#define SG_RK_GENERIC 4u               // order 3 or 4: the general product

#if defined(__CUDACC__)
__host__ __device__
#endif
static inline uint32_t sg_reac_fast_code(const sg_reac* r) {
    uint32_t kind = SG_RK_GENERIC, a = 0u, b = 0u;
    if (r->nlhs == 0) {
        kind = SG_RK_ZERO;
    } else if (r->nlhs == 1 && r->lhs_ord[0] == 1) {
        kind = SG_RK_ONE;
        a = (uint32_t)r->lhs_spec[0];
    } else if (r->nlhs == 1 && r->lhs_ord[0] == 2) {
        kind = SG_RK_DIMER;
        a = (uint32_t)r->lhs_spec[0];
    } else if (r->nlhs == 2 && r->lhs_ord[0] == 1 && r->lhs_ord[1] == 1) {
        kind = SG_RK_PAIR;
        a = (uint32_t)r->lhs_spec[0];
        b = (uint32_t)r->lhs_spec[1];
    }
    return kind | (a << 8) | (b << 16);
}

// One surface reaction of a patch (Patchdef sreac_lhs_S/I, sreac_upd_S/I,
// src/steps/solver/patchdef.hpp), optionally with a voltage-dependent constant
// (VDepSReacdef, src/steps/solver/vdepsreacdef.cpp:194-218).  Reactants and products on
// the triangle (S) and in its inner tet (I); outer-volume terms are not supported.
typedef struct sg_sreac {
    int32_t patch;
    int32_t order;                     // total lhs stoichiometry (surface + volume)
    int32_t surf_surf;                 // 1: no volume reactant -> area scaling of the constant
    int32_t vdep;                      // index of the k(V) table, -1 for a constant kcst
    int32_t nslhs, nilhs, nsupd, niupd;
    int32_t slhs_spec[SG_MAX_LHS], slhs_ord[SG_MAX_LHS];
    int32_t ilhs_spec[SG_MAX_LHS], ilhs_ord[SG_MAX_LHS];
    int32_t supd_spec[SG_MAX_UPD], supd_delta[SG_MAX_UPD];
    int32_t iupd_spec[SG_MAX_UPD], iupd_delta[SG_MAX_UPD];
} sg_sreac;

// k(V) table of a voltage-dependent surface reaction: k at vmin + i dv, i < n (V, /s ...).
typedef struct sg_vtab {
    double vmin;
    double dv;
    int32_t off;                       // offset into the concatenated table values
    int32_t n;
} sg_vtab;

// Ohmic current through one surface species (channel state) of a patch (OhmicCurrdef).
typedef struct sg_ohmic {
    int32_t patch;
    int32_t sspec;
    double g;                          // S per channel
    double erev;                       // V
} sg_ohmic;

// GHK current (ghkcurr.cpp:168-280): channel state sspec of a patch passes ion (valence z)
// with permeability perm (m^3/s per channel) against a fixed outer concentration voconc (M).
typedef struct sg_ghk {
    int32_t patch;
    int32_t sspec;
    int32_t ion;
    int32_t valence;
    double perm;
    double vshift;                     // V
    double voconc;                     // M
    int32_t realflux;                  // ions move (else charge only)
    int32_t pad_;
} sg_ghk;

// Surface part of the window kernel (null tables when the model has no membrane).
typedef struct sg_surf_args {
    uint32_t* tri_counts;              // [SS][M] surface species per membrane triangle
    const int32_t* tet_tris;           // [T][4] membrane triangles whose SSA unit is the tet, -1
    const int32_t* tri_patch;          // [M]
    const double* tri_area;            // [M] m^2
    const double* tri_V;               // [M] mV (EField), null without EField
    const sg_sreac* sreacs;            // [RS] grouped by patch
    const int32_t* patch_sreac_begin;  // [npatch + 1]
    const double* skcst;               // [RS]
    const sg_vtab* vtabs;
    const double* vtab_vals;
    double* spec_int;                  // [SS][M] time integral of surface counts (s) this EField step
    // Surface diffusion (sdiff.cpp): two-phase like the volume, 4 uint32 slots per (tri, species).
    uint32_t* tri_outflow;             // [2][SD][M][4] or null without surface diffusion
    double* tri_occ;                   // [SD][M] window integral of the count, written by the SSA
    const int32_t* sdiff_slot;         // [SS]: compact surface-diffusing index or -1
    const int32_t* sdiff_spec;         // [SD]
    const double* sdcst;               // [npatch][SS] surface diffusion constants (m^2/s), 0 = none
    const int32_t* snbr;               // [M][4]: (neighbour << 2) | its edge, -1 = none
    const float* sgeo;                 // [M][4]: conditional selectors c0, c1, 1, G = sum l/(A d)
    const int32_t* tri_inner;          // [M] inner tet (its realization owns the triangle)
    int32_t nsdiff;
    const sg_ghk* ghks;                // [nghk]
    long long* tri_echarge;            // [M] elementary charges carried out by GHK events this EField step
    double temp;                       // K
    int32_t nghk;
    int32_t nsspec;
    int32_t ntris;
    int32_t nsreac;
    int32_t max_sreac_per_patch;       // surface events per triangle: reactions + GHK currents of its patch
} sg_surf_args;

// Per realization bookkeeping, advanced on the device by the last block of each
// window launch so that the window kernel can be replayed from a CUDA graph.
typedef struct sg_real {
    int32_t tet_begin;                 // first tet of this realization
    int32_t tet_end;                   // one past its last tet
    double t;                          // current time (s)
    double t_end;                      // end time of the current run() call
    double period;                     // operator-split update period (s)
    unsigned long long window;         // windows completed since reset
    int32_t pending;                   // outflow of the last window not yet gathered
    int32_t pad_;
} sg_real;

// Device status word bits (checked by the host after every run()).
#define SG_ERR_CONSERVATION 1u         // species totals moved other than by reactions
#define SG_ERR_OVERFLOW 2u             // a count would exceed UINT32_MAX
#define SG_ERR_TABLE 4u                // a table index out of range
#define SG_ERR_CG 8u                   // EField CG did not converge
#define SG_ERR_NEGATIVE 16u            // a count would go below zero

// Window-kernel arguments.
typedef struct sg_window_args {
    uint32_t* counts;
    uint32_t* outflow;                 // base of [2][D][T] uint4 buffers (as uint32*)
    const int32_t* nbr;                // [T][4]
    const float* geo;                  // [T][4]
    const double* ivs;                 // [T]
    const int32_t* comp;               // [T] or null when every tet is in compartment 0
    const uint32_t* clamp;             // [T] bit per species, or null
    const sg_reac* reacs;              // [R]
    const int32_t* comp_reac_begin;    // [ncomp + 1]
    const double* kcst;                // [nreal][R]
    const double* dcst;                // [nreal][ncomp][S]
    const int32_t* diff_slot;          // [S]: compact diffusing index or -1
    sg_real* reals;                    // [nreal]
    unsigned long long* totals;        // [2][S]  species totals at window start
    unsigned long long* ext;           // [2][R]  reaction events per window
    unsigned long long* ext_total;     // [R]     reaction events since reset
    unsigned long long* diff_total;    // [1]     diffused molecules since reset
    unsigned long long* launch_state;  // [4]: done blocks, launch parity, active count, prev valid
    uint32_t* status;                  // device error word
    sg_surf_args surf;                 // membrane triangles (SURF kernels only)
    unsigned long long* surf_ext;      // [1] surface reaction events since reset
    double* tdel;                      // [D][T] change-time sums handed to the diffusion kernel (split mode)
    uint32_t* tmask;                   // [T] split mode: bit s set when tdel of species s is nonzero
                                       // (tdel is written only for those species)
    const int32_t* diff_spec;          // [D]: species of each diffusing index
    const int32_t* tet_list;           // [nlist] tets of this launch, or null for all tets
    int32_t nlist;
    // Work counters of the split-window kernels, [2][4] by launch parity: the next chunk
    // of 32 tets for the volume SSA (0), the membrane SSA (1) and the diffusion leave (2)
    // (3 unused).  Each window's last block zeroes the next parity's counters.  Null:
    // static schedule.
    unsigned int* work;
    // Diffusion boundaries (diffboundary.cpp, diff.cpp:307-398), null without any: per tet
    // the boundary of each face (byte f, 0xFF = none), the neighbour behind boundary faces
    // ((n << 2) | its face, -1), the face coefficients A / (V d), the two compartments of
    // each boundary and the rate table [nbnd][S][side]: -1 closed, -2 open at the source
    // compartment's constant, >= 0 open at that constant (m^2/s).
    const uint32_t* bface;
    const int32_t* bnbr;
    const float* bcoef;
    const int32_t* bcomps;
    const double* btab;
    int32_t nbnd;
    int32_t ntets;                     // total tets over realizations
    int32_t nspec;
    int32_t ndiff;
    int32_t nreac;
    int32_t ncomp;
    int32_t nreal;
    uint64_t seed;
} sg_window_args;
