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
// the triangle (S), in its inner tet (I) and in its outer tet (O).  As in the reference
// (SReacdef::inside / outside), the volume reactants are all on one side: ilhs holds them
// and vside says which tet they are counted in (and whose volume scales the constant).
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
    int32_t vside;                     // 0: volume reactants in the inner tet, 1: in the outer tet
    int32_t noupd;                     // outer-tet species changed
    int32_t oupd_spec[SG_MAX_UPD], oupd_delta[SG_MAX_UPD];
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
// with permeability perm (m^3/s per channel) against a fixed outer concentration voconc (M),
// or, with voconc < 0, against the concentration in the triangle's outer tet (the ions then
// move between the two tets).
typedef struct sg_ghk {
    int32_t patch;
    int32_t sspec;
    int32_t ion;
    int32_t valence;
    double perm;
    double vshift;                     // V
    double voconc;                     // M; < 0: the outer tet's concentration
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
    const int32_t* tri_outer;          // [M] outer tet, -1 none (null when no triangle has one)
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
#define SG_ERR_WAIT 32u                // a persistent window launch gave up waiting on a realization

// Merged SSA units.  A membrane triangle whose patch has surface reactions or GHK currents
// that count or change species of its outer tet couples that tet to its inner one (the
// reference keeps the triangle and both tets in one rank's SSA, sreac.cpp:200-300).  A
// connected group of coupled tets, together with every membrane triangle whose inner tet is
// in the group, is one SSA unit: elements are its tets (ascending) then its triangles
// (ascending), each with its own reactions; the unit's direct-method SSA selects the
// element through a binary sum tree of element propensities.
typedef struct sg_unit_args {
    const int32_t* tet_begin;          // [U + 1] into tets
    const int32_t* tets;               // tets of each unit, ascending
    const int32_t* tri_begin;          // [U + 1] into tris
    const int32_t* tris;               // membrane triangles of each unit, ascending
    const int32_t* elem_base;          // [U + 1]: first element of each unit (tets, then triangles)
    const int32_t* tree_base;          // [U + 1]: first node of each unit's tree (2 P doubles, P = 2^k >= elements)
    const int32_t* tet_unit;           // [T]: unit of a merged tet, -1 otherwise
    const int32_t* tet_adj;            // [E][4]: for tet elements, the unit's triangle elements whose rates read the tet (-1)
    const int32_t* tri_side;           // [M][2]: unit elements of a merged triangle's inner tet and coupled outer tet (-1)
    double* prop;                      // [E][rmax] element reaction propensities (scratch)
    double* tree;                      // sum trees (scratch)
    double* socc;                      // [SS][M] surface occupancy integrals within the window (scratch)
    double* slast;                     // [SS][M] time of the last change within the window (scratch)
    int32_t nunits;
    int32_t rmax;                      // reactions (and GHK currents) per element, at most
} sg_unit_args;

// One persistent launch that runs nwin windows of every batched realization.  Work items
// are (window, chunk) in window-major order; a chunk is tpw consecutive tets of one
// realization (32 lanes x tets per lane).  A warp takes the next item from the counter and
// waits (bounded) until its realization has completed the previous window; the warp that
// finishes the last chunk of a realization's window advances that realization's time and
// publishes the window.
typedef struct sg_persist_args {
    const int32_t* chunk_begin;        // [nreal + 1] first chunk of each realization
    unsigned int* done;                // [nreal] chunks finished in this launch
    unsigned int* ready;               // [nreal] windows completed in this launch
    unsigned long long* next;          // [1] next work item
    unsigned int* abort;               // [1] set when a wait gave up
    unsigned int spin_limit;           // polls of one wait before it gives up
    int32_t nchunks;                   // chunks of one window over all realizations
    int32_t nwin;                      // windows of this launch
    int32_t tpw;                       // tets per chunk
} sg_persist_args;

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
    // 1/x and ln x! for x below the mode-search table size in global memory (the values the
    // leave kernel keeps in shared memory), for kernels without room for them; may be null.
    const double* mode_rcpl;
    const double* mode_lnf;
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
    sg_unit_args units;                // merged SSA units (nunits = 0: none)
    int32_t ntets;                     // total tets over realizations
    int32_t nspec;
    int32_t ndiff;
    int32_t nreac;
    int32_t ncomp;
    int32_t nreal;
    uint64_t seed;
} sg_window_args;
