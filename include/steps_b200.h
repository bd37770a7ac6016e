/*
 * steps_b200 — C ABI of the B200 operator-split spatial SSA solver.
 *
 * The library replaces the implementation of STEPS' TetOpSplitP
 * (src/steps/mpi/tetopsplit/tetopsplit.hpp:79) behind the solver API of
 * src/steps/solver/api.hpp:58.  Plain C types only: pointers, sizes, indices.
 * Every function returns an sg_status; on failure sg_last_error() gives the
 * message (thread-local).  Status codes mirror the reference's exception
 * classes (src/steps/util/error.hpp:161-234): ArgErr, ProgErr, NotImplErr.
 *
 * Units follow the reference API: seconds, metres, m^3, molecule counts as
 * double at the boundary (fractional values are rounded stochastically),
 * reaction constants in the reference's units (M, s), diffusion constants m^2/s.
 *
 * Typical use (what a TetOpSplitP-replacement class does in its constructor):
 *   sg_create -> sg_set_nspecs -> sg_set_mesh -> sg_add_reac* -> sg_add_diff*
 *   [-> sg_set_realizations] -> sg_setup; then sg_run / getters / setters.
 */
#ifndef STEPS_B200_H
#define STEPS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_ABI_VERSION 1

typedef enum sg_status {
    SG_OK = 0,
    SG_EARG = 1,     /* steps::ArgErr      (bad argument)            */
    SG_EPROG = 2,    /* steps::ProgErr     (internal / usage error)  */
    SG_ENOTIMPL = 3, /* steps::NotImplErr                             */
    SG_ECUDA = 4,    /* CUDA runtime failure                          */
    SG_EDEVICE = 5   /* device status word: conservation, overflow, CG */
} sg_status;

typedef struct sg_solver sg_solver; /* opaque */

/* Message of the last failed call on this thread. */
const char* sg_last_error(void);
int sg_version(void);

/* ---- construction ------------------------------------------------------ */

/* Replaces TetOpSplitP::TetOpSplitP (tetopsplit.hpp:81-87, TOS:84-127).  seed keys
 * the Philox streams (the reference reads RNG::seed, rng.hpp:60). */
int sg_create(sg_solver** out, uint64_t seed, int device);
int sg_destroy(sg_solver* h);

/* Volume species count (global species of the Statedef, statedef.hpp:40). */
int sg_set_nspecs(sg_solver* h, int32_t nspec);

/* Mesh as the reference Tet objects see it (TOS:644-681): per tet volume (m^3), per
 * face neighbour tet (-1 = none), face area (m^2) and barycentre distance (m), and
 * the compartment of each tet (-1 = outside every compartment). */
int sg_set_mesh(sg_solver* h, int32_t ntets, const double* vol, const int32_t* neighb,
                const double* area, const double* dist, const int32_t* tet_comp, int32_t ncomp);

/* Diffusion boundaries (diffboundary.cpp): before sg_setup, face_bnd[4t+f] is the boundary
 * of face f of tet t (-1 none; both tets of a face name the same boundary) and
 * bnd_comps[2b], bnd_comps[2b+1] the two compartments boundary b joins.  All start closed. */
int sg_set_diff_boundaries(sg_solver* h, int32_t nbnd, const int32_t* face_bnd, const int32_t* bnd_comps);
/* setDiffBoundarySpecDiffusionActive (TOS:2745): open or close species spec across the
 * boundary in both directions, each side diffusing at its own compartment's constant. */
int sg_set_diff_boundary_active(sg_solver* h, int32_t bnd, int32_t spec, int32_t active);
int sg_get_diff_boundary_active(sg_solver* h, int32_t bnd, int32_t spec, int32_t* active);
/* setDiffBoundarySpecDcst (TOS:2865): constant across the boundary, for the direction into
 * direction_comp only (or both with -1); opens that direction.  A side whose compartment
 * has no positive constant for the species sends nothing (as the reference, whose boundary
 * directions belong to the source tet's diffusion rule). */
int sg_set_diff_boundary_dcst(sg_solver* h, int32_t bnd, int32_t spec, double dcst, int32_t direction_comp);

/* One volume reaction of a compartment: dense lhs/upd rows over nspec species as in
 * Compdef::reac_lhs / reac_upd (compdef.hpp:252-266); kcst as Reacdef kcst. */
int sg_add_reac(sg_solver* h, int32_t comp, const uint32_t* lhs, const int32_t* upd, double kcst,
                int32_t* out_idx);

/* One diffusion rule (Diffdef: ligand species, dcst in m^2/s) of a compartment. */
int sg_add_diff(sg_solver* h, int32_t comp, int32_t spec, double dcst, int32_t* out_idx);

/* Batched form: the mesh holds nreal independent realizations, realization r owning
 * tets [tet_offsets[r], tet_offsets[r+1]).  No reference counterpart (the reference runs
 * one realization per process). */
int sg_set_realizations(sg_solver* h, int32_t nreal, const int32_t* tet_offsets);

/* Flatten tables and upload (TOS:479-1088 _setup). */
int sg_setup(sg_solver* h);

/* ---- simulation control (api.hpp:103-140) ---------------------------------- */

int sg_reset(sg_solver* h);                       /* API::reset        TOS reset          */
int sg_run(sg_solver* h, double endtime);         /* API::run          TOS:1507           */
int sg_advance(sg_solver* h, double adv);         /* API::advance      TOS:1955           */
int sg_get_time(sg_solver* h, double* t);         /* API::getTime                          */
int sg_get_update_period(sg_solver* h, int32_t real, double* period); /* TOS:5373 updPeriod */
int sg_get_nsteps(sg_solver* h, uint64_t* n);     /* API::getNSteps                        */
int sg_get_niteration(sg_solver* h, uint64_t* n); /* TetOpSplitP::getNIteration TOS:8322   */
int sg_get_reac_extent(sg_solver* h, int32_t reac, uint64_t* n); /* getReacExtent TOS:8302 */
int sg_get_diff_extent(sg_solver* h, uint64_t* n);               /* getDiffExtent TOS:8314 */
int sg_set_diff_apply_threshold(sg_solver* h, int32_t threshold); /* TOS:8296 */
/* API::checkpoint / API::restore (TOS:217-451): the complete simulation state (counts,
 * time and window indices, constants, clamps, extents, membrane and EField state) in this
 * library's own binary format.  restore needs a solver built from the same mesh and
 * model; the continuation is identical to the uninterrupted run. */
int sg_checkpoint(sg_solver* h, const char* file_name);
int sg_restore(sg_solver* h, const char* file_name);

/* ---- counts (api.hpp:2324-2325, 2582-2583) --------------------------------- */

/* API::getTetSpecCount / setTetSpecCount -> TOS:3830 / TOS:3849. */
int sg_get_tet_count(sg_solver* h, int32_t tet, int32_t spec, double* n);
int sg_set_tet_count(sg_solver* h, int32_t tet, int32_t spec, double n);

/* API::getCompSpecCount / setCompSpecCount -> TOS:2045 / TOS:2051 (distribute_quantity).
 * real selects one realization, or -1 for all. */
int sg_get_comp_count(sg_solver* h, int32_t comp, int32_t spec, int32_t real, double* n);
int sg_set_comp_count(sg_solver* h, int32_t comp, int32_t spec, int32_t real, double n);

/* Whole species row over all tets: getBatchTetSpecCountsNP (TOS:5715) for every tet,
 * and its setter counterpart.  out/in hold ntets uint32 values. */
int sg_get_spec_counts(sg_solver* h, int32_t spec, uint32_t* out);
int sg_set_spec_counts(sg_solver* h, int32_t spec, const uint32_t* in);
/* Every species row at once ([nspec][ntets] uint32, species-major as the device state):
 * one copy and one stream synchronisation each way instead of one per species. */
int sg_get_all_counts(sg_solver* h, uint32_t* out);
int sg_set_all_counts(sg_solver* h, const uint32_t* in);
/* getBatchTetSpecCountsNP (TOS:5715): out[i] = count of spec in tets[i], gathered on the
 * device so that only the n selected values cross to the host. */
int sg_get_batch_tet_counts(sg_solver* h, int32_t spec, const int32_t* tets, int32_t n, double* out);

/* API::setTetSpecClamped (TOS setTetSpecClamped). */
int sg_set_tet_clamped(sg_solver* h, int32_t tet, int32_t spec, int32_t clamped);

/* API::setCompReacK / getCompReacK and setCompDiffD (api_comp.cpp). real = -1: all. */
int sg_set_reac_k(sg_solver* h, int32_t reac, int32_t real, double k);
int sg_get_reac_k(sg_solver* h, int32_t reac, int32_t real, double* k);
int sg_set_diff_d(sg_solver* h, int32_t comp, int32_t spec, int32_t real, double d);

/* ---- membrane triangles and surface reactions (Patchdef, Tri; tri.hpp:339) ------
 * Builder calls (before sg_setup).  The membrane triangles m = 0..ntris-1 each join the
 * SSA unit of their inner tet (the reference's Tri in the same rank as its iTet). */
int sg_set_surface(sg_solver* h, int32_t nsspec, int32_t ntris, const int32_t* tri_inner_tet,
                   const int32_t* tri_patch, const double* tri_area, int32_t npatch);
/* SReac (sreac.cpp:40-68, 305-520): dense rows slhs/supd over nsspec surface species and
 * ilhs/iupd over nspec inner-volume species; kcst in the reference's units. */
int sg_add_sreac(sg_solver* h, int32_t patch, const uint32_t* slhs, const uint32_t* ilhs, const int32_t* supd,
                 const int32_t* iupd, double kcst, int32_t* out_idx);
/* VDepSReac (vdepsreac.cpp:46-76, vdepsreacdef.cpp:194-218): k(V) tabulated at
 * vmin + i dv (V), i < ntab, interpolated linearly at the triangle potential. */
int sg_add_vdep_sreac(sg_solver* h, int32_t patch, const uint32_t* slhs, const uint32_t* ilhs,
                      const int32_t* supd, const int32_t* iupd, double vmin, double dv, int32_t ntab,
                      const double* ktab, int32_t* out_idx);
/* Outer tets of the membrane triangles (Tri::oTet, tri.hpp; -1 = none): the tet on the
 * side of the patch's outer compartment.  Needed when a surface reaction or GHK current
 * reaches the outer volume; the triangles of such patches then join one SSA unit with both
 * of their tets (sreac.cpp:200-300). */
int sg_set_tri_outer(sg_solver* h, const int32_t* tri_outer_tet);
/* Outer-volume terms of surface reaction sreac (Patchdef sreac_lhs_O / sreac_upd_O,
 * sreac.cpp:40-68, 305-520): olhs, dense over nspec, are reactants in the outer tet (then
 * the reaction has no inner-volume reactants and its constant scales with the outer tet's
 * volume, SReacdef::outside); oupd the changes of outer-tet species. */
int sg_set_sreac_outer(sg_solver* h, int32_t sreac, const uint32_t* olhs, const int32_t* oupd);
/* OhmicCurr (ohmiccurrdef): g (S per channel) through surface species sspec, erev (V). */
int sg_add_ohmic(sg_solver* h, int32_t patch, int32_t sspec, double g, double erev, int32_t* out_idx);
int sg_get_tri_count(sg_solver* h, int32_t tri, int32_t sspec, double* n);   /* TOS:4831 getTriSpecCount */
int sg_set_tri_count(sg_solver* h, int32_t tri, int32_t sspec, double n);    /* setTriSpecCount */
/* getPatchSpecCount / setPatchSpecCount; real selects the triangles whose inner tet is in
 * that realization, -1 all of them (counts are distributed by triangle area). */
int sg_get_patch_count(sg_solver* h, int32_t patch, int32_t sspec, int32_t real, double* n);
int sg_set_patch_count(sg_solver* h, int32_t patch, int32_t sspec, int32_t real, double n);
int sg_get_tri_ohmic_i(sg_solver* h, int32_t tri, double* amps);  /* getTriOhmicI: last EField step */
/* GHKcurr (ghkcurr.cpp:168-280, math/ghk.cpp:71-90): channel state sspec of patch passes
 * volume species ion of the given valence, permeability perm (m^3/s per channel), vshift
 * (V), against a fixed outer concentration voconc (M), or, with voconc < 0, against the
 * concentration in the triangle's outer tet (sg_set_tri_outer).  realflux = 1 moves the
 * ions (between the two tets when the outer tet is used); the carried charge is the
 * triangle's GHK current. */
int sg_add_ghk(sg_solver* h, int32_t patch, int32_t sspec, int32_t ion, int32_t valence, double perm,
               double vshift, double voconc, int32_t realflux, int32_t* out_idx);
int sg_set_temp(sg_solver* h, double kelvin);                     /* API::setTemp (default 293.15) */
int sg_get_temp(sg_solver* h, double* kelvin);                    /* API::getTemp */
int sg_get_tri_ghk_i(sg_solver* h, int32_t tri, double* amps);    /* getTriGHKI: last EField step */
/* Surface diffusion (SDiff, sdiff.cpp:62-83, 498-560; TOS:585-630 triangle neighbours):
 * for membrane triangle m and edge e, nbr[3m+e] is the membrane triangle across that edge
 * (-1 = none), nbr_edge its edge index, len the edge length (m) and dist the distance of
 * the two barycentres (m).  Diffusion runs towards neighbours of the same patch. */
int sg_set_tri_neighbours(sg_solver* h, const int32_t* nbr, const int32_t* nbr_edge, const double* len,
                          const double* dist);
/* One surface diffusion rule: surface species sspec diffuses on patch with dcst (m^2/s). */
int sg_add_sdiff(sg_solver* h, int32_t patch, int32_t sspec, double dcst, int32_t* out_idx);

/* ---- membrane potential (EField; api.hpp:140, 2874-2875; efield.hpp:59) ----------
 * Units at this boundary are the reference API's: V, A, s, F/m^2, ohm m, ohm m^2.
 * Inside, the EField works in um, ms, mV, pA, pF, nS like src/steps/solver/efield. */

/* Membrane mesh: all mesh vertices (m, [nverts][3]), every tet's 4 vertices (tets of a
 * compartment conduct; efield.cpp:48-112 initMesh), and the membrane triangles' vertices.
 * method: 0 = FP64 PCG, 1 = FP32 PCG inside FP64 residual refinement; both precondition
 * with Jacobi plus a dense coarse solve on spatial vertex aggregates.  Replaces
 * TetOpSplitP::_setupEField (TOS:1092-1279); switches run() to the EField loop (TOS:1851). */
int sg_set_efield_mesh(sg_solver* h, int32_t nverts, const double* verts, const int32_t* tet_verts,
                       int32_t ntris, const int32_t* tri_verts, int32_t method);
int sg_set_efield_dt(sg_solver* h, double dt);                     /* API::setEfieldDT  */
int sg_get_efield_dt(sg_solver* h, double* dt);                    /* API::getEfieldDT  */
/* Relative residual of the solve, of each FP32 inner solve, and the iteration cap. */
int sg_set_efield_tolerance(sg_solver* h, double rel_tol, double inner_rel_tol, int32_t max_iter);
int sg_set_memb_potential(sg_solver* h, double v);                 /* API::setMembPotential */
int sg_set_memb_capac(sg_solver* h, double cm);                    /* API::setMembCapac     */
int sg_set_memb_vol_res(sg_solver* h, double ra);                  /* API::setMembVolRes    */
int sg_set_memb_res(sg_solver* h, double ro, double vrev);         /* API::setMembRes       */
int sg_get_vert_v(sg_solver* h, int32_t vert, double* v);          /* API::getVertV  TOS:5215 */
int sg_set_vert_v(sg_solver* h, int32_t vert, double v);           /* API::setVertV  TOS:5225 */
int sg_get_tri_v(sg_solver* h, int32_t memb_tri, double* v);       /* API::getTriV (membrane index) */
int sg_set_vert_v_clamped(sg_solver* h, int32_t vert, int32_t clamped); /* API::setVertVClamped */
int sg_set_vert_iclamp(sg_solver* h, int32_t vert, double amps);   /* API::setVertIClamp    */
/* EField steps taken, CG iterations, device ms in the solves, last relative residual. */
int sg_get_efield_stats(sg_solver* h, uint64_t* steps, uint64_t* iterations, double* solve_ms,
                        double* last_rel_residual);

/* ---- device options (no reference counterpart) ------------------------------ */

/* EField accuracy check: after each step (either method) also solve the same system in
 * FP64 from zero to rel_tol (not counted in the solve time) and record the largest
 * per-vertex |V - V_fp64| / |V_fp64|; read it with sg_get_efield_check. */
int sg_set_efield_check(sg_solver* h, int32_t on, double rel_tol);
int sg_get_efield_check(sg_solver* h, uint64_t* steps, double* max_rel, double* last_rel);
/* EField solve form: 1 = every CG iteration inside one cooperative launch (grid barriers
 * between the phases), 0 = three kernel launches per iteration. */
int sg_set_efield_persistent(sg_solver* h, int32_t on);
/* Polls of one grid-barrier wait (about 100 ns each) after which the persistent EField
 * solve gives up: the launch ends and the step returns SG_EDEVICE ("a grid barrier wait
 * timed out"), with the device left usable.  Default 2^22 (about half a second).  No
 * counterpart in the reference (whose solve has no device-side waits); small values make
 * the error path testable. */
int sg_set_efield_barrier_limit(sg_solver* h, uint32_t polls);

/* Mixed method with the persistent solve: one FP32 CG with reliable updates (on, default;
 * the FP64 residual b - A x replaces the FP32 one whenever the FP32 residual norm has
 * fallen by the factor delta, default 0.1, since the last replacement) or restarted FP32
 * inner solves inside an FP64 refinement loop (off).  Replaces the PETSc solve's precision
 * choice (dVsolver_petsc.cpp:163-260); no reference counterpart for the factor. */
int sg_set_efield_reliable_updates(sg_solver* h, int32_t on, double delta);

/* Window-kernel launch shape: block in {64,128,256}; grid > 0 blocks, 0 = occupancy-sized
 * (blocks stride over the tets), -1 = one tet per thread. */
int sg_set_launch(sg_solver* h, int32_t block, int32_t grid);
int sg_get_launch(sg_solver* h, int32_t* block, int32_t* grid);
/* Autotune the launch shape at the next run() with more than 25 windows: after one
 * untimed window, twelve candidates are timed on one window each in list order and on one
 * more in reverse order (drift of the per-window work cancels): block {64,128,256} x grid
 * {occupancy-sized (0), one tet per thread (-1)}; block 256, grid -1 at a shared-memory
 * carveout of 75%; split windows at block 128 and 256, grid -1; the persistent form
 * (sg_set_persistent) at block 256 with 2, 4 and 8 tets per lane (skipped unless every
 * realization takes the same windows and the model has no membrane).  The fastest is kept (the sample path does not depend on the shape).  The
 * twelve sums (ms, in that order) are read back with sg_get_autotune_ms, the kept
 * carveout with sg_get_carveout. */
int sg_set_autotune(sg_solver* h, int32_t on);
int sg_get_carveout(sg_solver* h, int32_t* percent);
/* Window as two kernels: reactions (gather, SSA) with one thread per tet, then the
 * diffusion leave with one thread per tet over its diffusing species; the same results as
 * the fused kernel.  Models with membrane triangles run split by default and always when
 * they have merged SSA units.  The autotuner also tries it. */
int sg_set_split(sg_solver* h, int32_t on);
int sg_get_split(sg_solver* h, int32_t* on);
/* Persistent form of the batched window loop (TOS:1528-1839 for every realization): the
 * windows of a run() call (up to 64 per launch) of every realization in one cooperative
 * launch, warps taking chunks of 32 x tets_per_lane (1, 2, 4 or 8) tets of one realization
 * in window order and waiting, bounded, until that realization has finished the previous
 * window; inside a chunk the tets whose first draw falls in the window run their SSA 32 at
 * a time.  The same results as the window launches, bit for bit.  Used when the model has
 * no membrane triangles and every realization takes the same windows; the per-window
 * conservation check does not run inside it. */
int sg_set_persistent(sg_solver* h, int32_t on, int32_t tets_per_lane);
int sg_get_persistent(sg_solver* h, int32_t* on, int32_t* tets_per_lane);
/* Polls (about 100 ns each) a persistent launch's wait on a realization makes before it
 * gives up; run() then fails with "a persistent window launch gave up waiting" and the
 * state of that call is undefined.  Default 2^22 (about half a second). */
int sg_set_window_wait_limit(sg_solver* h, uint32_t polls);
int sg_get_autotune_ms(sg_solver* h, float* ms, int32_t cap, int32_t* count);
/* Replay window launches from a captured CUDA graph of 16 windows (on by default). */
int sg_set_graphs(sg_solver* h, int32_t on);
/* Per-window bit-exact molecule-conservation check (on by default). */
int sg_set_conservation_check(sg_solver* h, int32_t on);
/* Device status word (SG_ERR_* bits). */
int sg_get_status(sg_solver* h, uint32_t* status);
/* The CUDA stream (cudaStream_t) every kernel of this solver is launched on. */
int sg_get_stream(sg_solver* h, void** stream);
/* CUDA-event timing of the window launches of each run() (resets the totals).  The
 * reference's MPI_PROFILING timers (getCompTime etc., TOS:8330-8359) have this role. */
int sg_set_profiling(sg_solver* h, int32_t on);
/* Device ms spent in window launches and their count since profiling was switched on,
 * and the number of kernels this solver has launched since creation. */
int sg_get_profile(sg_solver* h, double* window_ms, uint64_t* windows, uint64_t* launches);

/* ---- allocation-free entry point (no counterpart in the reference) ----------
 *
 * For callers that cannot call cudaMalloc: host programs whose device memory comes only
 * from their own pool allocator (a simulator embedding this step next to other GPU
 * code that owns the device's memory), and long-running loops that must not pay an
 * allocation's implicit device-wide synchronisation on every call.
 * It advances one realization in one compartment (every tet) from t0 to t_end with the
 * same window kernel as sg_run, and returns with counts complete.  The caller owns all
 * inputs and outputs; the library allocates nothing.  Its scratch (packed mesh tables,
 * face-outflow double buffer, counters) is one fixed device array of
 * SG_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until exit.
 *
 * Limits: ntets <= SG_NOALLOC_MAX_TETS, ntets * nspec <= SG_NOALLOC_MAX_TET_SPECIES,
 * nspec <= 32, nreac <= SG_NOALLOC_MAX_REACS; larger problems return SG_EARG.
 *
 * Device buffers (current device): counts [nspec][ntets] uint32 (in/out); vol [ntets],
 * neighb [ntets][4] (-1 = none), area [ntets][4], dist [ntets][4] as in sg_set_mesh.
 * Host arrays: lhs / upd [nreac][nspec] dense rows as in sg_add_reac, kcst [nreac],
 * dcst [nspec] (0 = species does not diffuse).  seed, window0 (windows already run in
 * earlier calls: continues the same Philox streams) and t0 give the same results as a
 * solver created with that seed and run over the same times.  stream is a cudaStream_t
 * (NULL = legacy default stream).  The call synchronises that stream twice: once to
 * read the largest face coefficient (which sets the update period and the number of
 * windows) and once at the end to read the device status word.
 * windows_out / period_out (optional) receive the windows run and the update period.
 *
 * The first call on a device looks up the scratch array's device address (once per
 * device, cached for the process); make that first call before any stream capture
 * starts, and do not call this entry point after cudaDeviceReset on that device.
 * Every call reuses the same array and clears what must start at zero (counters,
 * status, face outflow); calls that overlap on the GPU race on it. */
#define SG_NOALLOC_MAX_TETS 65536
#define SG_NOALLOC_MAX_TET_SPECIES 262144
#define SG_NOALLOC_MAX_REACS 64
#define SG_NOALLOC_SCRATCH_BYTES 11022080
int sg_run_noalloc(int32_t ntets, int32_t nspec, int32_t nreac, uint32_t* counts, const double* vol,
                   const int32_t* neighb, const double* area, const double* dist, const uint32_t* lhs,
                   const int32_t* upd, const double* kcst, const double* dcst, uint64_t seed, double t0,
                   double t_end, uint64_t window0, void* stream, uint64_t* windows_out,
                   double* period_out);

#ifdef __cplusplus
}
#endif

#endif /* STEPS_B200_H */
