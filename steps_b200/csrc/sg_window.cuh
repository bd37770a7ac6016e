// One operator-split window for every unit (tet) of every active realization.
//
// Reference path restated (src/steps/mpi/tetopsplit/tetopsplit.cpp, "TOS"):
//   TOS:1528-1839  _runWithoutEField: SSA over the window, then diffusion, then sync.
//   TOS:1569-1588  SSA loop: dt ~ Exp(a0); stop when cumulative dt passes the window.
//   TOS:1633-1712  diffusion: population, occupancy-weighted mean, Bernoulli on the
//                  fraction, Binomial(mean_n, min(1, window * scaledDcst)).
//   diff.cpp:515-585  multinomial face split by sequential conditional binomials.
//   reac.cpp:184-251  propensity h_mu * ccst and apply with occupancy integration
//                  (tet.cpp:318-340).
//
// The reference runs one composition-rejection SSA over all reactions of a rank.
// Reactions only touch one tet, so an independent direct-method SSA per tet inside
// the window has the same law.  Diffusion is two-phase: each (tet, species) writes
// its per-face outflow in window w; window w+1 first gathers the inflow through
// the reverse-face table, so every tet only writes its own counts.
#pragma once
#include "sg_rng.cuh"
#include "sg_surf.cuh"
#include "sg_types.h"

namespace sg {

__device__ __forceinline__ double reac_ccst(const sg_reac* rc, double k, double ivs) {
    int o = rc->order;
    if (o == 1) return k;
    if (o == 0) return k / ivs;
    double c = k * ivs;
    for (int i = 2; i < o; ++i) c = c * ivs;
    return c;
}

// h_mu * ccst, counts read from this thread's column of shared memory.
__device__ __forceinline__ double reac_prop(const sg_reac* rc, const uint32_t* sc, int stride,
                                            double ccst) {
    double h = 1.0;
    int nl = rc->nlhs;
    for (int i = 0; i < nl; ++i) {
        int s = rc->lhs_spec[i];
        uint32_t o = (uint32_t)rc->lhs_ord[i];
        uint32_t c = sc[s * stride];
        if (o > c) return 0.0;
        if (o >= 4) h = h * (double)(c - 3);
        if (o >= 3) h = h * (double)(c - 2);
        if (o >= 2) h = h * (double)(c - 1);
        h = h * (double)c;
    }
    return h * ccst;
}

// h_mu * ccst through the reaction's closed form (sg_reac::fast); equal bit for bit to
// reac_prop for every count: the exact integer product rounded once is the value of the
// reference's double product of exact factors, and a zero factor gives +0 in both.
__device__ __forceinline__ double reac_prop_fast(const sg_reac* rc, const uint32_t* sc, int stride, double ccst) {
    const uint32_t code = rc->fast;
    const uint32_t kind = code & 0xFFu;
    if (kind == SG_RK_GENERIC) return reac_prop(rc, sc, stride, ccst);
    unsigned long long h = 1ull;
    if (kind != SG_RK_ZERO) {
        const uint32_t ca = sc[((code >> 8) & 0xFFu) * stride];
        uint32_t cb = 1u;
        if (kind == SG_RK_PAIR) cb = sc[(code >> 16) * stride];
        else if (kind == SG_RK_DIMER) cb = ca - 1u;  // ca = 0 wraps, and 0 * cb = 0
        h = (unsigned long long)ca * cb;
    }
    return (double)h * ccst;
}

// Margin of the first waiting-time test: with x = a0 T, (1 - u) > x (1 + 2^-40) implies
// -log(u) / a0 > T as the full computation rounds it (-log u >= 1 - u; the project log is
// within a few ulp and the division and the products round by 2^-53 each), so the log and
// the division can be skipped without changing any outcome.
#define SG_SQUEEZE 1.0000000000009095  // 1 + 2^-40

__device__ __forceinline__ int find_real(const sg_real* reals, int nreal, int t) {
    if (nreal == 1) return 0;
    int lo = 0, hi = nreal - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&reals[mid].tet_begin) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum of a uint32 over the 32 lanes as 64 bits, in every lane: two warp reductions of the
// 16-bit halves (neither can overflow 32 bits) instead of a 64-bit shuffle tree.
__device__ __forceinline__ unsigned long long warp_total_u32(uint32_t c) {
    const uint32_t lo = __reduce_add_sync(0xffffffffu, c & 0xFFFFu);
    const uint32_t hi = __reduce_add_sync(0xffffffffu, c >> 16);
    return (unsigned long long)lo + ((unsigned long long)hi << 16);
}

// First tet of the warp's next chunk of 32: from the launch's work counter (dynamic
// schedule) or the warp's fixed stride (static).  Uniform across the warp.
__device__ __forceinline__ int next_warp_base(unsigned int* ctr, int it, int BLOCK) {
    if (ctr) {
        unsigned int c = 0u;
        if ((threadIdx.x & 31) == 0) c = atomicAdd(ctr, 1u);
        return (int)__shfl_sync(0xffffffffu, c, 0) * 32;
    }
    return (int)((blockIdx.x + (unsigned)it * gridDim.x) * (unsigned)BLOCK + (threadIdx.x & ~31u));
}

// Asynchronous global -> shared copies (cp.async) of 4 and 8 bytes; a thread reads what it
// copied after sg_cp_async_wait.
__device__ __forceinline__ void sg_cp_async4(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void sg_cp_async8(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void sg_cp_async_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared-memory carve-up for a block of BLOCK threads.
struct smem_layout {
    uint32_t* cnt;             // [S][BLOCK]
    double* tdel;              // [S][BLOCK] sum over count changes of (change) x (time of change)
    double* prop;              // [R][BLOCK] propensities of this thread's tet
    sg_reac* reac;             // [R] copy of the reaction table
    unsigned long long* tot;   // [S]
    unsigned long long* moved; // [1]
    unsigned int* ext;         // [R]
    int* flag;                 // [2]
};

__host__ __device__ inline size_t smem_bytes(int block, int nspec, int nreac) {
    size_t b = (size_t)block * nspec * 4;
    b = (b + 15) & ~(size_t)15;
    b += (size_t)block * nspec * 8;
    b += (size_t)block * nreac * 8;
    b += (size_t)nreac * sizeof(sg_reac);
    b = (b + 7) & ~(size_t)7;
    b += (size_t)nspec * 8 + 8;
    b += (size_t)nreac * 4 + 4;
    b = (b + 7) & ~(size_t)7;
    b += 16;
    return b;
}

__device__ inline smem_layout carve(unsigned char* base, int block, int nspec, int nreac) {
    smem_layout L;
    size_t b = (size_t)block * nspec * 4;
    L.cnt = (uint32_t*)base;
    b = (b + 15) & ~(size_t)15;
    L.tdel = (double*)(base + b);
    b += (size_t)block * nspec * 8;
    L.prop = (double*)(base + b);
    b += (size_t)block * nreac * 8;
    L.reac = (sg_reac*)(base + b);
    b += (size_t)nreac * sizeof(sg_reac);
    b = (b + 7) & ~(size_t)7;
    L.tot = (unsigned long long*)(base + b);
    b += (size_t)nspec * 8;
    L.moved = (unsigned long long*)(base + b);
    b += 8;
    L.ext = (unsigned int*)(base + b);
    b += (size_t)nreac * 4 + 4;
    b = (b + 7) & ~(size_t)7;
    L.flag = (int*)(base + b);
    return L;
}

// SSA for one tet over [0, T): direct method with FP64 propensities, waiting
// times -log(U)/a0.  Occupancy: the time integral of a count over the window is
// c_end T - sum_k (change_k) t_k, so only sum_k (change_k) t_k is kept per species
// (tdel); the reference keeps the running integral and the last update time instead
// (tet.cpp:318-340), the same quantity up to rounding.
__device__ __forceinline__ void tet_ssa(const sg_window_args& a, const smem_layout& L, int tid,
                                        int BLOCK, int rb, int re, const double* K, double ivs,
                                        uint32_t clampm, double T, sg_stream* st) {
    uint32_t* sc = L.cnt + tid;
    double* sd = L.tdel + tid;
    double* sp = L.prop + tid;  // sp[q * BLOCK]: propensity of reaction q in this tet
    double tt = 0.0;
    // Propensities are kept per reaction and only the ones whose reactants changed are
    // re-evaluated after an event; a0 is always re-summed in reaction order, so every
    // value equals a full re-evaluation.
    uint32_t changed = 0xFFFFFFFFu;
    for (;;) {
        double a0 = 0.0;
        for (int q = rb; q < re; ++q) {
            const sg_reac* rc = &L.reac[q];
            if ((rc->lhs_mask & changed) || changed == 0xFFFFFFFFu)
                sp[q * BLOCK] = reac_prop_fast(rc, sc, BLOCK, reac_ccst(rc, __ldg(&K[q]), ivs));
            a0 = a0 + sp[q * BLOCK];
        }
        if (!(a0 > 0.0)) break;
        const double u = sg_u01_oc(sg_next_u32(st));
        // First draw of the window: most units see no event, decided without the log.
        if (tt == 0.0 && 1.0 - u > (a0 * T) * SG_SQUEEZE) break;
        double dt = -sg_log(u) / a0;
        if (tt + dt > T) break;
        tt = tt + dt;
        double target = sg_u01_co(sg_next_u32(st)) * a0;
        double cum = 0.0;
        int sel = -1, lastnz = -1;
        for (int q = rb; q < re; ++q) {
            double p = sp[q * BLOCK];
            if (p > 0.0) {
                lastnz = q;
                cum = cum + p;
                if (target < cum) {
                    sel = q;
                    break;
                }
            }
        }
        if (sel < 0) sel = lastnz;
        if (sel < 0) break;
        const sg_reac* rc = &L.reac[sel];
        changed = rc->upd_mask & ~clampm;
        int nu = rc->nupd;
        for (int i = 0; i < nu; ++i) {
            int s = rc->upd_spec[i];
            if ((clampm >> s) & 1u) continue;
            uint32_t old = sc[s * BLOCK];
            long long nc = (long long)old + rc->upd_delta[i];
            if (nc < 0 || nc > 0xFFFFFFFFll) {
                atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
                nc = nc < 0 ? 0 : 0xFFFFFFFFll;
            }
            sd[s * BLOCK] = sd[s * BLOCK] + (double)(nc - (long long)old) * tt;
            sc[s * BLOCK] = (uint32_t)nc;
        }
        atomicAdd(&L.ext[sel], 1u);
    }
}

// First pass of a split window's SSA: the tet's total propensity and its first draw.
// False when that draw shows, by the squeeze of tet_ssa, that no event falls in the window
// (the tet's SSA is then complete); true when the tet has to run tet_ssa, which sums the
// same propensities in the same order and redraws the same first uniform.
__device__ __forceinline__ bool tet_may_fire(const smem_layout& L, int tid, int BLOCK, int rb, int re,
                                             const double* K, double ivs, double T, sg_stream* st) {
    const uint32_t* sc = L.cnt + tid;
    double a0 = 0.0;
    for (int q = rb; q < re; ++q) {
        const sg_reac* rc = &L.reac[q];
        a0 = a0 + reac_prop_fast(rc, sc, BLOCK, reac_ccst(rc, __ldg(&K[q]), ivs));
    }
    if (!(a0 > 0.0)) return false;
    const double u = sg_u01_oc(sg_next_u32(st));
    return !(1.0 - u > (a0 * T) * SG_SQUEEZE);
}

// Whole SSA of tet t from its gathered counts (stored in counts by the first pass), with
// its stream restarted, so the draws are the ones the first pass took; then its counts,
// the nonzero change-time sums of its diffusing species and tmask.
__device__ __forceinline__ void tet_ssa_queued(const sg_window_args& a, const smem_layout& L, int tid, int BLOCK,
                                               int t) {
    const int S = a.nspec;
    const int r = find_real(a.reals, a.nreal, t);
    const sg_real* rl = &a.reals[r];
    const double rt = rl->t, rend = rl->t_end, per = rl->period;
    const double T = (rt + per > rend) ? rend - rt : per;
    const unsigned long long w = rl->window;
    const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
    const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
    for (int s = 0; s < S; ++s) {
        L.cnt[s * BLOCK + tid] = a.counts[(size_t)s * a.ntets + t];
        L.tdel[s * BLOCK + tid] = 0.0;
    }
    sg_stream st;
    sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)(t - rl->tet_begin), w, SG_PURPOSE_WINDOW);
    tet_ssa(a, L, tid, BLOCK, __ldg(&a.comp_reac_begin[comp]), __ldg(&a.comp_reac_begin[comp + 1]),
            a.kcst + (size_t)r * a.nreac, __ldg(&a.ivs[t]), clampm, T, &st);
    uint32_t tm = 0u;
    for (int s = 0; s < S; ++s) {
        const int ds = __ldg(&a.diff_slot[s]);
        const double sdv = L.tdel[s * BLOCK + tid];
        if (ds >= 0 && sdv != 0.0) {
            a.tdel[(size_t)ds * a.ntets + t] = sdv;
            tm |= 1u << s;
        }
        a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
    }
    if (a.tmask) a.tmask[t] = tm;
}

// SSA of a unit made of a tet and up to four membrane triangles (inner tet = this tet):
// volume reactions, then each triangle's surface reactions, in a fixed order.  All
// propensities are re-evaluated after every event (such units are few).  Triangle counts
// and their time integrals (ohmic currents) are written back at the end of the window.
static __device__ __noinline__ void tet_ssa_surf(const sg_window_args& a, const smem_layout& L, const surf_layout& SL,
                                          int tid, int BLOCK, int rb, int re, const double* K, double ivs,
                                          uint32_t clampm, double T, sg_stream* st, int4 tris,
                                          unsigned long long w, int pending) {
    const sg_surf_args& sa = a.surf;
    const int SS = sa.nsspec, RSP = sa.max_sreac_per_patch, M = sa.ntris;
    uint32_t* sc = L.cnt + tid;
    double* sd = L.tdel + tid;
    const int mm[4] = {tris.x, tris.y, tris.z, tris.w};
    int pb[4], pe[4], pj[4];
    double area[4], vm[4];
    for (int j = 0; j < 4; ++j) {
        pb[j] = pe[j] = 0;
        pj[j] = -1;
        area[j] = 0.0;
        vm[j] = 0.0;
        const int m = mm[j];
        if (m < 0) continue;
        const int p = sa.tri_patch[m];
        pj[j] = p;
        pb[j] = sa.patch_sreac_begin[p];
        pe[j] = sa.patch_sreac_begin[p + 1];
        area[j] = sa.tri_area[m];
        vm[j] = sa.tri_V ? sa.tri_V[m] : 0.0;
        for (int s = 0; s < SS; ++s) {
            uint32_t c = sa.tri_counts[(size_t)s * M + m];
            if (pending && sa.tri_outflow) {
                // Gather last window's surface-diffusion inflow (slot e: from the neighbour
                // across edge e).
                const int sd = sa.sdiff_slot[s];
                if (sd >= 0 && sa.sdcst[(size_t)p * SS + s] > 0.0) {
                    const uint4 v = reinterpret_cast<const uint4*>(
                        sa.tri_outflow + (size_t)((w + 1) & 1ull) * sa.nsdiff * M * 4)[(size_t)sd * M + m];
                    const int4 nb = reinterpret_cast<const int4*>(sa.snbr)[m];
                    unsigned long long sum = c;
                    if (nb.x >= 0) sum += v.x;
                    if (nb.y >= 0) sum += v.y;
                    if (nb.z >= 0) sum += v.z;
                    if (sum > 0xFFFFFFFFull) {
                        atomicOr(a.status, SG_ERR_OVERFLOW);
                        sum = 0xFFFFFFFFull;
                    }
                    c = (uint32_t)sum;
                }
            }
            SL.cnt[(j * SS + s) * BLOCK + tid] = c;
            SL.occ[(j * SS + s) * BLOCK + tid] = 0.0;
            SL.last[(j * SS + s) * BLOCK + tid] = 0.0;
        }
    }
    double tt = 0.0;
    for (;;) {
        double a0 = 0.0;
        for (int q = rb; q < re; ++q) {
            const sg_reac* rc = &L.reac[q];
            double pq = reac_prop(rc, sc, BLOCK, reac_ccst(rc, __ldg(&K[q]), ivs));
            L.prop[q * BLOCK + tid] = pq;
            a0 = a0 + pq;
        }
        for (int j = 0; j < 4; ++j) {
            for (int q = pb[j]; q < pe[j]; ++q) {
                const sg_sreac& r = sa.sreacs[q];
                double k = (r.vdep >= 0) ? vdep_k(sa, r.vdep, vm[j], a.status) : sa.skcst[q];
                double h = sreac_h(r, SL.cnt + (size_t)j * SS * BLOCK + tid, sc, BLOCK);
                double pq = h * sreac_ccst(r, k, ivs, area[j]);
                SL.prop[(j * RSP + (q - pb[j])) * BLOCK + tid] = pq;
                a0 = a0 + pq;
            }
            // GHK currents of the triangle's patch, after its reactions (ghkcurr.cpp:168).
            int kk = pe[j] - pb[j];
            for (int g = 0; g < sa.nghk && pj[j] >= 0; ++g) {
                const sg_ghk& gh = sa.ghks[g];
                if (gh.patch != pj[j]) continue;
                const double rt = ghk_rate(gh, vm[j], sc[gh.ion * BLOCK], SL.cnt[(j * SS + gh.sspec) * BLOCK + tid],
                                           ivs, sa.temp, a.status);
                const double pq = fabs(rt);
                SL.prop[(j * RSP + kk) * BLOCK + tid] = pq;
                a0 = a0 + pq;
                ++kk;
            }
        }
        if (!(a0 > 0.0)) break;
        double dt = -sg_log(sg_u01_oc(sg_next_u32(st))) / a0;
        if (tt + dt > T) break;
        tt = tt + dt;
        double target = sg_u01_co(sg_next_u32(st)) * a0;
        double cum = 0.0;
        int sj = -2, sq = -1, lj = -2, lq = -1;  // selected (slot or -1 = volume, index)
        for (int q = rb; q < re && sj == -2; ++q) {
            double pq = L.prop[q * BLOCK + tid];
            if (pq > 0.0) {
                lj = -1;
                lq = q;
                cum = cum + pq;
                if (target < cum) {
                    sj = -1;
                    sq = q;
                }
            }
        }
        for (int j = 0; j < 4 && sj == -2; ++j) {
            for (int q = pb[j]; q < pe[j]; ++q) {
                double pq = SL.prop[(j * RSP + (q - pb[j])) * BLOCK + tid];
                if (pq > 0.0) {
                    lj = j;
                    lq = q;
                    cum = cum + pq;
                    if (target < cum) {
                        sj = j;
                        sq = q;
                        break;
                    }
                }
            }
            // GHK events are coded as sq = -10 - g.
            int kk = pe[j] - pb[j];
            for (int g = 0; g < sa.nghk && pj[j] >= 0 && sj == -2; ++g) {
                if (sa.ghks[g].patch != pj[j]) continue;
                double pq = SL.prop[(j * RSP + kk) * BLOCK + tid];
                ++kk;
                if (pq > 0.0) {
                    lj = j;
                    lq = -10 - g;
                    cum = cum + pq;
                    if (target < cum) {
                        sj = j;
                        sq = -10 - g;
                    }
                }
            }
        }
        if (sj == -2) {
            sj = lj;
            sq = lq;
        }
        if (sq <= -10) {
            // GHK event on triangle slot sj (ghkcurr.cpp:230-280): one ion out (efflux) or in,
            // z elementary charges out or in for the triangle's current.
            const sg_ghk& gh = sa.ghks[-10 - sq];
            const int m = mm[sj];
            const double rt = ghk_rate(gh, vm[sj], sc[gh.ion * BLOCK], SL.cnt[(sj * SS + gh.sspec) * BLOCK + tid],
                                       ivs, sa.temp, a.status);
            const bool eff = rt >= 0.0;
            if (gh.realflux && !((clampm >> gh.ion) & 1u)) {
                const int s = gh.ion;
                const uint32_t old = sc[s * BLOCK];
                long long nc = (long long)old + (eff ? -1 : 1);
                if (nc < 0 || nc > 0xFFFFFFFFll) {
                    atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
                    nc = nc < 0 ? 0 : 0xFFFFFFFFll;
                }
                sd[s * BLOCK] = sd[s * BLOCK] + (double)(nc - (long long)old) * tt;
                sc[s * BLOCK] = (uint32_t)nc;
            }
            atomicAdd((unsigned long long*)&sa.tri_echarge[m],
                      (unsigned long long)(long long)(eff ? gh.valence : -gh.valence));
            atomicAdd(a.surf_ext, 1ull);
            continue;
        }
        if (sq < 0) break;
        if (sj == -1) {
            const sg_reac* rc = &L.reac[sq];
            for (int i = 0; i < rc->nupd; ++i) {
                int s = rc->upd_spec[i];
                if ((clampm >> s) & 1u) continue;
                uint32_t old = sc[s * BLOCK];
                long long nc = (long long)old + rc->upd_delta[i];
                if (nc < 0 || nc > 0xFFFFFFFFll) {
                    atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
                    nc = nc < 0 ? 0 : 0xFFFFFFFFll;
                }
                sd[s * BLOCK] = sd[s * BLOCK] + (double)(nc - (long long)old) * tt;
                sc[s * BLOCK] = (uint32_t)nc;
            }
            atomicAdd(&L.ext[sq], 1u);
        } else {
            const sg_sreac& r = sa.sreacs[sq];
            for (int i = 0; i < r.nsupd; ++i) {
                size_t o = (size_t)(sj * SS + r.supd_spec[i]) * BLOCK + tid;
                uint32_t old = SL.cnt[o];
                SL.occ[o] = SL.occ[o] + (double)old * (tt - SL.last[o]);
                SL.last[o] = tt;
                long long nc = (long long)old + r.supd_delta[i];
                if (nc < 0 || nc > 0xFFFFFFFFll) {
                    atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
                    nc = nc < 0 ? 0 : 0xFFFFFFFFll;
                }
                SL.cnt[o] = (uint32_t)nc;
            }
            for (int i = 0; i < r.niupd; ++i) {
                int s = r.iupd_spec[i];
                if ((clampm >> s) & 1u) continue;
                uint32_t old = sc[s * BLOCK];
                long long nc = (long long)old + r.iupd_delta[i];
                if (nc < 0 || nc > 0xFFFFFFFFll) {
                    atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
                    nc = nc < 0 ? 0 : 0xFFFFFFFFll;
                }
                sd[s * BLOCK] = sd[s * BLOCK] + (double)(nc - (long long)old) * tt;
                sc[s * BLOCK] = (uint32_t)nc;
            }
            atomicAdd(a.surf_ext, 1ull);
        }
    }
    for (int j = 0; j < 4; ++j) {
        const int m = mm[j];
        if (m < 0) continue;
        for (int s = 0; s < SS; ++s) {
            size_t o = (size_t)(j * SS + s) * BLOCK + tid;
            uint32_t c = SL.cnt[o];
            sa.tri_counts[(size_t)s * M + m] = c;
            const double occ = SL.occ[o] + (double)c * (T - SL.last[o]);
            sa.spec_int[(size_t)s * M + m] += occ;
            if (sa.tri_occ) {
                const int sd = sa.sdiff_slot[s];
                if (sd >= 0) sa.tri_occ[(size_t)sd * M + m] = occ;
            }
        }
    }
}

__device__ __forceinline__ uint4 leave_split(sg_stream* st, uint32_t mean_n, double t1, double c0, double c1,
                                             double c2, double odd1, double odd2, double odd3, const double* rcp,
                                             const double* rcpl, const double* lnf, uint32_t* out_kn);

// Inflow of species s through the diffusion-boundary faces of tet t (slots v.f of the tet's
// own inflow): counted when the tet behind face f diffuses s, because that tet then wrote
// the slot this window (0 while the boundary is closed in its direction).
__device__ __forceinline__ unsigned long long bnd_inflow(const sg_window_args& a, int t, int r, int s, uint4 v) {
    const uint32_t bf = __ldg(&a.bface[t]);
    if (bf == 0xFFFFFFFFu) return 0ull;
    const uint32_t vv[4] = {v.x, v.y, v.z, v.w};
    unsigned long long sum = 0ull;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (((bf >> (8 * f)) & 0xFFu) == 0xFFu) continue;
        const int n = __ldg(&a.bnbr[(size_t)t * 4 + f]) >> 2;
        const int cn = a.comp ? __ldg(&a.comp[n]) : 0;
        if (cn >= 0 && __ldg(&a.dcst[((size_t)r * a.ncomp + cn) * a.nspec + s]) > 0.0) sum += vv[f];
    }
    return sum;
}

// Rates of tet t for species s through its faces when some face is a diffusion boundary:
// same-compartment faces at D, boundary faces at the boundary's rate for the tet's side
// (closed: 0), each times the face coefficient A / (V d).  Returns the total and the
// conditional selectors in g (the last open face takes the rest), as the host builds them
// for tets without boundary faces.
__device__ __forceinline__ double bnd_split(const sg_window_args& a, int t, int comp, int s, double D, int4 nb,
                                            float4* g) {
    const uint32_t bf = __ldg(&a.bface[t]);
    const float4 cf = __ldg(reinterpret_cast<const float4*>(a.bcoef) + t);
    const float c4[4] = {cf.x, cf.y, cf.z, cf.w};
    const int n4[4] = {nb.x, nb.y, nb.z, nb.w};
    double r[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        r[f] = 0.0;
        if (n4[f] >= 0) {
            r[f] = (double)c4[f] * D;
        } else {
            const uint32_t b = (bf >> (8 * f)) & 0xFFu;
            if (b != 0xFFu) {
                const int side = (comp == __ldg(&a.bcomps[b * 2])) ? 0 : 1;
                const double v = __ldg(&a.btab[((size_t)b * a.nspec + s) * 2 + side]);
                if (v < -1.5) r[f] = (double)c4[f] * D;
                else if (v >= 0.0) r[f] = (double)c4[f] * v;
            }
        }
    }
    const double tot = r[0] + r[1] + r[2] + r[3];
    int lastf = -1;
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (r[f] > 0.0) lastf = f;
    double rem = tot;
    float cs[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        double c = 0.0;
        if (r[f] > 0.0) {
            c = (f == lastf) ? 1.0 : r[f] / rem;
            if (c > 1.0) c = 1.0;
            rem -= r[f];
        }
        cs[f] = (float)c;
    }
    *g = make_float4(cs[0], cs[1], cs[2], 0.0f);
    return tot;
}

// Scatter of the boundary faces' leavers into the neighbours' slots.
__device__ __forceinline__ void bnd_scatter(const sg_window_args& a, int t, uint32_t* po, uint4 k) {
    const uint32_t bf = __ldg(&a.bface[t]);
    const uint32_t kk[4] = {k.x, k.y, k.z, k.w};
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (((bf >> (8 * f)) & 0xFFu) != 0xFFu) po[__ldg(&a.bnbr[(size_t)t * 4 + f])] = kk[f];
}

// Diffusion leave of one (tet, species) with pop > 0 molecules (TOS:1633-1712,
// diff.cpp:473-585): the occupancy mean n = c_end - sd / T with a Bernoulli on its
// fraction, Binomial(n, min(1, t1)) leaving (t1 = T D G, or T times the summed face rates
// at a diffusion boundary), split over the faces by conditional
// binomials on the selectors c0..c2 (the last face takes the rest).  Each (tet, species)
// draws from its own stream (purpose SG_PURPOSE_DIFF + species), so the result does not
// depend on the SSA's draws, on the other species or on which kernel runs it.
__device__ __forceinline__ uint4 leave_species(uint64_t seed, uint32_t real, uint32_t unit, unsigned long long w,
                                               uint32_t s, uint32_t pop, double sd, double invT, double t1,
                                               const double* c, double odd1, double odd2, double odd3,
                                               const double* rcp, const double* rcpl, const double* lnf,
                                               sg_stream* st, uint32_t* out_kn) {
    sg_stream_init(st, seed, real, unit, w, SG_PURPOSE_DIFF + s);
    if (t1 >= 1.0) t1 = 1.0;
    uint32_t mean_n = pop;
    if (sd != 0.0) {
        double nbar = (double)pop - sd * invT;
        if (nbar > (double)pop) nbar = (double)pop;
        double nint = floor(nbar);
        double frc = nbar - nint;
        mean_n = (uint32_t)nint;
        if (frc > 0.0) {
            if (sg_u01_co(sg_next_u32(st)) < frc) mean_n += 1u;
        }
    }
    return leave_split(st, mean_n, t1, c[0], c[1], c[2], odd1, odd2, odd3, rcp, rcpl, lnf, out_kn);
}

// Below this many molecules the leave draws each molecule's fate (stay, or which face)
// instead of four binomials: the reference's own per-molecule direction draws for small
// counts (diff.cpp:473-512), with the leaving draw folded into the same uniform.
#define SG_PM_MAX 16u

// Threshold of a probability x in [0, 1] for a 32-bit draw v: v < sg_thr(x) exactly when
// v 2^-32 < x (the scaling by 2^32 is exact).
__host__ __device__ __forceinline__ uint64_t sg_thr(double x) {
    return x > 0.0 ? (uint64_t)ceil(x * 4294967296.0) : 0ull;
}

// Per-molecule leave of n <= SG_PM_MAX molecules with 0 < t1 <= 1: one uniform v per
// molecule; it leaves when v < t1 and then takes face f when v < t1 cum_f, cum_f the
// cumulative face probabilities of the conditional selectors (a selector of 1 sends all
// that remain to its face).  The joint law is the multinomial of Binomial(n, t1) and the
// conditional face binomials.
__device__ __forceinline__ uint4 leave_molecules(sg_stream* st, uint32_t n, double t1, double c0, double c1,
                                                 double c2, uint32_t* out_kn) {
    const double r0 = 1.0 - c0;
    const double cum0 = c0;
    const double cum1 = cum0 + c1 * r0;
    const double cum2 = cum1 + c2 * (r0 * (1.0 - c1));
    const uint64_t T3 = sg_thr(t1);
    uint64_t T2 = (c2 >= 1.0) ? T3 : sg_thr(t1 * cum2);
    uint64_t T1 = (c1 >= 1.0) ? T3 : sg_thr(t1 * cum1);
    uint64_t T0 = (c0 >= 1.0) ? T3 : sg_thr(t1 * cum0);
    if (c1 >= 1.0) T2 = T3;
    if (c0 >= 1.0) T1 = T2 = T3;
    T2 = T2 < T3 ? T2 : T3;
    T1 = T1 < T2 ? T1 : T2;
    T0 = T0 < T1 ? T0 : T1;
    uint32_t a0 = 0u, a1 = 0u, a2 = 0u, a3 = 0u;
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t v = sg_next_u32(st);
        a0 += v < T0 ? 1u : 0u;
        a1 += v < T1 ? 1u : 0u;
        a2 += v < T2 ? 1u : 0u;
        a3 += v < T3 ? 1u : 0u;
    }
    *out_kn = a3;
    return make_uint4(a0, a1 - a0, a2 - a1, a3 - a2);
}

// Binomial(mean_n, t1) molecules leave, split over the directions by conditional
// binomials on the selectors g.x, g.y, g.z; the last direction takes the rest.  Up to
// SG_PM_MAX molecules, molecule by molecule (leave_molecules).
__device__ __forceinline__ uint4 leave_split(sg_stream* st, uint32_t mean_n, double t1, double c0, double c1,
                                             double c2, double odd1, double odd2, double odd3, const double* rcp,
                                             const double* rcpl, const double* lnf, uint32_t* out_kn) {
    if (mean_n <= SG_PM_MAX) {
        if (mean_n == 0u || !(t1 > 0.0)) {
            *out_kn = 0u;
            return make_uint4(0u, 0u, 0u, 0u);
        }
        return leave_molecules(st, mean_n, t1 < 1.0 ? t1 : 1.0, c0, c1, c2, out_kn);
    }
    // Stage 0: molecules leaving; stages 1-3: the split.  One sampler call site.
    uint4 k = make_uint4(0u, 0u, 0u, 0u);
    uint32_t n = mean_n, Kn = 0u;
    double pst = t1;
    double ost = (t1 > 0.0 && t1 < 1.0) ? sg_binom_odds(t1) : 0.0;
#pragma unroll 1
    for (int stage = 0; stage < 4; ++stage) {
        uint32_t v = sg_binom_o(st, n, pst, ost, rcp, rcpl, lnf);
        if (stage == 0) {
            Kn = v;
            n = v;
            pst = c0;
            ost = odd1;
        } else if (stage == 1) {
            k.x = v;
            n -= v;
            pst = c1;
            ost = odd2;
        } else if (stage == 2) {
            k.y = v;
            n -= v;
            pst = c2;
            ost = odd3;
        } else {
            k.z = v;
            n -= v;
        }
    }
    k.w = n;
    *out_kn = Kn;
    return k;
}

// Leave of one (tet, species) with the face selectors and their odds read from this
// thread's slots in shared memory (selc[k * stride], k = c0, c1, c2, as float or double;
// selo[k * stride] their odds) instead of registers held across the species loop.
template <typename C>
__device__ __forceinline__ uint4 leave_split_sh(sg_stream* st, uint32_t mean_n, double t1, const C* selc,
                                                const double* selo, int stride, const double* rcp,
                                                const double* rcpl, const double* lnf, uint32_t* out_kn) {
    if (mean_n <= SG_PM_MAX) {
        if (mean_n == 0u || !(t1 > 0.0)) {
            *out_kn = 0u;
            return make_uint4(0u, 0u, 0u, 0u);
        }
        return leave_molecules(st, mean_n, t1 < 1.0 ? t1 : 1.0, (double)selc[0], (double)selc[stride],
                               (double)selc[2 * stride], out_kn);
    }
    uint4 k = make_uint4(0u, 0u, 0u, 0u);
    uint32_t n = mean_n, Kn = 0u;
    double pst = t1;
    double ost = (t1 > 0.0 && t1 < 1.0) ? sg_binom_odds(t1) : 0.0;
#pragma unroll 1
    for (int stage = 0; stage < 4; ++stage) {
        uint32_t v = sg_binom_o(st, n, pst, ost, rcp, rcpl, lnf);
        if (stage == 0) {
            Kn = v;
            n = v;
        } else if (stage == 1) {
            k.x = v;
            n -= v;
        } else if (stage == 2) {
            k.y = v;
            n -= v;
        } else {
            k.z = v;
            n -= v;
        }
        if (stage < 3) {
            pst = (double)selc[stage * stride];
            ost = selo[stage * stride];
        }
    }
    k.w = n;
    *out_kn = Kn;
    return k;
}

// Last block of a window: conservation check, counters, device-side time advance.
// flag is a 2-int shared scratch; parity is the launch parity read at kernel start.
__device__ __forceinline__ void window_last_block(const sg_window_args& a, int check, unsigned long long parity,
                                                  int* flag, int BLOCK) {
    const int S = a.nspec, R = a.nreac, tid = threadIdx.x, lane = tid & 31;
    const unsigned long long p = parity, q = parity ^ 1ull;
    int nact = 0;
    for (int i = tid; i < a.nreal; i += BLOCK) {
        const sg_real* rl = &a.reals[i];
        if (__ldcg(&rl->t) < __ldcg(&rl->t_end)) nact += 1;
    }
    for (int o = 16; o > 0; o >>= 1) nact += __shfl_down_sync(0xffffffffu, nact, o);
    if (lane == 0) atomicAdd(&flag[1], nact);
    __syncthreads();
    nact = flag[1];
    const bool do_check = check && __ldcg(&a.launch_state[3]) != 0ull &&
                          (unsigned long long)nact == __ldcg(&a.launch_state[2]);
    for (int s = tid; s < S && do_check; s += BLOCK) {
        long long expect = (long long)__ldcg(&a.totals[q * S + s]);
        for (int rr = 0; rr < R; ++rr) {
            const sg_reac* rc = &a.reacs[rr];
            for (int i = 0; i < rc->nupd; ++i)
                if (rc->upd_spec[i] == s)
                    expect += (long long)rc->upd_delta[i] * (long long)__ldcg(&a.ext[q * R + rr]);
        }
        if ((unsigned long long)expect != __ldcg(&a.totals[p * S + s]))
            atomicOr(a.status, SG_ERR_CONSERVATION);
    }
    __syncthreads();
    for (int rr = tid; rr < R; rr += BLOCK) {
        a.ext_total[rr] += __ldcg(&a.ext[p * R + rr]);
        a.ext[q * R + rr] = 0ull;
    }
    for (int s = tid; s < S; s += BLOCK) a.totals[q * S + s] = 0ull;
    if (a.work && tid < 4) a.work[q * 4 + tid] = 0u;
    for (int i = tid; i < a.nreal; i += BLOCK) {
        sg_real* rl = &a.reals[i];
        double rt = __ldcg(&rl->t), rend = __ldcg(&rl->t_end), per = __ldcg(&rl->period);
        if (rt < rend) {
            rl->t = (rt + per > rend) ? rend : rt + per;
            rl->window = __ldcg(&rl->window) + 1ull;
            rl->pending = 1;
        }
    }
    if (tid == 0) {
        a.launch_state[2] = (unsigned long long)nact;
        a.launch_state[3] = 1ull;
        a.launch_state[1] = p + 1ull;
        a.launch_state[0] = 0ull;
    }
}

// Count this block as finished; true in the last block of the launch (flag: 2 ints).
__device__ __forceinline__ bool window_block_done(const sg_window_args& a, int* flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long prev = atomicAdd(&a.launch_state[0], 1ull);
        flag[0] = (prev == (unsigned long long)(gridDim.x - 1)) ? 1 : 0;
        flag[1] = 0;
    }
    __syncthreads();
    if (!flag[0]) return false;
    __threadfence();
    return true;
}

// Resident threads per SM the window kernel is compiled for (caps registers per thread).
#ifndef SG_WINDOW_THREADS_PER_SM
#define SG_WINDOW_THREADS_PER_SM 1024
#endif

// Window kernel: gather (if pending) -> totals -> SSA -> diffusion leave -> store.
// SPLIT: reactions only (gather, SSA, counts and change-time sums to global memory); the
// diffusion leave and the end of the window run in leave_kernel.
template <int BLOCK, bool SURF = false, bool SPLIT = false>
__global__ void __launch_bounds__(BLOCK, SG_WINDOW_THREADS_PER_SM / BLOCK)
    window_kernel(sg_window_args a, int check) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_rcp[SG_RCP_TABLE];
    // Volume pass of a split window: per warp, up to 63 tets whose first draw may fall in
    // the window wait here and run their SSA 32 at a time (all lanes busy with events).
    __shared__ int s_q[(SPLIT && !SURF) ? 2 * BLOCK : 1];
    const int S = a.nspec;
    const int R = a.nreac;
    const int tid = threadIdx.x;
    smem_layout L = carve(smem_raw, BLOCK, S, R);
    surf_layout SLy;
    if (SURF)
        SLy = surf_carve(smem_raw + ((smem_bytes(BLOCK, S, R) + 15) & ~(size_t)15), BLOCK, a.surf.nsspec,
                         a.surf.max_sreac_per_patch);
    for (int i = tid; i < SG_RCP_TABLE; i += BLOCK) s_rcp[i] = (i == 0) ? 0.0 : 1.0 / (double)i;
    for (int i = tid; i < R; i += BLOCK) L.reac[i] = a.reacs[i];
    for (int i = tid; i < S; i += BLOCK) L.tot[i] = 0ull;
    for (int i = tid; i < R; i += BLOCK) L.ext[i] = 0u;
    if (tid == 0) L.moved[0] = 0ull;
    __syncthreads();

    const int lane = tid & 31;
    const unsigned long long parity = __ldcg(&a.launch_state[1]) & 1ull;
    const size_t plane = (size_t)a.ntets * 4;  // uint32 words per diffusing species
    unsigned long long moved = 0ull;
    // Split kernels take chunks of 32 tets per warp from the launch's work counter, so a
    // warp whose tets drew few events moves on instead of idling until its block ends.
    unsigned int* wctr = (SPLIT && a.work) ? a.work + parity * 4 + (SURF ? 1 : 0) : nullptr;

    int* wq = s_q + (SPLIT && !SURF ? (tid & ~31) * 2 : 0);  // this warp's queue
    int qn = 0;                                                 // its length (warp-uniform)

    // A tet list (split windows of membrane models) restricts the launch to those tets.
    const int nit = a.tet_list ? a.nlist : a.ntets;
    for (int it = 0;; ++it) {
        const int base = next_warp_base(wctr, it, BLOCK);
        if (base >= nit) {
            if (SPLIT && !SURF) {
                __syncwarp();
                if (lane < qn) tet_ssa_queued(a, L, tid, BLOCK, wq[lane]);
            }
            break;
        }
        bool active = base + lane < nit;
        const int t = !active ? 0 : (a.tet_list ? __ldg(&a.tet_list[base + lane]) : base + lane);
        int r = 0, comp = 0, tlocal = 0;
        double T = 0.0;
        unsigned long long w = 0;
        int pending = 0;
        if (active) {
            r = find_real(a.reals, a.nreal, t);
            const sg_real* rl = &a.reals[r];
            double rt = rl->t, rend = rl->t_end, per = rl->period;
            active = rt < rend;
            T = (rt + per > rend) ? rend - rt : per;
            w = rl->window;
            pending = rl->pending;
            tlocal = t - rl->tet_begin;
            if (a.comp) comp = __ldg(&a.comp[t]);
            if (comp < 0) active = false;
            if (SPLIT && !SURF && a.surf.tet_tris) {
                // Membrane tets run in the SURF launch over the membrane tet list.
                const int4 tr = __ldg(reinterpret_cast<const int4*>(a.surf.tet_tris) + t);
                if (tr.x >= 0 || tr.y >= 0 || tr.z >= 0 || tr.w >= 0) active = false;
            }
            // Tets of merged units run in unit_ssa_kernel.
            if (SPLIT && a.units.tet_unit && __ldg(&a.units.tet_unit[t]) >= 0) active = false;
        }
        int4 nb = make_int4(-1, -1, -1, -1);
        uint32_t clampm = 0u;
        const double* Dc = a.dcst;
        if (active) {
            nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
            if (a.clamp) clampm = __ldg(&a.clamp[t]);
            Dc = a.dcst + ((size_t)r * a.ncomp + comp) * S;
        }
        // Phase 1: gather last window's inflow, stage counts in shared memory.  The counts
        // and the inflow of the first GS diffusing species are copied in asynchronously, all
        // in flight at once, the inflow into this thread's change-time and propensity slots
        // (free until the SSA; two 8-byte halves per slot pair).
        const uint32_t* in = a.outflow + (size_t)((w + 1) & 1ull) * a.ndiff * plane;
        const int GS = (S + R) / 2 < a.ndiff ? (S + R) / 2 : a.ndiff;
        if (active) {
            for (int s = 0; s < S; ++s) sg_cp_async4(&L.cnt[s * BLOCK + tid], &a.counts[(size_t)s * a.ntets + t]);
            if (pending)
                for (int ds = 0; ds < GS; ++ds) {
                    const uint32_t* src = in + (size_t)ds * plane + (size_t)t * 4;
                    sg_cp_async8(&L.tdel[(2 * ds) * BLOCK + tid], src);
                    sg_cp_async8(&L.tdel[(2 * ds + 1) * BLOCK + tid], src + 2);
                }
            sg_cp_async_wait();
        }
        for (int s = 0; s < S; ++s) {
            uint32_t c = 0u;
            if (active) {
                c = L.cnt[s * BLOCK + tid];
                int ds = __ldg(&a.diff_slot[s]);
                if (pending && ds >= 0 && __ldg(&Dc[s]) > 0.0 && !((clampm >> s) & 1u)) {
                    // Slot f of this tet holds what the neighbour behind face f sent.
                    uint4 v;
                    if (ds < GS) {
                        const uint2 lo = *reinterpret_cast<const uint2*>(&L.tdel[(2 * ds) * BLOCK + tid]);
                        const uint2 hi = *reinterpret_cast<const uint2*>(&L.tdel[(2 * ds + 1) * BLOCK + tid]);
                        v = make_uint4(lo.x, lo.y, hi.x, hi.y);
                    } else {
                        v = __ldg(reinterpret_cast<const uint4*>(in + (size_t)ds * plane) + t);
                    }
                    unsigned long long sum = c;
                    if (nb.x >= 0) sum += v.x;
                    if (nb.y >= 0) sum += v.y;
                    if (nb.z >= 0) sum += v.z;
                    if (nb.w >= 0) sum += v.w;
                    if (a.bface) sum += bnd_inflow(a, t, r, s, v);
                    if (sum > 0xFFFFFFFFull) {
                        atomicOr(a.status, SG_ERR_OVERFLOW);
                        sum = 0xFFFFFFFFull;
                    }
                    c = (uint32_t)sum;
                }
            }
            L.cnt[s * BLOCK + tid] = c;
            const unsigned long long v = warp_total_u32(c);
            if (lane == 0 && v) atomicAdd(&L.tot[s], v);
        }
        if (active)
            for (int s = 0; s < S; ++s) L.tdel[s * BLOCK + tid] = 0.0;
        if (SPLIT && !SURF) {
            // First draw only; tets that may see an event join the warp's queue.
            bool fire = false;
            if (active) {
                const int rb = __ldg(&a.comp_reac_begin[comp]);
                const int re = __ldg(&a.comp_reac_begin[comp + 1]);
                if (re > rb) {
                    sg_stream st;
                    sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)tlocal, w, SG_PURPOSE_WINDOW);
                    fire = tet_may_fire(L, tid, BLOCK, rb, re, a.kcst + (size_t)r * R, __ldg(&a.ivs[t]), T, &st);
                }
                for (int s = 0; s < S; ++s) a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
                if (!fire && a.tmask) a.tmask[t] = 0u;  // no change-time sums
            }
            const unsigned bal = __ballot_sync(0xffffffffu, fire);
            if (fire) wq[qn + __popc(bal & ((1u << lane) - 1u))] = t;
            qn += __popc(bal);
            if (qn >= 32) {
                __syncwarp();
                tet_ssa_queued(a, L, tid, BLOCK, wq[qn - 32 + lane]);
                qn -= 32;
                __syncwarp();
            }
            continue;
        }
        if (!active) continue;

        sg_stream st;
        sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)tlocal, w, SG_PURPOSE_WINDOW);
        const double ivs = __ldg(&a.ivs[t]);
        const double* K = a.kcst + (size_t)r * R;
        const int rb = __ldg(&a.comp_reac_begin[comp]);
        const int re = __ldg(&a.comp_reac_begin[comp + 1]);

        // Phase 2: reaction SSA over the window (with the tet's membrane triangles, if any).
        if (SURF) {
            const int4 tr = __ldg(reinterpret_cast<const int4*>(a.surf.tet_tris) + t);
            if ((tr.x & tr.y & tr.z & tr.w) >= 0 || tr.x >= 0 || tr.y >= 0 || tr.z >= 0 || tr.w >= 0)
                tet_ssa_surf(a, L, SLy, tid, BLOCK, rb, re, K, ivs, clampm, T, &st, tr, w, pending);
            else if (re > rb)
                tet_ssa(a, L, tid, BLOCK, rb, re, K, ivs, clampm, T, &st);
        } else if (re > rb) {
            tet_ssa(a, L, tid, BLOCK, rb, re, K, ivs, clampm, T, &st);
        }

        if (SPLIT) {
            // Counts, and the change-time sums of the diffusing species that changed (their
            // bits in tmask; the leave reads the others as zero).
            uint32_t tm = 0u;
            for (int s = 0; s < S; ++s) {
                const int ds = __ldg(&a.diff_slot[s]);
                const double sdv = L.tdel[s * BLOCK + tid];
                if (ds >= 0 && sdv != 0.0) {
                    a.tdel[(size_t)ds * a.ntets + t] = sdv;
                    tm |= 1u << s;
                }
                a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
            }
            if (a.tmask) a.tmask[t] = tm;
            continue;
        }
        // Phase 3: diffusion leave, one (tet, species) at a time.
        const float4 g = __ldg(reinterpret_cast<const float4*>(a.geo) + t);
        const bool bt = a.bface && __ldg(&a.bface[t]) != 0xFFFFFFFFu;
        // The face selectors and their odds, once per tet.
        const double cs[3] = {(double)g.x, (double)g.y, (double)g.z};
        const double odd1 = sg_binom_odds(cs[0]);
        const double odd2 = sg_binom_odds(cs[1]);
        const double odd3 = sg_binom_odds(cs[2]);
        uint32_t* out = a.outflow + (size_t)(w & 1ull) * a.ndiff * plane;
        const double invT = 1.0 / T;  // one division per tet for the occupancy means
        for (int s = 0; s < S; ++s) {
            int ds = __ldg(&a.diff_slot[s]);
            if (ds < 0) continue;
            double D = __ldg(&Dc[s]);
            if (!(D > 0.0)) continue;
            uint32_t pop = L.cnt[s * BLOCK + tid];
            uint4 k = make_uint4(0u, 0u, 0u, 0u);
            if (pop > 0u) {
                uint32_t Kn = 0u;
                if (bt) {
                    // Diffusion-boundary tet: face rates, and so selectors, per species.
                    float4 gb;
                    const double tot = bnd_split(a, t, comp, s, D, nb, &gb);
                    const double cb[3] = {(double)gb.x, (double)gb.y, (double)gb.z};
                    k = leave_species(a.seed, (uint32_t)r, (uint32_t)tlocal, w, (uint32_t)s, pop, L.tdel[s * BLOCK + tid],
                                      invT, T * tot, cb, sg_binom_odds(cb[0]), sg_binom_odds(cb[1]),
                                      sg_binom_odds(cb[2]), s_rcp, nullptr, nullptr, &st, &Kn);
                } else {
                    k = leave_species(a.seed, (uint32_t)r, (uint32_t)tlocal, w, (uint32_t)s, pop, L.tdel[s * BLOCK + tid],
                                      invT, T * (D * (double)g.w), cs, odd1, odd2, odd3, s_rcp, nullptr, nullptr,
                                      &st, &Kn);
                }
                if (Kn > 0u) {
                    if (!((clampm >> s) & 1u)) L.cnt[s * BLOCK + tid] = pop - Kn;
                    moved += Kn;
                }
            }
            // Scatter into the receiving tets' slots: nb.f = (neighbour << 2) | its face, i.e.
            // the word index inside this species' plane.  Each slot has one writer.
            uint32_t* po = out + (size_t)ds * plane;
            if (nb.x >= 0) po[nb.x] = k.x;
            if (nb.y >= 0) po[nb.y] = k.y;
            if (nb.z >= 0) po[nb.z] = k.z;
            if (nb.w >= 0) po[nb.w] = k.w;
            if (bt) bnd_scatter(a, t, po, k);
        }
        // Phase 4: store counts.
        for (int s = 0; s < S; ++s) a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
    }

    // Block partials -> global accumulators of this launch parity.
    moved = warp_sum_u64(moved);
    if (lane == 0 && moved) atomicAdd(L.moved, moved);
    __syncthreads();
    for (int i = tid; i < S; i += BLOCK)
        if (L.tot[i]) atomicAdd(&a.totals[parity * S + i], L.tot[i]);
    for (int i = tid; i < R; i += BLOCK)
        if (L.ext[i]) atomicAdd(&a.ext[parity * R + i], (unsigned long long)L.ext[i]);
    if (tid == 0 && L.moved[0]) atomicAdd(a.diff_total, L.moved[0]);
    if (SPLIT) return;  // leave_kernel ends the window
    if (!window_block_done(a, L.flag)) return;
    window_last_block(a, check, parity, L.flag, BLOCK);
}

// Resident threads per SM the leave kernel is compiled for (caps registers per thread).
#ifndef SG_LEAVE_THREADS_PER_SM
#define SG_LEAVE_THREADS_PER_SM 1024
#endif

// Split window, second kernel: the diffusion leave.  One thread per tet loops over the
// diffusing species, so the tet's tables (neighbours, face selectors and their odds, the
// window length, realization, compartment, clamps) are read and derived once; warps take
// chunks of 32 tets from the launch's work counter, so no warp waits on slower ones until
// the work runs out.  Then the end of the window (last block).  Each (tet, species) draws
// from its own stream, so the results equal the fused kernel's bit for bit.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, SG_LEAVE_THREADS_PER_SM / BLOCK) leave_kernel(sg_window_args a, int check) {
    __shared__ double s_rcp[SG_RCP_TABLE];
    // Per-thread slots for what the species loop reads after each sampler call: the face
    // selectors c0, c1, c2 (floats, as in the geometry) and their odds, the window length
    // and its inverse.  Held in registers across the loop they forced spills at the
    // 64-register cap.  The mode search's tables (a.mode_rcpl, a.mode_lnf) and the
    // remaining spills are served by L1: the block's shared memory is kept small (about
    // 14 KB) so that the host can give L1 most of the SM's 256 KB (set_leave_carveout).
    __shared__ float s_selc[3 * BLOCK];
    __shared__ double s_selo[3 * BLOCK];
    __shared__ double s_T[2 * BLOCK];
    __shared__ int flag[2];
    __shared__ unsigned long long s_moved;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < SG_RCP_TABLE; i += BLOCK) s_rcp[i] = (i == 0) ? 0.0 : 1.0 / (double)i;
    if (tid == 0) s_moved = 0ull;
    __syncthreads();
    const unsigned long long parity = __ldcg(&a.launch_state[1]) & 1ull;
    unsigned int* wctr = a.work ? a.work + parity * 4 + 2 : nullptr;
    const size_t plane = (size_t)a.ntets * 4;
    const int S = a.nspec;
    float* selc = s_selc + tid;
    double* selo = s_selo + tid;
    unsigned long long moved = 0ull;
    for (int it = 0;; ++it) {
        const int base = next_warp_base(wctr, it, BLOCK);
        if (base >= a.ntets) break;
        const int t = base + lane;
        if (t >= a.ntets) continue;
        const int r = find_real(a.reals, a.nreal, t);
        const sg_real* rl = &a.reals[r];
        const double rt = rl->t, rend = rl->t_end, per = rl->period;
        if (!(rt < rend)) continue;
        const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
        if (comp < 0) continue;
        const double Tw = (rt + per > rend) ? rend - rt : per;
        const uint32_t tl = (uint32_t)(t - rl->tet_begin);
        const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
        const bool bt = a.bface && __ldg(&a.bface[t]) != 0xFFFFFFFFu;
        const double* Dc = a.dcst + ((size_t)r * a.ncomp + comp) * S;
        const float G = __ldg(reinterpret_cast<const float*>(a.geo) + (size_t)t * 4 + 3);
        if (!bt) {
            const float4 g = __ldg(reinterpret_cast<const float4*>(a.geo) + t);
            selc[0] = g.x;
            selc[BLOCK] = g.y;
            selc[2 * BLOCK] = g.z;
            selo[0] = sg_binom_odds((double)g.x);
            selo[BLOCK] = sg_binom_odds((double)g.y);
            selo[2 * BLOCK] = sg_binom_odds((double)g.z);
        }
        s_T[tid] = Tw;
        s_T[BLOCK + tid] = 1.0 / Tw;  // one division per tet for the occupancy means
        const uint32_t tm = a.tmask ? a.tmask[t] : 0u;
        for (int s = 0; s < S; ++s) {
            const double T = s_T[tid], invT = s_T[BLOCK + tid];
            const unsigned long long w = a.reals[r].window;
            const int ds = __ldg(&a.diff_slot[s]);
            if (ds < 0) continue;
            const double D = __ldg(&Dc[s]);
            if (!(D > 0.0)) continue;
            const size_t ci = (size_t)s * a.ntets + t;
            const uint32_t pop = a.counts[ci];
            uint4 k = make_uint4(0u, 0u, 0u, 0u);
            if (pop > 0u) {
                sg_stream st;
                uint32_t Kn = 0u;
                const double sd = ((tm >> s) & 1u) ? a.tdel[(size_t)ds * a.ntets + t] : 0.0;
                double t1;
                if (bt) {
                    const int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
                    float4 gb;
                    const double tot = bnd_split(a, t, comp, s, D, nb, &gb);
                    selc[0] = gb.x;
                    selc[BLOCK] = gb.y;
                    selc[2 * BLOCK] = gb.z;
                    selo[0] = sg_binom_odds((double)gb.x);
                    selo[BLOCK] = sg_binom_odds((double)gb.y);
                    selo[2 * BLOCK] = sg_binom_odds((double)gb.z);
                    t1 = T * tot;
                } else {
                    t1 = T * (D * (double)G);
                }
                sg_stream_init(&st, a.seed, (uint32_t)r, tl, w, SG_PURPOSE_DIFF + (uint32_t)s);
                if (t1 >= 1.0) t1 = 1.0;
                uint32_t mean_n = pop;
                if (sd != 0.0) {
                    double nbar = (double)pop - sd * invT;
                    if (nbar > (double)pop) nbar = (double)pop;
                    double nint = floor(nbar);
                    double frc = nbar - nint;
                    mean_n = (uint32_t)nint;
                    if (frc > 0.0) {
                        if (sg_u01_co(sg_next_u32(&st)) < frc) mean_n += 1u;
                    }
                }
                k = leave_split_sh(&st, mean_n, t1, selc, selo, BLOCK, s_rcp, a.mode_rcpl, a.mode_lnf, &Kn);
                if (Kn > 0u) {
                    if (!((clampm >> s) & 1u)) a.counts[ci] = pop - Kn;
                    moved += Kn;
                }
            }
            const int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
            uint32_t* po = a.outflow + (size_t)(w & 1ull) * a.ndiff * plane + (size_t)ds * plane;
            if (nb.x >= 0) po[nb.x] = k.x;
            if (nb.y >= 0) po[nb.y] = k.y;
            if (nb.z >= 0) po[nb.z] = k.z;
            if (nb.w >= 0) po[nb.w] = k.w;
            if (bt) bnd_scatter(a, t, po, k);
        }
    }
    moved = warp_sum_u64(moved);
    if (lane == 0 && moved) atomicAdd(&s_moved, moved);
    __syncthreads();
    if (tid == 0 && s_moved) atomicAdd(a.diff_total, s_moved);
    if (!window_block_done(a, flag)) return;
    window_last_block(a, check, parity, flag, BLOCK);
}

// Surface diffusion leave (TOS:1716-1793, sdiff.cpp:498-560), one thread per (surface-
// diffusing species, membrane triangle), between the SSA and leave_kernel of a split
// window: n = min(pop, window integral / T) with a Bernoulli on its fraction,
// Binomial(n, min(1, T D G)) leaving, conditional binomials over the three edges.  Each
// (triangle, species) draws from its own stream (purpose SG_PURPOSE_SDIFF + species).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) sdiffuse_kernel(sg_window_args a) {
    __shared__ double s_rcp[SG_RCP_TABLE];
    __shared__ unsigned long long s_moved;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < SG_RCP_TABLE; i += BLOCK) s_rcp[i] = (i == 0) ? 0.0 : 1.0 / (double)i;
    if (tid == 0) s_moved = 0ull;
    __syncthreads();
    const sg_surf_args& sa = a.surf;
    const int M = sa.ntris, SS = sa.nsspec;
    const long long total = (long long)sa.nsdiff * M;
    unsigned long long moved = 0ull;
    for (long long idx = (long long)blockIdx.x * BLOCK + tid; idx < total; idx += (long long)gridDim.x * BLOCK) {
        const int sd = (int)(idx / M);
        const int m = (int)(idx - (long long)sd * M);
        const int r = find_real(a.reals, a.nreal, __ldg(&sa.tri_inner[m]));
        const sg_real* rl = &a.reals[r];
        const double rt = rl->t, rend = rl->t_end, per = rl->period;
        if (!(rt < rend)) continue;
        const int s = __ldg(&sa.sdiff_spec[sd]);
        const double D = __ldg(&sa.sdcst[(size_t)__ldg(&sa.tri_patch[m]) * SS + s]);
        if (!(D > 0.0)) continue;
        const double T = (rt + per > rend) ? rend - rt : per;
        const unsigned long long w = rl->window;
        const size_t ci = (size_t)s * M + m;
        const uint32_t pop = sa.tri_counts[ci];
        uint4 k = make_uint4(0u, 0u, 0u, 0u);
        if (pop > 0u) {
            const float4 g = __ldg(reinterpret_cast<const float4*>(sa.sgeo) + m);
            double t1 = T * (D * (double)g.w);
            if (t1 >= 1.0) t1 = 1.0;
            double nd = sa.tri_occ[(size_t)sd * M + m] / T;
            if (nd > (double)pop) nd = (double)pop;
            const double nint = floor(nd);
            const double frc = nd - nint;
            uint32_t mean_n = (uint32_t)nint;
            sg_stream st;
            sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)m, w, SG_PURPOSE_SDIFF + (uint32_t)s);
            if (frc > 0.0) {
                if (sg_u01_co(sg_next_u32(&st)) < frc) mean_n += 1u;
            }
            uint32_t Kn = 0u;
            k = leave_split(&st, mean_n, t1, (double)g.x, (double)g.y, (double)g.z, sg_binom_odds((double)g.x),
                            sg_binom_odds((double)g.y), 0.0, s_rcp,
                            nullptr, nullptr, &Kn);
            if (Kn > 0u) {
                sa.tri_counts[ci] = pop - Kn;
                moved += Kn;
            }
        }
        const int4 nb = __ldg(reinterpret_cast<const int4*>(sa.snbr) + m);
        uint32_t* po = sa.tri_outflow + (size_t)(w & 1ull) * sa.nsdiff * M * 4 + (size_t)sd * M * 4;
        if (nb.x >= 0) po[nb.x] = k.x;
        if (nb.y >= 0) po[nb.y] = k.y;
        if (nb.z >= 0) po[nb.z] = k.z;
    }
    moved = warp_sum_u64(moved);
    if (lane == 0 && moved) atomicAdd(&s_moved, moved);
    __syncthreads();
    if (tid == 0 && s_moved) atomicAdd(a.diff_total, s_moved);
}

// ---- batched realizations in one persistent launch ----------------------------------

// The mode search's tables in global memory: 1/x and ln x! for x < SG_MODE_TABLE, computed
// by the same functions as the leave kernel's shared copies.
static __global__ void mode_tables_kernel(double* rcpl, double* lnf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < SG_MODE_TABLE; i += gridDim.x * blockDim.x) {
        rcpl[i] = (i == 0) ? 0.0 : 1.0 / (double)i;
        lnf[i] = sg_lnfact((uint32_t)i);
    }
}

__device__ __forceinline__ unsigned int sg_ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void sg_st_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The diffusion leave of tet t (the split window's leave kernel for one tet): its counts
// and change-time sums into this thread's shared-memory column, the leave, the scatter of
// its outflow, then its counts to global memory.  The face selectors and their odds sit in this
// thread's slots sel[k * BLOCK] (k = c0, c1, c2, odd1, odd2, odd3: its propensity column,
// free once its SSA is done) for the species loop.
__device__ __forceinline__ void leave_and_store(const sg_window_args& a, const smem_layout& L, int tid, int BLOCK,
                                                int t, int r, int tlocal, int comp, double T, unsigned long long w,
                                                const double* s_rcp, unsigned long long* moved) {
    const int S = a.nspec;
    // The counts and change-time sums the first pass or the queued SSA wrote (this warp).
    const uint32_t tm = a.tmask ? __ldcg(&a.tmask[t]) : 0u;
    for (int s = 0; s < S; ++s) {
        L.cnt[s * BLOCK + tid] = __ldcg(&a.counts[(size_t)s * a.ntets + t]);
        const int ds = __ldg(&a.diff_slot[s]);
        L.tdel[s * BLOCK + tid] = (ds >= 0 && ((tm >> s) & 1u)) ? __ldcg(&a.tdel[(size_t)ds * a.ntets + t]) : 0.0;
    }
    const size_t plane = (size_t)a.ntets * 4;
    double* sel = L.prop + tid;
    const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
    const double* Dc = a.dcst + ((size_t)r * a.ncomp + comp) * S;
    const float G = __ldg(reinterpret_cast<const float*>(a.geo) + (size_t)t * 4 + 3);
    const bool bt = a.bface && __ldg(&a.bface[t]) != 0xFFFFFFFFu;
    if (!bt) {
        const float4 g = __ldg(reinterpret_cast<const float4*>(a.geo) + t);
        sel[0] = (double)g.x;
        sel[BLOCK] = (double)g.y;
        sel[2 * BLOCK] = (double)g.z;
        sel[3 * BLOCK] = sg_binom_odds((double)g.x);
        sel[4 * BLOCK] = sg_binom_odds((double)g.y);
        sel[5 * BLOCK] = sg_binom_odds((double)g.z);
    }
    const double invT = 1.0 / T;
    for (int s = 0; s < S; ++s) {
        const int ds = __ldg(&a.diff_slot[s]);
        if (ds < 0) continue;
        const double D = __ldg(&Dc[s]);
        if (!(D > 0.0)) continue;
        const uint32_t pop = L.cnt[s * BLOCK + tid];
        uint4 k = make_uint4(0u, 0u, 0u, 0u);
        if (pop > 0u) {
            sg_stream st;
            uint32_t Kn = 0u;
            double t1;
            if (bt) {
                const int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
                float4 gb;
                const double tot = bnd_split(a, t, comp, s, D, nb, &gb);
                sel[0] = (double)gb.x;
                sel[BLOCK] = (double)gb.y;
                sel[2 * BLOCK] = (double)gb.z;
                sel[3 * BLOCK] = sg_binom_odds((double)gb.x);
                sel[4 * BLOCK] = sg_binom_odds((double)gb.y);
                sel[5 * BLOCK] = sg_binom_odds((double)gb.z);
                t1 = T * tot;
            } else {
                t1 = T * (D * (double)G);
            }
            sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)tlocal, w, SG_PURPOSE_DIFF + (uint32_t)s);
            if (t1 >= 1.0) t1 = 1.0;
            uint32_t mean_n = pop;
            const double sd = L.tdel[s * BLOCK + tid];
            if (sd != 0.0) {
                double nbar = (double)pop - sd * invT;
                if (nbar > (double)pop) nbar = (double)pop;
                const double nint = floor(nbar);
                const double frc = nbar - nint;
                mean_n = (uint32_t)nint;
                if (frc > 0.0) {
                    if (sg_u01_co(sg_next_u32(&st)) < frc) mean_n += 1u;
                }
            }
            k = leave_split_sh(&st, mean_n, t1, sel, sel + 3 * BLOCK, BLOCK, s_rcp, a.mode_rcpl, a.mode_lnf, &Kn);
            if (Kn > 0u) {
                if (!((clampm >> s) & 1u)) L.cnt[s * BLOCK + tid] = pop - Kn;
                *moved += Kn;
            }
        }
        const int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
        uint32_t* po = a.outflow + (size_t)(w & 1ull) * a.ndiff * plane + (size_t)ds * plane;
        if (nb.x >= 0) po[nb.x] = k.x;
        if (nb.y >= 0) po[nb.y] = k.y;
        if (nb.z >= 0) po[nb.z] = k.z;
        if (nb.w >= 0) po[nb.w] = k.w;
        if (bt) bnd_scatter(a, t, po, k);
    }
    for (int s = 0; s < S; ++s) a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
}

// First pass of tet t inside a persistent launch, as the split window's SSA kernel: its
// inflow gathered (counts and inflow read through L2: other SMs wrote them earlier in the
// same launch), its counts stored, its first waiting time drawn.  True when that draw may
// fall in the window (the tet then waits for coherent_queued); false when its SSA is
// complete (no change-time sums).
__device__ __forceinline__ bool coherent_first_pass(const sg_window_args& a, const smem_layout& L, int tid, int BLOCK,
                                                    int t, int r, int tlocal, double T, unsigned long long w,
                                                    int pending, const double* s_rcp, unsigned long long* moved) {
    const int S = a.nspec, R = a.nreac;
    const size_t plane = (size_t)a.ntets * 4;
    const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
    if (comp < 0) return false;
    const int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
    const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
    const double* Dc = a.dcst + ((size_t)r * a.ncomp + comp) * S;
    const uint32_t* in = a.outflow + (size_t)((w + 1) & 1ull) * a.ndiff * plane;
    for (int s = 0; s < S; ++s) {
        uint32_t c = __ldcg(&a.counts[(size_t)s * a.ntets + t]);
        const int ds = __ldg(&a.diff_slot[s]);
        if (pending && ds >= 0 && __ldg(&Dc[s]) > 0.0 && !((clampm >> s) & 1u)) {
            const uint4 v = __ldcg(reinterpret_cast<const uint4*>(in + (size_t)ds * plane) + t);
            unsigned long long sum = c;
            if (nb.x >= 0) sum += v.x;
            if (nb.y >= 0) sum += v.y;
            if (nb.z >= 0) sum += v.z;
            if (nb.w >= 0) sum += v.w;
            if (a.bface) sum += bnd_inflow(a, t, r, s, v);
            if (sum > 0xFFFFFFFFull) {
                atomicOr(a.status, SG_ERR_OVERFLOW);
                sum = 0xFFFFFFFFull;
            }
            c = (uint32_t)sum;
        }
        L.tdel[s * BLOCK + tid] = 0.0;
        L.cnt[s * BLOCK + tid] = c;
    }
    const int rb = __ldg(&a.comp_reac_begin[comp]);
    const int re = __ldg(&a.comp_reac_begin[comp + 1]);
    bool fire = false;
    if (re > rb) {
        sg_stream st;
        sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)tlocal, w, SG_PURPOSE_WINDOW);
        fire = tet_may_fire(L, tid, BLOCK, rb, re, a.kcst + (size_t)r * R, __ldg(&a.ivs[t]), T, &st);
    }
    for (int s = 0; s < S; ++s) a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
    if (!fire && a.tmask) a.tmask[t] = 0u;  // no change-time sums
    return fire;
}

// A queued tet of a persistent launch: its gathered counts back from global memory (this
// warp wrote them), its whole SSA on its restarted stream (the draws of the first pass
// again), then its counts, its nonzero change-time sums and tmask to global memory.
__device__ __forceinline__ void coherent_queued(const sg_window_args& a, const smem_layout& L, int tid, int BLOCK,
                                                int t, int r, int tlocal, double T, unsigned long long w,
                                                const double* s_rcp, unsigned long long* moved) {
    const int S = a.nspec, R = a.nreac;
    const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
    const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
    for (int s = 0; s < S; ++s) {
        L.cnt[s * BLOCK + tid] = __ldcg(&a.counts[(size_t)s * a.ntets + t]);
        L.tdel[s * BLOCK + tid] = 0.0;
    }
    sg_stream st;
    sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)tlocal, w, SG_PURPOSE_WINDOW);
    tet_ssa(a, L, tid, BLOCK, __ldg(&a.comp_reac_begin[comp]), __ldg(&a.comp_reac_begin[comp + 1]),
            a.kcst + (size_t)r * R, __ldg(&a.ivs[t]), clampm, T, &st);
    uint32_t tm = 0u;
    for (int s = 0; s < S; ++s) {
        const int ds = __ldg(&a.diff_slot[s]);
        const double sdv = L.tdel[s * BLOCK + tid];
        if (ds >= 0 && sdv != 0.0) {
            a.tdel[(size_t)ds * a.ntets + t] = sdv;
            tm |= 1u << s;
        }
        a.counts[(size_t)s * a.ntets + t] = L.cnt[s * BLOCK + tid];
    }
    if (a.tmask) a.tmask[t] = tm;
}

// P.nwin windows of every batched realization in one launch (all blocks resident: a
// cooperative launch).  Items are taken in window-major order, so every item a warp waits
// for was taken earlier by a resident warp that itself only waits on earlier items: the
// waits end.  Each wait is still bounded (P.spin_limit polls); a wait that runs out sets
// SG_ERR_WAIT and the abort word, and every warp then stops at its next wait or item.
// Reaction extents go straight to the run totals; the per-window conservation check of
// the window launches is replaced by the host's check over the whole run() call.
template <int BLOCK, int TPL>
__global__ void __launch_bounds__(BLOCK, SG_WINDOW_THREADS_PER_SM / BLOCK)
    persistent_window_kernel(sg_window_args a, sg_persist_args P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_rcp[SG_RCP_TABLE];
    __shared__ int s_q[2 * BLOCK];  // per warp: up to 63 queued tets
    const int S = a.nspec, R = a.nreac, tid = threadIdx.x, lane = tid & 31;
    // At least six propensity slots per thread: the leave keeps the selectors there.
    smem_layout L = carve(smem_raw, BLOCK, S, R > 6 ? R : 6);
    for (int i = tid; i < SG_RCP_TABLE; i += BLOCK) s_rcp[i] = (i == 0) ? 0.0 : 1.0 / (double)i;
    for (int i = tid; i < R; i += BLOCK) L.reac[i] = a.reacs[i];
    for (int i = tid; i < R; i += BLOCK) L.ext[i] = 0u;
    if (tid == 0) L.moved[0] = 0ull;
    __syncthreads();
    int* wq = s_q + (tid & ~31) * 2;
    int qn = 0;
    unsigned long long moved = 0ull;
    const unsigned long long nitems = (unsigned long long)P.nwin * (unsigned long long)P.nchunks;
    for (;;) {
        unsigned long long item = 0ull;
        if (lane == 0) item = atomicAdd(P.next, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= nitems) break;
        const int wrel = (int)(item / (unsigned long long)P.nchunks);
        const int j = (int)(item - (unsigned long long)wrel * (unsigned long long)P.nchunks);
        int lo = 0, hi = a.nreal - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(&P.chunk_begin[mid]) <= j) lo = mid;
            else hi = mid - 1;
        }
        const int r = lo;
        const int c0 = __ldg(&P.chunk_begin[r]);
        const unsigned int nch = (unsigned int)(__ldg(&P.chunk_begin[r + 1]) - c0);
        int ok = 1;
        if (lane == 0) {
            unsigned int polls = 0u;
            while (sg_ld_acquire(&P.ready[r]) < (unsigned int)wrel) {
                if (__ldcg(P.abort) != 0u || ++polls > P.spin_limit) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
            if (lane == 0) {
                atomicOr(P.abort, 1u);
                atomicOr(a.status, SG_ERR_WAIT);
            }
            break;
        }
        (void)sg_ld_acquire(&P.ready[r]);  // every lane reads the previous window's writes after this
        const sg_real* rl = &a.reals[r];
        const double rt = __ldcg(&rl->t), rend = __ldcg(&rl->t_end), per = __ldcg(&rl->period);
        const unsigned long long w = __ldcg(&rl->window);
        const int pending = __ldcg(&rl->pending);
        const int tb = __ldg(&rl->tet_begin), te = __ldg(&rl->tet_end);
        const bool live = rt < rend;
        const double T = (rt + per > rend) ? rend - rt : per;
        // The split window inside the chunk: first passes of its tets 32 at a time, tets
        // whose first draw may fall in the window waiting in the warp's queue and running
        // their SSA 32 at a time (all lanes busy); then the leave of every tet of the chunk.
#pragma unroll 1
        for (int k = 0; k < TPL; ++k) {
            const int t = tb + (j - c0) * 32 * TPL + k * 32 + lane;
            bool fire = false;
            if (live && t < te) fire = coherent_first_pass(a, L, tid, BLOCK, t, r, t - tb, T, w, pending, s_rcp, &moved);
            const unsigned bal = __ballot_sync(0xffffffffu, fire);
            if (fire) wq[qn + __popc(bal & ((1u << lane) - 1u))] = t;
            qn += __popc(bal);
            if (qn >= 32) {
                __syncwarp();
                const int tq = wq[qn - 32 + lane];
                coherent_queued(a, L, tid, BLOCK, tq, r, tq - tb, T, w, s_rcp, &moved);
                qn -= 32;
                __syncwarp();
            }
        }
        __syncwarp();
        if (lane < qn) {
            const int tq = wq[lane];
            coherent_queued(a, L, tid, BLOCK, tq, r, tq - tb, T, w, s_rcp, &moved);
        }
        qn = 0;
        __syncwarp();
        // The diffusion leave of the chunk's tets, all lanes at once.
#pragma unroll 1
        for (int k = 0; k < TPL; ++k) {
            const int t = tb + (j - c0) * 32 * TPL + k * 32 + lane;
            if (live && t < te) {
                const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
                if (comp >= 0) leave_and_store(a, L, tid, BLOCK, t, r, t - tb, comp, T, w, s_rcp, &moved);
            }
        }
        __syncwarp();
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            const unsigned int prev = atomicAdd(&P.done[r], 1u);
            if (prev + 1u == (unsigned int)(wrel + 1) * nch) {
                // Last chunk of this realization's window: advance it (as window_last_block)
                // and publish the window.
                sg_real* rw = &a.reals[r];
                if (live) {
                    rw->t = (rt + per > rend) ? rend : rt + per;
                    rw->window = w + 1ull;
                    rw->pending = 1;
                }
                __threadfence();
                sg_st_release(&P.ready[r], (unsigned int)(wrel + 1));
            }
        }
    }
    moved = warp_sum_u64(moved);
    if (lane == 0 && moved) atomicAdd(L.moved, moved);
    __syncthreads();
    for (int i = tid; i < R; i += BLOCK)
        if (L.ext[i]) atomicAdd(&a.ext_total[i], (unsigned long long)L.ext[i]);
    if (tid == 0 && L.moved[0]) atomicAdd(a.diff_total, L.moved[0]);
}

// ---- merged SSA units (surface reactions and GHK currents that reach the outer tet) ----
//
// The reference keeps a triangle, its inner tet and its outer tet in one rank's SSA
// (sreac.cpp:200-300 rejects any other placement), so the events of all tets linked through
// such triangles form one SSA.  Here each such unit runs on one thread: elements are the
// unit's tets (their volume reactions, reac.cpp:184-251) and triangles (surface reactions
// sreac.cpp:305-520, with inner or outer volume reactants and products, then GHK currents
// ghkcurr.cpp:168-280), selected through a binary tree of element propensity sums; after an
// event only the elements whose rates read a changed count are re-evaluated.  State lives in
// the global count arrays (units are few and touch scattered tets).

// Number of reactions (and GHK currents) of element e.
__device__ __forceinline__ int unit_elem_nq(const sg_window_args& a, int e, int nt, const int32_t* tets,
                                            const int32_t* tris) {
    if (e < nt) {
        const int comp = a.comp ? __ldg(&a.comp[tets[e]]) : 0;
        return __ldg(&a.comp_reac_begin[comp + 1]) - __ldg(&a.comp_reac_begin[comp]);
    }
    const sg_surf_args& sa = a.surf;
    const int p = sa.tri_patch[tris[e - nt]];
    int n = sa.patch_sreac_begin[p + 1] - sa.patch_sreac_begin[p];
    for (int g = 0; g < sa.nghk; ++g) n += sa.ghks[g].patch == p ? 1 : 0;
    return n;
}

// Propensities of element e into prop[0..nq); returns their sum in reaction order.
static __device__ __noinline__ double unit_elem_props(const sg_window_args& a, int e, int nt, const int32_t* tets,
                                                      const int32_t* tris, int r, double* prop) {
    const sg_surf_args& sa = a.surf;
    double sum = 0.0;
    if (e < nt) {
        const int t = tets[e];
        const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
        const int rb = __ldg(&a.comp_reac_begin[comp]), re = __ldg(&a.comp_reac_begin[comp + 1]);
        const double ivs = __ldg(&a.ivs[t]);
        const double* K = a.kcst + (size_t)r * a.nreac;
        for (int q = rb; q < re; ++q) {
            const sg_reac* rc = &a.reacs[q];
            const double p = reac_prop(rc, a.counts + t, a.ntets, reac_ccst(rc, __ldg(&K[q]), ivs));
            prop[q - rb] = p;
            sum = sum + p;
        }
        return sum;
    }
    const int M = sa.ntris;
    const int m = tris[e - nt];
    const int p = sa.tri_patch[m];
    const int pb = sa.patch_sreac_begin[p], pe = sa.patch_sreac_begin[p + 1];
    const int ti = sa.tri_inner[m];
    const int to = sa.tri_outer ? sa.tri_outer[m] : -1;
    const double area = sa.tri_area[m];
    const double vm = sa.tri_V ? sa.tri_V[m] : 0.0;
    const double ivs_i = __ldg(&a.ivs[ti]);
    const double ivs_o = to >= 0 ? __ldg(&a.ivs[to]) : 0.0;
    int kk = 0;
    for (int q = pb; q < pe; ++q, ++kk) {
        const sg_sreac& rs = sa.sreacs[q];
        const double k = (rs.vdep >= 0) ? vdep_k(sa, rs.vdep, vm, a.status) : sa.skcst[q];
        const int tv = rs.vside ? to : ti;
        double pq = 0.0;
        if (tv >= 0) {
            const double h = sreac_h2(rs, sa.tri_counts + m, M, a.counts + tv, a.ntets);
            pq = h * sreac_ccst(rs, k, rs.vside ? ivs_o : ivs_i, area);
        }
        prop[kk] = pq;
        sum = sum + pq;
    }
    for (int g = 0; g < sa.nghk; ++g) {
        const sg_ghk& gh = sa.ghks[g];
        if (gh.patch != p) continue;
        const uint32_t n = sa.tri_counts[(size_t)gh.sspec * M + m];
        const uint32_t ci = a.counts[(size_t)gh.ion * a.ntets + ti];
        double rt;
        if (gh.voconc >= 0.0 || to < 0)
            rt = ghk_rate(gh, vm, ci, n, ivs_i, sa.temp, a.status);
        else
            rt = ghk_rate_outer(gh, vm, ci, n, ivs_i, a.counts[(size_t)gh.ion * a.ntets + to], ivs_o, sa.temp,
                                a.status);
        const double pq = fabs(rt);
        prop[kk++] = pq;
        sum = sum + pq;
    }
    return sum;
}

// Count of volume species s in tet t changes by d at time tt of the window (skipped when
// clamped): bounds, and the change-time sum of a diffusing species.
__device__ __forceinline__ void unit_bump_tet(const sg_window_args& a, int t, int s, int d, double tt) {
    const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
    if ((clampm >> s) & 1u) return;
    uint32_t* pc = a.counts + (size_t)s * a.ntets + t;
    const uint32_t old = *pc;
    long long nc = (long long)old + d;
    if (nc < 0 || nc > 0xFFFFFFFFll) {
        atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
        nc = nc < 0 ? 0 : 0xFFFFFFFFll;
    }
    const int ds = __ldg(&a.diff_slot[s]);
    if (ds >= 0) {
        double* pd = a.tdel + (size_t)ds * a.ntets + t;
        *pd = *pd + (double)(nc - (long long)old) * tt;
    }
    *pc = (uint32_t)nc;
}

// Apply event (element e, reaction or GHK current sel) of a merged unit at time tt of the
// window; returns the elements whose propensities read a changed count (into aff, at most
// 16: the element, and the tets whose counts changed with their triangles).
static __device__ __noinline__ int unit_apply(const sg_window_args& a, int e, int sel, int eb, int nt,
                                              const int32_t* tets, const int32_t* tris, unsigned long long parity,
                                              double tt, int* aff) {
    const sg_unit_args& U = a.units;
    const sg_surf_args& sa = a.surf;
    const int M = sa.ntris;
    int n = 0;
    auto add_tet = [&](int f) {
        if (f < 0) return;
        aff[n++] = f;
        const int4 adj = __ldg(reinterpret_cast<const int4*>(U.tet_adj) + eb + f);
        if (adj.x >= 0) aff[n++] = adj.x;
        if (adj.y >= 0) aff[n++] = adj.y;
        if (adj.z >= 0) aff[n++] = adj.z;
        if (adj.w >= 0) aff[n++] = adj.w;
    };
    if (e < nt) {
        const int t = tets[e];
        const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
        const int q = __ldg(&a.comp_reac_begin[comp]) + sel;
        const sg_reac* rc = &a.reacs[q];
        for (int i = 0; i < rc->nupd; ++i) unit_bump_tet(a, t, rc->upd_spec[i], rc->upd_delta[i], tt);
        atomicAdd(&a.ext[parity * a.nreac + q], 1ull);
        add_tet(e);
        return n;
    }
    const int j = e - nt, m = tris[j];
    const int p = sa.tri_patch[m];
    const int pb = sa.patch_sreac_begin[p], npr = sa.patch_sreac_begin[p + 1] - pb;
    const int ti = sa.tri_inner[m];
    const int to = sa.tri_outer ? sa.tri_outer[m] : -1;
    const int ei = U.tri_side[2 * m], eo = U.tri_side[2 * m + 1];
    bool ci = false, co = false;
    if (sel < npr) {
        const sg_sreac& rs = sa.sreacs[pb + sel];
        for (int i = 0; i < rs.nsupd; ++i) {
            const size_t o = (size_t)rs.supd_spec[i] * M + m;
            const uint32_t old = sa.tri_counts[o];
            U.socc[o] = U.socc[o] + (double)old * (tt - U.slast[o]);
            U.slast[o] = tt;
            long long nc = (long long)old + rs.supd_delta[i];
            if (nc < 0 || nc > 0xFFFFFFFFll) {
                atomicOr(a.status, nc < 0 ? SG_ERR_NEGATIVE : SG_ERR_OVERFLOW);
                nc = nc < 0 ? 0 : 0xFFFFFFFFll;
            }
            sa.tri_counts[o] = (uint32_t)nc;
        }
        for (int i = 0; i < rs.niupd; ++i) unit_bump_tet(a, ti, rs.iupd_spec[i], rs.iupd_delta[i], tt);
        for (int i = 0; i < rs.noupd && to >= 0; ++i) unit_bump_tet(a, to, rs.oupd_spec[i], rs.oupd_delta[i], tt);
        ci = rs.niupd > 0;
        co = rs.noupd > 0;
    } else {
        // GHK current number sel - npr of the patch: one ion out of (efflux) or into the
        // inner tet, into or out of the outer tet when its concentration is used; z
        // elementary charges for the triangle's current.
        int g = 0, left = sel - npr;
        for (; g < sa.nghk; ++g)
            if (sa.ghks[g].patch == p && left-- == 0) break;
        const sg_ghk& gh = sa.ghks[g];
        const uint32_t nch = sa.tri_counts[(size_t)gh.sspec * M + m];
        const uint32_t cin = a.counts[(size_t)gh.ion * a.ntets + ti];
        const double vm = sa.tri_V ? sa.tri_V[m] : 0.0;
        const bool outer = gh.voconc < 0.0 && to >= 0;
        const double rtg = outer ? ghk_rate_outer(gh, vm, cin, nch, __ldg(&a.ivs[ti]),
                                                  a.counts[(size_t)gh.ion * a.ntets + to], __ldg(&a.ivs[to]), sa.temp,
                                                  a.status)
                                 : ghk_rate(gh, vm, cin, nch, __ldg(&a.ivs[ti]), sa.temp, a.status);
        const bool eff = rtg >= 0.0;
        if (gh.realflux) {
            unit_bump_tet(a, ti, gh.ion, eff ? -1 : 1, tt);
            if (outer) unit_bump_tet(a, to, gh.ion, eff ? 1 : -1, tt);
            ci = true;
            co = outer;
        }
        atomicAdd((unsigned long long*)&sa.tri_echarge[m],
                  (unsigned long long)(long long)(eff ? gh.valence : -gh.valence));
    }
    atomicAdd(a.surf_ext, 1ull);
    aff[n++] = e;
    if (ci) add_tet(ei);
    if (co) add_tet(eo);
    return n;
}

// SSA of every merged unit over its window, one warp per unit, between the volume and
// membrane SSA passes and the diffusion leave of a split window: gathers the unit's inflow,
// writes its tets' counts, change-time sums and tmask, its triangles' counts and occupancy
// integrals.  The unit draws from the window stream of its first tet.  Lane 0 runs the
// event loop (draws, the descent of the tree, the reaction within the element, the count
// changes); the lanes share the gather, the element propensities, the tree build and, after
// each event, the re-evaluation of the affected elements and of their paths to the root,
// level by level (a node is always the sum of its two children, so the order of the lanes'
// updates does not change any value).  SH: the tree and the element propensities sit in
// shared memory (the largest unit fits the launch's dynamic shared memory).
template <bool SH>
__global__ void __launch_bounds__(32) unit_ssa_kernel(sg_window_args a) {
    extern __shared__ __align__(16) unsigned char smem_u[];
    __shared__ int s_aff[16];
    const sg_unit_args& U = a.units;
    const sg_surf_args& sa = a.surf;
    const int lane = threadIdx.x;
    const unsigned long long parity = __ldcg(&a.launch_state[1]) & 1ull;
    const size_t plane = (size_t)a.ntets * 4;
    const int S = a.nspec, SS = sa.nsspec, M = sa.ntris;
    for (int u = blockIdx.x; u < U.nunits; u += gridDim.x) {
        const int tb = U.tet_begin[u], nt = U.tet_begin[u + 1] - tb;
        const int mb = U.tri_begin[u], nm = U.tri_begin[u + 1] - mb;
        const int32_t* tets = U.tets + tb;
        const int32_t* tris = U.tris + mb;
        const int r = find_real(a.reals, a.nreal, tets[0]);
        const sg_real* rl = &a.reals[r];
        const double rt = rl->t, rend = rl->t_end, per = rl->period;
        if (!(rt < rend)) continue;
        const double T = (rt + per > rend) ? rend - rt : per;
        const unsigned long long w = rl->window;
        const int pending = rl->pending;
        // Gather the last window's inflow into the unit's tets and triangles.
        const uint32_t* in = a.outflow + (size_t)((w + 1) & 1ull) * a.ndiff * plane;
        for (int k = lane; k < nt; k += 32) {
            const int t = tets[k];
            const int comp = a.comp ? __ldg(&a.comp[t]) : 0;
            const uint32_t clampm = a.clamp ? __ldg(&a.clamp[t]) : 0u;
            const int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
            const double* Dc = a.dcst + ((size_t)r * a.ncomp + comp) * S;
            for (int s = 0; s < S; ++s) {
                uint32_t c = a.counts[(size_t)s * a.ntets + t];
                const int ds = __ldg(&a.diff_slot[s]);
                if (pending && ds >= 0 && __ldg(&Dc[s]) > 0.0 && !((clampm >> s) & 1u)) {
                    const uint4 v = __ldg(reinterpret_cast<const uint4*>(in + (size_t)ds * plane) + t);
                    unsigned long long sum = c;
                    if (nb.x >= 0) sum += v.x;
                    if (nb.y >= 0) sum += v.y;
                    if (nb.z >= 0) sum += v.z;
                    if (nb.w >= 0) sum += v.w;
                    if (a.bface) sum += bnd_inflow(a, t, r, s, v);
                    if (sum > 0xFFFFFFFFull) {
                        atomicOr(a.status, SG_ERR_OVERFLOW);
                        sum = 0xFFFFFFFFull;
                    }
                    c = (uint32_t)sum;
                }
                if (ds >= 0) a.tdel[(size_t)ds * a.ntets + t] = 0.0;
                a.counts[(size_t)s * a.ntets + t] = c;
                if (c) atomicAdd(&a.totals[parity * S + s], (unsigned long long)c);
            }
        }
        for (int j = lane; j < nm; j += 32) {
            const int m = tris[j];
            const int p = sa.tri_patch[m];
            for (int s = 0; s < SS; ++s) {
                const size_t o = (size_t)s * M + m;
                uint32_t c = sa.tri_counts[o];
                if (pending && sa.tri_outflow) {
                    const int sd = sa.sdiff_slot[s];
                    if (sd >= 0 && sa.sdcst[(size_t)p * SS + s] > 0.0) {
                        const uint4 v = reinterpret_cast<const uint4*>(
                            sa.tri_outflow + (size_t)((w + 1) & 1ull) * sa.nsdiff * M * 4)[(size_t)sd * M + m];
                        const int4 nb = reinterpret_cast<const int4*>(sa.snbr)[m];
                        unsigned long long sum = c;
                        if (nb.x >= 0) sum += v.x;
                        if (nb.y >= 0) sum += v.y;
                        if (nb.z >= 0) sum += v.z;
                        if (sum > 0xFFFFFFFFull) {
                            atomicOr(a.status, SG_ERR_OVERFLOW);
                            sum = 0xFFFFFFFFull;
                        }
                        c = (uint32_t)sum;
                    }
                }
                sa.tri_counts[o] = c;
                U.socc[o] = 0.0;
                U.slast[o] = 0.0;
            }
        }
        __syncwarp();
        // Element sums and the tree (node i = node 2i + node 2i + 1; leaves P..2P-1).
        const int E = nt + nm;
        const int eb = U.elem_base[u];
        const int P = (U.tree_base[u + 1] - U.tree_base[u]) >> 1;
        double* tree = SH ? reinterpret_cast<double*>(smem_u) : U.tree + U.tree_base[u];
        double* prop = SH ? reinterpret_cast<double*>(smem_u) + 2 * P : U.prop + (size_t)eb * U.rmax;
        for (int e = lane; e < P; e += 32)
            tree[P + e] = e < E ? unit_elem_props(a, e, nt, tets, tris, r, prop + (size_t)e * U.rmax) : 0.0;
        __syncwarp();
        for (int h = P >> 1; h >= 1; h >>= 1) {
            for (int i = h + lane; i < 2 * h; i += 32) tree[i] = tree[2 * i] + tree[2 * i + 1];
            __syncwarp();
        }
        sg_stream st;
        sg_stream_init(&st, a.seed, (uint32_t)r, (uint32_t)(tets[0] - rl->tet_begin), w, SG_PURPOSE_WINDOW);
        double tt = 0.0;
        for (;;) {
            int naff = 0;
            if (lane == 0) {
                const double a0 = tree[1];
                int e = -1, sel = -1;
                if (a0 > 0.0) {
                    const double dt = -sg_log(sg_u01_oc(sg_next_u32(&st))) / a0;
                    if (tt + dt <= T) {
                        tt = tt + dt;
                        double target = sg_u01_co(sg_next_u32(&st)) * a0;
                        // Descend: left while the target falls below the left sum (or nothing is right).
                        int node = 1;
                        while (node < P) {
                            const double l = tree[2 * node], rr = tree[2 * node + 1];
                            if (target < l || !(rr > 0.0)) {
                                node = 2 * node;
                            } else {
                                target = target - l;
                                node = 2 * node + 1;
                            }
                        }
                        e = node - P;
                        const double* pq = prop + (size_t)e * U.rmax;
                        const int nq = unit_elem_nq(a, e, nt, tets, tris);
                        double cum = 0.0;
                        int lastnz = -1;
                        for (int q = 0; q < nq; ++q) {
                            const double pv = pq[q];
                            if (pv > 0.0) {
                                lastnz = q;
                                cum = cum + pv;
                                if (target < cum) {
                                    sel = q;
                                    break;
                                }
                            }
                        }
                        if (sel < 0) sel = lastnz;
                    }
                }
                if (sel >= 0) naff = unit_apply(a, e, sel, eb, nt, tets, tris, parity, tt, s_aff);
            }
            naff = __shfl_sync(0xffffffffu, naff, 0);
            if (naff == 0) break;
            __syncwarp();
            // The affected elements' propensities, then their paths to the root by levels.
            int node = 0;
            if (lane < naff) {
                const int f = s_aff[lane];
                node = P + f;
                tree[node] = unit_elem_props(a, f, nt, tets, tris, r, prop + (size_t)f * U.rmax);
            }
            __syncwarp();
            for (int h = P >> 1; h >= 1; h >>= 1) {
                node >>= 1;
                if (lane < naff) tree[node] = tree[2 * node] + tree[2 * node + 1];
                __syncwarp();
            }
        }
        __syncwarp();
        // Occupancy integrals of the triangles, change-time masks of the tets.
        for (int j = lane; j < nm; j += 32) {
            const int m = tris[j];
            for (int s = 0; s < SS; ++s) {
                const size_t o = (size_t)s * M + m;
                const uint32_t c = sa.tri_counts[o];
                const double occ = U.socc[o] + (double)c * (T - U.slast[o]);
                sa.spec_int[o] += occ;
                if (sa.tri_occ) {
                    const int sd = sa.sdiff_slot[s];
                    if (sd >= 0) sa.tri_occ[(size_t)sd * M + m] = occ;
                }
            }
        }
        for (int k = lane; k < nt && a.tmask; k += 32) {
            const int t = tets[k];
            uint32_t tm = 0u;
            for (int s = 0; s < S; ++s) {
                const int ds = __ldg(&a.diff_slot[s]);
                if (ds >= 0 && a.tdel[(size_t)ds * a.ntets + t] != 0.0) tm |= 1u << s;
            }
            a.tmask[t] = tm;
        }
        __syncwarp();
    }
}

// Apply the pending surface-diffusion inflow to the triangle counts (before host reads).
static __global__ void sflush_kernel(sg_window_args a) {
    const sg_surf_args& sa = a.surf;
    const int M = sa.ntris, SS = sa.nsspec;
    const long long total = (long long)sa.nsdiff * M;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int sd = (int)(idx / M);
        const int m = (int)(idx - (long long)sd * M);
        const sg_real* rl = &a.reals[find_real(a.reals, a.nreal, sa.tri_inner[m])];
        if (!rl->pending) continue;
        const int s = sa.sdiff_spec[sd];
        if (!(sa.sdcst[(size_t)sa.tri_patch[m] * SS + s] > 0.0)) continue;
        const uint4 v = reinterpret_cast<const uint4*>(sa.tri_outflow + (size_t)((rl->window + 1) & 1ull) *
                                                                            sa.nsdiff * M * 4)[(size_t)sd * M + m];
        const int4 nb = reinterpret_cast<const int4*>(sa.snbr)[m];
        unsigned long long sum = sa.tri_counts[(size_t)s * M + m];
        if (nb.x >= 0) sum += v.x;
        if (nb.y >= 0) sum += v.y;
        if (nb.z >= 0) sum += v.z;
        if (sum > 0xFFFFFFFFull) {
            atomicOr(a.status, SG_ERR_OVERFLOW);
            sum = 0xFFFFFFFFull;
        }
        sa.tri_counts[(size_t)s * M + m] = (uint32_t)sum;
    }
}

// Apply the pending inflow of the last window to the counts (enter phase only).
static __global__ void flush_kernel(sg_window_args a) {
    const size_t plane = (size_t)a.ntets * 4;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.ntets; t += gridDim.x * blockDim.x) {
        int r = find_real(a.reals, a.nreal, t);
        const sg_real* rl = &a.reals[r];
        if (!rl->pending) continue;
        int comp = a.comp ? a.comp[t] : 0;
        if (comp < 0) continue;
        int4 nb = __ldg(reinterpret_cast<const int4*>(a.nbr) + t);
        uint32_t clampm = a.clamp ? a.clamp[t] : 0u;
        const double* Dc = a.dcst + ((size_t)r * a.ncomp + comp) * a.nspec;
        const uint32_t* in = a.outflow + (size_t)((rl->window + 1) & 1ull) * a.ndiff * plane;
        for (int s = 0; s < a.nspec; ++s) {
            int ds = a.diff_slot[s];
            if (ds < 0 || !(Dc[s] > 0.0) || ((clampm >> s) & 1u)) continue;
            const uint4 v = reinterpret_cast<const uint4*>(in + (size_t)ds * plane)[t];
            unsigned long long sum = a.counts[(size_t)s * a.ntets + t];
            if (nb.x >= 0) sum += v.x;
            if (nb.y >= 0) sum += v.y;
            if (nb.z >= 0) sum += v.z;
            if (nb.w >= 0) sum += v.w;
            if (a.bface) sum += bnd_inflow(a, t, r, s, v);
            if (sum > 0xFFFFFFFFull) {
                atomicOr(a.status, SG_ERR_OVERFLOW);
                sum = 0xFFFFFFFFull;
            }
            a.counts[(size_t)s * a.ntets + t] = (uint32_t)sum;
        }
    }
}

static __global__ void clear_pending_kernel(sg_real* reals, int nreal) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nreal; i += gridDim.x * blockDim.x)
        reals[i].pending = 0;
}

}  // namespace sg
