// Surface part of an SSA unit: a tet together with the membrane triangles whose inner
// tet it is.  Restates src/steps/mpi/tetopsplit/sreac.cpp:40-68 (constant scaling by
// inner-tet volume or triangle area), :305-428 (propensity), :431-520 (apply),
// vdepsreac.cpp:46-76 / vdepsreacdef.cpp:194-218 (k(V) by table interpolation) and the
// ohmic-current time integrals of tri.cpp:544-561, 664-694 (integral of the channel-state
// count over the EField step).
#pragma once
#include "sg_rng.cuh"
#include "sg_types.h"

namespace sg {

#define SG_AVOGADRO 6.02214179e23  // src/steps/math/constants.hpp:45

// Shared-memory region of the surface state, appended after the volume layout.
struct surf_layout {
    uint32_t* cnt;   // [4*SS][BLOCK]
    double* occ;     // [4*SS][BLOCK]
    double* last;    // [4*SS][BLOCK]
    double* prop;    // [4*RSP][BLOCK]
};

__host__ __device__ inline size_t surf_smem_bytes(int block, int nss, int rsp) {
    size_t b = (size_t)4 * nss * block * 4;
    b = (b + 15) & ~(size_t)15;
    b += (size_t)4 * nss * block * 16;
    b += (size_t)4 * rsp * block * 8;
    return b;
}

__device__ inline surf_layout surf_carve(unsigned char* base, int block, int nss, int rsp) {
    surf_layout L;
    size_t b = (size_t)4 * nss * block * 4;
    L.cnt = (uint32_t*)base;
    b = (b + 15) & ~(size_t)15;
    L.occ = (double*)(base + b);
    b += (size_t)4 * nss * block * 8;
    L.last = (double*)(base + b);
    b += (size_t)4 * nss * block * 8;
    L.prop = (double*)(base + b);
    return L;
}

// k(V) of a voltage-dependent reaction: linear interpolation (vdepsreacdef.cpp:194-218).
__device__ inline double vdep_k(const sg_surf_args& sa, int tab, double v_mV, uint32_t* status) {
    const sg_vtab vt = sa.vtabs[tab];
    double v = v_mV * 1.0e-3;
    double v2 = (v - vt.vmin) / vt.dv;
    if (!(v2 >= 0.0) || v2 > (double)(vt.n - 1)) {
        atomicOr(status, SG_ERR_TABLE);
        v2 = v2 < 0.0 ? 0.0 : (double)(vt.n - 1);
    }
    double lv = floor(v2);
    int lo = (int)lv;
    int hi = (int)ceil(v2);
    double r = v2 - lv;
    return (1.0 - r) * sa.vtab_vals[vt.off + lo] + r * sa.vtab_vals[vt.off + hi];
}

#define SG_FARADAY 96485.3399       // src/steps/math/constants.hpp:49
#define SG_GAS_CONSTANT 8.314472    // constants.hpp:53
#define SG_E_CHARGE 1.602176487e-19 // constants.hpp:57

// Single-channel GHK current (A) of src/steps/math/ghk.cpp:71-90 at potential v (V), with
// inner/outer concentrations in mol/m^3: P z F nu (ci - co e^-nu) / (1 - e^-nu),
// nu = z v F / (R T); the limit P z F (ci - co) at nu = 0.  |nu| beyond the double range
// is an error, as in the reference.
__device__ inline double ghk_current(double P, double v, int z, double temp, double ci, double co,
                                     uint32_t* status) {
    const double nu = (double)z * v * SG_FARADAY / (SG_GAS_CONSTANT * temp);
    if (!(nu < 700.0 && nu > -700.0)) {
        atomicOr(status, SG_ERR_TABLE);
        return 0.0;
    }
    if (fabs(nu) > 2.220446049250313e-16) {
        const double e = sg_exp(-nu);
        return P * (double)z * SG_FARADAY * nu * (ci - co * e) / (1.0 - e);
    }
    return P * (double)z * SG_FARADAY * (ci - co);
}

// Signed rate (ions/s) of one GHK current on a triangle with n channels in the state, inner
// ion count c_ion in a tet of 1/(1e3 V N_A) = ivs, triangle potential vm (mV): positive is an
// efflux (ghkcurr.cpp:168-212).
__device__ inline double ghk_rate(const sg_ghk& g, double vm, uint32_t c_ion, uint32_t n, double ivs, double temp,
                                  uint32_t* status) {
    if (n == 0) return 0.0;
    const double ci = (double)c_ion * ivs * 1.0e3;  // M -> mol/m^3
    const double co = g.voconc * 1.0e3;
    const double I = ghk_current(g.perm, vm * 1.0e-3 + g.vshift, g.valence, temp, ci, co, status);
    return I / (SG_E_CHARGE * (double)g.valence) * (double)n;
}

// Signed rate of a GHK current whose outer concentration is that of the outer tet, c_out
// ions in a tet of 1/(1e3 V N_A) = ivs_out (ghkcurr.cpp:176-181 with voconc < 0).
__device__ inline double ghk_rate_outer(const sg_ghk& g, double vm, uint32_t c_ion, uint32_t n, double ivs,
                                        uint32_t c_out, double ivs_out, double temp, uint32_t* status) {
    if (n == 0) return 0.0;
    const double ci = (double)c_ion * ivs * 1.0e3;
    const double co = (double)c_out * ivs_out * 1.0e3;
    const double I = ghk_current(g.perm, vm * 1.0e-3 + g.vshift, g.valence, temp, ci, co, status);
    return I / (SG_E_CHARGE * (double)g.valence) * (double)n;
}

// Scaled constant of a surface reaction on triangle m whose inner tet has 1/(1e3 V N_A) = ivs.
__device__ inline double sreac_ccst(const sg_sreac& r, double k, double ivs, double area) {
    if (r.surf_surf) {
        double ascale = area * SG_AVOGADRO;  // comp_ccst_area (sreac.cpp:60-68)
        if (r.order == 0) return k * ascale;
        double c = k;
        for (int i = 1; i < r.order; ++i) c = c / ascale;
        return c;
    }
    if (r.order == 0) return k / ivs;        // comp_ccst_vol (sreac.cpp:40-58)
    double c = k;
    for (int i = 1; i < r.order; ++i) c = c * ivs;
    return c;
}

__device__ inline double falling(uint32_t c, uint32_t o) {
    double h = 1.0;
    if (o >= 4) h = h * (double)(c - 3);
    if (o >= 3) h = h * (double)(c - 2);
    if (o >= 2) h = h * (double)(c - 1);
    return h * (double)c;
}

// h_mu of a surface reaction: surface reactants on slot j, volume reactants in the tet.
__device__ inline double sreac_h(const sg_sreac& r, const uint32_t* scnt_slot, const uint32_t* vcnt, int stride) {
    double h = 1.0;
    for (int i = 0; i < r.nslhs; ++i) {
        uint32_t c = scnt_slot[r.slhs_spec[i] * stride];
        uint32_t o = (uint32_t)r.slhs_ord[i];
        if (o > c) return 0.0;
        h = h * falling(c, o);
    }
    for (int i = 0; i < r.nilhs; ++i) {
        uint32_t c = vcnt[r.ilhs_spec[i] * stride];
        uint32_t o = (uint32_t)r.ilhs_ord[i];
        if (o > c) return 0.0;
        h = h * falling(c, o);
    }
    return h;
}

// The same product with the surface and volume counts at their own strides (the merged
// units read them from the global count arrays); vcnt is the tet on the reactants' side.
__device__ inline double sreac_h2(const sg_sreac& r, const uint32_t* scnt, int sstride, const uint32_t* vcnt,
                                  int vstride) {
    double h = 1.0;
    for (int i = 0; i < r.nslhs; ++i) {
        uint32_t c = scnt[(size_t)r.slhs_spec[i] * sstride];
        uint32_t o = (uint32_t)r.slhs_ord[i];
        if (o > c) return 0.0;
        h = h * falling(c, o);
    }
    for (int i = 0; i < r.nilhs; ++i) {
        uint32_t c = vcnt[(size_t)r.ilhs_spec[i] * vstride];
        uint32_t o = (uint32_t)r.ilhs_ord[i];
        if (o > c) return 0.0;
        h = h * falling(c, o);
    }
    return h;
}

}  // namespace sg
