// EField: vertex-based membrane-potential solve on the GPU.
//
// Reference: src/steps/solver/efield/ (efield.cpp:48-112 initMesh, dVsolver.hpp:126-180
// _advance, tetcoupler.cpp:48-300 coupling coefficients, tetmesh.cpp:231-262 surface).
// Units as in the reference EField: um, ms, mV, pA, pF, nS.
//
// Each EField step assembles the backward-Euler system of dVsolver.hpp:126-180,
//     A_ii = C_i/dt + g_i + sum_j cc_ij,   A_ij = -cc_ij,
//     b_i  = I_i + g_i (V_ext - V_i) + sum_j cc_ij (V_j - V_i),
// solves A dV = b with CG preconditioned by Jacobi plus a coarse solve on spatial vertex
// aggregates (FP64, or FP32 CG inside an FP64 residual-refinement loop), warm-started
// from the previous step's dV, and updates V += dV on unclamped vertices.  Clamped rows
// are identity rows with b = 0, so their columns drop out and A stays SPD.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace sg {

enum EFieldMethod { EF_CG_FP64 = 0, EF_CG_MIXED = 1 };

struct EFieldStats {
    uint64_t steps = 0;
    uint64_t iterations = 0;        // inner CG iterations (FP32 ones in mixed mode)
    uint64_t refinements = 0;       // FP64 residual evaluations
    double last_rel_residual = 0.0;
    double solve_ms = 0.0;          // device time of the solves (CUDA events)
    // Per-step check of the solve against an FP64 solve of the same system to check_tol.
    uint64_t check_steps = 0;
    double check_max_rel = 0.0;     // max over steps and vertices of |V_mixed - V_fp64| / |V_fp64|
    double check_last_rel = 0.0;
};

struct EFieldSystem {
    // ---- host model ----
    int nverts = 0;
    int ntris = 0;                        // membrane triangles
    std::vector<int32_t> tri_verts;       // [ntris][3]
    std::vector<double> tri_area_um2;     // [ntris]
    std::vector<double> vert_area_um2;    // [nverts] membrane area attributed to the vertex
    std::vector<int32_t> nbr_ptr, nbr_idx;// vertex adjacency (CSR, no diagonal)
    std::vector<double> geo_cc;           // geometric coupling per adjacency entry (um)
    double cm = 0.01;                     // pF/um^2   (1 uF/cm^2, efield.cpp:81)
    double sigma = 1.0 / 1.0e-3;          // nS/um     (1 ohm m, efield.cpp:87)
    double g_leak = 0.0;                  // nS/um^2   surface conductance
    double v_leak = 0.0;                  // mV
    int method = EF_CG_FP64;
    double tol = 1.0e-10;                 // relative residual of the FP64 solve
    int max_iter = 20000;
    std::vector<uint8_t> vclamped;        // [nverts]
    std::vector<double> vert_iclamp;      // pA, [nverts]
    std::vector<double> tri_iclamp;       // pA, [ntris]

    // ---- device ----
    int width = 0;                        // ELL width (max off-diagonal entries per row)
    double* V = nullptr;                  // mV [nverts]
    double* tri_V = nullptr;              // mV [ntris]
    double* tri_I = nullptr;              // pA [ntris] (outward membrane current of the step)
    int32_t* d_tri_verts = nullptr;
    int32_t* d_vt_ptr = nullptr;          // vertex -> membrane tris (CSR)
    int32_t* d_vt_idx = nullptr;
    double* d_vert_iclamp = nullptr;
    double* d_tri_iclamp = nullptr;
    int32_t* ell_col = nullptr;           // [width][nverts], -1 = padding
    double* ell_cc = nullptr;             // [width][nverts] cc_ij (nS), all neighbours (RHS)
    double* ell_a64 = nullptr;            // [width][nverts] -cc_ij, clamped columns removed
    float* ell_a32 = nullptr;
    double* diag64 = nullptr;             // A_ii
    // The previous step length's diagonal and coarse inverses (swapped back in when dt
    // returns to it without a rebuild); alt_dt < 0: none.
    double alt_dt = -1.0;
    double* alt_diag64 = nullptr;
    double* alt_einv64 = nullptr;
    float* alt_einv32 = nullptr;
    double* cap_gext = nullptr;           // [2][nverts]: C_i (pF), g_i (nS)
    uint8_t* d_vclamped = nullptr;
    // Two-level preconditioner M^-1 = D^-1 + Z E^-1 Z^T: Z aggregates vertices into spatial
    // bins (piecewise-constant coarse space), E = Z^T A Z is inverted densely on the host.
    std::vector<double> verts_um;         // [nverts][3] for the aggregation
    int nagg = 0;
    int ncomp_v = 0;                      // connected components of the vertex graph
    std::vector<std::vector<int32_t>> comp_verts;  // their vertices, ascending
    size_t einv_len = 0;                  // sum over components of (aggregates)^2
    int32_t* d_agg_base = nullptr;        // [nagg] first aggregate of the aggregate's component
    int32_t* d_agg_len = nullptr;         // [nagg] aggregates in that component
    long long* d_agg_row = nullptr;       // [nagg] offset of the aggregate's row in the coarse inverse
    int32_t* d_agg = nullptr;             // [nverts] aggregate of each vertex, -1 for clamped
    // Vertex segments for the restriction Z^T r: one per aggregate (its vertices in
    // ascending order), then chunks of the vertices in no aggregate.
    int nseg = 0;
    int32_t* d_seg_ptr = nullptr;         // [nseg + 1]
    int32_t* d_seg_idx = nullptr;         // [nverts]
    int32_t* d_seg_agg = nullptr;         // [nseg], -1 = no aggregate
    double* d_einv64 = nullptr;           // per component a dense [m][m] block, m its aggregates
    float* d_einv32 = nullptr;
    double* d_c64 = nullptr;              // restricted residual [nagg]
    float* d_c32 = nullptr;
    int32_t* acol_dev = nullptr;          // [width][nverts] matrix columns (clamped ones removed)
    double inner_tol = 1.0e-4;            // relative residual of each FP32 inner solve
    // Mixed method, persistent solve: one FP32 solve with reliable updates (the FP64
    // residual replaces the FP32 one whenever the latter has fallen by ru_delta) instead of
    // restarted inner solves; ru_tol2 > 0 only while such a solve runs.
    bool reliable = true;
    double ru_delta = 0.1;
    double ru_tol2 = 0.0;
    bool check = false;                   // also solve each step in FP64 to check_tol and compare
    double check_tol = 1.0e-12;           // relative residual of the FP64 check solve
    double* xchk = nullptr;               // [nverts] dV of the FP64 check solve
    double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *p2 = nullptr, *q = nullptr;
    float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *p2_32 = nullptr, *q32 = nullptr, *x32 = nullptr,
          *s32 = nullptr;
    double* red = nullptr;                // reduction partials
    double* scal = nullptr;               // device scalars
    unsigned int* red_count = nullptr;
    unsigned int* d_bar = nullptr;        // grid barrier of the persistent solve: count, generation, error
    bool persistent = true;               // whole solve in one cooperative launch (else a launch per phase)
    unsigned int spin_limit = 1u << 22;   // polls of a grid-barrier wait before the persistent solve gives up
    double dt_built = -1.0;
    bool dirty = true;                    // clamps / membrane properties changed
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evc0 = nullptr, evc1 = nullptr;
    EFieldStats stats;
    int nsm = 148;

    // Mesh vertex index -> index in the device arrays (vertices are stored grouped by
    // connected component and coarse aggregate); every per-vertex array of this struct,
    // host or device, is in device order.
    std::vector<int32_t> vperm;
    int vid(int mesh_vertex) const { return vperm.empty() ? mesh_vertex : vperm[mesh_vertex]; }

    ~EFieldSystem();
    // verts in um, tets [ntet][4] (all tets that conduct), membrane tris [ntris][3] with areas,
    // all indexed by mesh vertex; renumbers the vertices (vperm) and calls setup_ordered.
    void setup(int nverts, const double* verts_um, int ntet, const int32_t* tets, int ntris,
               const int32_t* tris, cudaStream_t stream, int nsm);
    void setup_ordered(int nverts, const double* verts_um, int ntet, const int32_t* tets, int ntris,
                       const int32_t* tris, cudaStream_t stream, int nsm);
    void set_potential(double v_mV, cudaStream_t stream);
    void build_matrix(double dt_ms, cudaStream_t stream);
    // One EField step of dt_ms with tri_I already set on the device.
    void advance(double dt_ms, cudaStream_t stream);
    void release();
    // Grid of the warp-per-segment kernels: 8 segments per block, at most 1024 blocks (the
    // reduction partials hold 2 x 1024 values); warps stride over the rest.
    int seg_grid() const { return nseg > 0 ? std::min((nseg + 7) / 8, 1024) : 1; }
    template <typename T>
    void pcg(cudaStream_t stream, int n, int g, const T* a, T* xv, T* rv, T* zv, T* pv, T* pv2, T* qv,
             const T* einv, T* cvec, double* h);
    template <typename T>
    void pcg_persistent(cudaStream_t stream, int n, const T* a, T* xv, T* rv, T* zv, T* pv, T* pv2, T* qv,
                        const T* einv, T* cvec, double* h);
    template <typename T>
    void pcg_loop(cudaStream_t stream, int n, int g, const T* a, T* xv, T* rv, T* zv, T* pv, T* pv2, T* qv,
                  const T* einv, T* cvec, double* h);
};

// Geometric coupling of a tet mesh: for every edge ij, sum over tets of the linear-FEM
// stiffness -V_T grad(phi_i).grad(phi_j) (um).  Exposed for the tests.
void efield_couple(int nverts, const double* verts_um, int ntet, const int32_t* tets,
                   std::vector<int32_t>& ptr, std::vector<int32_t>& idx, std::vector<double>& cc);

}  // namespace sg
