// EField membrane-potential solve (see sg_efield.h for the equations and units).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <tuple>
#include <vector>

#include "sg_efield.h"
#include "sg_errors.h"
#include "sg_types.h"

namespace sg {

// ---------------------------------------------------------------------------
// Geometry: coupling between the vertices of every edge.  For a tet T with linear
// shape functions phi_i, the flux of the piecewise-linear field through the part of
// vertex i's barycentric dual cell inside T is sum_j -V_T grad(phi_i).grad(phi_j) V_j,
// the quantity tetcoupler.cpp:195-300 integrates face by face.  Summed over the tets
// of an edge this is the geometric coupling cc_ij (um); times the conductivity it is
// the conductance between the two vertices (nS).
// ---------------------------------------------------------------------------
void efield_couple(int nverts, const double* X, int ntet, const int32_t* tets, std::vector<int32_t>& ptr,
                   std::vector<int32_t>& idx, std::vector<double>& cc) {
    std::vector<std::tuple<int32_t, int32_t, double>> e;
    e.reserve((size_t)ntet * 6);
    for (int t = 0; t < ntet; ++t) {
        const int32_t* v = tets + (size_t)t * 4;
        for (int k = 0; k < 4; ++k)
            if (v[k] < 0 || v[k] >= nverts) throw ArgErr("tet vertex index out of range");
        double J[3][3];  // columns: x1-x0, x2-x0, x3-x0
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) J[r][c] = X[(size_t)v[c + 1] * 3 + r] - X[(size_t)v[0] * 3 + r];
        double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        if (!(std::fabs(det) > 0.0)) throw ArgErr("degenerate tetrahedron in the EField mesh");
        // Rows of J^-1 are the gradients of phi_1..phi_3.
        double inv[3][3];
        inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
        inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
        inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
        inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
        inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
        double gr[4][3];
        for (int c = 0; c < 3; ++c) {
            gr[1][c] = inv[0][c];
            gr[2][c] = inv[1][c];
            gr[3][c] = inv[2][c];
            gr[0][c] = -(inv[0][c] + inv[1][c] + inv[2][c]);
        }
        double vol = std::fabs(det) / 6.0;
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) {
                double k = vol * (gr[i][0] * gr[j][0] + gr[i][1] * gr[j][1] + gr[i][2] * gr[j][2]);
                int a = v[i], b = v[j];
                if (a > b) std::swap(a, b);
                e.emplace_back(a, b, -k);
            }
    }
    std::sort(e.begin(), e.end(), [](const auto& x, const auto& y) {
        return std::get<0>(x) != std::get<0>(y) ? std::get<0>(x) < std::get<0>(y) : std::get<1>(x) < std::get<1>(y);
    });
    // Reduce duplicates (one entry per tet sharing the edge), then mirror to both rows.
    std::vector<std::tuple<int32_t, int32_t, double>> u;
    for (auto& t : e) {
        if (!u.empty() && std::get<0>(u.back()) == std::get<0>(t) && std::get<1>(u.back()) == std::get<1>(t))
            std::get<2>(u.back()) += std::get<2>(t);
        else
            u.push_back(t);
    }
    std::vector<int32_t> deg(nverts, 0);
    for (auto& t : u) {
        deg[std::get<0>(t)]++;
        deg[std::get<1>(t)]++;
    }
    ptr.assign(nverts + 1, 0);
    for (int i = 0; i < nverts; ++i) ptr[i + 1] = ptr[i] + deg[i];
    idx.assign(ptr[nverts], 0);
    cc.assign(ptr[nverts], 0.0);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (auto& t : u) {
        int a = std::get<0>(t), b = std::get<1>(t);
        double w = std::get<2>(t);
        idx[fill[a]] = b;
        cc[fill[a]++] = w;
        idx[fill[b]] = a;
        cc[fill[b]++] = w;
    }
}

template <typename T>
static void dalloc(T*& p, size_t n) {
    if (p) cudaFree(p);
    p = nullptr;
    if (n) SG_CUDA(cudaMalloc((void**)&p, n * sizeof(T)));
}

template <typename T>
static void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

void EFieldSystem::release() {
    dfree(V);
    dfree(tri_V);
    dfree(tri_I);
    dfree(d_tri_verts);
    dfree(d_vt_ptr);
    dfree(d_vt_idx);
    dfree(d_vert_iclamp);
    dfree(d_tri_iclamp);
    dfree(ell_col);
    dfree(ell_cc);
    dfree(ell_a64);
    dfree(ell_a32);
    dfree(diag64);
    dfree(cap_gext);
    dfree(d_vclamped);
    dfree(b);
    dfree(x);
    dfree(r);
    dfree(z);
    dfree(p);
    dfree(q);
    dfree(r32);
    dfree(z32);
    dfree(p32);
    dfree(q32);
    dfree(x32);
    dfree(s32);
    dfree(acol_dev);
    dfree(red);
    dfree(scal);
    dfree(red_count);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
}

EFieldSystem::~EFieldSystem() { release(); }

void EFieldSystem::setup(int nv, const double* verts_um, int ntet, const int32_t* tets, int nt,
                         const int32_t* tris, cudaStream_t stream, int nsm_) {
    if (nv <= 0) throw ArgErr("EField needs vertices");
    nsm = nsm_;
    nverts = nv;
    ntris = nt;
    efield_couple(nv, verts_um, ntet, tets, nbr_ptr, nbr_idx, geo_cc);
    tri_verts.assign(tris, tris + (size_t)nt * 3);
    tri_area_um2.assign(nt, 0.0);
    vert_area_um2.assign(nv, 0.0);
    // Membrane area per vertex: a third of each adjacent membrane triangle (tetmesh.cpp:231-262).
    for (int t = 0; t < nt; ++t) {
        const int32_t* v = tris + (size_t)t * 3;
        for (int k = 0; k < 3; ++k)
            if (v[k] < 0 || v[k] >= nv) throw ArgErr("triangle vertex index out of range");
        double a[3], bb[3];
        for (int c = 0; c < 3; ++c) {
            a[c] = verts_um[(size_t)v[1] * 3 + c] - verts_um[(size_t)v[0] * 3 + c];
            bb[c] = verts_um[(size_t)v[2] * 3 + c] - verts_um[(size_t)v[0] * 3 + c];
        }
        double cx = a[1] * bb[2] - a[2] * bb[1], cy = a[2] * bb[0] - a[0] * bb[2], cz = a[0] * bb[1] - a[1] * bb[0];
        double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        tri_area_um2[t] = area;
        for (int k = 0; k < 3; ++k) vert_area_um2[v[k]] += area / 3.0;
    }
    width = 0;
    for (int i = 0; i < nv; ++i) width = std::max(width, nbr_ptr[i + 1] - nbr_ptr[i]);
    vclamped.assign(nv, 0);
    vert_iclamp.assign(nv, 0.0);
    tri_iclamp.assign(nt, 0.0);

    // Vertex -> membrane triangle adjacency for the current gather.
    std::vector<int32_t> vt_ptr(nv + 1, 0), vt_idx((size_t)nt * 3);
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < 3; ++k) vt_ptr[tris[(size_t)t * 3 + k] + 1]++;
    for (int i = 0; i < nv; ++i) vt_ptr[i + 1] += vt_ptr[i];
    std::vector<int32_t> fill(vt_ptr.begin(), vt_ptr.end() - 1);
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < 3; ++k) vt_idx[fill[tris[(size_t)t * 3 + k]]++] = t;

    release();
    SG_CUDA(cudaEventCreate(&ev0));
    SG_CUDA(cudaEventCreate(&ev1));
    dalloc(V, nv);
    dalloc(tri_V, std::max(nt, 1));
    dalloc(tri_I, std::max(nt, 1));
    dalloc(d_tri_verts, std::max(nt * 3, 1));
    dalloc(d_vt_ptr, nv + 1);
    dalloc(d_vt_idx, std::max(nt * 3, 1));
    dalloc(d_vert_iclamp, nv);
    dalloc(d_tri_iclamp, std::max(nt, 1));
    dalloc(ell_col, (size_t)width * nv);
    dalloc(ell_cc, (size_t)width * nv);
    dalloc(ell_a64, (size_t)width * nv);
    dalloc(ell_a32, (size_t)width * nv);
    dalloc(diag64, nv);
    dalloc(cap_gext, 2 * (size_t)nv);
    dalloc(d_vclamped, nv);
    dalloc(b, nv);
    dalloc(x, nv);
    dalloc(r, nv);
    dalloc(z, nv);
    dalloc(p, nv);
    dalloc(q, nv);
    dalloc(r32, nv);
    dalloc(z32, nv);
    dalloc(p32, nv);
    dalloc(q32, nv);
    dalloc(x32, nv);
    dalloc(s32, nv);
    dalloc(red, 4096);
    dalloc(scal, 32);
    dalloc(red_count, 4);
    if (nt) SG_CUDA(cudaMemcpyAsync(d_tri_verts, tris, (size_t)nt * 3 * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_vt_ptr, vt_ptr.data(), vt_ptr.size() * 4, cudaMemcpyHostToDevice, stream));
    if (nt) SG_CUDA(cudaMemcpyAsync(d_vt_idx, vt_idx.data(), vt_idx.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemsetAsync(d_vert_iclamp, 0, nv * 8, stream));
    SG_CUDA(cudaMemsetAsync(d_tri_iclamp, 0, std::max(nt, 1) * 8, stream));
    SG_CUDA(cudaMemsetAsync(tri_I, 0, std::max(nt, 1) * 8, stream));
    SG_CUDA(cudaMemsetAsync(x, 0, nv * 8, stream));
    SG_CUDA(cudaMemsetAsync(red_count, 0, 16, stream));
    SG_CUDA(cudaMemsetAsync(scal, 0, 32 * 8, stream));
    set_potential(-65.0, stream);  // efield.cpp:104 DEFAULT_MEMB_POT
    dirty = true;
    stats = EFieldStats();
}

// ---------------------------------------------------------------------------
// Device kernels
// ---------------------------------------------------------------------------
namespace {

constexpr int kBlock = 256;
// Device scalar slots.
enum { S_RZ = 0, S_PQ, S_ALPHA, S_BETA, S_RR, S_BB, S_DONE, S_ITER, S_TOL2, S_RZ0 };

__global__ void fill_kernel(double* v, int n, double x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = x;
}

// Per-vertex current and right-hand side of dVsolver.hpp:129-168.
__global__ void rhs_kernel(int n, int width, const double* V, const int32_t* col, const double* cc,
                           const double* cap_gext, double v_ext, const double* vclamp_cur,
                           const int32_t* vt_ptr, const int32_t* vt_idx, const double* tri_I,
                           const double* tri_clamp, const uint8_t* clamped, double* b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (clamped[i]) {
            b[i] = 0.0;
            continue;
        }
        double cur = vclamp_cur[i];
        for (int k = vt_ptr[i]; k < vt_ptr[i + 1]; ++k) {
            int t = vt_idx[k];
            cur += (-tri_I[t] + tri_clamp[t]) / 3.0;
        }
        double vi = V[i];
        double rhs = cur + cap_gext[n + i] * (v_ext - vi);
        for (int w = 0; w < width; ++w) {
            int j = col[(size_t)w * n + i];
            if (j < 0) break;
            rhs += cc[(size_t)w * n + i] * (V[j] - vi);
        }
        b[i] = rhs;
    }
}

// Fixed-order block reduction of NV values per thread: partials[blockIdx][k]; the last
// block to finish sums the partials in block order and calls fin(totals).
template <int NV, typename Fin>
__device__ void reduce_last(double (&v)[NV], double* partials, unsigned int* counter, Fin fin) {
    __shared__ double sh[NV][kBlock / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; ++k) {
            double s = 0.0;
            for (int w = 0; w < kBlock / 32; ++w) s += sh[k][w];
            partials[(size_t)blockIdx.x * NV + k] = s;
        }
        __threadfence();
        unsigned int prev = atomicAdd(counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x == 0) {
        __threadfence();
        double tot[NV];
        for (int k = 0; k < NV; ++k) tot[k] = 0.0;
        for (int blk = 0; blk < (int)gridDim.x; ++blk)
            for (int k = 0; k < NV; ++k) tot[k] += __ldcg(&partials[(size_t)blk * NV + k]);
        *counter = 0u;
        fin(tot);
    }
}

// q = A p (A = diag + off-diagonal ELL), partial p.q; last block: alpha = rz / pq.
template <typename T>
__global__ void spmv_dot_kernel(int n, int width, const int32_t* col, const T* a, const double* diag, const T* pv,
                                T* qv, double* partials, unsigned int* counter, double* scal) {
    if (scal[S_DONE] != 0.0) return;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T s = (T)diag[i] * pv[i];
        for (int w = 0; w < width; ++w) {
            int j = col[(size_t)w * n + i];
            if (j < 0) break;
            s += a[(size_t)w * n + i] * pv[j];
        }
        qv[i] = s;
        acc[0] += (double)pv[i] * (double)s;
    }
    reduce_last<1>(acc, partials, counter, [&](double* tot) {
        scal[S_PQ] = tot[0];
        scal[S_ALPHA] = (tot[0] != 0.0) ? scal[S_RZ] / tot[0] : 0.0;
    });
}

// x += alpha p; r -= alpha q; z = r / diag; partial r.z and r.r; last block: beta, convergence.
template <typename T>
__global__ void update_kernel(int n, const double* diag, T* xv, T* rv, T* zv, const T* pv, const T* qv,
                              double* partials, unsigned int* counter, double* scal, int max_iter) {
    if (scal[S_DONE] != 0.0) return;
    const T alpha = (T)scal[S_ALPHA];
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T xi = xv[i] + alpha * pv[i];
        T ri = rv[i] - alpha * qv[i];
        T zi = ri / (T)diag[i];
        xv[i] = xi;
        rv[i] = ri;
        zv[i] = zi;
        acc[0] += (double)ri * (double)zi;
        acc[1] += (double)ri * (double)ri;
    }
    reduce_last<2>(acc, partials, counter, [&](double* tot) {
        double rz_old = scal[S_RZ];
        scal[S_BETA] = (rz_old != 0.0) ? tot[0] / rz_old : 0.0;
        scal[S_RZ] = tot[0];
        scal[S_RR] = tot[1];
        scal[S_ITER] += 1.0;
        if (tot[1] <= scal[S_TOL2] || scal[S_ITER] >= (double)max_iter) scal[S_DONE] = 1.0;
    });
}

// p = z + beta p
template <typename T>
__global__ void direction_kernel(int n, const T* zv, T* pv, const double* scal) {
    if (scal[S_DONE] != 0.0) return;
    const T beta = (T)scal[S_BETA];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        pv[i] = zv[i] + beta * pv[i];
}

// Start of a CG solve of A x = rhs from x = 0: r = rhs, z = r / diag, p = z; r.z, r.r.
template <typename T>
__global__ void cg_start_kernel(int n, const double* diag, const T* rhs, T* xv, T* rv, T* zv, T* pv,
                                double* partials, unsigned int* counter, double* scal, double rel_tol) {
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        T ri = rhs[i];
        T zi = ri / (T)diag[i];
        xv[i] = (T)0;
        rv[i] = ri;
        zv[i] = zi;
        pv[i] = zi;
        acc[0] += (double)ri * (double)zi;
        acc[1] += (double)ri * (double)ri;
    }
    reduce_last<2>(acc, partials, counter, [&](double* tot) {
        scal[S_RZ] = tot[0];
        scal[S_RZ0] = tot[0];
        scal[S_RR] = tot[1];
        scal[S_BB] = tot[1];
        scal[S_TOL2] = rel_tol * rel_tol * tot[1];
        scal[S_ITER] = 0.0;
        scal[S_DONE] = (tot[1] <= 0.0) ? 1.0 : 0.0;
    });
}

// FP64 residual of the refinement loop: r64 = b - A x64, r32 = (float) r64, partial r.r.
__global__ void residual_kernel(int n, int width, const int32_t* col, const double* a, const double* diag,
                                const double* bv, const double* xv, double* rv, float* r32,
                                double* partials, unsigned int* counter, double* scal) {
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = diag[i] * xv[i];
        for (int w = 0; w < width; ++w) {
            int j = col[(size_t)w * n + i];
            if (j < 0) break;
            s += a[(size_t)w * n + i] * xv[j];
        }
        double ri = bv[i] - s;
        rv[i] = ri;
        r32[i] = (float)ri;
        acc[0] += ri * ri;
        acc[1] += bv[i] * bv[i];
    }
    reduce_last<2>(acc, partials, counter, [&](double* tot) {
        scal[S_RR] = tot[0];
        scal[S_BB] = tot[1];
    });
}

// Restart of FP64 CG from the residual r = b - A x0 of a warm start x0: z, p, r.z; the
// tolerance stays relative to |b| (set by residual_kernel).
__global__ void cg_restart_kernel(int n, const double* diag, const double* rv, double* zv, double* pv,
                                  double* partials, unsigned int* counter, double* scal, double rel_tol) {
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double zi = rv[i] / diag[i];
        zv[i] = zi;
        pv[i] = zi;
        acc[0] += rv[i] * zi;
    }
    reduce_last<1>(acc, partials, counter, [&](double* tot) {
        scal[S_RZ] = tot[0];
        scal[S_RZ0] = tot[0];
        scal[S_TOL2] = rel_tol * rel_tol * scal[S_BB];
        scal[S_ITER] = 0.0;
        scal[S_DONE] = (scal[S_RR] <= scal[S_TOL2]) ? 1.0 : 0.0;
    });
}

__global__ void add_correction_kernel(int n, double* xv, const float* d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) xv[i] += (double)d[i];
}

// V += dV on unclamped vertices; then triangle potentials (mean of the 3 vertices).
__global__ void apply_kernel(int n, double* V, const double* dv, const uint8_t* clamped) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!clamped[i]) V[i] += dv[i];
}

__global__ void tri_v_kernel(int nt, const int32_t* tv, const double* V, double* triV) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x)
        triV[t] = (V[tv[3 * t]] + V[tv[3 * t + 1]] + V[tv[3 * t + 2]]) / 3.0;
}

int grid_for(int n, int nsm) { return std::max(1, std::min((n + kBlock - 1) / kBlock, std::min(nsm * 8, 1024))); }

}  // namespace

void EFieldSystem::set_potential(double v_mV, cudaStream_t stream) {
    fill_kernel<<<grid_for(nverts, nsm), kBlock, 0, stream>>>(V, nverts, v_mV);
    SG_CUDA(cudaGetLastError());
    if (ntris) {
        fill_kernel<<<grid_for(ntris, nsm), kBlock, 0, stream>>>(tri_V, ntris, v_mV);
        SG_CUDA(cudaGetLastError());
    }
}

// A_ii = C_i/dt + g_i + sum_j cc_ij and A_ij = -cc_ij for unclamped rows and columns;
// clamped rows are identity rows (dVsolver.hpp:146-166).
void EFieldSystem::build_matrix(double dt_ms, cudaStream_t stream) {
    const int n = nverts;
    std::vector<int32_t> col((size_t)width * n, -1);
    std::vector<double> cc((size_t)width * n, 0.0), a64((size_t)width * n, 0.0), diag(n), cg(2 * (size_t)n);
    std::vector<float> a32((size_t)width * n, 0.0f);
    for (int i = 0; i < n; ++i) {
        double C = cm * vert_area_um2[i];
        double g = g_leak * vert_area_um2[i];
        cg[i] = C;
        cg[n + i] = g;
        double d = C / dt_ms + g;
        int w = 0;
        for (int k = nbr_ptr[i]; k < nbr_ptr[i + 1]; ++k, ++w) {
            double c = sigma * geo_cc[k];
            col[(size_t)w * n + i] = nbr_idx[k];  // RHS: every neighbour
            cc[(size_t)w * n + i] = c;
            d += c;
        }
        diag[i] = vclamped[i] ? 1.0 : d;
    }
    // Matrix columns: unclamped neighbours of unclamped rows, packed to the front.
    std::vector<int32_t> acol((size_t)width * n, -1);
    for (int i = 0; i < n; ++i) {
        if (vclamped[i]) continue;
        int wa = 0;
        for (int k = nbr_ptr[i]; k < nbr_ptr[i + 1]; ++k) {
            if (vclamped[nbr_idx[k]]) continue;
            double a = -sigma * geo_cc[k];
            acol[(size_t)wa * n + i] = nbr_idx[k];
            a64[(size_t)wa * n + i] = a;
            a32[(size_t)wa * n + i] = (float)a;
            ++wa;
        }
    }
    if (!acol_dev) dalloc(acol_dev, (size_t)width * n);
    SG_CUDA(cudaMemcpyAsync(ell_col, col.data(), col.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(acol_dev, acol.data(), acol.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(ell_cc, cc.data(), cc.size() * 8, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(ell_a64, a64.data(), a64.size() * 8, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(ell_a32, a32.data(), a32.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(diag64, diag.data(), diag.size() * 8, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(cap_gext, cg.data(), cg.size() * 8, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_vclamped, vclamped.data(), vclamped.size(), cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_vert_iclamp, vert_iclamp.data(), vert_iclamp.size() * 8, cudaMemcpyHostToDevice,
                            stream));
    if (ntris)
        SG_CUDA(cudaMemcpyAsync(d_tri_iclamp, tri_iclamp.data(), tri_iclamp.size() * 8, cudaMemcpyHostToDevice,
                                stream));
    SG_CUDA(cudaStreamSynchronize(stream));  // host vectors above are temporaries
    dt_built = dt_ms;
    dirty = false;
}

// One EField step: RHS from the current V and currents, CG solve, V update.
void EFieldSystem::advance(double dt_ms, cudaStream_t stream) {
    if (dirty || dt_ms != dt_built) build_matrix(dt_ms, stream);
    const int n = nverts;
    const int g = grid_for(n, nsm);
    SG_CUDA(cudaEventRecord(ev0, stream));
    rhs_kernel<<<g, kBlock, 0, stream>>>(n, width, V, ell_col, ell_cc, cap_gext, v_leak, d_vert_iclamp, d_vt_ptr,
                                         d_vt_idx, tri_I, d_tri_iclamp, d_vclamped, b);
    SG_CUDA(cudaGetLastError());
    const int chunk = 16;
    double h[10];
    if (method == EF_CG_FP64) {
        // Warm start from the previous step's dV (x keeps it).
        residual_kernel<<<g, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, red, red_count,
                                                  scal);
        cg_restart_kernel<<<g, kBlock, 0, stream>>>(n, diag64, r, z, p, red, red_count, scal, tol);
        for (int it = 0; it < max_iter; it += chunk) {
            for (int c = 0; c < chunk; ++c) {
                spmv_dot_kernel<double><<<g, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, p, q, red,
                                                                   red_count, scal);
                update_kernel<double><<<g, kBlock, 0, stream>>>(n, diag64, x, r, z, p, q, red, red_count, scal,
                                                                max_iter);
                direction_kernel<double><<<g, kBlock, 0, stream>>>(n, z, p, scal);
            }
            SG_CUDA(cudaGetLastError());
            SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
            SG_CUDA(cudaStreamSynchronize(stream));
            if (h[S_DONE] != 0.0) break;
        }
        stats.iterations += (uint64_t)h[S_ITER];
        stats.last_rel_residual = h[S_BB] > 0.0 ? std::sqrt(h[S_RR] / h[S_BB]) : 0.0;
        if (h[S_BB] > 0.0 && h[S_RR] > h[S_TOL2]) throw DeviceErr("EField CG did not converge");
    } else {
        // Mixed precision: FP32 CG on the correction, FP64 residuals and accumulation,
        // warm-started from the previous step's dV.
        residual_kernel<<<g, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, red, red_count,
                                                  scal);
        SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
        SG_CUDA(cudaStreamSynchronize(stream));
        const double bb = h[S_BB];
        double rr = h[S_RR];
        int outer = 0;
        while (bb > 0.0 && rr > tol * tol * bb && outer < 50) {
            // Inner FP32 solve of A d = r32: s32 is its residual, q32 = A p32.
            cg_start_kernel<float><<<g, kBlock, 0, stream>>>(n, diag64, r32, x32, s32, z32, p32, red, red_count, scal,
                                                             inner_tol);
            for (int it = 0; it < max_iter; it += chunk) {
                for (int c = 0; c < chunk; ++c) {
                    spmv_dot_kernel<float><<<g, kBlock, 0, stream>>>(n, width, acol_dev, ell_a32, diag64, p32, q32,
                                                                     red, red_count, scal);
                    update_kernel<float><<<g, kBlock, 0, stream>>>(n, diag64, x32, s32, z32, p32, q32, red,
                                                                   red_count, scal, max_iter);
                    direction_kernel<float><<<g, kBlock, 0, stream>>>(n, z32, p32, scal);
                }
                SG_CUDA(cudaGetLastError());
                SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
                SG_CUDA(cudaStreamSynchronize(stream));
                if (h[S_DONE] != 0.0) break;
            }
            stats.iterations += (uint64_t)h[S_ITER];
            add_correction_kernel<<<g, kBlock, 0, stream>>>(n, x, x32);
            residual_kernel<<<g, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, red,
                                                      red_count, scal);
            SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
            SG_CUDA(cudaStreamSynchronize(stream));
            rr = h[S_RR];
            stats.refinements += 1;
            ++outer;
        }
        stats.last_rel_residual = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
        if (bb > 0.0 && rr > tol * tol * bb) throw DeviceErr("EField refinement did not converge");
    }
    apply_kernel<<<g, kBlock, 0, stream>>>(n, V, x, d_vclamped);
    if (ntris) tri_v_kernel<<<grid_for(ntris, nsm), kBlock, 0, stream>>>(ntris, d_tri_verts, V, tri_V);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaEventRecord(ev1, stream));
    SG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    SG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    stats.solve_ms += ms;
    stats.steps += 1;
}

}  // namespace sg
