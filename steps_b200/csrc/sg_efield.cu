// EField membrane-potential solve (see sg_efield.h for the equations and units).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <tuple>
#include <type_traits>
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
    dfree(alt_diag64);
    dfree(alt_einv64);
    dfree(alt_einv32);
    alt_dt = -1.0;
    dfree(cap_gext);
    dfree(d_vclamped);
    dfree(b);
    dfree(x);
    dfree(r);
    dfree(z);
    dfree(p);
    dfree(p2);
    dfree(q);
    dfree(r32);
    dfree(z32);
    dfree(p32);
    dfree(p2_32);
    dfree(q32);
    dfree(x32);
    dfree(s32);
    dfree(xchk);
    dfree(acol_dev);
    dfree(d_agg);
    dfree(d_agg_base);
    dfree(d_agg_len);
    dfree(d_agg_row);
    einv_len = 0;
    dfree(d_seg_ptr);
    dfree(d_seg_idx);
    dfree(d_seg_agg);
    nseg = 0;
    dfree(d_einv64);
    dfree(d_einv32);
    dfree(d_c64);
    dfree(d_c32);
    nagg = 0;
    dfree(red);
    dfree(scal);
    dfree(red_count);
    dfree(d_bar);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evc0) cudaEventDestroy(evc0);
    if (evc1) cudaEventDestroy(evc1);
    ev0 = ev1 = evc0 = evc1 = nullptr;
}

EFieldSystem::~EFieldSystem() { release(); }

static std::vector<int32_t> aggregate_order(int nv, const double* X, int ntet, const int32_t* tets);

void EFieldSystem::setup(int nv, const double* verts_um, int ntet, const int32_t* tets, int nt,
                         const int32_t* tris, cudaStream_t stream, int nsm_) {
    if (nv <= 0) throw ArgErr("EField needs vertices");
    for (size_t k = 0; k < (size_t)nt * 3; ++k)
        if (tris[k] < 0 || tris[k] >= nv) throw ArgErr("triangle vertex index out of range");
    std::vector<int32_t> perm = aggregate_order(nv, verts_um, ntet, tets);
    std::vector<double> X((size_t)nv * 3);
    for (int v = 0; v < nv; ++v)
        for (int c = 0; c < 3; ++c) X[(size_t)perm[v] * 3 + c] = verts_um[(size_t)v * 3 + c];
    std::vector<int32_t> tv((size_t)ntet * 4), rv((size_t)nt * 3);
    for (size_t k = 0; k < tv.size(); ++k) tv[k] = perm[tets[k]];
    for (size_t k = 0; k < rv.size(); ++k) rv[k] = perm[tris[k]];
    setup_ordered(nv, X.data(), ntet, tv.data(), nt, rv.data(), stream, nsm_);
    vperm = std::move(perm);
}

void EFieldSystem::setup_ordered(int nv, const double* verts_um, int ntet, const int32_t* tets, int nt,
                                 const int32_t* tris, cudaStream_t stream, int nsm_) {
    nsm = nsm_;
    nverts = nv;
    ntris = nt;
    efield_couple(nv, verts_um, ntet, tets, nbr_ptr, nbr_idx, geo_cc);
    this->verts_um.assign(verts_um, verts_um + (size_t)nv * 3);
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
    // Connected components of the vertex graph (batched realizations are disjoint copies).
    {
        std::vector<int32_t> comp(nv, -1), stack;
        comp_verts.clear();
        for (int s0 = 0; s0 < nv; ++s0) {
            if (comp[s0] >= 0) continue;
            const int c = (int)comp_verts.size();
            comp_verts.emplace_back();
            comp[s0] = c;
            stack.assign(1, s0);
            while (!stack.empty()) {
                const int v = stack.back();
                stack.pop_back();
                comp_verts[c].push_back(v);
                for (int k = nbr_ptr[v]; k < nbr_ptr[v + 1]; ++k)
                    if (comp[nbr_idx[k]] < 0) {
                        comp[nbr_idx[k]] = c;
                        stack.push_back(nbr_idx[k]);
                    }
            }
            std::sort(comp_verts[c].begin(), comp_verts[c].end());
        }
        ncomp_v = (int)comp_verts.size();
    }
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
    dalloc(p2, nv);
    dalloc(q, nv);
    dalloc(r32, nv);
    dalloc(z32, nv);
    dalloc(p32, nv);
    dalloc(p2_32, nv);
    dalloc(q32, nv);
    dalloc(x32, nv);
    dalloc(s32, nv);
    dalloc(red, 8192);
    dalloc(scal, 32);
    dalloc(red_count, 4);
    dalloc(d_bar, 4);
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
enum { S_RZ = 0, S_PQ, S_ALPHA, S_BETA, S_RR, S_BB, S_DONE, S_ITER, S_TOL2, S_RZ0, S_CHK, S_NRU };
constexpr int kScalOut = 12;  // device scalars copied back after a solve (S_RZ .. S_NRU)

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
    // The whole last block sums the block partials: thread t takes blocks t, t + kBlock, ...
    // in order, then a fixed shuffle tree and the warps in order (deterministic).
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int blk = threadIdx.x; blk < (int)gridDim.x; blk += kBlock)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(size_t)blk * NV + k]);
    __syncthreads();  // sh is reused below
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = acc[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[NV];
        for (int k = 0; k < NV; ++k) {
            tot[k] = 0.0;
            for (int w = 0; w < kBlock / 32; ++w) tot[k] += sh[k][w];
        }
        *counter = 0u;
        fin(tot);
    }
}

// Direction and product in one pass: p' = z + beta p (computed for the row and for every
// neighbour it reads, so no separate direction kernel), q = A p' with A = diag + ELL,
// partial p'.q; last block: alpha = rz / pq.  p' goes to pout (p is double-buffered).
template <typename T>
__global__ void spmv_kernel(int n, int width, const int32_t* col, const T* a, const double* diag, const T* zv,
                            const T* pin, T* pout, T* qv, double* partials, unsigned int* counter, double* scal) {
    if (scal[S_DONE] != 0.0) return;
    const T beta = (T)scal[S_BETA];
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T pi = zv[i] + beta * pin[i];
        T s = (T)diag[i] * pi;
        // Padding (-1) is skipped per entry rather than ending the loop, so the unrolled
        // column and neighbour loads are all in flight together.
#pragma unroll 4
        for (int w = 0; w < width; ++w) {
            const int j = col[(size_t)w * n + i];
            if (j >= 0) s += a[(size_t)w * n + i] * (zv[j] + beta * pin[j]);
        }
        pout[i] = pi;
        qv[i] = s;
        acc[0] += (double)pi * (double)s;
    }
    reduce_last<1>(acc, partials, counter, [&](double* tot) {
        scal[S_PQ] = tot[0];
        scal[S_ALPHA] = (tot[0] != 0.0) ? scal[S_RZ] / tot[0] : 0.0;
    });
}

// Vertex segments: segment sg lists the vertices seg_idx[seg_ptr[sg] .. seg_ptr[sg + 1]) of
// aggregate seg_agg[sg] in ascending order (-1: vertices in no aggregate).  One warp walks
// a segment and writes its restriction c[agg] = sum of r with a fixed shuffle tree, so the
// coarse right-hand side is the same in every run (no floating-point atomics).
struct Segs {
    int n;
    const int32_t* ptr;
    const int32_t* idx;
    const int32_t* agg;
};

template <typename T>
__device__ __forceinline__ void seg_store(const Segs& sg, int k, T c, T* cvec) {
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    const int ag = sg.agg[k];
    if ((threadIdx.x & 31) == 0 && ag >= 0 && cvec) cvec[ag] = c;
}

// x += alpha p; r -= alpha q; restriction c = Z^T r; partial r.r; last block: convergence.
template <typename T>
__global__ void update_kernel(Segs sg, T* xv, T* rv, const T* pv, const T* qv, T* cvec, double* partials,
                              unsigned int* counter, double* scal, int max_iter) {
    if (scal[S_DONE] != 0.0) return;
    const T alpha = (T)scal[S_ALPHA];
    const int lane = threadIdx.x & 31;
    double acc[1] = {0.0};
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < sg.n; k += (gridDim.x * blockDim.x) >> 5) {
        T c = (T)0;
        for (int m = sg.ptr[k] + lane; m < sg.ptr[k + 1]; m += 32) {
            const int i = sg.idx[m];
            T xi = xv[i] + alpha * pv[i];
            T ri = rv[i] - alpha * qv[i];
            xv[i] = xi;
            rv[i] = ri;
            c += ri;
            acc[0] += (double)ri * (double)ri;
        }
        seg_store(sg, k, c, cvec);
    }
    reduce_last<1>(acc, partials, counter, [&](double* tot) {
        scal[S_RR] = tot[0];
        scal[S_ITER] += 1.0;
        if (tot[0] <= scal[S_TOL2] || scal[S_ITER] >= (double)max_iter) scal[S_DONE] = 1.0;
    });
}

// Solve start from x = 0 with right-hand side rhs: r = rhs, restriction, r.r (= rhs.rhs).
template <typename T>
__global__ void init_kernel(Segs sg, const T* rhs, T* xv, T* rv, T* cvec, double* partials, unsigned int* counter,
                            double* scal, double rel_tol) {
    const int lane = threadIdx.x & 31;
    double acc[1] = {0.0};
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < sg.n; k += (gridDim.x * blockDim.x) >> 5) {
        T c = (T)0;
        for (int m = sg.ptr[k] + lane; m < sg.ptr[k + 1]; m += 32) {
            const int i = sg.idx[m];
            T ri = rhs[i];
            xv[i] = (T)0;
            rv[i] = ri;
            c += ri;
            acc[0] += (double)ri * (double)ri;
        }
        seg_store(sg, k, c, cvec);
    }
    reduce_last<1>(acc, partials, counter, [&](double* tot) {
        scal[S_RR] = tot[0];
        scal[S_BB] = tot[0];
        scal[S_TOL2] = rel_tol * rel_tol * tot[0];
        scal[S_ITER] = 0.0;
        scal[S_DONE] = (tot[0] <= 0.0) ? 1.0 : 0.0;
    });
}

// Coarse inverse layout: one dense block per connected component; aggregate a's row
// starts at row[a] and spans the len[a] aggregates of its component, base[a] the first.
struct Coarse {
    const int32_t* base;
    const int32_t* len;
    const long long* row;
};

// Two-level preconditioner, one warp per vertex segment: the warp of aggregate a forms
// y_a = (E^-1 c)_a (row a of the component's dense coarse inverse times the restricted
// residual of that component) and
// sets z = r / diag + y_a on the aggregate's vertices; vertices in no aggregate get
// z = r / diag.  Partial r.z; last block: beta = r.z / previous r.z (0 at the start of a
// solve, where p = z is also written as the first direction).
// Row `row` of a component's coarse inverse times the component's restricted residual
// `cb` (len entries), summed over the warp: four independent accumulators per lane so
// that eight loads are in flight, combined and shuffled in a fixed order.
template <typename T>
__device__ __forceinline__ T coarse_row_dot(const T* row, const T* cb, int len, int lane) {
    T y0 = (T)0, y1 = (T)0, y2 = (T)0, y3 = (T)0;
    int j = lane;
    for (; j + 96 < len; j += 128) {
        y0 += __ldg(&row[j]) * __ldcg(&cb[j]);
        y1 += __ldg(&row[j + 32]) * __ldcg(&cb[j + 32]);
        y2 += __ldg(&row[j + 64]) * __ldcg(&cb[j + 64]);
        y3 += __ldg(&row[j + 96]) * __ldcg(&cb[j + 96]);
    }
    for (; j < len; j += 32) y0 += __ldg(&row[j]) * __ldcg(&cb[j]);
    T y = (y0 + y1) + (y2 + y3);
    for (int o = 16; o > 0; o >>= 1) y += __shfl_down_sync(0xffffffffu, y, o);
    return __shfl_sync(0xffffffffu, y, 0);
}

template <typename T>
__global__ void precond_kernel(Segs sg, Coarse cs, const double* diag, const T* rv, T* zv, T* pv, const T* einv,
                               const T* cvec, double* partials, unsigned int* counter, double* scal, int start) {
    if (scal[S_DONE] != 0.0 && !start) return;
    const int lane = threadIdx.x & 31;
    double acc[1] = {0.0};
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < sg.n; k += (gridDim.x * blockDim.x) >> 5) {
        const int ag = sg.agg[k];
        T y = (T)0;
        if (ag >= 0) {
            y = coarse_row_dot(einv + cs.row[ag], cvec + cs.base[ag], cs.len[ag], lane);
        }
        for (int m = sg.ptr[k] + lane; m < sg.ptr[k + 1]; m += 32) {
            const int i = sg.idx[m];
            const T ri = rv[i];
            const T zi = ri / (T)diag[i] + y;
            zv[i] = zi;
            if (start) pv[i] = zi;
            acc[0] += (double)ri * (double)zi;
        }
    }
    reduce_last<1>(acc, partials, counter, [&](double* tot) {
        if (start) {
            scal[S_BETA] = 0.0;
            if (scal[S_RR] <= scal[S_TOL2]) scal[S_DONE] = 1.0;
        } else {
            double rz_old = scal[S_RZ];
            scal[S_BETA] = (rz_old != 0.0) ? tot[0] / rz_old : 0.0;
        }
        scal[S_RZ] = tot[0];
    });
}

// ---------------------------------------------------------------------------
// The whole PCG solve in one cooperative launch (all blocks co-resident): the three
// phases of an iteration are separated by grid barriers instead of kernel boundaries,
// and each scalar (p.q, r.r, r.z) is reduced by every block from the same block
// partials in the same order, so all blocks take identical decisions without a second
// barrier.  Vectors written by other blocks inside the launch are read with __ldcg (L2),
// never from a stale L1 line.  The barrier waits are bounded: a block that waits longer
// than the solve's poll limit (kSpinLimit unless set otherwise) sets bar[2] and every block
// leaves at its next barrier.
// ---------------------------------------------------------------------------
constexpr unsigned int kSpinLimit = 1u << 22;  // x ~100 ns polls: about half a second
// The persistent solve is launched with at most 2048 blocks (3 x 2048 reduction partials
// fit the 8192-value buffer); a 32-register bound keeps 8 blocks of 256 per SM resident.

// GPU-scope acquire/release accesses of the barrier words.  __syncthreads orders the
// block's writes before thread 0's release (releases are cumulative), and the block reads
// other blocks' writes only after thread 0's acquire and the closing __syncthreads.
__device__ __forceinline__ unsigned int atom_add_acq_rel_gpu(unsigned int* p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks, unsigned int& gen,
                                             unsigned int limit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int g = gen;
        if (atom_add_acq_rel_gpu(&bar[0], 1u) == nblocks - 1u) {
            bar[0] = 0u;  // nobody arrives at the next barrier before the release below
            st_release_gpu(&bar[1], g + 1u);
        } else {
            unsigned int spins = 0;
            while (ld_acquire_gpu(&bar[1]) == g) {
                if (++spins > limit) {
                    atomicOr(&bar[2], 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
    }
    __syncthreads();
    gen += 1u;
    return *(volatile unsigned int*)&bar[2] == 0u;
}

// Block partial of v -> partials[blockIdx]; barrier; the sum over all blocks in block
// order (thread-strided, fixed shuffle tree, warps in order), the same in every block.
__device__ __forceinline__ bool grid_sum(double v, double* partials, unsigned int* bar, unsigned int& gen,
                                         unsigned int limit, double* out) {
    __shared__ double sh[kBlock / 32];
    __shared__ double tot;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) s += sh[w];
        partials[blockIdx.x] = s;
    }
    if (!grid_barrier(bar, gridDim.x, gen, limit)) return false;
    double a = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) a += __ldcg(&partials[b]);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) sh[wid] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) s += sh[w];
        tot = s;
    }
    __syncthreads();
    *out = tot;
    __syncthreads();  // sh and tot are reused by the next call
    return true;
}

template <typename T>
struct PcgArgs {
    int n, width, max_iter;
    Coarse cs;
    const int32_t* col;
    const T* a;
    const double* diag;
    const T* einv;
    Segs sg;
    T *x, *r, *z, *p, *p2, *q, *c;
    double* partials;  // [3][gridDim]
    double* scal;
    unsigned int* bar;  // count, generation, error
    unsigned int spin_limit;  // polls of a barrier wait before the solve gives up
    // Reliable updates (FP32 solve of the FP64 system, T = float only): x is the FP32
    // correction accumulated since the last update; when the FP32 residual norm has fallen
    // by delta2 from its largest value since the last update (or below tol2_64), x64 += x,
    // x = 0 and r is replaced by the FP64 residual b - A64 x64 (rounded to FP32); the solve
    // ends when that FP64 residual meets tol2_64.  The search direction is kept.
    int ru;
    double delta2, tol2_64;
    const double* a64;
    const double* b64;
    double* x64;
    double* r64;
};

constexpr int kSegPass = 4;   // segments per block per preconditioner pass
constexpr int kEllFast = 16;  // ELL widths up to this take the fully unrolled SpMV row
constexpr int kMinbSmall = 3; // blocks per SM of the latency-bound (one-pass) solve

// Two-level PCG from a started state (r and its restriction c set, scal[S_RR], scal[S_TOL2]
// set).  The same algorithm as the multi-kernel loop (z = r / d + y, p' = z + beta p,
// q = A p', x += alpha p', r -= alpha q); sums run in a different order.
// MINB: resident blocks per SM the kernel is compiled for.  kMinbSmall (85 registers) for
// systems that fit in one pass of the grid, where every phase is latency-bound: the SpMV row is
// fully unrolled and the preconditioner is block-cooperative.  8 for larger systems
// (bandwidth-bound SpMV, many segments per block): a warp per segment.
template <typename T, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) pcg_persistent_kernel(PcgArgs<T> P) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    const unsigned int G = gridDim.x;
    unsigned int gen = *(volatile unsigned int*)&P.bar[1];
    double* part0 = P.partials;
    double* part1 = P.partials + G;
    double* part2 = P.partials + 2 * G;
    double rr = __ldcg(&P.scal[S_RR]);
    const double tol2 = P.ru ? P.tol2_64 : __ldcg(&P.scal[S_TOL2]);
    double rz = 0.0, beta = 0.0, rmax2 = rr;
    int iter = 0, nru = 0;
    bool ok = true;

    // Phase C: z = M^-1 r (p = z at the start), r.z.  Block-cooperative: a pass takes the
    // segments k = k0 + i G (i < kSegPass) of this block; the whole block forms their
    // coarse values y = (E^-1 c)[aggregate] together (thread t sums the row entries t,
    // t + kBlock, ... in order, then a fixed shuffle tree and the warps in order, so y does
    // not depend on the grid) with every segment's loads in flight at once, then applies
    // z = r / d + y to the segments' vertices.
    __shared__ T sy[kSegPass][kBlock / 32];
    const int wid = threadIdx.x >> 5;
    auto precond = [&](bool start) -> double {
        double acc = 0.0;
        const int nseg = P.sg.n;
        if (MINB > kMinbSmall || nseg > (int)G * kSegPass) {
            // A warp per segment (coarse row dot by the warp).
            for (int k = gw; k < nseg; k += nw) {
                const int ag = __ldg(&P.sg.agg[k]);
                T y = (T)0;
                if (ag >= 0)
                    y = coarse_row_dot(P.einv + __ldg(&P.cs.row[ag]), P.c + __ldg(&P.cs.base[ag]),
                                       __ldg(&P.cs.len[ag]), lane);
                const int m1 = __ldg(&P.sg.ptr[k + 1]);
                for (int m = __ldg(&P.sg.ptr[k]) + lane; m < m1; m += 32) {
                    const int iv = __ldg(&P.sg.idx[m]);
                    const T ri = __ldcg(&P.r[iv]);
                    const T zi = ri / (T)__ldg(&P.diag[iv]) + y;
                    P.z[iv] = zi;
                    if (start) P.p[iv] = zi;
                    acc += (double)ri * (double)zi;
                }
            }
            return acc;
        }
        for (int k0 = blockIdx.x; k0 < nseg; k0 += (int)G * kSegPass) {
            const T* rw[kSegPass];
            const T* cb[kSegPass];
            int len[kSegPass];
            int lmax = 0;
#pragma unroll
            for (int i = 0; i < kSegPass; ++i) {
                const int k = k0 + i * (int)G;
                const int ag = (k < nseg) ? __ldg(&P.sg.agg[k]) : -1;
                len[i] = (ag >= 0) ? __ldg(&P.cs.len[ag]) : 0;
                rw[i] = (ag >= 0) ? P.einv + __ldg(&P.cs.row[ag]) : P.einv;
                cb[i] = (ag >= 0) ? P.c + __ldg(&P.cs.base[ag]) : P.c;
                lmax = max(lmax, len[i]);
            }
            T part[kSegPass];
#pragma unroll
            for (int i = 0; i < kSegPass; ++i) part[i] = (T)0;
#pragma unroll 2
            for (int j = threadIdx.x; j < lmax; j += kBlock) {
#pragma unroll
                for (int i = 0; i < kSegPass; ++i)
                    if (j < len[i]) part[i] += __ldg(&rw[i][j]) * __ldcg(&cb[i][j]);
            }
#pragma unroll
            for (int i = 0; i < kSegPass; ++i) {
                T v = part[i];
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) sy[i][wid] = v;
            }
            __syncthreads();
            T y[kSegPass];
#pragma unroll
            for (int i = 0; i < kSegPass; ++i) {
                T v = (T)0;
                for (int w = 0; w < kBlock / 32; ++w) v += sy[i][w];
                y[i] = v;
            }
            __syncthreads();  // sy is rewritten by the next pass
#pragma unroll
            for (int i = 0; i < kSegPass; ++i) {
                const int k = k0 + i * (int)G;
                if (k >= nseg) break;
                const int m1 = __ldg(&P.sg.ptr[k + 1]);
                for (int m = __ldg(&P.sg.ptr[k]) + threadIdx.x; m < m1; m += kBlock) {
                    const int iv = __ldg(&P.sg.idx[m]);
                    const T ri = __ldcg(&P.r[iv]);
                    const T zi = ri / (T)__ldg(&P.diag[iv]) + y[i];
                    P.z[iv] = zi;
                    if (start) P.p[iv] = zi;
                    acc += (double)ri * (double)zi;
                }
            }
        }
        return acc;
    };

    if (rr > tol2) {
        double v = precond(true);
        ok = grid_sum(v, part0, P.bar, gen, P.spin_limit, &rz);
        T* pin = P.p;
        T* pout = P.p2;
        while (ok) {
            // Phase A: p' = z + beta p, q = A p', p'.q.
            const T bt = (T)beta;
            double acc = 0.0;
            for (int i = gt; i < P.n; i += nt) {
                const T pi = __ldcg(&P.z[i]) + bt * __ldcg(&pin[i]);
                T s = (T)__ldg(&P.diag[i]) * pi;
                if (MINB <= kMinbSmall && P.width <= kEllFast) {
                    // All column indices first, then every gather: two dependent rounds.
                    int jv[kEllFast];
#pragma unroll
                    for (int w = 0; w < kEllFast; ++w) jv[w] = (w < P.width) ? __ldg(&P.col[(size_t)w * P.n + i]) : -1;
#pragma unroll
                    for (int w = 0; w < kEllFast; ++w) {
                        const int j = jv[w];
                        if (j >= 0) s += __ldg(&P.a[(size_t)w * P.n + i]) * (__ldcg(&P.z[j]) + bt * __ldcg(&pin[j]));
                    }
                } else {
#pragma unroll 4
                    for (int w = 0; w < P.width; ++w) {
                        const int j = __ldg(&P.col[(size_t)w * P.n + i]);
                        if (j >= 0) s += __ldg(&P.a[(size_t)w * P.n + i]) * (__ldcg(&P.z[j]) + bt * __ldcg(&pin[j]));
                    }
                }
                pout[i] = pi;
                P.q[i] = s;
                acc += (double)pi * (double)s;
            }
            double pq = 0.0;
            if (!(ok = grid_sum(acc, part1, P.bar, gen, P.spin_limit, &pq))) break;
            const T alpha = (T)((pq != 0.0) ? rz / pq : 0.0);
            // Phase B: x += alpha p', r -= alpha q, restriction c, r.r.
            acc = 0.0;
            for (int k = gw; k < P.sg.n; k += nw) {
                T cs = (T)0;
                const int m1 = __ldg(&P.sg.ptr[k + 1]);
                for (int m = __ldg(&P.sg.ptr[k]) + lane; m < m1; m += 32) {
                    const int i = __ldg(&P.sg.idx[m]);
                    const T xi = __ldcg(&P.x[i]) + alpha * __ldcg(&pout[i]);
                    const T ri = __ldcg(&P.r[i]) - alpha * __ldcg(&P.q[i]);
                    P.x[i] = xi;
                    P.r[i] = ri;
                    cs += ri;
                    acc += (double)ri * (double)ri;
                }
                for (int o = 16; o > 0; o >>= 1) cs += __shfl_down_sync(0xffffffffu, cs, o);
                const int ag = __ldg(&P.sg.agg[k]);
                if (lane == 0 && ag >= 0) P.c[ag] = cs;
            }
            if (!(ok = grid_sum(acc, part2, P.bar, gen, P.spin_limit, &rr))) break;
            ++iter;
            if constexpr (std::is_same<T, float>::value) {
                if (P.ru) {
                    rmax2 = fmax(rmax2, rr);
                    if (rr <= P.delta2 * rmax2 || rr <= P.tol2_64 || iter >= P.max_iter) {
                        // Reliable update: fold the correction into x64, FP64 residual.
                        for (int i = gt; i < P.n; i += nt) {
                            P.x64[i] += (double)__ldcg(&P.x[i]);
                            P.x[i] = 0.0f;
                        }
                        if (!(ok = grid_barrier(P.bar, G, gen, P.spin_limit))) break;
                        double acc64 = 0.0;
                        for (int k = gw; k < P.sg.n; k += nw) {
                            float cs = 0.0f;
                            const int m1 = __ldg(&P.sg.ptr[k + 1]);
                            for (int m = __ldg(&P.sg.ptr[k]) + lane; m < m1; m += 32) {
                                const int i = __ldg(&P.sg.idx[m]);
                                double sx = __ldg(&P.diag[i]) * __ldcg(&P.x64[i]);
                                for (int w = 0; w < P.width; ++w) {
                                    const int j = __ldg(&P.col[(size_t)w * P.n + i]);
                                    if (j >= 0) sx += __ldg(&P.a64[(size_t)w * P.n + i]) * __ldcg(&P.x64[j]);
                                }
                                const double ri = __ldg(&P.b64[i]) - sx;
                                P.r64[i] = ri;
                                const float r32 = (float)ri;
                                P.r[i] = r32;
                                cs += r32;
                                acc64 += ri * ri;
                            }
                            for (int o = 16; o > 0; o >>= 1) cs += __shfl_down_sync(0xffffffffu, cs, o);
                            const int ag = __ldg(&P.sg.agg[k]);
                            if (lane == 0 && ag >= 0) P.c[ag] = cs;
                        }
                        if (!(ok = grid_sum(acc64, part2, P.bar, gen, P.spin_limit, &rr))) break;
                        ++nru;
                        rmax2 = rr;
                        if (rr <= P.tol2_64 || iter >= P.max_iter) break;
                    }
                } else if (rr <= tol2 || iter >= P.max_iter) {
                    break;
                }
            } else {
                if (rr <= tol2 || iter >= P.max_iter) break;
            }
            // Phase C: z = M^-1 r, r.z, beta.
            double rzn = 0.0;
            if (!(ok = grid_sum(precond(false), part0, P.bar, gen, P.spin_limit, &rzn))) break;
            beta = (rz != 0.0) ? rzn / rz : 0.0;
            rz = rzn;
            T* tp = pin;
            pin = pout;
            pout = tp;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.scal[S_RR] = rr;
        P.scal[S_ITER] = (double)iter;
        P.scal[S_RZ] = rz;
        P.scal[S_DONE] = 1.0;
        P.scal[S_NRU] = (double)nru;
    }
}

// FP64 residual r64 = b - A x64 (warm starts and the refinement loop), r32 = (float) r64,
// optional restriction into cvec; partial r.r and b.b.
__global__ void residual_kernel(int n, int width, const int32_t* col, const double* a, const double* diag,
                                const double* bv, const double* xv, double* rv, float* r32, Segs sg, double* cvec,
                                double* partials, unsigned int* counter, double* scal) {
    const int lane = threadIdx.x & 31;
    double acc[2] = {0.0, 0.0};
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < sg.n; k += (gridDim.x * blockDim.x) >> 5) {
        double c = 0.0;
        for (int m = sg.ptr[k] + lane; m < sg.ptr[k + 1]; m += 32) {
            const int i = sg.idx[m];
            double s = diag[i] * xv[i];
#pragma unroll 4
            for (int w = 0; w < width; ++w) {
                const int j = col[(size_t)w * n + i];
                if (j >= 0) s += a[(size_t)w * n + i] * xv[j];
            }
            double ri = bv[i] - s;
            rv[i] = ri;
            r32[i] = (float)ri;
            c += ri;
            acc[0] += ri * ri;
            acc[1] += bv[i] * bv[i];
        }
        seg_store(sg, k, c, cvec);
    }
    reduce_last<2>(acc, partials, counter, [&](double* tot) {
        scal[S_RR] = tot[0];
        scal[S_BB] = tot[1];
    });
}

// Tolerance and counters of an FP64 solve warm-started by residual_kernel.
__global__ void warm_start_kernel(double* scal, double rel_tol) {
    scal[S_TOL2] = rel_tol * rel_tol * scal[S_BB];
    scal[S_ITER] = 0.0;
    scal[S_DONE] = (scal[S_BB] <= 0.0) ? 1.0 : 0.0;
}

__global__ void add_correction_kernel(int n, double* xv, const float* d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) xv[i] += (double)d[i];
}

// Check of a mixed-precision step: max over unclamped vertices of |dV - dV64| / |V + dV64|
// into scal[S_CHK] (non-negative doubles order like their bit patterns, so the max is an
// integer atomic and independent of thread order).
__global__ void check_kernel(int n, const double* V, const double* dv, const double* dv64, const uint8_t* clamped,
                             double* scal) {
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (clamped[i]) continue;
        double ref = fabs(V[i] + dv64[i]);
        double e = fabs(dv[i] - dv64[i]);
        double rel = ref > 0.0 ? e / ref : e;
        m = rel > m ? rel : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double y = __shfl_down_sync(0xffffffffu, m, o);
        m = y > m ? y : m;
    }
    if ((threadIdx.x & 31) == 0 && m > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(&scal[S_CHK]), (unsigned long long)__double_as_longlong(m));
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

// In-place inverse of a dense SPD matrix through its Cholesky factor (row-major n x n).
static void spd_inverse(int n, std::vector<double>& E) {
    std::vector<double> L((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double s = E[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(s > 0.0)) throw DeviceErr("EField coarse matrix is not positive definite");
        double d = std::sqrt(s);
        L[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double t = E[(size_t)i * n + j];
            const double* li = &L[(size_t)i * n];
            const double* lj = &L[(size_t)j * n];
            for (int k = 0; k < j; ++k) t -= li[k] * lj[k];
            L[(size_t)i * n + j] = t / d;
        }
    }
    // W = L^-1 (lower triangular), then E^-1 = W^T W.
    std::vector<double> W((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        W[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
        for (int i = j + 1; i < n; ++i) {
            double t = 0.0;
            for (int k = j; k < i; ++k) t -= L[(size_t)i * n + k] * W[(size_t)k * n + j];
            W[(size_t)i * n + j] = t / L[(size_t)i * n + i];
        }
    }
    for (int a = 0; a < n; ++a)
        for (int b = a; b < n; ++b) {
            double t = 0.0;
            for (int k = b; k < n; ++k) t += W[(size_t)k * n + a] * W[(size_t)k * n + b];
            E[(size_t)a * n + b] = t;
            E[(size_t)b * n + a] = t;
        }
}

// Coarse bins of one connected component: its bounding box cut into bins of about
// `target` vertices (bins per axis in proportion to the box's extent); lin[q] is the
// linear bin index of verts[q].
static void component_bins(const std::vector<int32_t>& verts, const double* X, int target, std::vector<long>& lin) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i : verts)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], X[(size_t)i * 3 + c]);
            hi[c] = std::max(hi[c], X[(size_t)i * 3 + c]);
        }
    double ext[3], vol = 1.0;
    for (int c = 0; c < 3; ++c) {
        ext[c] = std::max(hi[c] - lo[c], 1e-12);
        vol *= ext[c];
    }
    double k = std::max(1.0, (double)verts.size() / target);
    double s = std::cbrt(vol / k);
    long nb[3];
    for (int c = 0; c < 3; ++c) nb[c] = std::max(1L, (long)std::llround(ext[c] / s));
    lin.resize(verts.size());
    for (size_t q = 0; q < verts.size(); ++q) {
        const int i = verts[q];
        long id[3];
        for (int c = 0; c < 3; ++c)
            id[c] = std::min(nb[c] - 1, (long)((X[(size_t)i * 3 + c] - lo[c]) / ext[c] * nb[c]));
        lin[q] = id[0] + nb[0] * (id[1] + nb[1] * id[2]);
    }
}

// Vertices per aggregate a component of n vertices is cut into (about 1000 aggregates).
static int aggregate_target(size_t n) { return std::max(16, (int)(n / 1000)); }

// Aggregates of one connected component: its occupied coarse bins, clamped vertices in
// none.  Aggregate ids start at `base`; returns how many this component has.
static int make_aggregates(const std::vector<int32_t>& verts, const std::vector<double>& X,
                           const std::vector<uint8_t>& clamped, int target, int base, std::vector<int32_t>& agg) {
    std::vector<long> lin, keys;
    component_bins(verts, X.data(), target, lin);
    for (size_t q = 0; q < verts.size(); ++q)
        if (!clamped[verts[q]]) keys.push_back(lin[q]);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    for (size_t q = 0; q < verts.size(); ++q) {
        const int i = verts[q];
        agg[i] = clamped[i] ? -1
                            : base + (int32_t)(std::lower_bound(keys.begin(), keys.end(), lin[q]) - keys.begin());
    }
    return (int)keys.size();
}

// Device vertex order: by connected component (in order of their smallest mesh index),
// then by coarse bin, then by mesh index.  Every aggregate is then one run of consecutive
// device indices (clamped vertices leave holes), so the warp-per-aggregate phases of the
// solve read and write consecutive addresses.  Returns mesh index -> device index.
static std::vector<int32_t> aggregate_order(int nv, const double* X, int ntet, const int32_t* tets) {
    std::vector<int32_t> up(nv);
    for (int i = 0; i < nv; ++i) up[i] = i;
    auto root = [&](int v) {
        while (up[v] != v) {
            up[v] = up[up[v]];
            v = up[v];
        }
        return v;
    };
    for (int t = 0; t < ntet; ++t) {
        const int32_t* tv = tets + (size_t)t * 4;
        for (int k = 0; k < 4; ++k)
            if (tv[k] < 0 || tv[k] >= nv) throw ArgErr("tet vertex index out of range");
        const int r0 = root(tv[0]);
        for (int k = 1; k < 4; ++k) {
            const int rk = root(tv[k]);
            if (rk != r0) up[std::max(rk, r0)] = std::min(rk, r0);
        }
    }
    // Roots are the smallest vertex of their component; label components in that order.
    std::vector<int32_t> label(nv, -1);
    std::vector<std::vector<int32_t>> comps;
    for (int i = 0; i < nv; ++i) {
        const int r = root(i);
        if (label[r] < 0) {
            label[r] = (int32_t)comps.size();
            comps.emplace_back();
        }
        comps[label[r]].push_back(i);
    }
    std::vector<int32_t> perm(nv);
    int32_t next = 0;
    std::vector<long> lin;
    std::vector<std::pair<long, int32_t>> key;
    for (const auto& cv : comps) {
        component_bins(cv, X, aggregate_target(cv.size()), lin);
        key.resize(cv.size());
        for (size_t q = 0; q < cv.size(); ++q) key[q] = {lin[q], cv[q]};
        std::sort(key.begin(), key.end());
        for (const auto& kv : key) perm[kv.second] = next++;
    }
    return perm;
}

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
    // Coarse space of the two-level preconditioner, per connected component of the vertex
    // graph (no edge joins two components, so E = Z^T A Z is block diagonal): about 1000
    // aggregates (>= 16 vertices each) per component, each block inverted densely and
    // stored row-major one after another.
    std::vector<int32_t> agg(n, -1);
    std::vector<int32_t> cbase(ncomp_v + 1, 0);
    for (int c = 0; c < ncomp_v; ++c) {
        const int target = aggregate_target(comp_verts[c].size());
        cbase[c + 1] = cbase[c] + make_aggregates(comp_verts[c], verts_um, vclamped, target, cbase[c], agg);
    }
    const int na = cbase[ncomp_v];
    std::vector<int32_t> h_agg_base(std::max(na, 1), 0), h_agg_len(std::max(na, 1), 0);
    std::vector<long long> h_agg_row(std::max(na, 1), 0), boff(ncomp_v + 1, 0);
    for (int c = 0; c < ncomp_v; ++c) {
        const long long m = cbase[c + 1] - cbase[c];
        boff[c + 1] = boff[c] + m * m;
        for (int a = cbase[c]; a < cbase[c + 1]; ++a) {
            h_agg_base[a] = cbase[c];
            h_agg_len[a] = (int32_t)m;
            h_agg_row[a] = boff[c] + (long long)(a - cbase[c]) * m;
        }
    }
    std::vector<double> E((size_t)boff[ncomp_v], 0.0);
    for (int i = 0; i < n; ++i) {
        const int ai = agg[i];
        if (ai < 0) continue;
        double* row = &E[(size_t)h_agg_row[ai]];
        const int b0 = h_agg_base[ai];
        row[ai - b0] += diag[i];
        for (int w = 0; w < width; ++w) {
            int j = acol[(size_t)w * n + i];
            if (j < 0) break;
            row[agg[j] - b0] += a64[(size_t)w * n + i];
        }
    }
    // The components' blocks are independent: invert them on all host cores.
    bool spd_ok = true;
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < ncomp_v; ++c) {
        const int m = cbase[c + 1] - cbase[c];
        if (m == 0) continue;
        std::vector<double> blk(E.begin() + boff[c], E.begin() + boff[c + 1]);
        try {
            spd_inverse(m, blk);
        } catch (...) {
#pragma omp atomic write
            spd_ok = false;
            continue;
        }
        std::copy(blk.begin(), blk.end(), E.begin() + boff[c]);
    }
    if (!spd_ok) throw DeviceErr("EField coarse matrix is not positive definite");
    std::vector<float> E32(E.begin(), E.end());
    if (na != nagg || (size_t)boff[ncomp_v] != einv_len || !d_agg) {
        dfree(d_einv64);
        dfree(d_einv32);
        dfree(alt_diag64);
        dfree(alt_einv64);
        dfree(alt_einv32);
        alt_dt = -1.0;
        dfree(d_c64);
        dfree(d_c32);
        dfree(d_agg_base);
        dfree(d_agg_len);
        dfree(d_agg_row);
        size_t m = std::max(na, 1);
        einv_len = (size_t)boff[ncomp_v];
        dalloc(d_einv64, std::max<size_t>(einv_len, 1));
        dalloc(d_einv32, std::max<size_t>(einv_len, 1));
        dalloc(d_c64, m);
        dalloc(d_c32, m);
        dalloc(d_agg_base, m);
        dalloc(d_agg_len, m);
        dalloc(d_agg_row, m);
        if (!d_agg) dalloc(d_agg, n);
        nagg = na;
    }
    SG_CUDA(cudaMemcpyAsync(d_agg, agg.data(), agg.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_agg_base, h_agg_base.data(), h_agg_base.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_agg_len, h_agg_len.data(), h_agg_len.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_agg_row, h_agg_row.data(), h_agg_row.size() * 8, cudaMemcpyHostToDevice, stream));
    // Segments: each aggregate's vertices in ascending order, then the vertices of no
    // aggregate (clamped) in chunks of 256.
    std::vector<int32_t> sptr(1, 0), sidx, sagg;
    {
        std::vector<int32_t> cnt(na + 1, 0);
        for (int i = 0; i < n; ++i)
            if (agg[i] >= 0) cnt[agg[i] + 1]++;
        for (int a = 0; a < na; ++a) cnt[a + 1] += cnt[a];
        sidx.assign(n, 0);
        std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
        int nfree = 0;
        for (int i = 0; i < n; ++i)
            if (agg[i] >= 0) sidx[fill[agg[i]]++] = i;
        for (int a = 0; a < na; ++a) {
            sptr.push_back(cnt[a + 1]);
            sagg.push_back(a);
        }
        int pos = cnt[na];
        for (int i = 0; i < n; ++i)
            if (agg[i] < 0) {
                sidx[pos++] = i;
                if (++nfree == 256) {
                    sptr.push_back(pos);
                    sagg.push_back(-1);
                    nfree = 0;
                }
            }
        if (nfree) {
            sptr.push_back(pos);
            sagg.push_back(-1);
        }
    }
    nseg = (int)sagg.size();
    dalloc(d_seg_ptr, sptr.size());
    dalloc(d_seg_idx, std::max<size_t>(sidx.size(), 1));
    dalloc(d_seg_agg, std::max<size_t>(sagg.size(), 1));
    SG_CUDA(cudaMemcpyAsync(d_seg_ptr, sptr.data(), sptr.size() * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_seg_idx, sidx.data(), sidx.size() * 4, cudaMemcpyHostToDevice, stream));
    if (nseg) SG_CUDA(cudaMemcpyAsync(d_seg_agg, sagg.data(), sagg.size() * 4, cudaMemcpyHostToDevice, stream));
    if (!E.empty()) {
        SG_CUDA(cudaMemcpyAsync(d_einv64, E.data(), E.size() * 8, cudaMemcpyHostToDevice, stream));
        SG_CUDA(cudaMemcpyAsync(d_einv32, E32.data(), E32.size() * 4, cudaMemcpyHostToDevice, stream));
    }
    SG_CUDA(cudaStreamSynchronize(stream));  // host vectors above are temporaries
    dt_built = dt_ms;
    dirty = false;
}

// Two-level PCG iterations from a started state (r, its restriction in c, and the
// scalars S_RR, S_TOL2, S_ITER, S_DONE set): preconditioned start, then chunks of three
// kernels per iteration, {p = z + beta p, q = A p, alpha} -> {x, r, restriction c} ->
// {coarse solve, z, beta}, until the device flag S_DONE is set; h receives the final
// scalars.  pv and pv2 alternate as the direction buffer.
template <typename T>
void EFieldSystem::pcg_loop(cudaStream_t stream, int n, int g, const T* a, T* xv, T* rv, T* zv, T* pv, T* pv2,
                            T* qv, const T* einv, T* cvec, double* h) {
    const Segs sg{nseg, d_seg_ptr, d_seg_idx, d_seg_agg};
    const int gs = seg_grid();
    const Coarse cs{d_agg_base, d_agg_len, d_agg_row};
    precond_kernel<T><<<gs, kBlock, 0, stream>>>(sg, cs, diag64, rv, zv, pv, einv, cvec, red, red_count, scal, 1);
    T* pin = pv;
    T* pout = pv2;
    const int chunk = 8;
    for (int it = 0; it < max_iter; it += chunk) {
        for (int c = 0; c < chunk; ++c) {
            spmv_kernel<T><<<g, kBlock, 0, stream>>>(n, width, acol_dev, a, diag64, zv, pin, pout, qv, red, red_count,
                                                     scal);
            update_kernel<T><<<gs, kBlock, 0, stream>>>(sg, xv, rv, pout, qv, cvec, red, red_count, scal, max_iter);
            precond_kernel<T><<<gs, kBlock, 0, stream>>>(sg, cs, diag64, rv, zv, nullptr, einv, cvec, red,
                                                         red_count, scal, 0);
            std::swap(pin, pout);
        }
        SG_CUDA(cudaGetLastError());
        SG_CUDA(cudaMemcpyAsync(h, scal, kScalOut * sizeof(double), cudaMemcpyDeviceToHost, stream));
        SG_CUDA(cudaStreamSynchronize(stream));
        if (h[S_DONE] != 0.0) break;
    }
}

// The persistent form of pcg_loop: one cooperative launch runs every iteration.
template <typename T>
void EFieldSystem::pcg_persistent(cudaStream_t stream, int n, const T* a, T* xv, T* rv, T* zv, T* pv, T* pv2,
                                  T* qv, const T* einv, T* cvec, double* h) {
    // Systems whose rows fit one pass of a kMinbSmall-blocks-per-SM grid take the
    // latency-bound form.
    const void* kern = (n <= kMinbSmall * nsm * kBlock) ? (const void*)pcg_persistent_kernel<T, kMinbSmall>
                                                        : (const void*)pcg_persistent_kernel<T, 8>;
    int per_sm = 0;
    SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, 0));
    const int want = std::max((n + kBlock - 1) / kBlock, (nseg + 7) / 8);
    const int G = std::max(1, std::min(std::min(want, std::max(per_sm, 1) * nsm), 2048));
    PcgArgs<T> P;
    P.n = n;
    P.width = width;
    P.cs = Coarse{d_agg_base, d_agg_len, d_agg_row};
    P.max_iter = max_iter;
    P.col = acol_dev;
    P.a = a;
    P.diag = diag64;
    P.einv = einv;
    P.sg = Segs{nseg, d_seg_ptr, d_seg_idx, d_seg_agg};
    P.x = xv;
    P.r = rv;
    P.z = zv;
    P.p = pv;
    P.p2 = pv2;
    P.q = qv;
    P.c = cvec;
    P.partials = red;
    P.scal = scal;
    P.bar = d_bar;
    P.spin_limit = spin_limit;
    P.ru = 0;
    P.delta2 = 0.0;
    P.tol2_64 = 0.0;
    P.a64 = nullptr;
    P.b64 = nullptr;
    P.x64 = nullptr;
    P.r64 = nullptr;
    if (std::is_same<T, float>::value && ru_tol2 > 0.0) {
        P.ru = 1;
        P.delta2 = ru_delta * ru_delta;
        P.tol2_64 = ru_tol2;
        P.a64 = ell_a64;
        P.b64 = b;
        P.x64 = x;
        P.r64 = r;
    }
    SG_CUDA(cudaMemsetAsync(d_bar, 0, 4 * sizeof(unsigned int), stream));
    void* args[] = {&P};
    SG_CUDA(cudaLaunchCooperativeKernel(kern, dim3(G), dim3(kBlock), args, 0, stream));
    unsigned int err = 0;
    SG_CUDA(cudaMemcpyAsync(h, scal, kScalOut * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(cudaMemcpyAsync(&err, d_bar + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(cudaStreamSynchronize(stream));
    if (err) throw DeviceErr("EField solve: a grid barrier wait timed out");
}

template <typename T>
void EFieldSystem::pcg(cudaStream_t stream, int n, int g, const T* a, T* xv, T* rv, T* zv, T* pv, T* pv2, T* qv,
                       const T* einv, T* cvec, double* h) {
    if (persistent)
        pcg_persistent<T>(stream, n, a, xv, rv, zv, pv, pv2, qv, einv, cvec, h);
    else
        pcg_loop<T>(stream, n, g, a, xv, rv, zv, pv, pv2, qv, einv, cvec, h);
}

// One EField step: RHS from the current V and currents, CG solve, V update.  The matrix
// is rebuilt when the step length changes by more than rounding (the truncated last step
// of a run), or when clamps or membrane properties change.
void EFieldSystem::advance(double dt_ms, cudaStream_t stream) {
    if (dirty || std::fabs(dt_ms - dt_built) > 1e-9 * dt_built) {
        // The diagonal and the coarse inverses depend on dt; the previous step length's
        // are kept, so a run that ends on a short step and resumes at the regular one (or
        // alternates two lengths) swaps instead of rebuilding on the host.
        const bool keep = !dirty && dt_built > 0.0 && d_einv64;
        if (keep && alt_dt > 0.0 && std::fabs(dt_ms - alt_dt) <= 1e-9 * alt_dt) {
            std::swap(diag64, alt_diag64);
            std::swap(d_einv64, alt_einv64);
            std::swap(d_einv32, alt_einv32);
            std::swap(dt_built, alt_dt);
        } else {
            if (keep) {
                if (!alt_diag64) {
                    dalloc(alt_diag64, nverts);
                    dalloc(alt_einv64, std::max<size_t>(einv_len, 1));
                    dalloc(alt_einv32, std::max<size_t>(einv_len, 1));
                }
                std::swap(diag64, alt_diag64);
                std::swap(d_einv64, alt_einv64);
                std::swap(d_einv32, alt_einv32);
                alt_dt = dt_built;
            } else {
                alt_dt = -1.0;
            }
            build_matrix(dt_ms, stream);
        }
    }
    const int n = nverts;
    const int g = grid_for(n, nsm);
    const Segs sg{nseg, d_seg_ptr, d_seg_idx, d_seg_agg};
    const int gs = seg_grid();
    SG_CUDA(cudaEventRecord(ev0, stream));
    rhs_kernel<<<g, kBlock, 0, stream>>>(n, width, V, ell_col, ell_cc, cap_gext, v_leak, d_vert_iclamp, d_vt_ptr,
                                         d_vt_idx, tri_I, d_tri_iclamp, d_vclamped, b);
    SG_CUDA(cudaGetLastError());
    double h[kScalOut];
    double check_ms = 0.0;
    if (method == EF_CG_FP64) {
        // Warm start from the previous step's dV (x keeps it): r = b - A x, restricted.
        residual_kernel<<<gs, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, sg, d_c64, red,
                                                   red_count, scal);
        warm_start_kernel<<<1, 1, 0, stream>>>(scal, tol);
        pcg<double>(stream, n, g, ell_a64, x, r, z, p, p2, q, d_einv64, d_c64, h);
        stats.iterations += (uint64_t)h[S_ITER];
        stats.last_rel_residual = h[S_BB] > 0.0 ? std::sqrt(h[S_RR] / h[S_BB]) : 0.0;
        if (h[S_BB] > 0.0 && h[S_RR] > h[S_TOL2]) throw DeviceErr("EField CG did not converge");
    } else {
        // Mixed precision: FP32 two-level PCG on the correction, FP64 residuals and
        // accumulation, warm-started from the previous step's dV.
        residual_kernel<<<gs, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, sg, nullptr,
                                                   red, red_count, scal);
        SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
        SG_CUDA(cudaStreamSynchronize(stream));
        const double bb = h[S_BB];
        double rr = h[S_RR];
        int outer = 0;
        if (persistent && reliable && bb > 0.0 && rr > tol * tol * bb) {
            // One FP32 solve with reliable updates to the FP64 tolerance (x32 = 0, s32 = r32).
            init_kernel<float><<<gs, kBlock, 0, stream>>>(sg, r32, x32, s32, d_c32, red, red_count, scal, inner_tol);
            ru_tol2 = tol * tol * bb;
            pcg<float>(stream, n, g, ell_a32, x32, s32, z32, p32, p2_32, q32, d_einv32, d_c32, h);
            ru_tol2 = 0.0;
            stats.iterations += (uint64_t)h[S_ITER];
            stats.refinements += (uint64_t)h[S_NRU];
            rr = h[S_RR];
            if (bb > 0.0 && rr > tol * tol * bb) {
                // Stopped above the tolerance: the refinement loop below starts from the
                // FP32 residual, which the reliable-update solve does not keep current.
                residual_kernel<<<gs, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, sg,
                                                           nullptr, red, red_count, scal);
                SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
                SG_CUDA(cudaStreamSynchronize(stream));
                rr = h[S_RR];
            }
        }
        while (bb > 0.0 && rr > tol * tol * bb && outer < 50) {
            // Inner FP32 solve of A d = r32: s32 is its residual, q32 = A p32.
            init_kernel<float><<<gs, kBlock, 0, stream>>>(sg, r32, x32, s32, d_c32, red, red_count, scal, inner_tol);
            pcg<float>(stream, n, g, ell_a32, x32, s32, z32, p32, p2_32, q32, d_einv32, d_c32, h);
            stats.iterations += (uint64_t)h[S_ITER];
            add_correction_kernel<<<g, kBlock, 0, stream>>>(n, x, x32);
            residual_kernel<<<gs, kBlock, 0, stream>>>(n, width, acol_dev, ell_a64, diag64, b, x, r, r32, sg, nullptr,
                                                       red, red_count, scal);
            SG_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
            SG_CUDA(cudaStreamSynchronize(stream));
            rr = h[S_RR];
            stats.refinements += 1;
            ++outer;
        }
        stats.last_rel_residual = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
        if (bb > 0.0 && rr > tol * tol * bb) throw DeviceErr("EField refinement did not converge");
    }
    if (check) {
        // FP64 solve of the same system from zero, then the per-vertex comparison.
        if (!xchk) dalloc(xchk, n);
        if (!evc0) {
            SG_CUDA(cudaEventCreate(&evc0));
            SG_CUDA(cudaEventCreate(&evc1));
        }
        SG_CUDA(cudaEventRecord(evc0, stream));
        init_kernel<double><<<gs, kBlock, 0, stream>>>(sg, b, xchk, r, d_c64, red, red_count, scal, check_tol);
        pcg<double>(stream, n, g, ell_a64, xchk, r, z, p, p2, q, d_einv64, d_c64, h);
        SG_CUDA(cudaMemsetAsync(scal + S_CHK, 0, sizeof(double), stream));
        check_kernel<<<g, kBlock, 0, stream>>>(n, V, x, xchk, d_vclamped, scal);
        double e = 0.0;
        SG_CUDA(cudaMemcpyAsync(&e, scal + S_CHK, sizeof(double), cudaMemcpyDeviceToHost, stream));
        SG_CUDA(cudaEventRecord(evc1, stream));
        SG_CUDA(cudaEventSynchronize(evc1));
        float cms = 0.0f;
        SG_CUDA(cudaEventElapsedTime(&cms, evc0, evc1));
        check_ms = cms;
        stats.check_steps += 1;
        stats.check_last_rel = e;
        stats.check_max_rel = std::max(stats.check_max_rel, e);
    }
    apply_kernel<<<g, kBlock, 0, stream>>>(n, V, x, d_vclamped);
    if (ntris) tri_v_kernel<<<grid_for(ntris, nsm), kBlock, 0, stream>>>(ntris, d_tri_verts, V, tri_V);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaEventRecord(ev1, stream));
    SG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    SG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    stats.solve_ms += ms - check_ms;  // the check solve is not part of the step's cost
    stats.steps += 1;
}

}  // namespace sg
