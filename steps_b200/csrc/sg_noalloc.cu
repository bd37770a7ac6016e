// Allocation-free entry point: operator-split windows on caller-owned device buffers.
//
// Some callers cannot call cudaMalloc: host programs whose device memory comes only
// from their own pool allocator (the step embedded next to other GPU code that owns
// the device's memory), and long-running loops where an allocation's implicit
// device-wide synchronisation on every call is not acceptable.  For them
// sg_run_noalloc() runs the same window kernel as the solver object, but keeps every
// piece of scratch the kernel needs (packed mesh tables, the double-buffered face
// outflow, counters, the realization record, the status word) in one file-scope
// device array, g_noalloc_scratch, instead of memory allocated per solver.
//
// The array has a fixed size (SG_NOALLOC_SCRATCH_BYTES, about 11 MiB) that every GPU
// which loads this library holds until the process exits.  All calls share it and it
// keeps the contents of the last call: each call clears the counters, the status word
// and the face outflow it relies on, and calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race on it and must be serialised by the caller.
// A call synchronises the caller's stream twice (after the table build, to read the
// largest face coefficient, and at the end, to read the status word).
#include <cuda_runtime.h>

#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "sg_errors.h"
#include "sg_rng.cuh"
#include "sg_types.h"
#include "sg_window.cuh"
#include "../../include/steps_b200.h"

namespace {

constexpr size_t kMaxTets = SG_NOALLOC_MAX_TETS;
constexpr size_t kMaxTetSpecies = SG_NOALLOC_MAX_TET_SPECIES;
constexpr size_t kMaxSpecs = 32;
constexpr size_t kMaxReacs = SG_NOALLOC_MAX_REACS;

// Byte offsets of the regions inside the scratch array (all 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffNbr = 0;                                               // int32 [T][4]
constexpr size_t kOffGeo = align256(kOffNbr + kMaxTets * 16);               // float [T][4]
constexpr size_t kOffIvs = align256(kOffGeo + kMaxTets * 16);               // double [T]
constexpr size_t kOffOut = align256(kOffIvs + kMaxTets * 8);                // uint4 [2][S][T]
constexpr size_t kOffReacs = align256(kOffOut + 2 * kMaxTetSpecies * 16);   // sg_reac [R]
constexpr size_t kOffKcst = align256(kOffReacs + kMaxReacs * sizeof(sg_reac));
constexpr size_t kOffDcst = align256(kOffKcst + kMaxReacs * 8);             // double [S]
constexpr size_t kOffSlot = align256(kOffDcst + kMaxSpecs * 8);             // int32 [S]
constexpr size_t kOffCrb = align256(kOffSlot + kMaxSpecs * 4);              // int32 [2]
constexpr size_t kOffReal = align256(kOffCrb + 8);                          // sg_real [1]
constexpr size_t kOffCounters = align256(kOffReal + sizeof(sg_real));       // u64 counters
constexpr size_t kCounterWords = 2 * kMaxSpecs + 2 * kMaxReacs + kMaxReacs + 1 + 4;
constexpr size_t kOffStatus = align256(kOffCounters + kCounterWords * 8);   // u32 status, float gmax
constexpr size_t kScratchBytes = align256(kOffStatus + 16);
static_assert(kScratchBytes == SG_NOALLOC_SCRATCH_BYTES, "header size constant out of date");

}  // namespace

// The scratch itself.  In host code this name is only a stand-in for the device
// symbol: its device address is obtained with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

const double kAvogadro = 6.02214179e23;  // src/steps/math/constants.hpp:45

// Per-tet tables from the raw mesh arrays, exactly as the solver object builds them on
// the host (diff.cpp:41-90 face coefficients; one compartment holding every tet), plus
// the largest G over the mesh for the update period.
__global__ void noalloc_tables_kernel(int ntets, const double* vol, const int32_t* neighb,
                                      const double* area, const double* dist, int32_t* nbrp,
                                      float* geo, double* ivs, unsigned int* gmax_bits,
                                      uint32_t* status) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntets; t += gridDim.x * blockDim.x) {
        double v = vol[t];
        // A non-positive or non-finite volume would give infinite rates.
        if (!(v > 0.0) || !(v < 1.0e300)) atomicOr(status, SG_ERR_TABLE);
        ivs[t] = 1.0 / (1.0e3 * v * kAvogadro);
        double g[4] = {0.0, 0.0, 0.0, 0.0};
        for (int f = 0; f < 4; ++f) {
            int n = neighb[(size_t)t * 4 + f];
            nbrp[(size_t)t * 4 + f] = -1;
            if (n == -1) continue;
            if (n < -1 || n >= ntets) {
                atomicOr(status, SG_ERR_TABLE);
                continue;
            }
            int rf = -1;
            for (int j = 0; j < 4; ++j)
                if (neighb[(size_t)n * 4 + j] == t) rf = j;
            if (rf < 0) {
                atomicOr(status, SG_ERR_TABLE);
                continue;
            }
            double d = dist[(size_t)t * 4 + f];
            // Both sides must agree on whether the face is open: a face open on one side
            // only would send molecules into a slot the other side never reads.
            if ((d > 0.0) != (dist[(size_t)n * 4 + rf] > 0.0)) {
                atomicOr(status, SG_ERR_TABLE);
                continue;
            }
            if (d > 0.0) {
                g[f] = area[(size_t)t * 4 + f] / (v * d);
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
        float Gf = (float)G;
        geo[(size_t)t * 4 + 3] = Gf;
        atomicMax(gmax_bits, __float_as_uint(Gf));  // G >= 0: bit order is value order
    }
}

std::mutex g_symbol_mutex;
void* g_symbol_addr[128] = {nullptr};

// Device address of the scratch array on the current device, looked up once per device
// and cached for the life of the process (a cudaDeviceReset would invalidate it; the
// header says not to call this entry point after one).
unsigned char* scratch_on(int device) {
    if (device < 0 || device >= 128) throw sg::ArgErr("device index out of range");
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    if (!g_symbol_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw sg::CudaErr(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                              cudaGetErrorString(e));
        g_symbol_addr[device] = p;
    }
    return static_cast<unsigned char*>(g_symbol_addr[device]);
}

bool almost_equal(double x, double y) {  // src/steps/util/collections.hpp:144-148
    double d = std::fabs(x - y);
    return d <= std::numeric_limits<double>::epsilon() * std::fabs(x + y) * 4 ||
           d < std::numeric_limits<double>::min();
}

// Dense lhs/upd rows -> compact reaction records (same rules as sg_add_reac).
std::vector<sg_reac> compact_reacs(int nspec, int nreac, const uint32_t* lhs, const int32_t* upd) {
    std::vector<sg_reac> out(nreac);
    for (int q = 0; q < nreac; ++q) {
        sg_reac r;
        std::memset(&r, 0, sizeof(r));
        for (int i = 0; i < nspec; ++i) {
            uint32_t l = lhs[(size_t)q * nspec + i];
            if (l == 0) continue;
            if (l > 4) throw sg::ArgErr("reactant stoichiometry above 4 is not supported");
            if (r.nlhs == SG_MAX_LHS) throw sg::ArgErr("more than 4 distinct reactants");
            r.lhs_spec[r.nlhs] = i;
            r.lhs_ord[r.nlhs] = (int32_t)l;
            r.nlhs += 1;
            r.order += (int32_t)l;
            r.lhs_mask |= 1u << i;
        }
        if (r.order > 4) throw sg::ArgErr("reaction order above 4 is not supported");
        for (int i = 0; i < nspec; ++i) {
            int32_t u = upd[(size_t)q * nspec + i];
            if (u == 0) continue;
            if (r.nupd == SG_MAX_UPD) throw sg::ArgErr("a reaction changes more than 8 species");
            r.upd_spec[r.nupd] = i;
            r.upd_delta[r.nupd] = u;
            r.nupd += 1;
            r.upd_mask |= 1u << i;
        }
        r.fast = sg_reac_fast_code(&r);
        out[q] = r;
    }
    return out;
}

void run_noalloc(int32_t ntets, int32_t nspec, int32_t nreac, uint32_t* counts, const double* vol,
                 const int32_t* neighb, const double* area, const double* dist, const uint32_t* lhs,
                 const int32_t* upd, const double* kcst, const double* dcst, uint64_t seed, double t0,
                 double t_end, uint64_t window0, void* stream_v, uint64_t* windows_out,
                 double* period_out) {
    if (ntets <= 0 || (size_t)ntets > kMaxTets)
        throw sg::ArgErr("sg_run_noalloc: ntets must be in 1.." + std::to_string(kMaxTets) +
                         " (the scratch array has a fixed size)");
    if (nspec <= 0 || (size_t)nspec > kMaxSpecs)
        throw sg::ArgErr("sg_run_noalloc: nspec must be in 1..32");
    if ((size_t)ntets * (size_t)nspec > kMaxTetSpecies)
        throw sg::ArgErr("sg_run_noalloc: ntets * nspec must not exceed " + std::to_string(kMaxTetSpecies) +
                         " (the scratch array has a fixed size)");
    if (nreac < 0 || (size_t)nreac > kMaxReacs)
        throw sg::ArgErr("sg_run_noalloc: nreac must be in 0.." + std::to_string(kMaxReacs));
    if (!counts || !vol || !neighb || !area || !dist || !dcst)
        throw sg::ArgErr("sg_run_noalloc: null buffer");
    if (nreac > 0 && (!lhs || !upd || !kcst)) throw sg::ArgErr("sg_run_noalloc: null reaction table");
    if (!(t_end >= t0)) throw sg::ArgErr("Endtime is before current simulation time");
    for (int q = 0; q < nreac; ++q)
        if (!(kcst[q] >= 0.0)) throw sg::ArgErr("reaction constant must be non-negative");
    for (int s = 0; s < nspec; ++s)
        if (!(dcst[s] >= 0.0)) throw sg::ArgErr("diffusion constant must be non-negative");

    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    int device = 0;
    SG_CUDA(cudaGetDevice(&device));
    unsigned char* base = scratch_on(device);

    std::vector<sg_reac> reacs = compact_reacs(nspec, nreac, lhs, upd);
    std::vector<int32_t> slot(nspec);
    for (int s = 0; s < nspec; ++s) slot[s] = s;
    int32_t crb[2] = {0, nreac};

    int32_t* d_nbr = reinterpret_cast<int32_t*>(base + kOffNbr);
    float* d_geo = reinterpret_cast<float*>(base + kOffGeo);
    double* d_ivs = reinterpret_cast<double*>(base + kOffIvs);
    uint32_t* d_out = reinterpret_cast<uint32_t*>(base + kOffOut);
    sg_reac* d_reacs = reinterpret_cast<sg_reac*>(base + kOffReacs);
    double* d_kcst = reinterpret_cast<double*>(base + kOffKcst);
    double* d_dcst = reinterpret_cast<double*>(base + kOffDcst);
    int32_t* d_slot = reinterpret_cast<int32_t*>(base + kOffSlot);
    int32_t* d_crb = reinterpret_cast<int32_t*>(base + kOffCrb);
    sg_real* d_real = reinterpret_cast<sg_real*>(base + kOffReal);
    unsigned long long* d_ctr = reinterpret_cast<unsigned long long*>(base + kOffCounters);
    uint32_t* d_status = reinterpret_cast<uint32_t*>(base + kOffStatus);
    unsigned int* d_gmax = reinterpret_cast<unsigned int*>(base + kOffStatus + 4);

    // Everything that must start at zero: counters, launch state, status, G max, and the
    // face-outflow double buffer of this problem's size (an earlier call's values must
    // never be gathered as inflow).
    SG_CUDA(cudaMemsetAsync(d_ctr, 0, kCounterWords * 8, stream));
    SG_CUDA(cudaMemsetAsync(d_status, 0, 8, stream));
    SG_CUDA(cudaMemsetAsync(d_out, 0, 2 * (size_t)nspec * (size_t)ntets * 16, stream));
    if (nreac) SG_CUDA(cudaMemcpyAsync(d_reacs, reacs.data(), reacs.size() * sizeof(sg_reac),
                                       cudaMemcpyHostToDevice, stream));
    if (nreac) SG_CUDA(cudaMemcpyAsync(d_kcst, kcst, (size_t)nreac * 8, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_dcst, dcst, (size_t)nspec * 8, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_slot, slot.data(), (size_t)nspec * 4, cudaMemcpyHostToDevice, stream));
    SG_CUDA(cudaMemcpyAsync(d_crb, crb, sizeof(crb), cudaMemcpyHostToDevice, stream));

    int nsm = 148;
    SG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    int tg = std::max(1, std::min((ntets + 255) / 256, nsm * 8));
    noalloc_tables_kernel<<<tg, 256, 0, stream>>>(ntets, vol, neighb, area, dist, d_nbr, d_geo, d_ivs,
                                                  d_gmax, d_status);
    SG_CUDA(cudaGetLastError());
    uint32_t head[2] = {0u, 0u};  // status, G max bits
    SG_CUDA(cudaMemcpyAsync(head, d_status, 8, cudaMemcpyDeviceToHost, stream));
    SG_CUDA(cudaStreamSynchronize(stream));
    if (head[0])
        throw sg::ArgErr("sg_run_noalloc: invalid mesh tables (a volume that is not positive and finite, a "
                         "neighbour index out of range or not symmetric, or a face open on one side only)");
    float gmax_f;
    std::memcpy(&gmax_f, &head[1], 4);
    double mx = 0.0;
    for (int s = 0; s < nspec; ++s) {
        double sd = dcst[s] * (double)gmax_f;
        if (sd > mx) mx = sd;
    }
    const double period = (mx > 0.0) ? 1.0 / mx : std::numeric_limits<double>::infinity();
    if (period_out) *period_out = period;

    uint64_t n = 0;
    if (!almost_equal(t0, t_end)) {
        double t = t0;
        while (t < t_end) {
            t = (t + period > t_end) ? t_end : t + period;
            n += 1;
        }
    }
    if (windows_out) *windows_out = n;
    if (n == 0) return;

    sg_real rl;
    std::memset(&rl, 0, sizeof(rl));
    rl.tet_begin = 0;
    rl.tet_end = ntets;
    rl.t = t0;
    rl.t_end = t_end;
    rl.period = period;
    rl.window = window0;
    rl.pending = 0;
    SG_CUDA(cudaMemcpyAsync(d_real, &rl, sizeof(rl), cudaMemcpyHostToDevice, stream));

    sg_window_args a;
    std::memset(&a, 0, sizeof(a));
    a.counts = counts;
    a.outflow = d_out;
    a.nbr = d_nbr;
    a.geo = d_geo;
    a.ivs = d_ivs;
    a.comp = nullptr;
    a.clamp = nullptr;
    a.reacs = d_reacs;
    a.comp_reac_begin = d_crb;
    a.kcst = d_kcst;
    a.dcst = d_dcst;
    a.diff_slot = d_slot;
    a.reals = d_real;
    a.totals = d_ctr;
    a.ext = d_ctr + 2 * kMaxSpecs;
    a.ext_total = d_ctr + 2 * kMaxSpecs + 2 * kMaxReacs;
    a.diff_total = d_ctr + 2 * kMaxSpecs + 3 * kMaxReacs;
    a.launch_state = d_ctr + 2 * kMaxSpecs + 3 * kMaxReacs + 1;
    a.status = d_status;
    a.ntets = ntets;
    a.nspec = nspec;
    a.ndiff = nspec;
    a.nreac = nreac;
    a.ncomp = 1;
    a.nreal = 1;
    a.seed = seed;

    constexpr int kBlock = 128;
    size_t sm = sg::smem_bytes(kBlock, nspec, nreac);
    if (sm > 48 * 1024)
        SG_CUDA(cudaFuncSetAttribute(sg::window_kernel<kBlock>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
    SG_CUDA(cudaFuncSetAttribute(sg::window_kernel<kBlock>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 0;
    SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sg::window_kernel<kBlock>, kBlock, sm));
    long need = ((long)ntets + kBlock - 1) / kBlock;
    int g = (int)std::max(1L, std::min(need, (long)std::max(per_sm, 1) * nsm));
    for (uint64_t i = 0; i < n; ++i) {
        sg::window_kernel<kBlock><<<g, kBlock, sm, stream>>>(a, 1);
        SG_CUDA(cudaGetLastError());
    }
    // Apply the inflow of the last window so that counts is complete on return.
    sg::flush_kernel<<<tg, 256, 0, stream>>>(a);
    SG_CUDA(cudaGetLastError());
    uint32_t st = 0;
    SG_CUDA(cudaMemcpyAsync(&st, d_status, 4, cudaMemcpyDeviceToHost, stream));
    SG_CUDA(cudaStreamSynchronize(stream));
    if (st) throw sg::DeviceErr("sg_run_noalloc: device status error " + std::to_string(st) +
                                " (1 conservation, 2 overflow, 16 negative count)");
}

}  // namespace

extern "C" int sg_run_noalloc(int32_t ntets, int32_t nspec, int32_t nreac, uint32_t* counts,
                              const double* vol, const int32_t* neighb, const double* area,
                              const double* dist, const uint32_t* lhs, const int32_t* upd,
                              const double* kcst, const double* dcst, uint64_t seed, double t0,
                              double t_end, uint64_t window0, void* stream, uint64_t* windows_out,
                              double* period_out) {
    try {
        run_noalloc(ntets, nspec, nreac, counts, vol, neighb, area, dist, lhs, upd, kcst, dcst, seed, t0,
                    t_end, window0, stream, windows_out, period_out);
        return SG_OK;
    } catch (const sg::ArgErr& e) {
        sg::set_last_error(e.what());
        return SG_EARG;
    } catch (const sg::CudaErr& e) {
        sg::set_last_error(e.what());
        return SG_ECUDA;
    } catch (const sg::DeviceErr& e) {
        sg::set_last_error(e.what());
        return SG_EDEVICE;
    } catch (const std::exception& e) {
        sg::set_last_error(e.what());
        return SG_EPROG;
    }
}
