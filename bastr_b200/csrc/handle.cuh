// Internals shared by the translation units of the library: the solver handle, its error
// reporting, launch helpers and the persistent-grid sizing of the pass kernels.  The 2D and 3D
// step schedules (steps2d.cuh, steps3d.cuh) are compiled in their own translation units, one per
// compute precision, so that the library builds in parallel; capi.cu holds the C ABI.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/bastr_gpu.h"
#include <nvtx3/nvToolsExt.h>
#ifndef BASTR_PDL
#define BASTR_PDL 1
#endif
// 2D: the forward y pass of RK stages 1 and 2 (and CN sweeps 1-5) also runs the next stage's
// inverse y pass (k2d_yfwd_inv).
#ifndef BASTR_FUSE_Y
#define BASTR_FUSE_Y 1
#endif
// Returns the launch error from the enclosing cudaError_t function.
#define LAUNCH(...)                                 \
    do {                                            \
        cudaError_t le_ = (__VA_ARGS__);            \
        if (le_ != cudaSuccess) return le_;         \
    } while (0)
#include "solver.cuh"
#include "tma.cuh"

using namespace bastr;

namespace bastr_impl {

constexpr int kChunk = 256;   // records kept on the device per batch chunk

struct Twiddles {
    int n = 0;
    double2* d64 = nullptr;
    float2* d32 = nullptr;
};

}  // namespace bastr_impl

using bastr_impl::kChunk;
using bastr_impl::Twiddles;

struct bastr_handle {
    bastr_params p{};
    Geo g{};
    int fp32 = 0;
    int allkmax = 0;
    int nshell = 0;            // shells 0..K cover every kept mode
    int64_t nstep = 0;
    double time = 0.0;
    bool have_state = false;
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // device buffers
    double2* u0 = nullptr;     // truncated state, FP64
    void* us = nullptr;        // stage input (compute precision)
    void* acc = nullptr;       // RK accumulator (compute precision)
    void* ma = nullptr;        // mixed fields after the first inverse pass(es)
    void* mb = nullptr;        // mixed fields before the last forward pass(es)
    void* mc = nullptr;        // 3D only: second mixed buffer
    double* phys = nullptr;    // physical fields for set/get (d * npts)
    double* vg_part = nullptr;
    double* en_part = nullptr;
    unsigned int* done = nullptr;  // completion tickets of last-block reductions [kTickets]
    int share_log2 = 0;            // plan: persistent grids use 1/2^share_log2 of the resident blocks
    bool ma_ready = false;         // 2D: MA already holds pass A of the next stage
    float* closure_buf = nullptr;  // 3D closure: tau_hat [3][n] (allocated on first use)
    double2* tr_buf = nullptr;     // transfer spectra: full complex grids (allocated on first use)
    double* tr_modes = nullptr;    // transfer spectra: per-mode values, item partials, shell sums
    double* hg_part = nullptr;     // initial-field generators: per-block partial sums
    double* sg_buf = nullptr;      // filtered fields / subgrid term: work buffers (allocated on first use)
    double2* sg_tw = nullptr;      // ... and the coarse grid's twiddle tables
    int sg_r = 0;                  // filter width the work buffers were sized for
    double2* pend = nullptr;       // (pending, factor) of a linear-forcing scale not yet applied
    unsigned long long* rng = nullptr;  // forcing calls so far: counter of the random-phase stream
    bool scale_pending = false;    // host view: a step with linear forcing ran since the last spectra
    double* rec = nullptr;     // [kChunk][R_COUNT]
    double* shells_dev = nullptr; // [kChunk][2][allkmax+1]
    // read-back of a batch in one copy (bastr_step_records): device gather buffer and pinned
    // host copy, [2 words + kChunk records + kChunk shell pairs]; allocated on first use
    double* stage_dev = nullptr;
    double* stage_host = nullptr;
    int64_t dev_bytes = 0;
    size_t n_state = 0;        // complex entries of the truncated state (all components)
    int n_vg_blocks = 0;
    int n_en_blocks = 0;
    int launches_per_step = 0;
    int chunk_used = 0;        // records written by the last async batch
    int64_t batch_n0 = 0;      // nstep and time at the start of that batch
    double batch_t0 = 0.0;
    Twiddles tw[3];            // per axis x, y, z
    size_t n_disk = 0;         // kept modes with |k| < K (state entries the spectra kernel reads, per component)
    // shell mode lists for the spectra (CSR): modes grouped by shell, cut into work items
    int* sp_modes = nullptr;
    int* sp_item_lo = nullptr;   // [n_items + 1]
    int* sp_shell_item = nullptr; // [nshell + 1]
    double* sp_item_part = nullptr;
    int n_items = 0;
    int band_lo = 0, band_hi = 0;   // the forcing band's entries in sp_modes (shell forcek)
    // per-launch profiling (bastr_profile): CUDA events around every launch
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    struct ProfRec { const char* name; size_t ev; double bytes; };
    std::vector<ProfRec> prof;
    std::vector<double> kn;
    std::vector<int64_t> ecount;
    // TMA tensor maps of the mixed-field buffers (2D, compute precision), built at creation
    CUtensorMap tm[5] = {};
    CUtensorMap tm3[4] = {};
    // the handle's device buffers as [begin, end) byte ranges: every tensor map is checked to lie
    // inside one at creation, and the index-checking build copies them to chk_table (Geo::chk)
    std::vector<std::pair<uint64_t, uint64_t>> ranges;
    CheckTable* chk_table = nullptr;
};

namespace bastr_impl {

// Slots of h->done: one per kind of last-block reduction (each stays 0 between launches), the
// batch's stop word and the kernels' error word (Geo::halt, Geo::err).
enum Ticket : int { T_SPECTRA = 0, T_HALT = 1, T_ERR = 2, kTickets = 4 };

// Tensor maps of a 2D handle (bastr_handle::tm):
//   TM_XA4 / TM_XA8  MA records [kx][ftot/4][y][4 fields] (ftot 4 / 8), box = 4 fields x 1 row x BK kx
//   TM_XB8           the (q1, q2) pieces of the second record (ftot 8), box = 2 fields x 1 row x BK kx
//   TM_YMB32/64      MB records [y/2][kx][2 rows][2 comps] in FP32 / FP64, box = 4 values x 1 kx x
//                    BY row pairs (the FP64 one also serves the state transform of FP32 handles)
// and of a 3D handle whose x pass stages with TMA (FP32, one warp's worth of threads per row):
//   TM_X3MB9/13      MB [z][kx][f][y] of the product fields (9) / with the velocity-gradient
//                    fields (13), FP32 values; box = 4 consecutive y x every f x every kx x 1 z
//   TM_Y3MA6/10      MA [kx][kyi][f][z] of the y-inverse pass's inputs (6 / 10 fields), FP32;
//                    box = 4 consecutive z x (fields + 1, the last read as zeros) x every kyi x 1 kx
enum TensorMapSlot : int { TM_XA4 = 0, TM_XA8 = 1, TM_XB8 = 2, TM_YMB32 = 3, TM_YMB64 = 4, kTensorMaps = 5 };
enum TensorMapSlot3 : int { TM_X3MB9 = 0, TM_X3MB13 = 1, TM_Y3MA6 = 2, TM_Y3MA10 = 3 };

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point (no link to libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// Records a device buffer of the handle (see bastr_handle::ranges); with the index-checking
// build the device copy of the table is refreshed, so a buffer allocated after creation is
// known to the checked kernels too.  Not for use while a stream is being captured.
inline cudaError_t track_alloc(bastr_handle* h, const void* p, size_t bytes) {
    if (!p) return cudaSuccess;
    h->ranges.push_back({(uint64_t)p, (uint64_t)p + bytes});
#ifdef BASTR_CHECKED
    if (!h->chk_table) {
        const cudaError_t e = cudaMalloc(&h->chk_table, sizeof(CheckTable));
        if (e != cudaSuccess) return e;
        h->g.chk = h->chk_table;
    }
    // BASTR_CHECK_SHRINK=n (tests of the checker itself): each registered range loses its last n
    // bytes, so in-bounds accesses near a buffer's end are reported (and go to the scratch line)
    // although no access leaves its buffer
    static const uint64_t shrink = [] {
        const char* v = std::getenv("BASTR_CHECK_SHRINK");
        return v ? (uint64_t)std::strtoull(v, nullptr, 10) : 0ull;
    }();
    CheckTable t{};
    t.n = (int)std::min<size_t>(h->ranges.size(), kCheckRanges);
    for (int i = 0; i < t.n; ++i) {
        t.lo[i] = h->ranges[i].first;
        t.hi[i] = std::max(h->ranges[i].first, h->ranges[i].second - std::min(shrink, h->ranges[i].second));
    }
    return cudaMemcpy(h->chk_table, &t, sizeof t, cudaMemcpyHostToDevice);
#else
    return cudaSuccess;
#endif
}

// A tiled tensor map of `rank` dimensions over a buffer of this GPU (dims innermost first, in
// elements of `elem` bytes; strides of dims 1.. in bytes); swizzle in bytes (0, 32, 64, 128).
// Out-of-range box elements read as zero.  Returns false when the driver rejects it, or when
// the map's extent (the last element's byte offset plus its size) reaches past the handle's
// buffer that holds `base`: the copy engine would read outside the allocation.
inline bool encode_map(const bastr_handle* h, CUtensorMap* m, const void* base, int elem, int rank,
                       const uint64_t* dims, const uint64_t* strides, const uint32_t* box, int swizzle) {
    uint64_t extent = (dims[0] - 1) * (uint64_t)elem + (uint64_t)elem;
    for (int i = 1; i < rank; ++i) extent += (dims[i] - 1) * strides[i - 1];
    const uint64_t a = (uint64_t)base;
    bool inside = false;
    for (const auto& r : h->ranges) inside = inside || (a >= r.first && a + extent <= r.second);
    if (!inside) return false;
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn) return false;
    cuuint64_t gd[5], gs[4];
    cuuint32_t bx[5], es[5];
    for (int i = 0; i < rank; ++i) {
        gd[i] = dims[i];
        bx[i] = box[i];
        es[i] = 1;
        if (i + 1 < rank) gs[i] = strides[i];
    }
    const CUtensorMapSwizzle sw = swizzle == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                                : swizzle == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                : swizzle == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE;
    const CUtensorMapDataType dt = elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return fn(m, dt, (cuuint32_t)rank, const_cast<void*>(base), gd, gs, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int fail(bastr_handle* h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(h, BASTR_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                              \
    } while (0)

inline bool is_pow2(int n) { return n >= 16 && n <= 2048 && (n & (n - 1)) == 0; }

// Brackets one kernel launch with CUDA events when profiling is on; `bytes` is the launch's
// algorithmic traffic (unique global reads plus writes of its inputs and outputs).
// Tracing: every pass launch, step batch and state transfer is an NVTX range named after it
// (header-only NVTX; the calls cost nothing measurable when no tool is attached).
#ifndef BASTR_NVTX
#define BASTR_NVTX 1
#endif
struct NvtxRange {
    explicit NvtxRange(const char* name) {
#if BASTR_NVTX
        nvtxRangePushA(name);
#else
        (void)name;
#endif
    }
    ~NvtxRange() {
#if BASTR_NVTX
        nvtxRangePop();
#endif
    }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct ProfScope {
    bastr_handle* h;
    size_t ev = 0;
    bool on = false;
    NvtxRange range;
    ProfScope(bastr_handle* hh, const char* name, double bytes) : h(hh), range(name) {
        if (!h->prof_on || h->ev_used + 2 > h->ev_pool.size()) return;
        ev = h->ev_used;
        h->ev_used += 2;
        on = true;
        cudaEventRecord(h->ev_pool[ev], h->stream);
        h->prof.push_back({name, ev, bytes});
    }
    ~ProfScope() {
        if (on) cudaEventRecord(h->ev_pool[ev + 1], h->stream);
    }
};

// Global traffic of the state-side reads/writes of one epilogue over n entries.
inline double epi_bytes(int epi, bool from_u0, double n, double cs) {
    switch (epi) {
        case EPI_STORE: return n * 16;
        case EPI_RK1: return n * 16 + 2 * n * cs;
        case EPI_RK2: return 2 * n * cs + n * 16 + 2 * n * cs;
        case EPI_RK3: return 2 * n * cs + n * 16 + n * 16;
        case EPI_CN_MID: return from_u0 ? n * 16 + n * cs : 2 * n * cs + n * 16;
        case EPI_CN_LAST: return n * cs + 2 * n * 16;
    }
    return 0;
}

template <typename T> const cplx<T>* twp(const Twiddles& t);
template <> inline const cplx<double>* twp<double>(const Twiddles& t) { return t.d64; }
template <> inline const cplx<float>* twp<float>(const Twiddles& t) { return t.d32; }

// Launches a kernel of the step on the handle's stream with programmatic dependent launch: it may
// start while the previous kernel drains, and waits for it on the device (pdl_wait).
template <typename... KArgs, typename... Args>
cudaError_t launch_k(bastr_handle* h, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                     Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = BASTR_PDL;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Enables the dynamic shared memory a kernel instance asks for and returns how many of its
// blocks fit on one SM.  The shared-memory limit is an attribute of the kernel, not of one
// launch size, and some kernels ask for a size that depends on the grid (the 3D y-forward pass's
// tile follows KY): the limit set per (device, kernel) only ever grows, so a smaller request
// never lowers it under a larger one made before.  Occupancy is cached per (device, kernel,
// size).
inline std::mutex g_prep_mu;
inline std::map<std::tuple<int, const void*, size_t>, int> g_prepped;
inline std::map<std::pair<int, const void*>, size_t> g_smem_limit;
inline int g_num_sms[64] = {};
template <typename K> cudaError_t prep(K kernel, size_t smem, int nt = 0, int* blocks_per_sm = nullptr) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const auto key = std::make_tuple(dev, (const void*)kernel, smem);
    std::lock_guard<std::mutex> lk(g_prep_mu);
    if (smem > 48 * 1024) {
        size_t& limit = g_smem_limit[std::make_pair(dev, (const void*)kernel)];
        if (smem > limit) {
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            limit = smem;
        }
    }
    auto it = g_prepped.find(key);
    if (it == g_prepped.end()) {
        int nb = 1;
        if (nt > 0) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, nt, smem);
            if (e != cudaSuccess) return e;
            if (nb < 1) nb = 1;
        }
        if (dev >= 0 && dev < 64 && g_num_sms[dev] == 0) {
            e = cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
        }
        it = g_prepped.emplace(key, nb).first;
    }
    if (blocks_per_sm) *blocks_per_sm = it->second;
    return cudaSuccess;
}

// Grid of a persistent pass: as many blocks as fit on the device, at most one per work item.
// The handle's plan may restrict its persistent grids to 1/2^share of that (an ensemble runs
// many handles at once, each on a share of the SMs).
template <typename K> cudaError_t persistent_grid(const bastr_handle* h, K kernel, size_t smem, int nt, int nitems,
                                                  int* grid) {
    int nb = 1;
    cudaError_t e = prep(kernel, smem, nt, &nb);
    if (e != cudaSuccess) return e;
    int dev = 0;
    cudaGetDevice(&dev);
    const int sms = (dev >= 0 && dev < 64 && g_num_sms[dev] > 0) ? g_num_sms[dev] : 148;
    *grid = std::max(1, std::min(nitems, (nb * sms) >> h->share_log2));
    return cudaSuccess;
}

#define SIZE_CASES(N, ...)                      \
    switch (N) {                                 \
        case 16: { constexpr int NN = 16; __VA_ARGS__; } break;     \
        case 32: { constexpr int NN = 32; __VA_ARGS__; } break;     \
        case 64: { constexpr int NN = 64; __VA_ARGS__; } break;     \
        case 128: { constexpr int NN = 128; __VA_ARGS__; } break;   \
        case 256: { constexpr int NN = 256; __VA_ARGS__; } break;   \
        case 512: { constexpr int NN = 512; __VA_ARGS__; } break;   \
        case 1024: { constexpr int NN = 1024; __VA_ARGS__; } break; \
        case 2048: { constexpr int NN = 2048; __VA_ARGS__; } break; \
        default: return cudaErrorInvalidValue;   \
    }

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

#define SIZE_CASES3(N, ...)                                  \
    switch (N) {                                              \
        case 16: { constexpr int NN = 16; __VA_ARGS__; } break;     \
        case 32: { constexpr int NN = 32; __VA_ARGS__; } break;     \
        case 64: { constexpr int NN = 64; __VA_ARGS__; } break;     \
        case 128: { constexpr int NN = 128; __VA_ARGS__; } break;   \
        case 256: { constexpr int NN = 256; __VA_ARGS__; } break;   \
        case 512: { constexpr int NN = 512; __VA_ARGS__; } break;   \
        default: return cudaErrorInvalidValue;                \
    }

// Mixed-field buffer sizes (bytes) of a 3D handle for compute element size cs.
inline void sizes3d(bastr_handle* h, size_t cs, size_t& ma, size_t& mb, size_t& mc) {
    const Geo& g = h->g;
    const size_t K = g.K, KY = g.KY, NY = g.ny, NZ = g.nz;
    const size_t c64 = sizeof(double2);
    ma = std::max({K * NZ * KY * 10 * cs, K * KY * NZ * 3 * cs, K * NZ * KY * 3 * c64, K * KY * NZ * 3 * c64});
    mb = std::max(NZ * NY * K * 13 * cs, NZ * NY * K * 3 * c64);
    mc = std::max(NZ * K * NY * 3 * cs, NZ * K * NY * 3 * c64);
}

// One right-hand-side evaluation F(u_s) with its stage combination (epi: EpiMode), and the
// FP64 physical <-> truncated spectral transforms of the state; defined per dimension and
// compute precision in steps2d_*.cu / steps3d_*.cu.
template <typename T> cudaError_t rhs2d(bastr_handle* h, int epi, bool from_u0, bool vg);
template <typename T> cudaError_t rhs3d(bastr_handle* h, int epi, bool from_u0, bool vg);
extern template cudaError_t rhs2d<float>(bastr_handle*, int, bool, bool);
extern template cudaError_t rhs2d<double>(bastr_handle*, int, bool, bool);
extern template cudaError_t rhs3d<float>(bastr_handle*, int, bool, bool);
extern template cudaError_t rhs3d<double>(bastr_handle*, int, bool, bool);
cudaError_t state2d_to_spectral(bastr_handle* h);
cudaError_t state2d_to_physical(bastr_handle* h);
cudaError_t state3d_to_spectral(bastr_handle* h);
cudaError_t state3d_to_physical(bastr_handle* h);

}  // namespace bastr_impl
