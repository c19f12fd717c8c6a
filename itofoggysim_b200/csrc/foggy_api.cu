// C ABI of libfoggy_b200 (include/foggy_gpu.h).  Host orchestration of the device kernels:
// scene upload, Mie coefficients, right-hand side, operator, device GMRES, cross-sections and
// the octree keys.  Every entry point returns a status code; no exception crosses the ABI.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "foggy_kernels.cuh"

using namespace foggy;

namespace {
const double kPi = 3.14159265358979323846264338327950288;
// error of the calling thread's last failing foggy_create / handle-less call (per thread, as
// errno, so that threads creating handles side by side read their own message)
thread_local std::string g_err;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// NVTX range over a scope: the phases of a solve (scene, pair tables, operator applications,
// ML-FMM passes) on a profiler's timeline, as the reference's _TRACE_ timings per pass
// (libmlfmm/src/lib/lib_ml_fmm.f90:339-372).  Without a tool attached it costs a branch.
struct Trace {
    explicit Trace(const char* name) { nvtxRangePushA(name); }
    ~Trace() { nvtxRangePop(); }
    Trace(const Trace&) = delete;
    Trace& operator=(const Trace&) = delete;
};

}  // namespace

struct foggy_handle_s {
    foggy_params prm{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;   // the device's stream-ordered pool (device_pool)
    std::string err;
    std::vector<void*> allocs;   // every device allocation, freed in destroy
    std::map<void*, size_t> alloc_bytes;   // their sizes, returned to the budget when freed
    std::vector<void*> direct_allocs;      // the ones made by cudaMalloc (kPoolMax and above)
    size_t bytes_in_use = 0;
    size_t budget = 0;

    // scene (host)
    int N = 0, NP = 0, pmax = 0, pg = 0;
    std::vector<double> centres;
    std::vector<int> pidx, p_s, p_param, couple;
    std::vector<int64_t> off;
    int64_t n_unk = 0;
    std::vector<double> mre, mim, radius;
    std::vector<int> nr;
    // scene (device)
    double* d_centres = nullptr;
    int* d_p = nullptr;
    int64_t* d_off = nullptr;
    cplx* d_an = nullptr;
    cplx* d_bn = nullptr;
    cplx* d_an_p = nullptr;
    cplx* d_bn_p = nullptr;
    int* d_couple = nullptr;
    double* d_g = nullptr;
    // translation tables
    int tab_pmax = -1;
    int ax_pmax = 0;   // degree of the axial (3j) tables, built on demand
    int32_t* d_axoff = nullptr;
    double* d_ga = nullptr;
    double* d_gb = nullptr;
    int64_t* d_koff = nullptr;
    double* d_gab = nullptr;
    int64_t* d_koffS = nullptr;   // scalar Gaunt table (build_scalar_gaunt_qmajor)
    double* d_gs = nullptr;
    int gs_nm = 0;
    // per-pair scalar coaxial coefficients (geometry only), when they fit the memory budget
    cplx* d_stab = nullptr;
    cplxf* d_stab32 = nullptr;   // the pair tables in single precision (mixed-precision solves)
    bool stab32_ready = false;
    int64_t* d_pair_off = nullptr;
    int stab_z = 0;
    bool stab_ready = false;
    double* d_sqrt_binom = nullptr;
    double* d_rs = nullptr;
    double* d_irs = nullptr;
    double* d_rj = nullptr;
    double* d_delta = nullptr;    // d^j(pi/2), build_delta_table
    float* d_delta32 = nullptr;   // the same in single precision
    int K = 0;
    // operator launches: (target bucket, source bucket) pairs of truncation-order buckets
    std::vector<DirectBucket> launches_direct;
    int* d_bucket_lists = nullptr;
    int nbuckets = 0, cmax = 1;
    // waves and right-hand side
    std::vector<WaveDev> waves;
    std::vector<GaussDev> beams;
    bool rhs_ready = false;
    cplx* d_b = nullptr;
    cplx* d_pq = nullptr;
    // operator scratch
    int chunks_unused = 0;
    cplx* d_partial = nullptr;
    cplx* d_tmp_in = nullptr;    // ragged work vectors
    cplx* d_tmp_out = nullptr;
    cplx* d_ref_a = nullptr;     // reference-layout staging (host-pointer calls)
    cplx* d_ref_b = nullptr;
    // GMRES workspace
    int ws_restart = 0;
    cplx* d_V = nullptr;
    cplx* d_w = nullptr;
    cplx* d_x = nullptr;
    cplx* d_r = nullptr;
    cplx* d_H = nullptr;
    cplx* d_cs = nullptr;
    double* d_sn = nullptr;
    cplx* d_gv = nullptr;
    cplx* d_h = nullptr;
    cplx* d_c = nullptr;
    cplx* d_y = nullptr;
    cplx* d_part = nullptr;
    double* d_npart = nullptr;
    double* d_scal = nullptr;    // [0] hn, [1] beta, [2] res_est, [3] bnorm
    int* d_flags = nullptr;
    double* h_pin = nullptr;     // pinned: res_est, beta, bnorm
    int* h_pin_flags = nullptr;
    double last_berr = -1.0;
    int64_t launches = 0;        // kernels launched by the current solve
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evm0 = nullptr, evm1 = nullptr;
    std::vector<cudaEvent_t> ev_pool;   // operator timing events of gmres(), reused across solves
    cudaEvent_t ev_step[2] = {nullptr, nullptr};   // read-back of the Arnoldi steps in flight
    // tree
    unsigned long long* d_keys = nullptr;
    int* d_idx = nullptr;
    unsigned long long* d_keys_sorted = nullptr;
    int* d_idx_sorted = nullptr;
    int tree_lmax = 0, tree_lmin = 0;
    bool tree_ready = false;
    // ML-FMM: octree lists, box coefficients, final-summation slabs
    bool fmm_ready = false;
    FmmTree fmm;
    double fmm_xmin[3] = {0, 0, 0};
    double* d_fmm_c = nullptr;       // box centres
    int* d_fmm_p = nullptr;          // box orders (the global order)
    int64_t* d_fmm_off = nullptr;    // box coefficient offsets
    cplx* d_fmm_C = nullptr;         // outgoing coefficients of every box
    cplx* d_fmm_D = nullptr;         // incoming coefficients of every box
    int* d_fmm_list = nullptr;       // CSR lists of the passes, concatenated
    int fmm_lofs[12] = {0};          // offsets of (ptr, idx) of: aggregation, children, I4, parent,
                                     // box-to-sphere, near field
    int fmm_ltotal = 0;              // entries of the twelve lists
    cplx* d_fmm_slab = nullptr;      // box-to-sphere and near-field sums, 2 x n_unk
    cplx* d_fmm_chunks = nullptr;    // partial sums of passes split into source chunks
    cplx* d_fmm_chunks2 = nullptr;   // the same for the near-field pass, which runs beside the others
    cudaStream_t side = nullptr;     // the near-field pass's stream, joined before the sum
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cplx* d_fmm_tab = nullptr;       // coaxial blocks of the passes' distinct translations
    int64_t* d_fmm_taboff = nullptr; // per list entry, its block's offset in d_fmm_tab
    cplxf* d_fmm_tab32 = nullptr;    // the blocks in single precision (mixed-precision solves)
    bool fmm_tab_ready = false;
    int fmm_pmax = 0;                // largest box order (the global order, or per-level orders)
    std::vector<int> fmm_list_host;  // the twelve pass lists, read back once (chunk counts)
    int fmm_tab_key[5] = {0, 0, 0, 0, 0};   // (convention, z_coupling, z_translation_gt_r, on, precision)
    // several right-hand sides in one block (foggy_solve_block, foggy_matvec_block): vectors of
    // nrhs slots, n_unk entries apart
    int blk_nrhs = 0, blk_m = 0;
    cplx* d_bV = nullptr;            // Krylov basis: vector i of slot b at (i nrhs + b) n_unk
    cplx* d_bW = nullptr;            // operator output
    cplx* d_bX = nullptr;            // iterates, slot order
    cplx* d_bB = nullptr;            // right-hand sides, slot order
    cplx* d_bR = nullptr;            // residuals
    cplx* d_bsmall = nullptr;        // H, cs, g, h, c, y of every slot, dots partials
    double* d_breal = nullptr;       // sn, norms, betas, tolerances, estimates, norm partials
    int* d_bint = nullptr;           // live, kend, flags
};

namespace {

int fail(foggy_handle h, int code, const std::string& msg) {
    if (h) {
        h->err = msg;
    } else {
        g_err = msg;
    }
    return code;
}

#define CK(h, call)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(h, FOGGY_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CKL(h)                                                                              \
    do {                                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                \
        if (e_ != cudaSuccess)                                                              \
            return fail(h, FOGGY_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// Host to device on the handle's stream, then wait.  The kernels that read dst run on that
// non-blocking stream, which a blocking cudaMemcpy on the legacy stream does not order (from
// pageable memory it may return before the DMA lands), and the source is often a temporary.
static cudaError_t d2h(foggy_handle h, void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(h->stream) : e;
}

static cudaError_t h2d(foggy_handle h, void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(h->stream) : e;
}

// Device memory of every handle comes from one stream-ordered pool per device: allocations and
// frees are ordered on the handle's stream, so a handle that sets up or tears down while others
// solve does not synchronise the device (cudaMalloc and cudaFree would serialise every stream of
// co-resident solves).  Memory freed to the pool beyond kPoolKeep bytes goes back to the driver at
// the next synchronisation; a freed block is reused by another stream only once its free has run
// (no dependencies between handles' streams are inserted).
constexpr uint64_t kPoolKeep = 4ull << 30;
// Allocations of kPoolMax bytes and more (the pair tables and Krylov bases of large scenes, made
// once per scene) come from cudaMalloc instead: measured on the 2000-sphere scene, the operator runs
// 4 % faster over cudaMalloc's mapping of its 107 GB of pair tables than over the pool's, and the
// pool takes 0.6-1.5 s longer to give them back.
constexpr uint64_t kPoolMax = 1ull << 30;

cudaMemPool_t device_pool(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = kPoolKeep;
    int no = 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    pools[device] = pool;
    return pool;
}

// per-call device scratch, stream-ordered like dalloc (not counted in the handle's budget)
template <class T>
cudaError_t talloc(foggy_handle h, T** p, size_t bytes) {
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), std::max<size_t>(bytes, 16), h->pool, h->stream);
}
inline void tfree(foggy_handle h, void* p) {
    if (p) cudaFreeAsync(p, h->stream);
}

// The handles' small page-locked read-back buffers, 256-byte slots carved from 1 MiB blocks that
// are allocated once and kept: cudaMallocHost per handle would serialise the device's streams.
constexpr size_t kPinSlot = 256;
struct PinnedSlots {
    std::mutex mu;
    std::vector<char*> free;
};
PinnedSlots& pinned_slots() {
    static PinnedSlots P;
    return P;
}
char* pinned_slot() {
    PinnedSlots& P = pinned_slots();
    std::lock_guard<std::mutex> lk(P.mu);
    if (P.free.empty()) {
        char* block = nullptr;
        if (cudaMallocHost(reinterpret_cast<void**>(&block), 1 << 20) != cudaSuccess) return nullptr;
        for (size_t i = 0; i < (size_t(1) << 20) / kPinSlot; ++i) P.free.push_back(block + i * kPinSlot);
    }
    char* q = P.free.back();
    P.free.pop_back();
    return q;
}
void pinned_release(char* q) {
    if (!q) return;
    PinnedSlots& P = pinned_slots();
    std::lock_guard<std::mutex> lk(P.mu);
    P.free.push_back(q);
}

template <class T>
int dalloc(foggy_handle h, T** p, size_t count) {
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    if (h->budget && h->bytes_in_use + bytes > h->budget)
        return fail(h, FOGGY_ERR_NOMEM, "device memory budget exceeded (" + std::to_string(h->bytes_in_use + bytes) +
                                            " > " + std::to_string(h->budget) + " bytes)");
    const bool direct = bytes >= kPoolMax;
    cudaError_t e = direct ? cudaMalloc(reinterpret_cast<void**>(p), bytes)
                           : cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, h->pool, h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(h, FOGGY_ERR_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    if (direct) h->direct_allocs.push_back(*p);
    h->allocs.push_back(*p);
    h->alloc_bytes[*p] = bytes;
    h->bytes_in_use += bytes;
    return FOGGY_OK;
}

template <class T>
void dfree(foggy_handle h, T*& p) {
    if (!p) return;
    auto it = std::find(h->allocs.begin(), h->allocs.end(), (void*)p);
    if (it != h->allocs.end()) h->allocs.erase(it);
    auto sz = h->alloc_bytes.find((void*)p);
    if (sz != h->alloc_bytes.end()) {
        h->bytes_in_use -= std::min(h->bytes_in_use, sz->second);
        h->alloc_bytes.erase(sz);
    }
    auto d = std::find(h->direct_allocs.begin(), h->direct_allocs.end(), (void*)p);
    if (d != h->direct_allocs.end()) {
        h->direct_allocs.erase(d);
        cudaFree(p);   // waits for the device, so for the stream's uses of p
    } else {
        cudaFreeAsync(p, h->stream);
    }
    p = nullptr;
}

#define TRY(x)                      \
    do {                            \
        int r_ = (x);               \
        if (r_ != FOGGY_OK) return r_; \
    } while (0)

void to_spherical(const double* c, double* rho, double* theta, double* phi) {
    double r = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    *rho = r;
    *theta = (r == 0.0) ? 0.0 : std::acos(c[2] / r);
    *phi = (c[0] == 0.0 && c[1] == 0.0) ? 0.0 : std::atan2(c[1], c[0]);
}

double wavenumber(const foggy_params& p) { return 2.0 * kPi * p.n_medium / p.lambda_0; }

SceneView scene_view(foggy_handle h) {
    SceneView s;
    s.n = h->N;
    s.pmax = h->pmax;
    s.k = wavenumber(h->prm);
    s.centres = h->d_centres;
    s.p = h->d_p;
    s.off = h->d_off;
    s.an = h->d_an;
    s.bn = h->d_bn;
    s.couple = h->d_couple;
    return s;
}

// Host tables that depend on the truncation degree alone: the scalar Gaunt sums, d-table helper
// tables, d^j(pi/2) and g_nm.  Built once per degree in the process and shared by every handle (a
// solve server creates one handle per request, so they are not rebuilt per request).
struct OrderTables {
    int K = 0;
    std::vector<int64_t> koffS;
    std::vector<double> gs, sb, rs, irs, rj, delta, g;
    std::vector<float> delta32;
};

std::shared_ptr<const OrderTables> order_tables(int pmax) {
    static std::mutex mu;
    static std::map<int, std::shared_ptr<const OrderTables>> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(pmax);
    if (it != cache.end()) return it->second;
    auto t = std::make_shared<OrderTables>();
    const int K = pmax + 1;   // the scalar-coefficient relation reads sqrt((nu+1)^2 - k^2) at nu = pmax
    t->K = K;
    build_scalar_gaunt_qmajor(pmax + 1, t->koffS, t->gs);
    t->sb.assign((size_t)(K + 1) * (2 * K + 1), 0.0);
    t->rs.assign((size_t)(K + 1) * (K + 1), 0.0);
    t->irs.assign((size_t)(K + 1) * (K + 1), 0.0);
    t->rj.assign(2 * (size_t)(K + 2), 0.0);
    for (int J = 0; J <= K; ++J)
        for (int m = -J; m <= J; ++m) {
            long double c = 1.0L;   // C(2J, J+m)
            int a = J + m, b = J - m;
            for (int i = 1; i <= b; ++i) c = c * (a + i) / i;
            t->sb[(size_t)J * (2 * K + 1) + (m + K)] = (double)std::sqrt(c);
        }
    for (int j = 0; j <= K; ++j)
        for (int m = 0; m <= j; ++m) {
            double v = std::sqrt((double)j * j - (double)m * m);
            t->rs[(size_t)j * (K + 1) + m] = v;
            t->irs[(size_t)j * (K + 1) + m] = (v > 0) ? 1.0 / v : 0.0;
        }
    for (int j = 2; j <= K; ++j) {
        t->rj[2 * j] = 1.0 / ((double)j * (j - 1));
        t->rj[2 * j + 1] = 1.0 / ((double)(j - 1) * (2.0 * j - 1.0));
    }
    build_delta_table(pmax, t->delta);
    t->delta32.assign(t->delta.begin(), t->delta.end());
    build_g_table(pmax, t->g);
    cache[pmax] = t;
    return t;
}

// the operator's order tables for degrees <= pmax on the device
int ensure_tables(foggy_handle h, int pmax) {
    if (h->tab_pmax >= pmax) return FOGGY_OK;
    for (double** q : {&h->d_gs, &h->d_sqrt_binom, &h->d_rs, &h->d_irs, &h->d_rj, &h->d_g, &h->d_delta}) dfree(h, *q);
    dfree(h, h->d_koffS);
    dfree(h, h->d_delta32);
    const std::shared_ptr<const OrderTables> t = order_tables(pmax);
    auto up = [&](auto** d, const auto& v) -> int {
        TRY(dalloc(h, d, v.size()));
        CK(h, cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice, h->stream));
        return FOGGY_OK;
    };
    TRY(up(&h->d_koffS, t->koffS));
    TRY(up(&h->d_gs, t->gs));
    TRY(up(&h->d_sqrt_binom, t->sb));
    TRY(up(&h->d_rs, t->rs));
    TRY(up(&h->d_irs, t->irs));
    TRY(up(&h->d_rj, t->rj));
    TRY(up(&h->d_delta, t->delta));
    TRY(up(&h->d_delta32, t->delta32));
    TRY(up(&h->d_g, t->g));
    // the cached host vectors outlive the copies (the cache keeps them), so no synchronisation here
    h->gs_nm = pmax + 1;
    h->K = t->K;
    h->tab_pmax = pmax;
    h->ax_pmax = 0;
    return FOGGY_OK;
}

// 3j (axial) tables of the explicit translation coefficients, for degrees <= the order tables'
int ensure_axial_tables(foggy_handle h) {
    if (h->ax_pmax >= h->tab_pmax) return FOGGY_OK;
    dfree(h, h->d_axoff);
    dfree(h, h->d_ga);
    dfree(h, h->d_gb);
    dfree(h, h->d_koff);
    dfree(h, h->d_gab);
    AxialTables t;
    build_axial_tables(h->tab_pmax, t);
    std::vector<int64_t> koff;
    std::vector<double> gab;
    build_axial_tables_qmajor(t, koff, gab);
    TRY(dalloc(h, &h->d_axoff, t.offset.size()));
    TRY(dalloc(h, &h->d_ga, t.ga.size()));
    TRY(dalloc(h, &h->d_gb, t.gb.size()));
    TRY(dalloc(h, &h->d_koff, koff.size()));
    TRY(dalloc(h, &h->d_gab, gab.size()));
    CK(h, h2d(h, h->d_koff, koff.data(), koff.size() * sizeof(int64_t)));
    CK(h, h2d(h, h->d_gab, gab.data(), gab.size() * sizeof(double)));
    CK(h, h2d(h, h->d_axoff, t.offset.data(), t.offset.size() * sizeof(int32_t)));
    CK(h, h2d(h, h->d_ga, t.ga.data(), t.ga.size() * sizeof(double)));
    CK(h, h2d(h, h->d_gb, t.gb.data(), t.gb.size() * sizeof(double)));
    h->ax_pmax = h->tab_pmax;
    return FOGGY_OK;
}

DTabs dtabs(foggy_handle h) {
    DTabs t;
    t.sqrt_binom = h->d_sqrt_binom;
    t.rs = h->d_rs;
    t.irs = h->d_irs;
    t.rj = h->d_rj;
    t.K = h->K;
    return t;
}

DirectArgs direct_args(foggy_handle h, const cplx* x) {
    DirectArgs a;
    a.sc = scene_view(h);
    a.delta = h->d_delta;
    a.g = SGaunt{h->d_koffS, h->d_gs, h->gs_nm};
    a.dt = dtabs(h);
    // tables of another radial function are never read
    const bool zok = h->stab_z == h->prm.z_coupling;
    a.pt.stab = (zok && h->stab_ready) ? h->d_stab : nullptr;
    a.pt.stab32 = (zok && h->stab32_ready) ? h->d_stab32 : nullptr;
    a.delta32 = h->d_delta32;
    a.fp32 = 0;
    a.pt.pair_off = h->d_pair_off;
    a.z = h->prm.z_coupling;
    a.x = x;
    a.partial = h->d_partial;
    a.cmax = h->cmax;
    a.n_unk = h->n_unk;
    return a;
}

// Upper bounds of the truncation-order buckets: steps of 4 degrees up to the largest order a
// sphere may have (kMaxDegree, the reference's cap), so every sphere is in one bucket.
constexpr int kBucketBounds[] = {0, 4, 8, 12, 16, 20, 24, 28, 32, 36, 40, 44, 48};
constexpr int kNumBounds = (int)(sizeof(kBucketBounds) / sizeof(kBucketBounds[0]));
static_assert(kBucketBounds[kNumBounds - 1] >= kMaxDegree, "every order needs a bucket");

// Truncation-order buckets of the spheres and the (target bucket, source bucket) launches of
// the direct operator.  Bucket upper bounds grow in steps of 4 degrees; each launch gets enough
// CTAs per target to fill the GPU.
int plan_direct(foggy_handle h) {
    const int* bounds = kBucketBounds;
    std::vector<std::vector<int>> members;
    std::vector<int> bp;
    for (int bi = 1; bi < kNumBounds; ++bi) {
        std::vector<int> v;
        for (int j = 0; j < h->N; ++j)
            if (h->p_s[j] > bounds[bi - 1] && h->p_s[j] <= bounds[bi]) v.push_back(j);
        if (!v.empty()) {
            int pm = 0;
            for (int j : v) pm = std::max(pm, h->p_s[j]);
            members.push_back(v);
            bp.push_back(pm);
        }
    }
    h->nbuckets = (int)members.size();
    const int want = 148 * 6;
    h->cmax = 1;
    std::vector<int> chunks(h->nbuckets);
    for (int t = 0; t < h->nbuckets; ++t) {
        int nt = (int)members[t].size();
        int c = std::max(1, std::min(32, (want + nt - 1) / nt));
        chunks[t] = c;
        h->cmax = std::max(h->cmax, c);
    }
    std::vector<int> flat;
    std::vector<int> start;
    for (auto& v : members) {
        start.push_back((int)flat.size());
        flat.insert(flat.end(), v.begin(), v.end());
    }
    dfree(h, h->d_bucket_lists);
    TRY(dalloc(h, &h->d_bucket_lists, flat.size()));
    CK(h, h2d(h, h->d_bucket_lists, flat.data(), flat.size() * sizeof(int)));
    h->launches_direct.clear();
    for (int t = 0; t < h->nbuckets; ++t)
        for (int s = 0; s < h->nbuckets; ++s) {
            DirectBucket b;
            b.targets = h->d_bucket_lists + start[t];
            b.ntargets = (int)members[t].size();
            b.sources = h->d_bucket_lists + start[s];
            b.nsources = (int)members[s].size();
            b.slab = s * h->cmax;
            b.chunks = std::min(chunks[t], std::max(1, b.nsources));
            b.pp = std::max(bp[t], bp[s]);
            h->launches_direct.push_back(b);
        }
    return FOGGY_OK;
}

// The pair tables over groups of pairs (k_pair_tables.cu).  The pairs are grouped by
// M2 = max(p_s, p_t) + 2 (a group shares its Gaunt coefficients) and, within a group, ordered by
// min(p_s, p_t) from the largest down, so that the pairs of a tile have blocks of similar size.
// FP64 tables (fp64): tiles of kPairs64 pairs, their row tiles in runs of 16, summed on the CUDA
// cores.  FP32 tables (fp32): tiles of 64 pairs (16 above order 34), runs of 8 row tiles, as
// tensor-core products.  One CTA per run.
int build_pair_tables(foggy_handle h, const SGaunt& g, bool fp64, bool fp32) {
    const int n = h->N;
    const int nm = h->pmax + 3;   // M2 = 3..pmax + 2, min order 1..pmax
    std::vector<int64_t> start((size_t)nm * nm + 1, 0);
    auto bucket = [&](int ps, int pt) { return (size_t)(std::max(ps, pt) + 2) * nm + (nm - 1 - std::min(ps, pt)); };
    for (int s = 0; s < n; ++s)
        for (int t = s + 1; t < n; ++t) start[bucket(h->p_s[s], h->p_s[t]) + 1]++;
    for (size_t b = 0; b < (size_t)nm * nm; ++b) start[b + 1] += start[b];
    const int64_t npairs = start[(size_t)nm * nm];
    std::vector<int2> pairs((size_t)npairs);
    {
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int s = 0; s < n; ++s)
            for (int t = s + 1; t < n; ++t) pairs[(size_t)fill[bucket(h->p_s[s], h->p_s[t])]++] = make_int2(s, t);
    }
    auto tiles_of = [&](int64_t first) {
        const int2 st = pairs[(size_t)first];
        return (int)((pair_block_size(h->p_s[st.x], h->p_s[st.y]) + 127) / 128);
    };
    std::vector<TcGroup> groups;
    std::vector<int64_t> gbeg, gend;
    int64_t a_floats = 0;
    for (int M2 = 3; M2 < nm; ++M2) {
        const int64_t g0 = start[(size_t)M2 * nm], g1 = start[(size_t)(M2 + 1) * nm];
        if (g0 == g1) continue;
        TcGroup gr;
        gr.M2 = M2;
        gr.K = tc_group_k(M2);
        gr.np = tc_group_pairs(gr.K);
        gr.mtiles = tiles_of(g0);
        gr.a_off = a_floats;
        if (fp32) a_floats += (int64_t)gr.mtiles * 2 * 128 * gr.K;
        groups.push_back(gr);
        gbeg.push_back(g0);
        gend.push_back(g1);
    }
    // tiles of np pairs per group, their row tiles in runs of `run`; tile0[i] = first tile of group i
    auto make_tiles = [&](bool tc, int run, std::vector<TcTile>& tiles, std::vector<int>& tile0) {
        for (size_t i = 0; i < groups.size(); ++i) {
            tile0.push_back((int)tiles.size());
            const int np = tc ? groups[i].np : kPairs64;
            for (int64_t f = gbeg[i]; f < gend[i]; f += np) {
                const int mt = tiles_of(f), cnt = (int)std::min<int64_t>(np, gend[i] - f);
                for (int m = 0; m < mt; m += run) tiles.push_back(TcTile{(int)i, (int)f, cnt, m, std::min(mt, m + run)});
            }
        }
        tile0.push_back((int)tiles.size());
    };
    std::vector<TcTile> t64, t32;
    std::vector<int> t64_0, t32_0;
    if (fp64) make_tiles(false, 16, t64, t64_0);
    if (fp32) make_tiles(true, 8, t32, t32_0);
    int2* d_pairs = nullptr;
    TcTile* d_t64 = nullptr;
    TcTile* d_t32 = nullptr;
    TcGroup* d_groups = nullptr;
    float* d_a = nullptr;
    int* d_err = nullptr;
    auto fin = [&](int rc) {
        tfree(h, d_pairs);
        tfree(h, d_t64);
        tfree(h, d_t32);
        tfree(h, d_groups);
        tfree(h, d_a);
        tfree(h, d_err);
        return rc;
    };
    if (talloc(h, &d_pairs, pairs.size() * sizeof(int2)) != cudaSuccess ||
        talloc(h, &d_t64, std::max<size_t>(t64.size(), 1) * sizeof(TcTile)) != cudaSuccess ||
        talloc(h, &d_t32, std::max<size_t>(t32.size(), 1) * sizeof(TcTile)) != cudaSuccess ||
        talloc(h, &d_groups, groups.size() * sizeof(TcGroup)) != cudaSuccess ||
        talloc(h, &d_a, (size_t)std::max<int64_t>(a_floats, 1) * sizeof(float)) != cudaSuccess ||
        talloc(h, &d_err, sizeof(int)) != cudaSuccess)
        return fin(fail(h, FOGGY_ERR_NOMEM, "pair tables: device scratch"));
    cudaError_t e = h2d(h, d_pairs, pairs.data(), pairs.size() * sizeof(int2));
    if (e == cudaSuccess && fp64) e = h2d(h, d_t64, t64.data(), t64.size() * sizeof(TcTile));
    if (e == cudaSuccess && fp32) e = h2d(h, d_t32, t32.data(), t32.size() * sizeof(TcTile));
    if (e == cudaSuccess) e = h2d(h, d_groups, groups.data(), groups.size() * sizeof(TcGroup));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return fin(fail(h, FOGGY_ERR_CUDA, std::string("pair tables: ") + cudaGetErrorString(e)));
    if (fp64) {
        PairArgs pa{scene_view(h), h->prm.z_coupling, d_pairs, d_t64, d_groups, g, h->d_pair_off, h->d_stab};
        for (size_t i = 0; i < groups.size(); ++i) {
            launch_pair_s_group(pa, t64_0[i], t64_0[i + 1] - t64_0[i], groups[i].M2, h->stream);
            h->launches += 1;
        }
    }
    if (fp32) {
        TcArgs ta{scene_view(h), h->prm.z_coupling, d_pairs, d_t32, d_groups, d_a, h->d_pair_off, h->d_stab32, d_err};
        for (size_t i = 0; i < groups.size(); ++i) {
            launch_tc_pack_a(g, groups[i], d_a, h->stream);
            launch_pair_tc(ta, t32_0[i], t32_0[i + 1] - t32_0[i], groups[i].K, groups[i].np, h->stream);
            h->launches += 2;
        }
    }
    e = cudaGetLastError();
    int err = 0;
    if (e == cudaSuccess) e = d2h(h, &err, d_err, sizeof(int));
    if (e != cudaSuccess) return fin(fail(h, FOGGY_ERR_CUDA, std::string("pair tables: ") + cudaGetErrorString(e)));
    if (err) return fin(fail(h, FOGGY_ERR_CUDA, "tensor-core pair tables: a wait for a copy or the tensor core timed out"));
    return fin(FOGGY_OK);
}

// Scalar coaxial coefficients of all unordered sphere pairs (geometry and z only), built once
// and read by every operator application.  Skipped when they do not fit (pair_tables = 0) or
// when switched off (pair_tables = -1).  The double-precision tables are FP64 sums on the CUDA
// cores, the single-precision ones tensor-core products in 3xTF32 (build_pair_tables).
int ensure_pair_tables(foggy_handle h) {
    const bool mixed = h->prm.precision == 1;
    if (h->prm.pair_tables < 0 || h->N < 2) {
        h->stab_ready = false;
        h->stab32_ready = false;
        return FOGGY_OK;
    }
    // both precisions' tables were built for one radial function; a new one invalidates both,
    // whichever of them this call rebuilds
    if (h->stab_z != h->prm.z_coupling) {
        h->stab_ready = false;
        h->stab32_ready = false;
    }
    if (mixed ? h->stab32_ready : h->stab_ready) return FOGGY_OK;
    const int64_t npairs = (int64_t)h->N * (h->N - 1) / 2;
    // total size from the counts of each truncation order
    std::vector<int64_t> cnt(h->pmax + 1, 0);
    for (int j = 0; j < h->N; ++j) cnt[h->p_s[j]]++;
    int64_t tot = 0;
    for (int a = 1; a <= h->pmax; ++a)
        for (int b = a; b <= h->pmax; ++b) {
            if (!cnt[a] || !cnt[b]) continue;
            int64_t pairs = (a == b) ? cnt[a] * (cnt[a] - 1) / 2 : cnt[a] * cnt[b];
            tot += pairs * pair_block_size(a, b);
        }
    // keep room for the Krylov basis of the solve and 4 GiB for everything else; a mixed-precision
    // solve needs the single-precision tables and keeps the double ones too when both fit (its
    // true residuals then use them; otherwise they sum S per application)
    const size_t offb = h->d_pair_off ? 0 : (size_t)npairs * 2 * sizeof(int64_t);
    const size_t b64 = h->d_stab ? 0 : (size_t)tot * sizeof(cplx);
    const size_t b32 = h->d_stab32 ? 0 : (size_t)tot * sizeof(cplxf);
    const size_t room = h->budget > h->bytes_in_use ? h->budget - h->bytes_in_use : 0;
    const size_t reserve = (size_t)(h->prm.gmres_restart + 4) * (size_t)h->n_unk * sizeof(cplx) + ((size_t)4 << 30);
    const bool force = h->prm.pair_tables == 1;
    const bool want32 = mixed && (force || offb + b32 + reserve <= room);
    const bool want64 = mixed ? (force || offb + b32 + b64 + reserve <= room) : (force || offb + b64 + reserve <= room);
    if (!want32 && !want64) {
        h->stab_ready = false;
        h->stab32_ready = false;
        return FOGGY_OK;
    }
    if (!h->d_pair_off) {
        TRY(dalloc(h, &h->d_pair_off, npairs + 1));
        int64_t* d_sizes = nullptr;
        CK(h, talloc(h, &d_sizes, npairs * sizeof(int64_t)));
        k_pair_sizes<<<h->N, 256, 0, h->stream>>>(scene_view(h), d_sizes);
        size_t tmp = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_sizes, h->d_pair_off, npairs, h->stream);
        void* d_tmp = nullptr;
        cudaError_t e = talloc(h, &d_tmp, tmp);
        if (e == cudaSuccess) {
            cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_sizes, h->d_pair_off, npairs, h->stream);
            e = cudaStreamSynchronize(h->stream);
        }
        tfree(h, d_tmp);
        tfree(h, d_sizes);
        if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("pair offsets: ") + cudaGetErrorString(e));
    }
    Trace tr("pair tables");
    SGaunt g{h->d_koffS, h->d_gs, h->gs_nm};
    if (want64 && !h->d_stab) TRY(dalloc(h, &h->d_stab, (size_t)tot));
    if (want32 && !h->d_stab32) TRY(dalloc(h, &h->d_stab32, (size_t)tot));
    TRY(build_pair_tables(h, g, want64, want32));
    if (want64) h->stab_ready = true;
    if (want32) h->stab32_ready = true;
    CKL(h);
    h->stab_z = h->prm.z_coupling;
    return FOGGY_OK;
}

// ---- ML-FMM (lib_ml_fmm_run, libmlfmm/src/lib/lib_ml_fmm.f90:231-262) ---------------------------
int build_tree_dev(foggy_handle h) {
    if (h->tree_ready) return FOGGY_OK;
    int n = h->N;
    if (!h->d_keys) {
        TRY(dalloc(h, &h->d_keys, n));
        TRY(dalloc(h, &h->d_idx, n));
        TRY(dalloc(h, &h->d_keys_sorted, n));
        TRY(dalloc(h, &h->d_idx_sorted, n));
    }
    double* d_mm = nullptr;
    int* d_lmax = nullptr;
    CK(h, talloc(h, &d_mm, 6 * sizeof(double)));
    CK(h, talloc(h, &d_lmax, sizeof(int)));
    k_minmax<<<1, 256, 0, h->stream>>>(n, h->d_centres, d_mm);
    k_morton<<<(n + 255) / 256, 256, 0, h->stream>>>(n, h->d_centres, d_mm, h->d_keys, h->d_idx);
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, h->d_keys, h->d_keys_sorted, h->d_idx, h->d_idx_sorted, n, 0,
                                    63, h->stream);
    void* d_tmp = nullptr;
    CK(h, talloc(h, &d_tmp, tmp_bytes));
    cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, h->d_keys, h->d_keys_sorted, h->d_idx, h->d_idx_sorted, n, 0,
                                    63, h->stream);
    int one = 1;
    CK(h, cudaMemcpyAsync(d_lmax, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    int s = std::max(1, h->prm.tree_s_opt);
    if (n > s) k_level_max<<<(n + 255) / 256, 256, 0, h->stream>>>(n, s, h->d_keys_sorted, d_lmax);
    int lmax = 1;
    cudaError_t e = cudaMemcpyAsync(&lmax, d_lmax, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    tfree(h, d_tmp);
    tfree(h, d_mm);
    tfree(h, d_lmax);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("tree: ") + cudaGetErrorString(e));
    CKL(h);
    // l_min = 1 + floor(log(k + 1) / log(2)) for k = 1 (lib_tree.f90:1162-1170)
    h->tree_lmin = (int)(1 + std::floor(std::log(2.0f) / std::log(2.0f)));
    h->tree_lmax = h->prm.tree_l_max > 0 ? h->prm.tree_l_max : lmax;
    h->tree_ready = true;
    return FOGGY_OK;
}


void free_fmm(foggy_handle h) {
    dfree(h, h->d_fmm_c);
    dfree(h, h->d_fmm_p);
    dfree(h, h->d_fmm_off);
    dfree(h, h->d_fmm_C);
    dfree(h, h->d_fmm_D);
    dfree(h, h->d_fmm_list);
    dfree(h, h->d_fmm_slab);
    dfree(h, h->d_fmm_chunks);
    dfree(h, h->d_fmm_chunks2);
    dfree(h, h->d_fmm_tab);
    dfree(h, h->d_fmm_taboff);
    dfree(h, h->d_fmm_tab32);
    h->fmm_tab_ready = false;
    h->fmm_pmax = 0;
    h->fmm_list_host.clear();
    h->fmm = FmmTree();
    h->fmm_ready = false;
}

// ML-FMM passes with fewer than kFmmFill targets run kFmmFill / targets CTAs per target (at most
// kFmmChunks), each over every chunks-th source of the target's list, so that the upper levels'
// few boxes still fill the GPU; their partial sums need fewer than 2 kFmmFill slabs of one target.
constexpr int kFmmFill = 148 * 6;
constexpr int kFmmChunks = 16;

// Expansion order of the boxes of level l.  The reference expands every box to its global order
// p_g (digits = 0).  With digits > 0: the excess-bandwidth order L = kd + 1.8 digits^(2/3) (kd)^(1/3)
// of the level's box diagonal d = sqrt(3) D 2^-l (D the scaled domain's edge), rounded up, never
// below p_g, at most kMaxDegree.
int fmm_level_order(double k, double D, int l, double digits, int pg) {
    if (!(digits > 0.0)) return pg;
    const double kd = k * std::sqrt(3.0) * std::ldexp(D, -l);
    const double L = std::ceil(std::fma(1.8 * std::pow(digits, 2.0 / 3.0), std::cbrt(kd), kd));
    return (int)std::min<double>(kMaxDegree, std::max<double>(pg, L));
}

// Octree hierarchy and ML-FMM pass lists of the current scene and tree parameters, built on the
// device from the sorted keys (k_tree.cu); the host keeps the level bounds only.
int ensure_fmm(foggy_handle h) {
    if (h->fmm_ready) return FOGGY_OK;
    free_fmm(h);
    // boxes carry the global order, which may exceed every sphere's
    TRY(ensure_tables(h, std::max(h->pg, 1)));
    TRY(build_tree_dev(h));
    const int n = h->N;
    int lmin = h->tree_lmin, lmax = h->tree_lmax;
    if (lmax < lmin) lmin = lmax;
    const int nlev = lmax - lmin + 1;
    const size_t nl = (size_t)nlev * n;
    std::vector<void*> scratch;
    auto sc_alloc = [&](auto** p, size_t count) -> cudaError_t {
        void* q = nullptr;
        cudaError_t e = talloc(h, &q, std::max<size_t>(count, 1) * sizeof(**p));
        if (e == cudaSuccess) scratch.push_back(q);
        *p = static_cast<std::remove_reference_t<decltype(*p)>>(q);
        return e;
    };
    auto cleanup = [&]() {
        for (void* q : scratch) tfree(h, q);
        scratch.clear();
    };
    auto bad = [&](cudaError_t e, const char* what) {
        cleanup();
        return fail(h, FOGGY_ERR_CUDA, std::string("ML-FMM tree (") + what + "): " + cudaGetErrorString(e));
    };
    int *flag, *incl, *run_start, *run_end, *parent, *box_level, *level_base, *cnt, *ptr;
    long long* box_n;
    double* mm;
    cudaError_t e = cudaSuccess;
    for (auto* pp : {&flag, &incl, &run_start, &run_end, &parent, &box_level})
        if (e == cudaSuccess) e = sc_alloc(pp, nl + 1);
    if (e == cudaSuccess) e = sc_alloc(&level_base, nlev + 1);
    if (e == cudaSuccess) e = sc_alloc(&cnt, std::max(nl, (size_t)n) + 1);
    if (e == cudaSuccess) e = sc_alloc(&ptr, 4 * (std::max(nl, (size_t)n) + 1));
    if (e == cudaSuccess) e = sc_alloc(&box_n, nl + 1);
    if (e == cudaSuccess) e = sc_alloc(&mm, 6);
    if (e != cudaSuccess) return bad(e, "scratch");
    // CUB scans: one temporary buffer of the largest size any of them needs
    size_t tmp_bytes = 0, t2 = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, flag, incl, (int)nl, h->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, t2, cnt, ptr, (int)std::max(nl, (size_t)n) + 1, h->stream);
    void* tmp = nullptr;
    e = sc_alloc(reinterpret_cast<char**>(&tmp), std::max(tmp_bytes, t2));
    if (e != cudaSuccess) return bad(e, "scan storage");
    tmp_bytes = std::max(tmp_bytes, t2);
    auto exscan = [&](const int* in, int* out, int items) {
        size_t tb = tmp_bytes;
        cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, items, h->stream);
    };
    auto blocks = [](size_t items) { return (unsigned)((items + 255) / 256); };
    const unsigned long long* keys = h->d_keys_sorted;
    const int* order = h->d_idx_sorted;
    k_minmax<<<1, 256, 0, h->stream>>>(n, h->d_centres, mm);
    k_tree_flags<<<blocks(nl), 256, 0, h->stream>>>(n, nlev, lmin, keys, flag);
    {
        size_t tb = tmp_bytes;
        cub::DeviceScan::InclusiveSum(tmp, tb, flag, incl, (int)nl, h->stream);
    }
    k_tree_boxes<<<blocks(nl), 256, 0, h->stream>>>(n, nlev, lmin, keys, incl, box_n, box_level, run_start, level_base);
    std::vector<int> lb(nlev + 1);
    double mmh[6];
    e = cudaMemcpyAsync(lb.data(), level_base, (nlev + 1) * sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mmh, mm, sizeof(mmh), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return bad(e, "boxes");
    const int nbox = lb[nlev];
    const int lb1 = nlev > 1 ? lb[1] : nbox;
    const int leaf0 = lb[nlev - 1], nleaf = nbox - leaf0;
    h->launches += 4;
    k_tree_links<<<blocks(nbox), 256, 0, h->stream>>>(nbox, n, nlev, incl, level_base, run_start, run_end, parent);
    // per-item counts and their exclusive scans: I4 per box, E2 per leaf, near field per sphere,
    // aggregation per leaf
    int* i4ptr = ptr;
    int* e2ptr = ptr + (nl + 1);
    int* nearptr = ptr + 2 * (nl + 1);
    int* aggptr = ptr + 3 * (nl + 1);
    int* e2cnt = nullptr;
    int* nearcnt = nullptr;
    int* aggcnt = nullptr;
    if ((e = sc_alloc(&e2cnt, nleaf + 1)) != cudaSuccess || (e = sc_alloc(&nearcnt, n + 1)) != cudaSuccess ||
        (e = sc_alloc(&aggcnt, nleaf + 1)) != cudaSuccess)
        return bad(e, "counts");
    cudaMemsetAsync(cnt, 0, (nbox + 1) * sizeof(int), h->stream);
    cudaMemsetAsync(e2cnt, 0, (nleaf + 1) * sizeof(int), h->stream);
    cudaMemsetAsync(nearcnt, 0, (n + 1) * sizeof(int), h->stream);
    cudaMemsetAsync(aggcnt, 0, (nleaf + 1) * sizeof(int), h->stream);
    k_tree_i4<<<blocks(nbox), 256, 0, h->stream>>>(nbox, nlev, level_base, box_n, box_level, nullptr, cnt, nullptr);
    exscan(cnt, i4ptr, nbox + 1);
    k_tree_e2<<<blocks(nleaf), 256, 0, h->stream>>>(nleaf, leaf0, nbox, lmax, box_n, run_start, run_end, order, nullptr,
                                                    e2cnt, nullptr);
    exscan(e2cnt, e2ptr, nleaf + 1);
    const int* incl_leaf = incl + (size_t)(nlev - 1) * n;
    k_fmm_counts<<<blocks(std::max(n, nleaf)), 256, 0, h->stream>>>(n, nleaf, leaf0, order, h->d_couple, incl_leaf,
                                                                     run_start, run_end, e2cnt, nearcnt, aggcnt);
    exscan(nearcnt, nearptr, n + 1);
    exscan(aggcnt, aggptr, nleaf + 1);
    int tot[4] = {0, 0, 0, 0};   // I4, E2, near field, aggregation entries
    e = cudaMemcpyAsync(&tot[0], i4ptr + nbox, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tot[1], e2ptr + nleaf, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tot[2], nearptr + n, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tot[3], aggptr + nleaf, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return bad(e, "list sizes");
    h->launches += 8;
    int* e2idx = nullptr;
    if ((e = sc_alloc(&e2idx, tot[1] + 1)) != cudaSuccess) return bad(e, "E2");
    k_tree_e2<<<blocks(nleaf), 256, 0, h->stream>>>(nleaf, leaf0, nbox, lmax, box_n, run_start, run_end, order, e2ptr,
                                                    nullptr, e2idx);
    // the twelve lists of the passes, one buffer: aggregation, children, I4, parent, box to sphere,
    // near field (pointers then indices each)
    const int sizes[12] = {nleaf + 1, tot[3], nbox + 1, nbox - lb1, nbox + 1, tot[0],
                           nbox + 1, nbox - lb1, n + 1, n, n + 1, tot[2]};
    int total = 0;
    for (int i = 0; i < 12; ++i) {
        h->fmm_lofs[i] = total;
        total += sizes[i];
    }
    h->fmm_ltotal = total;
    {
        const int rc = dalloc(h, &h->d_fmm_list, (size_t)total + 1);
        if (rc) {
            cleanup();
            return rc;
        }
    }
    cudaMemsetAsync(h->d_fmm_list, 0, ((size_t)total + 1) * sizeof(int), h->stream);
    k_fmm_child_ptr<<<blocks(nbox), 256, 0, h->stream>>>(nbox, lb1, parent, h->d_fmm_list + h->fmm_lofs[2]);
    k_tree_i4<<<blocks(nbox), 256, 0, h->stream>>>(nbox, nlev, level_base, box_n, box_level, i4ptr, nullptr,
                                                   h->d_fmm_list + h->fmm_lofs[5]);
    FmmListArgs la{};
    la.n = n;
    la.nbox = nbox;
    la.nleaf = nleaf;
    la.leaf0 = leaf0;
    la.lb1 = lb1;
    la.order = order;
    la.couple = h->d_couple;
    la.incl_leaf = incl_leaf;
    la.run_start = run_start;
    la.run_end = run_end;
    la.parent = parent;
    la.e2_ptr = e2ptr;
    la.e2_idx = e2idx;
    la.agg_ptr = aggptr;
    la.i4_ptr = i4ptr;
    la.near_ptr = nearptr;
    for (int i = 0; i < 12; ++i) la.lofs[i] = h->fmm_lofs[i];
    la.list = h->d_fmm_list;
    k_fmm_lists<<<blocks((size_t)std::max(n, nbox) + 1), 256, 0, h->stream>>>(la);
    h->launches += 4;
    // box centres, orders and coefficient offsets; the boxes' expansions, level by level
    FmmLevels lv{};
    lv.lmin = lmin;
    double Dm = 0.0;   // the scaled domain's edge, as k_fmm_boxes computes it
    for (int d = 0; d < 3; ++d) Dm = std::max(Dm, (mmh[3 + d] - mmh[d]) * (1.0 + 2.220446049250313e-16));
    int pmax = h->pg;
    int64_t box_entries = 0;
    for (int li = 0; li < nlev; ++li) {
        const int L = fmm_level_order(wavenumber(h->prm), Dm, lmin + li, h->prm.fmm_digits, h->pg);
        lv.order[li] = L;
        lv.base[li] = lb[li];
        lv.off[li] = box_entries;
        box_entries += (int64_t)(lb[li + 1] - lb[li]) * 2 * L * (L + 2);
        pmax = std::max(pmax, L);
    }
    h->fmm_pmax = pmax;
    const int Pm = pmax * (pmax + 2);
    int rc = ensure_tables(h, pmax);
    if (!rc) rc = dalloc(h, &h->d_fmm_c, 3 * (size_t)nbox);
    if (!rc) rc = dalloc(h, &h->d_fmm_p, (size_t)nbox);
    if (!rc) rc = dalloc(h, &h->d_fmm_off, (size_t)nbox);
    if (!rc) rc = dalloc(h, &h->d_fmm_C, (size_t)box_entries);
    if (!rc) rc = dalloc(h, &h->d_fmm_D, (size_t)box_entries);
    if (!rc) rc = dalloc(h, &h->d_fmm_slab, 2 * (size_t)h->n_unk);
    if (!rc) rc = dalloc(h, &h->d_fmm_chunks, (size_t)2 * kFmmFill * 2 * Pm);
    if (!rc) rc = dalloc(h, &h->d_fmm_chunks2, (size_t)2 * kFmmFill * 2 * Pm);
    if (rc) {
        cleanup();
        return rc;
    }
    k_fmm_boxes<<<blocks(nbox), 256, 0, h->stream>>>(nbox, box_n, box_level, mm, lv, h->d_fmm_c, h->d_fmm_p,
                                                     h->d_fmm_off);
    h->launches += 1;
    e = cudaGetLastError();
    h->fmm_list_host.assign((size_t)h->fmm_ltotal + 1, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->fmm_list_host.data(), h->d_fmm_list, ((size_t)h->fmm_ltotal + 1) * sizeof(int),
                            cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cleanup();
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("ML-FMM lists: ") + cudaGetErrorString(e));
    for (int d = 0; d < 3; ++d) h->fmm_xmin[d] = mmh[d];
    FmmTree& t = h->fmm;
    t = FmmTree();
    t.lmin = lmin;
    t.lmax = lmax;
    t.level_base = lb;
    h->fmm_ready = true;
    return FOGGY_OK;
}

// One ML-FMM pass: targets tbase .. tbase + ntgt - 1 of tg over their lists (ptr list lp, index list
// li) of sources in sr, displacement sign and shift, radial function z; in -> out (add: out +=).
struct FmmPass {
    PointSet tg, sr;
    const cplx* in;
    cplx* out;
    int lp, li, tbase, ntgt;
    double sign;
    int z, add;
    bool shift;
};

TransArgs fmm_pass_args(foggy_handle h, const TransArgs& base, const FmmPass& q) {
    TransArgs a = base;
    const int* L = h->d_fmm_list;
    const int* lo = h->fmm_lofs;
    a.slab = h->d_fmm_chunks;
    a.slab_ld = 2 * (int64_t)h->fmm_pmax * (h->fmm_pmax + 2);
    a.tgt = q.tg;
    a.src = q.sr;
    a.x = q.in;
    a.out = q.out;
    a.lptr = L + lo[q.lp] + (q.lp == 0 || q.lp >= 8 ? 0 : q.tbase);
    a.lidx = L + lo[q.li];
    a.tbase = q.tbase;
    a.sign = q.sign;
    for (int d = 0; d < 3; ++d) a.sh[d] = q.shift ? h->fmm_xmin[d] : 0.0;
    a.z = q.z;
    a.add = q.add;
    return a;
}

// The coaxial blocks of the passes' translations, cached like the direct operator's pair tables
// (pair_tables -1 = off, 0 = when they fit beside the Krylov basis, 1 = always).  Translations of
// one index list share their radial function, displacement rule and degrees, and within a level
// the box displacements repeat, so each list keeps one block per distinct (length, target degree,
// source degree): the lengths come from the device (k_fmm_rho, rounded as the passes round them),
// the host groups them, and k_fmm_tab sums each block once, as the passes would sum it per
// translation.  The passes then read S from the blocks, with the same result bit for bit.
int ensure_fmm_tables(foggy_handle h, const TransArgs& base, const std::vector<FmmPass>& passes) {
    const int key[5] = {h->prm.fmm_convention, h->prm.z_coupling, h->prm.z_translation_gt_r, h->prm.pair_tables >= 0,
                        h->prm.precision};
    if (h->fmm_tab_ready && std::equal(key, key + 5, h->fmm_tab_key)) return FOGGY_OK;
    dfree(h, h->d_fmm_tab);
    dfree(h, h->d_fmm_taboff);
    dfree(h, h->d_fmm_tab32);
    h->fmm_tab_ready = false;
    std::copy(key, key + 5, h->fmm_tab_key);
    if (h->prm.pair_tables < 0) {
        h->fmm_tab_ready = true;   // off: the passes sum S from the Gaunt table
        return FOGGY_OK;
    }
    const int total = h->fmm_ltotal;
    double* d_rho = nullptr;
    int2* d_deg = nullptr;
    CK(h, talloc(h, &d_rho, (size_t)total * sizeof(double)));
    CK(h, talloc(h, &d_deg, (size_t)total * sizeof(int2)));
    CK(h, cudaMemsetAsync(d_deg, 0xff, (size_t)total * sizeof(int2), h->stream));   // -1: no pass
    int z_of[12];
    std::fill(z_of, z_of + 12, 0);
    for (const FmmPass& q : passes) {
        if (q.ntgt <= 0) continue;
        const TransArgs a = fmm_pass_args(h, base, q);
        k_fmm_rho<<<q.ntgt, 128, 0, h->stream>>>(a, d_rho + h->fmm_lofs[q.li], d_deg + h->fmm_lofs[q.li]);
        h->launches += 1;
        z_of[q.li] = q.z;
    }
    std::vector<double> rho(total);
    std::vector<int2> deg(total);
    cudaError_t e = cudaMemcpyAsync(rho.data(), d_rho, (size_t)total * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(deg.data(), d_deg, (size_t)total * sizeof(int2), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    tfree(h, d_rho);
    tfree(h, d_deg);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("ML-FMM tables: ") + cudaGetErrorString(e));
    // per index list, one block per distinct (length bits, degrees)
    std::vector<int64_t> off(total, -1);
    std::vector<FmmTabEntry> uniq;
    std::vector<std::pair<int, int>> list_range;   // (first unique entry, count) per index list
    int64_t entries = 0;
    for (int li = 1; li < 12; li += 2) {
        const int lo = h->fmm_lofs[li], hi = li + 1 < 12 ? h->fmm_lofs[li + 1] : total;
        std::map<std::tuple<uint64_t, int, int>, int64_t> seen;
        const int first = (int)uniq.size();
        for (int i = lo; i < hi; ++i) {
            if (deg[i].x < 0) continue;
            uint64_t bits;
            std::memcpy(&bits, &rho[i], sizeof(bits));
            const auto k = std::make_tuple(bits, deg[i].x, deg[i].y);
            auto it = seen.find(k);
            if (it == seen.end()) {
                it = seen.emplace(k, entries).first;
                uniq.push_back(FmmTabEntry{rho[i], deg[i].x, deg[i].y, entries});
                entries += pair_block_size(deg[i].y, deg[i].x);
            }
            off[i] = it->second;
        }
        list_range.emplace_back(first, (int)uniq.size() - first);
    }
    const bool mixed = h->prm.precision == 1;
    const size_t need = (size_t)entries * (sizeof(cplx) + (mixed ? sizeof(cplxf) : 0)) + (size_t)total * sizeof(int64_t);
    const size_t room = h->budget > h->bytes_in_use ? h->budget - h->bytes_in_use : 0;
    const size_t reserve = (size_t)(h->prm.gmres_restart + 4) * (size_t)h->n_unk * sizeof(cplx) + ((size_t)1 << 30);
    if (h->prm.pair_tables == 0 && need + reserve > room) {
        h->fmm_tab_ready = true;   // do not fit: the passes sum S from the Gaunt table
        return FOGGY_OK;
    }
    Trace tr("ML-FMM tables");
    TRY(dalloc(h, &h->d_fmm_tab, (size_t)std::max<int64_t>(entries, 1)));
    TRY(dalloc(h, &h->d_fmm_taboff, (size_t)total));
    FmmTabEntry* d_u = nullptr;
    CK(h, talloc(h, &d_u, std::max<size_t>(uniq.size(), 1) * sizeof(FmmTabEntry)));
    e = cudaMemcpyAsync(h->d_fmm_taboff, off.data(), (size_t)total * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && !uniq.empty())
        e = cudaMemcpyAsync(d_u, uniq.data(), uniq.size() * sizeof(FmmTabEntry), cudaMemcpyHostToDevice, h->stream);
    const SGaunt g{h->d_koffS, h->d_gs, h->gs_nm};
    for (int r = 0; r < (int)list_range.size() && e == cudaSuccess; ++r) {
        const int li = 2 * r + 1;
        if (list_range[r].second == 0) continue;
        k_fmm_tab<<<list_range[r].second, 256, 0, h->stream>>>(d_u + list_range[r].first, g, z_of[li], h->d_fmm_tab);
        h->launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && mixed) {
        const int rc = dalloc(h, &h->d_fmm_tab32, (size_t)std::max<int64_t>(entries, 1));
        if (rc) {
            tfree(h, d_u);
            return rc;
        }
        k_narrow<<<(unsigned)std::min<int64_t>((entries + 255) / 256 + 1, 148 * 8), 256, 0, h->stream>>>(
            h->d_fmm_tab, h->d_fmm_tab32, entries);
        h->launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);   // the host vectors go out of scope
    tfree(h, d_u);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("ML-FMM tables: ") + cudaGetErrorString(e));
    h->fmm_tab_ready = true;
    return FOGGY_OK;
}

// y = A x by the ML-FMM passes (upward :387-640, downward :656-982, final summation :994-1204;
// the Mie handles lib_mie_ms_ml_fmm_interface.f90:259-981), in the device layout.
// fp32: translations in single precision (the Arnoldi steps of a mixed-precision solve); the box
// coefficients, the chunks' partial sums and y stay FP64.
int apply_operator_fmm(foggy_handle h, const cplx* x, cplx* y, bool fp32 = false) {
    TRY(ensure_fmm(h));
    const FmmTree& t = h->fmm;
    const int conv = h->prm.fmm_convention;
    const int zi = h->prm.z_coupling;
    const int z_reg = conv == 0 ? zi : 1;                            // aggregation, M2M, L2L
    const int z_dor = conv == 0 ? h->prm.z_translation_gt_r : 1;     // box to sphere
    const double sts = conv == 0 ? -1.0 : 1.0;                       // aggregation, M2L, box to sphere
    const int nlev = t.lmax - t.lmin + 1;
    const int nbox = t.level_base[nlev];
    const int leaf0 = t.level_base[nlev - 1];
    SceneView sv = scene_view(h);
    TransArgs base{};
    base.delta = h->d_delta;
    base.dt = dtabs(h);
    base.g = SGaunt{h->d_koffS, h->d_gs, h->gs_nm};
    base.k = sv.k;
    base.pp = std::max(h->pg, h->fmm_pmax);
    base.fp32 = fp32 ? 1 : 0;
    base.delta32 = h->d_delta32;
    const PointSet S{h->d_centres, h->d_p, h->d_off};
    const PointSet B{h->d_fmm_c, h->d_fmm_p, h->d_fmm_off};
    // the passes in order: upward (aggregation at the leaves, then M2M level by level), downward
    // (M2L on every level, then L2L from the coarsest level down), final summation (box to
    // sphere, near field)
    std::vector<FmmPass> passes;
    const char* names[6] = {"aggregation", "M2M", "M2L", "L2L", "box to sphere", "near field"};
    std::vector<int> stage;
    auto add = [&](int st, PointSet tg, PointSet sr, const cplx* in, cplx* out, int lp, int li, int tbase, int ntgt,
                   double sign, int z, int addflag, bool shift) {
        passes.push_back(FmmPass{tg, sr, in, out, lp, li, tbase, ntgt, sign, z, addflag, shift});
        stage.push_back(st);
    };
    add(0, B, S, x, h->d_fmm_C, 0, 1, leaf0, nbox - leaf0, sts, z_reg, 0, false);
    for (int li = nlev - 2; li >= 0; --li)
        add(1, B, B, h->d_fmm_C, h->d_fmm_C, 2, 3, t.level_base[li], t.level_base[li + 1] - t.level_base[li], 1.0,
            z_reg, 0, false);
    // M2L of every level in one launch: each box's incoming sum depends only on the outgoing
    // expansions of its own level
    add(2, B, B, h->d_fmm_C, h->d_fmm_D, 4, 5, 0, nbox, sts, zi, 0, false);
    for (int li = 1; li < nlev; ++li)
        add(3, B, B, h->d_fmm_D, h->d_fmm_D, 6, 7, t.level_base[li], t.level_base[li + 1] - t.level_base[li], 1.0,
            z_reg, 1, false);
    add(4, S, B, h->d_fmm_D, h->d_fmm_slab, 8, 9, 0, h->N, sts, z_dor, 0, conv == 0);
    add(5, S, S, x, h->d_fmm_slab + h->n_unk, 10, 11, 0, h->N, 1.0, zi, 0, false);
    TRY(ensure_fmm_tables(h, base, passes));
    const bool tabs = h->d_fmm_taboff != nullptr && (!fp32 || h->d_fmm_tab32 != nullptr);
    // the near field needs only x: it runs on a second stream beside the box passes
    if (!h->side) {
        if (cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess)
            return fail(h, FOGGY_ERR_CUDA, "ML-FMM side stream");
    }
    CK(h, cudaEventRecord(h->ev_fork, h->stream));
    CK(h, cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    Trace tr(fp32 ? "ML-FMM operator (FP32)" : "ML-FMM operator");
    for (size_t i = 0; i < passes.size(); ++i) {
        const FmmPass& q = passes[i];
        const bool near = stage[i] == 5;
        Trace tp(names[stage[i]]);
        TransArgs a = fmm_pass_args(h, base, q);
        if (near) a.slab = h->d_fmm_chunks2;
        if (tabs) {
            a.tab = h->d_fmm_tab;
            a.tab32 = h->d_fmm_tab32;
            a.tab_off = h->d_fmm_taboff + h->fmm_lofs[q.li];
        }
        // passes with few targets split each target's sources over several CTAs, no more than the
        // longest of its source lists
        int longest = 0;
        if (q.ntgt > 0) {
            const int* ptr = h->fmm_list_host.data() + h->fmm_lofs[q.lp] + (q.lp == 0 || q.lp >= 8 ? 0 : q.tbase);
            for (int b = 0; b < q.ntgt; ++b) longest = std::max(longest, ptr[b + 1] - ptr[b]);
        }
        const int chunks =
            q.ntgt > 0 ? std::max(1, std::min({kFmmChunks, (kFmmFill + q.ntgt - 1) / q.ntgt, longest})) : 1;
        launch_translate(a, q.ntgt, chunks, near ? h->side : h->stream);
        if (q.ntgt > 0) h->launches += chunks > 1 ? 2 : 1;
    }
    // join first, so that whatever follows on the handle's stream (frees included) comes after the side
    cudaEventRecord(h->ev_join, h->side);
    cudaStreamWaitEvent(h->stream, h->ev_join, 0);
    CKL(h);
    k_direct_finish<<<h->N, 256, 0, h->stream>>>(sv, x, h->d_fmm_slab, 2, h->n_unk, y);
    h->launches += 1;
    CKL(h);
    return FOGGY_OK;
}

// y = A x in the device layout
// fp32: the single-precision operator (mixed-precision solves' Arnoldi steps), when its tables exist
int apply_operator(foggy_handle h, const cplx* x, cplx* y, bool fp32 = false) {
    if (h->prm.matvec_mode == FOGGY_MATVEC_MLFMM) return apply_operator_fmm(h, x, y, fp32);
    TRY(ensure_pair_tables(h));
    DirectArgs a = direct_args(h, x);
    a.fp32 = (fp32 && h->stab32_ready) ? 1 : 0;
    Trace tr(a.fp32 ? "operator (FP32)" : "operator (FP64)");
    for (const DirectBucket& b : h->launches_direct) {
        launch_direct(a, b, h->stream);
        h->launches += 1;
    }
    CKL(h);
    k_direct_finish<<<h->N, 256, 0, h->stream>>>(a.sc, x, h->d_partial, h->nbuckets * h->cmax, h->n_unk, y);
    h->launches += 1;
    CKL(h);
    return FOGGY_OK;
}

int ensure_rhs(foggy_handle h) {
    if (h->rhs_ready) return FOGGY_OK;
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    if (h->waves.empty() && h->beams.empty()) return fail(h, FOGGY_ERR_STATE, "no plane waves or beams set");
    const int nw = (int)h->waves.size(), nb = (int)h->beams.size();
    const size_t nl = (size_t)h->N * nb;   // local plane waves of the beams, per sphere
    const size_t S = (size_t)(h->pmax + 1) * (h->pmax + 1);
    // one allocation: waves, local waves, beams, then the pi / tau tables of both
    const size_t nwav = (size_t)nw + nl;
    const size_t bytes = nwav * sizeof(WaveDev) + (size_t)nb * sizeof(GaussDev) + 2 * nwav * S * sizeof(double);
    void* buf = nullptr;
    CK(h, talloc(h, &buf, bytes));
    WaveDev* d_w = static_cast<WaveDev*>(buf);
    WaveDev* d_l = d_w + nw;
    GaussDev* d_g = reinterpret_cast<GaussDev*>(d_l + nl);
    double* d_pi = reinterpret_cast<double*>(d_g + nb);
    double* d_tau = d_pi + nwav * S;
    cudaError_t e = cudaSuccess;
    if (nw) e = cudaMemcpyAsync(d_w, h->waves.data(), nw * sizeof(WaveDev), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && nb)
        e = cudaMemcpyAsync(d_g, h->beams.data(), nb * sizeof(GaussDev), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && nb) {
        k_gauss_local<<<(unsigned)((nl + 127) / 128), 128, 0, h->stream>>>(scene_view(h), nb, d_g, h->prm.lambda_0,
                                                                           h->prm.n_medium, d_l);
        h->launches += 1;
    }
    if (e == cudaSuccess) {
        // pi / tau of the shared waves and of the local waves are one table set
        k_pitau<<<(unsigned)nwav, h->pmax + 1, 0, h->stream>>>((int)nwav, d_w, h->pmax, d_pi, d_tau);
        k_rhs<<<h->N, 128, 0, h->stream>>>(scene_view(h), nw, d_w, h->pmax, d_pi, d_tau, nb, d_l, d_pi + nw * S,
                                           d_tau + nw * S, h->d_b, h->d_pq);
        h->launches += 2;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    tfree(h, buf);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("rhs: ") + cudaGetErrorString(e));
    h->rhs_ready = true;
    return FOGGY_OK;
}

void free_block(foggy_handle h) {
    dfree(h, h->d_bV);
    dfree(h, h->d_bW);
    dfree(h, h->d_bX);
    dfree(h, h->d_bB);
    dfree(h, h->d_bR);
    dfree(h, h->d_bsmall);
    dfree(h, h->d_breal);
    dfree(h, h->d_bint);
    h->blk_nrhs = 0;
    h->blk_m = 0;
}

void free_scene(foggy_handle h) {
    dfree(h, h->d_centres);
    dfree(h, h->d_p);
    dfree(h, h->d_off);
    dfree(h, h->d_an);
    dfree(h, h->d_bn);
    dfree(h, h->d_an_p);
    dfree(h, h->d_bn_p);
    dfree(h, h->d_couple);
    dfree(h, h->d_b);
    dfree(h, h->d_pq);
    dfree(h, h->d_partial);
    dfree(h, h->d_stab);
    dfree(h, h->d_stab32);
    h->stab32_ready = false;
    dfree(h, h->d_pair_off);
    h->stab_ready = false;
    dfree(h, h->d_tmp_in);
    dfree(h, h->d_tmp_out);
    dfree(h, h->d_ref_a);
    dfree(h, h->d_ref_b);
    dfree(h, h->d_V);
    dfree(h, h->d_w);
    dfree(h, h->d_x);
    dfree(h, h->d_r);
    dfree(h, h->d_keys);
    dfree(h, h->d_idx);
    dfree(h, h->d_keys_sorted);
    dfree(h, h->d_idx_sorted);
    h->ws_restart = 0;
    h->tree_ready = false;
    h->rhs_ready = false;
    free_fmm(h);
    free_block(h);
}

int ensure_workspace(foggy_handle h, int restart) {
    if (h->ws_restart >= restart && h->d_V) return FOGGY_OK;
    dfree(h, h->d_V);
    dfree(h, h->d_H);
    dfree(h, h->d_cs);
    dfree(h, h->d_sn);
    dfree(h, h->d_gv);
    dfree(h, h->d_h);
    dfree(h, h->d_c);
    dfree(h, h->d_y);
    dfree(h, h->d_part);
    TRY(dalloc(h, &h->d_V, (size_t)(restart + 1) * h->n_unk));
    if (!h->d_w) TRY(dalloc(h, &h->d_w, h->n_unk));
    if (!h->d_x) TRY(dalloc(h, &h->d_x, h->n_unk));
    if (!h->d_r) TRY(dalloc(h, &h->d_r, h->n_unk));
    TRY(dalloc(h, &h->d_H, (size_t)(restart + 1) * restart));
    TRY(dalloc(h, &h->d_cs, restart));
    TRY(dalloc(h, &h->d_sn, restart));
    TRY(dalloc(h, &h->d_gv, restart + 1));
    TRY(dalloc(h, &h->d_h, restart + 1));
    TRY(dalloc(h, &h->d_c, restart + 1));
    TRY(dalloc(h, &h->d_y, restart + 1));
    TRY(dalloc(h, &h->d_part, (size_t)kRedBlocks * (restart + 1)));
    if (!h->d_npart) TRY(dalloc(h, &h->d_npart, kRedBlocks));
    if (!h->d_scal) TRY(dalloc(h, &h->d_scal, 8));
    if (!h->d_flags) TRY(dalloc(h, &h->d_flags, 4));
    h->ws_restart = restart;
    return FOGGY_OK;
}

int norm_dev(foggy_handle h, const cplx* v, double* out_dev) {
    k_norm_partial<<<kRedBlocks, 256, 0, h->stream>>>(v, h->n_unk, h->d_npart);
    k_norm_reduce<<<1, 256, 0, h->stream>>>(h->d_npart, out_dev);
    h->launches += 2;
    CKL(h);
    return FOGGY_OK;
}

int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 8); }

// GMRES(m) with classical Gram-Schmidt and one reorthogonalisation (CGS2), Givens rotations
// and the explicit residual at each restart.
int gmres(foggy_handle h, foggy_stats* st) {
    const int m = h->prm.gmres_restart;
    const int maxit = h->prm.gmres_max_iterations;
    const double tol = h->prm.gmres_tolerance;
    const int64_t n = h->n_unk;
    const int G = grid_for(n);
    double* d_hn = h->d_scal + 0;
    double* d_beta = h->d_scal + 1;
    double* d_res = h->d_scal + 2;
    double* d_bn = h->d_scal + 3;
    for (cudaEvent_t& e : h->ev_step)
        if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return fail(h, FOGGY_ERR_CUDA, "cudaEventCreate");
    // operator timing: one pair of events per application, from the handle's pool (created once,
    // reused by later solves, destroyed with the handle)
    size_t nmv = 0;
    // Arnoldi steps of a mixed-precision solve use the FP32 operator; the true residuals (start and
    // every restart) the FP64 one, so the restarts refine the solution to the FP64 tolerance
    const bool mixed = h->prm.precision == 1;
    auto matvec = [&](const cplx* x, cplx* y, bool arnoldi) -> int {
        while (h->ev_pool.size() < 2 * (nmv + 1)) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, "cudaEventCreate");
            h->ev_pool.push_back(e);
        }
        cudaEventRecord(h->ev_pool[2 * nmv], h->stream);
        int r = apply_operator(h, x, y, arnoldi && mixed);
        cudaEventRecord(h->ev_pool[2 * nmv + 1], h->stream);
        ++nmv;
        st->matvecs++;
        return r;
    };
    auto cleanup = [&]() {
        cudaStreamSynchronize(h->stream);
        for (size_t i = 0; i < nmv; ++i) {
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev_pool[2 * i], h->ev_pool[2 * i + 1]);
            st->ms_matvec += ms;
        }
        nmv = 0;
    };
    TRY(norm_dev(h, h->d_b, d_bn));
    TRY(matvec(h->d_x, h->d_w, false));
    k_sub<<<G, 256, 0, h->stream>>>(h->d_b, h->d_w, h->d_r, n);
    h->launches += 1;
    TRY(norm_dev(h, h->d_r, d_beta));
    CK(h, cudaMemcpyAsync(h->h_pin, h->d_scal, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    double bnorm = h->h_pin[3];
    double beta = h->h_pin[1];
    if (bnorm == 0.0) {
        CK(h, cudaMemsetAsync(h->d_x, 0, n * sizeof(cplx), h->stream));
        st->backward_error = 0.0;
        cleanup();
        return FOGGY_OK;
    }
    double berr = beta / bnorm;
    int status = FOGGY_OK;
    if (!std::isfinite(berr)) {
        cleanup();
        st->backward_error = berr;
        return FOGGY_ERR_NAN;
    }
    while (berr > tol && st->iterations < maxit) {
        k_scale_copy<<<G, 256, 0, h->stream>>>(h->d_r, d_beta, h->d_V, n);
        k_init_cycle<<<1, 64, 0, h->stream>>>(h->d_gv, m + 1, d_beta, h->d_flags);
        h->launches += 2;
        // Arnoldi step k; its residual estimate, H[k+1][k] and flags are copied into pinned slot
        // k & 1, and the slot's event marks when they have landed
        auto enqueue_step = [&](int k) -> int {
            cplx* vk = h->d_V + (size_t)k * n;
            cplx* vk1 = h->d_V + (size_t)(k + 1) * n;
            TRY(matvec(vk, h->d_w, true));
            k_dots_partial<<<kRedBlocks, 256, 0, h->stream>>>(h->d_V, n, k + 1, h->d_w, n, h->d_part);
            k_dots_reduce<<<k + 1, 256, 0, h->stream>>>(h->d_part, k + 1, h->d_h, 0);
            k_axpy_multi<<<G, 256, 0, h->stream>>>(h->d_V, n, k + 1, h->d_h, h->d_w, n);
            k_dots_partial<<<kRedBlocks, 256, 0, h->stream>>>(h->d_V, n, k + 1, h->d_w, n, h->d_part);
            k_dots_reduce<<<k + 1, 256, 0, h->stream>>>(h->d_part, k + 1, h->d_c, 0);
            k_axpy_multi<<<G, 256, 0, h->stream>>>(h->d_V, n, k + 1, h->d_c, h->d_w, n);
            TRY(norm_dev(h, h->d_w, d_hn));
            k_scale_copy<<<G, 256, 0, h->stream>>>(h->d_w, d_hn, vk1, n);
            k_givens<<<1, 1, 0, h->stream>>>(h->d_H, m, h->d_cs, h->d_sn, h->d_gv, h->d_h, h->d_c, d_hn, k, d_res,
                                             h->d_flags);
            CKL(h);
            h->launches += 8;
            const int sl = k & 1;
            CK(h, cudaMemcpyAsync(h->h_pin + 4 * sl, h->d_scal, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaMemcpyAsync(h->h_pin_flags + sl, h->d_flags, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaEventRecord(h->ev_step[sl], h->stream));
            return FOGGY_OK;
        };
        // One step of lookahead: step k + 1 is queued before step k is read back, so the GPU does
        // not idle while the host tests convergence.  If step k ends the cycle, step k + 1 has only
        // written column k + 1 of H and entries k + 1, k + 2 of g, which the k + 1 columns solved
        // below never read; it costs one operator application.
        int k = 0;
        bool queued = false;   // step k is on the stream already
        for (; k < m && st->iterations < maxit; ++k) {
            if (!queued) TRY(enqueue_step(k));
            queued = k + 1 < m && st->iterations + 1 < maxit;
            if (queued) TRY(enqueue_step(k + 1));
            CK(h, cudaEventSynchronize(h->ev_step[k & 1]));
            st->iterations++;
            const double* pin = h->h_pin + 4 * (k & 1);
            const int flag = h->h_pin_flags[k & 1];
            if (flag == 2) { status = FOGGY_ERR_NAN; break; }
            if (flag == 1) { status = FOGGY_ERR_BREAKDOWN; break; }
            if (pin[2] / bnorm <= tol || pin[0] == 0.0) { ++k; break; }
        }
        if (status == FOGGY_ERR_NAN) break;
        if (status == FOGGY_ERR_BREAKDOWN) {
            if (k == 0) break;
            status = FOGGY_OK;   // solve with the columns built so far
        }
        if (k > 0) {
            k_trisolve<<<1, 1, 0, h->stream>>>(h->d_H, m, h->d_gv, k, h->d_y);
            k_update_x<<<G, 256, 0, h->stream>>>(h->d_x, h->d_V, n, h->d_y, k, n);
            h->launches += 2;
        }
        st->restarts++;
        TRY(matvec(h->d_x, h->d_w, false));
        k_sub<<<G, 256, 0, h->stream>>>(h->d_b, h->d_w, h->d_r, n);
        h->launches += 1;
        TRY(norm_dev(h, h->d_r, d_beta));
        CK(h, cudaMemcpyAsync(h->h_pin, h->d_scal, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        beta = h->h_pin[1];
        berr = beta / bnorm;
        if (!std::isfinite(berr)) { status = FOGGY_ERR_NAN; break; }
    }
    cleanup();
    st->backward_error = berr;
    if (status == FOGGY_OK && berr > tol) status = FOGGY_ERR_NOT_CONVERGED;
    return status;
}

}  // namespace

// =====================================================================================
extern "C" {

void foggy_default_params(foggy_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->lambda_0 = 0.55;
    p->n_medium = 1.0;
    p->n_range[0] = 1;
    p->n_range[1] = 1;
    p->z_coupling = 1;
    p->reference_row_rule = 1;
    p->matvec_mode = FOGGY_MATVEC_DIRECT;
    p->use_initial_guess = 0;
    p->gmres_restart = 10;
    p->gmres_max_iterations = 1000;
    p->gmres_tolerance = 1e-6;
    p->tree_l_max = 0;
    p->tree_s_opt = 10;
    p->fmm_digits = 0.0;
    p->device_memory_budget = 0;
    p->pair_tables = 0;
    p->fmm_convention = 0;
    p->z_translation_gt_r = 3;
}

static int check_params(foggy_handle h, const foggy_params* p) {
    if (!p) return fail(h, FOGGY_ERR_ARGUMENT, "params is NULL");
    if (!(p->lambda_0 > 0) || !(p->n_medium > 0)) return fail(h, FOGGY_ERR_ARGUMENT, "lambda_0 and n_medium must be > 0");
    if (p->n_range[0] != 1) return fail(h, FOGGY_ERR_UNSUPPORTED, "n_range(1) must be 1");
    if (p->n_range[1] < 1 || p->n_range[1] > kMaxDegree)
        return fail(h, FOGGY_ERR_ARGUMENT, "n_range(2) must be in [1, 45]");
    if (p->z_coupling < 1 || p->z_coupling > 4) return fail(h, FOGGY_ERR_ARGUMENT, "z_coupling must be 1..4");
    if (p->gmres_restart < 1 || p->gmres_restart > 60) return fail(h, FOGGY_ERR_ARGUMENT, "gmres_restart must be 1..60");
    if (p->gmres_max_iterations < 1) return fail(h, FOGGY_ERR_ARGUMENT, "gmres_max_iterations must be >= 1");
    if (!(p->fmm_digits >= 0.0) || p->fmm_digits > 16.0)
        return fail(h, FOGGY_ERR_ARGUMENT, "fmm_digits must be in [0, 16] (0: the global order on every level)");
    if (!(p->gmres_tolerance > 0)) return fail(h, FOGGY_ERR_ARGUMENT, "gmres_tolerance must be > 0");
    if (p->matvec_mode != FOGGY_MATVEC_DIRECT && p->matvec_mode != FOGGY_MATVEC_MLFMM)
        return fail(h, FOGGY_ERR_ARGUMENT, "matvec_mode");
    if (p->fmm_convention != 0 && p->fmm_convention != 1)
        return fail(h, FOGGY_ERR_ARGUMENT, "fmm_convention must be 0 or 1");
    if (p->z_translation_gt_r < 1 || p->z_translation_gt_r > 4)
        return fail(h, FOGGY_ERR_ARGUMENT, "z_translation_gt_r must be 1..4");
    if (p->precision != 0 && p->precision != 1) return fail(h, FOGGY_ERR_ARGUMENT, "precision must be 0 (FP64) or 1 (mixed)");
    return FOGGY_OK;
}

int32_t foggy_create(const foggy_params* params, int32_t device, foggy_handle* out) {
    if (!out) return fail(nullptr, FOGGY_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    int rc = check_params(nullptr, params);
    if (rc) return rc;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(nullptr, FOGGY_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(nullptr, FOGGY_ERR_ARGUMENT, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, FOGGY_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    foggy_handle h = new (std::nothrow) foggy_handle_s();
    if (!h) return fail(nullptr, FOGGY_ERR_NOMEM, "host allocation");
    h->prm = *params;
    h->device = device;
    char* pin = nullptr;
    h->pool = device_pool(device);
    if (!h->pool || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        !(pin = pinned_slot())) {
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return fail(nullptr, FOGGY_ERR_CUDA, "memory pool, stream or pinned allocation failed");
    }
    h->h_pin = reinterpret_cast<double*>(pin);             // 8 doubles
    h->h_pin_flags = reinterpret_cast<int*>(pin + 128);    // 4 ints
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    // memory the pool holds but no allocation uses is free for this handle too
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(h->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(h->pool, cudaMemPoolAttrUsedMemCurrent, &used);
    if (reserved > used) fr += (size_t)(reserved - used);
    h->budget = params->device_memory_budget > 0 ? (size_t)params->device_memory_budget : (size_t)(0.9 * fr);
    *out = h;
    return FOGGY_OK;
}

int32_t foggy_destroy(foggy_handle h) {
    if (!h) return FOGGY_OK;
    cudaSetDevice(h->device);
    for (void* p : h->allocs)
        if (std::find(h->direct_allocs.begin(), h->direct_allocs.end(), p) == h->direct_allocs.end())
            cudaFreeAsync(p, h->stream);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : h->direct_allocs) cudaFree(p);
    h->direct_allocs.clear();
    h->allocs.clear();
    pinned_release(reinterpret_cast<char*>(h->h_pin));
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    if (h->side) cudaStreamSynchronize(h->side);
    for (cudaEvent_t e : {h->ev0, h->ev1, h->evm0, h->evm1, h->ev_step[0], h->ev_step[1], h->ev_fork, h->ev_join})
        if (e) cudaEventDestroy(e);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return FOGGY_OK;
}

const char* foggy_last_error(foggy_handle h) {
    if (h) return h->err.c_str();
    return g_err.c_str();
}

int32_t foggy_set_params(foggy_handle h, const foggy_params* params) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    TRY(check_params(h, params));
    bool scene_change = params->n_range[1] != h->prm.n_range[1] || params->lambda_0 != h->prm.lambda_0 ||
                        params->n_medium != h->prm.n_medium ||
                        params->reference_row_rule != h->prm.reference_row_rule;
    foggy_params old = h->prm;
    h->prm = *params;
    if (params->z_coupling != old.z_coupling) {
        // the pair tables hold S for the old radial function
        h->stab_ready = false;
        h->stab32_ready = false;
    }
    if (params->tree_l_max != old.tree_l_max || params->tree_s_opt != old.tree_s_opt ||
        params->fmm_digits != old.fmm_digits) {
        h->tree_ready = false;
        free_fmm(h);
    }
    if (scene_change && h->N > 0) {
        // rebuild the scene with the new global settings
        std::vector<double> c = h->centres, mr, rad = h->radius;
        std::vector<int> pi = h->pidx, nr = h->nr;
        for (int i = 0; i < h->NP; ++i) {
            mr.push_back(h->mre[i]);
            mr.push_back(h->mim[i]);
        }
        int rc = foggy_set_spheres(h, h->N, c.data(), pi.data(), h->NP, mr.data(), rad.data(), nr.data());
        if (rc) {
            h->prm = old;
            return rc;
        }
    }
    return FOGGY_OK;
}

// The scene of foggy_set_spheres on a handle whose previous scene is freed; the input is checked.
static int32_t load_scene(foggy_handle h, int32_t n_spheres, const double* centres, const int32_t* param_index,
                          int32_t n_param, const double* refractive_index, const double* radius,
                          const int32_t* n_range) {
    const int pg = h->prm.n_range[1];
    h->N = n_spheres;
    h->NP = n_param;
    h->pg = pg;
    h->centres.assign(centres, centres + 3 * (size_t)n_spheres);
    h->pidx.assign(param_index, param_index + n_spheres);
    h->mre.resize(n_param);
    h->mim.resize(n_param);
    h->radius.assign(radius, radius + n_param);
    h->nr.assign(n_range, n_range + 2 * n_param);
    h->p_param.resize(n_param);
    for (int i = 0; i < n_param; ++i) {
        h->mre[i] = refractive_index[2 * i] / h->prm.n_medium;
        h->mim[i] = refractive_index[2 * i + 1] / h->prm.n_medium;
        h->p_param[i] = std::min(n_range[2 * i + 1], pg);
    }
    h->p_s.resize(n_spheres);
    h->couple.resize(n_spheres);
    h->off.resize(n_spheres + 1);
    h->pmax = 0;
    int64_t o = 0;
    for (int j = 0; j < n_spheres; ++j) {
        int ip = param_index[j];
        int p = h->p_param[ip];
        h->p_s[j] = p;
        h->pmax = std::max(h->pmax, p);
        // rows of spheres whose range does not cover the global one carry no coupling
        // (lib_mie_ms_solver_interface.f90:965-978)
        h->couple[j] = (h->prm.reference_row_rule && n_range[2 * ip + 1] < pg) ? 0 : 1;
        h->off[j] = o;
        o += 2 * (int64_t)p * (p + 2);
    }
    h->off[n_spheres] = o;
    h->n_unk = o;
    TRY(ensure_tables(h, std::max(h->pmax, 1)));
    // device scene
    TRY(dalloc(h, &h->d_centres, 3 * (size_t)n_spheres));
    TRY(dalloc(h, &h->d_p, n_spheres));
    TRY(dalloc(h, &h->d_off, n_spheres + 1));
    TRY(dalloc(h, &h->d_couple, n_spheres));
    TRY(dalloc(h, &h->d_an, (size_t)n_spheres * h->pmax));
    TRY(dalloc(h, &h->d_bn, (size_t)n_spheres * h->pmax));
    TRY(dalloc(h, &h->d_an_p, (size_t)n_param * h->pmax));
    TRY(dalloc(h, &h->d_bn_p, (size_t)n_param * h->pmax));
    TRY(dalloc(h, &h->d_b, h->n_unk));
    TRY(dalloc(h, &h->d_pq, h->n_unk));
    TRY(dalloc(h, &h->d_tmp_in, h->n_unk));
    TRY(dalloc(h, &h->d_tmp_out, h->n_unk));
    TRY(plan_direct(h));
    TRY(dalloc(h, &h->d_partial, (size_t)h->nbuckets * h->cmax * h->n_unk));
    CK(h, h2d(h, h->d_centres, centres, 3 * (size_t)n_spheres * sizeof(double)));
    CK(h, h2d(h, h->d_p, h->p_s.data(), n_spheres * sizeof(int)));
    CK(h, h2d(h, h->d_off, h->off.data(), (n_spheres + 1) * sizeof(int64_t)));
    CK(h, h2d(h, h->d_couple, h->couple.data(), n_spheres * sizeof(int)));
    // Mie coefficients per parameter (FP64, device) then gathered per sphere
    std::vector<double> xs(n_param);
    for (int i = 0; i < n_param; ++i) xs[i] = 2.0 * kPi * h->prm.n_medium * radius[i] / h->prm.lambda_0;
    double *d_x = nullptr, *d_mr = nullptr, *d_mi = nullptr;
    int* d_pp = nullptr;
    int* d_pidx = nullptr;
    CK(h, talloc(h, &d_x, n_param * sizeof(double)));
    CK(h, talloc(h, &d_mr, n_param * sizeof(double)));
    CK(h, talloc(h, &d_mi, n_param * sizeof(double)));
    CK(h, talloc(h, &d_pp, n_param * sizeof(int)));
    CK(h, talloc(h, &d_pidx, n_spheres * sizeof(int)));
    CK(h, h2d(h, d_x, xs.data(), n_param * sizeof(double)));
    CK(h, h2d(h, d_mr, h->mre.data(), n_param * sizeof(double)));
    CK(h, h2d(h, d_mi, h->mim.data(), n_param * sizeof(double)));
    CK(h, h2d(h, d_pp, h->p_param.data(), n_param * sizeof(int)));
    CK(h, h2d(h, d_pidx, param_index, n_spheres * sizeof(int)));
    k_mie_ab<<<(n_param + 63) / 64, 64, 0, h->stream>>>(n_param, d_x, d_mr, d_mi, d_pp, h->pmax, h->d_an_p, h->d_bn_p);
    k_gather_an<<<n_spheres, 64, 0, h->stream>>>(n_spheres, d_pidx, h->pmax, h->d_an_p, h->d_bn_p, h->d_an, h->d_bn);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    tfree(h, d_x);
    tfree(h, d_mr);
    tfree(h, d_mi);
    tfree(h, d_pp);
    tfree(h, d_pidx);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("mie: ") + cudaGetErrorString(e));
    CKL(h);
    h->rhs_ready = false;
    return FOGGY_OK;
}

int32_t foggy_set_spheres(foggy_handle h, int32_t n_spheres, const double* centres, const int32_t* param_index,
                          int32_t n_param, const double* refractive_index, const double* radius,
                          const int32_t* n_range) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (n_spheres < 1 || n_param < 1 || !centres || !param_index || !refractive_index || !radius || !n_range)
        return fail(h, FOGGY_ERR_ARGUMENT, "empty or NULL sphere input");
    // all of the input is checked before the handle's scene is touched, so a refused call leaves
    // the previous scene in place
    const int pg = h->prm.n_range[1];
    for (int i = 0; i < n_param; ++i) {
        if (n_range[2 * i] != 1 || n_range[2 * i + 1] < 1)
            return fail(h, FOGGY_ERR_ARGUMENT, "parameter n_range must be [1, n_max], n_max >= 1");
        if (!(radius[i] > 0) || !std::isfinite(radius[i]))
            return fail(h, FOGGY_ERR_ARGUMENT, "radius must be finite and > 0");
        if (!std::isfinite(refractive_index[2 * i]) || !std::isfinite(refractive_index[2 * i + 1]))
            return fail(h, FOGGY_ERR_ARGUMENT, "non-finite refractive index");
    }
    int pmax = 0;
    for (int j = 0; j < n_spheres; ++j) {
        const int ip = param_index[j];
        if (ip < 0 || ip >= n_param) return fail(h, FOGGY_ERR_ARGUMENT, "param_index out of range");
        for (int d = 0; d < 3; ++d)
            if (!std::isfinite(centres[3 * (size_t)j + d])) return fail(h, FOGGY_ERR_ARGUMENT, "non-finite centre");
        pmax = std::max(pmax, std::min(n_range[2 * ip + 1], pg));
    }
    Trace tr("foggy_set_spheres");
    CK(h, cudaSetDevice(h->device));
    free_scene(h);
    const int32_t rc = load_scene(h, n_spheres, centres, param_index, n_param, refractive_index, radius, n_range);
    if (rc != FOGGY_OK) {
        // a device failure part way: no scene rather than a partial one
        free_scene(h);
        h->N = 0;
        h->NP = 0;
        h->n_unk = 0;
    }
    return rc;
}

int32_t foggy_set_plane_waves(foggy_handle h, int32_t nw, const double* theta, const double* phi,
                              const double* jones, const double* g, const double* phase, const double* d_0_i) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (nw < 0 || (nw > 0 && (!theta || !phi || !jones || !g)))
        return fail(h, FOGGY_ERR_ARGUMENT, "negative count or NULL wave input");
    h->waves.clear();
    double k = wavenumber(h->prm);
    for (int i = 0; i < nw; ++i) {
        WaveDev w{};
        // the reference stores the direction as a cartesian vector and converts it back
        // (lib_mie_illumination.f90:421-425, 330-333)
        double rs = k * std::sin(theta[i]);
        w.kc[0] = rs * std::cos(phi[i]);
        w.kc[1] = rs * std::sin(phi[i]);
        w.kc[2] = k * std::cos(theta[i]);
        double rho;
        to_spherical(w.kc, &rho, &w.alpha, &w.beta);
        double ph = phase ? phase[i] : 0.0;
        w.ax = std::hypot(jones[4 * i], jones[4 * i + 1]);
        w.phx = std::atan2(jones[4 * i + 1], jones[4 * i]) + ph;
        w.ay = std::hypot(jones[4 * i + 2], jones[4 * i + 3]);
        w.phy = std::atan2(jones[4 * i + 3], jones[4 * i + 2]) + ph;
        w.g = g[i];
        for (int d = 0; d < 3; ++d) w.d0[d] = d_0_i ? d_0_i[3 * i + d] : 0.0;
        h->waves.push_back(w);
    }
    h->rhs_ready = false;
    return FOGGY_OK;
}

int32_t foggy_set_gaussian_beams(foggy_handle h, int32_t nb, const double* waist, const int32_t* tem,
                                 const double* theta, const double* phi, const double* jones, const double* g,
                                 const double* phase, const double* d_0_i, const int32_t* convention) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (nb < 0 || (nb > 0 && (!waist || !tem || !theta || !phi || !jones || !g)))
        return fail(h, FOGGY_ERR_ARGUMENT, "negative count or NULL beam input");
    std::vector<GaussDev> v;
    for (int i = 0; i < nb; ++i) {
        GaussDev b{};
        b.wx0 = waist[2 * i];
        b.wy0 = waist[2 * i + 1];
        b.tem_m = tem[2 * i];
        b.tem_n = tem[2 * i + 1];
        if (!(b.wx0 > 0.0) || !(b.wy0 > 0.0) || b.tem_m < 0 || b.tem_n < 0 || b.tem_m > 30 || b.tem_n > 30)
            return fail(h, FOGGY_ERR_ARGUMENT, "beam waist must be > 0 and TEM orders in 0..30");
        b.jxr = jones[4 * i];
        b.jxi = jones[4 * i + 1];
        b.jyr = jones[4 * i + 2];
        b.jyi = jones[4 * i + 3];
        if (b.jxr == 0.0 && b.jxi == 0.0 && b.jyr == 0.0 && b.jyi == 0.0)
            return fail(h, FOGGY_ERR_ARGUMENT, "beam Jones vector is zero");
        b.theta = theta[i];
        b.phi = phi[i];
        b.phase = phase ? phase[i] : 0.0;
        b.g = g[i];
        for (int d = 0; d < 3; ++d) b.d0[d] = d_0_i ? d_0_i[3 * i + d] : 0.0;
        b.convention = convention ? convention[i] : 1;
        if (b.convention != 1 && b.convention != 2) return fail(h, FOGGY_ERR_ARGUMENT, "beam convention must be 1 or 2");
        v.push_back(b);
    }
    h->beams = v;
    h->rhs_ready = false;
    return FOGGY_OK;
}

int64_t foggy_vector_length(foggy_handle h) {
    if (!h || h->N == 0) return 0;
    int C = (h->pg + 1) * (h->pg + 1) - 1;
    return (int64_t)2 * C * h->N;
}

int32_t foggy_get_mie_coefficients(foggy_handle h, int32_t ip, double* a, double* b) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (ip < 0 || ip >= h->NP || !a || !b) return fail(h, FOGGY_ERR_ARGUMENT, "parameter index");
    int p = h->p_param[ip];
    CK(h, d2h(h, a, h->d_an_p + (size_t)ip * h->pmax, p * sizeof(cplx)));
    CK(h, d2h(h, b, h->d_bn_p + (size_t)ip * h->pmax, p * sizeof(cplx)));
    return FOGGY_OK;
}

static int stage_ref_buffers(foggy_handle h) {
    size_t len = (size_t)foggy_vector_length(h);
    if (!h->d_ref_a) TRY(dalloc(h, &h->d_ref_a, len));
    if (!h->d_ref_b) TRY(dalloc(h, &h->d_ref_b, len));
    return FOGGY_OK;
}

int32_t foggy_get_vector_b(foggy_handle h, double* b, int32_t mem) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!b) return fail(h, FOGGY_ERR_ARGUMENT, "b is NULL");
    CK(h, cudaSetDevice(h->device));
    TRY(ensure_rhs(h));
    size_t len = (size_t)foggy_vector_length(h);
    cplx* dst = reinterpret_cast<cplx*>(b);
    if (mem == FOGGY_MEM_HOST) {
        TRY(stage_ref_buffers(h));
        dst = h->d_ref_b;
    }
    k_pack<<<h->N, 128, 0, h->stream>>>(scene_view(h), h->pg, h->d_g, h->d_b, nullptr, dst);
    CKL(h);
    if (mem == FOGGY_MEM_HOST)
        CK(h, cudaMemcpyAsync(b, dst, len * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return FOGGY_OK;
}

int32_t foggy_matvec(foggy_handle h, const double* x, double* y, int32_t mem) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x || !y) return fail(h, FOGGY_ERR_ARGUMENT, "x or y is NULL");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    CK(h, cudaSetDevice(h->device));
    size_t len = (size_t)foggy_vector_length(h);
    const cplx* xr = reinterpret_cast<const cplx*>(x);
    cplx* yr = reinterpret_cast<cplx*>(y);
    if (mem == FOGGY_MEM_HOST) {
        TRY(stage_ref_buffers(h));
        CK(h, cudaMemcpyAsync(h->d_ref_a, x, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream));
        xr = h->d_ref_a;
        yr = h->d_ref_b;
    }
    SceneView sv = scene_view(h);
    k_unpack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, xr, h->d_tmp_in);
    TRY(apply_operator(h, h->d_tmp_in, h->d_tmp_out));
    k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, h->d_tmp_out, xr, yr);
    CKL(h);
    if (mem == FOGGY_MEM_HOST)
        CK(h, cudaMemcpyAsync(y, yr, len * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return FOGGY_OK;
}

int32_t foggy_solve(foggy_handle h, const double* x0, double* x, int32_t mem, foggy_stats* stats) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x) return fail(h, FOGGY_ERR_ARGUMENT, "x is NULL");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    Trace tr("foggy_solve");
    CK(h, cudaSetDevice(h->device));
    foggy_stats st{};
    h->launches = 0;
    if (!h->ev0) {
        cudaEventCreate(&h->ev0);
        cudaEventCreate(&h->ev1);
    }
    CK(h, cudaEventRecord(h->ev0, h->stream));
    TRY(ensure_rhs(h));
    TRY(ensure_workspace(h, h->prm.gmres_restart));
    size_t len = (size_t)foggy_vector_length(h);
    SceneView sv = scene_view(h);
    if (x0) {
        const cplx* src = reinterpret_cast<const cplx*>(x0);
        if (mem == FOGGY_MEM_HOST) {
            TRY(stage_ref_buffers(h));
            CK(h, cudaMemcpyAsync(h->d_ref_a, x0, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream));
            src = h->d_ref_a;
        }
        k_unpack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, src, h->d_x);
        h->launches += 1;
    } else if (h->prm.use_initial_guess) {
        // x0 = single-sphere solution a_n p, b_n q (lib_mie_single_sphere.f90:1312-1395)
        CK(h, cudaMemcpyAsync(h->d_x, h->d_b, h->n_unk * sizeof(cplx), cudaMemcpyDeviceToDevice, h->stream));
    } else {
        CK(h, cudaMemsetAsync(h->d_x, 0, h->n_unk * sizeof(cplx), h->stream));
    }
    CKL(h);
    int status = gmres(h, &st);
    if (status == FOGGY_ERR_CUDA || status == FOGGY_ERR_UNSUPPORTED || status == FOGGY_ERR_NOMEM) return status;
    cplx* dst = reinterpret_cast<cplx*>(x);
    if (mem == FOGGY_MEM_HOST) {
        TRY(stage_ref_buffers(h));
        dst = h->d_ref_b;
    }
    k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, h->d_x, nullptr, dst);
    h->launches += 1;
    CKL(h);
    if (mem == FOGGY_MEM_HOST)
        CK(h, cudaMemcpyAsync(x, dst, len * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaEventRecord(h->ev1, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    st.ms_total = ms;
    st.kernel_launches = h->launches;
    st.status = status;
    h->last_berr = st.backward_error;
    if (stats) *stats = st;
    if (status != FOGGY_OK) {
        const char* what = status == FOGGY_ERR_NOT_CONVERGED ? "GMRES did not reach the tolerance"
                           : status == FOGGY_ERR_BREAKDOWN   ? "GMRES breakdown"
                                                             : "NaN or Inf in the residual";
        fail(h, status, what);
    }
    return status;
}

double foggy_get_backward_error(foggy_handle h) { return h ? h->last_berr : -1.0; }

int32_t foggy_get_field(foggy_handle h, const double* x, int32_t mem, int32_t npoints, const double* points,
                        double e_field_0, double* e_out, double* h_out) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x || !points || !e_out || !h_out) return fail(h, FOGGY_ERR_ARGUMENT, "x, points, e_out or h_out is NULL");
    if (npoints < 0) return fail(h, FOGGY_ERR_ARGUMENT, "npoints must be >= 0");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    if (npoints == 0) return FOGGY_OK;
    Trace tr("foggy_get_field");
    CK(h, cudaSetDevice(h->device));
    const size_t len = (size_t)foggy_vector_length(h);
    const int C = (h->pg + 1) * (h->pg + 1) - 1;
    std::vector<double> rad(h->N);
    for (int j = 0; j < h->N; ++j) rad[j] = h->radius[h->pidx[j]];
    const cplx* xd = reinterpret_cast<const cplx*>(x);
    const double* pd = points;
    cplx* ed = reinterpret_cast<cplx*>(e_out);
    cplx* hd = reinterpret_cast<cplx*>(h_out);
    // per-call buffers: sphere radii, and the points and fields when they live on the host
    void* tmp = nullptr;
    const size_t np = (size_t)npoints;
    size_t bytes = rad.size() * sizeof(double);
    if (mem == FOGGY_MEM_HOST) bytes += len * sizeof(cplx) + 3 * np * sizeof(double) + 6 * np * sizeof(cplx);
    CK(h, talloc(h, &tmp, bytes));
    double* d_rad = static_cast<double*>(tmp);
    char* q = reinterpret_cast<char*>(d_rad + rad.size());
    cudaError_t e = cudaMemcpyAsync(d_rad, rad.data(), rad.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (mem == FOGGY_MEM_HOST) {
        cplx* xs = reinterpret_cast<cplx*>(q);
        double* ps = reinterpret_cast<double*>(xs + len);
        ed = reinterpret_cast<cplx*>(ps + 3 * np);
        hd = ed + 3 * np;
        if (e == cudaSuccess) e = cudaMemcpyAsync(xs, x, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ps, points, 3 * np * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        xd = xs;
        pd = ps;
    }
    if (e == cudaSuccess) {
        k_field<<<npoints, 128, 0, h->stream>>>(scene_view(h), d_rad, h->pg, C, xd, pd, e_field_0,
                                                h->prm.n_medium / 299792458.0, ed, hd);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && mem == FOGGY_MEM_HOST) {
        e = cudaMemcpyAsync(e_out, ed, 3 * np * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, hd, 3 * np * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    tfree(h, tmp);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("field: ") + cudaGetErrorString(e));
    return FOGGY_OK;
}

int32_t foggy_solve_rhs(foggy_handle h, int32_t nrhs, const double* x0, double* x, int32_t mem, foggy_stats* stats,
                        double* cross_sections) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x) return fail(h, FOGGY_ERR_ARGUMENT, "x is NULL");
    if (nrhs < 1 || nrhs != (int)h->waves.size())
        return fail(h, FOGGY_ERR_ARGUMENT, "nrhs must equal the number of plane waves set (one right-hand side each)");
    if (!h->beams.empty()) return fail(h, FOGGY_ERR_ARGUMENT, "one right-hand side per plane wave excludes Gaussian beams");
    const size_t len = (size_t)foggy_vector_length(h);
    const std::vector<WaveDev> all = h->waves;
    foggy_stats tot{};
    int status = FOGGY_OK;
    for (int r = 0; r < nrhs && status != FOGGY_ERR_CUDA; ++r) {
        h->waves.assign(1, all[r]);
        h->rhs_ready = false;
        foggy_stats st{};
        double* xr = x + 2 * len * r;
        const double* x0r = x0 ? x0 + 2 * len * r : nullptr;
        const int rc = foggy_solve(h, x0r, xr, mem, &st);
        if (rc == FOGGY_ERR_CUDA || rc == FOGGY_ERR_ARGUMENT || rc == FOGGY_ERR_STATE || rc == FOGGY_ERR_NOMEM ||
            rc == FOGGY_ERR_UNSUPPORTED) {
            h->waves = all;
            h->rhs_ready = false;
            return rc;
        }
        if (rc != FOGGY_OK && status == FOGGY_OK) status = rc;
        if (cross_sections) {
            const int rc2 = foggy_cross_sections(h, xr, mem, cross_sections + 3 * r);
            if (rc2 != FOGGY_OK) {
                h->waves = all;
                h->rhs_ready = false;
                return rc2;
            }
        }
        tot.iterations += st.iterations;
        tot.restarts += st.restarts;
        tot.matvecs += st.matvecs;
        tot.backward_error = std::max(tot.backward_error, st.backward_error);
        tot.ms_total += st.ms_total;
        tot.ms_matvec += st.ms_matvec;
        tot.ms_setup += st.ms_setup;
        tot.kernel_launches += st.kernel_launches;
    }
    h->waves = all;
    h->rhs_ready = false;
    tot.status = status;
    if (stats) *stats = tot;
    return status;
}

}  // extern "C"

namespace foggy {
void raise_smem_ceiling(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> ceiling;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    size_t& c = ceiling[{func, dev}];
    if (bytes > c && cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess)
        c = bytes;
}

// Device bytes a direct-operator solve of this scene holds at its peak, from the same plan the
// handle follows (scene arrays, operator slabs, Krylov workspace, host staging, pair tables).
int64_t estimate_solve_bytes(const foggy_params& prm, int N, const int* param_index, int NP, const int* n_range,
                             int pair_tables, int64_t* table_bytes_out) {
    const int pg = prm.n_range[1];
    std::vector<int> pp(NP);
    for (int i = 0; i < NP; ++i) pp[i] = std::max(1, std::min(n_range[2 * i + 1], pg));
    int64_t n_unk = 0;
    int pmax = 1;
    const int* bounds = kBucketBounds;
    std::vector<int64_t> bucket(kNumBounds, 0), cnt(kMaxDegree + 1, 0);
    for (int j = 0; j < N; ++j) {
        const int p = pp[param_index[j]];
        n_unk += 2 * (int64_t)p * (p + 2);
        pmax = std::max(pmax, p);
        cnt[std::min(p, kMaxDegree)]++;
        for (int b = 1; b < kNumBounds; ++b)
            if (p > bounds[b - 1] && p <= bounds[b]) bucket[b]++;
    }
    int nbuckets = 0, cmax = 1;
    for (int b = 1; b < kNumBounds; ++b)
        if (bucket[b]) {
            ++nbuckets;
            cmax = std::max(cmax, (int)std::max<int64_t>(1, std::min<int64_t>(32, (148 * 6 + bucket[b] - 1) / bucket[b])));
        }
    const int64_t C = (int64_t)(pg + 1) * (pg + 1) - 1, len = 2 * C * N;
    const int64_t v = (int64_t)sizeof(cplx);
    int64_t bytes = 0;
    bytes += (int64_t)N * 64 + (int64_t)(N + NP) * pmax * 2 * v + 4 * n_unk * v;     // scene, b, pq, scratch
    bytes += (int64_t)nbuckets * cmax * n_unk * v;                                        // operator slabs
    bytes += (int64_t)(prm.gmres_restart + 4) * n_unk * v + (int64_t)(prm.gmres_restart + 2) * 2048 * v;
    bytes += 2 * len * v;                                                                 // host staging
    const int64_t q = 2 * pmax + 2;
    bytes += 256 * q * q * q + ((int64_t)64 << 20);                                      // order tables
    if (prm.matvec_mode == FOGGY_MATVEC_MLFMM) {
        // the ML-FMM's box expansions (every sphere's box on every level, at most), the partial sums of
        // its chunked passes on both streams, and its lists; its cached translation blocks are kept only
        // when they fit beside all this
        const int depth = prm.tree_l_max > 0 ? prm.tree_l_max
                                             : std::min(21, 3 + (int)std::ceil(std::log((double)std::max(N, 2)) /
                                                                                std::log(8.0)));
        const int Lb = prm.fmm_digits > 0.0 ? kMaxDegree : pg;
        const int64_t Pb = (int64_t)Lb * (Lb + 2), nbox = (int64_t)N * depth;
        bytes += 2 * nbox * 2 * Pb * v + 2 * (int64_t)2 * kFmmFill * 2 * Pb * v + nbox * 220 * 4 + (int64_t)N * 256;
    }
    int64_t tb = 0;
    if (pair_tables >= 0 && N > 1) {
        for (int a = 1; a <= kMaxDegree; ++a)
            for (int b = a; b <= kMaxDegree; ++b) {
                if (!cnt[a] || !cnt[b]) continue;
                const int64_t pairs = (a == b) ? cnt[a] * (cnt[a] - 1) / 2 : cnt[a] * cnt[b];
                tb += pairs * pair_block_size(a, b) * v;
            }
        tb += (int64_t)N * (N - 1) / 2 * 16 + 16;
    }
    if (prm.precision == 1) tb += tb / 2;   // single-precision tables beside the double ones
    if (table_bytes_out) *table_bytes_out = tb;
    return bytes + (pair_tables == 1 ? tb : 0);
}

int64_t estimate_block_bytes(const foggy_params& prm, int N, const int* param_index, int NP, const int* n_range,
                             int nrhs) {
    const int pg = prm.n_range[1];
    int64_t n_unk = 0;
    for (int j = 0; j < N; ++j) {
        const int p = std::max(1, std::min(n_range[2 * param_index[j] + 1], pg));
        n_unk += 2 * (int64_t)p * (p + 2);
    }
    const int64_t m = prm.gmres_restart, v = (int64_t)sizeof(cplx);
    return (m + 5) * nrhs * n_unk * v + nrhs * ((m + 1) * (m + 5 + kRedBlocks) * v + (m + 5 + kRedBlocks) * 8 + 12);
}
}  // namespace foggy

extern "C" {

// y_v = A x_v for nrhs vectors (reference layout, len entries apart), one operator application each
int32_t foggy_matvec_rhs(foggy_handle h, int32_t nrhs, const double* x, double* y, int32_t mem) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x || !y || nrhs < 1) return fail(h, FOGGY_ERR_ARGUMENT, "x or y is NULL, or nrhs < 1");
    const size_t len = (size_t)foggy_vector_length(h);
    for (int v = 0; v < nrhs; ++v) TRY(foggy_matvec(h, x + 2 * (size_t)v * len, y + 2 * (size_t)v * len, mem));
    return FOGGY_OK;
}

int32_t foggy_cross_sections(foggy_handle h, const double* x, int32_t mem, double* out) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x || !out) return fail(h, FOGGY_ERR_ARGUMENT, "x or out is NULL");
    CK(h, cudaSetDevice(h->device));
    TRY(ensure_rhs(h));
    size_t len = (size_t)foggy_vector_length(h);
    const cplx* src = reinterpret_cast<const cplx*>(x);
    if (mem == FOGGY_MEM_HOST) {
        TRY(stage_ref_buffers(h));
        CK(h, cudaMemcpyAsync(h->d_ref_a, x, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream));
        src = h->d_ref_a;
    }
    SceneView sv = scene_view(h);
    k_unpack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, src, h->d_tmp_in);
    double* d_part = nullptr;
    CK(h, talloc(h, &d_part, 2 * (size_t)h->N * sizeof(double)));
    k_cross_sections<<<h->N, 256, 0, h->stream>>>(sv, h->d_tmp_in, h->d_pq, d_part);
    std::vector<double> part(2 * (size_t)h->N);
    cudaError_t e = cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    tfree(h, d_part);
    if (e != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("cross sections: ") + cudaGetErrorString(e));
    double se = 0, sa = 0;
    for (int j = 0; j < h->N; ++j) {
        se += part[2 * j];
        sa += part[2 * j + 1];
    }
    double k = wavenumber(h->prm);
    double f = 4.0 * kPi / (k * k);
    out[1] = f * se;
    out[2] = f * sa;
    out[0] = out[1] - out[2];
    return FOGGY_OK;
}

double foggy_wigner_3j(int32_t j1, int32_t j2, int32_t j3, int32_t m1, int32_t m2, int32_t m3) {
    return wigner3j(j1, j2, j3, m1, m2, m3);
}

int32_t foggy_translation_coefficients(double x, double theta, double phi, const int32_t n_range[2],
                                       const int32_t nu_range[2], int32_t z_selector, double* A, double* B) {
    if (!n_range || !nu_range || !A || !B) return fail(nullptr, FOGGY_ERR_ARGUMENT, "NULL argument");
    if (n_range[0] < 1 || nu_range[0] < 1 || n_range[1] < n_range[0] || nu_range[1] < nu_range[0] ||
        n_range[1] > 32 || nu_range[1] > 32)
        return fail(nullptr, FOGGY_ERR_ARGUMENT, "degree ranges must lie in [1, 32]");
    if (z_selector < 1 || z_selector > 4) return fail(nullptr, FOGGY_ERR_ARGUMENT, "z_selector must be 1..4");
    if (!(x > 0)) return fail(nullptr, FOGGY_ERR_ARGUMENT, "x must be > 0");
    foggy_params p;
    foggy_default_params(&p);
    int dev = 0;
    cudaGetDevice(&dev);
    foggy_handle h = nullptr;
    int rc = foggy_create(&p, dev, &h);
    if (rc) return rc;
    int pn = n_range[1], pnu = nu_range[1];
    int pmax = std::max(pn, pnu);
    rc = ensure_tables(h, pmax);
    if (rc == FOGGY_OK) rc = ensure_axial_tables(h);
    if (rc) {
        fail(nullptr, rc, h->err);
        foggy_destroy(h);
        return rc;
    }
    AxialView ax{h->tab_pmax, h->d_axoff, h->d_ga, h->d_gb, h->d_koff, reinterpret_cast<const double2*>(h->d_gab)};
    int Pn = pn * (pn + 2), Pnu = pnu * (pnu + 2);
    cplx *dA = nullptr, *dB = nullptr;
    std::vector<cplx> hA((size_t)Pn * Pnu), hB((size_t)Pn * Pnu);
    cudaError_t e = talloc(h, &dA, hA.size() * sizeof(cplx));
    if (e == cudaSuccess) e = talloc(h, &dB, hB.size() * sizeof(cplx));
    if (e == cudaSuccess) {
        size_t smem = translation_pair_smem_bytes(pmax);
        raise_smem_ceiling(reinterpret_cast<const void*>(k_translation_pair), smem);
        k_translation_pair<<<1, 256, smem, h->stream>>>(ax, dtabs(h), x, theta, phi, pn, pnu, z_selector, dA, dB);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hA.data(), dA, hA.size() * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hB.data(), dB, hB.size() * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    tfree(h, dA);
    tfree(h, dB);
    std::vector<double> g;
    build_g_table(pmax, g);
    foggy_destroy(h);
    if (e != cudaSuccess) return fail(nullptr, FOGGY_ERR_CUDA, std::string("translation: ") + cudaGetErrorString(e));
    // back to the reference basis and the requested ranges
    int n1 = n_range[0], nu1 = nu_range[0];
    int cnu = (nu_range[1] + 1) * (nu_range[1] + 1) - nu1 * nu1;
    cplx* Ao = reinterpret_cast<cplx*>(A);
    cplx* Bo = reinterpret_cast<cplx*>(B);
    for (int n = n1; n <= pn; ++n)
        for (int m = -n; m <= n; ++m)
            for (int nu = nu1; nu <= pnu; ++nu)
                for (int mu = -nu; mu <= nu; ++mu) {
                    int r = n * n - 1 + n + m, c = nu * nu - 1 + nu + mu;
                    double sc = g[n * (n + 1) + m] / g[nu * (nu + 1) + mu];
                    size_t o = (size_t)(n * n - n1 * n1 + n + m) * cnu + (nu * nu - nu1 * nu1 + nu + mu);
                    Ao[o] = sc * hA[(size_t)r * Pnu + c];
                    Bo[o] = sc * hB[(size_t)r * Pnu + c];
                }
    return FOGGY_OK;
}

// ---- octree -------------------------------------------------------------------------------
int32_t foggy_build_tree(foggy_handle h, int64_t* uindex_out, int32_t* order_out, int32_t* l_min_out,
                         int32_t* l_max_out) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    CK(h, cudaSetDevice(h->device));
    h->tree_ready = false;
    TRY(build_tree_dev(h));
    int n = h->N;
    if (uindex_out || order_out) {
        std::vector<unsigned long long> ks(n);
        std::vector<int> is(n);
        CK(h, d2h(h, ks.data(), h->d_keys_sorted, n * sizeof(unsigned long long)));
        CK(h, d2h(h, is.data(), h->d_idx_sorted, n * sizeof(int)));
        int sh = 3 * (21 - h->tree_lmax);
        for (int i = 0; i < n; ++i) {
            if (order_out) order_out[i] = is[i];
            if (uindex_out) uindex_out[is[i]] = (int64_t)(ks[i] >> sh);
        }
    }
    if (l_min_out) *l_min_out = h->tree_lmin;
    if (l_max_out) *l_max_out = h->tree_lmax;
    return FOGGY_OK;
}

int32_t foggy_universal_index(int32_t n, const double* points, int32_t l, int64_t* out) {
    if (n < 1 || !points || !out) return fail(nullptr, FOGGY_ERR_ARGUMENT, "empty or NULL input");
    if (l < 1 || l > 21) return fail(nullptr, FOGGY_ERR_ARGUMENT, "level must be 1..21");
    double* dp = nullptr;
    long long* dout = nullptr;
    cudaError_t e = cudaMalloc(&dp, 3 * (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dout, (size_t)n * sizeof(long long));
    if (e == cudaSuccess) e = cudaMemcpy(dp, points, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_uindex_points<<<(n + 255) / 256, 256>>>(n, dp, l, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, (size_t)n * sizeof(long long), cudaMemcpyDeviceToHost);
    cudaFree(dp);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(nullptr, FOGGY_ERR_CUDA, std::string("universal index: ") + cudaGetErrorString(e));
    return FOGGY_OK;
}

int32_t foggy_estimate_solve_bytes(const foggy_params* params, int32_t n_spheres, const int32_t* param_index,
                                   int32_t n_param, const int32_t* n_range, int64_t* solve_bytes,
                                   int64_t* table_bytes) {
    TRY(check_params(nullptr, params));
    if (n_spheres < 1 || n_param < 1 || !param_index || !n_range || !solve_bytes || !table_bytes)
        return fail(nullptr, FOGGY_ERR_ARGUMENT, "empty or NULL input");
    int pmax = 0;
    for (int i = 0; i < n_param; ++i)
        if (n_range[2 * i] != 1 || n_range[2 * i + 1] < 1)
            return fail(nullptr, FOGGY_ERR_ARGUMENT, "parameter n_range must be [1, n_max], n_max >= 1");
    for (int j = 0; j < n_spheres; ++j) {
        if (param_index[j] < 0 || param_index[j] >= n_param)
            return fail(nullptr, FOGGY_ERR_ARGUMENT, "param_index out of range");
        pmax = std::max(pmax, std::min(n_range[2 * param_index[j] + 1], params->n_range[1]));
    }
    *solve_bytes = estimate_solve_bytes(*params, n_spheres, param_index, n_param, n_range, 0, table_bytes);
    return FOGGY_OK;
}

// ---- libtree box arithmetic: integer work on universal indices, on the host ------------------
static int check_box(int64_t n, int32_t l) {
    if (l < 0 || l > 21) return fail(nullptr, FOGGY_ERR_ARGUMENT, "level must be 0..21");
    // every non-negative int64 is a level-21 box (8^21 = 2^63)
    if (n < 0 || (l < 21 && n >= ((int64_t)1 << (3 * l))))
        return fail(nullptr, FOGGY_ERR_ARGUMENT, "box index outside 0..8^l - 1");
    return FOGGY_OK;
}

int32_t foggy_tree_parent(int64_t n, int32_t l, int32_t step, int64_t* parent) {
    if (!parent) return fail(nullptr, FOGGY_ERR_ARGUMENT, "parent is NULL");
    TRY(check_box(n, l));
    if (step < 1 || step > l) return fail(nullptr, FOGGY_ERR_ARGUMENT, "step must be 1..l");
    *parent = n >> (3 * step);
    return FOGGY_OK;
}

int32_t foggy_tree_children(int64_t n, int32_t l, int64_t* children) {
    if (!children) return fail(nullptr, FOGGY_ERR_ARGUMENT, "children is NULL");
    TRY(check_box(n, l));
    if (l == 21) return fail(nullptr, FOGGY_ERR_ARGUMENT, "level 21 boxes have no children");
    for (int j = 0; j < 8; ++j) children[j] = (n << 3) + j;
    return FOGGY_OK;
}

int32_t foggy_tree_centre_of_box(int64_t n, int32_t l, double* centre) {
    if (!centre) return fail(nullptr, FOGGY_ERR_ARGUMENT, "centre is NULL");
    TRY(check_box(n, l));
    box_centre(n, l, centre);
    return FOGGY_OK;
}

int32_t foggy_tree_neighbours(int64_t n, int32_t l, int64_t* out, int32_t* count) {
    if (!out || !count) return fail(nullptr, FOGGY_ERR_ARGUMENT, "out or count is NULL");
    TRY(check_box(n, l));
    std::vector<int64_t> nb;
    tree_i2(n, l, nb);   // own box first, then the neighbours inside the domain
    std::sort(nb.begin() + 1, nb.end());
    *count = (int32_t)nb.size() - 1;
    std::copy(nb.begin() + 1, nb.end(), out);
    return FOGGY_OK;
}

int32_t foggy_tree_boxes(foggy_handle h, int32_t l, int64_t* boxes, int32_t* count) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!count) return fail(h, FOGGY_ERR_ARGUMENT, "count is NULL");
    if (l < 0 || l > 21) return fail(h, FOGGY_ERR_ARGUMENT, "level must be 0..21");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    CK(h, cudaSetDevice(h->device));
    TRY(build_tree_dev(h));
    int n = h->N;
    std::vector<unsigned long long> ks(n);
    CK(h, d2h(h, ks.data(), h->d_keys_sorted, n * sizeof(unsigned long long)));
    int sh = 3 * (21 - l);
    std::vector<int64_t> u;
    for (int i = 0; i < n; ++i) {
        int64_t v = (int64_t)(ks[i] >> sh);
        if (u.empty() || u.back() != v) u.push_back(v);
    }
    if (boxes) {
        if (*count < (int)u.size()) return fail(h, FOGGY_ERR_ARGUMENT, "boxes buffer too small");
        std::copy(u.begin(), u.end(), boxes);
    }
    *count = (int)u.size();
    return FOGGY_OK;
}

int32_t foggy_tree_domain(foggy_handle h, int32_t l, int64_t n, int32_t kind, int64_t* out, int32_t* count) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!count) return fail(h, FOGGY_ERR_ARGUMENT, "count is NULL");
    if (l < 0 || l > 21) return fail(h, FOGGY_ERR_ARGUMENT, "level must be 0..21");
    if (n < 0 || (l < 21 && n >= ((int64_t)1 << (3 * l)))) return fail(h, FOGGY_ERR_ARGUMENT, "box index out of range");
    if (kind != 1 && kind != 2 && kind != 4) return fail(h, FOGGY_ERR_ARGUMENT, "kind must be 1 (E1), 2 (E2) or 4 (I4)");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    CK(h, cudaSetDevice(h->device));
    std::vector<int64_t> v;
    if (kind == 4) {
        tree_i4(n, l, v);
    } else {
        TRY(build_tree_dev(h));
        const int N = h->N;
        std::vector<unsigned long long> ks(N);
        std::vector<int> is(N);
        CK(h, d2h(h, ks.data(), h->d_keys_sorted, N * sizeof(unsigned long long)));
        CK(h, d2h(h, is.data(), h->d_idx_sorted, N * sizeof(int)));
        std::vector<int64_t> boxes;
        if (kind == 1) boxes.push_back(n);
        else tree_i2(n, l, boxes);
        std::sort(boxes.begin(), boxes.end());
        const int sh = 3 * (21 - l);
        for (int64_t b : boxes)
            for (int i = 0; i < N; ++i)
                if ((int64_t)(ks[i] >> sh) == b) v.push_back(is[i]);
    }
    if (out) {
        if (*count < (int)v.size()) return fail(h, FOGGY_ERR_ARGUMENT, "out buffer too small");
        std::copy(v.begin(), v.end(), out);
    }
    *count = (int)v.size();
    return FOGGY_OK;
}

// The ML-FMM's pass lists as built on the device (CSR, pointers then indices): part 0/1
// aggregation (leaf <- spheres), 2/3 children, 4/5 I4, 6/7 parent, 8/9 box to sphere, 10/11 near
// field (sphere <- E2 of its leaf without itself).  Boxes are numbered level by level from l_min
// in ascending Morton order, leaves from the first leaf box.  No counterpart in the reference,
// whose lists live in its hash tables (lib_tree.f90:492-1143).
int32_t foggy_fmm_lists(foggy_handle h, int32_t part, int32_t* out, int32_t* count) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!count) return fail(h, FOGGY_ERR_ARGUMENT, "count is NULL");
    if (part < 0 || part > 11) return fail(h, FOGGY_ERR_ARGUMENT, "part must be 0..11");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    CK(h, cudaSetDevice(h->device));
    TRY(ensure_fmm(h));
    const int beg = h->fmm_lofs[part];
    const int end = part < 11 ? h->fmm_lofs[part + 1] : h->fmm_ltotal;
    if (out) {
        if (*count < end - beg) return fail(h, FOGGY_ERR_ARGUMENT, "out buffer too small");
        if (end > beg) {
            CK(h, cudaMemcpyAsync(out, h->d_fmm_list + beg, (end - beg) * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
        }
    }
    *count = end - beg;
    return FOGGY_OK;
}

}  // extern "C"

// ---- operator without allocation ------------------------------------------------------------
// Working memory of foggy_matvec_static: the two scaled work vectors and one partial-sum slab
// per truncation-order bucket.  It is a fixed array in device memory that exists on every GPU
// this library is loaded on, for the life of the process, and is shared by all calls on that
// GPU.
namespace {
constexpr size_t kStaticScratchBytes = (size_t)32 << 20;   // 32 MiB
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
constexpr int kMaxDevices = 64;
void* g_static_scratch_ptr[kMaxDevices] = {};
std::mutex g_static_mu;
}  // namespace

extern "C" int32_t foggy_matvec_static(foggy_handle h, const double* x, double* y) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x || !y) return fail(h, FOGGY_ERR_ARGUMENT, "x or y is NULL");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    if (h->prm.matvec_mode != FOGGY_MATVEC_DIRECT)
        return fail(h, FOGGY_ERR_UNSUPPORTED, "foggy_matvec_static: only the direct operator");
    if (h->device < 0 || h->device >= kMaxDevices) return fail(h, FOGGY_ERR_ARGUMENT, "device index too large");
    CK(h, cudaSetDevice(h->device));
    // the array's device address, looked up once per GPU on the first call there
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_scratch_ptr[h->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess)
                return fail(h, FOGGY_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_static_scratch_ptr[h->device] = p;
        }
        base = g_static_scratch_ptr[h->device];
    }
    const size_t need = (size_t)h->n_unk * sizeof(cplx) * (2 + (size_t)h->nbuckets);
    if (need > kStaticScratchBytes)
        return fail(h, FOGGY_ERR_ARGUMENT,
                    "foggy_matvec_static: the scene needs " + std::to_string(need) +
                        " bytes of working memory, above the fixed " + std::to_string(kStaticScratchBytes) +
                        " (use foggy_matvec)");
    cplx* xin = reinterpret_cast<cplx*>(base);
    cplx* yout = xin + h->n_unk;
    cplx* partial = yout + h->n_unk;
    // every slab entry that k_direct_finish reads is written by this call's k_direct launches,
    // so nothing in the array needs clearing first
    SceneView sv = scene_view(h);
    const cplx* xr = reinterpret_cast<const cplx*>(x);
    k_unpack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, xr, xin);
    DirectArgs a = direct_args(h, xin);
    a.partial = partial;
    a.cmax = 1;
    for (const DirectBucket& b : h->launches_direct) {
        DirectBucket b1 = b;
        b1.chunks = 1;
        b1.slab = b.slab / h->cmax;
        launch_direct(a, b1, h->stream);
    }
    CKL(h);
    k_direct_finish<<<h->N, 256, 0, h->stream>>>(sv, xin, partial, h->nbuckets, h->n_unk, yout);
    k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, yout, xr, reinterpret_cast<cplx*>(y));
    CKL(h);
    CK(h, cudaStreamSynchronize(h->stream));
    return FOGGY_OK;
}

// ---- several right-hand sides in one block ------------------------------------------------------
// The reference solves each illumination with its own GMRES run (lib_mie_ms_solver_run,
// FoggySim/src/lib/mie_theory/lib_mie_ms_solver_interface.f90:143-154, around
// lib_solver_GMRES.f90:116-316).  Here the right-hand sides of one scene share every operator
// application: k_direct_block applies the operator to a block of vectors, each of its CTAs to a
// tile of R of them, and the Krylov spaces of all right-hand sides advance in lock step (one
// GMRES(m) recurrence per right-hand side, CGS2, Givens, explicit residual at each restart, as in
// gmres()).  Right-hand sides that reach the tolerance at a restart leave the block.
namespace {

// Tile width R per launch shape, chosen by timing: (FP32, pair tables, largest degree, log2 of the
// target count, block width up to 8) -> R.  Process-wide, as the choice depends on the shape only.
std::mutex g_tile_mu;
std::map<std::tuple<int, int, int, int, int>, int> g_tile_cache;

int smem_optin(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    return v;
}

std::vector<int> tile_candidates(bool fp32, int pp, bool tabs, int nrhs, int smem_max) {
    std::vector<int> out;
    const std::vector<int> all = fp32 ? std::vector<int>{1, 2, 4, 8, 16} : std::vector<int>{1, 2, 4, 8};
    for (int R : all) {
        if (R > 1 && R / 2 >= nrhs) break;   // a tile wider than the block would idle
        if (block_smem_bytes(pp, tabs, fp32, R) <= (size_t)smem_max) out.push_back(R);
    }
    return out;
}

auto tile_key(const BlockArgs& ba, const DirectBucket& b, bool tabs) {
    int lt = 0;
    while ((1 << (lt + 1)) <= b.ntargets) ++lt;
    return std::make_tuple(ba.d.fp32, (int)tabs, b.pp, lt, std::min(ba.nrhs, 16));
}

// The autotuner: every candidate width runs the launch's first 296 targets (two CTAs per SM)
// against its first 48 sources for min(nrhs, 16) vectors into a scratch output, once to warm up
// and once timed; the fastest wins.
int choose_tile(foggy_handle h, const BlockArgs& ba, const DirectBucket& b, bool tabs, int* R_out) {
    const auto key = tile_key(ba, b, tabs);
    {
        std::lock_guard<std::mutex> lk(g_tile_mu);
        auto it = g_tile_cache.find(key);
        if (it != g_tile_cache.end()) {
            *R_out = it->second;
            return FOGGY_OK;
        }
    }
    const std::vector<int> cand = tile_candidates(ba.d.fp32, b.pp, tabs, ba.nrhs, smem_optin(h->device));
    if (cand.empty()) return fail(h, FOGGY_ERR_UNSUPPORTED, "no tile width of the block operator fits this degree");
    int best = cand[0];
    if (cand.size() > 1) {
        const int nrt = std::min(ba.nrhs, 16);
        cplx* scratch = nullptr;
        CK(h, talloc(h, &scratch, (size_t)nrt * h->n_unk * sizeof(cplx)));
        BlockArgs bt = ba;
        bt.y = scratch;
        bt.nrhs = nrt;
        DirectBucket db = b;
        db.ntargets = std::min(b.ntargets, 296);
        db.nsources = std::min(b.nsources, 48);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best_ms = 1e30f;
        cudaError_t err = cudaSuccess;
        for (int R : cand) {
            launch_direct_block(bt, db, R, h->stream);
            cudaEventRecord(e0, h->stream);
            launch_direct_block(bt, db, R, h->stream);
            cudaEventRecord(e1, h->stream);
            err = cudaEventSynchronize(e1);
            if (err == cudaSuccess) err = cudaGetLastError();
            if (err != cudaSuccess) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best_ms) {
                best_ms = ms;
                best = R;
            }
            h->launches += 2;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        tfree(h, scratch);
        if (err != cudaSuccess) return fail(h, FOGGY_ERR_CUDA, std::string("block tile tuning: ") + cudaGetErrorString(err));
    }
    std::lock_guard<std::mutex> lk(g_tile_mu);
    g_tile_cache[key] = best;
    *R_out = best;
    return FOGGY_OK;
}

BlockArgs block_args(foggy_handle h, const cplx* X, cplx* Y, int nrhs, bool fp32) {
    BlockArgs ba{};
    ba.d = direct_args(h, nullptr);
    ba.d.fp32 = fp32 ? 1 : 0;
    ba.x = X;
    ba.y = Y;
    ba.nrhs = nrhs;
    ba.ld = h->n_unk;
    return ba;
}

// Y_r = A X_r for r < nrhs (device layout, n_unk apart), FP64 or FP32 translation arithmetic
int apply_operator_block(foggy_handle h, const cplx* X, cplx* Y, int nrhs, bool fp32) {
    if (h->prm.matvec_mode == FOGGY_MATVEC_MLFMM) {
        // the ML-FMM passes one vector after another (their translations are per box, not per pair)
        for (int r = 0; r < nrhs; ++r)
            TRY(apply_operator_fmm(h, X + (size_t)r * h->n_unk, Y + (size_t)r * h->n_unk, fp32));
        return FOGGY_OK;
    }
    TRY(ensure_pair_tables(h));
    const BlockArgs ba = block_args(h, X, Y, nrhs, fp32);
    const bool tabs = fp32 ? ba.d.pt.stab32 != nullptr : ba.d.pt.stab != nullptr;
    Trace tr(fp32 ? "block operator (FP32)" : "block operator (FP64)");
    CK(h, cudaMemcpyAsync(Y, X, (size_t)nrhs * h->n_unk * sizeof(cplx), cudaMemcpyDeviceToDevice, h->stream));
    for (const DirectBucket& b : h->launches_direct) {
        int R = 1;
        TRY(choose_tile(h, ba, b, tabs, &R));
        launch_direct_block(ba, b, R, h->stream);
        h->launches += 1;
    }
    CKL(h);
    return FOGGY_OK;
}

// Workspace of a block of nrhs right-hand sides with restart m; allocated before the pair tables
// so that those are only kept when they fit beside it.
int ensure_block_ws(foggy_handle h, int nrhs, int m) {
    if (h->blk_nrhs >= nrhs && h->blk_m >= m && h->d_bV) return FOGGY_OK;
    free_block(h);
    const size_t n = (size_t)h->n_unk, nb = (size_t)nrhs;
    TRY(dalloc(h, &h->d_bV, (size_t)(m + 1) * nb * n));
    TRY(dalloc(h, &h->d_bW, nb * n));
    TRY(dalloc(h, &h->d_bX, nb * n));
    TRY(dalloc(h, &h->d_bB, nb * n));
    TRY(dalloc(h, &h->d_bR, nb * n));
    // H (m+1) m, cs m, g, h, c, y (m+1) each per slot; dots partials (m+1) kRedBlocks per slot
    TRY(dalloc(h, &h->d_bsmall, nb * ((size_t)(m + 1) * m + m + 4 * (size_t)(m + 1) + (size_t)(m + 1) * kRedBlocks)));
    // sn m, bnorm, beta, hn, tol, res per slot; norm partials kRedBlocks per slot
    TRY(dalloc(h, &h->d_breal, nb * ((size_t)m + 5 + kRedBlocks)));
    TRY(dalloc(h, &h->d_bint, 3 * nb));
    h->blk_nrhs = nrhs;
    h->blk_m = m;
    return FOGGY_OK;
}

struct BlockPtrs {
    cplx *H, *cs, *g, *hh, *c, *y, *part;
    double *sn, *bnorm, *beta, *hn, *tol, *res, *npart;
    int *live, *kend, *flags;
};

BlockPtrs block_ptrs(foggy_handle h) {
    const size_t nb = (size_t)h->blk_nrhs, m = (size_t)h->blk_m;
    BlockPtrs p;
    cplx* c = h->d_bsmall;
    p.H = c;     c += nb * (m + 1) * m;
    p.cs = c;    c += nb * m;
    p.g = c;     c += nb * (m + 1);
    p.hh = c;    c += nb * (m + 1);
    p.c = c;     c += nb * (m + 1);
    p.y = c;     c += nb * (m + 1);
    p.part = c;
    double* d = h->d_breal;
    p.sn = d;    d += nb * m;
    p.bnorm = d; d += nb;
    p.beta = d;  d += nb;
    p.hn = d;    d += nb;
    p.tol = d;   d += nb;
    p.res = d;   d += nb;
    p.npart = d;
    p.live = h->d_bint;
    p.kend = h->d_bint + nb;
    p.flags = h->d_bint + 2 * nb;
    return p;
}

// ||W_b|| for the first ns slots into out[b]
int block_norms(foggy_handle h, const cplx* W, int ns, const int* live, double* out, const BlockPtrs& p) {
    k_norm_partial_b<<<dim3(kRedBlocks, ns), 256, 0, h->stream>>>(W, h->n_unk, h->n_unk, live, p.npart);
    k_norm_reduce_b<<<dim3(1, ns), 256, 0, h->stream>>>(p.npart, live, out, 1);
    h->launches += 2;
    CKL(h);
    return FOGGY_OK;
}

// Batched GMRES over nrhs right-hand sides.  On entry h->d_bB and h->d_bX hold the right-hand sides
// and initial guesses in right-hand-side order (slot r = right-hand side r); slots are reordered as
// right-hand sides leave the block, and emit(a, r) stores slot a's iterate as the solution of
// right-hand side r when it does.  iters / berr / rstatus: per right-hand side.
template <class Emit>
int block_gmres(foggy_handle h, int nrhs, foggy_stats* st, std::vector<int>& iters, std::vector<double>& berr,
                std::vector<int>& rstatus, Emit emit) {
    const int m = h->prm.gmres_restart;
    const int maxit = h->prm.gmres_max_iterations;
    const double tol = h->prm.gmres_tolerance;
    const int64_t n = h->n_unk;
    const size_t vb = (size_t)n * sizeof(cplx);
    const bool mixed = h->prm.precision == 1;
    const int G = grid_for(n);
    const BlockPtrs p = block_ptrs(h);
    const size_t ldi = (size_t)h->blk_nrhs * n;   // basis vector i -> i + 1 of one slot
    iters.assign(nrhs, 0);
    berr.assign(nrhs, 0.0);
    rstatus.assign(nrhs, FOGGY_OK);
    std::vector<int> rhs_of(nrhs);
    for (int r = 0; r < nrhs; ++r) rhs_of[r] = r;
    cudaEvent_t ea, eb;
    cudaEventCreate(&ea);
    cudaEventCreate(&eb);
    auto matvec = [&](const cplx* Xin, cplx* Yout, int ns, bool arnoldi) -> int {
        cudaEventRecord(ea, h->stream);
        const int r = apply_operator_block(h, Xin, Yout, ns, arnoldi && mixed);
        cudaEventRecord(eb, h->stream);
        cudaEventSynchronize(eb);
        float ms = 0;
        cudaEventElapsedTime(&ms, ea, eb);
        st->ms_matvec += ms;
        st->matvecs += ns;
        return r;
    };
    auto done = [&]() {
        cudaEventDestroy(ea);
        cudaEventDestroy(eb);
    };
    int nact = nrhs;
    TRY(block_norms(h, h->d_bB, nact, nullptr, p.bnorm, p));
    std::vector<double> hb(nrhs), hbeta(nrhs);
    std::vector<int> hlive(nrhs), hflags(nrhs);
    CK(h, cudaMemcpyAsync(hb.data(), p.bnorm, nrhs * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    // residuals of the current iterates; slots that meet the tolerance (or failed) leave the block
    auto residuals = [&]() -> int {
        int r_ = matvec(h->d_bX, h->d_bW, nact, false);
        if (r_) return r_;
        k_sub_b<<<dim3(G, nact), 256, 0, h->stream>>>(h->d_bB, h->d_bW, h->d_bR, n, n);
        h->launches += 1;
        TRY(block_norms(h, h->d_bR, nact, nullptr, p.beta, p));
        CK(h, cudaMemcpyAsync(hbeta.data(), p.beta, nact * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        for (int a = nact - 1; a >= 0; --a) {
            const int r = rhs_of[a];
            const double e = hb[a] == 0.0 ? 0.0 : hbeta[a] / hb[a];
            berr[r] = e;
            int out = -1;
            if (!std::isfinite(e)) out = FOGGY_ERR_NAN;
            else if (e <= tol) out = FOGGY_OK;
            else if (iters[r] >= maxit) out = FOGGY_ERR_NOT_CONVERGED;
            else if (rstatus[r] == FOGGY_ERR_BREAKDOWN) out = FOGGY_ERR_BREAKDOWN;
            if (out == -1) continue;
            rstatus[r] = out;
            if (hb[a] == 0.0) CK(h, cudaMemsetAsync(h->d_bX + (size_t)a * n, 0, vb, h->stream));
            TRY(emit(a, r));
            const int last = nact - 1;
            if (a != last) {
                CK(h, cudaMemcpyAsync(h->d_bX + (size_t)a * n, h->d_bX + (size_t)last * n, vb, cudaMemcpyDeviceToDevice, h->stream));
                CK(h, cudaMemcpyAsync(h->d_bB + (size_t)a * n, h->d_bB + (size_t)last * n, vb, cudaMemcpyDeviceToDevice, h->stream));
                CK(h, cudaMemcpyAsync(h->d_bR + (size_t)a * n, h->d_bR + (size_t)last * n, vb, cudaMemcpyDeviceToDevice, h->stream));
                rhs_of[a] = rhs_of[last];
                hb[a] = hb[last];
                hbeta[a] = hbeta[last];
            }
            --nact;
        }
        CK(h, cudaMemcpyAsync(p.bnorm, hb.data(), nact * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(h, cudaMemcpyAsync(p.beta, hbeta.data(), nact * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        return FOGGY_OK;
    };
    int rc = residuals();
    if (rc) { done(); return rc; }
    std::vector<double> htol(nrhs);
    while (nact > 0) {
        for (int a = 0; a < nact; ++a) htol[a] = tol * hb[a];
        CK(h, cudaMemcpyAsync(p.tol, htol.data(), nact * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        k_scale_copy_b<<<dim3(G, nact), 256, 0, h->stream>>>(h->d_bR, n, p.beta, 1, h->d_bV, n, n, nullptr);
        k_init_cycle_b<<<(nact + 63) / 64, 64, 0, h->stream>>>(p.g, m + 1, p.beta, nact, p.live, p.kend);
        CK(h, cudaMemsetAsync(p.flags, 0, nact * sizeof(int), h->stream));
        h->launches += 2;
        // the cycle's steps; a slot may stop early (converged estimate, breakdown, iteration limit)
        int steps = m;
        for (int a = 0; a < nact; ++a) steps = std::min(steps, std::max(1, maxit - iters[rhs_of[a]]));
        for (int k = 0; k < m; ++k) {
            cplx* Vk = h->d_bV + (size_t)k * ldi;
            cplx* Vk1 = h->d_bV + (size_t)(k + 1) * ldi;
            rc = matvec(Vk, h->d_bW, nact, true);
            if (rc) { done(); return rc; }
            for (int pass = 0; pass < 2; ++pass) {
                cplx* coef = pass ? p.c : p.hh;
                k_dots_partial_b<<<dim3(kRedBlocks, nact), 256, 0, h->stream>>>(h->d_bV, ldi, n, k + 1, h->d_bW, n,
                                                                                p.live, p.part);
                k_dots_reduce_b<<<dim3(k + 1, nact), 256, 0, h->stream>>>(p.part, k + 1, p.live, coef, m + 1);
                k_axpy_multi_b<<<dim3(G, nact), 256, 0, h->stream>>>(h->d_bV, ldi, n, k + 1, coef, m + 1, h->d_bW, n,
                                                                     p.live);
            }
            TRY(block_norms(h, h->d_bW, nact, p.live, p.hn, p));
            k_scale_copy_b<<<dim3(G, nact), 256, 0, h->stream>>>(h->d_bW, n, p.hn, 1, Vk1, n, n, p.live);
            k_givens_b<<<(nact + 63) / 64, 64, 0, h->stream>>>(p.H, m, p.cs, p.sn, p.g, p.hh, p.c, p.hn, k, p.tol,
                                                                p.res, p.flags, p.live, p.kend, nact);
            h->launches += 8;
            CKL(h);
            // slots live at this step did an Arnoldi step
            std::vector<int> was(hlive.begin(), hlive.begin() + nact);
            if (k == 0) std::fill(was.begin(), was.end(), 1);
            CK(h, cudaMemcpyAsync(hlive.data(), p.live, nact * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaMemcpyAsync(hflags.data(), p.flags, nact * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
            int any = 0;
            for (int a = 0; a < nact; ++a) {
                if (was[a]) iters[rhs_of[a]]++, st->iterations++;
                if (hflags[a] == 2) rstatus[rhs_of[a]] = FOGGY_ERR_NAN;
                // a breakdown before any column leaves nothing to update with; later ones solve with
                // the columns built so far, as gmres() does
                if (hflags[a] == 1 && k == 0) rstatus[rhs_of[a]] = FOGGY_ERR_BREAKDOWN;
                any |= hlive[a];
            }
            if (!any || k + 1 >= steps) break;
        }
        k_trisolve_b<<<(nact + 63) / 64, 64, 0, h->stream>>>(p.H, m, p.g, p.kend, p.y, nact);
        k_update_x_b<<<dim3(G, nact), 256, 0, h->stream>>>(h->d_bX, n, h->d_bV, ldi, p.y, m + 1, p.kend, n);
        h->launches += 2;
        CKL(h);
        st->restarts++;
        rc = residuals();
        if (rc) { done(); return rc; }
    }
    done();
    int status = FOGGY_OK;
    double worst = 0.0;
    for (int r = 0; r < nrhs; ++r) {
        worst = std::max(worst, berr[r]);
        if (rstatus[r] != FOGGY_OK && status == FOGGY_OK) status = rstatus[r];
    }
    st->backward_error = worst;
    return status;
}

}  // namespace

extern "C" {

int32_t foggy_matvec_block(foggy_handle h, int32_t nrhs, int32_t precision, const double* x, double* y, int32_t mem) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x || !y || nrhs < 1) return fail(h, FOGGY_ERR_ARGUMENT, "x or y is NULL, or nrhs < 1");
    if (precision != 0 && precision != 1) return fail(h, FOGGY_ERR_ARGUMENT, "precision must be 0 (FP64) or 1 (FP32)");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    CK(h, cudaSetDevice(h->device));
    TRY(stage_ref_buffers(h));
    const size_t len = (size_t)foggy_vector_length(h);
    const size_t n = (size_t)h->n_unk;
    cplx* X = nullptr;
    TRY(dalloc(h, &X, 2 * (size_t)nrhs * n));
    cplx* Y = X + (size_t)nrhs * n;
    SceneView sv = scene_view(h);
    auto fin = [&](int rc) {
        dfree(h, X);
        return rc;
    };
    for (int r = 0; r < nrhs; ++r) {
        const cplx* src = reinterpret_cast<const cplx*>(x) + r * len;
        if (mem == FOGGY_MEM_HOST) {
            if (cudaMemcpyAsync(h->d_ref_a, src, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
                return fin(fail(h, FOGGY_ERR_CUDA, "foggy_matvec_block: host to device copy"));
            src = h->d_ref_a;
        }
        k_unpack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, src, X + (size_t)r * n);
    }
    int rc = apply_operator_block(h, X, Y, nrhs, precision == 1);
    if (rc) return fin(rc);
    for (int r = 0; r < nrhs; ++r) {
        const cplx* xr = reinterpret_cast<const cplx*>(x) + r * len;
        cplx* dst = reinterpret_cast<cplx*>(y) + r * len;
        if (mem == FOGGY_MEM_HOST) {
            // the identity rows above a sphere's degree come from x, staged again
            cudaMemcpyAsync(h->d_ref_a, xr, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream);
            xr = h->d_ref_a;
            k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, Y + (size_t)r * n, xr, h->d_ref_b);
            cudaMemcpyAsync(dst, h->d_ref_b, len * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream);
        } else {
            k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, Y + (size_t)r * n, xr, dst);
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fin(fail(h, FOGGY_ERR_CUDA, std::string("foggy_matvec_block: ") + cudaGetErrorString(e)));
    return fin(FOGGY_OK);
}

int32_t foggy_solve_block(foggy_handle h, int32_t nrhs, const double* x0, double* x, int32_t mem, foggy_stats* stats,
                          double* cross_sections, int32_t* iterations, double* backward_errors) {
    if (!h) return fail(nullptr, FOGGY_ERR_ARGUMENT, "handle is NULL");
    if (!x) return fail(h, FOGGY_ERR_ARGUMENT, "x is NULL");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    if (nrhs < 1 || nrhs != (int)h->waves.size())
        return fail(h, FOGGY_ERR_ARGUMENT, "nrhs must equal the number of plane waves set (one right-hand side each)");
    if (!h->beams.empty()) return fail(h, FOGGY_ERR_ARGUMENT, "one right-hand side per plane wave excludes Gaussian beams");
    if (h->prm.gmres_restart < 1 || h->prm.gmres_restart > 63)
        return fail(h, FOGGY_ERR_ARGUMENT, "gmres_restart must be 1..63 for the block solve");
    Trace tr("foggy_solve_block");
    CK(h, cudaSetDevice(h->device));
    foggy_stats st{};
    h->launches = 0;
    if (!h->ev0) {
        cudaEventCreate(&h->ev0);
        cudaEventCreate(&h->ev1);
    }
    CK(h, cudaEventRecord(h->ev0, h->stream));
    TRY(ensure_block_ws(h, nrhs, h->prm.gmres_restart));
    TRY(stage_ref_buffers(h));
    const size_t len = (size_t)foggy_vector_length(h);
    const size_t n = (size_t)h->n_unk;
    SceneView sv = scene_view(h);
    // right-hand sides, one per plane wave, and initial guesses, in right-hand-side order
    const std::vector<WaveDev> all = h->waves;
    int rc = FOGGY_OK;
    for (int r = 0; r < nrhs && rc == FOGGY_OK; ++r) {
        h->waves.assign(1, all[r]);
        h->rhs_ready = false;
        rc = ensure_rhs(h);
        if (rc) break;
        cudaError_t e = cudaMemcpyAsync(h->d_bB + r * n, h->d_b, n * sizeof(cplx), cudaMemcpyDeviceToDevice, h->stream);
        if (e == cudaSuccess) {
            if (x0) {
                const cplx* src = reinterpret_cast<const cplx*>(x0) + r * len;
                if (mem == FOGGY_MEM_HOST) {
                    e = cudaMemcpyAsync(h->d_ref_a, src, len * sizeof(cplx), cudaMemcpyHostToDevice, h->stream);
                    src = h->d_ref_a;
                }
                k_unpack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, src, h->d_bX + r * n);
                h->launches += 1;
            } else if (h->prm.use_initial_guess) {
                e = cudaMemcpyAsync(h->d_bX + r * n, h->d_b, n * sizeof(cplx), cudaMemcpyDeviceToDevice, h->stream);
            } else {
                e = cudaMemsetAsync(h->d_bX + r * n, 0, n * sizeof(cplx), h->stream);
            }
        }
        if (e != cudaSuccess) rc = fail(h, FOGGY_ERR_CUDA, std::string("foggy_solve_block: ") + cudaGetErrorString(e));
    }
    h->waves = all;
    h->rhs_ready = false;
    if (rc) return rc;
    // a right-hand side that leaves the block is written to x at once (reference layout)
    auto emit = [&](int a, int r) -> int {
        cplx* dst = reinterpret_cast<cplx*>(x) + (size_t)r * len;
        if (mem == FOGGY_MEM_HOST) {
            k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, h->d_bX + (size_t)a * n, nullptr, h->d_ref_b);
            CK(h, cudaMemcpyAsync(dst, h->d_ref_b, len * sizeof(cplx), cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
        } else {
            k_pack<<<h->N, 128, 0, h->stream>>>(sv, h->pg, h->d_g, h->d_bX + (size_t)a * n, nullptr, dst);
        }
        h->launches += 1;
        CKL(h);
        return FOGGY_OK;
    };
    std::vector<int> its, rst;
    std::vector<double> be;
    const int status = block_gmres(h, nrhs, &st, its, be, rst, emit);
    if (status == FOGGY_ERR_CUDA || status == FOGGY_ERR_UNSUPPORTED || status == FOGGY_ERR_NOMEM) return status;
    CK(h, cudaEventRecord(h->ev1, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    st.ms_total = ms;
    st.kernel_launches = h->launches;
    st.status = status;
    h->last_berr = st.backward_error;
    for (int r = 0; r < nrhs; ++r) {
        if (iterations) iterations[r] = its[r];
        if (backward_errors) backward_errors[r] = be[r];
    }
    if (cross_sections) {
        for (int r = 0; r < nrhs; ++r) {
            h->waves.assign(1, all[r]);
            h->rhs_ready = false;
            const int rc2 = foggy_cross_sections(h, x + 2 * len * r, mem, cross_sections + 3 * r);
            if (rc2 != FOGGY_OK) {
                h->waves = all;
                h->rhs_ready = false;
                return rc2;
            }
        }
        h->waves = all;
        h->rhs_ready = false;
    }
    if (stats) *stats = st;
    if (status != FOGGY_OK) {
        const char* what = status == FOGGY_ERR_NOT_CONVERGED ? "GMRES did not reach the tolerance for every right-hand side"
                           : status == FOGGY_ERR_BREAKDOWN   ? "GMRES breakdown"
                                                             : "NaN or Inf in a residual";
        fail(h, status, what);
    }
    return status;
}

// Tile width of each operator launch (tuned on first use) for a block of nrhs vectors:
// out[4 i .. 4 i + 3] = (targets, sources, largest degree, tile width) of launch i.
int32_t foggy_block_tiles(foggy_handle h, int32_t precision, int32_t nrhs, int32_t* out, int32_t* count) {
    if (!h || !count) return fail(h, FOGGY_ERR_ARGUMENT, "handle or count is NULL");
    if (h->N == 0) return fail(h, FOGGY_ERR_STATE, "no spheres set");
    if (nrhs < 1) return fail(h, FOGGY_ERR_ARGUMENT, "nrhs < 1");
    CK(h, cudaSetDevice(h->device));
    *count = (int)h->launches_direct.size();
    if (!out) return FOGGY_OK;
    TRY(ensure_pair_tables(h));
    // the tuner reads the first min(nrhs, 16) vectors of the block: zeros serve
    cplx* X = nullptr;
    const int nrt = std::min(nrhs, 16);
    TRY(dalloc(h, &X, (size_t)nrt * h->n_unk));
    CK(h, cudaMemsetAsync(X, 0, (size_t)nrt * h->n_unk * sizeof(cplx), h->stream));
    BlockArgs ba = block_args(h, X, nullptr, nrhs, precision == 1);
    const bool tabs = ba.d.fp32 ? ba.d.pt.stab32 != nullptr : ba.d.pt.stab != nullptr;
    int rc = FOGGY_OK;
    for (size_t i = 0; i < h->launches_direct.size() && rc == FOGGY_OK; ++i) {
        const DirectBucket& b = h->launches_direct[i];
        int R = 0;
        rc = choose_tile(h, ba, b, tabs, &R);
        out[4 * i] = b.ntargets;
        out[4 * i + 1] = b.nsources;
        out[4 * i + 2] = b.pp;
        out[4 * i + 3] = R;
    }
    dfree(h, X);
    return rc;
}

}  // extern "C"
