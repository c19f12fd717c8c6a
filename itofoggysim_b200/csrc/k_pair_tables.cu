// Pair tables of every sphere pair, kept in HBM for the operator: the single-precision ones (the
// mixed-precision operator) as tensor-core products, tcgen05.mma kind::tf32 with every operand split
// into a TF32 high and low part (3xTF32: hi*hi + hi*lo + lo*hi, FP32 accumulation in tensor memory);
// the double-precision ones summed in FP64 on the CUDA cores over the same groups of pairs.
//
// Row e of the block of an unordered sphere pair (s, t) is the scalar coaxial coefficient
// S(k; a, b) that k_pair_s sums (k = 0..min(p_s, p_t), a, b = k..M+1, M = max(p_s, p_t)):
//     S[e] = sum_p G[e][p] zeta_p,   zeta_p = i^p z_p(k |d_t - d_s|),
//     G[e][p] = (2p+1)(a b p; -k k 0)(a b p; 0 0 0) for p = a + b - 2q, q = 0..min(a, b), else 0.
// G depends on M2 = M + 2 alone (a pair with a smaller min(p_s, p_t) owns a prefix of the rows of
// the block of two spheres of order M), so the tables of all pairs of one M2 are one product
//     T[e][n] = sum_p G[e][p] Z[n][p],   column n = (pair, re | im),
// M = 128 rows e per MMA, N = 2 x the pairs of a CTA, K = the degrees p = 0..2 M2 - 2 padded to 8.
// G is packed once per handle in the operand layout of the MMA (k_tc_pack_a, split in FP64); each
// CTA computes the Bessel functions of its pairs, splits their zeta into the B operand, and walks a
// run of up to 8 of the 128-row tiles of its group: a bulk copy brings tile m + 2 while the MMAs of
// tile m + 1 run and eight epilogue warps (two per TMEM lane quarter, one per half of the columns)
// read tile m out of tensor memory (two accumulators) into the tables.
#include <algorithm>
#include <cstdint>

#include "foggy_kernels.cuh"
#include "k_common.cuh"
#include "k_special.cuh"

namespace foggy {

namespace {

constexpr int kTcRows = 128;            // rows e per tile (M of one MMA)
constexpr int kTcEpiWarps = 8;          // warps 0-7: epilogue (warp w: TMEM lanes 32 (w % 4).., column half w / 4)
constexpr int kTcThreads = 32 * (kTcEpiWarps + 1);   // + warp 8: bulk copies and MMAs
constexpr uint32_t kTcCols = 256;       // TMEM columns: two accumulators of up to 128 columns
constexpr long long kTcSpin = 4000000000LL;   // clock cycles a wait may take before it gives up (~2 s)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// round to the nearest TF32 (10 explicit mantissa bits), ties away from zero
__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Float offset of element (r, k) of a K-major tile of R rows in the MMA's canonical layout without
// swizzle: 8-row x 16-byte core matrices, 128 bytes each, the R/8 row groups of one 4-wide K chunk
// one after the other (stride 128 bytes), then the next K chunk (stride 16 R bytes).
__host__ __device__ __forceinline__ int64_t tc_canon(int r, int k, int R) {
    return ((int64_t)(k >> 2) * (R >> 3) + (r >> 3)) * 32 + (r & 7) * 4 + (k & 3);
}

// shared-memory matrix descriptor: start, leading (K chunk) and stride (row group) byte offsets,
// descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor of kind::tf32: FP32 accumulator, A and B TF32 and K-major, N and M
__host__ __device__ __forceinline__ uint32_t tc_idesc(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of the given parity to complete, at most kTcSpin cycles; a wait that runs out
// raises the CTA's abort flag, and every wait gives up once the flag is raised.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
    const long long t0 = clock64();
    while (!mbar_test(bar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > kTcSpin) {
            *abort = 1;
            return false;
        }
    }
    return true;
}
// the same without looking at the abort flag (draining copies and MMAs in flight after an abort)
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_test(bar, parity) && clock64() - t0 <= kTcSpin) {
    }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// rows (k, a, b) of the full block of M2 (two spheres of order M2 - 2)
__host__ __device__ __forceinline__ int64_t tc_rows(int M2) { return pair_block_offset(M2 - 1, M2, M2); }

}  // namespace

int64_t tc_group_rows(int M2) { return tc_rows(M2); }
int tc_group_k(int M2) { return ((2 * M2 - 1) + 7) / 8 * 8; }
int tc_group_pairs(int K) { return K <= 72 ? 64 : 16; }
size_t tc_smem_bytes(int K, int np) {
    // two A tiles (hi, lo) of 128 x K, the B operand (hi, lo) of 2 np x K, 128 bytes of alignment;
    // at least 80 KB so that no more than two CTAs (2 x 256 TMEM columns) share an SM
    size_t b = 2 * (size_t)(2 * kTcRows * K) * 4 + (size_t)(2 * 2 * np * K) * 4 + 128;
    return b < 80 * 1024 ? 80 * 1024 : b;
}

// G of one M2 in the A layout: tile m (rows 128 m .. 128 m + 127) at out + a_off + 2 * 128 * K * m,
// its TF32 high parts then its low parts, rows past the block zero.
__global__ void k_tc_pack_a(SGaunt g, TcGroup gr, float* out) {
    const int K = gr.K, M2 = gr.M2, km = M2 - 2;
    const int64_t rows = tc_rows(M2);
    const int64_t total = (int64_t)gr.mtiles * kTcRows * K;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = idx / K;
        const int p = (int)(idx - e * K);
        double c = 0.0;
        if (e < rows) {
            int k = 0;
            while (k < km && pair_block_offset(k + 1, M2, M2) <= e) ++k;
            const int64_t r = e - pair_block_offset(k, M2, M2);
            const int cols = M2 - k;
            const int aa = k + (int)(r / cols), bb = k + (int)(r % cols);
            const int lo = aa > bb ? aa - bb : bb - aa;
            if (p >= lo && p <= aa + bb && ((aa + bb - p) & 1) == 0) {
                const int q = (aa + bb - p) >> 1;
                const int W = g.NM - k + 1;
                c = g.gs[g.koff[k] + (size_t)q * W * W + (size_t)(aa - k) * W + (bb - k)];
            }
        }
        const float hi = tf32_rna((float)c);
        const float lo = tf32_rna((float)(c - (double)hi));
        const int64_t m = e / kTcRows;
        const int rr = (int)(e - m * kTcRows);
        float* t = out + gr.a_off + m * 2 * kTcRows * K;
        const int64_t o = tc_canon(rr, p, kTcRows);
        t[o] = hi;
        t[(int64_t)kTcRows * K + o] = lo;
    }
}

// One CTA per tile of up to np pairs of one group: B operand from the pairs' zeta, then the 128-row
// tiles of A through two shared-memory buffers and two TMEM accumulators.
__global__ void __launch_bounds__(kTcThreads) k_pair_tc(TcArgs a, int tile0) {
    extern __shared__ __align__(128) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t bar_full[2], bar_mma[2], bar_empty[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    __shared__ int64_t s_off[64], s_tot[64];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TcTile tl = a.tiles[tile0 + blockIdx.x];
    const TcGroup gr = a.groups[tl.group];
    const int K = gr.K, np = gr.np, N = 2 * np, P = 2 * gr.M2 - 2, m0 = tl.m0, mt = tl.m1 - tl.m0;

    const uint32_t raw = smem_u32(tc_smem_raw);
    unsigned char* base = tc_smem_raw + (((raw + 127u) & ~127u) - raw);
    float* abuf0 = reinterpret_cast<float*>(base);
    float* abuf1 = abuf0 + 2 * kTcRows * K;
    float* bhi = abuf1 + 2 * kTcRows * K;
    float* blo = bhi + N * K;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bar_full[b]), 1);
            mbar_init(smem_u32(&bar_mma[b]), 1);
            mbar_init(smem_u32(&bar_empty[b]), kTcEpiWarps * 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    // the pairs' Bessel functions in the (not yet used) A buffers: pair i at scr + 2 (P + 1) i
    double* scr = reinterpret_cast<double*>(abuf0);
    for (int i = tid; i < tl.count; i += kTcThreads) {
        const int2 st = a.pairs[tl.first + i];
        const double* cs = a.sc.centres + 3 * (size_t)st.x;
        const double* ct = a.sc.centres + 3 * (size_t)st.y;
        const double d0 = a.sc.k * (ct[0] - cs[0]), d1 = a.sc.k * (ct[1] - cs[1]), d2 = a.sc.k * (ct[2] - cs[2]);
        const double rho = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double* jb = scr + (size_t)2 * (P + 1) * i;
        dev_sph_jn(rho, P, jb);
        if (a.z != 1) dev_sph_yn(rho, P, jb + P + 1);
        s_off[i] = a.pair_off[pair_index(st.x, st.y, a.sc.n)];
        s_tot[i] = pair_block_size(a.sc.p[st.x], a.sc.p[st.y]);
    }
    __syncthreads();
    // B operand: row 2i the real parts of pair i's zeta_p, row 2i + 1 the imaginary parts
    for (int idx = tid; idx < N * K; idx += kTcThreads) {
        const int n = idx / K, p = idx - n * K, i = n >> 1;
        float hi = 0.f, lo = 0.f;
        if (i < tl.count && p <= P) {
            const double* jb = scr + (size_t)2 * (P + 1) * i;
            const cplx zc = zeta_of(a.z, p, jb, jb + P + 1);
            const double v = (n & 1) ? zc.y : zc.x;
            hi = tf32_rna((float)v);
            lo = tf32_rna((float)(v - (double)hi));
        }
        const int64_t o = tc_canon(n, p, N);
        bhi[o] = hi;
        blo[o] = lo;
    }
    // the generic-proxy writes above (B, and the scratch the bulk copies will overwrite) before any
    // tensor-core read or bulk copy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (warp == kTcEpiWarps) {
        if (lane == 0) {
            const uint32_t abytes = (uint32_t)(2 * kTcRows * K * 4);
            const float* ga = a.a + gr.a_off;
            const uint32_t sa[2] = {smem_u32(abuf0), smem_u32(abuf1)};
            const uint32_t sbh = smem_u32(bhi), sbl = smem_u32(blo);
            const uint32_t idesc = tc_idesc(kTcRows, N);
            const uint32_t lbo_a = 16 * kTcRows, lbo_b = 16 * N;   // bytes between K chunks
            const uint32_t step_a = 32 * kTcRows, step_b = 32 * N;  // bytes per K slice of 8
            const uint32_t lo_a = (uint32_t)(kTcRows * K * 4);
            int loaded = 0, consumed = 0, issued = 0;
            // j: the CTA's own tile count (buffers and phases), m0 + j: the tile of the group
            auto load = [&](int j) {
                const int b = j & 1;
                mbar_expect_tx(smem_u32(&bar_full[b]), abytes);
                bulk_g2s(sa[b], ga + (size_t)(m0 + j) * 2 * kTcRows * K, abytes, smem_u32(&bar_full[b]));
                ++loaded;
            };
            load(0);
            if (mt > 1) load(1);
            for (int m = 0; m < mt; ++m) {
                const int b = m & 1;
                if (!mbar_wait(smem_u32(&bar_full[b]), (m >> 1) & 1, &s_abort)) break;
                consumed = m + 1;
                if (m >= 2 && !mbar_wait(smem_u32(&bar_empty[b]), ((m - 2) >> 1) & 1, &s_abort)) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * 128);
                for (int s = 0; s < K / 8; ++s) {
                    const uint64_t ah = tc_desc(sa[b] + s * step_a, lbo_a, 128);
                    const uint64_t al = tc_desc(sa[b] + lo_a + s * step_a, lbo_a, 128);
                    const uint64_t bh = tc_desc(sbh + s * step_b, lbo_b, 128);
                    const uint64_t bl = tc_desc(sbl + s * step_b, lbo_b, 128);
                    tc_mma(d, al, bh, idesc, s > 0 ? 1u : 0u);
                    tc_mma(d, ah, bl, idesc, 1u);
                    tc_mma(d, ah, bh, idesc, 1u);
                }
                tc_commit(smem_u32(&bar_mma[b]));
                issued = m + 1;
                if (m + 2 < mt) {
                    // shared buffer b is free once the MMAs of tile m have read it
                    if (!mbar_wait(smem_u32(&bar_mma[b]), (m >> 1) & 1, &s_abort)) break;
                    load(m + 2);
                }
            }
            if (s_abort) {
                for (int m = consumed; m < loaded; ++m) mbar_drain(smem_u32(&bar_full[m & 1]), (m >> 1) & 1);
                if (issued > 0) mbar_drain(smem_u32(&bar_mma[(issued - 1) & 1]), ((issued - 1) >> 1) & 1);
            }
        }
        __syncwarp();
    } else {
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        for (int m = 0; m < mt; ++m) {
            const int b = m & 1;
            const bool ok = mbar_wait(smem_u32(&bar_mma[b]), (m >> 1) & 1, &s_abort);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc_fence_after();
            const int64_t e = (int64_t)(m0 + m) * kTcRows + quarter * 32 + lane;
            for (int c = half * np; c < (half + 1) * np; c += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + lane_base + (uint32_t)(b * 128 + c), v);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int i = (c >> 1) + j;
                    if (i < tl.count && e < s_tot[i])
                        a.stab[s_off[i] + e] = cplxf{__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1])};
                }
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&bar_empty[b]));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
    }
    if (tid == 0 && s_abort) atomicExch(a.err, 1);
}

// ---------------------------------------------------------------------------------------------
// Double-precision tables on the CUDA cores, over the same groups (one M2 = max order + 2): one CTA
// per run of up to 16 row tiles of up to 32 pairs.  The pairs' zeta_p sit in shared memory; each
// thread takes one row e = (k, a, b), keeps its Gaunt coefficients in registers and sums
// S = sum_q G_q zeta_{a+b-2q} for every second pair of the tile.  The sum runs over q ascending with
// one FMA per term, as the per-pair sum it replaces did, so the tables are bit-identical to it.
template <int QMAX>
__global__ void __launch_bounds__(256) k_pair_s_group(PairArgs a, int tile0) {
    extern __shared__ __align__(16) unsigned char ps_smem[];
    __shared__ int64_t s_off[kPairs64], s_tot[kPairs64];
    const int tid = threadIdx.x;
    const TcTile tl = a.tiles[tile0 + blockIdx.x];
    const int M2 = a.groups[tl.group].M2, P = 2 * M2 - 2, km = M2 - 2;
    cplx* zeta = reinterpret_cast<cplx*>(ps_smem);                              // [kPairs64][P + 1]
    double* scr = reinterpret_cast<double*>(zeta + (size_t)kPairs64 * (P + 1));  // [kPairs64][2 (P + 1)]
    for (int i = tid; i < tl.count; i += 256) {
        const int2 st = a.pairs[tl.first + i];
        const double* cs = a.sc.centres + 3 * (size_t)st.x;
        const double* ct = a.sc.centres + 3 * (size_t)st.y;
        double d0 = a.sc.k * (ct[0] - cs[0]);
        double d1 = a.sc.k * (ct[1] - cs[1]);
        double d2 = a.sc.k * (ct[2] - cs[2]);
        const double rho = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        double* jb = scr + (size_t)2 * (P + 1) * i;
        dev_sph_jn(rho, P, jb);
        if (a.z != 1) dev_sph_yn(rho, P, jb + P + 1);
        s_off[i] = a.pair_off[pair_index(st.x, st.y, a.sc.n)];
        s_tot[i] = pair_block_size(a.sc.p[st.x], a.sc.p[st.y]);
    }
    __syncthreads();
    for (int idx = tid; idx < tl.count * (P + 1); idx += 256) {
        const int i = idx / (P + 1), p = idx - i * (P + 1);
        const double* jb = scr + (size_t)2 * (P + 1) * i;
        zeta[idx] = zeta_of(a.z, p, jb, jb + P + 1);
    }
    __syncthreads();
    const int r = tid & 127, half = tid >> 7;
    for (int m = tl.m0; m < tl.m1; ++m) {
        const int64_t e = (int64_t)m * 128 + r;
        if (e >= s_tot[0]) break;   // the tile's first pair has its largest block
        int k = 0;
        while (k < km && pair_block_offset(k + 1, M2, M2) <= e) ++k;
        const int64_t rr = e - pair_block_offset(k, M2, M2);
        const int cols = M2 - k;
        const int aa = k + (int)(rr / cols), bb = k + (int)(rr % cols);
        const int W = a.g.NM - k + 1;
        const size_t plane = (size_t)W * W;
        const double* gp = a.g.gs + a.g.koff[k] + (size_t)(aa - k) * W + (bb - k);
        const int qm = min(aa, bb), p0 = aa + bb;
        double c[QMAX];
#pragma unroll
        for (int q = 0; q < QMAX; ++q) c[q] = q <= qm ? __ldg(gp + q * plane) : 0.0;
        for (int i = half; i < tl.count; i += 2) {
            if (e >= s_tot[i]) break;   // blocks shrink along the tile
            const cplx* zi = zeta + (size_t)(P + 1) * i + p0;
            double sx = 0.0, sy = 0.0;
#pragma unroll
            for (int q = 0; q < QMAX; ++q) {
                if (q <= qm) {
                    const cplx zz = zi[-2 * q];
                    sx += c[q] * zz.x;
                    sy += c[q] * zz.y;
                }
            }
            a.stab[s_off[i] + e] = cplx{sx, sy};
        }
    }
}

size_t pair_s_group_smem_bytes(int M2) { return (size_t)kPairs64 * (2 * M2 - 1) * 32; }

void launch_pair_s_group(const PairArgs& a, int tile0, int ntiles, int M2, cudaStream_t s) {
    const size_t smem = pair_s_group_smem_bytes(M2);
    if (M2 <= 16) {
        raise_smem_ceiling(reinterpret_cast<const void*>(k_pair_s_group<16>), smem);
        k_pair_s_group<16><<<ntiles, 256, smem, s>>>(a, tile0);
    } else if (M2 <= 32) {
        raise_smem_ceiling(reinterpret_cast<const void*>(k_pair_s_group<32>), smem);
        k_pair_s_group<32><<<ntiles, 256, smem, s>>>(a, tile0);
    } else {
        raise_smem_ceiling(reinterpret_cast<const void*>(k_pair_s_group<48>), smem);
        k_pair_s_group<48><<<ntiles, 256, smem, s>>>(a, tile0);
    }
}

void launch_pair_tc(const TcArgs& a, int tile0, int ntiles, int K, int np, cudaStream_t s) {
    const size_t smem = tc_smem_bytes(K, np);
    raise_smem_ceiling(reinterpret_cast<const void*>(k_pair_tc), smem);
    k_pair_tc<<<ntiles, kTcThreads, smem, s>>>(a, tile0);
}

void launch_tc_pack_a(SGaunt g, const TcGroup& gr, float* out, cudaStream_t s) {
    const int64_t total = (int64_t)gr.mtiles * kTcRows * gr.K;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
    k_tc_pack_a<<<blocks, 256, 0, s>>>(g, gr, out);
}

}  // namespace foggy
