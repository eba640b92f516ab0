// cs_synth_tc.cu -- tensor-core profile synthesis + zero-baseline boxcar gate
// (the mixed-precision form of k_synth_fp32).
//
// The c2r transform of every decimation level is linear in the amplitude
// stack, so all levels come out of ONE product per 128-trial tile:
//   D[trial][col] = sum_k A[trial][k] * B[col][k]
// with A = (Re X_1, Im X_1, Re X_2, ..., Im X_60) in BF16/FP16 and B the
// host-built FP64 twiddles rounded once, one column per profile bin of every
// level followed by that level's first wmax bins again (the wrapped tail of
// the boxcar prefix sums, src/search.jl:571-578).  tcgen05.mma (M=128, K=16
// per instruction, FP32 accumulation in TMEM) computes D; each epilogue thread
// owns one trial's TMEM row.  It first bounds its gate by the largest window
// energy of its bins (a one-width scan of x^2); a warp whose trials all stay
// below the medcut test skips the rest.  Otherwise it streams its bins through
// a register ring of prefix sums to the zero-baseline gate value
// (src/search.jl:743-779).  The gate only selects the trials that take the
// exact FP32 rescan, so the reported S/N never depends on the reduced precision.
//
// Layout: SWIZZLE_NONE K-major canonical UMMA layout -- 8-row x 16-byte core
// matrices.  B (twiddles): K-adjacent core matrices 128 B apart (LBO), 8-row
// groups 2048 B apart (SBO).  A (amplitudes): the other way round, LBO 2048 B
// and SBO 128 B, so that a tile's K chunk is contiguous.  One persistent CTA per SM (it holds all 512 TMEM columns).
#include "cs_internal.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace cs {

namespace {

constexpr int kTM = 128;            // trials per tile (MMA M)
constexpr int kK = 128;             // padded K: 2*nharms <= 128
constexpr int kSBO = (kK / 8) * 128;  // bytes between 8-row groups
constexpr int kABytes = kTM * kK * 2;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo = 128, uint32_t sbo = kSBO) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);                 // start address
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;             // LBO: K-adjacent core matrices
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;             // SBO: 8-row groups
    d |= (uint64_t)1 << 46;                                 // descriptor version (sm_100)
    return d;                                               // base offset 0, SWIZZLE_NONE
}

// A tiles are laid out K-chunk by K-chunk: the 16 core matrices (8 trials x 8
// K values, 128 bytes each) of one K chunk are adjacent (8-row groups 128 B
// apart) and K-adjacent chunks 2 KB apart, so each chunk of a tile -- the
// four harmonics one interpolation CTA computes -- is one contiguous 2 KB run.
constexpr uint32_t kALBO = (kTM / 8) * 128;   // 2048
constexpr uint32_t kASBO = 128;

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float v[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Three-input maximum (sm_100 max.f32 a, b, c): exact, like two fmaxf.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Zero-baseline gate of one level streamed out of TMEM: wrapped prefix sums
// ps[e] over the level's columns (nbins bins, then its first wmax bins again,
// then zero padding to a multiple of HM), ring[e mod HM] holding the prefix at
// each start position (+inf once the start would lie past the profile, so
// windows that would start there -- including every window through the zero
// padding -- never count), and per width w the max of ps[e] - ps[e-w].
// MASK (bit w-1 per width) is a compile-time width set; MASK == 0 reads the
// runtime mask instead.
template <int HM, uint32_t MASK>
struct GateScan {
    float ring[HM];
    float mw[HM];
    float ps;
    uint32_t wm;

    __device__ __forceinline__ void init(uint32_t runtime_mask) {
#pragma unroll
        for (int d = 0; d < HM; ++d) { ring[d] = INFINITY; mw[d] = -INFINITY; }
        ring[0] = 0.0f;
        ps = 0.0f;
        wm = MASK ? MASK : runtime_mask;
    }
    // Two bins at columns e_bin, e_bin+1 (ring slots SLOT, SLOT+1): two
    // sequential prefix adds, each width's maximum taken over both columns by
    // one three-input max.  FAST: both columns lie before the profile's last
    // bin, so the ring takes the prefix sums without a test.
    template <int SLOT, bool FAST>
    __device__ __forceinline__ void step2(float x0, float x1, int e_bin, int nbins) {
        const float ps0 = ps + x0;
        const float ps1 = ps0 + x1;
        const float r0 = FAST ? ps0 : ((e_bin + 1 < nbins) ? ps0 : INFINITY);
        const float r1 = FAST ? ps1 : ((e_bin + 2 < nbins) ? ps1 : INFINITY);
#pragma unroll
        for (int w = 1; w <= HM; ++w) {
            const bool on = MASK ? ((MASK >> (w - 1)) & 1u) : ((wm >> (w - 1)) & 1u);
            if (on) {
                const float d0 = ps0 - ring[(SLOT - w + HM) % HM];
                const float d1 = ps1 - (w == 1 ? r0 : ring[(SLOT + 1 - w + HM) % HM]);
                mw[w - 1] = fmax3(mw[w - 1], d0, d1);
            }
        }
        ring[SLOT % HM] = r0;
        ring[(SLOT + 1) % HM] = r1;
        ps = ps1;
    }
    __device__ __forceinline__ float finish(const float* __restrict__ rsq) const {
        float best = -INFINITY;
#pragma unroll
        for (int w = 1; w <= HM; ++w) {
            const bool on = MASK ? ((MASK >> (w - 1)) & 1u) : ((wm >> (w - 1)) & 1u);
            if (on) best = fmaxf(best, mw[w - 1] * rsq[w - 1]);
        }
        return best;
    }
};

template <int U, int N, bool FAST, class G>
struct Unroll2 {
    __device__ __forceinline__ static void run(G& g, const float* x, int base, int nbins) {
        g.template step2<U + 1, FAST>(x[U], x[U + 1], base + U, nbins);
        Unroll2<U + 2, N, FAST, G>::run(g, x, base, nbins);
    }
};
template <int N, bool FAST, class G>
struct Unroll2<N, N, FAST, G> {
    __device__ __forceinline__ static void run(G&, const float*, int, int) {}
};

// Streams pw columns out of TMEM through the scan g.
// pw (the level's padded column count) is a multiple of HM.
template <class G>
__device__ __forceinline__ void scan_cols(G& g, uint32_t tcol, int nbins, int pw) {
    for (int c0 = 0; c0 < pw; c0 += 32) {
        if (c0 + 32 <= pw) {
            float x[32];
            tmem_ld32(tcol + c0, x);
            if (c0 + 32 < nbins)
                Unroll2<0, 32, true, G>::run(g, x, c0, nbins);
            else
                Unroll2<0, 32, false, G>::run(g, x, c0, nbins);
        } else {
            for (int c1 = c0; c1 < pw; c1 += 8) {   // HM == 8 here: pw is a multiple of 8
                float x[8];
                tmem_ld8(tcol + c1, x);
                Unroll2<0, 8, false, G>::run(g, x, c1, nbins);
            }
        }
    }
}

__host__ __device__ constexpr int top_width(uint32_t m) {
    int w = 0;
    while (m) { ++w; m >>= 1; }
    return w;
}

// Gate value of one unit (its starts [0, nbins), columns [0, pw)).
//
// Window-energy bound: a boxcar of width w <= W (the widest of the level) lies
// inside the width-W window at its start, so by Cauchy-Schwarz
//   S_w(p) / sqrt(w) <= sqrt(sum of x^2 over [p, p+W)) <= sqrt(L),
// L the largest width-W sum of squares over the unit's starts -- a one-width
// scan of x^2, a third of the cost of the full gate scan.  B below adds the
// rounding of both scans (prefix sums of at most 512 columns: an error of at
// most 2^-14 of the sum of |x| in the gate, 2^-14 of the sum of x^2 in L) and
// 2^-16 for the rest, so B >= the gate value the full scan would compute.  When
// B < cut for every valid trial of the warp (cut: the value below which a gate
// can neither be flagged for the rescan nor pushed as a candidate; -inf when
// the exact gate values are wanted), the warp skips the full scan and returns
// -inf, which leaves the flagged set and the candidates unchanged.
// The largest sum of squares over W consecutive columns, streamed like
// GateScan: prefix sums q of x^2 (one fused multiply-add per column) and a ring
// of them.  Every window that ends inside the pw columns counts, also those
// starting past the unit's last start: a larger maximum is still a bound, and
// no column needs a test.
template <int HM, int W>
struct EnergyScan {
    float ring[HM];
    float q;
    float mx;

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int d = 0; d < HM; ++d) ring[d] = INFINITY;   // no window starts before column 0
        ring[0] = 0.0f;
        q = 0.0f;
        mx = -INFINITY;
    }
    template <int SLOT, bool FAST>
    __device__ __forceinline__ void step2(float x0, float x1, int, int) {
        const float q0 = fmaf(x0, x0, q);
        const float q1 = fmaf(x1, x1, q0);
        const float d0 = q0 - ring[(SLOT - W + HM) % HM];
        const float d1 = q1 - (W == 1 ? q0 : ring[(SLOT + 1 - W + HM) % HM]);
        mx = fmax3(mx, d0, d1);
        ring[SLOT % HM] = q0;
        ring[(SLOT + 1) % HM] = q1;
        q = q1;
    }
};

template <int HM, int W>
__device__ __forceinline__ float energy_bound(uint32_t tcol, int nbins, int pw) {
    EnergyScan<HM, W> e;
    e.init();
    scan_cols(e, tcol, nbins, pw);
    return (sqrtf(e.mx + e.q * 0x1p-13f) + 0x1p-13f * sqrtf((float)pw * e.q)) * (1.0f + 0x1p-16f);
}

template <int HM, uint32_t MASK>
__device__ __noinline__ float full_gate(uint32_t tcol, int nbins, int pw, uint32_t wmask,
                                        const float* __restrict__ rsq) {
    GateScan<HM, MASK> g;
    g.init(wmask);
    scan_cols(g, tcol, nbins, pw);
    return g.finish(rsq);
}

template <int HM, uint32_t MASK>
__device__ __noinline__ float gate_level(uint32_t tcol, int nbins, int pw, uint32_t wmask,
                                         const float* __restrict__ rsq, float cut, bool valid) {
    if constexpr (MASK != 0u) {
        if (cut > 0.0f) {   // cut is the level's: warp-uniform
            const float B = energy_bound<HM, top_width(MASK)>(tcol, nbins, pw);
            if (__all_sync(0xffffffffu, !valid || B < cut)) return -INFINITY;
        }
    }
    return full_gate<HM, MASK>(tcol, nbins, pw, wmask, rsq);
}

// Width sets of the decimation ladder and of the plain geometric bank.
constexpr uint32_t kMaskLadderBase = 0x2Fu;   // {1,2,3,4,6}
constexpr uint32_t kMaskLadderDeep = 0x2Eu;   // {2,3,4,6}

template <int HM>
__device__ __forceinline__ float gate_dispatch(uint32_t tcol, int nbins, int pw, uint32_t wmask,
                                               const float* __restrict__ rsq, float cut, bool valid) {
    if (HM == 8) {
        if (wmask == kMaskLadderBase)
            return gate_level<8, kMaskLadderBase>(tcol, nbins, pw, wmask, rsq, cut, valid);
        if (wmask == kMaskLadderDeep)
            return gate_level<8, kMaskLadderDeep>(tcol, nbins, pw, wmask, rsq, cut, valid);
        return gate_level<8, 0u>(tcol, nbins, pw, wmask, rsq, cut, valid);
    }
    if (wmask == 0x4112Fu)   // {1,..,13,19}
        return gate_level<32, 0x4112Fu>(tcol, nbins, pw, wmask, rsq, cut, valid);
    if (wmask == 0x804112Fu)
        return gate_level<32, 0x804112Fu>(tcol, nbins, pw, wmask, rsq, cut, valid);
    return gate_level<32, 0u>(tcol, nbins, pw, wmask, rsq, cut, valid);
}

}  // namespace

constexpr int kEpiThreads = 512;   // 4 warpgroups share the epilogue

// Named barriers of 256 threads (two warpgroups), for the split epilogue
// (t.dbuf == 2): id 1 for warpgroups 0-1, id 2 for warpgroups 2-3 (id 0 is
// __syncthreads).  The reductions return the same value to every thread.
__device__ __forceinline__ void group_sync(int id) {
    asm volatile("barrier.cta.sync %0, 256;" ::"r"(id) : "memory");
}
__device__ __forceinline__ bool group_and(bool v, int id) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "barrier.cta.red.and.pred p, %2, 256, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ bool group_or(bool v, int id) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "barrier.cta.red.or.pred p, %2, 256, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}

// One persistent CTA per SM walks the tiles blockIdx.x, +gridDim.x, ...
// Thread 0 issues each tile's product (one commit per tile) as soon as its A
// tile has landed and the TMEM columns it writes are free: with two base-level
// slots that is right after the decimated levels of the current tile have been
// scanned, so the next product runs under the base level's scan and the
// medcut pass.  A tiles are double-buffered in shared memory (one buffer for
// split tiles), each refilled as soon as the product that read it completed.
template <int HM>
__global__ void __launch_bounds__(kEpiThreads, 1) k_synth_tc(WaveArgs a, TcArgs t, const uint4* __restrict__ Bg,
                                                      int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int abytes = kABytes * t.split;     // one tile's A bytes (hi, then lo when split)
    const int nbuf = t.split == 2 ? 1 : 2;
    uint8_t* As0 = smem;                      // nbuf A buffers, abytes each
    uint8_t* Bs = smem + nbuf * abytes;       // ncols_total * kK * 2
    __shared__ uint64_t mbar;                 // product completion, one phase per tile
    __shared__ uint64_t lbar[2];              // A-tile arrival, one per buffer
    __shared__ uint32_t tmem_base_sh;
    __shared__ int mma_ok_sh;                 // 0 once a product could not be issued
    __shared__ TcLevel lev_sh[kMaxLevels];
    __shared__ TcUnit unit_sh[kMaxUnits];
    __shared__ TcMma mma_sh[kMaxMma];
    __shared__ float part_sh[kMaxUnits][kTM];   // per-unit gate partials of the tile
    __shared__ uint8_t lu_start[kMaxLevels + 1], lu_idx[kMaxUnits];
    __shared__ float inv_sh[kMaxLevels];        // 1/sigma of the tile's block, per level
    __shared__ int nv_sh[kMaxLevels];           // valid trials of the tile's block, per level
    __shared__ float cut_sh[kMaxLevels];        // gate bound for skipping a warp's scan, per level
    __shared__ float gup_sh;                    // 2^s: undoes the tile's block's FP16 scale
    __shared__ float gup_chunk_sh[kMaxSpecChunks];   // 2^s of a block whose last spectrum chunk is c
    // split epilogue (t.dbuf == 2): base-level products per slot, A buffers
    // released by both groups, and the counts the final drain waits for
    __shared__ uint64_t mbar_b2[2];             // base-level product of the slot's tiles
    __shared__ int afree_sh[2];                 // arrivals of the two groups at an A buffer
    __shared__ int nload_sh[2];                 // A loads issued into each buffer
    __shared__ int ncommit_sh[3];               // products committed: decimated, base slot 0, base slot 1
    __shared__ uint8_t grp_lev[2][kMaxLevels];  // each group's levels (group 0: warpgroups 0-1)
    __shared__ int grp_nlev[2];
    __shared__ int grp_ok_sh[2];                // 0 once a group's product could not be issued
    __shared__ float gup2_sh[2];                // each group's tile scale 2^s

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int tiles_per_blk = a.tiles_per_blk;
    const int ntiles = a.nblk * tiles_per_blk;
    const int my_ntiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    // B once per CTA.
    const int bwords = t.ncols_total * kK * 2 / 16;
    for (int i = tid; i < bwords; i += blockDim.x) reinterpret_cast<uint4*>(Bs)[i] = Bg[i];
    if (tid < t.nlev) lev_sh[tid] = t.lev[tid];
    if (tid < t.nunit) unit_sh[tid] = t.unit[tid];
    if (tid < t.nmma) mma_sh[tid] = t.mma[tid];
    // the chunk maxima are the search's constants: each chunk index's scale,
    // once per CTA, so that a tile needs only its block's chunk index
    if (tid >= 32 && tid < 32 + kMaxSpecChunks)
        gup_chunk_sh[tid - 32] = a.fp16 ? pow2f(ascale_exp(a.amax_bits, tid - 32)) : 1.0f;
    if (tid == 0) {
        // each level's units, listed contiguously, for the per-level gate maximum
        int c = 0;
        for (int l = 0; l < t.nlev; ++l) {
            lu_start[l] = (uint8_t)c;
            for (int u = 0; u < t.nunit; ++u)
                if (t.unit[u].lev == l) lu_idx[c++] = (uint8_t)u;
        }
        lu_start[t.nlev] = (uint8_t)c;
        mma_ok_sh = 1;
        mbar_init(&mbar, 1);
        mbar_init(&lbar[0], 1);
        mbar_init(&lbar[1], 1);
        mbar_init(&mbar_b2[0], 1);
        mbar_init(&mbar_b2[1], 1);
        afree_sh[0] = afree_sh[1] = 0;
        nload_sh[0] = nload_sh[1] = 0;
        ncommit_sh[0] = ncommit_sh[1] = ncommit_sh[2] = 0;
        // the split epilogue's level lists: a level belongs to the group of its units
        grp_nlev[0] = grp_nlev[1] = 0;
        for (int l = 0; l < t.nlev; ++l) {
            int g = 1;
            for (int u = 0; u < t.nunit; ++u)
                if (t.unit[u].lev == l && t.unit[u].phase == 1) g = 0;
            if (l == 0) g = 0;
            grp_lev[g][grp_nlev[g]++] = (uint8_t)l;
        }
        grp_ok_sh[0] = grp_ok_sh[1] = 1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_sh)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    const uint32_t idesc_base = (1u << 4) | ((uint32_t)(t.fp16 ? 0 : 1) << 7) |
                                ((uint32_t)(t.fp16 ? 0 : 1) << 10) | ((uint32_t)(kTM >> 4) << 24);
    const uint32_t b_addr = smem_u32(Bs);

    // Thread 0's bookkeeping: loads issued per A buffer, products issued.
    int nload[2] = {0, 0};
    int nmma_issued = 0;
    // Local tile it sits in A buffer it % nbuf; the n-th load into a buffer
    // completes that buffer's barrier phase n.
    auto a_buf = [&](int it) { return nbuf == 2 ? (it & 1) : 0; };
    auto load_a = [&](int it) {
        const int b = a_buf(it);
        bulk_load(smem_u32(As0 + b * abytes), a.Atile + (int64_t)((int)blockIdx.x + it * (int)gridDim.x) * abytes,
                  abytes, &lbar[b]);
        ++nload[b];
    };
    // Product of local tile it: wait for its A tile, then every column range
    // into TMEM (the base level into the slot of the tile's parity), one commit.
    auto issue_mma = [&](int it) -> bool {
        const int b = a_buf(it);
        const uint32_t par = (uint32_t)((nbuf == 2 ? (it >> 1) : it) & 1);
        if (!mbar_wait(&lbar[b], par)) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_addr = smem_u32(As0 + b * abytes);
        for (int q = 0; q < t.nmma; ++q) {
            const TcMma M = mma_sh[q];
            const uint32_t idesc = idesc_base | ((uint32_t)(M.n >> 3) << 17);
            const uint32_t dcol = (uint32_t)((it & 1) ? M.tcol1 : M.tcol);
            // split: the hi tile's K steps, then the lo tile's against the
            // same twiddles, into one FP32 accumulator
            for (int kk = 0; kk < t.split * (kK / 16); ++kk) {
                const int sp = kk / (kK / 16), ks = kk - sp * (kK / 16);
                const uint64_t da = umma_desc(a_addr + sp * kABytes + ks * 2 * kALBO, kALBO, kASBO);
                const uint64_t db = umma_desc(b_addr + (M.bcol / 8) * kSBO + ks * 256);
                const uint32_t acc = kk > 0;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem + dcol), "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(smem_u32(&mbar)) : "memory");
        ++nmma_issued;
        return true;
    };

    bool ok = true;
    if (t.dbuf != 2 && tid == 0 && my_ntiles > 0) {
        load_a(0);
        if (nbuf == 2 && my_ntiles > 1) load_a(1);
        if (!issue_mma(0)) mma_ok_sh = 0;
    }
    // The per-level sigma and valid counts of the first tile's block; each
    // iteration then loads the next tile's while its own epilogue runs.
    // (the split epilogue: thread 0 keeps the base level's, threads 256+l the
    // decimated level l's)
    int plev = tid < t.nlev ? tid : -1;
    if (t.dbuf == 2) {
        // the split epilogue: warpgroups 0-1's levels to threads l, 2-3's to 256+l
        plev = -1;
        const int g = tid < 256 ? 0 : 1;
        for (int i = 0; i < grp_nlev[g]; ++i)
            if (grp_lev[g][i] == (tid & 255)) plev = tid & 255;
    }
    float sig_next = 0.0f;
    int nv_next = 0, cidx_next = kMaxSpecChunks - 1;   // the block's last spectrum chunk: its FP16 scale
    if (plev >= 0 && my_ntiles > 0) {
        const int b0 = (int)blockIdx.x / tiles_per_blk;
        sig_next = a.sigma[b0 * a.nlev + plev];
        nv_next = a.nvalid[b0 * a.nlev + plev];
        if (a.blk_cidx) cidx_next = a.blk_cidx[b0];
    }
    ok = __syncthreads_and(mma_ok_sh != 0) != 0;
    if (!ok && tid == 0) atomicExch(err, 2);

    const int wg = warp >> 2;
    const int row = (warp & 3) * 32 + (tid & 31);
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);

    if (t.dbuf == 2) {
        // Split epilogue.  Warpgroups 0-1 (group A, named barrier 1) scan the
        // base level from the slot of the tile's parity; warpgroups 2-3
        // (group B, barrier 2) scan the decimated levels.  Each group's first
        // thread issues its own products: A the base level of tile it+2 into
        // the slot it just read, B the decimated levels of tile it+1, so
        // neither group waits for the other's scan.  Tile it's A buffer is
        // refilled with tile it+2 by whichever group is done with it second.
        const bool grpA = tid < 256;
        const int gid = grpA ? 0 : 1;
        const int bar_id = grpA ? 1 : 2;
        const int gtid = tid & 255;
        auto load2 = [&](int it) {
            const int b = it & 1;
            bulk_load(smem_u32(As0 + b * abytes),
                      a.Atile + (int64_t)((int)blockIdx.x + it * (int)gridDim.x) * abytes, abytes, &lbar[b]);
            atomicAdd(&nload_sh[b], 1);
        };
        // This group's products of tile it (its A tile waited for, bounded):
        // warpgroups 0-1 the base level's ranges (phase 1) into the slot of
        // the tile's parity, 2-3 the decimated levels' (phase 0).
        auto issue2 = [&](int it) -> bool {
            const int b = it & 1;
            if (!mbar_wait(&lbar[b], (uint32_t)((it >> 1) & 1))) return false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_addr = smem_u32(As0 + b * abytes);
            for (int q = 0; q < t.nmma; ++q) {
                const TcMma M = mma_sh[q];
                if ((M.phase == 1) != grpA) continue;
                const uint32_t idesc = idesc_base | ((uint32_t)(M.n >> 3) << 17);
                const uint32_t dcol = (uint32_t)((it & 1) ? M.tcol1 : M.tcol);
                for (int ks = 0; ks < kK / 16; ++ks) {
                    const uint64_t da = umma_desc(a_addr + ks * 2 * kALBO, kALBO, kASBO);
                    const uint64_t db = umma_desc(b_addr + (M.bcol / 8) * kSBO + ks * 256);
                    const uint32_t acc = ks > 0;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(tmem + dcol), "l"(da), "l"(db), "r"(idesc), "r"(acc));
                }
            }
            uint64_t* done = grpA ? &mbar_b2[it & 1] : &mbar;
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(done)) : "memory");
            atomicAdd(&ncommit_sh[grpA ? 1 + (it & 1) : 0], 1);
            return true;
        };
        if (gtid == 0 && my_ntiles > 0 && ok) {
            bool good = true;
            if (grpA) {
                load2(0);
                if (my_ntiles > 1) load2(1);
                good = issue2(0) && (my_ntiles < 2 || issue2(1));
            } else {
                good = issue2(0);
            }
            if (!good) grp_ok_sh[gid] = 0;
        }
        ok = group_and(ok, bar_id);
        for (int it = 0; it < my_ntiles && ok; ++it) {
            const int tile = (int)blockIdx.x + it * (int)gridDim.x;
            const int blk = tile / tiles_per_blk;
            const int j0 = (tile % tiles_per_blk) * kTM;
            if (plev >= 0) {
                // this group's level(s): 1/sigma times the tile scale, valid count, skip bound
                const float gup = gup_chunk_sh[cidx_next];
                gup2_sh[gid] = gup;   // (every owner of the group writes the same value)
                const float inv = inv_sigma(sig_next) * gup;
                inv_sh[plev] = inv;
                nv_sh[plev] = nv_next;
                float cut = -INFINITY;
                const float c = fminf(a.medcut_gate, a.threshold);
                if (!a.Q0 && inv > 0.0f && c > 0.0f) cut = (c / inv) * (1.0f - 0x1p-16f);
                cut_sh[plev] = cut;
                if (it + 1 < my_ntiles) {
                    const int bn = (tile + (int)gridDim.x) / tiles_per_blk;
                    sig_next = a.sigma[bn * a.nlev + plev];
                    nv_next = a.nvalid[bn * a.nlev + plev];
                    if (a.blk_cidx) cidx_next = a.blk_cidx[bn];
                }
            }
            // this tile's product for the group has landed (bounded)
            const bool landed = grpA ? mbar_wait(&mbar_b2[it & 1], (uint32_t)((it >> 1) & 1))
                                     : mbar_wait(&mbar, (uint32_t)(it & 1));
            ok = group_and(landed && grp_ok_sh[gid] != 0, bar_id);
            if (!ok) {
                if (gtid == 0) atomicExch(err, 2);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // both groups' products of tile it are done with its A buffer
            if (gtid == 0 && it + 2 < my_ntiles) {
                __threadfence_block();
                if (atomicAdd(&afree_sh[it & 1], 1) & 1) {
                    __threadfence_block();
                    load2(it + 2);
                }
            }
            const int par = it & 1;
            bool need = false;
            for (int u = 0; u < t.nunit; ++u) {
                const TcUnit& U = unit_sh[u];
                if (U.phase != (grpA ? 1 : 0) || U.wg != wg) continue;           // warp-uniform
                if (j0 >= nv_sh[U.lev]) continue;                                // warp-uniform
                const TcLevel& L = lev_sh[U.lev];
                const float cut = cut_sh[U.lev];
                const uint32_t col = (uint32_t)(par ? U.col1 : U.col);
                const float v = gate_dispatch<HM>(lane_base + col, U.nstart, U.pw, L.wmask, L.rsq, cut,
                                                  j0 + row < nv_sh[U.lev]);
                part_sh[u][row] = v;
                need |= !(cut > 0.0f) || v != -INFINITY;
            }
            // the group's columns are read: its next product may land in them
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            need = group_or(need, bar_id);
            if (gtid == 0) {
                // the base level two tiles on into the slot just read; the
                // decimated levels of the next tile into their one slot
                const int nxt = grpA ? it + 2 : it + 1;
                if (nxt < my_ntiles && !issue2(nxt)) grp_ok_sh[gid] = 0;
            }
            if (need) {
                // gate = max over the level's units, then the medcut test
                const int nl = grp_nlev[gid];
                for (int idx = gtid; idx < nl * kTM; idx += 256) {
                    const int l = grp_lev[gid][idx / kTM], r = idx % kTM;
                    const int j = j0 + r;
                    if (j >= nv_sh[l]) continue;
                    float g = -INFINITY;
                    for (int i = lu_start[l]; i < lu_start[l + 1]; ++i) g = fmaxf(g, part_sh[lu_idx[i]][r]);
                    if (a.Q0) a.Q0[((int64_t)blk * a.nlev + l) * a.Nprof + j] = g * gup2_sh[gid];
                    gate_flag(a, blk, l, j, g, inv_sh[l]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            ok = group_and(grp_ok_sh[gid] != 0, bar_id);
            if (!ok && gtid == 0) atomicExch(err, 2);
        }
    } else
    for (int it = 0; it < my_ntiles && ok; ++it) {
        const int tile = (int)blockIdx.x + it * (int)gridDim.x;
        const int blk = tile / tiles_per_blk;
        const int j0 = (tile % tiles_per_blk) * kTM;
        // the block's per-level sigma and valid counts, for the epilogue
        // (the previous tile's epilogue finished at the last barrier)
        if (tid < t.nlev) {
            // 1/sigma times the A tiles' scale 2^s (exact): the gate in true units
            const float gup = gup_chunk_sh[cidx_next];
            if (tid == 0) gup_sh = gup;
            const float inv = inv_sigma(sig_next) * gup;
            inv_sh[tid] = inv;
            nv_sh[tid] = nv_next;
            // a gate g (TMEM units) with g < cut has g*inv below both medcut_gate
            // and the threshold, so gate_flag would neither flag nor push it
            float cut = -INFINITY;
            const float c = fminf(a.medcut_gate, a.threshold);
            if (!a.Q0 && inv > 0.0f && c > 0.0f) cut = (c / inv) * (1.0f - 0x1p-16f);
            cut_sh[tid] = cut;
            if (it + 1 < my_ntiles) {
                const int bn = (tile + (int)gridDim.x) / tiles_per_blk;
                sig_next = a.sigma[bn * a.nlev + tid];
                nv_next = a.nvalid[bn * a.nlev + tid];
                if (a.blk_cidx) cidx_next = a.blk_cidx[bn];
            }
        }
        // this tile's product has completed: its accumulators are readable and
        // its A buffer may be refilled
        ok = __syncthreads_and(mbar_wait(&mbar, (uint32_t)(it & 1))) != 0;
        if (!ok) {
            if (tid == 0) atomicExch(err, 2);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            if (nbuf == 2 && it + 2 < my_ntiles) load_a(it + 2);
            if (nbuf == 1 && it + 1 < my_ntiles) load_a(it + 1);
        }
        const int par = it & 1;
        // Epilogue: warpgroup wg scans its units of a phase; the thread owns TMEM
        // row (warp%4)*32 + lane.  need: a gate of the tile may be flagged or
        // pushed.  A -inf gate whose level could skip (cut > 0, so 1/sigma > 0)
        // is neither, so a tile whose every unit returned -inf there needs no
        // medcut pass.
        auto scan_units = [&](int ph) -> bool {
            bool nd = false;
            for (int u = 0; u < t.nunit; ++u) {
                const TcUnit& U = unit_sh[u];
                if (U.wg != wg || U.phase != ph) continue;              // warp-uniform
                if (j0 >= nv_sh[U.lev]) continue;                       // warp-uniform
                const TcLevel& L = lev_sh[U.lev];
                const float cut = cut_sh[U.lev];
                const uint32_t col = (uint32_t)(par ? U.col1 : U.col);
                const float v = gate_dispatch<HM>(lane_base + col, U.nstart, U.pw, L.wmask, L.rsq, cut,
                                                  j0 + row < nv_sh[U.lev]);
                part_sh[u][row] = v;
                nd |= !(cut > 0.0f) || v != -INFINITY;
            }
            return nd;
        };
        bool need = scan_units(0);
        // The columns phase 0 read are free: the next tile's product may land
        // in them (and in the other base-level slot) while phase 1 and the
        // medcut pass run.
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0 && it + 1 < my_ntiles && !issue_mma(it + 1)) mma_ok_sh = 0;
        if (t.dbuf) need |= scan_units(1);
        // gate = max over the level's units, then the medcut test
        if (__syncthreads_or(need)) for (int idx = tid; idx < t.nlev * kTM; idx += blockDim.x) {
            const int l = idx / kTM, r = idx % kTM;
            const int j = j0 + r;
            if (j >= nv_sh[l]) continue;
            float g = -INFINITY;
            for (int i = lu_start[l]; i < lu_start[l + 1]; ++i) g = fmaxf(g, part_sh[lu_idx[i]][r]);
            if (a.Q0) a.Q0[((int64_t)blk * a.nlev + l) * a.Nprof + j] = g * gup_sh;
            gate_flag(a, blk, l, j, g, inv_sh[l]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        ok = __syncthreads_and(mma_ok_sh != 0) != 0;
        if (!ok && tid == 0) atomicExch(err, 2);
    }
    if (t.dbuf == 2) __syncthreads();   // both groups are out of their loops: the counts are final
    if (tid == 0) {
        // bounded: let every product and A-tile copy this CTA issued land
        // before its TMEM and shared memory go away (all have on the normal path)
        if (t.dbuf == 2) {
            if (ncommit_sh[0] > 0) mbar_wait(&mbar, (uint32_t)((ncommit_sh[0] - 1) & 1));
            for (int sl = 0; sl < 2; ++sl)
                if (ncommit_sh[1 + sl] > 0) mbar_wait(&mbar_b2[sl], (uint32_t)((ncommit_sh[1 + sl] - 1) & 1));
            for (int b = 0; b < 2; ++b)
                if (nload_sh[b] > 0) mbar_wait(&lbar[b], (uint32_t)((nload_sh[b] - 1) & 1));
        } else {
            if (nmma_issued > 0) mbar_wait(&mbar, (uint32_t)((nmma_issued - 1) & 1));
            for (int b = 0; b < 2; ++b)
                if (nload[b] > 0) mbar_wait(&lbar[b], (uint32_t)((nload[b] - 1) & 1));
        }
    }
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

// ---------------------------------------------------------------------------
// Host side: the twiddle matrix, the level layout and the launch.
// ---------------------------------------------------------------------------

static uint16_t to_half_bits(float v, int fp16) {
    if (fp16) {
        __half h = __float2half_rn(v);
        return *reinterpret_cast<uint16_t*>(&h);
    }
    __nv_bfloat16 b = __float2bfloat16_rn(v);
    return *reinterpret_cast<uint16_t*>(&b);
}

int prepare_tc(const DevLevel* dl, int nlev, int nharms, int fp16, int split, TcPlanHost* out, int div0, int div1,
               int allow_dbuf) {
    if (2 * nharms > kK || nlev < 1) return -1;
    TcArgs& t = out->args;
    t = TcArgs{};
    t.nlev = nlev;
    t.fp16 = fp16;
    t.split = split;
    int wmax = 0;
    for (int l = 0; l < nlev; ++l) wmax = wmax > dl[l].wmax ? wmax : dl[l].wmax;
    t.hm = wmax <= 8 ? 8 : (wmax <= 32 ? 32 : 0);
    if (!t.hm) return -2;
    auto pad16 = [](int x) { return (x + 15) / 16 * 16; };
    auto pad32 = [](int x) { return (x + 31) / 32 * 32; };
    // Each level's columns: its bins followed by its first wmax bins.  The
    // decimated levels lie one after another (offsets relative to the first);
    // the base level's B columns come first, their count fixed below.
    int rcol = 0;
    for (int l = 0; l < nlev; ++l) {
        TcLevel& L = t.lev[l];
        L.nbins = dl[l].nbins;
        L.ncol = dl[l].nbins + dl[l].wmax;
        L.pw = (L.ncol + t.hm - 1) / t.hm * t.hm;
        L.col = l == 0 ? 0 : rcol;
        if (l > 0) rcol += L.pw;
        L.wmask = 0;
        for (int i = 0; i < 32; ++i) L.rsq[i] = 0.0f;
        for (int i = 0; i < dl[l].nw; ++i) {
            const int w = dl[l].widths[i];
            L.wmask |= 1u << (w - 1);
            L.rsq[w - 1] = dl[l].rsqrtw[i];
        }
    }
    const int g1 = pad16(rcol);          // decimated levels
    if (g1 + pad16(t.lev[0].pw) > 512) return -3;
    int try_dbuf = 1;
    int mode = 0;
    auto phase_of = [&](int l) { return (try_dbuf && l == 0) ? 1 : 0; };
    struct UC { int lev, p0, nst; double c; };
    auto seg_cost = [&](int l, int nst) { return (double)(nst + dl[l].wmax) * (1 + 2 * dl[l].nw); };
    // The units of one phase for a segment target of (phase cost / div), and
    // their longest-processing-time placement on the 4 warpgroups.
    // (mode 2: the base level's units on warpgroups 0-1, the decimated levels'
    // on 2-3, the two groups scanning side by side)
    auto build_phase = [&](int ph, int div, UC* uc, int* wg_of, double* maxload) -> int {
        const int wg0 = mode == 2 ? (ph == 1 ? 0 : 2) : 0, nwg = mode == 2 ? 2 : 4;
        double ph_cost = 0.0;
        for (int l = 0; l < nlev; ++l)
            if (phase_of(l) == ph) ph_cost += seg_cost(l, dl[l].nbins);
        int nu = 0;
        for (int l = 0; l < nlev; ++l) {
            if (phase_of(l) != ph) continue;
            int nseg = (int)(seg_cost(l, dl[l].nbins) / (ph_cost / div) + 0.5);
            nseg = nseg < 1 ? 1 : nseg;
            while (nseg > 1 && dl[l].nbins / nseg < 8) --nseg;
            if (nu + nseg > kMaxUnits) return -1;
            for (int sgi = 0; sgi < nseg; ++sgi) {
                // segment boundaries on multiples of 8 columns
                const int p0 = (int)(((int64_t)dl[l].nbins * sgi / nseg) / 8 * 8);
                const int p1 =
                    sgi + 1 == nseg ? dl[l].nbins : (int)(((int64_t)dl[l].nbins * (sgi + 1) / nseg) / 8 * 8);
                uc[nu++] = {l, p0, p1 - p0, seg_cost(l, p1 - p0)};
            }
        }
        double load[4] = {0.0, 0.0, 0.0, 0.0};
        bool used[kMaxUnits] = {false};
        for (int k = 0; k < nu; ++k) {
            int best = -1;
            for (int i = 0; i < nu; ++i)
                if (!used[i] && (best < 0 || uc[i].c > uc[best].c)) best = i;
            used[best] = true;
            int g = wg0;
            for (int q = wg0 + 1; q < wg0 + nwg; ++q) if (load[q] < load[g]) g = q;
            load[g] += uc[best].c;
            wg_of[best] = g;
        }
        *maxload = std::max(std::max(load[0], load[1]), std::max(load[2], load[3]));
        return nu;
    };
    // Epilogue units: each level's boxcar starts split into segments (every
    // segment re-reads wmax columns), then placed on the 4 warpgroups.  With
    // two base-level slots the decimated levels are scanned first (phase 0)
    // and the base level second (phase 1), while the next tile's product
    // lands in the other slot and in the freed decimated columns.  Per phase,
    // the segment size that gives the lightest heaviest warpgroup wins.  A
    // slot spans every column its units read (each unit reads a multiple of
    // the ring size from its first start), so that no scan reaches into the
    // other slot, which the next tile's product may be writing.
    UC all_uc[kMaxUnits];
    int all_wg[kMaxUnits], all_ph[kMaxUnits];
    int nall = 0;
    int slot_w = t.lev[0].pw;
    for (mode = allow_dbuf >= 2 && split == 1 && nlev >= 2 ? 2 : (allow_dbuf ? 1 : 0); mode >= 0; --mode) {
        try_dbuf = mode > 0 ? 1 : 0;
        nall = 0;
        bool okp = true;
        for (int ph = 0; ph < 2 && okp; ++ph) {
            UC best_uc[kMaxUnits], uc[kMaxUnits];
            int best_wg[kMaxUnits], wg_of[kMaxUnits];
            int best_nu = 0;
            double best_load = 0.0;
            for (int div : {2, 3, 4, 5, 6, 8, 10, 12, 16}) {
                const int forced = ph ? div1 : div0;   // a tuned divisor replaces the search
                if (forced > 0 && div != forced) continue;
                double ml = 0.0;
                const int nu = build_phase(ph, div, uc, wg_of, &ml);
                if (nu < 0 || nall + nu > kMaxUnits) continue;
                if (best_nu == 0 || ml < best_load) {
                    best_nu = nu;
                    best_load = ml;
                    std::copy(uc, uc + nu, best_uc);
                    std::copy(wg_of, wg_of + nu, best_wg);
                }
            }
            bool any = false;
            for (int l = 0; l < nlev; ++l) any |= phase_of(l) == ph;
            if (any && best_nu == 0) okp = false;
            for (int i = 0; i < best_nu; ++i) {
                all_uc[nall] = best_uc[i];
                all_wg[nall] = best_wg[i];
                all_ph[nall++] = ph;
            }
        }
        if (!okp) continue;
        slot_w = t.lev[0].pw;
        for (int i = 0; i < nall; ++i)
            if (all_uc[i].lev == 0) {
                const int upw = (all_uc[i].nst + dl[0].wmax + t.hm - 1) / t.hm * t.hm;
                slot_w = std::max(slot_w, all_uc[i].p0 + upw);
            }
        slot_w = pad16(slot_w);
        if (!try_dbuf || pad32(g1) + pad32(slot_w) + slot_w <= 512) break;
    }
    if (mode < 0) return -4;
    t.dbuf = mode;
    // B columns: the base level's slot width (its bins, its wrapped tail and
    // zero columns up to the reach of its scans, so that every column a scan
    // reads is written by the product), then the decimated levels.
    const int g0 = slot_w;
    const int total = g0 + g1;
    if (total > 512) return -3;
    for (int l = 1; l < nlev; ++l) t.lev[l].col += g0;
    // TMEM: the decimated levels at [0, g1), then the base level's slot for
    // even tiles and, with two slots, the one for odd tiles (32-column aligned).
    const int slot0 = t.dbuf ? pad32(g1) : g1, slot1 = t.dbuf ? slot0 + pad32(slot_w) : slot0;
    if (slot0 + slot_w > 512) return -3;
    auto tcol_of = [&](int l, int odd) { return l == 0 ? (odd ? slot1 : slot0) : t.lev[l].col - g0; };
    t.nmma = 0;
    for (int c = 0; c < g0; c += 256) {
        const int n = g0 - c < 256 ? g0 - c : 256;
        t.mma[t.nmma++] = {(int16_t)c, (int16_t)n, (int16_t)(slot0 + c), (int16_t)(slot1 + c), 1, 0};
    }
    // the decimated levels (issued by warpgroups 2-3 in the split epilogue)
    for (int c = 0; c < g1; c += 256) {
        const int n = g1 - c < 256 ? g1 - c : 256;
        if (t.nmma >= kMaxMma) return -4;
        t.mma[t.nmma++] = {(int16_t)(g0 + c), (int16_t)n, (int16_t)c, (int16_t)c, 0, 0};
    }
    t.nunit = nall;
    for (int l = 0; l < nlev; ++l) t.lev[l].nunits = 0;
    for (int i = 0; i < nall; ++i) {
        TcUnit& U = t.unit[i];
        const int l = all_uc[i].lev;
        t.lev[l].nunits += 1;
        U.lev = (int16_t)l;
        U.wg = (int16_t)all_wg[i];
        U.nstart = (int16_t)all_uc[i].nst;
        U.pw = (int16_t)((all_uc[i].nst + dl[l].wmax + t.hm - 1) / t.hm * t.hm);
        U.col = (int16_t)(tcol_of(l, 0) + all_uc[i].p0);
        U.col1 = (int16_t)(tcol_of(l, 1) + all_uc[i].p0);
        U.phase = (int16_t)all_ph[i];
        U.pad = 0;
        if (U.col + U.pw > 512 || U.col1 + U.pw > 512) return -3;
    }
    t.ncols_total = total;
    out->B.assign((size_t)total * kK, 0);
    for (int l = 0; l < nlev; ++l) {
        const DevLevel& d = dl[l];
        const TcLevel& L = t.lev[l];
        for (int c = 0; c < L.ncol; ++c) {
            const int nbin = c % d.nbins;
            const int n = L.col + c;
            for (int jh = 1; jh <= d.Hk; ++jh) {
                const int h = jh * d.k;          // base harmonic
                double cre, cim;
                if (jh < d.Hk) {
                    const double ang = 2.0 * M_PI * (double)(((int64_t)jh * nbin) % d.nbins) / (double)d.nbins;
                    cre = 2.0 * std::cos(ang);
                    cim = -2.0 * std::sin(ang);
                } else {
                    cre = (nbin & 1) ? -1.0 : 1.0;   // Nyquist term: real part only
                    cim = 0.0;
                }
                for (int part = 0; part < 2; ++part) {
                    const int k = 2 * (h - 1) + part;
                    const size_t off = ((size_t)(n >> 3) * kSBO + (size_t)(k >> 3) * 128 + (n & 7) * 16 +
                                        (k & 7) * 2) / 2;
                    out->B[off] = to_half_bits((float)(part ? cim : cre), fp16);
                }
            }
        }
    }
    out->smem = (size_t)(split == 2 ? 1 : 2) * kABytes * split + (size_t)total * kK * 2;
    return 0;
}

cudaError_t launch_synth_tc(const WaveArgs& a, const TcPlanHost& tp, const void* dB, int* err, cudaStream_t st,
                            int num_sms) {
    const int tiles = a.nblk * ((a.Nprof + kTM - 1) / kTM);
    const int grid = tiles < num_sms ? tiles : num_sms;
    if (tp.args.hm == 8) {
        cudaFuncSetAttribute(k_synth_tc<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tp.smem);
        k_synth_tc<8><<<grid, kEpiThreads, tp.smem, st>>>(a, tp.args, static_cast<const uint4*>(dB), err);
    } else {
        cudaFuncSetAttribute(k_synth_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tp.smem);
        k_synth_tc<32><<<grid, kEpiThreads, tp.smem, st>>>(a, tp.args, static_cast<const uint4*>(dB), err);
    }
    return cudaGetLastError();
}

}  // namespace cs
