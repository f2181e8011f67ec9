// tgb_gemm.cu -- Blackwell (sm_100a) GEMM for the GAP sparse-set kernel.
//
// A persistent CTA per SM walks 128 x 256 tiles of C = A . B^T:
//   warp 0  : TMA producer (one lane) feeding a shared-memory operand ring of
//             3 stages (modes whose epilogue stages bf16 or fp32 outputs for TMA
//             stores) or 4 stages (the plain fp32 store),
//   warp 1  : allocates 512 TMEM columns (two 256-column accumulators, so one
//             tile's epilogue overlaps the next tile's MMAs); one lane issues
//             tcgen05.mma (M=128, N=256, K=16, bf16 -> fp32) and tcgen05.commit,
//   warps 2.. : epilogue, kGemmEpiGroups (GAP, plain store: 8 warps) or
//             kGemmMlpEpiGroups (MLP modes: 16 warps) warps per TMEM lane
//             quarter; warp w reads TMEM lanes 32*(w%4) .. +31 and its column
//             group of the tile with tcgen05.ld, then runs the fused epilogue.
// Operand tiles are [rows x 64] bf16 with the 128-byte swizzle, which is the
// canonical K-major layout of the UMMA shared-memory descriptor.
// Every mbarrier wait is bounded by wall time; on expiry the waiting role sets
// an error bit, stops issuing and lets the CTA drain and free its TMEM.

#include "tgb_gemm.cuh"

#include <cudaTypedefs.h>

namespace tgb {

namespace {

constexpr uint64_t kWaitLimitNs = 2000000000ull;   // 2 s per wait

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr unsigned kTimeoutBits = DEV_ERR_TIMEOUT_TMA | DEV_ERR_TIMEOUT_MMA | DEV_ERR_TIMEOUT_EPI;

// Bounded wait: true when the phase with the given parity completed. Gives up
// after kWaitLimitNs, or at once when another CTA has already timed out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const unsigned *err) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 0) {
            if (*reinterpret_cast<const volatile unsigned *>(err) & kTimeoutBits) return false;
            if (global_ns() - t0 > kWaitLimitNs) return false;
        }
    }
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// UMMA shared-memory descriptor, K-major, 128-byte swizzle: start address>>4,
// leading byte offset 1 (unused for swizzled K-major), stride byte offset
// 1024 B (8 rows x 128 B) >> 4, descriptor version 1, layout SWIZZLE_128B (2).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: fp32 accumulator, bf16 A and B, both K-major, N>>3, M>>4.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// 32 consecutive accumulator columns of this warp's 32 TMEM lanes (one row per
// lane). The wait names the destination registers as operands, so no use of
// them can be scheduled before the load has completed.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31]) : : "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ double ipow_d(double x, int e) {
    double r = 1.0;
    for (int k = 0; k < e; ++k) r *= x;
    return r;
}

constexpr int BM = kGemmBM, BN = kGemmBN, BK = kGemmBK, STAGES = kGemmStages;
constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2;
// column parameters staged per epilogue warp: one double2 per accumulator column
// of the tile and lane quarter, whatever the warp count
constexpr size_t PRM_BYTES = (size_t)4 * BN * sizeof(double2);
// Epilogue staging for TMA tensor stores: 32 x 32 blocks, a bf16 hi and lo (or h
// and silu') pair of 64-byte-row blocks, or one fp32 block of 128-byte rows.
constexpr uint32_t STG_HALF = 32 * 32 * 2;           // one 32 x 32 bf16 block
constexpr uint32_t STG_BUF = 2 * STG_HALF;           // hi + lo, or one 32 x 32 fp32 block
constexpr uint32_t TMEM_COLS = 2 * BN;   // two accumulators: epilogue of tile i overlaps tile i+1

// Epilogue variants (compile-time, so the element loop has no mode branches).
enum {
    MODE_GAP_Z4 = 0, MODE_GAP_ZINT = 1, MODE_GAP_ZREAL = 2, MODE_STORE = 3, MODE_MLP_L1 = 4,
    MODE_MLP_L2 = 5, MODE_MLP_L2B = 6, MODE_MLP_L1B = 7, N_MODES = 8
};

// The MLP epilogues round their outputs to bf16 (8-bit significand); the fast
// exponential (a few ulp at the |z| of the hidden layers) and the correctly rounded
// reciprocal are ample and keep the per-element work in the epilogue short.
__device__ __forceinline__ float sigmoid_f(float z) { return __frcp_rn(1.f + __expf(-z)); }


template <int MODE>
__device__ __forceinline__ double kpow_m1(double K, const GemmEpi &ep) {
    if (MODE == MODE_GAP_Z4) return (K * K) * K;
    if (MODE == MODE_GAP_ZINT) return ipow_d(K, ep.zeta_int - 1);
    return pow(K, ep.zeta_f - 1.0);
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Per-mode plan. The GAP epilogue (long K loop) has kGemmEpiGroups warps per TMEM
// lane quarter, each with two staging buffers. The MLP epilogues follow short K
// loops (256 .. 1232), so their element work is what bounds them: they run
// kGemmMlpEpiGroups warps per quarter (twice the warps in flight) with one staging
// buffer each. Staged modes (every output but the plain fp32 store) run a 3-stage
// operand ring, the plain store 4.
__host__ __device__ constexpr bool gap_mode(int mode) { return mode <= MODE_GAP_ZREAL; }
__host__ __device__ constexpr bool mlp_mode(int mode) { return mode >= MODE_MLP_L1; }
__host__ __device__ constexpr bool staged_mode(int mode) { return mode != MODE_STORE; }
__host__ __device__ constexpr int epi_groups(int mode) {
    return mlp_mode(mode) ? kGemmMlpEpiGroups : kGemmEpiGroups;
}
__host__ __device__ constexpr int epi_warps(int mode) { return 4 * epi_groups(mode); }
__host__ __device__ constexpr int threads_for(int mode) { return 64 + 32 * epi_warps(mode); }
__host__ __device__ constexpr int cols_per_warp(int mode) { return BN / epi_groups(mode); }
__host__ __device__ constexpr int chunks_for(int mode) { return cols_per_warp(mode) / 32; }
__host__ __device__ constexpr int stage_bufs(int mode) { return mlp_mode(mode) ? 1 : 2; }
__host__ __device__ constexpr int stages_for(int mode) { return staged_mode(mode) ? 3 : STAGES; }
__host__ __device__ constexpr size_t stg_offset(int mode) {   // from the 1024-aligned base
    return ((size_t)stages_for(mode) * (A_BYTES + B_BYTES) + 256 + PRM_BYTES + 1023) / 1024 * 1024;
}
__host__ __device__ constexpr size_t smem_bytes_for(int mode) {
    return 1024 + stg_offset(mode) +
           (staged_mode(mode) ? (size_t)epi_warps(mode) * stage_bufs(mode) * STG_BUF : 0);
}
static_assert(smem_bytes_for(MODE_GAP_Z4) <= 232448 && smem_bytes_for(MODE_STORE) <= 232448 &&
                  smem_bytes_for(MODE_MLP_L1) <= 232448,
              "shared memory plan exceeds 227 KB");
static_assert(threads_for(MODE_MLP_L1) <= 1024 && chunks_for(MODE_MLP_L1) >= 1 &&
                  chunks_for(MODE_GAP_Z4) >= 1,
              "epilogue warp plan");

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z),
                 "r"(v.w)
                 : "memory");
}

// Lane r's 32 bf16 values as row r of a 32 x 32 staging block: 64-byte rows with
// the 64-byte swizzle of the store map (16-byte chunk u sits at u ^ ((r >> 1) & 3)).
__device__ __forceinline__ void stage_row(uint32_t buf, int lane, const __nv_bfloat16 (&v)[32]) {
    const uint4 *v4 = reinterpret_cast<const uint4 *>(v);
#pragma unroll
    for (int u = 0; u < 4; ++u)
        st_shared_v4(buf + (uint32_t)lane * 64u + (uint32_t)((u ^ ((lane >> 1) & 3)) * 16), v4[u]);
}

// Before a warp refills a staging buffer: the bulk group that last read it has
// finished reading (two chunks ago with two buffers, the previous chunk with one).
template <int NBUF>
__device__ __forceinline__ void stage_acquire(int lane) {
    if (lane == 0) {
        if constexpr (NBUF == 2) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
        else asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
    __syncwarp();
}

// Lane r's 32 fp32 values as row r of a 32 x 32 fp32 staging block: 128-byte rows
// with the 128-byte swizzle of the store map (16-byte chunk u at u ^ (r & 7)).
__device__ __forceinline__ void stage_row_f32(uint32_t buf, int lane, const float (&v)[32]) {
    const uint4 *v4 = reinterpret_cast<const uint4 *>(v);
#pragma unroll
    for (int u = 0; u < 8; ++u)
        st_shared_v4(buf + (uint32_t)lane * 128u + (uint32_t)((u ^ (lane & 7)) * 16), v4[u]);
}
// After the warp's shared stores: make them visible to the async proxy.
__device__ __forceinline__ void stage_release() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
}

// TMA tensor store of a staged block (shared -> global), tracked by a bulk group
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, uint32_t src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}

// Column tile of linear tile t. Column tiles run fastest, so the CTAs of one
// wave that share a row tile read its A rows from L2 once. With rotate set (the
// grid is then a multiple of n_tiles_n, so a row tile never straddles two waves)
// wave w shifts the column tiles of every row by w, and the short last column
// tile moves from CTA to CTA instead of always landing on the same ones.
__device__ __forceinline__ int tile_col(int t, int n_tiles_n, int rotate) {
    const int n = t % n_tiles_n;
    return rotate ? (n + t / (int)gridDim.x) % n_tiles_n : n;
}

// Persistent: CTA b processes tiles b, b + gridDim.x, ... (see tile_col). Stage
// counters of the shared-memory ring run across tiles; accumulator it % 2 is
// reused every second tile once all epilogue warps have released it. With
// last_rows > 0 the last column tile loads its B operand through tmBl (a box of
// last_rows rows) and its MMAs are last_rows wide; the epilogues read no column
// past N.
template <int MODE>
__global__ void __launch_bounds__(threads_for(MODE), 1)
    k_gemm_tn(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmBl,
              int num_kb, int n_tiles_m, int n_tiles_n, int last_rows, int rotate, GemmEpi ep,
              unsigned *err) {
    constexpr int NST = stages_for(MODE);
    constexpr int EPI_WARPS = epi_warps(MODE), GROUPS = epi_groups(MODE);
    constexpr int COLS_PER_WARP = cols_per_warp(MODE), CHUNKS = chunks_for(MODE);
    constexpr int NBUF = stage_bufs(MODE);
    constexpr uint32_t STG_WARP = NBUF * STG_BUF;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *gbase = smem_raw + (base - raw);
    const uint32_t sA = base, sB = base + NST * A_BYTES;
    // barriers: full[NST], empty[NST], acc_full[2], acc_empty[2], then the TMEM
    // slot; the per-warp column-parameter slots follow the 256-byte block, the kd
    // staging buffers (GAP modes) the next 1024-byte boundary
    const uint32_t bars = sB + NST * B_BYTES;
    const uint32_t full0 = bars, empty0 = bars + 8 * NST;
    const uint32_t accf0 = bars + 16 * NST, acce0 = accf0 + 16;
    const uint32_t stg0 = base + (uint32_t)stg_offset(MODE);
    const uint32_t slot_addr = acce0 + 16;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gbase + (slot_addr - base));
    double2 *prm_all = reinterpret_cast<double2 *>(gbase + (bars + 256 - base));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // rows known only on the device (a compacted row list): tiles past them are
    // skipped by every role alike
    int rows = ep.rows;
    if (ep.rows_dev) rows = min(rows, max(*ep.rows_dev, 0));
    const int n_tiles = min(n_tiles_m, (rows + BM - 1) / BM) * n_tiles_n;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(accf0 + 8 * a, 1);           // tcgen05.commit of the last k-block
            mbar_init(acce0 + 8 * a, EPI_WARPS);   // one arrive per epilogue warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_addr),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- TMA producer
        int g = 0;   // k-blocks issued so far (all tiles)
        bool ok = ep.stall_test == 0;   // the failure test issues nothing
        for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
            const int tn = tile_col(t, n_tiles_n, rotate);
            const int m0 = (t / n_tiles_n) * BM, n0 = tn * BN;
            const bool short_tile = last_rows > 0 && tn == n_tiles_n - 1;
            const uint32_t b_bytes = short_tile ? (uint32_t)last_rows * BK * 2 : B_BYTES;
            const int ak = ep.bd_block > 0 ? (n0 / ep.bd_block) * ep.bd_block : 0;
            for (int kb = 0; kb < num_kb; ++kb, ++g) {
                const int s = g % NST;
                const uint32_t ph = (uint32_t)(g / NST) & 1u;
                if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, err)) {
                    atomicOr(err, (unsigned)DEV_ERR_TIMEOUT_TMA);
                    ok = false;
                    break;
                }
                mbar_expect_tx(full0 + 8 * s, A_BYTES + b_bytes);
                int ax = ak + kb * BK;
                if (ep.a_krep > 0 && ax >= ep.a_krep) ax -= ep.a_krep;
                tma_load_2d(sA + s * A_BYTES, &tmA, ax, m0, full0 + 8 * s);
                tma_load_2d(sB + s * B_BYTES, short_tile ? &tmBl : &tmB, kb * BK, n0,
                            full0 + 8 * s);
            }
        }
        // Drain: the last load of every stage has landed before the CTA may exit
        // (already true on the normal path, where the MMA consumed them).
        for (int k = g > NST ? g - NST : 0; k < g; ++k)
            (void)mbar_wait(full0 + 8 * (k % NST), (uint32_t)(k / NST) & 1u, err);
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer
        constexpr uint32_t idesc_full = make_idesc(BM, BN);
        int g = 0, it = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, ++it) {
            const bool short_tile = last_rows > 0 && tile_col(t, n_tiles_n, rotate) == n_tiles_n - 1;
            const uint32_t idesc = short_tile ? make_idesc(BM, last_rows) : idesc_full;
            const int a = it & 1;
            const uint32_t use = (uint32_t)(it >> 1);
            if (!mbar_wait(acce0 + 8 * a, (use & 1u) ^ 1u, err)) {
                atomicOr(err, (unsigned)DEV_ERR_TIMEOUT_MMA);
                break;
            }
            tc_fence_after();
            const uint32_t dacc = tmem + (uint32_t)(a * BN);
            for (int kb = 0; kb < num_kb; ++kb, ++g) {
                const int s = g % NST;
                const uint32_t ph = (uint32_t)(g / NST) & 1u;
                if (!mbar_wait(full0 + 8 * s, ph, err)) {
                    atomicOr(err, (unsigned)DEV_ERR_TIMEOUT_MMA);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = sA + s * A_BYTES, b0 = sB + s * B_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk)
                    tc_mma(dacc, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32), idesc,
                           (kb > 0 || kk > 0) ? 1u : 0u);
                tc_commit(empty0 + 8 * s);
            }
            tc_commit(accf0 + 8 * a);
        }
    } else if (warp >= 2) {
      // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (the lane quarter
      // the hardware lets it access) and column group (w - 2) / 4 of the tile
      const int q = warp & 3;
      const int grp = (warp - 2) >> 2;
      double2 *prm = prm_all + (warp - 2) * CHUNKS * 32;
      const uint32_t stg_warp = stg0 + (uint32_t)(warp - 2) * STG_WARP;
      int nbuf = 0;   // kd staging buffers used so far (alternating)
      int it = 0;
      for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
        const int a = it & 1;
        const uint32_t use = (uint32_t)(it >> 1);
        const int tile_n = tile_col(t, n_tiles_n, rotate);
        const int m0 = (t / n_tiles_n) * BM, n0 = tile_n * BN;
        const int row = m0 + q * 32 + lane;
        const bool row_ok = row < rows;
        // MLP epilogues: the tile's global inputs (column parameters; the bf16
        // silu'(z1) factors of L2B) are requested before the wait for the
        // accumulator, so their latency overlaps the MMA of this tile
        float a0[mlp_mode(MODE) ? CHUNKS : 1], a1[mlp_mode(MODE) ? CHUNKS : 1];
        uint4 pre[MODE == MODE_MLP_L2B ? CHUNKS : 1][4];
        if constexpr (mlp_mode(MODE) && MODE != MODE_MLP_L2B) {
#pragma unroll
            for (int c = 0; c < CHUNKS; ++c) {
                const int cl = n0 + grp * COLS_PER_WARP + c * 32 + lane;
                a0[c] = 0.f;
                a1[c] = 0.f;
                if (cl < ep.cols) {
                    if (ep.p0) a0[c] = ep.p0[cl];
                    if constexpr (MODE == MODE_MLP_L2) a1[c] = ep.p1[cl];
                }
            }
        }
        if constexpr (MODE == MODE_MLP_L2B) {
#pragma unroll
            for (int c = 0; c < CHUNKS; ++c) {
                const int gcol = n0 + grp * COLS_PER_WARP + c * 32;
                if (row_ok && gcol < ep.cols) {
                    const uint4 *s4 = reinterpret_cast<const uint4 *>(ep.in_b + (size_t)row * ep.ldi + gcol);
#pragma unroll
                    for (int u = 0; u < 4; ++u) pre[c][u] = s4[u];
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u) pre[c][u] = make_uint4(0, 0, 0, 0);
                }
            }
        }
        const bool ready = mbar_wait(accf0 + 8 * a, use & 1u, err);
        if (!ready) {
            if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_TIMEOUT_EPI);
            break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem + (uint32_t)(a * BN) + ((uint32_t)(q * 32) << 16);
        if constexpr (MODE >= MODE_MLP_L1) {
            // the MLP epilogues: float column parameters staged per warp like the GAP ones
            float2 *pfall = reinterpret_cast<float2 *>(prm);
            if constexpr (MODE != MODE_MLP_L2B) {
                __syncwarp();
#pragma unroll
                for (int c = 0; c < CHUNKS; ++c) pfall[c * 32 + lane] = make_float2(a0[c], a1[c]);
                __syncwarp();
            }
            float racc = 0.f;
#pragma unroll
            for (int c = 0; c < CHUNKS; ++c) {
                const int col = grp * COLS_PER_WARP + c * 32;
                const int gcol = n0 + col;
                if (gcol >= ep.cols) break;   // warp-uniform
                const float2 *pf = pfall + c * 32;
                float v[32];
                tmem_ld32(taddr + (uint32_t)col, v);
                if constexpr (MODE == MODE_MLP_L1) {
                    __align__(16) __nv_bfloat16 hb[32], sb[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const float z = v[j] + pf[j].x, sg = sigmoid_f(z);
                        hb[j] = __float2bfloat16_rn(z * sg);
                        sb[j] = __float2bfloat16_rn(sg * (1.f + z * (1.f - sg)));
                    }
                    // h1 and silu'(z1) blocks of one [rows x 2 HH] matrix (s at x2 + col)
                    const uint32_t sbuf = stg_warp + (NBUF == 2 ? (uint32_t)(nbuf & 1) * STG_BUF : 0u);
                    stage_acquire<NBUF>(lane);
                    stage_row(sbuf, lane, hb);
                    stage_row(sbuf + STG_HALF, lane, sb);
                    stage_release();
                    const int y = m0 + q * 32;
                    if (lane == 0 && y < rows) {
                        tma_store_2d(&tmC, sbuf, gcol, y);
                        tma_store_2d(&tmC, sbuf + STG_HALF, ep.x2 + gcol, y);
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    }
                    ++nbuf;
                } else if constexpr (MODE == MODE_MLP_L2) {
                    __align__(16) __nv_bfloat16 ub[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const float2 q2 = pf[j];
                        const float z = v[j] + q2.x, sg = sigmoid_f(z);
                        racc += q2.y * z * sg;
                        ub[j] = __float2bfloat16_rn(q2.y * sg * (1.f + z * (1.f - sg)));
                    }
                    const uint32_t sbuf = stg_warp + (NBUF == 2 ? (uint32_t)(nbuf & 1) * STG_BUF : 0u);
                    stage_acquire<NBUF>(lane);
                    stage_row(sbuf, lane, ub);
                    stage_release();
                    const int y = m0 + q * 32;
                    if (lane == 0 && y < rows) {
                        tma_store_2d(&tmC, sbuf, gcol, y);
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    }
                    ++nbuf;
                } else if constexpr (MODE == MODE_MLP_L2B) {
                    __align__(16) __nv_bfloat16 sf[32], ub[32];
                    uint4 *t4 = reinterpret_cast<uint4 *>(sf);
#pragma unroll
                    for (int u = 0; u < 4; ++u) t4[u] = pre[c][u];
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        ub[j] = __float2bfloat16_rn(v[j] * __bfloat162float(sf[j]));
                    const uint32_t sbuf = stg_warp + (NBUF == 2 ? (uint32_t)(nbuf & 1) * STG_BUF : 0u);
                    stage_acquire<NBUF>(lane);
                    stage_row(sbuf, lane, ub);
                    stage_release();
                    const int y = m0 + q * 32;
                    if (lane == 0 && y < rows) {
                        tma_store_2d(&tmC, sbuf, gcol, y);
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    }
                    ++nbuf;
                } else {   // MODE_MLP_L1B
                    __align__(16) float ov[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) ov[j] = ep.scale * v[j] - pf[j].x;
                    const int y = m0 + q * 32;   // warp-uniform
                    if (y + 32 <= rows) {
                        // a whole 32-row block: staged and written by one TMA store,
                        // which clips the columns at the map's width (ep.cols)
                        stage_acquire<NBUF>(lane);
                        stage_row_f32(stg_warp, lane, ov);
                        stage_release();
                        if (lane == 0) {
                            tma_store_2d(&tmC, stg_warp, gcol, y);
                            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                        }
                    } else if (row_ok) {   // the last, partial block: plain stores
                        float *o = ep.out + (size_t)row * ep.ldo + gcol;
                        if (gcol + 32 <= ep.cols) {
                            float4 *o4 = reinterpret_cast<float4 *>(o);
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                o4[j] = make_float4(ov[4 * j], ov[4 * j + 1], ov[4 * j + 2],
                                                    ov[4 * j + 3]);
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (gcol + j < ep.cols) o[j] = ov[j];
                        }
                    }
                }
            }
            if constexpr (MODE == MODE_MLP_L2) {
                if (row_ok)
                    ep.rowpart[(size_t)row * ep.rowpart_ld + tile_n * GROUPS + grp] = racc;
            }
        } else if constexpr (MODE != MODE_STORE) {
            double e4[4] = {0, 0, 0, 0}, k4[4] = {0, 0, 0, 0};
            const double qo = row_ok ? ep.qoff[row] : 0.0;
            const float c0f = (float)ep.c0;
            // column parameters (alpha_s, mu . q_s) of all this warp's chunks: lane l
            // loads column l of each chunk (all loads in flight together), the element
            // loop reads them back as shared-memory broadcasts
            {
                double a0[CHUNKS], a1[CHUNKS];
#pragma unroll
                for (int c = 0; c < CHUNKS; ++c) {
                    const int cl = n0 + grp * COLS_PER_WARP + c * 32 + lane;
                    a0[c] = cl < ep.Mpad ? ep.alpha[cl] : 0.0;
                    a1[c] = cl < ep.Mpad ? ep.aoff[cl] : 0.0;
                }
                __syncwarp();
#pragma unroll
                for (int c = 0; c < CHUNKS; ++c) prm[c * 32 + lane] = make_double2(a0[c], a1[c]);
                __syncwarp();
            }
            for (int c = 0; c < CHUNKS; ++c) {
                const int col = grp * COLS_PER_WARP + c * 32;
                const int gcol = n0 + col;
                if (gcol >= ep.Mpad) break;   // warp-uniform; Mpad is a multiple of 32
                const double2 *pc = prm + c * 32;
                float v[32];
                tmem_ld32(taddr + (uint32_t)col, v);
                __align__(16) __nv_bfloat16 hi[32], lo[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const double2 p = pc[j];
                    const double K = ((double)v[j] + p.y) + qo;
                    // alpha_s K^(zeta-1); with a real zeta a padding column (alpha 0,
                    // K = delta . mu, which may be negative) must give 0, not 0 x NaN
                    double t1;
                    if constexpr (MODE == MODE_GAP_ZREAL) t1 = p.x != 0.0 ? p.x * kpow_m1<MODE>(K, ep) : 0.0;
                    else t1 = p.x * kpow_m1<MODE>(K, ep);
                    k4[j & 3] += t1;
                    e4[j & 3] = fma(t1, K, e4[j & 3]);
                    // kd_s - kcoef_s = zeta delta^2 (alpha_s K^(zeta-1) - alpha_s)
                    bf16_split((float)(t1 - p.x) * c0f, hi[j], lo[j]);
                }
                // Stage the 32 x 32 hi / lo blocks (64-byte rows, 64-byte swizzle: the
                // 16-byte chunk u of row r sits at chunk u ^ ((r >> 1) & 3)) and let TMA
                // write them out as whole lines. Rows past the tensor are clipped by TMA.
                const uint32_t sbuf = stg_warp + (NBUF == 2 ? (uint32_t)(nbuf & 1) * STG_BUF : 0u);
                stage_acquire<NBUF>(lane);
                stage_row(sbuf, lane, hi);
                if (ep.nsplit == 3) stage_row(sbuf + STG_HALF, lane, lo);
                stage_release();
                const int y = m0 + q * 32;   // warp-uniform
                if (lane == 0 && y < rows) {   // partial blocks are clipped by TMA
                    tma_store_2d(&tmC, sbuf, gcol, y);
                    if (ep.nsplit == 3) tma_store_2d(&tmC, sbuf + STG_HALF, ep.Mpad + gcol, y);
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
                ++nbuf;
            }
            if (row_ok) {
                const size_t o = ((size_t)row * n_tiles_n + tile_n) * GROUPS + grp;
                ep.epart[o] = (e4[0] + e4[1]) + (e4[2] + e4[3]);
                ep.kdsum[o] = ep.c0 * ((k4[0] + k4[1]) + (k4[2] + k4[3]));
            }
        } else {
            for (int c = 0; c < COLS_PER_WARP / 32; ++c) {
                const int col = grp * COLS_PER_WARP + c * 32;
                const int gcol = n0 + col;
                if (gcol >= ep.cols) break;   // warp-uniform
                float v[32];
                tmem_ld32(taddr + (uint32_t)col, v);
                if (!row_ok) continue;
                float *o = ep.out + (size_t)row * ep.ldo + gcol;
                if (gcol + 32 <= ep.cols) {
                    float4 *o4 = reinterpret_cast<float4 *>(o);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        o4[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (gcol + j < ep.cols) o[j] = v[j];
                }
            }
        }
        // release accumulator a to the MMA issuer
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * a);
      }
      if constexpr (staged_mode(MODE)) {   // the staged stores have landed before the CTA exits
          if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
          __syncwarp();
      }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder() {
    if (g_encode) return TG_OK;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
        set_error("cuTensorMapEncodeTiled not available from the driver");
        return TG_ERR_CUDA;
    }
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return TG_OK;
}

}  // namespace

int make_tma_bf16(TmaMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld,
                  int box_rows) {
    TGB_TRY(get_encoder());
    TGB_CHECK(((uintptr_t)base & 15) == 0, TG_ERR_ARG, "TMA base address not 16-byte aligned");
    TGB_CHECK((ld * 2) % 16 == 0, TG_ERR_ARG, "TMA row stride %lld B not a multiple of 16",
              (long long)(ld * 2));
    TGB_CHECK(rows >= 1 && cols >= 1, TG_ERR_ARG, "empty TMA extent");
    cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {(cuuint32_t)kGemmBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(&m->map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base),
                          gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    TGB_CHECK(r == CUDA_SUCCESS, TG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TG_OK;
}

int make_tma_store_bf16(TmaMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld) {
    TGB_TRY(get_encoder());
    TGB_CHECK(((uintptr_t)base & 15) == 0, TG_ERR_ARG, "TMA base address not 16-byte aligned");
    TGB_CHECK((ld * 2) % 16 == 0, TG_ERR_ARG, "TMA row stride %lld B not a multiple of 16",
              (long long)(ld * 2));
    TGB_CHECK(rows >= 1 && cols >= 1, TG_ERR_ARG, "empty TMA extent");
    cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(&m->map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base),
                          gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    TGB_CHECK(r == CUDA_SUCCESS, TG_ERR_CUDA, "cuTensorMapEncodeTiled (store) failed (%d)", (int)r);
    return TG_OK;
}

int make_tma_store_f32(TmaMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld) {
    TGB_TRY(get_encoder());
    TGB_CHECK(((uintptr_t)base & 15) == 0, TG_ERR_ARG, "TMA base address not 16-byte aligned");
    TGB_CHECK((ld * 4) % 16 == 0, TG_ERR_ARG, "TMA row stride %lld B not a multiple of 16",
              (long long)(ld * 4));
    TGB_CHECK(rows >= 1 && cols >= 1, TG_ERR_ARG, "empty TMA extent");
    cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)(ld * 4)};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(&m->map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base),
                          gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    TGB_CHECK(r == CUDA_SUCCESS, TG_ERR_CUDA, "cuTensorMapEncodeTiled (fp32 store) failed (%d)", (int)r);
    return TG_OK;
}

int launch_gemm_tn(const TmaMap &A, const TmaMap &B, int M, int N, int K, const GemmEpi &ep,
                   unsigned *err, cudaStream_t st, const TmaMap *C, const TmaMap *Blast) {
    TGB_CHECK(K % kGemmBK == 0, TG_ERR_ARG, "GEMM K=%d must be a multiple of %d", K, kGemmBK);
    // 16-byte vector stores in the epilogues
    TGB_CHECK(ep.mode != EPI_STORE_F32 || (ep.ldo % 4 == 0 && ((uintptr_t)ep.out & 15) == 0),
              TG_ERR_ARG, "fp32 output rows must be 16-byte aligned (ldo %% 4 == 0)");
    TGB_CHECK(ep.mode != EPI_GAP_KERNEL || (ep.K2 % 8 == 0 && ep.Mpad % 32 == 0 &&
                                            ((uintptr_t)ep.kd & 15) == 0 && C != nullptr),
              TG_ERR_ARG, "GAP epilogue: 16-byte kd rows, Mpad %% 32 == 0 and a kd store map");
    if (M <= 0 || N <= 0) return TG_OK;
    TGB_CHECK(ep.mode < EPI_MLP_L1 || ep.mode == EPI_MLP_L1B || (C != nullptr && N % 32 == 0 &&
                                                                   ep.x2 % 32 == 0),
              TG_ERR_ARG, "bf16 MLP outputs need a store map, N %% 32 == 0 and x2 %% 32 == 0");
    TGB_CHECK(ep.mode != EPI_MLP_L2B || (ep.ldi % 8 == 0 && ((uintptr_t)ep.in_b & 15) == 0),
              TG_ERR_ARG, "bf16 MLP factor rows must be 16-byte aligned");
    TGB_CHECK(ep.mode != EPI_MLP_L1B || (ep.ldo % 4 == 0 && ((uintptr_t)ep.out & 15) == 0 &&
                                         C != nullptr),
              TG_ERR_ARG, "MLP fp32 output: 16-byte aligned rows (ldo %% 4 == 0) and a store map");
    int mode = MODE_STORE;
    switch (ep.mode) {
        case EPI_GAP_KERNEL:
            mode = ep.zeta_int == 4 ? MODE_GAP_Z4 : ep.zeta_int > 0 ? MODE_GAP_ZINT : MODE_GAP_ZREAL;
            break;
        case EPI_MLP_L1: mode = MODE_MLP_L1; break;
        case EPI_MLP_L2: mode = MODE_MLP_L2; break;
        case EPI_MLP_L2B: mode = MODE_MLP_L2B; break;
        case EPI_MLP_L1B: mode = MODE_MLP_L1B; break;
        default: mode = MODE_STORE;
    }
    using Kern = void (*)(CUtensorMap, CUtensorMap, CUtensorMap, CUtensorMap, int, int, int, int,
                          int, GemmEpi, unsigned *);
    static const Kern kerns[N_MODES] = {
        k_gemm_tn<MODE_GAP_Z4>, k_gemm_tn<MODE_GAP_ZINT>, k_gemm_tn<MODE_GAP_ZREAL>,
        k_gemm_tn<MODE_STORE>, k_gemm_tn<MODE_MLP_L1>, k_gemm_tn<MODE_MLP_L2>,
        k_gemm_tn<MODE_MLP_L2B>, k_gemm_tn<MODE_MLP_L1B>};
    static bool attr[N_MODES] = {};
    if (!attr[mode]) {
        TGB_CUDA(cudaFuncSetAttribute(kerns[mode], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_bytes_for(mode)));
        attr[mode] = true;
    }
    static int n_sm = 0;
    if (!n_sm) {
        int dev = 0;
        TGB_CUDA(cudaGetDevice(&dev));
        TGB_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    }
    const int tm = (M + BM - 1) / BM, tn = (N + BN - 1) / BN;
    int grid = std::min(tm * tn, n_sm);   // persistent: one CTA per SM
    const int last_rows = Blast ? gemm_last_box_rows(N) : 0;
    // A short last column tile among at most four pays for the SMs a grid that is
    // a multiple of the column-tile count may leave idle (none with two tiles on
    // 148 SMs): the waves then rotate the short tile over the CTAs.
    const int rotate = (last_rows > 0 && tn > 1 && tn <= 4 && grid == n_sm) ? 1 : 0;
    if (rotate) grid = n_sm / tn * tn;
    kerns[mode]<<<grid, threads_for(mode), smem_bytes_for(mode), st>>>(
        A.map, B.map, C ? C->map : A.map, Blast ? Blast->map : B.map, K / kGemmBK, tm, tn, last_rows,
        rotate, ep, err);
    TGB_CUDA(cudaGetLastError());
    return TG_OK;
}

}  // namespace tgb
