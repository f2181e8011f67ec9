// tgb_capi.cu -- context, sparse-set blocks, the get_gap_soap path, the neighbour
// list entry point and the device-resident MD engine behind include/tgb200.h.

#include "tgb_common.cuh"
#include "tgb_gemm.cuh"
#include "tgb_mlp.cuh"
#include "tgb_comm.cuh"
#include "tgb_family.cuh"
#include "tgb_neighbors.cuh"
#include "tgb_soap.cuh"

#include <cub/device/device_scan.cuh>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

namespace tgb {

// ---------------------------------------------------------------- errors
static thread_local char g_err[2048] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char *last_error() { return g_err; }

int init_soap_constants();

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    int ensure(size_t m) {
        if (m <= n && p) return TG_OK;
        dev_free(p);
        n = 0;
        TGB_TRY(dev_alloc(&p, m));
        n = m;
        return TG_OK;
    }
    void release() {
        dev_free(p);
        n = 0;
    }
    ~DBuf() { release(); }
};

static int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Largest compressed descriptor accepted (the GEMM operands grow with it).
constexpr int kMaxCompressedDim = 16384;

// ---------------------------------------------------------------- blocks
struct Block {
    int key = 0, precision = TG_PREC_BF16X3;
    SoapHostHypers hh{};
    int ns = 0, amax = 0, lmax = 0, ntot = 0, nlm = 0, dim = 0;
    // dim: entries of the descriptor rows the GEMMs see. Uncompressed, dim = dimf
    // (the power spectrum); compressed, dim = dimc (the transformation's own dim)
    // rounded up to a multiple of 8 with zero entries.
    int dimf = 0, dimc = 0;
    int M = 0, Mpad = 0, K1 = 0, K2 = 0, nsplit = 3, n_etiles = 0, tw = 0;
    int KD = 0;   // stored kd row: [hi | lo] (bf16x3) or [hi]; GEMM 2 reads hi twice
    double delta = 1.0, zeta = 1.0, rcut_max = 0.0;
    int zeta_int = 0;
    signed char zmap[kMaxZ], zmap2[kMaxZ];   // first and second descriptor species of a global id
    int n_inst = 1;                          // 2 when a global species appears twice
    DBuf<float> table, selfR;
    DBuf<float4> table_fd;   // the descriptor's (f, f') interval copy
    DBuf<__nv_bfloat16> QsA, QsT;
    DBuf<double> alpha, mu, aoff, g0;
    DBuf<float> g0f;       // g0 in fp32: subtracted from the MLP's dE/dq rows
    DBuf<float> muf;       // mu in fp32
    double mu2 = 0.0, g0mu = 0.0;   // mu . mu, g0 . mu
    DBuf<int> ref_index;   // [dim]: reference position of internal descriptor entry d (-1: padding)
    TmaMap tmB1{}, tmB2{};
    TmaMap tmB1l{}, tmB2l{};   // the short last column tile's B maps (N % kGemmBN != 0)
    const TmaMap *last1() const { return gemm_last_box_rows(Mpad) ? &tmB1l : nullptr; }
    const TmaMap *last2() const { return gemm_last_box_rows(dim) ? &tmB2l : nullptr; }
    // compression matrix C (dim x dimf) as CSR by row and by column
    DBuf<int> c_row_ptr, c_row_col, c_col_idx, c_col_ptr, c_col_row;
    DBuf<double> c_row_val, c_col_val;
    int c_ncols = 0;

    bool compressed() const { return dimc > 0; }
    CompressArgs cargs() const {
        return CompressArgs{dimf, c_row_ptr.p, c_row_col.p, c_row_val.p,
                            c_ncols, c_col_idx.p, c_col_ptr.p, c_col_row.p, c_col_val.p};
    }

    SoapParams params(int n_atoms) const {
        SoapParams P{};
        P.ns = ns; P.amax = amax; P.lmax = lmax; P.ntot = ntot; P.nlm = nlm; P.dim = dim;
        P.nsplit = nsplit; P.K1 = K1; P.tw = tw; P.n_atoms = n_atoms;
        std::memcpy(P.zmap, zmap, sizeof(zmap));
        std::memcpy(P.zmap2, zmap2, sizeof(zmap2));
        P.n_inst = n_inst;
        for (int s = 0; s < ns; ++s) {
            P.rcut[s] = (float)hh.rcut_hard[s];
            P.tab_h[s] = (float)(hh.rcut_hard[s] / kTableIntervals);
            P.tab_inv_h[s] = (float)(kTableIntervals / hh.rcut_hard[s]);
        }
        P.table = table.p;
        P.table_fd = table_fd.p;
        P.self_R = selfR.p;
        P.mu = mu.p;
        P.g0 = g0.p;
        P.muf = muf.p;
        P.g0f = g0f.p;
        P.mu2 = mu2;
        P.g0mu = g0mu;
        P.raw = compressed() ? 1 : 0;
        return P;
    }
};

// The kd scratch (GEMM 1's split kernel derivative, GEMM 2's A operand) is
// bounded: the two GEMMs run over row chunks of kd_chunk_rows() sites, so kd
// holds one chunk. Chunks are whole 128-row tiles; the per-row arithmetic does
// not depend on the chunking.
constexpr size_t kKdScratchBytes = size_t(1) << 30;

static int kd_chunk_rows(const Block &b, int n_sites) {
    long long rows = (long long)(kKdScratchBytes / (sizeof(__nv_bfloat16) * (size_t)b.KD));
    if (const char *e = std::getenv("TGB_KD_CHUNK_ROWS")) {   // tests: force several chunks
        const long long v = std::atoll(e);
        if (v > 0) rows = v;
    }
    rows = std::max<long long>(kGemmBM, rows / kGemmBM * kGemmBM);
    const long long n = std::max(n_sites, 1);
    return (int)std::min<long long>(rows, (n + kGemmBM - 1) / kGemmBM * kGemmBM);
}

// Per-block evaluation buffers, sized by the number of central sites.
struct Workspace {
    int cap = 0;
    int kd_rows = 0;           // rows of kd (one GEMM row chunk)
    DBuf<__nv_bfloat16> qsplit, kd;
    DBuf<float> q, c, g;
    DBuf<double> praw;         // compressed blocks: p, [n][dimf]
    DBuf<float> gfull;         //   and dE/dp
    DBuf<double> pnorm, epart, kdsum, qoff, vpart;
    TmaMap tmA1{}, tmA2{}, tmKd{};   // tmKd: the GAP epilogue's TMA stores into kd
    int tm_rows = -1, tm_k1 = -1, tm_kd = -1, tm_kdrows = -1;
    const void *tm_p1 = nullptr, *tm_p2 = nullptr;
    int tile_desc = 0, tile_force = 0;   // CTA tiles of the two SOAP passes (autotuned)

    int ensure(const Block &b, int n_sites) {
        const int n = n_sites > 0 ? n_sites : 1;
        const int R = kd_chunk_rows(b, n);
        if (n > cap || q.n < (size_t)n * b.dim || kd.n < (size_t)R * b.KD ||
            qsplit.n < (size_t)n * b.K1 || c.n < (size_t)n * b.ntot * b.nlm ||
            epart.n < (size_t)n * b.n_etiles || kdsum.n < (size_t)n * b.n_etiles ||
            (b.compressed() && (praw.n < (size_t)n * b.dimf || gfull.n < (size_t)n * b.dimf))) {
            const int nc = n > cap ? n : cap;
            TGB_TRY(qsplit.ensure((size_t)nc * b.K1));
            TGB_TRY(kd.ensure((size_t)R * b.KD));
            TGB_TRY(q.ensure((size_t)nc * b.dim));
            TGB_TRY(g.ensure((size_t)nc * b.dim));
            TGB_TRY(c.ensure((size_t)nc * b.ntot * b.nlm));
            TGB_TRY(pnorm.ensure(nc));
            TGB_TRY(epart.ensure((size_t)nc * b.n_etiles));
            TGB_TRY(kdsum.ensure((size_t)nc * b.n_etiles));
            TGB_TRY(qoff.ensure(nc));
            TGB_TRY(vpart.ensure((size_t)9 * ((nc + 1) / 2 + 1)));   // the 2-site tile
            if (b.compressed()) {
                TGB_TRY(praw.ensure((size_t)nc * b.dimf));
                TGB_TRY(gfull.ensure((size_t)nc * b.dimf));
            }
            cap = nc;
        }
        kd_rows = R;
        if (tm_rows != n || tm_p1 != qsplit.p || tm_p2 != kd.p || tm_k1 != b.K1 || tm_kd != b.KD ||
            tm_kdrows != R) {
            TGB_TRY(make_tma_bf16(&tmA1, qsplit.p, n, b.K1, b.K1, kGemmBM));
            TGB_TRY(make_tma_bf16(&tmA2, kd.p, R, b.KD, b.KD, kGemmBM));
            TGB_TRY(make_tma_store_bf16(&tmKd, kd.p, R, b.KD, b.KD));
            tm_rows = n;
            tm_p1 = qsplit.p;
            tm_p2 = kd.p;
            tm_k1 = b.K1;
            tm_kd = b.KD;
            tm_kdrows = R;
        }
        return TG_OK;
    }
};

namespace {

__global__ void k_prep_sparse(const double *__restrict__ Qs, const double *__restrict__ mu, int M,
                              int Mpad, int dim, int K1, int K2, int nsplit,
                              __nv_bfloat16 *__restrict__ QsA, __nv_bfloat16 *__restrict__ QsT) {
    // Operands hold q_s - mu. B-side pattern per segment: [hi | lo | hi] (nsplit 3)
    // or [hi] (nsplit 1); the A side is [hi | hi | lo], so the three products are
    // hi.hi + hi.lo + lo.hi.
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nA = (int64_t)Mpad * K1, nT = (int64_t)dim * K2;
    if (t < nA) {
        const int s = (int)(t / K1), k = (int)(t % K1);
        float v = 0.f;
        int seg = k / dim, d = k % dim;
        if (s < M && seg < nsplit) {
            const float x = (float)(Qs[(size_t)s * dim + d] - mu[d]);
            __nv_bfloat16 hi, lo;
            bf16_split(x, hi, lo);
            v = __bfloat162float(seg == 1 ? lo : hi);
        }
        QsA[t] = __float2bfloat16_rn(v);
    } else if (t < nA + nT) {
        const int64_t u = t - nA;
        const int d = (int)(u / K2), k = (int)(u % K2);
        const int seg = k / Mpad, s = k % Mpad;
        float v = 0.f;
        if (s < M && seg < nsplit) {
            const float x = (float)(Qs[(size_t)s * dim + d] - mu[d]);
            __nv_bfloat16 hi, lo;
            bf16_split(x, hi, lo);
            v = __bfloat162float(seg == 1 ? lo : hi);
        }
        QsT[u] = __float2bfloat16_rn(v);
    }
}

__global__ void k_prep_alpha(const double *__restrict__ al, int M, int Mpad,
                             double *__restrict__ alpha) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= Mpad) return;
    alpha[s] = s < M ? al[s] : 0.0;
}

}  // namespace

// Optional CUDA-event log of the passes of a step: mark(pass) records an event
// on the stream; the time since the previous mark is booked to that pass.
enum Pass {
    PASS_NEIGH = 0, PASS_DESC, PASS_GEMM1, PASS_GEMM2, PASS_FORCE, PASS_INTEGRATE, PASS_MLP, N_PASS
};

// A host-side NVTX range over one C-ABI call, so that a profiler's timeline
// (ncu --nvtx, nsys) shows which entry point launched which kernels. NVTX v3 is
// header-only: without a tool attached a range costs a few nanoseconds.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

struct EventLog {
    std::vector<cudaEvent_t> ev;
    std::vector<int> pass;
    size_t used = 0;
    int mark(int p, cudaStream_t st) {
        if (used == ev.size()) {
            cudaEvent_t e;
            TGB_CUDA(cudaEventCreate(&e));
            ev.push_back(e);
            pass.push_back(p);
        }
        pass[used] = p;
        TGB_CUDA(cudaEventRecord(ev[used], st));
        ++used;
        return TG_OK;
    }
    // accumulate ms per pass over the recorded marks (stream must be synchronised)
    int collect(double *ms) {
        for (size_t i = 1; i < used; ++i) {
            float t = 0.f;
            TGB_CUDA(cudaEventElapsedTime(&t, ev[i - 1], ev[i]));
            if (pass[i] >= 0) ms[pass[i]] += t;
        }
        used = 0;
        return TG_OK;
    }
    ~EventLog() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

#define TGB_MARK(log, p, st)                     \
    do {                                         \
        if (log) TGB_TRY((log)->mark((p), (st))); \
    } while (0)

// The descriptor pass: the SOAP expansion and power spectrum, and for a
// compressed block the compression after it (the expansion then leaves the raw
// power spectrum in praw).
int descriptor_pass(const Block &b, Workspace &w, const SoapParams &P, const SiteArgs &S,
                    cudaStream_t st, int tile) {
    DescOut O{w.qsplit.p, w.q.p, w.qoff.p, w.pnorm.p, w.c.p, w.praw.p};
    TGB_TRY(launch_soap_expand(P, S, O, st, tile));
    if (!b.compressed()) return TG_OK;
    return launch_compress_forward(P, b.cargs(), S.n_sites, w.praw.p, O, st);
}

// The force pass; a compressed block first takes dE/dq back to dE/dp.
int force_pass(const Block &b, Workspace &w, const SoapParams &P, const SiteArgs &S, ForceIn I,
               const ForceOut &FO, int *nblk, cudaStream_t st, int tile) {
    if (b.compressed()) {
        TGB_TRY(launch_compress_adjoint(P, b.cargs(), S.n_sites, I, w.gfull.p, st));
        I.g = w.gfull.p;
    }
    return launch_soap_force(P, S, I, FO, nblk, st, tile);
}

// GEMM 1's epilogue parameters for a block (rows and per-row outputs set by the caller).
static GemmEpi gap_epilogue(const Block &b, const Workspace &w) {
    GemmEpi e1{};
    e1.mode = EPI_GAP_KERNEL;
    e1.cols = b.Mpad;
    e1.alpha = b.alpha.p;
    e1.c0 = b.zeta * b.delta * b.delta;
    e1.zeta_int = b.zeta_int;
    e1.zeta_f = b.zeta;
    e1.aoff = b.aoff.p;
    e1.kd = w.kd.p;
    e1.K2 = b.KD;
    e1.Mpad = b.Mpad;
    e1.nsplit = b.nsplit;
    return e1;
}

// Descriptor, GEMM 1 (kernel + energy epilogue), GEMM 2 (dE/dq), forces. The
// GEMMs run chunk by chunk over w.kd_rows sites, GEMM 2 of a chunk right after
// its GEMM 1, so kd holds one chunk.
int evaluate_block(Block &b, Workspace &w, const SiteArgs &S, int n_atoms, double *forces,
                   double *energies, double *virial, unsigned *err, cudaStream_t st,
                   EventLog *log = nullptr, const int *atom_struct = nullptr,
                   double *vir_struct = nullptr, double *pair_grad = nullptr) {
    if (S.n_sites <= 0) return TG_OK;
    TGB_TRY(w.ensure(b, S.n_sites));
    const SoapParams P = b.params(n_atoms);
    TGB_TRY(descriptor_pass(b, w, P, S, st, w.tile_desc));
    TGB_MARK(log, PASS_DESC, st);
    const int n = S.n_sites, R = w.kd_rows;
    for (int r0 = 0; r0 < n; r0 += R) {
        const int nr = std::min(R, n - r0);
        TmaMap a1c;
        const TmaMap *a1 = &w.tmA1;
        if (nr < n) {   // this chunk's rows of the split-q operand
            TGB_TRY(make_tma_bf16(&a1c, w.qsplit.p + (size_t)r0 * b.K1, nr, b.K1, b.K1, kGemmBM));
            a1 = &a1c;
        }
        GemmEpi e1 = gap_epilogue(b, w);
        e1.rows = nr;
        e1.epart = w.epart.p + (size_t)r0 * b.n_etiles;
        e1.kdsum = w.kdsum.p + (size_t)r0 * b.n_etiles;
        e1.qoff = w.qoff.p + r0;
        TGB_TRY(launch_gemm_tn(*a1, b.tmB1, nr, b.Mpad, b.K1, e1, err, st, &w.tmKd, b.last1()));
        TGB_MARK(log, PASS_GEMM1, st);
        GemmEpi e2{};
        e2.mode = EPI_STORE_F32;
        e2.rows = nr;
        e2.cols = b.dim;
        e2.out = w.g.p + (size_t)r0 * b.dim;
        e2.ldo = b.dim;
        e2.a_krep = b.nsplit == 3 ? b.Mpad : 0;
        TGB_TRY(launch_gemm_tn(w.tmA2, b.tmB2, nr, b.dim, b.K2, e2, err, st, nullptr, b.last2()));
        TGB_MARK(log, PASS_GEMM2, st);
    }
    ForceIn I{w.g.p,     w.q.p,      w.pnorm.p,         w.c.p,   w.epart.p,
              w.kdsum.p, b.n_etiles, b.delta * b.delta, w.qoff.p};
    ForceOut FO{forces, energies, w.vpart.p, err, atom_struct, vir_struct, pair_grad};
    int nblk = 0;
    TGB_TRY(force_pass(b, w, P, S, I, FO, &nblk, st, w.tile_force));
    TGB_TRY(launch_virial_reduce(w.vpart.p, nblk, virial, st));
    TGB_MARK(log, PASS_FORCE, st);
    return TG_OK;
}

static unsigned grid_for(int64_t n, int tb = 256) { return (unsigned)((n + tb - 1) / tb); }

// The project's autotuner: with the run's own sites and lists in place, time
// every CTA tile of the descriptor and the force pass (one warm launch, then
// `reps` launches between CUDA events) and keep the fastest of each. The tiles
// change only how central sites are grouped into CTAs and the register budget,
// so descriptor values do not depend on the choice; the extra force launches
// add into forces, energies and the virial partials, which every evaluation
// clears before it starts. TGB_AUTOTUNE=0 keeps the default tiles; TGB_SOAP_TILE
// pins one.
bool autotune_enabled() {
    const char *e = std::getenv("TGB_AUTOTUNE");
    return !(e && e[0] == '0') && !std::getenv("TGB_SOAP_TILE");
}

// TGB_SOAP_TILE=t pins every block to tile t (0 .. kForceTiles - 1) instead of
// tuning; returns -1 when unset.
int pinned_tile() {
    const char *e = std::getenv("TGB_SOAP_TILE");
    if (!e) return -1;
    const int t = std::atoi(e);
    return t < 0 ? 0 : (t >= kForceTiles ? kForceTiles - 1 : t);
}

// A pinned tile for a block: the descriptor pass has tiles 0 .. kSoapTiles - 1,
// the force pass also the tensor-core tile where the block's shape allows it.
void pin_tiles(const Block &b, Workspace &w, int t) {
    w.tile_desc = std::min(t, kSoapTiles - 1);
    w.tile_force = (t == kForceTileMma && !soap_force_mma_supported(b.params(1))) ? 0 : t;
}

int autotune_block(Block &b, Workspace &w, const SiteArgs &S, int n_atoms, double *forces,
                   double *energies, double *virial, unsigned *err, cudaStream_t st, int reps = 3) {
    if (S.n_sites <= 0) return TG_OK;
    TGB_TRY(evaluate_block(b, w, S, n_atoms, forces, energies, virial, err, st));
    const SoapParams P = b.params(n_atoms);
    // the tiles apply to the expansion and force kernels (a compressed block's
    // expansion writes praw and its force kernel reads gfull)
    DescOut O{w.qsplit.p, w.q.p, w.qoff.p, w.pnorm.p, w.c.p, w.praw.p};
    ForceIn I{b.compressed() ? w.gfull.p : w.g.p, w.q.p, w.pnorm.p, w.c.p, w.epart.p, w.kdsum.p,
              b.n_etiles, b.delta * b.delta, w.qoff.p};
    ForceOut FO{forces, energies, w.vpart.p, err};
    cudaEvent_t e0, e1;
    TGB_CUDA(cudaEventCreate(&e0));
    TGB_CUDA(cudaEventCreate(&e1));
    auto time_tile = [&](bool force, int t, float &ms) -> int {
        int nblk = 0;
        for (int r = 0; r <= reps; ++r) {
            if (r == 1) TGB_CUDA(cudaEventRecord(e0, st));
            if (force) TGB_TRY(launch_soap_force(P, S, I, FO, &nblk, st, t));
            else TGB_TRY(launch_soap_expand(P, S, O, st, t));
        }
        TGB_CUDA(cudaEventRecord(e1, st));
        TGB_CUDA(cudaEventSynchronize(e1));
        TGB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return TG_OK;
    };
    int rc = TG_OK;
    for (int pass = 0; pass < 2 && rc == TG_OK; ++pass) {
        float best = 0.f;
        int arg = 0;
        const int n_tiles = pass == 1 ? kForceTiles : kSoapTiles;
        for (int t = 0; t < n_tiles && rc == TG_OK; ++t) {
            if (pass == 1 && t == kForceTileMma && !soap_force_mma_supported(P)) continue;
            float ms = 0.f;
            rc = time_tile(pass == 1, t, ms);
            if (rc == TG_OK && (t == 0 || ms < best)) {
                best = ms;
                arg = t;
            }
        }
        if (pass == 0) w.tile_desc = arg;
        else w.tile_force = arg;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// ---------------------------------------------------------------- mixed form
// Sites whose ensemble spread exceeds the gate go back to the exact GAP kernel:
// they are compacted on the device and the two GEMMs run over the compacted
// rows, their count read on the device (the step stays one CUDA graph).

// one thread per site: MLP sites get epart = E / delta^2 and kdsum = 0 (their g
// rows already hold dE/dq - g0, so that the force pass's g0 + g is the MLP's
// dE/dq); gated sites are appended to gidx
// One thread per (row, energy tile), so the stores of consecutive threads are
// consecutive; the thread of tile 0 also gates its row.
__global__ void k_mlp_mix(int n, int n_et, const double *__restrict__ emean,
                          const double *__restrict__ estd, double gate, double inv_delta2,
                          double *__restrict__ epart, double *__restrict__ kdsum,
                          int *__restrict__ gidx, int *__restrict__ gcount) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n_et) return;
    const int row = (int)(e / n_et), t = (int)(e - (size_t)row * n_et);
    const bool gated = !(estd[row] <= gate);   // a NaN spread is gated too
    if (gated && t == 0) gidx[atomicAdd(gcount, 1)] = row;
    epart[e] = (!gated && t == 0) ? emean[row] * inv_delta2 : 0.0;
    kdsum[e] = 0.0;
}

// compacted GEMM-1 operand rows of the gated sites and their delta.mu. The mixed
// form's descriptor writes only its network's bf16 input, so the rows are split
// here from the fp32 delta rows, exactly as the descriptor splits them.
__global__ void k_gather_gated(const int *__restrict__ gcount, const int *__restrict__ gidx, int D,
                               int K1, int nsplit, const float *__restrict__ q,
                               const double *__restrict__ qoff, __nv_bfloat16 *__restrict__ Qg,
                               double *__restrict__ qoff_g) {
    const int cnt = *gcount;
    for (int r = blockIdx.x; r < cnt; r += gridDim.x) {
        const int site = gidx[r];
        const float *src = q + (size_t)site * D;
        __nv_bfloat16 *dst = Qg + (size_t)r * K1;
        for (int d = threadIdx.x; d < D; d += blockDim.x) {
            __nv_bfloat16 hi, lo;
            bf16_split(src[d], hi, lo);
            dst[d] = hi;
            if (nsplit == 3) {
                dst[D + d] = hi;
                dst[2 * D + d] = lo;
            }
        }
        for (int k = nsplit * D + threadIdx.x; k < K1; k += blockDim.x)
            dst[k] = __float2bfloat16_rn(0.f);
        if (threadIdx.x == 0) qoff_g[r] = qoff[site];
    }
}

__global__ void k_scatter_gated(const int *__restrict__ gcount, const int *__restrict__ gidx, int D,
                                int n_et, const double *__restrict__ epart_g,
                                const double *__restrict__ kdsum_g, const float *__restrict__ g_g,
                                double *__restrict__ epart, double *__restrict__ kdsum,
                                float *__restrict__ g) {
    const int cnt = *gcount;
    for (int r = blockIdx.x; r < cnt; r += gridDim.x) {
        const int site = gidx[r];
        for (int d = threadIdx.x; d < D; d += blockDim.x)
            g[(size_t)site * D + d] = g_g[(size_t)r * D + d];
        for (int t = threadIdx.x; t < n_et; t += blockDim.x) {
            epart[(size_t)site * n_et + t] = epart_g[(size_t)r * n_et + t];
            kdsum[(size_t)site * n_et + t] = kdsum_g[(size_t)r * n_et + t];
        }
    }
}

// training triples of a block after an exact evaluation: E = delta^2 sum epart,
// dE/dq = (sum kdsum) mu + g0 + g (one warp per site)
__global__ void k_collect(int n, int D, int n_et, double delta2, const double *__restrict__ epart,
                          const double *__restrict__ kdsum, const double *__restrict__ mu,
                          const double *__restrict__ g0, const float *__restrict__ g,
                          double *__restrict__ E, float *__restrict__ G) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    double ks = 0.0, e = 0.0;
    for (int t = 0; t < n_et; ++t) {
        ks += kdsum[(size_t)row * n_et + t];
        e += epart[(size_t)row * n_et + t];
    }
    for (int d = lane; d < D; d += 32)
        G[(size_t)row * D + d] = (float)(ks * mu[d] + g0[d] + (double)g[(size_t)row * D + d]);
    if (lane == 0) E[row] = delta2 * e;
}

// gated rows of each GEMM row chunk: min(R, max(0, count - c R))
__global__ void k_chunk_counts(const int *__restrict__ gcount, int R, int nch,
                               int *__restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    out[c] = max(0, min(R, *gcount - c * R));
}

struct MixedRun {
    Mlp *mlp = nullptr;
    MlpInferWork *iw = nullptr;   // this block's inference buffers
    double gate = 0.0;
    int cap = 0;
    DBuf<__nv_bfloat16> Qg;
    DBuf<double> qoff_g, epart_g, kdsum_g, emean, estd;
    DBuf<float> g_g;
    DBuf<int> gidx, gcount, chunk_cnt;
    TmaMap tmQg{};

    int ensure(const Block &b, int n_sites) {
        const int n = n_sites > 0 ? n_sites : 1;
        if (n <= cap) return TG_OK;
        TGB_TRY(Qg.ensure((size_t)n * b.K1));
        TGB_TRY(qoff_g.ensure(n));
        TGB_TRY(epart_g.ensure((size_t)n * b.n_etiles));
        TGB_TRY(kdsum_g.ensure((size_t)n * b.n_etiles));
        TGB_TRY(emean.ensure(n));
        TGB_TRY(estd.ensure(n));
        TGB_TRY(g_g.ensure((size_t)n * b.dim));
        TGB_TRY(gidx.ensure(n));
        TGB_TRY(gcount.ensure(1));
        TGB_TRY(chunk_cnt.ensure((size_t)(n + kGemmBM - 1) / kGemmBM));
        TGB_TRY(make_tma_bf16(&tmQg, Qg.p, n, b.K1, b.K1, kGemmBM));
        cap = n;
        return TG_OK;
    }
    ~MixedRun() { mlp_infer_work_delete(iw); }
};

// Descriptor, MLP ensemble, gate; exact GAP for the gated sites; forces.
int evaluate_block_mixed(Block &b, Workspace &w, MixedRun &x, const SiteArgs &S, int n_atoms,
                         double *forces, double *energies, double *virial, unsigned *err,
                         cudaStream_t st, EventLog *log = nullptr) {
    const int n = S.n_sites;
    if (n <= 0) return TG_OK;
    TGB_TRY(w.ensure(b, n));
    TGB_TRY(x.ensure(b, n));
    TGB_CHECK(x.mlp->L.D == b.dim, TG_ERR_ARG, "MLP input size %d does not match block dim %d",
              x.mlp->L.D, b.dim);
    // the descriptor writes the network's input only: the bf16 row of delta,
    // zero-padded to the network's input length (the gated rows are split below)
    TGB_CHECK(x.mlp->L.Dp <= b.K1, TG_ERR_ARG, "MLP input length %d exceeds the row length %d",
              x.mlp->L.Dp, b.K1);
    SoapParams P = b.params(n_atoms);
    P.nsplit = 1;
    P.fill_to = x.mlp->L.Dp;
    TGB_TRY(descriptor_pass(b, w, P, S, st, w.tile_desc));
    TGB_MARK(log, PASS_DESC, st);
    TGB_TRY(mlp_infer(*x.mlp, *x.iw, n, w.qsplit.p, b.K1, x.emean.p, x.estd.p, w.g.p, b.dim,
                      b.g0f.p, st));
    TGB_CUDA(cudaMemsetAsync(x.gcount.p, 0, sizeof(int), st));
    k_mlp_mix<<<grid_for((int64_t)n * b.n_etiles), 256, 0, st>>>(
        n, b.n_etiles, x.emean.p, x.estd.p, x.gate, 1.0 / (b.delta * b.delta), w.epart.p, w.kdsum.p,
        x.gidx.p, x.gcount.p);
    const unsigned gg = (unsigned)std::min(n, 1184);   // grid-stride over the gated rows
    k_gather_gated<<<gg, 128, 0, st>>>(x.gcount.p, x.gidx.p, b.dim, b.K1, b.nsplit, w.q.p,
                                      w.qoff.p, x.Qg.p, x.qoff_g.p);
    TGB_CUDA(cudaGetLastError());
    TGB_MARK(log, PASS_MLP, st);
    // both GEMMs over the compacted gated rows in chunks of w.kd_rows, each chunk's
    // row count taken on the device from the gated count
    const int R = w.kd_rows, nch = (n + R - 1) / R;
    k_chunk_counts<<<grid_for(nch), 256, 0, st>>>(x.gcount.p, R, nch, x.chunk_cnt.p);
    TGB_CUDA(cudaGetLastError());
    for (int c = 0; c < nch; ++c) {
        const int r0 = c * R, nr = std::min(R, n - r0);
        TmaMap a1c;
        const TmaMap *a1 = &x.tmQg;
        if (nr < n) {
            TGB_TRY(make_tma_bf16(&a1c, x.Qg.p + (size_t)r0 * b.K1, nr, b.K1, b.K1, kGemmBM));
            a1 = &a1c;
        }
        GemmEpi e1 = gap_epilogue(b, w);
        e1.rows = nr;
        e1.rows_dev = x.chunk_cnt.p + c;
        e1.epart = x.epart_g.p + (size_t)r0 * b.n_etiles;
        e1.kdsum = x.kdsum_g.p + (size_t)r0 * b.n_etiles;
        e1.qoff = x.qoff_g.p + r0;
        TGB_TRY(launch_gemm_tn(*a1, b.tmB1, nr, b.Mpad, b.K1, e1, err, st, &w.tmKd, b.last1()));
        TGB_MARK(log, PASS_GEMM1, st);
        GemmEpi e2{};
        e2.mode = EPI_STORE_F32;
        e2.rows = nr;
        e2.rows_dev = x.chunk_cnt.p + c;
        e2.cols = b.dim;
        e2.out = x.g_g.p + (size_t)r0 * b.dim;
        e2.ldo = b.dim;
        e2.a_krep = b.nsplit == 3 ? b.Mpad : 0;
        TGB_TRY(launch_gemm_tn(w.tmA2, b.tmB2, nr, b.dim, b.K2, e2, err, st, nullptr, b.last2()));
        TGB_MARK(log, PASS_GEMM2, st);
    }
    k_scatter_gated<<<gg, 128, 0, st>>>(x.gcount.p, x.gidx.p, b.dim, b.n_etiles, x.epart_g.p,
                                       x.kdsum_g.p, x.g_g.p, w.epart.p, w.kdsum.p, w.g.p);
    TGB_CUDA(cudaGetLastError());
    TGB_MARK(log, PASS_GEMM2, st);
    ForceIn I{w.g.p,     w.q.p,      w.pnorm.p,         w.c.p,   w.epart.p,
              w.kdsum.p, b.n_etiles, b.delta * b.delta, w.qoff.p};
    ForceOut FO{forces, energies, w.vpart.p, err};
    int nblk = 0;
    TGB_TRY(force_pass(b, w, P, S, I, FO, &nblk, st, w.tile_force));
    TGB_TRY(launch_virial_reduce(w.vpart.p, nblk, virial, st));
    TGB_MARK(log, PASS_FORCE, st);
    return TG_OK;
}

// ---------------------------------------------------------------- context
struct Engine;

struct Context {
    int device = -1;
    cudaStream_t st = nullptr;
    std::map<int, std::unique_ptr<Block>> blocks;
    // blocks replaced under their key by a begin of another shape: engines made
    // before the replacement still point at them, so they live until finalize
    std::vector<std::unique_ptr<Block>> retired;
    std::map<int, std::unique_ptr<Family>> families;   // 2b / 3b / core_pot, same key space
    std::map<int, std::unique_ptr<Workspace>> ws;
    Block *current = nullptr;
    DBuf<unsigned> err;
    // staging of the get_gap_soap path
    DBuf<int> nn, nl, nbr, spb, spa, flag, site_row, site_atom, seen, cnt;
    DBuf<int64_t> pstart;
    DBuf<double> rjs, xyz, en, fo, vir;
    DBuf<char> scan;
};

static Context *g_ctx = nullptr;

static int need_ctx() {
    TGB_CHECK(g_ctx != nullptr, TG_ERR_STATE, "tg_context_init has not been called");
    return TG_OK;
}

static int check_err_word(Context &c, unsigned *err_dev) {
    unsigned e = 0;
    TGB_CUDA(cudaMemcpyAsync(&e, err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c.st));
    TGB_CUDA(cudaStreamSynchronize(c.st));
    if (e) {
        TGB_CUDA(cudaMemsetAsync(err_dev, 0, sizeof(unsigned), c.st));
        if (e & (DEV_ERR_TIMEOUT_TMA | DEV_ERR_TIMEOUT_MMA | DEV_ERR_TIMEOUT_EPI)) {
            set_error("device wait timed out (error word 0x%x)", e);
            return TG_ERR_TIMEOUT;
        }
        set_error("device error word 0x%x%s", e,
                  (e & DEV_ERR_NEIGH_CAPACITY) ? " (neighbour pair capacity exceeded)" : "");
        return TG_ERR_DEVICE;
    }
    return TG_OK;
}

}  // namespace tgb

using namespace tgb;

// ============================================================== C-ABI
extern "C" {

const char *tg_last_error(void) { return tgb::last_error(); }

int tg_context_init(int32_t rank, int32_t device, int32_t *n_omp) {
    if (n_omp) *n_omp = 1;
    if (g_ctx) return TG_OK;
    int ndev = 0;
    TGB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 && ndev > 0) device = (rank < 0 ? 0 : rank) % ndev;   // one rank per GPU
    TGB_CHECK(device >= 0 && device < ndev, TG_ERR_ARG, "device %d not present (%d devices)", device,
              ndev);
    TGB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    TGB_CUDA(cudaGetDeviceProperties(&prop, device));
    TGB_CHECK(prop.major == 10 && prop.minor == 0, TG_ERR_ARG,
              "this backend is built for sm_100a (B200); device %d is sm_%d%d", device, prop.major,
              prop.minor);
    auto *c = new Context();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        set_error("cudaStreamCreate failed");
        return TG_ERR_CUDA;
    }
    int r = init_soap_constants();
    if (r == TG_OK) r = c->err.ensure(1);
    if (r == TG_OK && cudaMemset(c->err.p, 0, sizeof(unsigned)) != cudaSuccess) r = TG_ERR_CUDA;
    if (r != TG_OK) {
        cudaStreamDestroy(c->st);
        delete c;
        return r;
    }
    g_ctx = c;
    return TG_OK;
}

int tg_context_finalize(void) {
    if (!g_ctx) return TG_OK;
    cudaStreamSynchronize(g_ctx->st);
    cudaStream_t st = g_ctx->st;
    delete g_ctx;
    g_ctx = nullptr;
    cudaStreamDestroy(st);
    return TG_OK;
}

int tg_memory_budget(double *max_gbytes) {
    TGB_TRY(need_ctx());
    size_t fr = 0, tot = 0;
    TGB_CUDA(cudaMemGetInfo(&fr, &tot));
    // Batches are a host-memory device in the reference; on the device the whole
    // step is resident, so the budget is what is free, less a 10 % reserve.
    if (max_gbytes) *max_gbytes = 0.9 * (double)fr / (1024.0 * 1024.0 * 1024.0);
    return TG_OK;
}

// Whether a cached block can stand for a begin with these arguments: the same
// sparse-set size, precision and descriptor shape (species, alpha_max, l_max,
// compression), so that every buffer a caller sizes from the hypers matches.
static bool same_shape(const Block &b, const tg_soap_hypers &h, int n_sparse, int precision) {
    if (b.M != n_sparse || b.precision != precision || b.hh.ns != h.n_species ||
        b.hh.lmax != h.l_max || b.hh.central_species != h.central_species)
        return false;
    for (int s = 0; s < b.hh.ns; ++s)
        if (b.hh.alpha_max[s] != h.alpha_max[s] || b.hh.species_z[s] != h.species_z[s]) return false;
    const int dimc = h.compress_P_nonzero > 0 ? h.dim : 0;
    return b.dimc == dimc && (dimc == 0 || b.c_row_col.n == (size_t)h.compress_P_nonzero);
}

// The compression matrix of a block as two CSR copies on the device: by
// compressed row (forward pass) and by internal power-spectrum column (adjoint).
// Entries keep the caller's order within a row or column.
static int upload_compression(Block &b, const tg_soap_hypers &h) {
    std::vector<int> inv(b.dimf);
    for (int d = 0; d < b.dimf; ++d) inv[descriptor_ref_index(d, b.ntot, b.lmax + 1)] = d;
    const int nz = h.compress_P_nonzero;
    std::vector<int> rp(b.dim + 1, 0), cp(b.dimf + 1, 0), rc(nz), cr(nz);
    std::vector<double> rv(nz), cv(nz);
    for (int k = 0; k < nz; ++k) {
        ++rp[h.compress_P_i[k]];
        ++cp[inv[h.compress_P_j[k] - 1] + 1];
    }
    for (int i = 0; i < b.dim; ++i) rp[i + 1] += rp[i];
    for (int j = 0; j < b.dimf; ++j) cp[j + 1] += cp[j];
    std::vector<int> rf(rp.begin(), rp.end() - 1), cf(cp.begin(), cp.end() - 1);
    for (int k = 0; k < nz; ++k) {
        const int i = h.compress_P_i[k] - 1, j = inv[h.compress_P_j[k] - 1];
        rc[rf[i]] = j;
        rv[rf[i]++] = h.compress_P_el[k];
        cr[cf[j]] = i;
        cv[cf[j]++] = h.compress_P_el[k];
    }
    // the adjoint walks only the columns that have entries
    std::vector<int> cidx, cptr(1, 0);
    for (int j = 0; j < b.dimf; ++j)
        if (cp[j + 1] > cp[j]) {
            cidx.push_back(j);
            cptr.push_back(cp[j + 1]);
        }
    b.c_ncols = (int)cidx.size();
    TGB_TRY(b.c_row_ptr.ensure(b.dim + 1));
    TGB_TRY(b.c_col_idx.ensure(b.c_ncols));
    TGB_TRY(b.c_col_ptr.ensure(b.c_ncols + 1));
    TGB_TRY(b.c_row_col.ensure(nz));
    TGB_TRY(b.c_col_row.ensure(nz));
    TGB_TRY(b.c_row_val.ensure(nz));
    TGB_TRY(b.c_col_val.ensure(nz));
    TGB_CUDA(cudaMemcpy(b.c_row_ptr.p, rp.data(), sizeof(int) * rp.size(), cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemcpy(b.c_col_idx.p, cidx.data(), sizeof(int) * cidx.size(), cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemcpy(b.c_col_ptr.p, cptr.data(), sizeof(int) * cptr.size(), cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemcpy(b.c_row_col.p, rc.data(), sizeof(int) * nz, cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemcpy(b.c_col_row.p, cr.data(), sizeof(int) * nz, cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemcpy(b.c_row_val.p, rv.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    TGB_CUDA(cudaMemcpy(b.c_col_val.p, cv.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    return TG_OK;
}

int tg_soap_begin(int32_t block_key, const tg_soap_hypers *h, int32_t n_sparse, const double *Qs,
                  const double *alphas, double delta, double zeta, int32_t precision) {
    NvtxRange nvtx_range("tg_soap_begin");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(!C.families.count(block_key), TG_ERR_ARG, "key %d already names a 2b/3b/core_pot family",
              block_key);
    TGB_CHECK(h && Qs && alphas, TG_ERR_ARG, "null hypers/Qs/alphas");
    auto it = C.blocks.find(block_key);
    if (it != C.blocks.end() && same_shape(*it->second, *h, n_sparse, precision)) {
        C.current = it->second.get();
        return TG_OK;
    }
    TGB_CHECK(h->n_species >= 1 && h->n_species <= kMaxSpecies, TG_ERR_ARG,
              "n_species %d outside 1..%d", h->n_species, kMaxSpecies);
    TGB_CHECK(precision == TG_PREC_BF16X3 || precision == TG_PREC_BF16, TG_ERR_ARG,
              "precision must be TG_PREC_BF16X3 or TG_PREC_BF16");
    TGB_CHECK(n_sparse >= 1, TG_ERR_ARG, "n_sparse must be positive");
    auto b = std::make_unique<Block>();
    b->key = block_key;
    b->precision = precision;
    SoapHostHypers &hh = b->hh;
    hh.ns = h->n_species;
    hh.lmax = h->l_max;
    hh.radial_enhancement = h->radial_enhancement;
    hh.central_species = h->central_species;
    TGB_CHECK(hh.radial_enhancement >= 0 && hh.radial_enhancement <= 2, TG_ERR_ARG,
              "radial_enhancement must be 0..2");
    TGB_CHECK(hh.central_species >= 0 && hh.central_species <= hh.ns, TG_ERR_ARG,
              "central_species out of range");
    for (int s = 0; s < hh.ns; ++s) {
        hh.alpha_max[s] = h->alpha_max[s];
        hh.species_z[s] = h->species_z[s];
        hh.rcut_hard[s] = h->rcut_hard[s];
        hh.rcut_soft[s] = h->rcut_soft[s];
        hh.nf[s] = h->nf[s];
        hh.global_scaling[s] = h->global_scaling[s];
        hh.sigma_r[s] = h->atom_sigma_r[s];
        hh.sigma_r_scaling[s] = h->atom_sigma_r_scaling[s];
        hh.sigma_t[s] = h->atom_sigma_t[s];
        hh.sigma_t_scaling[s] = h->atom_sigma_t_scaling[s];
        hh.amplitude_scaling[s] = h->amplitude_scaling[s];
        hh.central_weight[s] = h->central_weight[s];
        TGB_CHECK(hh.alpha_max[s] == hh.alpha_max[0], TG_ERR_ARG,
                  "the device path needs the same alpha_max for every species");
        TGB_CHECK(hh.species_z[s] >= 1 && hh.species_z[s] < kMaxZ, TG_ERR_ARG,
                  "species id %d outside 1..%d", hh.species_z[s], kMaxZ - 1);
        TGB_CHECK(hh.rcut_hard[s] > 0.0 && hh.sigma_r[s] > 0.0 && hh.sigma_t[s] > 0.0, TG_ERR_ARG,
                  "rcut and atom sigmas must be positive");
    }
    b->ns = hh.ns;
    b->amax = hh.alpha_max[0];
    b->lmax = hh.lmax;
    TGB_CHECK(soap_shape_supported(b->ns, b->amax, b->lmax), TG_ERR_ARG,
              "unsupported SOAP shape: n_species %d alpha_max %d l_max %d", b->ns, b->amax, b->lmax);
    b->ntot = b->ns * b->amax;
    b->nlm = (b->lmax + 1) * (b->lmax + 1);
    b->dimf = b->ntot * (b->ntot + 1) / 2 * (b->lmax + 1);
    b->dimc = 0;
    b->dim = b->dimf;
    if (h->compress_P_nonzero > 0) {
        // read_files.f90:5166-5231: q_c(i) = sum P_el p(P_j) over P_i = i (1-based)
        TGB_CHECK(h->compress_P_i && h->compress_P_j && h->compress_P_el, TG_ERR_ARG,
                  "compression entries are null");
        TGB_CHECK(h->dim >= 1 && h->dim <= kMaxCompressedDim, TG_ERR_ARG,
                  "compressed dim %d outside 1..%d", h->dim, kMaxCompressedDim);
        for (int k = 0; k < h->compress_P_nonzero; ++k)
            TGB_CHECK(h->compress_P_i[k] >= 1 && h->compress_P_i[k] <= h->dim &&
                          h->compress_P_j[k] >= 1 && h->compress_P_j[k] <= b->dimf,
                      TG_ERR_ARG, "compression entry %d (%d, %d) outside %d x %d", k + 1,
                      h->compress_P_i[k], h->compress_P_j[k], h->dim, b->dimf);
        b->dimc = h->dim;
        b->dim = round_up(h->dim, 8);
    }
    b->nsplit = precision == TG_PREC_BF16X3 ? 3 : 1;
    b->M = n_sparse;
    b->Mpad = round_up(n_sparse, 64);
    b->K1 = round_up(b->nsplit * b->dim, kGemmBK);
    b->K2 = b->nsplit * b->Mpad;
    b->KD = (b->nsplit == 3 ? 2 : 1) * b->Mpad;
    b->n_etiles = gemm_n_etiles(b->Mpad);
    b->tw = table_width(b->amax, b->lmax);
    b->delta = delta;
    b->rcut_max = 0.0;
    for (int s = 0; s < hh.ns; ++s) b->rcut_max = std::max(b->rcut_max, hh.rcut_hard[s]);
    // gap.f90:115-121: zeta within 1e-5 of an integer is snapped to it
    if (std::fabs(zeta - (double)(int)zeta) < 1.e-5 && (int)zeta >= 1) {
        b->zeta_int = (int)zeta;
        b->zeta = (double)b->zeta_int;
    } else {
        b->zeta_int = 0;
        b->zeta = zeta;
    }
    // species multiplicity (gap_interface.f90:180-199): a global species listed
    // twice feeds both descriptor species, each with its own hypers. The device
    // shapes have at most two species, so two matches is the most there can be.
    for (int z = 0; z < kMaxZ; ++z) b->zmap[z] = b->zmap2[z] = -1;
    b->n_inst = 1;
    for (int s = 0; s < hh.ns; ++s) {
        const int z = hh.species_z[s];
        if (b->zmap[z] < 0) {
            b->zmap[z] = (signed char)s;
        } else {
            TGB_CHECK(b->zmap2[z] < 0, TG_ERR_ARG, "species %d listed more than twice in one block", z);
            b->zmap2[z] = (signed char)s;
            b->n_inst = 2;
        }
    }
    TGB_TRY(b->table.ensure((size_t)hh.ns * (kTableIntervals + 1) * b->tw));
    TGB_TRY(b->selfR.ensure((size_t)hh.ns * b->amax));
    TGB_TRY(b->QsA.ensure((size_t)b->Mpad * b->K1));
    TGB_TRY(b->QsT.ensure((size_t)b->dim * b->K2));
    TGB_TRY(b->alpha.ensure(b->Mpad));
    TGB_TRY(b->mu.ensure(b->dim));
    TGB_TRY(b->aoff.ensure(b->Mpad));
    TGB_TRY(b->g0.ensure(b->dim));
    TGB_TRY(b->ref_index.ensure(b->dim));
    // The device keeps power-spectrum entries in its internal order (l-major);
    // the sparse set is permuted into that order once here. A compressed block's
    // entries stay in the transformation's order, padded with zeros to dim, and
    // the transformation's columns are permuted instead.
    std::vector<int> ref(b->dim);
    const int qdim = b->compressed() ? b->dimc : b->dim;   // rows of the caller's Qs
    if (b->compressed()) {
        for (int d = 0; d < b->dim; ++d) ref[d] = d < b->dimc ? d : -1;
        TGB_TRY(upload_compression(*b, *h));
    } else {
        for (int d = 0; d < b->dim; ++d) ref[d] = descriptor_ref_index(d, b->ntot, b->lmax + 1);
    }
    std::vector<double> Qi((size_t)n_sparse * b->dim, 0.0);
    for (int s = 0; s < n_sparse; ++s)
        for (int d = 0; d < b->dim; ++d)
            if (ref[d] >= 0) Qi[(size_t)s * b->dim + d] = Qs[(size_t)s * qdim + ref[d]];
    Qs = Qi.data();
    TGB_CUDA(cudaMemcpy(b->ref_index.p, ref.data(), sizeof(int) * b->dim, cudaMemcpyHostToDevice));
    // Centre of the sparse set (FP64): the GEMMs run on q - mu and q_s - mu, the
    // exact rank-1 terms mu.q_s and (q - mu).mu are added in the epilogue.
    {
        std::vector<double> mu(b->dim, 0.0), aoff(b->Mpad, 0.0);
        for (int s = 0; s < n_sparse; ++s)
            for (int d = 0; d < b->dim; ++d) mu[d] += Qs[(size_t)s * b->dim + d];
        for (int d = 0; d < b->dim; ++d) mu[d] /= (double)n_sparse;
        for (int s = 0; s < n_sparse; ++s) {
            double a = 0.0;
            for (int d = 0; d < b->dim; ++d) a += mu[d] * Qs[(size_t)s * b->dim + d];
            aoff[s] = a;
        }
        // g0 = sum_s zeta delta^2 alpha_s (q_s - mu): dE/dq of an atom with K = 1 to
        // every sparse point; GEMM 2 only carries the deviation from it.
        std::vector<double> g0(b->dim, 0.0);
        const double zd2 = b->zeta * delta * delta;
        for (int s = 0; s < n_sparse; ++s) {
            const double c = zd2 * alphas[s];
            for (int d = 0; d < b->dim; ++d) g0[d] += c * (Qs[(size_t)s * b->dim + d] - mu[d]);
        }
        TGB_CUDA(cudaMemcpy(b->g0.p, g0.data(), sizeof(double) * b->dim, cudaMemcpyHostToDevice));
        std::vector<float> g0f(g0.begin(), g0.end()), muf(mu.begin(), mu.end());
        TGB_TRY(b->g0f.ensure(b->dim));
        TGB_TRY(b->muf.ensure(b->dim));
        TGB_CUDA(cudaMemcpy(b->g0f.p, g0f.data(), sizeof(float) * b->dim, cudaMemcpyHostToDevice));
        TGB_CUDA(cudaMemcpy(b->muf.p, muf.data(), sizeof(float) * b->dim, cudaMemcpyHostToDevice));
        b->mu2 = 0.0;
        b->g0mu = 0.0;
        for (int d = 0; d < b->dim; ++d) {
            b->mu2 += mu[d] * mu[d];
            b->g0mu += g0[d] * mu[d];
        }
        TGB_CUDA(cudaMemcpy(b->mu.p, mu.data(), sizeof(double) * b->dim, cudaMemcpyHostToDevice));
        TGB_CUDA(cudaMemcpy(b->aoff.p, aoff.data(), sizeof(double) * b->Mpad, cudaMemcpyHostToDevice));
    }
    DBuf<double> tq, ta;
    TGB_TRY(tq.ensure((size_t)n_sparse * b->dim));
    TGB_TRY(ta.ensure(n_sparse));
    TGB_CUDA(cudaMemcpyAsync(tq.p, Qs, sizeof(double) * n_sparse * b->dim, cudaMemcpyHostToDevice, C.st));
    TGB_CUDA(cudaMemcpyAsync(ta.p, alphas, sizeof(double) * n_sparse, cudaMemcpyHostToDevice, C.st));
    const int64_t tot = (int64_t)b->Mpad * b->K1 + (int64_t)b->dim * b->K2;
    k_prep_sparse<<<(unsigned)((tot + 255) / 256), 256, 0, C.st>>>(tq.p, b->mu.p, b->M, b->Mpad,
                                                                   b->dim, b->K1, b->K2, b->nsplit,
                                                                   b->QsA.p, b->QsT.p);
    k_prep_alpha<<<(b->Mpad + 255) / 256, 256, 0, C.st>>>(ta.p, b->M, b->Mpad, b->alpha.p);
    TGB_CUDA(cudaGetLastError());
    TGB_TRY(b->table_fd.ensure((size_t)hh.ns * (b->amax + b->lmax + 1) * kTableIntervals));
    TGB_TRY(build_soap_tables(hh, b->table.p, b->selfR.p, C.st, b->table_fd.p));
    TGB_TRY(make_tma_bf16(&b->tmB1, b->QsA.p, b->Mpad, b->K1, b->K1, kGemmBN));
    TGB_TRY(make_tma_bf16(&b->tmB2, b->QsT.p, b->dim, b->K2, b->K2, kGemmBN));
    if (b->last1())
        TGB_TRY(make_tma_bf16(&b->tmB1l, b->QsA.p, b->Mpad, b->K1, b->K1,
                              gemm_last_box_rows(b->Mpad)));
    if (b->last2())
        TGB_TRY(make_tma_bf16(&b->tmB2l, b->QsT.p, b->dim, b->K2, b->K2,
                              gemm_last_box_rows(b->dim)));
    TGB_CUDA(cudaStreamSynchronize(C.st));
    C.current = b.get();
    auto old = C.blocks.find(block_key);
    if (old != C.blocks.end()) C.retired.push_back(std::move(old->second));
    C.blocks[block_key] = std::move(b);
    return TG_OK;
}

int tg_soap_end(void) {
    TGB_TRY(need_ctx());
    g_ctx->current = nullptr;
    return TG_OK;
}

}  // extern "C"

namespace tgb {
namespace {

__global__ void k_central_flags(int n, const int *__restrict__ spb, const signed char *zfirst,
                                int cs, int *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int z = spb[i];
    int first = (z >= 0 && z < kMaxZ) ? zfirst[z] + 1 : 0;   // 1-based, 0 if absent
    flag[i] = (cs == 0 || first == cs) ? 1 : 0;
}

__global__ void k_sites(int n, const int *__restrict__ flag, const int *__restrict__ incl,
                        const int64_t *__restrict__ pstart, const int *__restrict__ nl1,
                        int n_total, int *__restrict__ site_row, int *__restrict__ site_atom) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int idx = incl[i] - 1;
    site_row[idx] = i;
    site_atom[idx] = (nl1[pstart[i]] - 1) % n_total;
}

__global__ void k_to0(int64_t P, const int *__restrict__ nl1, int *__restrict__ nbr) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < P) nbr[p] = nl1[p] - 1;
}

// Atoms a block "sees" (gap_interface.f90:204-232): kept pairs of central sites.
__global__ void k_seen(int n_sites, const int *__restrict__ site_row, const int64_t *__restrict__ pstart,
                       const int *__restrict__ nbr, const double *__restrict__ rjs,
                       const int *__restrict__ spa, const signed char *zfirst, double rcut_max,
                       int n_total, int *__restrict__ seen) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sites) return;
    const int row = site_row[i];
    for (int64_t p = pstart[row]; p < pstart[row + 1]; ++p) {
        const int j = nbr[p] % n_total;
        const int z = spa[j];
        if (rjs[p] < rcut_max && z >= 0 && z < kMaxZ && zfirst[z] >= 0) seen[j] = 1;
    }
}

// q = mu + delta (rows of dim)
// q = mu + delta, written back in the reference order of the descriptor entries.
__global__ void k_d2f(int64_t n, int dim, int dim_out, const float *__restrict__ a,
                      const double *__restrict__ mu, const int *__restrict__ ref_index,
                      double *__restrict__ b) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t site = i / dim;
    const int d = (int)(i - site * dim);
    const int r = ref_index[d];
    if (r >= 0) b[site * dim_out + r] = mu[d] + (double)a[i];
}

__global__ void k_gather_species(int64_t P, const int *__restrict__ nbr, const int *__restrict__ sp,
                                 int *__restrict__ out) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < P) out[p] = sp[nbr[p]];
}

__global__ void k_is_self(int n, const int64_t *__restrict__ pstart, int *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && pstart[i + 1] > pstart[i]) flag[pstart[i]] = 1;
}

__global__ void k_add1(int64_t P, int *__restrict__ v) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < P) v[p] += 1;
}

// energies(i) = e0(species(i)) (turbogap.f90:1253-1261)
// e0 of the sites in [beg, end) (the sites this rank owns), zero elsewhere
__global__ void k_energy_e0(int n, const int *__restrict__ sp, const double *__restrict__ e0, int nz,
                            int beg, int end, double *__restrict__ en) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int z = sp[i];
    en[i] = (i >= beg && i < end && z >= 1 && z <= nz) ? e0[z - 1] : 0.0;
}

}  // namespace


// Shared front half of tg_get_gap_soap / tg_get_soap: uploads the batch and
// builds the central-site list (gap_interface.f90:178-309 semantics).
static int stage_batch(Context &C, Block &b, int n_total, int n_sites0, const int32_t *n_neigh0,
                       const int32_t *nl0, const double *rjs0, const double *xyz0,
                       const int32_t *spb, const int32_t *spa, int64_t *P_out, int *n_central,
                       DBuf<signed char> &zf) {
    int64_t P = 0;
    for (int i = 0; i < n_sites0; ++i) {
        TGB_CHECK(n_neigh0[i] >= 1, TG_ERR_ARG, "site %d has no self pair (n_neigh0 = %d)", i,
                  n_neigh0[i]);
        P += n_neigh0[i];
    }
    for (int64_t p = 0; p < P; ++p)
        TGB_CHECK(nl0[p] >= 1, TG_ERR_ARG, "neighbors_list0(%lld) = %d is not a 1-based index",
                  (long long)(p + 1), nl0[p]);
    *P_out = P;
    cudaStream_t st = C.st;
    TGB_TRY(C.nn.ensure(n_sites0));
    TGB_TRY(C.pstart.ensure((size_t)n_sites0 + 1));
    TGB_TRY(C.nl.ensure(P));
    TGB_TRY(C.nbr.ensure(P));
    TGB_TRY(C.rjs.ensure(P));
    TGB_TRY(C.xyz.ensure(3 * P));
    TGB_TRY(C.spb.ensure(n_sites0));
    TGB_TRY(C.spa.ensure(n_total));
    TGB_TRY(C.flag.ensure(n_sites0));
    TGB_TRY(C.cnt.ensure((size_t)n_sites0 + 1));
    TGB_TRY(C.site_row.ensure(n_sites0));
    TGB_TRY(C.site_atom.ensure(n_sites0));
    TGB_CUDA(cudaMemcpyAsync(C.nn.p, n_neigh0, sizeof(int) * n_sites0, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(C.nl.p, nl0, sizeof(int) * P, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(C.rjs.p, rjs0, sizeof(double) * P, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(C.xyz.p, xyz0, sizeof(double) * 3 * P, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(C.spb.p, spb, sizeof(int) * n_sites0, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(C.spa.p, spa, sizeof(int) * n_total, cudaMemcpyHostToDevice, st));
    signed char zfirst[kMaxZ];
    for (int z = 0; z < kMaxZ; ++z) zfirst[z] = b.zmap[z];
    TGB_TRY(zf.ensure(kMaxZ));
    TGB_CUDA(cudaMemcpyAsync(zf.p, zfirst, kMaxZ, cudaMemcpyHostToDevice, st));
    size_t need = 0;
    cub::DeviceScan::InclusiveSum(nullptr, need, C.nn.p, C.pstart.p + 1, n_sites0);
    size_t need2 = 0;
    cub::DeviceScan::InclusiveSum(nullptr, need2, C.flag.p, C.cnt.p, n_sites0);
    TGB_TRY(C.scan.ensure(std::max(need, need2)));
    TGB_CUDA(cudaMemsetAsync(C.pstart.p, 0, sizeof(int64_t), st));
    size_t bytes = C.scan.n;
    TGB_CUDA(cub::DeviceScan::InclusiveSum(C.scan.p, bytes, C.nn.p, C.pstart.p + 1, n_sites0, st));
    k_central_flags<<<grid_for(n_sites0), 256, 0, st>>>(n_sites0, C.spb.p, zf.p, b.hh.central_species,
                                                        C.flag.p);
    bytes = C.scan.n;
    TGB_CUDA(cub::DeviceScan::InclusiveSum(C.scan.p, bytes, C.flag.p, C.cnt.p, n_sites0, st));
    k_sites<<<grid_for(n_sites0), 256, 0, st>>>(n_sites0, C.flag.p, C.cnt.p, C.pstart.p, C.nl.p,
                                                n_total, C.site_row.p, C.site_atom.p);
    k_to0<<<grid_for(P), 256, 0, st>>>(P, C.nl.p, C.nbr.p);
    TGB_CUDA(cudaGetLastError());
    int nc = 0;
    TGB_CUDA(cudaMemcpyAsync(&nc, C.cnt.p + (n_sites0 - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    *n_central = nc;
    return TG_OK;
}

}  // namespace tgb

extern "C" {

int tg_get_gap_soap(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                    const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                    const int32_t *species_batch, const int32_t *species_all, double *energies0,
                    double *forces0, double *virial) {
    NvtxRange nvtx_range("tg_get_gap_soap");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(C.current, TG_ERR_STATE, "no block is open (call tg_soap_begin first)");
    TGB_CHECK(n_total_sites >= 1 && n_sites0 >= 0, TG_ERR_ARG, "bad site counts");
    if (virial)
        for (int q = 0; q < 9; ++q) virial[q] = 0.0;
    if (n_sites0 == 0) return TG_OK;
    Block &b = *C.current;
    DBuf<signed char> zf;
    int64_t P = 0;
    int nc = 0;
    TGB_TRY(stage_batch(C, b, n_total_sites, n_sites0, n_neigh0, neighbors_list0, rjs0, xyz0,
                        species_batch, species_all, &P, &nc, zf));
    cudaStream_t st = C.st;
    TGB_TRY(C.en.ensure(n_total_sites));
    TGB_TRY(C.fo.ensure(3 * (size_t)n_total_sites));
    TGB_TRY(C.vir.ensure(9));
    TGB_TRY(C.seen.ensure(n_total_sites));
    TGB_CUDA(cudaMemsetAsync(C.en.p, 0, sizeof(double) * n_total_sites, st));
    TGB_CUDA(cudaMemsetAsync(C.fo.p, 0, sizeof(double) * 3 * n_total_sites, st));
    TGB_CUDA(cudaMemsetAsync(C.vir.p, 0, sizeof(double) * 9, st));
    TGB_CUDA(cudaMemsetAsync(C.seen.p, 0, sizeof(int) * n_total_sites, st));
    auto &wp = C.ws[b.key];
    if (!wp) wp = std::make_unique<Workspace>();
    SiteArgs S{nc, C.site_row.p, C.site_atom.p, C.pstart.p, C.nbr.p, C.xyz.p, C.spa.p};
    TGB_TRY(evaluate_block(b, *wp, S, n_total_sites, C.fo.p, C.en.p, C.vir.p, C.err.p, st));
    k_seen<<<grid_for(nc), 256, 0, st>>>(nc, C.site_row.p, C.pstart.p, C.nbr.p, C.rjs.p, C.spa.p,
                                          zf.p, b.rcut_max, n_total_sites, C.seen.p);
    TGB_CUDA(cudaGetLastError());
    TGB_TRY(check_err_word(C, C.err.p));
    std::vector<double> en(n_total_sites), fo(3 * (size_t)n_total_sites), vr(9);
    std::vector<int> seen(n_total_sites), rows(nc), atoms(nc);
    TGB_CUDA(cudaMemcpyAsync(en.data(), C.en.p, sizeof(double) * n_total_sites, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(fo.data(), C.fo.p, sizeof(double) * 3 * n_total_sites, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(vr.data(), C.vir.p, sizeof(double) * 9, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(seen.data(), C.seen.p, sizeof(int) * n_total_sites, cudaMemcpyDeviceToHost, st));
    if (nc > 0)
        TGB_CUDA(cudaMemcpyAsync(atoms.data(), C.site_atom.p, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    // gap_interface.f90:422-431: assignment to the sites this block touched
    if (energies0)
        for (int i = 0; i < nc; ++i) energies0[atoms[i]] = en[atoms[i]];
    if (forces0)
        for (int j = 0; j < n_total_sites; ++j)
            if (seen[j])
                for (int q = 0; q < 3; ++q) forces0[3 * (size_t)j + q] = fo[3 * (size_t)j + q];
    if (virial)
        for (int q = 0; q < 9; ++q) virial[q] = vr[q];
    return TG_OK;
}

int tg_family_begin(int32_t key, const tg_family *family) {
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(family, TG_ERR_ARG, "null family");
    TGB_CHECK(!C.blocks.count(key), TG_ERR_ARG, "key %d already names a soap_turbo block", key);
    auto &slot = C.families[key];
    if (!slot) slot = std::make_unique<Family>();
    TGB_CUDA(cudaDeviceSynchronize());   // an engine may be using the old parameters
    const int rc = family_create(*family, *slot);
    if (rc != TG_OK) {
        C.families.erase(key);
        return rc;
    }
    slot->key = key;
    return TG_OK;
}

int tg_get_family(int32_t key, int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                  const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                  const int32_t *species_all, double *energies0, double *forces0, double *virial) {
    NvtxRange nvtx_range("tg_get_family");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    auto fi = C.families.find(key);
    TGB_CHECK(fi != C.families.end(), TG_ERR_STATE, "family key %d was never begun", key);
    TGB_CHECK(n_total_sites >= 1 && n_sites0 >= 0, TG_ERR_ARG, "bad site counts");
    if (n_sites0 == 0) return TG_OK;
    TGB_CHECK(n_neigh0 && neighbors_list0 && rjs0 && xyz0 && species_all, TG_ERR_ARG,
              "null neighbour arrays");
    // host: list offsets, 0-based neighbours and the site of each list (its self pair)
    std::vector<int64_t> ps(n_sites0 + 1, 0);
    for (int i = 0; i < n_sites0; ++i) {
        TGB_CHECK(n_neigh0[i] >= 1, TG_ERR_ARG, "site %d has no self pair", i);
        ps[i + 1] = ps[i] + n_neigh0[i];
    }
    const int64_t P = ps[n_sites0];
    std::vector<int> nb(P), rows(n_sites0), atoms(n_sites0);
    for (int64_t k = 0; k < P; ++k) {
        TGB_CHECK(neighbors_list0[k] >= 1, TG_ERR_ARG, "neighbour indices are 1-based");
        nb[k] = neighbors_list0[k] - 1;
    }
    for (int i = 0; i < n_sites0; ++i) {
        rows[i] = i;
        atoms[i] = nb[ps[i]] % n_total_sites;
    }
    cudaStream_t st = C.st;
    DBuf<int64_t> d_ps;
    DBuf<int> d_nb, d_rows, d_atoms, d_sp;
    DBuf<double> d_rjs, d_xyz, d_en, d_fo, d_vir;
    TGB_TRY(d_ps.ensure(n_sites0 + 1)); TGB_TRY(d_nb.ensure(P)); TGB_TRY(d_rows.ensure(n_sites0));
    TGB_TRY(d_atoms.ensure(n_sites0)); TGB_TRY(d_sp.ensure(n_total_sites)); TGB_TRY(d_rjs.ensure(P));
    TGB_TRY(d_xyz.ensure(3 * (size_t)P)); TGB_TRY(d_en.ensure(n_total_sites));
    TGB_TRY(d_fo.ensure(3 * (size_t)n_total_sites)); TGB_TRY(d_vir.ensure(9));
    TGB_CUDA(cudaMemcpyAsync(d_ps.p, ps.data(), sizeof(int64_t) * (n_sites0 + 1), cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(d_nb.p, nb.data(), sizeof(int) * P, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(d_rows.p, rows.data(), sizeof(int) * n_sites0, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(d_atoms.p, atoms.data(), sizeof(int) * n_sites0, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(d_sp.p, species_all, sizeof(int) * n_total_sites, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(d_rjs.p, rjs0, sizeof(double) * P, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(d_xyz.p, xyz0, sizeof(double) * 3 * P, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemsetAsync(d_en.p, 0, sizeof(double) * n_total_sites, st));
    TGB_CUDA(cudaMemsetAsync(d_fo.p, 0, sizeof(double) * 3 * n_total_sites, st));
    TGB_CUDA(cudaMemsetAsync(d_vir.p, 0, sizeof(double) * 9, st));
    SiteArgs S{n_sites0, d_rows.p, d_atoms.p, d_ps.p, d_nb.p, d_xyz.p, d_sp.p};
    TGB_TRY(evaluate_family(*fi->second, S, d_rjs.p, n_total_sites, d_en.p, d_fo.p, d_vir.p, st));
    std::vector<double> en(n_total_sites), fo(3 * (size_t)n_total_sites), vr(9);
    TGB_CUDA(cudaMemcpyAsync(en.data(), d_en.p, sizeof(double) * n_total_sites, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(fo.data(), d_fo.p, sizeof(double) * 3 * n_total_sites, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(vr.data(), d_vir.p, sizeof(double) * 9, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    if (energies0)
        for (int i = 0; i < n_total_sites; ++i) energies0[i] += en[i];
    if (forces0)
        for (size_t q = 0; q < fo.size(); ++q) forces0[q] += fo[q];
    if (virial)
        for (int q = 0; q < 9; ++q) virial[q] += vr[q];
    return TG_OK;
}

// One block's GAP sum delta^2 sum_s alpha_s K_is^zeta (no e0) per central site and,
// when der is given, its gradient d/dr_j for every pair of the sites' lists (the
// self pair holding d/dr_i), through the get_gap_soap remap. Host outputs: the
// sums by atom (en, n_total_sites), the sites' batch rows and atoms, the list
// starts (ps, n_sites0 + 1) and der (3 P).
static int property_eval(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                         const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                         const int32_t *species_batch, const int32_t *species_all, double *der,
                         std::vector<double> &en, std::vector<int> &rows, std::vector<int> &atoms,
                         std::vector<int64_t> &ps, int *n_central) {
    Context &C = *g_ctx;
    Block &b = *C.current;
    DBuf<signed char> zf;
    int64_t P = 0;
    int nc = 0;
    TGB_TRY(stage_batch(C, b, n_total_sites, n_sites0, n_neigh0, neighbors_list0, rjs0, xyz0,
                        species_batch, species_all, &P, &nc, zf));
    cudaStream_t st = C.st;
    DBuf<double> pg;
    TGB_TRY(C.en.ensure(n_total_sites));
    TGB_TRY(C.fo.ensure(3 * (size_t)n_total_sites));
    TGB_TRY(C.vir.ensure(9));
    TGB_CUDA(cudaMemsetAsync(C.en.p, 0, sizeof(double) * n_total_sites, st));
    TGB_CUDA(cudaMemsetAsync(C.fo.p, 0, sizeof(double) * 3 * n_total_sites, st));
    TGB_CUDA(cudaMemsetAsync(C.vir.p, 0, sizeof(double) * 9, st));
    if (der) {
        TGB_TRY(pg.ensure(3 * (size_t)P));
        TGB_CUDA(cudaMemsetAsync(pg.p, 0, sizeof(double) * 3 * P, st));
    }
    auto &wp = C.ws[b.key];
    if (!wp) wp = std::make_unique<Workspace>();
    SiteArgs S{nc, C.site_row.p, C.site_atom.p, C.pstart.p, C.nbr.p, C.xyz.p, C.spa.p};
    TGB_TRY(evaluate_block(b, *wp, S, n_total_sites, C.fo.p, C.en.p, C.vir.p, C.err.p, st, nullptr,
                           nullptr, nullptr, der ? pg.p : nullptr));
    TGB_TRY(check_err_word(C, C.err.p));
    en.assign(n_total_sites, 0.0);
    rows.assign(nc, 0);
    atoms.assign(nc, 0);
    ps.assign(n_sites0 + 1, 0);
    TGB_CUDA(cudaMemcpyAsync(en.data(), C.en.p, sizeof(double) * n_total_sites, cudaMemcpyDeviceToHost, st));
    if (nc > 0) {
        TGB_CUDA(cudaMemcpyAsync(atoms.data(), C.site_atom.p, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaMemcpyAsync(rows.data(), C.site_row.p, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
    }
    TGB_CUDA(cudaMemcpyAsync(ps.data(), C.pstart.p, sizeof(int64_t) * (n_sites0 + 1), cudaMemcpyDeviceToHost, st));
    if (der) TGB_CUDA(cudaMemcpyAsync(der, pg.p, sizeof(double) * 3 * P, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    *n_central = nc;
    return TG_OK;
}

int tg_get_local_property(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                          const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                          const int32_t *species_batch, const int32_t *species_all, double v0,
                          double *values, double *value_der, int32_t *n_central) {
    NvtxRange nvtx_range("tg_get_local_property");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(C.current, TG_ERR_STATE, "no block is open (call tg_soap_begin first)");
    TGB_CHECK(n_total_sites >= 1 && n_sites0 >= 0 && values && n_central, TG_ERR_ARG,
              "bad local-property arguments");
    *n_central = 0;
    if (n_sites0 == 0) return TG_OK;
    std::vector<double> en;
    std::vector<int> rows, atoms;
    std::vector<int64_t> ps;
    int nc = 0;
    TGB_TRY(property_eval(n_total_sites, n_sites0, n_neigh0, neighbors_list0, rjs0, xyz0,
                          species_batch, species_all, value_der, en, rows, atoms, ps, &nc));
    // local_properties.f90:244-270 (and hirshfeld_predict, vdw.f90:39-159): V =
    // delta^2 sum_s alpha_s K^zeta + V0, negative values clamped to zero together
    // with their derivatives
    for (int i = 0; i < nc; ++i) {
        double v = en[atoms[i]] + v0;
        if (v < 0.0) {
            v = 0.0;
            if (value_der)
                for (int64_t p = ps[rows[i]]; p < ps[rows[i] + 1]; ++p)
                    for (int q = 0; q < 3; ++q) value_der[3 * p + q] = 0.0;
        }
        values[i] = v;
    }
    *n_central = nc;
    return TG_OK;
}

int tg_get_soap_dipole(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                       const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                       const int32_t *species_batch, const int32_t *species_all, double *dipoles,
                       double *energies, int32_t *n_central) {
    NvtxRange nvtx_range("tg_get_soap_dipole");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(C.current, TG_ERR_STATE, "no block is open (call tg_soap_begin first)");
    TGB_CHECK(n_total_sites >= 1 && n_sites0 >= 0 && dipoles && n_central, TG_ERR_ARG,
              "bad dipole arguments");
    *n_central = 0;
    if (n_sites0 == 0) return TG_OK;
    int64_t P = 0;
    for (int i = 0; i < n_sites0; ++i) P += n_neigh0[i];
    std::vector<double> der(3 * (size_t)std::max<int64_t>(P, 1)), en;
    std::vector<int> rows, atoms;
    std::vector<int64_t> ps;
    int nc = 0;
    TGB_TRY(property_eval(n_total_sites, n_sites0, n_neigh0, neighbors_list0, rjs0, xyz0,
                          species_batch, species_all, der.data(), en, rows, atoms, ps, &nc));
    // gap.f90:378-387: mu_i = Qss_i . d(soap_i)/d(r_i), the self pair (first of
    // the site's list) of the fictitious energy's gradient; no e0, no clamp
    for (int i = 0; i < nc; ++i) {
        const int64_t self = ps[rows[i]];
        for (int q = 0; q < 3; ++q) dipoles[3 * (size_t)i + q] = der[3 * self + q];
        if (energies) energies[i] = en[atoms[i]];
    }
    *n_central = nc;
    return TG_OK;
}

int tg_get_soap(int32_t n_total_sites, int32_t n_sites0, const int32_t *n_neigh0,
                const int32_t *neighbors_list0, const double *rjs0, const double *xyz0,
                const int32_t *species_batch, const int32_t *species_all, double *soap,
                int32_t *n_central) {
    NvtxRange nvtx_range("tg_get_soap");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(C.current, TG_ERR_STATE, "no block is open (call tg_soap_begin first)");
    if (n_central) *n_central = 0;
    if (n_sites0 == 0) return TG_OK;
    Block &b = *C.current;
    DBuf<signed char> zf;
    int64_t P = 0;
    int nc = 0;
    TGB_TRY(stage_batch(C, b, n_total_sites, n_sites0, n_neigh0, neighbors_list0, rjs0, xyz0,
                        species_batch, species_all, &P, &nc, zf));
    if (n_central) *n_central = nc;
    if (nc == 0) return TG_OK;
    auto &wp = C.ws[b.key];
    if (!wp) wp = std::make_unique<Workspace>();
    TGB_TRY(wp->ensure(b, nc));
    SiteArgs S{nc, C.site_row.p, C.site_atom.p, C.pstart.p, C.nbr.p, C.xyz.p, C.spa.p};
    const SoapParams Pm = b.params(n_total_sites);
    TGB_TRY(descriptor_pass(b, *wp, Pm, S, C.st, 0));
    const int dout = b.compressed() ? b.dimc : b.dim;
    DBuf<double> out;
    TGB_TRY(out.ensure((size_t)nc * dout));
    k_d2f<<<grid_for((int64_t)nc * b.dim), 256, 0, C.st>>>((int64_t)nc * b.dim, b.dim, dout, wp->q.p,
                                                            b.mu.p, b.ref_index.p, out.p);
    TGB_CUDA(cudaGetLastError());
    TGB_CUDA(cudaMemcpyAsync(soap, out.p, sizeof(double) * nc * dout, cudaMemcpyDeviceToHost, C.st));
    TGB_CUDA(cudaStreamSynchronize(C.st));
    return TG_OK;
}

int tg_build_neighbors_list(int32_t n_sites_supercell, const double *positions, int32_t n_sites,
                            double *a_box, double *b_box, double *c_box, double rcut_max,
                            const int32_t *indices, const int32_t *species_supercell,
                            const int32_t *do_list, int64_t cap, int32_t *n_neigh,
                            int32_t *neighbors_list, double *rjs, double *thetas, double *phis,
                            double *xyz, int32_t *neighbor_species, int64_t *n_pairs) {
    NvtxRange nvtx_range("tg_build_neighbors_list");
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(n_sites >= 1 && n_sites_supercell >= n_sites, TG_ERR_ARG, "bad site counts");
    Box bx = make_box(a_box, b_box, c_box);
    if (bx.ortho) {   // neighbors.f90:372-384: snap the off-diagonal noise to zero
        a_box[1] = a_box[2] = b_box[0] = b_box[2] = c_box[0] = c_box[1] = 0.0;
        bx = make_box(a_box, b_box, c_box);
    }
    bool use_cells = false;
    const CellGrid g = plan_cells(bx, rcut_max, indices, &use_cells);
    cudaStream_t st = C.st;
    NeighborList nl;
    DBuf<double> pos;
    DBuf<int> dl, sp, nsp, selff;
    TGB_TRY(pos.ensure(3 * (size_t)n_sites_supercell));
    TGB_TRY(dl.ensure(n_sites));
    TGB_TRY(sp.ensure(n_sites_supercell));
    TGB_CUDA(cudaMemcpyAsync(pos.p, positions, sizeof(double) * 3 * n_sites_supercell, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(sp.p, species_supercell, sizeof(int) * n_sites_supercell, cudaMemcpyHostToDevice, st));
    if (do_list) TGB_CUDA(cudaMemcpyAsync(dl.p, do_list, sizeof(int) * n_sites, cudaMemcpyHostToDevice, st));
    int64_t pcap = std::max<int64_t>(cap, 1);
    int rc = nl.reserve(n_sites, n_sites_supercell, pcap, g);
    if (rc == TG_OK && cudaMemsetAsync(nl.err, 0, sizeof(unsigned), st) != cudaSuccess) rc = TG_ERR_CUDA;
    if (rc == TG_OK)
        rc = nl_build(nl, n_sites, n_sites_supercell, pos.p, bx, g, use_cells, rcut_max,
                      do_list ? dl.p : nullptr, st);
    int64_t P = 0;
    if (rc == TG_OK) {
        if (cudaMemcpyAsync(&P, nl.pstart + n_sites, sizeof(int64_t), cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = TG_ERR_CUDA;
    }
    if (rc == TG_OK) {
        if (n_pairs) *n_pairs = P;
        if (P > cap) {
            set_error("neighbour arrays hold %lld pairs, %lld needed", (long long)cap, (long long)P);
            rc = TG_ERR_CAPACITY;
        }
    }
    if (rc == TG_OK) {
        rc = selff.ensure(P);
        if (rc == TG_OK) rc = nsp.ensure(P);
        DBuf<double> th, ph;
        if (rc == TG_OK) rc = th.ensure(P);
        if (rc == TG_OK) rc = ph.ensure(P);
        if (rc == TG_OK && P > 0) {
            cudaMemsetAsync(selff.p, 0, sizeof(int) * P, st);
            k_is_self<<<grid_for(n_sites), 256, 0, st>>>(n_sites, nl.pstart, selff.p);
            rc = launch_angles(P, nl.rjs, nl.xyz, selff.p, th.p, ph.p, st);
            k_gather_species<<<grid_for(P), 256, 0, st>>>(P, nl.nbr, sp.p, nsp.p);
            k_add1<<<grid_for(P), 256, 0, st>>>(P, nl.nbr);
            if (cudaGetLastError() != cudaSuccess) rc = TG_ERR_CUDA;
            if (rc == TG_OK) {
                cudaMemcpyAsync(n_neigh, nl.n_neigh, sizeof(int) * n_sites, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(neighbors_list, nl.nbr, sizeof(int) * P, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(rjs, nl.rjs, sizeof(double) * P, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(xyz, nl.xyz, sizeof(double) * 3 * P, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(thetas, th.p, sizeof(double) * P, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(phis, ph.p, sizeof(double) * P, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(neighbor_species, nsp.p, sizeof(int) * P, cudaMemcpyDeviceToHost, st);
                if (cudaStreamSynchronize(st) != cudaSuccess) {
                    set_error("copy-back of the neighbour list failed");
                    rc = TG_ERR_CUDA;
                }
            }
        } else if (rc == TG_OK) {
            cudaMemcpyAsync(n_neigh, nl.n_neigh, sizeof(int) * n_sites, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
        }
    }
    if (rc == TG_OK) rc = check_err_word(C, nl.err);
    nl.release();
    return rc;
}

int tg_velocity_verlet(int32_t n, double *positions, double *positions_prev, double *velocities,
                       const double *forces, double *forces_prev, const double *masses, double dt,
                       double *dt_prev, int32_t first_step) {
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    cudaStream_t st = C.st;
    DBuf<double> p, pp, v, f, fp, m;
    const size_t b3 = sizeof(double) * 3 * n;
    TGB_TRY(p.ensure(3 * n)); TGB_TRY(pp.ensure(3 * n)); TGB_TRY(v.ensure(3 * n));
    TGB_TRY(f.ensure(3 * n)); TGB_TRY(fp.ensure(3 * n)); TGB_TRY(m.ensure(n));
    TGB_CUDA(cudaMemcpyAsync(p.p, positions, b3, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(v.p, velocities, b3, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(f.p, forces, b3, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(fp.p, forces_prev, b3, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(m.p, masses, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    TGB_TRY(launch_velocity_verlet(n, p.p, pp.p, v.p, f.p, fp.p, m.p, dt, dt_prev ? *dt_prev : dt,
                                   first_step, st));
    TGB_CUDA(cudaMemcpyAsync(positions, p.p, b3, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(positions_prev, pp.p, b3, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(velocities, v.p, b3, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(forces_prev, fp.p, b3, cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    if (dt_prev) *dt_prev = dt;
    return TG_OK;
}

}  // extern "C"

// ============================================================== engine
namespace tgb {

struct BlockRun {
    Block *b = nullptr;
    std::unique_ptr<Workspace> w;
    std::unique_ptr<MixedRun> mix;   // set: the block runs in the mixed (MLP + gate) form
    DBuf<int> sites;
    int n_sites = 0;
};

// a 2b / 3b / core_pot family of an engine and its central sites
struct FamilyRun {
    Family *f = nullptr;
    DBuf<int> sites;
    int n_sites = 0;
};

struct Engine {
    int n = 0, nsc = 0, indices[3] = {1, 1, 1};
    bool use_cells = false;
    CellGrid g{1, 1, 1};
    Box box{}, box_prim{};
    double rcut = 0.0;
    int nz = 0;
    DBuf<double> pos, pos_sc, pos_prev, vel, f, f_prev, mass, en, vir, e0, acc4, ekin, abc;
    DBuf<int> species;
    DBuf<unsigned> err;
    NeighborList nl;
    std::vector<std::unique_ptr<BlockRun>> runs;
    std::vector<std::unique_ptr<FamilyRun>> fams;
    cudaGraphExec_t graph = nullptr;
    double graph_dt = 0.0;
    bool first_step = true;
    // Verlet-skin lists (neighbors_buffer > 0 on the cell path, no supercell)
    bool skin = false;
    double skin_thresh = 0.0;            // neighbors_buffer / 2, compared with |displacement|^2
    DBuf<int> nl_when;                   // nonzero: the next evaluation rebuilds
    DBuf<double> disp;                   // displacement since the last rebuild (3, n)
    DBuf<long long> nl_counts;           // rebuilds, evaluations
    std::vector<int> species_h;          // host copy, for the site lists
    int site_beg = 0, site_end = 0;      // central sites of this rank
    // a rank's share of a sharded structure lists its own sites only: list flags
    // (1 inside [site_beg, site_end)) for the neighbour search, unset for the whole
    DBuf<int> do_list;
    bool ranged = false;
    Comm *comm = nullptr;                // set: forces/energies/virial summed over ranks
    bool frame_prev = false;    // the last evaluation saw pos_prev (an MD step ran)
    double dt_prev = 0.0;
    cudaStream_t st = nullptr;
    // blocks after the first run on their own streams (forked after the neighbour
    // list, joined before integration), so one block's kernels fill the SMs the
    // other block's tail waves leave idle
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev_side;
    cudaEvent_t ev_fork = nullptr;

    ~Engine() {
        if (graph) cudaGraphExecDestroy(graph);   // before the communicator its NCCL nodes use
        if (st) cudaStreamSynchronize(st);
        comm_destroy(comm);
        nl.release();
        for (auto e : ev_side) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (auto s2 : side) cudaStreamDestroy(s2);
        if (st) cudaStreamDestroy(st);
    }

    int ensure_streams() {
        const size_t need = runs.size() > 1 ? runs.size() - 1 : 0;
        if (!ev_fork) TGB_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        while (side.size() < need) {
            cudaStream_t s2;
            cudaEvent_t e2;
            TGB_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
            TGB_CUDA(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
            side.push_back(s2);
            ev_side.push_back(e2);
        }
        return TG_OK;
    }

    EventLog prof;

    int compute_ef(EventLog *log = nullptr) {
        TGB_MARK(log, -1, st);
        const double *p = pos.p;
        if (nsc > n) {
            TGB_TRY(launch_supercell(n, pos.p, abc.p, indices, pos_sc.p, st));
            p = pos_sc.p;
        }
        if (skin) {
            // neighbors_buffer > 0: rebuild only when the previous step asked for it,
            // otherwise refresh the kept pairs (decided on the device, inside the graph)
            TGB_TRY(nl_build(nl, n, nsc, p, box, g, use_cells, rcut, ranged ? do_list.p : nullptr,
                             st, nl_when.p));
            TGB_TRY(launch_nl_refresh(n, p, box, nl, nl_when.p, st));
            TGB_TRY(launch_skin_reset(n, nl_when.p, disp.p, nl_counts.p, st));
            TGB_CUDA(cudaMemsetAsync(nl_when.p, 0, sizeof(int), st));
        } else {
            TGB_TRY(nl_build(nl, n, nsc, p, box, g, use_cells, rcut, ranged ? do_list.p : nullptr, st));
        }
        TGB_TRY(launch_pair_species(n, nl, species.p, n, st));
        TGB_MARK(log, PASS_NEIGH, st);
        k_energy_e0<<<grid_for(n), 256, 0, st>>>(n, species.p, e0.p, nz, site_beg, site_end, en.p);
        TGB_CUDA(cudaMemsetAsync(f.p, 0, sizeof(double) * 3 * n, st));
        TGB_CUDA(cudaMemsetAsync(vir.p, 0, sizeof(double) * 9, st));
        // with a pass log every block runs on the main stream, so the marks time passes
        const bool fork = !log && runs.size() > 1;
        if (fork) {
            TGB_TRY(ensure_streams());
            TGB_CUDA(cudaEventRecord(ev_fork, st));
            for (size_t k = 1; k < runs.size(); ++k) TGB_CUDA(cudaStreamWaitEvent(side[k - 1], ev_fork, 0));
        }
        for (size_t k = 0; k < runs.size(); ++k) {
            auto &r = runs[k];
            cudaStream_t sk = (fork && k > 0) ? side[k - 1] : st;
            SiteArgs S{r->n_sites, r->sites.p, r->sites.p, nl.pstart, nl.nbr, nl.xyz, species.p};
            S.nsp = nl.nsp;
            if (r->mix)
                TGB_TRY(evaluate_block_mixed(*r->b, *r->w, *r->mix, S, n, f.p, en.p, vir.p, err.p,
                                             sk, log));
            else
                TGB_TRY(evaluate_block(*r->b, *r->w, S, n, f.p, en.p, vir.p, err.p, sk, log));
        }
        if (fork)
            for (size_t k = 1; k < runs.size(); ++k) {
                TGB_CUDA(cudaEventRecord(ev_side[k - 1], side[k - 1]));
                TGB_CUDA(cudaStreamWaitEvent(st, ev_side[k - 1], 0));
            }
        // the other GAP families on the same lists (gap_backend_cpu.f90:79-267),
        // timed with the force pass
        for (auto &fr : fams) {
            SiteArgs S{fr->n_sites, fr->sites.p, fr->sites.p, nl.pstart, nl.nbr, nl.xyz, species.p};
            TGB_TRY(evaluate_family(*fr->f, S, nl.rjs, n, en.p, f.p, vir.p, st));
        }
        if (!fams.empty()) TGB_MARK(log, PASS_FORCE, st);
        // sharded structure: every rank holds its own sites' share; the sum over
        // ranks is the whole (turbogap.f90:1876-1885)
        if (comm) TGB_TRY(comm_allreduce3(comm, f.p, 3 * (size_t)n, en.p, n, vir.p, 9, st));
        return TG_OK;
    }

    // central sites of each block within [site_beg, site_end); species never
    // change during MD
    int assign_sites() {
        ranged = site_beg > 0 || site_end < n;
        if (ranged) {
            std::vector<int> flags(n, 0);
            for (int i = site_beg; i < site_end; ++i) flags[i] = 1;
            TGB_TRY(do_list.ensure(n));
            TGB_CUDA(cudaMemcpyAsync(do_list.p, flags.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        }
        for (auto &run : runs) {
            const Block *b = run->b;
            std::vector<int> s;
            for (int i = site_beg; i < site_end; ++i) {
                const int z = species_h[i];
                int first = 0;
                for (int q = 0; q < b->ns; ++q)
                    if (b->hh.species_z[q] == z) { first = q + 1; break; }
                if (b->hh.central_species == 0 || first == b->hh.central_species) s.push_back(i);
            }
            run->n_sites = (int)s.size();
            TGB_TRY(run->sites.ensure(std::max<size_t>(s.size(), 1)));
            if (!s.empty())
                TGB_CUDA(cudaMemcpyAsync(run->sites.p, s.data(), sizeof(int) * s.size(),
                                         cudaMemcpyHostToDevice, st));
            TGB_TRY(run->w->ensure(*b, run->n_sites));
            if (run->mix) TGB_TRY(run->mix->ensure(*b, run->n_sites));
        }
        for (auto &fr : fams) {
            std::vector<int> s;
            family_sites(*fr->f, species_h.data(), site_beg, site_end, s);
            fr->n_sites = (int)s.size();
            TGB_TRY(fr->sites.ensure(std::max<size_t>(s.size(), 1)));
            if (!s.empty())
                TGB_CUDA(cudaMemcpyAsync(fr->sites.p, s.data(), sizeof(int) * s.size(),
                                         cudaMemcpyHostToDevice, st));
        }
        TGB_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }

    int md_step(double dt, bool first, EventLog *log = nullptr) {
        TGB_TRY(compute_ef(log));
        TGB_TRY(launch_wrap(n, pos.p, box_prim, st));
        TGB_TRY(launch_remove_cm(n, vel.p, mass.p, acc4.p, st));
        TGB_TRY(launch_velocity_verlet(n, pos.p, pos_prev.p, vel.p, f.p, f_prev.p, mass.p, dt,
                                       first ? dt : dt_prev, first ? 1 : 0, st));
        if (skin) TGB_TRY(launch_skin_check(n, pos.p, pos_prev.p, disp.p, skin_thresh, nl_when.p, st));
        TGB_MARK(log, PASS_INTEGRATE, st);
        return TG_OK;
    }

    // picks the CTA tiles of every block's SOAP passes on this structure
    int autotune() {
        if (pinned_tile() >= 0)
            for (auto &r : runs) pin_tiles(*r->b, *r->w, pinned_tile());
        if (!autotune_enabled() || runs.empty()) return TG_OK;
        const double *p = pos.p;
        if (nsc > n) {
            TGB_TRY(launch_supercell(n, pos.p, abc.p, indices, pos_sc.p, st));
            p = pos_sc.p;
        }
        TGB_TRY(nl_build(nl, n, nsc, p, box, g, use_cells, rcut, nullptr, st));
        TGB_TRY(launch_pair_species(n, nl, species.p, n, st));
        TGB_CUDA(cudaMemsetAsync(f.p, 0, sizeof(double) * 3 * n, st));
        TGB_CUDA(cudaMemsetAsync(en.p, 0, sizeof(double) * n, st));
        TGB_CUDA(cudaMemsetAsync(vir.p, 0, sizeof(double) * 9, st));
        for (auto &r : runs) {
            SiteArgs S{r->n_sites, r->sites.p, r->sites.p, nl.pstart, nl.nbr, nl.xyz, species.p};
            S.nsp = nl.nsp;
            TGB_TRY(autotune_block(*r->b, *r->w, S, n, f.p, en.p, vir.p, err.p, st));
        }
        TGB_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }

    // the next evaluation rebuilds the list (positions replaced from outside)
    int force_rebuild() {
        if (!skin) return TG_OK;
        const int one = 1;
        TGB_CUDA(cudaMemcpyAsync(nl_when.p, &one, sizeof(int), cudaMemcpyHostToDevice, st));
        TGB_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }
};

}  // namespace tgb

struct tg_engine {
    tgb::Engine e;
};

extern "C" {

static int engine_errors(Engine &E);

int tg_engine_create(int32_t n_atoms, const double *positions, const int32_t *species,
                     const double *masses, const double *a_box, const double *b_box,
                     const double *c_box, int32_t n_blocks, const int32_t *block_keys,
                     const double *e0_by_species, int32_t n_species_total, double neighbors_buffer,
                     tg_engine **out) {
    NvtxRange nvtx_range("tg_engine_create");
    TGB_TRY(need_ctx());
    TGB_CHECK(out && n_atoms >= 1 && n_blocks >= 1, TG_ERR_ARG, "bad engine arguments");
    Context &C = *g_ctx;
    auto holder = std::make_unique<tg_engine>();
    Engine &E = holder->e;
    E.n = n_atoms;
    TGB_CUDA(cudaStreamCreateWithFlags(&E.st, cudaStreamNonBlocking));
    double rcut = 0.0;
    for (int k = 0; k < n_blocks; ++k) {
        auto it = C.blocks.find(block_keys[k]);
        auto fi = C.families.find(block_keys[k]);
        TGB_CHECK(it != C.blocks.end() || fi != C.families.end(), TG_ERR_STATE,
                  "block key %d was never begun", block_keys[k]);
        rcut = std::max(rcut, it != C.blocks.end() ? it->second->rcut_max : fi->second->rcut);
    }
    rcut += neighbors_buffer;   // turbogap_setup.f90:284-285
    E.rcut = rcut;
    // read_files.f90:320-380: supercell when the box cannot hold a cutoff sphere
    host_unit_cells(a_box, b_box, c_box, rcut, E.indices);
    // a triclinic box takes the reference's O(N N_supercell) list search
    // (neighbors.f90:474-514) and its triclinic wrap_pbc
    E.box_prim = make_box(a_box, b_box, c_box);
    double A[3], B[3], Cc[3];
    for (int q = 0; q < 3; ++q) {
        A[q] = a_box[q] * E.indices[0];
        B[q] = b_box[q] * E.indices[1];
        Cc[q] = c_box[q] * E.indices[2];
    }
    E.box = make_box(A, B, Cc);
    E.nsc = n_atoms * E.indices[0] * E.indices[1] * E.indices[2];
    E.g = plan_cells(E.box, rcut, E.indices, &E.use_cells);
    const size_t n3 = 3 * (size_t)n_atoms;
    TGB_TRY(E.pos.ensure(n3)); TGB_TRY(E.pos_prev.ensure(n3)); TGB_TRY(E.vel.ensure(n3));
    TGB_TRY(E.f.ensure(n3)); TGB_TRY(E.f_prev.ensure(n3)); TGB_TRY(E.mass.ensure(n_atoms));
    TGB_TRY(E.en.ensure(n_atoms)); TGB_TRY(E.vir.ensure(9)); TGB_TRY(E.acc4.ensure(4));
    TGB_TRY(E.ekin.ensure(1)); TGB_TRY(E.species.ensure(n_atoms)); TGB_TRY(E.err.ensure(1));
    TGB_TRY(E.abc.ensure(9));
    E.nz = std::max(n_species_total, 1);
    TGB_TRY(E.e0.ensure(E.nz));
    std::vector<double> e0(E.nz, 0.0);
    if (e0_by_species)
        for (int z = 0; z < n_species_total; ++z) e0[z] = e0_by_species[z];
    const double abc_h[9] = {a_box[0], a_box[1], a_box[2], b_box[0], b_box[1],
                             b_box[2], c_box[0], c_box[1], c_box[2]};
    if (E.nsc > E.n) TGB_TRY(E.pos_sc.ensure(3 * (size_t)E.nsc));
    cudaStream_t st = E.st;
    TGB_CUDA(cudaMemcpyAsync(E.pos.p, positions, sizeof(double) * n3, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemsetAsync(E.vel.p, 0, sizeof(double) * n3, st));
    TGB_CUDA(cudaMemsetAsync(E.f_prev.p, 0, sizeof(double) * n3, st));
    TGB_CUDA(cudaMemcpyAsync(E.mass.p, masses, sizeof(double) * n_atoms, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.species.p, species, sizeof(int) * n_atoms, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.e0.p, e0.data(), sizeof(double) * E.nz, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.abc.p, abc_h, sizeof(abc_h), cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemsetAsync(E.err.p, 0, sizeof(unsigned), st));
    E.species_h.assign(species, species + n_atoms);
    E.site_beg = 0;
    E.site_end = n_atoms;
    for (int k = 0; k < n_blocks; ++k) {
        auto fi = C.families.find(block_keys[k]);
        if (fi != C.families.end()) {
            auto fr = std::make_unique<FamilyRun>();
            fr->f = fi->second.get();
            E.fams.push_back(std::move(fr));
            continue;
        }
        auto run = std::make_unique<BlockRun>();
        run->b = C.blocks[block_keys[k]].get();
        run->w = std::make_unique<Workspace>();
        E.runs.push_back(std::move(run));
    }
    TGB_TRY(E.assign_sites());
    // size the pair arrays from a first build, with 40 % headroom for MD
    const double *p0 = E.pos.p;
    if (E.nsc > E.n) {
        TGB_TRY(launch_supercell(E.n, E.pos.p, E.abc.p, E.indices, E.pos_sc.p, st));
        p0 = E.pos_sc.p;
    }
    TGB_TRY(E.nl.reserve(E.n, E.nsc, (int64_t)E.n * 48, E.g));
    TGB_CUDA(cudaMemsetAsync(E.nl.err, 0, sizeof(unsigned), st));
    TGB_TRY(nl_build(E.nl, E.n, E.nsc, p0, E.box, E.g, E.use_cells, rcut, nullptr, st));
    int64_t P = 0;
    TGB_CUDA(cudaMemcpyAsync(&P, E.nl.pstart + E.n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    TGB_TRY(E.nl.reserve(E.n, E.nsc, (int64_t)(P * 1.4) + 64, E.g));
    if (E.use_cells) {
        // slot rows of the one-pass build: the largest count with 25 % headroom (a
        // site that outgrows them sends that build to the filling search);
        // TGB_NL_SLOTS=s sets the rows, 0 keeps the two-pass build
        std::vector<int> cnt(E.n);
        TGB_CUDA(cudaMemcpyAsync(cnt.data(), E.nl.n_neigh, sizeof(int) * E.n,
                                 cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaStreamSynchronize(st));
        int mx = 1;
        for (int c : cnt) mx = std::max(mx, c);
        int slots = (mx + mx / 4 + 8 + 15) / 16 * 16;
        if (const char *e = std::getenv("TGB_NL_SLOTS")) slots = std::max(0, std::atoi(e));
        if (slots > 0 && slots <= 256) TGB_TRY(E.nl.reserve_slots(E.n, slots));
    }
    TGB_CUDA(cudaMemsetAsync(E.nl.err, 0, sizeof(unsigned), st));
    // turbogap_md.f90:453-470: a supercell always rebuilds; otherwise a positive
    // buffer keeps the list until an atom has moved far enough
    E.skin = neighbors_buffer > 0.0 && E.nsc == E.n && E.use_cells;
    if (E.skin) {
        E.skin_thresh = neighbors_buffer / 2.0;
        TGB_TRY(E.nl_when.ensure(1));
        TGB_TRY(E.disp.ensure(n3));
        TGB_TRY(E.nl_counts.ensure(2));
        TGB_CUDA(cudaMemsetAsync(E.disp.p, 0, sizeof(double) * n3, st));
        TGB_CUDA(cudaMemsetAsync(E.nl_counts.p, 0, sizeof(long long) * 2, st));
        TGB_TRY(E.force_rebuild());
    }
    TGB_TRY(E.autotune());
    TGB_TRY(engine_errors(E));
    TGB_CUDA(cudaStreamSynchronize(st));
    *out = holder.release();
    return TG_OK;
}

int tg_engine_destroy(tg_engine *e) {
    if (!e) return TG_OK;
    cudaStreamSynchronize(e->e.st);
    delete e;
    return TG_OK;
}

int tg_engine_set_state(tg_engine *eh, const double *positions, const double *velocities) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    const size_t b3 = sizeof(double) * 3 * E.n;
    if (positions) TGB_CUDA(cudaMemcpyAsync(E.pos.p, positions, b3, cudaMemcpyHostToDevice, E.st));
    if (velocities) TGB_CUDA(cudaMemcpyAsync(E.vel.p, velocities, b3, cudaMemcpyHostToDevice, E.st));
    E.first_step = true;
    E.frame_prev = false;
    if (positions) TGB_TRY(E.force_rebuild());
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

static int engine_errors(Engine &E) {
    unsigned e1 = 0, e2 = 0;
    TGB_CUDA(cudaMemcpyAsync(&e1, E.err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaMemcpyAsync(&e2, E.nl.err, sizeof(unsigned), cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    const unsigned e = e1 | e2;
    if (!e) return TG_OK;
    TGB_CUDA(cudaMemsetAsync(E.err.p, 0, sizeof(unsigned), E.st));
    TGB_CUDA(cudaMemsetAsync(E.nl.err, 0, sizeof(unsigned), E.st));
    if (e & (DEV_ERR_TIMEOUT_TMA | DEV_ERR_TIMEOUT_MMA | DEV_ERR_TIMEOUT_EPI)) {
        set_error("device wait timed out (error word 0x%x)", e);
        return TG_ERR_TIMEOUT;
    }
    set_error("device error word 0x%x%s", e,
              (e & DEV_ERR_NEIGH_CAPACITY) ? " (neighbour pair capacity exceeded)" : "");
    return TG_ERR_DEVICE;
}

int tg_engine_compute_device(tg_engine *eh) {
    NvtxRange nvtx_range("tg_engine_compute_device");
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    eh->e.frame_prev = false;
    return eh->e.compute_ef();
}

int tg_engine_compute(tg_engine *eh, double *energies, double *forces, double *virial) {
    NvtxRange nvtx_range("tg_engine_compute");
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    E.frame_prev = false;
    TGB_TRY(E.compute_ef());
    if (energies)
        TGB_CUDA(cudaMemcpyAsync(energies, E.en.p, sizeof(double) * E.n, cudaMemcpyDeviceToHost, E.st));
    if (forces)
        TGB_CUDA(cudaMemcpyAsync(forces, E.f.p, sizeof(double) * 3 * E.n, cudaMemcpyDeviceToHost, E.st));
    if (virial) TGB_CUDA(cudaMemcpyAsync(virial, E.vir.p, sizeof(double) * 9, cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return engine_errors(E);
}

int tg_engine_md(tg_engine *eh, int32_t n_steps, double dt, double *e_pot, double *e_kin) {
    NvtxRange nvtx_range("tg_engine_md");
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    for (int s = 0; s < n_steps; ++s) {
        if (E.first_step) {
            TGB_TRY(E.md_step(dt, true));
            E.first_step = false;
            E.dt_prev = dt;
            TGB_TRY(engine_errors(E));
            continue;
        }
        if (!E.graph || E.graph_dt != dt) {
            if (E.graph) {
                cudaGraphExecDestroy(E.graph);
                E.graph = nullptr;
            }
            cudaGraph_t gr;
            TGB_CUDA(cudaStreamBeginCapture(E.st, cudaStreamCaptureModeThreadLocal));
            int r = E.md_step(dt, false);
            cudaError_t ce = cudaStreamEndCapture(E.st, &gr);
            TGB_TRY(r);
            TGB_CUDA(ce);
            ce = cudaGraphInstantiate(&E.graph, gr, 0);
            cudaGraphDestroy(gr);
            TGB_CUDA(ce);
            E.graph_dt = dt;
        }
        TGB_CUDA(cudaGraphLaunch(E.graph, E.st));
        E.dt_prev = dt;
    }
    if (n_steps > 0) E.frame_prev = true;
    TGB_TRY(engine_errors(E));
    if (e_kin) {
        TGB_TRY(launch_kinetic(E.n, E.vel.p, E.mass.p, E.ekin.p, E.st));
        TGB_CUDA(cudaMemcpyAsync(e_kin, E.ekin.p, sizeof(double), cudaMemcpyDeviceToHost, E.st));
    }
    if (e_pot) {
        std::vector<double> en(E.n);
        TGB_CUDA(cudaMemcpyAsync(en.data(), E.en.p, sizeof(double) * E.n, cudaMemcpyDeviceToHost, E.st));
        TGB_CUDA(cudaStreamSynchronize(E.st));
        double s = 0.0;
        for (double v : en) s += v;
        *e_pot = s;
    }
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

int tg_engine_get_state(tg_engine *eh, double *positions, double *velocities, double *forces) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    const size_t b3 = sizeof(double) * 3 * E.n;
    if (positions) TGB_CUDA(cudaMemcpyAsync(positions, E.pos.p, b3, cudaMemcpyDeviceToHost, E.st));
    if (velocities) TGB_CUDA(cudaMemcpyAsync(velocities, E.vel.p, b3, cudaMemcpyDeviceToHost, E.st));
    if (forces) TGB_CUDA(cudaMemcpyAsync(forces, E.f.p, b3, cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

int tg_engine_get_frame(tg_engine *eh, double *positions, double *velocities, double *forces,
                        double *energies, double *virial) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    const size_t b3 = sizeof(double) * 3 * E.n;
    // after an MD step the evaluation saw pos_prev (turbogap_md.f90:357-358: the
    // trajectory holds positions_prev, synchronous with the velocities)
    const double *p = E.frame_prev ? E.pos_prev.p : E.pos.p;
    if (positions) TGB_CUDA(cudaMemcpyAsync(positions, p, b3, cudaMemcpyDeviceToHost, E.st));
    if (velocities) TGB_CUDA(cudaMemcpyAsync(velocities, E.vel.p, b3, cudaMemcpyDeviceToHost, E.st));
    if (forces) TGB_CUDA(cudaMemcpyAsync(forces, E.f.p, b3, cudaMemcpyDeviceToHost, E.st));
    if (energies)
        TGB_CUDA(cudaMemcpyAsync(energies, E.en.p, sizeof(double) * E.n, cudaMemcpyDeviceToHost, E.st));
    if (virial) TGB_CUDA(cudaMemcpyAsync(virial, E.vir.p, sizeof(double) * 9, cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

int tg_engine_set_site_range(tg_engine *eh, int32_t site_beg, int32_t site_end) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    TGB_CHECK(site_beg >= 0 && site_beg <= site_end && site_end <= E.n, TG_ERR_ARG,
              "site range [%d, %d) outside [0, %d)", site_beg, site_end, E.n);
    TGB_CUDA(cudaStreamSynchronize(E.st));
    if (E.graph) {   // the captured step holds the old site lists
        cudaGraphExecDestroy(E.graph);
        E.graph = nullptr;
    }
    E.site_beg = site_beg;
    E.site_end = site_end;
    return E.assign_sites();
}

int tg_nccl_unique_id(void *id128) { return comm_unique_id(id128); }

int tg_engine_set_comm(tg_engine *eh, const void *id128, int32_t n_ranks, int32_t rank) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    TGB_CUDA(cudaStreamSynchronize(E.st));
    if (E.graph) {
        cudaGraphExecDestroy(E.graph);
        E.graph = nullptr;
    }
    comm_destroy(E.comm);
    E.comm = nullptr;
    if (!id128) return TG_OK;
    return comm_init(id128, n_ranks, rank, &E.comm);
}

int tg_engine_neighbor_stats(tg_engine *eh, int64_t *n_builds, int64_t *n_evaluations) {
    TGB_CHECK(eh && n_builds && n_evaluations, TG_ERR_ARG, "null argument");
    Engine &E = eh->e;
    *n_builds = *n_evaluations = -1;
    if (!E.skin) return TG_OK;
    long long c[2] = {0, 0};
    TGB_CUDA(cudaMemcpyAsync(c, E.nl_counts.p, sizeof(c), cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    *n_builds = c[0];
    *n_evaluations = c[1];
    return TG_OK;
}

int tg_engine_tiles(tg_engine *eh, int32_t *tiles, int32_t n, int32_t *n_blocks) {
    TGB_CHECK(eh && tiles && n_blocks, TG_ERR_ARG, "null argument");
    Engine &E = eh->e;
    TGB_CHECK(n >= 2 * (int)E.runs.size(), TG_ERR_CAPACITY, "tiles needs %d entries",
              2 * (int)E.runs.size());
    *n_blocks = (int32_t)E.runs.size();
    for (size_t k = 0; k < E.runs.size(); ++k) {
        tiles[2 * k] = E.runs[k]->w->tile_desc;
        tiles[2 * k + 1] = E.runs[k]->w->tile_force;
    }
    return TG_OK;
}

int tg_engine_n_pairs(tg_engine *eh, int64_t *n_pairs) {
    TGB_CHECK(eh && n_pairs, TG_ERR_ARG, "null argument");
    Engine &E = eh->e;
    TGB_CUDA(cudaMemcpyAsync(n_pairs, E.nl.pstart + E.n, sizeof(int64_t), cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

int tg_engine_profile(tg_engine *eh, int32_t n_steps, double dt, double *ms_per_pass,
                      int32_t *n_passes) {
    NvtxRange nvtx_range("tg_engine_profile");
    TGB_CHECK(eh && ms_per_pass && n_steps >= 1, TG_ERR_ARG, "bad profile arguments");
    Engine &E = eh->e;
    double acc[N_PASS] = {0};
    for (int s = 0; s < n_steps; ++s) {
        const bool first = E.first_step;
        TGB_TRY(E.md_step(dt, first, &E.prof));
        E.first_step = false;
        E.frame_prev = true;
        E.dt_prev = dt;
        TGB_CUDA(cudaStreamSynchronize(E.st));
        TGB_TRY(E.prof.collect(acc));
    }
    for (int p = 0; p < N_PASS; ++p) ms_per_pass[p] = acc[p] / n_steps;
    if (n_passes) *n_passes = N_PASS;
    return engine_errors(E);
}

int tg_engine_graph_kernels(tg_engine *eh, int32_t *n_kernels) {
    TGB_CHECK(eh && n_kernels, TG_ERR_ARG, "null argument");
    Engine &E = eh->e;
    *n_kernels = 0;
    if (!E.graph) return TG_OK;
    cudaGraph_t g;
    TGB_CUDA(cudaStreamBeginCapture(E.st, cudaStreamCaptureModeThreadLocal));
    int r = E.md_step(E.graph_dt, false);
    cudaError_t ce = cudaStreamEndCapture(E.st, &g);
    TGB_TRY(r);
    TGB_CUDA(ce);
    size_t n = 0;
    ce = cudaGraphGetNodes(g, nullptr, &n);
    std::vector<cudaGraphNode_t> nodes(n);
    if (ce == cudaSuccess && n) ce = cudaGraphGetNodes(g, nodes.data(), &n);
    int k = 0;
    for (size_t i = 0; ce == cudaSuccess && i < n; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    cudaGraphDestroy(g);
    TGB_CUDA(ce);
    *n_kernels = k;
    return TG_OK;
}

int tg_engine_stream(tg_engine *eh, void **stream) {
    TGB_CHECK(eh && stream, TG_ERR_ARG, "null argument");
    *stream = (void *)eh->e.st;
    return TG_OK;
}

// ---------------------------------------------------------------- learned surrogate
struct tg_mlp {
    tgb::Mlp *m = nullptr;
};

int tg_mlp_create(int32_t dim, int32_t hidden, int32_t n_members, uint64_t seed, tg_mlp **out) {
    TGB_TRY(need_ctx());
    TGB_CHECK(out, TG_ERR_ARG, "null output");
    Mlp *m = nullptr;
    TGB_TRY(mlp_create(dim, hidden, n_members, (unsigned long long)seed, &m));
    *out = new tg_mlp{m};
    return TG_OK;
}

int tg_mlp_destroy(tg_mlp *h) {
    if (!h) return TG_OK;
    mlp_destroy(h->m);
    delete h;
    return TG_OK;
}

int tg_mlp_set_member(tg_mlp *h, int32_t member, const double *W1, const double *b1,
                      const double *W2, const double *b2, const double *w3, double b3) {
    TGB_CHECK(h, TG_ERR_ARG, "null MLP");
    return mlp_set_member(*h->m, member, W1, b1, W2, b2, w3, b3);
}

int tg_mlp_get_member(tg_mlp *h, int32_t member, double *W1, double *b1, double *W2, double *b2,
                      double *w3, double *b3) {
    TGB_CHECK(h, TG_ERR_ARG, "null MLP");
    return mlp_get_member(*h->m, member, W1, b1, W2, b2, w3, b3);
}

int tg_mlp_set_normalisation(tg_mlp *h, double sigma_x, double mean_e, double sigma_e) {
    TGB_CHECK(h, TG_ERR_ARG, "null MLP");
    TGB_CHECK(sigma_x > 0.0 && sigma_e > 0.0, TG_ERR_ARG, "scales must be positive");
    Mlp &m = *h->m;
    m.sx = sigma_x;
    m.muE = mean_e;
    m.sE = sigma_e;
    for (int k = 0; k < m.n_members; ++k) {   // rebuild the inference copies
        std::vector<double> W1((size_t)m.L.H * m.L.D), b1(m.L.H), W2((size_t)m.L.H * m.L.H),
            b2(m.L.H), w3(m.L.H);
        double b3 = 0.0;
        TGB_TRY(mlp_get_member(m, k, W1.data(), b1.data(), W2.data(), b2.data(), w3.data(), &b3));
        const long long t = m.adam_t[k];
        TGB_TRY(mlp_set_member(m, k, W1.data(), b1.data(), W2.data(), b2.data(), w3.data(), b3));
        m.adam_t[k] = t;
    }
    return TG_OK;
}

int tg_mlp_get_normalisation(tg_mlp *h, double *sigma_x, double *mean_e, double *sigma_e) {
    TGB_CHECK(h, TG_ERR_ARG, "null MLP");
    if (sigma_x) *sigma_x = h->m->sx;
    if (mean_e) *mean_e = h->m->muE;
    if (sigma_e) *sigma_e = h->m->sE;
    return TG_OK;
}

int tg_mlp_add_samples(tg_mlp *h, int32_t n, const float *delta, const double *energy,
                       const float *dedq) {
    TGB_TRY(need_ctx());
    TGB_CHECK(h && n >= 0 && (n == 0 || (delta && energy && dedq)), TG_ERR_ARG, "bad samples");
    if (n == 0) return TG_OK;
    Context &C = *g_ctx;
    Mlp &m = *h->m;
    const int D = m.L.D;
    DBuf<float> x, g;
    DBuf<double> e;
    TGB_TRY(x.ensure((size_t)n * D));
    TGB_TRY(g.ensure((size_t)n * D));
    TGB_TRY(e.ensure(n));
    TGB_CUDA(cudaMemcpyAsync(x.p, delta, sizeof(float) * n * D, cudaMemcpyHostToDevice, C.st));
    TGB_CUDA(cudaMemcpyAsync(g.p, dedq, sizeof(float) * n * D, cudaMemcpyHostToDevice, C.st));
    TGB_CUDA(cudaMemcpyAsync(e.p, energy, sizeof(double) * n, cudaMemcpyHostToDevice, C.st));
    TGB_TRY(mlp_append_device(m, n, x.p, D, e.p, g.p, D, C.st));
    TGB_CUDA(cudaStreamSynchronize(C.st));
    return TG_OK;
}

int tg_mlp_add_engine_samples(tg_mlp *h, tg_engine *eh, int32_t block) {
    NvtxRange nvtx_range("tg_mlp_add_engine_samples");
    TGB_CHECK(h && eh, TG_ERR_ARG, "null argument");
    Engine &E = eh->e;
    TGB_CHECK(block >= 0 && block < (int)E.runs.size(), TG_ERR_ARG, "block %d out of range", block);
    BlockRun &r = *E.runs[block];
    TGB_CHECK(!r.mix, TG_ERR_STATE, "block %d runs the mixed form; samples come from exact steps",
              block);
    Block &b = *r.b;
    Mlp &m = *h->m;
    TGB_CHECK(m.L.D == b.dim, TG_ERR_ARG, "MLP input size %d does not match block dim %d", m.L.D,
              b.dim);
    const int n = r.n_sites;
    if (n == 0) return TG_OK;
    Workspace &w = *r.w;
    DBuf<float> G;
    DBuf<double> e;
    TGB_TRY(G.ensure((size_t)n * b.dim));
    TGB_TRY(e.ensure(n));
    k_collect<<<grid_for((int64_t)n * 32), 256, 0, E.st>>>(n, b.dim, b.n_etiles, b.delta * b.delta,
                                                           w.epart.p, w.kdsum.p, b.mu.p, b.g0.p,
                                                           w.g.p, e.p, G.p);
    TGB_CUDA(cudaGetLastError());
    TGB_TRY(mlp_append_device(m, n, w.q.p, b.dim, e.p, G.p, b.dim, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

int tg_mlp_n_samples(tg_mlp *h, int64_t *n) {
    TGB_CHECK(h && n, TG_ERR_ARG, "null argument");
    *n = h->m->n_data;
    return TG_OK;
}

int tg_mlp_train(tg_mlp *h, int32_t epochs, int32_t batch, double lr, double force_weight,
                 uint64_t seed, double *loss_per_epoch) {
    NvtxRange nvtx_range("tg_mlp_train");
    TGB_TRY(need_ctx());
    TGB_CHECK(h, TG_ERR_ARG, "null MLP");
    return mlp_train(*h->m, epochs, batch, lr, force_weight, (unsigned long long)seed,
                     loss_per_epoch, g_ctx->st);
}

__global__ void k_rows_to_bf16(int n, int D, int Dp, const float *__restrict__ x,
                               __nv_bfloat16 *__restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * Dp) return;
    const int64_t r = i / Dp;
    const int d = (int)(i - r * Dp);
    out[i] = __float2bfloat16_rn(d < D ? x[r * D + d] : 0.f);
}

int tg_mlp_predict(tg_mlp *h, int32_t n, const float *delta, double *energy_mean,
                   double *energy_std, double *dedq_mean) {
    NvtxRange nvtx_range("tg_mlp_predict");
    TGB_TRY(need_ctx());
    TGB_CHECK(h && n >= 0 && (n == 0 || (delta && energy_mean)), TG_ERR_ARG, "bad arguments");
    if (n == 0) return TG_OK;
    Context &C = *g_ctx;
    Mlp &m = *h->m;
    const int D = m.L.D, Dp = m.L.Dp;
    const int ldg = (D + 3) / 4 * 4;
    DBuf<float> x, g;
    DBuf<__nv_bfloat16> xb;
    DBuf<double> em, es;
    TGB_TRY(x.ensure((size_t)n * D));
    TGB_TRY(g.ensure((size_t)n * ldg));
    TGB_TRY(xb.ensure((size_t)n * Dp));
    TGB_TRY(em.ensure(n));
    TGB_TRY(es.ensure(n));
    TGB_CUDA(cudaMemcpyAsync(x.p, delta, sizeof(float) * n * D, cudaMemcpyHostToDevice, C.st));
    k_rows_to_bf16<<<grid_for((int64_t)n * Dp), 256, 0, C.st>>>(n, D, Dp, x.p, xb.p);
    TGB_CUDA(cudaGetLastError());
    std::unique_ptr<MlpInferWork, void (*)(MlpInferWork *)> iw(mlp_infer_work_new(),
                                                                mlp_infer_work_delete);
    TGB_TRY(mlp_infer(m, *iw, n, xb.p, Dp, em.p, es.p, g.p, ldg, nullptr, C.st));
    TGB_TRY(mlp_check_err(m, C.st));
    TGB_CUDA(cudaMemcpyAsync(energy_mean, em.p, sizeof(double) * n, cudaMemcpyDeviceToHost, C.st));
    if (energy_std)
        TGB_CUDA(cudaMemcpyAsync(energy_std, es.p, sizeof(double) * n, cudaMemcpyDeviceToHost, C.st));
    std::vector<float> gh;
    if (dedq_mean) {
        gh.resize((size_t)n * ldg);
        TGB_CUDA(cudaMemcpyAsync(gh.data(), g.p, sizeof(float) * n * ldg, cudaMemcpyDeviceToHost, C.st));
    }
    TGB_CUDA(cudaStreamSynchronize(C.st));
    if (dedq_mean)
        for (int r = 0; r < n; ++r)
            for (int d = 0; d < D; ++d) dedq_mean[(size_t)r * D + d] = gh[(size_t)r * ldg + d];
    return TG_OK;
}

int tg_engine_set_mlp(tg_engine *eh, int32_t block, tg_mlp *h, double gate_ev) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    TGB_CHECK(block >= 0 && block < (int)E.runs.size(), TG_ERR_ARG, "block %d out of range", block);
    BlockRun &r = *E.runs[block];
    TGB_TRY(engine_errors(E));
    if (E.graph) {   // the captured step no longer matches
        cudaGraphExecDestroy(E.graph);
        E.graph = nullptr;
    }
    if (!h) {
        r.mix.reset();
        return TG_OK;
    }
    TGB_CHECK(h->m->L.D == r.b->dim, TG_ERR_ARG, "MLP input size %d does not match block dim %d",
              h->m->L.D, r.b->dim);
    TGB_CHECK(h->m->infer_ready, TG_ERR_STATE, "MLP has no inference weights");
    TGB_CHECK(gate_ev >= 0.0, TG_ERR_ARG, "negative gate");
    r.mix = std::make_unique<MixedRun>();
    r.mix->mlp = h->m;
    r.mix->iw = mlp_infer_work_new();
    r.mix->gate = gate_ev;
    TGB_TRY(r.mix->ensure(*r.b, r.n_sites));
    return TG_OK;
}

int tg_engine_mlp_stats(tg_engine *eh, int32_t block, int32_t *n_gated, int32_t *n_sites) {
    TGB_CHECK(eh, TG_ERR_ARG, "null engine");
    Engine &E = eh->e;
    TGB_CHECK(block >= 0 && block < (int)E.runs.size(), TG_ERR_ARG, "block %d out of range", block);
    BlockRun &r = *E.runs[block];
    if (n_sites) *n_sites = r.n_sites;
    if (n_gated) {
        *n_gated = r.n_sites;
        if (r.mix) {
            TGB_CUDA(cudaMemcpyAsync(n_gated, r.mix->gcount.p, sizeof(int), cudaMemcpyDeviceToHost, E.st));
            TGB_CUDA(cudaStreamSynchronize(E.st));
        }
    }
    return TG_OK;
}

}  // extern "C"

// ============================================================== batches
// Many independent orthorhombic structures evaluated together (energies, forces
// and a virial per structure): one batched neighbour list over all of them, then
// every block's kernels over the concatenated central sites, all in one CUDA
// graph after the first evaluation.
namespace tgb {

struct BatchEngine {
    int n = 0, ns = 0, nz = 1;
    double rcut = 0.0;
    DBuf<double> pos, f, en, vir, vir_s, e0, xyz, cell_pos;
    DBuf<int> species, atom_struct, cell_id, cell_count, cell_start, cell_fill, cell_atoms, n_neigh,
        nbr, snbr, ovf;
    DBuf<double> sxyz;
    DBuf<int64_t> pstart;
    DBuf<BatchStruct> sdev;
    DBuf<char> scan_tmp;
    DBuf<unsigned> err;
    DBuf<signed char> nsp;     // per-pair neighbour species (launch_pair_species)
    BatchNL nl;
    std::vector<std::unique_ptr<BlockRun>> runs;
    std::vector<int> n_atoms_h;
    cudaStream_t st = nullptr;
    cudaGraphExec_t graph = nullptr;

    ~BatchEngine() {
        if (graph) cudaGraphExecDestroy(graph);
        if (st) cudaStreamDestroy(st);
    }

    EventLog prof;

    int autotune() {
        if (pinned_tile() >= 0)
            for (auto &r : runs) pin_tiles(*r->b, *r->w, pinned_tile());
        if (!autotune_enabled()) return TG_OK;
        TGB_TRY(batch_nl_build(nl, pos.p, rcut, st));
        TGB_TRY(launch_pair_species(nl.pstart + n, nl.cap, nl.nbr, species.p, n, nsp.p, st));
        TGB_CUDA(cudaMemsetAsync(f.p, 0, sizeof(double) * 3 * n, st));
        TGB_CUDA(cudaMemsetAsync(en.p, 0, sizeof(double) * n, st));
        TGB_CUDA(cudaMemsetAsync(vir.p, 0, sizeof(double) * 9, st));
        for (auto &r : runs) {
            SiteArgs S{r->n_sites, r->sites.p, r->sites.p, nl.pstart, nl.nbr, nl.xyz, species.p};
            S.nsp = nsp.p;
            TGB_TRY(autotune_block(*r->b, *r->w, S, n, f.p, en.p, vir.p, err.p, st));
        }
        TGB_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }

    int compute_ef(EventLog *log = nullptr) {
        TGB_MARK(log, -1, st);
        TGB_TRY(batch_nl_build(nl, pos.p, rcut, st));
        TGB_TRY(launch_pair_species(nl.pstart + n, nl.cap, nl.nbr, species.p, n, nsp.p, st));
        TGB_MARK(log, PASS_NEIGH, st);
        k_energy_e0<<<grid_for(n), 256, 0, st>>>(n, species.p, e0.p, nz, 0, n, en.p);
        TGB_CUDA(cudaMemsetAsync(f.p, 0, sizeof(double) * 3 * n, st));
        TGB_CUDA(cudaMemsetAsync(vir.p, 0, sizeof(double) * 9, st));
        TGB_CUDA(cudaMemsetAsync(vir_s.p, 0, sizeof(double) * 9 * ns, st));
        for (auto &r : runs) {
            SiteArgs S{r->n_sites, r->sites.p, r->sites.p, nl.pstart, nl.nbr, nl.xyz, species.p};
            S.nsp = nsp.p;
            TGB_TRY(evaluate_block(*r->b, *r->w, S, n, f.p, en.p, vir.p, err.p, st, log,
                                   atom_struct.p, vir_s.p));
        }
        return TG_OK;
    }

    int errors() {
        unsigned e1 = 0, e2 = 0;
        TGB_CUDA(cudaMemcpyAsync(&e1, err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaMemcpyAsync(&e2, nl.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaStreamSynchronize(st));
        if (!(e1 | e2)) return TG_OK;
        TGB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), st));
        TGB_CUDA(cudaMemsetAsync(nl.err, 0, sizeof(unsigned), st));
        set_error("device error word 0x%x%s", e1 | e2,
                  (e2 & DEV_ERR_NEIGH_CAPACITY) ? " (neighbour pair capacity exceeded)" : "");
        return (e1 & (DEV_ERR_TIMEOUT_TMA | DEV_ERR_TIMEOUT_MMA | DEV_ERR_TIMEOUT_EPI)) ? TG_ERR_TIMEOUT
                                                                                        : TG_ERR_DEVICE;
    }

    // pair arrays sized from a counting build (with 25 % headroom for moved atoms)
    int size_pairs() {
        nl.cap = 0;
        TGB_TRY(batch_nl_build(nl, pos.p, rcut, st));
        int64_t P = 0;
        TGB_CUDA(cudaMemcpyAsync(&P, nl.pstart + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        TGB_CUDA(cudaStreamSynchronize(st));
        const int64_t cap = P + P / 4 + 64;
        TGB_TRY(nbr.ensure(cap));
        TGB_TRY(xyz.ensure(3 * (size_t)cap));
        TGB_TRY(nsp.ensure(cap));
        nl.nbr = nbr.p;
        nl.xyz = xyz.p;
        nl.cap = cap;
        // slot rows of the one-pass build: the largest count with 25 % headroom
        // (an atom that outgrows them sends that build to the second search)
        std::vector<int> cnt(n);
        TGB_CUDA(cudaMemcpyAsync(cnt.data(), nl.n_neigh, sizeof(int) * n, cudaMemcpyDeviceToHost,
                                 st));
        TGB_CUDA(cudaStreamSynchronize(st));
        int mx = 1;
        for (int c : cnt) mx = std::max(mx, c);
        int slots = (mx + mx / 4 + 8 + 15) / 16 * 16;
        // TGB_BATCH_SLOTS=s sets the rows (0: the two-pass build), e.g. to make
        // the overflow fallback run
        if (const char *e = std::getenv("TGB_BATCH_SLOTS")) slots = std::max(0, std::atoi(e));
        nl.slots = 0;
        if (slots > 0 && slots <= 256) {
            TGB_TRY(snbr.ensure((size_t)n * slots));
            TGB_TRY(sxyz.ensure((size_t)3 * n * slots));
            TGB_TRY(ovf.ensure(1));
            nl.snbr = snbr.p;
            nl.sxyz = sxyz.p;
            nl.ovf = ovf.p;
            nl.slots = slots;
        }
        TGB_CUDA(cudaMemsetAsync(nl.err, 0, sizeof(unsigned), st));
        TGB_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }
};

}  // namespace tgb

struct tg_batch {
    tgb::BatchEngine e;
};

extern "C" {

int tg_batch_create(int32_t n_structs, const int32_t *n_atoms, const double *positions,
                    const int32_t *species, const double *boxes, int32_t n_blocks,
                    const int32_t *block_keys, const double *e0_by_species,
                    int32_t n_species_total, tg_batch **out) {
    NvtxRange nvtx_range("tg_batch_create");
    TGB_TRY(need_ctx());
    TGB_CHECK(out && n_structs >= 1 && n_atoms && positions && species && boxes && n_blocks >= 1 &&
                  block_keys,
              TG_ERR_ARG, "bad batch arguments");
    Context &C = *g_ctx;
    auto holder = std::make_unique<tg_batch>();
    BatchEngine &E = holder->e;
    TGB_CUDA(cudaStreamCreateWithFlags(&E.st, cudaStreamNonBlocking));
    double rcut = 0.0;
    for (int k = 0; k < n_blocks; ++k) {
        auto it = C.blocks.find(block_keys[k]);
        TGB_CHECK(!C.families.count(block_keys[k]), TG_ERR_ARG,
                  "key %d is a 2b/3b/core_pot family: batches take soap_turbo blocks", block_keys[k]);
        TGB_CHECK(it != C.blocks.end(), TG_ERR_STATE, "block key %d was never begun", block_keys[k]);
        rcut = std::max(rcut, it->second->rcut_max);
    }
    E.rcut = rcut;
    E.ns = n_structs;
    std::vector<BatchStruct> sh(n_structs);
    std::vector<int> as;
    int off = 0, ncells = 0, ncell_atoms = 0;
    for (int s = 0; s < n_structs; ++s) {
        const double *bx = boxes + 9 * (size_t)s;
        TGB_CHECK(n_atoms[s] >= 1, TG_ERR_ARG, "structure %d has no atoms", s);
        const Box b = make_box(bx, bx + 3, bx + 6);
        TGB_CHECK(b.ortho, TG_ERR_ARG, "structure %d: batches take orthorhombic boxes", s);
        BatchStruct &q = sh[s];
        q.off = off;
        q.n = n_atoms[s];
        for (int k = 0; k < 3; ++k) q.L[k] = b.L[k];
        q.coff = ncells;
        ncells += batch_plan_struct(q, rcut);
        if (q.mode == 0) ncell_atoms += q.n;
        for (int i = 0; i < q.n; ++i) as.push_back(s);
        off += q.n;
    }
    E.n = off;
    E.n_atoms_h.assign(n_atoms, n_atoms + n_structs);
    const int n = E.n;
    const size_t n3 = 3 * (size_t)n;
    cudaStream_t st = E.st;
    TGB_TRY(E.pos.ensure(n3)); TGB_TRY(E.f.ensure(n3)); TGB_TRY(E.en.ensure(n));
    TGB_TRY(E.vir.ensure(9)); TGB_TRY(E.vir_s.ensure(9 * (size_t)n_structs));
    TGB_TRY(E.species.ensure(n)); TGB_TRY(E.atom_struct.ensure(n)); TGB_TRY(E.err.ensure(1));
    TGB_TRY(E.sdev.ensure(n_structs)); TGB_TRY(E.cell_id.ensure(n)); TGB_TRY(E.n_neigh.ensure(n));
    TGB_TRY(E.pstart.ensure((size_t)n + 1));
    const int nc = std::max(ncells, 1);
    TGB_TRY(E.cell_count.ensure(nc)); TGB_TRY(E.cell_start.ensure(nc));
    TGB_TRY(E.cell_fill.ensure(nc)); TGB_TRY(E.cell_atoms.ensure(n));
    TGB_TRY(E.cell_pos.ensure(3 * (size_t)n));
    size_t need1 = 0, need2 = 0;
    cub::DeviceScan::InclusiveSum(nullptr, need1, E.n_neigh.p, E.pstart.p + 1, n);
    cub::DeviceScan::ExclusiveSum(nullptr, need2, E.cell_count.p, E.cell_start.p, nc);
    TGB_TRY(E.scan_tmp.ensure(std::max(need1, need2)));
    E.nz = std::max(n_species_total, 1);
    TGB_TRY(E.e0.ensure(E.nz));
    std::vector<double> e0(E.nz, 0.0);
    if (e0_by_species)
        for (int z = 0; z < n_species_total; ++z) e0[z] = e0_by_species[z];
    TGB_CUDA(cudaMemcpyAsync(E.pos.p, positions, sizeof(double) * n3, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.species.p, species, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.atom_struct.p, as.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.sdev.p, sh.data(), sizeof(BatchStruct) * n_structs,
                             cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemcpyAsync(E.e0.p, e0.data(), sizeof(double) * E.nz, cudaMemcpyHostToDevice, st));
    TGB_CUDA(cudaMemsetAsync(E.err.p, 0, sizeof(unsigned), st));
    BatchNL &nl = E.nl;
    nl.n_atoms = n;
    nl.n_structs = n_structs;
    nl.n_cells = ncells;
    nl.st = E.sdev.p;
    nl.atom_struct = E.atom_struct.p;
    nl.cell_id = E.cell_id.p;
    nl.cell_count = E.cell_count.p;
    nl.cell_start = E.cell_start.p;
    nl.cell_fill = E.cell_fill.p;
    nl.cell_atoms = E.cell_atoms.p;
    nl.cell_pos = E.cell_pos.p;
    nl.n_cell_atoms = ncell_atoms;
    nl.n_neigh = E.n_neigh.p;
    nl.pstart = E.pstart.p;
    nl.scan_tmp = E.scan_tmp.p;
    nl.scan_bytes = E.scan_tmp.n;
    nl.err = E.err.p;
    for (int k = 0; k < n_blocks; ++k) {
        Block *b = C.blocks[block_keys[k]].get();
        auto run = std::make_unique<BlockRun>();
        run->b = b;
        run->w = std::make_unique<Workspace>();
        std::vector<int> sites;
        for (int i = 0; i < n; ++i) {
            const int z = species[i];
            int first = 0;
            for (int q = 0; q < b->ns; ++q)
                if (b->hh.species_z[q] == z) { first = q + 1; break; }
            if (b->hh.central_species == 0 || first == b->hh.central_species) sites.push_back(i);
        }
        run->n_sites = (int)sites.size();
        TGB_TRY(run->sites.ensure(sites.size()));
        if (!sites.empty())
            TGB_CUDA(cudaMemcpyAsync(run->sites.p, sites.data(), sizeof(int) * sites.size(),
                                     cudaMemcpyHostToDevice, st));
        TGB_TRY(run->w->ensure(*b, run->n_sites));
        E.runs.push_back(std::move(run));
    }
    TGB_TRY(E.size_pairs());
    TGB_TRY(E.autotune());
    TGB_TRY(E.errors());
    *out = holder.release();
    return TG_OK;
}

int tg_batch_destroy(tg_batch *b) {
    if (!b) return TG_OK;
    cudaStreamSynchronize(b->e.st);
    delete b;
    return TG_OK;
}

int tg_batch_set_positions(tg_batch *bh, const double *positions) {
    TGB_CHECK(bh && positions, TG_ERR_ARG, "null argument");
    BatchEngine &E = bh->e;
    TGB_CUDA(cudaMemcpyAsync(E.pos.p, positions, sizeof(double) * 3 * E.n, cudaMemcpyHostToDevice,
                             E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

// Evaluation without copies out: the first call runs eagerly, later calls replay
// one CUDA graph of the whole evaluation.
int tg_batch_compute_device(tg_batch *bh) {
    NvtxRange nvtx_range("tg_batch_compute_device");
    TGB_CHECK(bh, TG_ERR_ARG, "null batch");
    BatchEngine &E = bh->e;
    if (!E.graph) {
        TGB_TRY(E.compute_ef());
        TGB_TRY(E.errors());
        cudaGraph_t gr;
        TGB_CUDA(cudaStreamBeginCapture(E.st, cudaStreamCaptureModeThreadLocal));
        int r = E.compute_ef();
        cudaError_t ce = cudaStreamEndCapture(E.st, &gr);
        TGB_TRY(r);
        TGB_CUDA(ce);
        ce = cudaGraphInstantiate(&E.graph, gr, 0);
        cudaGraphDestroy(gr);
        TGB_CUDA(ce);
        return TG_OK;
    }
    TGB_CUDA(cudaGraphLaunch(E.graph, E.st));
    return TG_OK;
}

int tg_batch_compute(tg_batch *bh, double *energies, double *forces, double *virials) {
    NvtxRange nvtx_range("tg_batch_compute");
    TGB_CHECK(bh, TG_ERR_ARG, "null batch");
    BatchEngine &E = bh->e;
    TGB_TRY(tg_batch_compute_device(bh));
    if (energies)
        TGB_CUDA(cudaMemcpyAsync(energies, E.en.p, sizeof(double) * E.n, cudaMemcpyDeviceToHost, E.st));
    if (forces)
        TGB_CUDA(cudaMemcpyAsync(forces, E.f.p, sizeof(double) * 3 * E.n, cudaMemcpyDeviceToHost, E.st));
    if (virials)
        TGB_CUDA(cudaMemcpyAsync(virials, E.vir_s.p, sizeof(double) * 9 * E.ns, cudaMemcpyDeviceToHost,
                                 E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return E.errors();
}

int tg_batch_stream(tg_batch *bh, void **stream) {
    TGB_CHECK(bh && stream, TG_ERR_ARG, "null argument");
    *stream = (void *)bh->e.st;
    return TG_OK;
}

int tg_batch_profile(tg_batch *bh, int32_t n_evals, double *ms_per_pass, int32_t *n_passes) {
    NvtxRange nvtx_range("tg_batch_profile");
    TGB_CHECK(bh && ms_per_pass && n_evals >= 1, TG_ERR_ARG, "bad profile arguments");
    BatchEngine &E = bh->e;
    double acc[N_PASS] = {0};
    for (int s = 0; s < n_evals; ++s) {
        TGB_TRY(E.compute_ef(&E.prof));
        TGB_CUDA(cudaStreamSynchronize(E.st));
        TGB_TRY(E.prof.collect(acc));
    }
    for (int p = 0; p < N_PASS; ++p) ms_per_pass[p] = acc[p] / n_evals;
    if (n_passes) *n_passes = N_PASS;
    return E.errors();
}

int tg_batch_graph_kernels(tg_batch *bh, int32_t *n_kernels) {
    TGB_CHECK(bh && n_kernels, TG_ERR_ARG, "null argument");
    BatchEngine &E = bh->e;
    cudaGraph_t g;
    TGB_CUDA(cudaStreamBeginCapture(E.st, cudaStreamCaptureModeThreadLocal));
    int r = E.compute_ef();
    cudaError_t ce = cudaStreamEndCapture(E.st, &g);
    TGB_TRY(r);
    TGB_CUDA(ce);
    size_t n = 0;
    ce = cudaGraphGetNodes(g, nullptr, &n);
    std::vector<cudaGraphNode_t> nodes(n);
    if (ce == cudaSuccess && n) ce = cudaGraphGetNodes(g, nodes.data(), &n);
    int k = 0;
    for (size_t i = 0; ce == cudaSuccess && i < n; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    cudaGraphDestroy(g);
    TGB_CUDA(ce);
    *n_kernels = k;
    return TG_OK;
}

int tg_batch_tiles(tg_batch *bh, int32_t *tiles, int32_t n, int32_t *n_blocks) {
    TGB_CHECK(bh && tiles && n_blocks, TG_ERR_ARG, "null argument");
    BatchEngine &E = bh->e;
    TGB_CHECK(n >= 2 * (int)E.runs.size(), TG_ERR_CAPACITY, "tiles needs %d entries",
              2 * (int)E.runs.size());
    *n_blocks = (int32_t)E.runs.size();
    for (size_t k = 0; k < E.runs.size(); ++k) {
        tiles[2 * k] = E.runs[k]->w->tile_desc;
        tiles[2 * k + 1] = E.runs[k]->w->tile_force;
    }
    return TG_OK;
}

int tg_batch_n_pairs(tg_batch *bh, int64_t *n_pairs) {
    TGB_CHECK(bh && n_pairs, TG_ERR_ARG, "null argument");
    BatchEngine &E = bh->e;
    TGB_CUDA(cudaMemcpyAsync(n_pairs, E.nl.pstart + E.n, sizeof(int64_t), cudaMemcpyDeviceToHost, E.st));
    TGB_CUDA(cudaStreamSynchronize(E.st));
    return TG_OK;
}

}  // extern "C"

// ============================================================== test-only
#include "../../include/tgb200_test.h"

extern "C" int tgx_gemm_bf16_tn(int32_t M, int32_t N, int32_t K, const uint16_t *A,
                                const uint16_t *B, float *Cout) {
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(M > 0 && N > 0 && K > 0 && K % kGemmBK == 0, TG_ERR_ARG, "bad GEMM shape");
    DBuf<__nv_bfloat16> a, b;
    DBuf<float> c;
    TGB_TRY(a.ensure((size_t)M * K));
    TGB_TRY(b.ensure((size_t)N * K));
    TGB_TRY(c.ensure((size_t)M * N));
    TGB_CUDA(cudaMemcpyAsync(a.p, A, sizeof(uint16_t) * M * K, cudaMemcpyHostToDevice, C.st));
    TGB_CUDA(cudaMemcpyAsync(b.p, B, sizeof(uint16_t) * N * K, cudaMemcpyHostToDevice, C.st));
    TGB_CUDA(cudaMemsetAsync(c.p, 0, sizeof(float) * M * N, C.st));
    TmaMap ta{}, tb{}, tl{};
    TGB_TRY(make_tma_bf16(&ta, a.p, M, K, K, kGemmBM));
    TGB_TRY(make_tma_bf16(&tb, b.p, N, K, K, kGemmBN));
    const int lr = gemm_last_box_rows(N);   // the short last column tile, as the blocks run it
    if (lr) TGB_TRY(make_tma_bf16(&tl, b.p, N, K, K, lr));
    GemmEpi ep{};
    ep.mode = EPI_STORE_F32;
    ep.rows = M;
    ep.cols = N;
    ep.out = c.p;
    ep.ldo = N;
    TGB_TRY(launch_gemm_tn(ta, tb, M, N, K, ep, C.err.p, C.st, nullptr, lr ? &tl : nullptr));
    TGB_TRY(check_err_word(C, C.err.p));
    TGB_CUDA(cudaMemcpyAsync(Cout, c.p, sizeof(float) * M * N, cudaMemcpyDeviceToHost, C.st));
    TGB_CUDA(cudaStreamSynchronize(C.st));
    return TG_OK;
}

// The GEMM with its producer silenced: the MMA issuer's first bounded wait
// (2 s) runs out, every role leaves, TMEM is freed and the call returns
// TG_ERR_TIMEOUT with the device error word in *err_word; nothing faults and
// the context stays usable.
extern "C" int tgx_gemm_stall_probe(int32_t M, int32_t N, int32_t K, uint32_t *err_word) {
    TGB_TRY(need_ctx());
    Context &C = *g_ctx;
    TGB_CHECK(M > 0 && N > 0 && K > 0 && K % kGemmBK == 0 && err_word, TG_ERR_ARG,
              "bad GEMM shape");
    DBuf<__nv_bfloat16> a, b;
    DBuf<float> c;
    TGB_TRY(a.ensure((size_t)M * K));
    TGB_TRY(b.ensure((size_t)N * K));
    TGB_TRY(c.ensure((size_t)M * N));
    TGB_CUDA(cudaMemsetAsync(a.p, 0, sizeof(__nv_bfloat16) * M * K, C.st));
    TGB_CUDA(cudaMemsetAsync(b.p, 0, sizeof(__nv_bfloat16) * N * K, C.st));
    TmaMap ta{}, tb{};
    TGB_TRY(make_tma_bf16(&ta, a.p, M, K, K, kGemmBM));
    TGB_TRY(make_tma_bf16(&tb, b.p, N, K, K, kGemmBN));
    GemmEpi ep{};
    ep.mode = EPI_STORE_F32;
    ep.rows = M;
    ep.cols = N;
    ep.out = c.p;
    ep.ldo = N;
    ep.stall_test = 1;
    TGB_TRY(launch_gemm_tn(ta, tb, M, N, K, ep, C.err.p, C.st));
    unsigned e = 0;
    TGB_CUDA(cudaMemcpyAsync(&e, C.err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, C.st));
    TGB_CUDA(cudaStreamSynchronize(C.st));
    *err_word = e;
    return check_err_word(C, C.err.p);
}

extern "C" int tgx_mlp_batch_grads(tg_mlp *h, int32_t member, int32_t B, const float *x,
                                   const float *y, const float *gref, double lam, double *grads,
                                   double *loss, float *E, float *G) {
    TGB_TRY(need_ctx());
    TGB_CHECK(h, TG_ERR_ARG, "null MLP");
    return mlp_batch_grads(*h->m, member, B, x, y, gref, lam, grads, loss, E, G, g_ctx->st);
}

extern "C" int tgx_mlp_layout(tg_mlp *h, int64_t *offsets) {
    TGB_CHECK(h && offsets, TG_ERR_ARG, "null argument");
    const MlpLayout &L = h->m->L;
    const int64_t v[9] = {L.D, L.Dp, L.H, (int64_t)L.oW1, (int64_t)L.ob1, (int64_t)L.oW2,
                          (int64_t)L.ob2, (int64_t)L.ow3, (int64_t)L.ob3};
    for (int i = 0; i < 9; ++i) offsets[i] = v[i];
    return TG_OK;
}
