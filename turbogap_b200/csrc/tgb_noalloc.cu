// tgb_noalloc.cu -- neighbour-list build for callers that cannot allocate.
//
// Some callers may not call cudaMalloc at all: a host that owns every device
// byte through its own arena (an OpenACC/OpenMP-offload Fortran driver, a
// framework with a pooled allocator), or code running under a memory budget
// where allocation during the time step is forbidden. They hand in their own
// input and output buffers and need the library to allocate nothing.
//
// tg_build_neighbors_list_noalloc runs the same cell-list kernels as
// tg_build_neighbors_list, but its scratch (cell grid, cell member lists, the
// prefix-scan workspace, the error word) lives in one file-scope __device__
// array of fixed size, allocated once per GPU when the module is loaded and
// held until the process exits. Limits: kNoAllocMaxSites sites and
// kNoAllocMaxCells cells. Orthorhombic boxes of at least 2 rcut (the cell path)
// only.
//
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress (and sizes the scan workspace); make that first call
// outside any stream capture. Under lazy module loading (the CUDA 12 default)
// that first call is also what loads this file's module, and with it the
// array and the kernels: the device memory they take appears then, once per
// device, and no later call changes it. Every call shares the array and leaves its
// contents behind, so the counters that must start at zero are cleared on each
// call; calls that overlap on the GPU (different streams, or another thread)
// race on the shared array and must be serialised by the caller.

#include "tgb_neighbors.cuh"

#include <cub/device/device_scan.cuh>

#include <cmath>
#include <mutex>

namespace tgb {
namespace {

constexpr int kNoAllocMaxSites = 131072;
constexpr int kNoAllocMaxCells = 131072;
constexpr size_t kScanBytes = 1u << 20;   // prefix-scan workspace (checked at set-up)

// Byte layout of the scratch array (each region 256-byte aligned).
constexpr size_t al256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffCellXyz = 0;
constexpr size_t kOffCellCount = kOffCellXyz + al256(3 * sizeof(int) * kNoAllocMaxSites);
constexpr size_t kOffCellStart = kOffCellCount + al256(sizeof(int) * kNoAllocMaxCells);
constexpr size_t kOffCellFill = kOffCellStart + al256(sizeof(int) * (kNoAllocMaxCells + 1));
constexpr size_t kOffCellAtoms = kOffCellFill + al256(sizeof(int) * kNoAllocMaxCells);
constexpr size_t kOffErr = kOffCellAtoms + al256(sizeof(int) * kNoAllocMaxSites);
constexpr size_t kOffScan = kOffErr + 256;
constexpr size_t kScratchBytes = kOffScan + kScanBytes;   // about 4.2 MB

static __device__ __align__(256) unsigned char g_nl_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_dev[kMaxDevices] = {};

__global__ void k_to_one_based(int64_t n, int *__restrict__ v) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] += 1;
}

// Device address of the scratch array on the current device (set-up on first use).
int scratch_for_current_device(unsigned char **out) {
    int dev = 0;
    TGB_CUDA(cudaGetDevice(&dev));
    TGB_CHECK(dev >= 0 && dev < kMaxDevices, TG_ERR_ARG, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        void *p = nullptr;
        TGB_CUDA(cudaGetSymbolAddress(&p, g_nl_scratch));
        cudaFuncAttributes fa;   // loads the module's kernels now, not inside a later call
        TGB_CUDA(cudaFuncGetAttributes(&fa, k_to_one_based));
        // the scan workspace must fit its region for the largest sizes allowed
        size_t need_sites = 0, need_cells = 0;
        TGB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, need_sites, (const int *)nullptr,
                                               (int64_t *)nullptr, kNoAllocMaxSites));
        TGB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, need_cells, (const int *)nullptr,
                                               (int *)nullptr, kNoAllocMaxCells));
        TGB_CHECK(need_sites <= kScanBytes && need_cells <= kScanBytes, TG_ERR_STATE,
                  "scan workspace of %zu/%zu bytes exceeds the %zu-byte region", need_sites,
                  need_cells, kScanBytes);
        g_scratch_dev[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_dev[dev];
    return TG_OK;
}

}  // namespace
}  // namespace tgb

using namespace tgb;

extern "C" int tg_build_neighbors_list_noalloc(int32_t n_sites, const double *positions,
                                               const double *a_box, const double *b_box,
                                               const double *c_box, double rcut_max,
                                               int64_t cap, int32_t *n_neigh, int64_t *pstart,
                                               int32_t *neighbors_list, double *rjs, double *xyz,
                                               int64_t *n_pairs, void *stream) {
    TGB_CHECK(n_sites >= 1 && positions && n_neigh && pstart && neighbors_list && rjs && xyz &&
                  n_pairs && a_box && b_box && c_box,
              TG_ERR_ARG, "null or empty argument");
    TGB_CHECK(n_sites <= kNoAllocMaxSites, TG_ERR_CAPACITY,
              "%d sites exceed the no-allocation limit of %d (use tg_build_neighbors_list)",
              n_sites, kNoAllocMaxSites);
    TGB_CHECK(std::isfinite(rcut_max) && rcut_max > 0.0, TG_ERR_ARG,
              "rcut_max must be positive and finite (got %g)", rcut_max);
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) a[k] = a_box[k], b[k] = b_box[k], c[k] = c_box[k];
    for (int k = 0; k < 3; ++k)
        TGB_CHECK(std::isfinite(a[k]) && std::isfinite(b[k]) && std::isfinite(c[k]), TG_ERR_ARG,
                  "non-finite lattice vector component");
    TGB_CHECK(a[0] > 0.0 && b[1] > 0.0 && c[2] > 0.0, TG_ERR_ARG,
              "the no-allocation entry point takes orthorhombic boxes with positive edges");
    // Cells per axis are int(L / rcut) (neighbors.f90:391-396); bound them, and
    // their product, in floating point before any integer conversion, so that the
    // grid can never outgrow the fixed scratch array.
    {
        const double lx = std::fabs(a[0]) / rcut_max, ly = std::fabs(b[1]) / rcut_max,
                     lz = std::fabs(c[2]) / rcut_max;
        TGB_CHECK(lx <= kNoAllocMaxCells && ly <= kNoAllocMaxCells && lz <= kNoAllocMaxCells &&
                      std::floor(lx) * std::floor(ly) * std::floor(lz) <= (double)kNoAllocMaxCells,
                  TG_ERR_CAPACITY, "box / rcut_max gives more cells than the no-allocation limit of %d",
                  kNoAllocMaxCells);
    }
    Box bx = make_box(a, b, c);
    if (bx.ortho) {   // neighbors.f90:372-384: snap the off-diagonal noise to zero
        a[1] = a[2] = b[0] = b[2] = c[0] = c[1] = 0.0;
        bx = make_box(a, b, c);
    }
    const int one[3] = {1, 1, 1};
    int ind[3];
    host_unit_cells(a, b, c, rcut_max, ind);
    TGB_CHECK(bx.ortho && ind[0] == 1 && ind[1] == 1 && ind[2] == 1, TG_ERR_ARG,
              "the no-allocation entry point takes orthorhombic boxes of at least 2 rcut");
    bool use_cells = false;
    const CellGrid g = plan_cells(bx, rcut_max, one, &use_cells);
    TGB_CHECK(use_cells, TG_ERR_ARG, "box too small for the cell list");
    const int64_t ncells = (int64_t)g.mx * g.my * g.mz;
    TGB_CHECK(ncells <= kNoAllocMaxCells, TG_ERR_CAPACITY,
              "%lld cells exceed the no-allocation limit of %d", (long long)ncells,
              kNoAllocMaxCells);
    unsigned char *base = nullptr;
    TGB_TRY(scratch_for_current_device(&base));
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // A non-owning view: scratch from the static array, outputs from the caller.
    NeighborList nl;
    nl.cap = cap;
    nl.n_neigh = n_neigh;
    nl.pstart = pstart;
    nl.nbr = neighbors_list;
    nl.rjs = rjs;
    nl.xyz = xyz;
    nl.cell_xyz = reinterpret_cast<int *>(base + kOffCellXyz);
    nl.cell_count = reinterpret_cast<int *>(base + kOffCellCount);
    nl.cell_start = reinterpret_cast<int *>(base + kOffCellStart);
    nl.cell_fill = reinterpret_cast<int *>(base + kOffCellFill);
    nl.cell_atoms = reinterpret_cast<int *>(base + kOffCellAtoms);
    nl.err = reinterpret_cast<unsigned *>(base + kOffErr);
    nl.scan_tmp = base + kOffScan;
    nl.scan_bytes = kScanBytes;
    TGB_CUDA(cudaMemsetAsync(nl.err, 0, sizeof(unsigned), st));   // left over from the last call
    int rc = nl_build(nl, n_sites, n_sites, positions, bx, g, true, rcut_max, nullptr, st);
    if (rc != TG_OK) return rc;
    int64_t P = 0;
    unsigned err = 0;
    TGB_CUDA(cudaMemcpyAsync(&P, pstart + n_sites, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaMemcpyAsync(&err, nl.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    TGB_CUDA(cudaStreamSynchronize(st));
    *n_pairs = P;
    if (P > cap || (err & DEV_ERR_NEIGH_CAPACITY)) {
        set_error("neighbour arrays hold %lld pairs, %lld needed", (long long)cap, (long long)P);
        return TG_ERR_CAPACITY;
    }
    TGB_CHECK(err == 0, TG_ERR_DEVICE, "device error word 0x%x", err);
    if (P > 0) {
        k_to_one_based<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(P, neighbors_list);
        TGB_CUDA(cudaGetLastError());
        TGB_CUDA(cudaStreamSynchronize(st));
    }
    return TG_OK;
}
