// tgb_comm.cu -- NCCL communicator of a sharded engine (host code).
//
// NCCL is resolved with dlopen/dlsym, so libtgb200.so has no link-time
// dependency on it. The communicator is non-blocking: initialisation and each
// grouped all-reduce are polled on the host with a deadline (default 120 s,
// TGB_NCCL_TIMEOUT_S), after which the communicator is aborted and the call
// returns TG_ERR_TIMEOUT instead of waiting for a rank that never arrives.
// TGB_NCCL_LIBRARY selects the library to load (default libnccl.so.2).
#include "tgb_comm.cuh"
#include "tgb_common.cuh"

#include <nccl.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <thread>

namespace tgb {
namespace {

struct NcclApi {
    void *h = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
    ncclResult_t (*init_rank_config)(ncclComm_t *, int, ncclUniqueId, int, ncclConfig_t *) = nullptr;
    ncclResult_t (*get_async_error)(ncclComm_t, ncclResult_t *) = nullptr;
    ncclResult_t (*abort)(ncclComm_t) = nullptr;
    ncclResult_t (*destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t,
                               ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    const char *(*error_string)(ncclResult_t) = nullptr;
};

NcclApi g_api;
std::mutex g_api_mu;

template <typename F>
bool sym(void *h, const char *name, F &f) {
    f = reinterpret_cast<F>(dlsym(h, name));
    return f != nullptr;
}

int api(NcclApi **out) {
    std::lock_guard<std::mutex> lk(g_api_mu);
    if (!g_api.h) {
        void *h = nullptr;
        // TGB_NCCL_LIBRARY names another build of the library (a path or a soname)
        if (const char *lib = std::getenv("TGB_NCCL_LIBRARY")) {
            h = dlopen(lib, RTLD_NOW | RTLD_GLOBAL);
            TGB_CHECK(h, TG_ERR_STATE, "NCCL library %s could not be loaded: %s", lib, dlerror());
        }
        for (const char *name : {"libnccl.so.2", "libnccl.so"})
            if (h || (h = dlopen(name, RTLD_NOW | RTLD_GLOBAL))) break;
        TGB_CHECK(h, TG_ERR_STATE, "NCCL (libnccl.so.2) could not be loaded: %s", dlerror());
        NcclApi a;
        a.h = h;
        const bool ok = sym(h, "ncclGetUniqueId", a.get_unique_id) &&
                        sym(h, "ncclCommInitRankConfig", a.init_rank_config) &&
                        sym(h, "ncclCommGetAsyncError", a.get_async_error) &&
                        sym(h, "ncclCommAbort", a.abort) && sym(h, "ncclCommDestroy", a.destroy) &&
                        sym(h, "ncclAllReduce", a.all_reduce) &&
                        sym(h, "ncclGroupStart", a.group_start) &&
                        sym(h, "ncclGroupEnd", a.group_end) &&
                        sym(h, "ncclGetErrorString", a.error_string);
        TGB_CHECK(ok, TG_ERR_STATE, "the loaded NCCL lacks an entry point the backend needs");
        g_api = a;
    }
    *out = &g_api;
    return TG_OK;
}

double timeout_s() {
    const char *e = std::getenv("TGB_NCCL_TIMEOUT_S");
    const double t = e ? std::atof(e) : 0.0;
    return t > 0.0 ? t : 120.0;
}

}  // namespace

struct Comm {
    ncclComm_t c = nullptr;
    int n = 0, rank = 0;
};

// Polls a non-blocking communicator until its pending work is issued.
static int settle(NcclApi *a, Comm *c, ncclResult_t r, const char *what) {
    const auto t0 = std::chrono::steady_clock::now();
    const double lim = timeout_s();
    while (r == ncclInProgress) {
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > lim) {
            a->abort(c->c);
            c->c = nullptr;
            set_error("NCCL %s did not complete within %.0f s (communicator aborted)", what, lim);
            return TG_ERR_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
        if (a->get_async_error(c->c, &r) != ncclSuccess) break;
    }
    TGB_CHECK(r == ncclSuccess, TG_ERR_DEVICE, "NCCL %s: %s", what, a->error_string(r));
    return TG_OK;
}

int comm_unique_id(void *id128) {
    TGB_CHECK(id128, TG_ERR_ARG, "null id buffer");
    NcclApi *a = nullptr;
    TGB_TRY(api(&a));
    ncclUniqueId id;
    const ncclResult_t r = a->get_unique_id(&id);
    TGB_CHECK(r == ncclSuccess, TG_ERR_DEVICE, "ncclGetUniqueId: %s", a->error_string(r));
    static_assert(sizeof(id) == 128, "ncclUniqueId is 128 bytes");
    std::memcpy(id128, &id, sizeof(id));
    return TG_OK;
}

int comm_init(const void *id128, int n_ranks, int rank, Comm **out) {
    TGB_CHECK(id128 && out && n_ranks >= 1 && rank >= 0 && rank < n_ranks, TG_ERR_ARG,
              "bad communicator arguments (n_ranks %d, rank %d)", n_ranks, rank);
    NcclApi *a = nullptr;
    TGB_TRY(api(&a));
    ncclUniqueId id;
    std::memcpy(&id, id128, sizeof(id));
    ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
    cfg.blocking = 0;
    Comm *c = new Comm;
    c->n = n_ranks;
    c->rank = rank;
    const ncclResult_t r = a->init_rank_config(&c->c, n_ranks, id, rank, &cfg);
    if (r != ncclSuccess && r != ncclInProgress) {
        set_error("ncclCommInitRankConfig: %s", a->error_string(r));
        delete c;
        return TG_ERR_DEVICE;
    }
    const int s = settle(a, c, r, "communicator initialisation");
    if (s != TG_OK) {
        if (c->c) a->abort(c->c);
        delete c;
        return s;
    }
    *out = c;
    return TG_OK;
}

void comm_destroy(Comm *c) {
    if (!c) return;
    NcclApi *a = nullptr;
    if (c->c && api(&a) == TG_OK) {
        const ncclResult_t r = a->destroy(c->c);
        if (r == ncclInProgress) settle(a, c, r, "communicator destruction");
    }
    delete c;
}

int comm_size(const Comm *c) { return c ? c->n : 1; }

int comm_allreduce3(Comm *c, double *x, size_t nx, double *y, size_t ny, double *z, size_t nz,
                    cudaStream_t st) {
    TGB_CHECK(c && c->c, TG_ERR_STATE, "no live communicator");
    NcclApi *a = nullptr;
    TGB_TRY(api(&a));
    ncclResult_t r = a->group_start();
    TGB_CHECK(r == ncclSuccess, TG_ERR_DEVICE, "ncclGroupStart: %s", a->error_string(r));
    double *bufs[3] = {x, y, z};
    const size_t counts[3] = {nx, ny, nz};
    for (int k = 0; k < 3; ++k) {
        if (!counts[k]) continue;
        r = a->all_reduce(bufs[k], bufs[k], counts[k], ncclFloat64, ncclSum, c->c, st);
        if (r != ncclSuccess && r != ncclInProgress) {
            a->group_end();
            set_error("ncclAllReduce: %s", a->error_string(r));
            return TG_ERR_DEVICE;
        }
    }
    r = a->group_end();
    return settle(a, c, r, "all-reduce of forces, energies and virial");
}

}  // namespace tgb

// Failure test: a communicator of n_ranks, then one grouped all-reduce with no
// data, then its destruction, host code only (the deadline logic of a sharded
// engine's exchange step without a GPU). Returns the first failing status.
extern "C" int tgx_comm_probe(const void *id128, int32_t n_ranks, int32_t rank) {
    tgb::Comm *c = nullptr;
    int rc = tgb::comm_init(id128, n_ranks, rank, &c);
    if (rc != TG_OK) return rc;
    rc = tgb::comm_allreduce3(c, nullptr, 0, nullptr, 0, nullptr, 0, nullptr);
    tgb::comm_destroy(c);
    return rc;
}
