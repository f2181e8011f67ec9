/* A stand-in for the NCCL entry points the backend loads, for failure tests
 * on CPU ranks. Communicator initialisation is non-blocking: it reports
 * "in progress" until every rank of the communicator has called it, which the
 * ranks announce by creating a file rank_<r> in the directory $FAKE_NCCL_DIR.
 * A rank that never calls leaves the others in progress until their deadline.
 * Grouped collectives complete at once and move no data. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef int ncclResult_t;
enum { kSuccess = 0, kInvalidArgument = 4, kInProgress = 7 };
typedef struct { char internal[128]; } ncclUniqueId;
typedef struct FakeComm { int n, rank; } *ncclComm_t;

static int marker(int r, char *path, size_t len) {
    const char *dir = getenv("FAKE_NCCL_DIR");
    if (!dir) return -1;
    snprintf(path, len, "%s/rank_%d", dir, r);
    return 0;
}

ncclResult_t ncclGetUniqueId(ncclUniqueId *id) {
    memset(id, 0, sizeof(*id));
    strcpy(id->internal, "fake-nccl");
    return kSuccess;
}

ncclResult_t ncclCommInitRankConfig(ncclComm_t *comm, int n, ncclUniqueId id, int rank,
                                    void *config) {
    (void)id; (void)config;
    char path[4096];
    if (marker(rank, path, sizeof path) != 0) return kInvalidArgument;
    FILE *f = fopen(path, "w");
    if (!f) return kInvalidArgument;
    fclose(f);
    struct FakeComm *c = (struct FakeComm *)malloc(sizeof *c);
    c->n = n;
    c->rank = rank;
    *comm = c;
    return kInProgress;
}

ncclResult_t ncclCommGetAsyncError(ncclComm_t comm, ncclResult_t *state) {
    char path[4096];
    for (int r = 0; r < comm->n; ++r) {
        if (marker(r, path, sizeof path) != 0 || access(path, F_OK) != 0) {
            *state = kInProgress;
            return kSuccess;
        }
    }
    *state = kSuccess;
    return kSuccess;
}

ncclResult_t ncclCommAbort(ncclComm_t comm) { free(comm); return kSuccess; }
ncclResult_t ncclCommDestroy(ncclComm_t comm) { free(comm); return kSuccess; }
ncclResult_t ncclAllReduce(const void *s, void *r, size_t n, int t, int op, ncclComm_t c,
                           void *stream) {
    (void)s; (void)r; (void)n; (void)t; (void)op; (void)c; (void)stream;
    return kSuccess;
}
ncclResult_t ncclGroupStart(void) { return kSuccess; }
ncclResult_t ncclGroupEnd(void) { return kSuccess; }
const char *ncclGetErrorString(ncclResult_t r) { return r == kSuccess ? "success" : "fake error"; }
