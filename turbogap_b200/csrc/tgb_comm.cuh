// tgb_comm.cuh -- the force exchange of a sharded structure over NCCL.
//
// The reference splits central atoms over MPI ranks and sums per-atom energies,
// forces and the virial of every rank into every atom (turbogap.f90:930-942,
// 1876-1885). Here each GPU is one rank: its engine evaluates its own central
// sites, and one grouped NCCL all-reduce (sum) of forces, energies and the
// virial on the engine's stream replaces the MPI reduction. NCCL is loaded at
// run time (dlopen) the first time a communicator is made, so the library
// loads on hosts without it.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace tgb {

struct Comm;

// 128 opaque bytes that rank 0 makes and every rank passes to comm_init.
int comm_unique_id(void *id128);
// Collective over all n_ranks processes (each calls it with the same id).
int comm_init(const void *id128, int n_ranks, int rank, Comm **out);
void comm_destroy(Comm *c);
// In-place sums of three double buffers, grouped into one NCCL launch group.
int comm_allreduce3(Comm *c, double *a, size_t na, double *b, size_t nb, double *d, size_t nd,
                    cudaStream_t st);
int comm_size(const Comm *c);

}  // namespace tgb
