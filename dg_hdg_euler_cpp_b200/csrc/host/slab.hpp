// Communicators of the slab domain decomposition (dgh_comm_*, dgh_ctx_create_slab).
//
// The 2D mesh is split into slabs of whole cell rows, one per rank.  A slab context holds its
// rows plus one ghost row below and one above (local rows 0 and rows+1); a volume vector of the
// slab is (rows + 2) * row_len contiguous doubles, row_len = nx * 4 (k+1)^2.  A communicator
// provides the two exchanges the DG Newton update needs: the sum or maximum of a few doubles
// over all ranks (norms, Arnoldi coefficients, the CFL rate, status bits) and the halo exchange
// that fills a vector's ghost rows from the neighbouring slabs.  Two kinds exist:
//  - nccl:  one rank per process and GPU; collectives are NCCL calls on the caller's stream
//           (ncclAllReduce, grouped ncclSend/ncclRecv), libnccl resolved at run time;
//  - local: several ranks inside one process (one host thread each, any devices), exchanging
//           through host barriers after synchronising their streams, so that no kernel ever
//           waits on another rank's kernel.  Several slabs on one GPU test the decomposition.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

// A collective that could not complete: a peer failed, or did not arrive in time.
struct dgh_comm_failure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct dgh_comm {
    int rank = 0, size = 1;
    virtual ~dgh_comm() = default;
    virtual const char *kind() const = 0;
    // In place over all ranks: op 0 sums, op 1 takes the maximum of count doubles at dev; ordered
    // on stream.  Every rank receives the same bits.
    virtual void allreduce(double *dev, int count, int op, cudaStream_t stream) = 0;
    // Fills the ghost rows of a slab vector: local row 0 from the top interior row of the rank
    // below, local row rows+1 from the bottom interior row of the rank above (periodic in rank).
    virtual void halo(double *vec, long long row_len, int rows, cudaStream_t stream) = 0;
    // Marks the group failed so that peers waiting in (or entering) a collective end with an error.
    virtual void fail(const std::string &why) noexcept = 0;
};

namespace dgh_slab {
// The rows of rank `rank`: ny = size * base + extra; the first `extra` ranks take base + 1.
inline void rows_of(int ny, int size, int rank, int &row0, int &rows) {
    const int base = ny / size, extra = ny % size;
    rows = base + (rank < extra ? 1 : 0);
    row0 = rank * base + (rank < extra ? rank : extra);
}
}  // namespace dgh_slab
