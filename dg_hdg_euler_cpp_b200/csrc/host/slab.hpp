// Communicators of the slab domain decomposition (dgh_comm_*, dgh_ctx_create_slab).
//
// The 2D mesh is split into slabs of whole cell rows, one per rank.  A slab context holds its
// rows plus ghost rows (one below; one above for the DG operator, two for HDG, whose top ghost
// cells are condensed and need their own upper faces).  A communicator provides the two
// exchanges a Newton update needs: the sum or maximum of a few doubles over all ranks (norms,
// Arnoldi coefficients, the CFL rate, status bits) and a halo exchange that copies regions of a
// vector between neighbouring slabs (ghost cell rows of a volume vector, ghost face rows of a
// trace vector).  Two kinds exist:
//  - nccl:  one rank per process and GPU; collectives are NCCL calls on the caller's stream
//           (ncclAllReduce, grouped ncclSend/ncclRecv), libnccl resolved at run time;
//  - local: several ranks inside one process (one host thread each, any devices), exchanging
//           through host barriers after synchronising their streams, so that no kernel ever
//           waits on another rank's kernel.  Several slabs on one GPU test the decomposition.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

// A collective that could not complete: a peer failed, or did not arrive in time.
struct dgh_comm_failure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// A region of a vector: `count` doubles from `offset`.
struct dgh_region {
    long long offset = 0, count = 0;
};
// Regions sent to the rank below and to the rank above, and regions received from the rank above
// and from the rank below, each list in order.
struct dgh_halo_plan {
    std::vector<dgh_region> to_below, to_above, from_above, from_below;
};

struct dgh_comm {
    int rank = 0, size = 1;
    virtual ~dgh_comm() = default;
    virtual const char *kind() const = 0;
    // In place over all ranks: op 0 sums, op 1 takes the maximum of count doubles at dev; ordered
    // on stream.  Every rank receives the same bits.
    virtual void allreduce(double *dev, int count, int op, cudaStream_t stream) = 0;
    // The halo exchange of one vector under `plan`: the i-th region sent to a neighbour lands in
    // that neighbour's i-th region received from this side (below and above are periodic in rank;
    // every rank uses a plan of the same shape).
    virtual void exchange(double *vec, const dgh_halo_plan &plan, cudaStream_t stream) = 0;
    // Marks the group failed so that peers waiting in (or entering) a collective end with an error.
    virtual void fail(const std::string &why) noexcept = 0;
    // How long a rank waits for its peers, in milliseconds (see the kinds' wait rules).
    virtual void set_timeout(int timeout_ms) = 0;
    // Waits for the work queued on `stream` (which may include this rank's collectives).  A CUDA
    // error is thrown as std::runtime_error; the NCCL kind gives up after its timeout (a peer that
    // never joins a collective), aborts its communicator so that its own NCCL kernels end, and
    // throws dgh_comm_failure.
    virtual void wait(cudaStream_t stream) {
        const cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) throw std::runtime_error(std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
    }
};

namespace dgh_slab {
// The rows of rank `rank`: ny = size * base + extra; the first `extra` ranks take base + 1.
inline void rows_of(int ny, int size, int rank, int &row0, int &rows) {
    const int base = ny / size, extra = ny % size;
    rows = base + (rank < extra ? 1 : 0);
    row0 = rank * base + (rank < extra ? rank : extra);
}
// The halo of a volume vector (row_len doubles per cell row; local row 0 the ghost row below,
// rows 1..rows the slab's, then `above` ghost rows): rows 1..above go to the rank below (its
// upper ghost rows), row `rows` to the rank above (its ghost row 0).
inline dgh_halo_plan volume_plan(long long row_len, int rows, int above) {
    const long long rl = row_len, R = rows, A = above;
    dgh_halo_plan p;
    p.to_below = {{rl, A * rl}};
    p.to_above = {{R * rl, rl}};
    p.from_above = {{(R + 1) * rl, A * rl}};
    p.from_below = {{0, rl}};
    return p;
}
// The halo of a trace vector (x faces, then y faces from y0; face_row doubles per face row; a
// face belongs to the cell left of or below it): row 1's x and upper y faces go to the rank below
// (its first ghost row above), row `rows`' upper y faces to the rank above (its ghost row 0's).
inline dgh_halo_plan trace_plan(long long face_row, long long y0, int rows) {
    const long long fr = face_row, R = rows;
    dgh_halo_plan p;
    p.to_below = {{fr, fr}, {y0 + fr, fr}};
    p.to_above = {{y0 + R * fr, fr}};
    p.from_above = {{(R + 1) * fr, fr}, {y0 + (R + 1) * fr, fr}};
    p.from_below = {{y0, fr}};
    return p;
}
}  // namespace dgh_slab
