// Slab communicators (slab.hpp): the in-process group of ranks and the NCCL communicator, and
// their C ABI (dgh_comm_*, dgh_slab_rows in dgh_gpu.h).
#include "slab.hpp"

#include "dgh_gpu.h"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {
thread_local std::string g_comm_error;

void cuda_ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw dgh_comm_failure(std::string(what) + ": " + cudaGetErrorString(e));
}
double larger(double a, double b) { return (b > a || std::isnan(b)) ? b : a; }

// Copies one row between slab vectors that may live on different devices.
void copy_row(double *dst, int dst_dev, const double *src, int src_dev, size_t bytes, cudaStream_t st) {
    if (dst_dev == src_dev) cuda_ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st), "halo copy");
    else cuda_ck(cudaMemcpyPeerAsync(dst, dst_dev, src, src_dev, bytes, st), "halo peer copy");
}

// ---- in-process group ------------------------------------------------------------------------
// The ranks of one group share this state.  A collective is two host barriers: every rank
// publishes its operand (values read back to the host, or a device pointer after synchronising
// its stream), waits for all, computes or copies its result, and waits again before the slots
// may be reused.  Reductions run on the host in rank order, so every rank gets the same bits.
struct LocalGroup {
    int size = 1;
    std::chrono::milliseconds timeout{60000};
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    unsigned long long generation = 0;
    bool failed = false;
    std::string why;
    std::vector<std::vector<double>> vals;
    std::vector<double *> vec;
    std::vector<const dgh_halo_plan *> plan;
    std::vector<int> device;

    void barrier(int rank) {
        std::unique_lock<std::mutex> lk(mu);
        if (failed) throw dgh_comm_failure("slab group failed: " + why);
        const unsigned long long gen = generation;
        if (++arrived == size) {
            arrived = 0;
            ++generation;
            cv.notify_all();
            return;
        }
        if (!cv.wait_for(lk, timeout, [&] { return generation != gen || failed; })) {
            failed = true;
            why = "rank " + std::to_string(rank) + " waited " + std::to_string(timeout.count()) +
                  " ms in a collective that a peer did not enter";
            cv.notify_all();
        }
        if (generation == gen) throw dgh_comm_failure("slab group failed: " + why);
    }
    void fail(const std::string &w) {
        std::lock_guard<std::mutex> lk(mu);
        if (!failed) {
            failed = true;
            why = w;
        }
        cv.notify_all();
    }
};

struct LocalComm final : dgh_comm {
    std::shared_ptr<LocalGroup> g;
    LocalComm(std::shared_ptr<LocalGroup> group, int r) : g(std::move(group)) {
        rank = r;
        size = g->size;
    }
    const char *kind() const override { return "local"; }
    void allreduce(double *dev, int count, int op, cudaStream_t st) override {
        if (size == 1) return;
        auto &mine = g->vals[rank];
        mine.assign(count, 0.);
        cuda_ck(cudaMemcpyAsync(mine.data(), dev, count * sizeof(double), cudaMemcpyDeviceToHost, st), "collective read");
        cuda_ck(cudaStreamSynchronize(st), "collective read");
        g->barrier(rank);
        std::vector<double> res(g->vals[0]);
        bool same = true;
        for (int r = 0; r < size; ++r) same = same && (int)g->vals[r].size() == count;
        if (same)
            for (int r = 1; r < size; ++r)
                for (int i = 0; i < count; ++i) res[i] = op == 0 ? res[i] + g->vals[r][i] : larger(res[i], g->vals[r][i]);
        g->barrier(rank);
        if (!same) {
            fail("ranks entered a collective with different counts");
            throw dgh_comm_failure("slab ranks entered a collective with different counts");
        }
        cuda_ck(cudaMemcpyAsync(dev, res.data(), count * sizeof(double), cudaMemcpyHostToDevice, st), "collective write");
        cuda_ck(cudaStreamSynchronize(st), "collective write");
    }
    void exchange(double *v, const dgh_halo_plan &p, cudaStream_t st) override {
        int dev = 0;
        cuda_ck(cudaGetDevice(&dev), "cudaGetDevice");
        if (size == 1) {  // the periodic wrap inside one slab: this rank is its own neighbour
            copy_regions(v, dev, p.from_below, v, dev, p.to_above, st);
            copy_regions(v, dev, p.from_above, v, dev, p.to_below, st);
            return;
        }
        cuda_ck(cudaStreamSynchronize(st), "halo");
        g->vec[rank] = v;
        g->plan[rank] = &p;
        g->device[rank] = dev;
        g->barrier(rank);
        const int below = (rank + size - 1) % size, above = (rank + 1) % size;
        const bool same = matches(p.from_below, g->plan[below]->to_above) && matches(p.from_above, g->plan[above]->to_below);
        if (same) {
            copy_regions(v, dev, p.from_below, g->vec[below], g->device[below], g->plan[below]->to_above, st);
            copy_regions(v, dev, p.from_above, g->vec[above], g->device[above], g->plan[above]->to_below, st);
            cuda_ck(cudaStreamSynchronize(st), "halo");
        }
        g->barrier(rank);
        if (!same) {
            fail("neighbouring slabs exchange regions of different sizes");
            throw dgh_comm_failure("neighbouring slabs exchange regions of different sizes");
        }
    }
    static bool matches(const std::vector<dgh_region> &a, const std::vector<dgh_region> &b) {
        if (a.size() != b.size()) return false;
        for (size_t i = 0; i < a.size(); ++i)
            if (a[i].count != b[i].count) return false;
        return true;
    }
    static void copy_regions(double *dst, int dst_dev, const std::vector<dgh_region> &into, const double *src, int src_dev,
                             const std::vector<dgh_region> &from, cudaStream_t st) {
        for (size_t i = 0; i < into.size() && i < from.size(); ++i)
            copy_row(dst + into[i].offset, dst_dev, src + from[i].offset, src_dev,
                     (size_t)into[i].count * sizeof(double), st);
    }
    void fail(const std::string &why) noexcept override {
        try {
            g->fail("rank " + std::to_string(rank) + ": " + why);
        } catch (...) {
        }
    }
    void set_timeout(int timeout_ms) override {
        std::lock_guard<std::mutex> lk(g->mu);
        g->timeout = std::chrono::milliseconds(timeout_ms);
    }
};

// ---- NCCL --------------------------------------------------------------------------------------
// libnccl is resolved when the first NCCL communicator is made: the copy already loaded into the
// process (by torch, for instance) if there is one, else DGH_NCCL_LIBRARY, else libnccl.so.2.
struct NcclApi {
    std::string why;
    ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
    ncclResult_t (*init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*abort)(ncclComm_t) = nullptr;
    ncclResult_t (*allreduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    const char *(*error_string)(ncclResult_t) = nullptr;
    bool ok() const { return why.empty(); }
};
template <class F> void resolve(void *h, const char *name, F &f, std::string &why) {
    f = reinterpret_cast<F>(dlsym(h, name));
    if (!f && why.empty()) why = std::string("libnccl lacks ") + name;
}
NcclApi load_nccl() {
    NcclApi a;
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) {
        if (const char *path = std::getenv("DGH_NCCL_LIBRARY")) h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
    }
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
        const char *e = dlerror();
        a.why = std::string("cannot load libnccl: ") + (e ? e : "not found");
        return a;
    }
    resolve(h, "ncclGetUniqueId", a.get_unique_id, a.why);
    resolve(h, "ncclCommInitRank", a.init_rank, a.why);
    resolve(h, "ncclCommDestroy", a.destroy, a.why);
    resolve(h, "ncclCommAbort", a.abort, a.why);
    resolve(h, "ncclAllReduce", a.allreduce, a.why);
    resolve(h, "ncclSend", a.send, a.why);
    resolve(h, "ncclRecv", a.recv, a.why);
    resolve(h, "ncclGroupStart", a.group_start, a.why);
    resolve(h, "ncclGroupEnd", a.group_end, a.why);
    resolve(h, "ncclGetErrorString", a.error_string, a.why);
    return a;
}
NcclApi &nccl() {
    static NcclApi api = load_nccl();
    return api;
}
void nccl_ck(ncclResult_t r, const char *what) {
    if (r != ncclSuccess) throw dgh_comm_failure(std::string(what) + ": " + nccl().error_string(r));
}

struct NcclComm final : dgh_comm {
    ncclComm_t comm = nullptr;
    int device = 0;
    bool failed = false;
    std::string why;
    std::chrono::milliseconds timeout{300000};
    const char *kind() const override { return "nccl"; }
    void check() const {
        if (failed) throw dgh_comm_failure("slab communicator failed: " + why);
    }
    void allreduce(double *dev, int count, int op, cudaStream_t st) override {
        check();
        nccl_ck(nccl().allreduce(dev, dev, (size_t)count, ncclDouble, op == 0 ? ncclSum : ncclMax, comm, st),
                "ncclAllReduce");
    }
    void exchange(double *v, const dgh_halo_plan &p, cudaStream_t st) override {
        check();
        if (size == 1) {
            for (size_t i = 0; i < p.from_below.size(); ++i)
                copy_row(v + p.from_below[i].offset, device, v + p.to_above[i].offset, device,
                         (size_t)p.from_below[i].count * sizeof(double), st);
            for (size_t i = 0; i < p.from_above.size(); ++i)
                copy_row(v + p.from_above[i].offset, device, v + p.to_below[i].offset, device,
                         (size_t)p.from_above[i].count * sizeof(double), st);
            return;
        }
        // With two ranks both neighbours are the same peer, and NCCL matches that peer's
        // messages in posting order: every rank sends its to_below regions, then its to_above
        // regions, and receives its from_above regions (the peer's to_below), then its
        // from_below regions (the peer's to_above).
        const int below = (rank + size - 1) % size, above = (rank + 1) % size;
        nccl_ck(nccl().group_start(), "ncclGroupStart");
        for (const auto &r : p.to_below) nccl_ck(nccl().send(v + r.offset, (size_t)r.count, ncclDouble, below, comm, st), "ncclSend");
        for (const auto &r : p.to_above) nccl_ck(nccl().send(v + r.offset, (size_t)r.count, ncclDouble, above, comm, st), "ncclSend");
        for (const auto &r : p.from_above) nccl_ck(nccl().recv(v + r.offset, (size_t)r.count, ncclDouble, above, comm, st), "ncclRecv");
        for (const auto &r : p.from_below) nccl_ck(nccl().recv(v + r.offset, (size_t)r.count, ncclDouble, below, comm, st), "ncclRecv");
        nccl_ck(nccl().group_end(), "ncclGroupEnd");
    }
    void fail(const std::string &w) noexcept override {
        if (failed) return;
        failed = true;
        why = w;
        if (comm) nccl().abort(comm);  // peers blocked on this rank see the communicator go away
        comm = nullptr;
    }
    void set_timeout(int timeout_ms) override { timeout = std::chrono::milliseconds(timeout_ms); }
    // Polls the stream instead of blocking in it, so that a rank whose peer never joins a
    // collective (the peer failed on its own) gives up after the timeout: it aborts its
    // communicator, which ends its own waiting NCCL kernels, and reports the failure.
    void wait(cudaStream_t st) override {
        const auto start = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t e = cudaStreamQuery(st);
            if (e == cudaSuccess) return;
            if (e != cudaErrorNotReady)
                throw std::runtime_error(std::string("cudaStreamQuery: ") + cudaGetErrorString(e));
            if (std::chrono::steady_clock::now() - start > timeout) {
                const std::string w = "rank " + std::to_string(rank) + " waited " + std::to_string(timeout.count()) +
                                      " ms for its stream (a collective that a peer did not enter)";
                fail(w);
                throw dgh_comm_failure("slab communicator failed: " + w);
            }
            std::this_thread::yield();
        }
    }
    ~NcclComm() override {
        if (comm) nccl().destroy(comm);
    }
};

template <class F> int comm_guard(F &&f) {
    g_comm_error.clear();
    try {
        f();
        return DGH_OK;
    } catch (const dgh_comm_failure &e) {
        g_comm_error = e.what();
        return DGH_ERR_COMM;
    } catch (const std::exception &e) {
        g_comm_error = e.what();
        return DGH_ERR_COMM;
    }
}
}  // namespace

extern "C" {

const char *dgh_comm_error(void) { return g_comm_error.c_str(); }

int dgh_slab_rows(int ny, int size, int rank, int out[4]) {
    if (!out || size < 1 || rank < 0 || rank >= size || ny < size) return DGH_ERR_INVALID;
    dgh_slab::rows_of(ny, size, rank, out[0], out[1]);
    out[2] = (rank + size - 1) % size;
    out[3] = (rank + 1) % size;
    return DGH_OK;
}

int dgh_slab_halo_plan(int nx, int degree, int rows, int above, int trace, int64_t regions[16], int counts[4]) {
    if (!regions || !counts || nx < 1 || degree < 0 || degree > 8 || rows < above || above < 1 || above > 2)
        return DGH_ERR_INVALID;
    const long long n = degree + 1, fw = 4 * n, cells = (long long)nx * (rows + 1 + above);
    const dgh_halo_plan p = trace ? dgh_slab::trace_plan(nx * fw, cells * fw, rows)
                                  : dgh_slab::volume_plan(nx * 4 * n * n, rows, above);
    int k = 0, j = 0;
    for (const auto *list : {&p.to_below, &p.to_above, &p.from_above, &p.from_below}) {
        counts[j++] = (int)list->size();
        for (const auto &r : *list) {
            regions[k++] = r.offset;
            regions[k++] = r.count;
        }
    }
    return DGH_OK;
}

int dgh_comm_local_create(int size, int timeout_ms, dgh_comm **ranks) {
    return comm_guard([&] {
        if (!ranks || size < 1 || timeout_ms < 1) throw dgh_comm_failure("invalid group size, timeout or output");
        auto g = std::make_shared<LocalGroup>();
        g->size = size;
        g->timeout = std::chrono::milliseconds(timeout_ms);
        g->vals.resize(size);
        g->vec.assign(size, nullptr);
        g->plan.assign(size, nullptr);
        g->device.assign(size, 0);
        for (int r = 0; r < size; ++r) ranks[r] = new LocalComm(g, r);
    });
}

int dgh_comm_nccl_unique_id(unsigned char id[128]) {
    return comm_guard([&] {
        if (!id) throw dgh_comm_failure("null output");
        if (!nccl().ok()) throw dgh_comm_failure(nccl().why);
        ncclUniqueId u;
        nccl_ck(nccl().get_unique_id(&u), "ncclGetUniqueId");
        static_assert(sizeof(u.internal) == 128, "NCCL unique id size");
        std::memcpy(id, u.internal, 128);
    });
}

int dgh_comm_nccl_create(const unsigned char id[128], int size, int rank, int device, dgh_comm **out) {
    return comm_guard([&] {
        if (!id || !out || size < 1 || rank < 0 || rank >= size) throw dgh_comm_failure("invalid rank, size or id");
        *out = nullptr;
        if (!nccl().ok()) throw dgh_comm_failure(nccl().why);
        cuda_ck(cudaSetDevice(device), "cudaSetDevice");
        ncclUniqueId u;
        std::memcpy(u.internal, id, 128);
        auto c = std::make_unique<NcclComm>();
        c->rank = rank;
        c->size = size;
        c->device = device;
        nccl_ck(nccl().init_rank(&c->comm, size, u, rank), "ncclCommInitRank");
        *out = c.release();
    });
}

int dgh_comm_info(const dgh_comm *comm, int out[3]) {
    if (!comm || !out) return DGH_ERR_INVALID;
    out[0] = comm->rank;
    out[1] = comm->size;
    out[2] = std::strcmp(comm->kind(), "nccl") == 0 ? 1 : 0;
    return DGH_OK;
}

int dgh_comm_set_timeout(dgh_comm *comm, int timeout_ms) {
    if (!comm || timeout_ms < 1) return DGH_ERR_INVALID;
    comm->set_timeout(timeout_ms);
    return DGH_OK;
}

int dgh_comm_fail(dgh_comm *comm, const char *why) {
    if (!comm) return DGH_ERR_INVALID;
    comm->fail(why ? why : "failed by its host");
    return DGH_OK;
}

int dgh_comm_destroy(dgh_comm *comm) {
    delete comm;
    return DGH_OK;
}

}  // extern "C"
