// Batched uneven problems (no counterpart in the reference): independent member problems, each
// with its own mesh, degree, method and precision, advanced together on one device.  Every
// member owns a context (its own non-blocking stream and device memory) and an integrator; a
// persistent host thread per member issues that member's work, so the members' kernels overlap
// on the device while each member computes exactly what its single-problem run computes (same
// kernels, same launch shapes, same order on its stream).  Small members, which cannot fill
// 148 SMs alone and are launch-latency bound, share the device with the large ones.
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dgh_gpu.h"

struct dgh_batch {
    int count = 0;
    std::vector<dgh_config> cfg;
    std::vector<dgh_ctx *> ctx;
    std::vector<dgh_integrator *> it;
    std::vector<double *> buf;  // per-member device state used to start a stage
    std::vector<int64_t> size;  // volume unknowns per member
    std::vector<int> status;
    std::vector<std::string> errors;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable go, done;
    uint64_t generation = 0;
    int pending = 0;
    bool quit = false;
    std::function<int(int)> job;
    // lockstep groups of the members' GMRES solves (dgh_batch_lockstep): one per class of members
    // that can share one (2D, collocated rule, block Jacobi, same method, precision and restart)
    std::vector<dgh_lockstep *> groups;
    std::vector<int> group_size, group_of;  // members per group; each member's group or -1
    void drop_groups() {
        for (auto *g : groups) dgh_lockstep_destroy(g);
        groups.clear();
        group_size.clear();
        group_of.assign(count, -1);
    }

    void worker(int i) {
        cudaSetDevice(cfg[i].device);
        uint64_t seen = 0;
        for (;;) {
            std::function<int(int)> f;
            {
                std::unique_lock<std::mutex> lk(mu);
                go.wait(lk, [&] { return quit || generation != seen; });
                if (quit) return;
                seen = generation;
                f = job;
            }
            const int rc = f(i);
            std::lock_guard<std::mutex> lk(mu);
            status[i] = rc;
            if (--pending == 0) done.notify_all();
        }
    }
    // Runs f(member) on every member's thread and waits for all; the first non-zero status of
    // the lowest member index is returned, every member's status stays in `status`.
    int run(std::function<int(int)> f) {
        {
            std::lock_guard<std::mutex> lk(mu);
            job = std::move(f);
            pending = count;
            ++generation;
        }
        go.notify_all();
        std::unique_lock<std::mutex> lk(mu);
        done.wait(lk, [&] { return pending == 0; });
        for (int i = 0; i < count; ++i)
            if (status[i] != DGH_OK) return status[i];
        return DGH_OK;
    }
    void release() {
        drop_groups();
        {
            std::lock_guard<std::mutex> lk(mu);
            quit = true;
        }
        go.notify_all();
        for (auto &w : workers) w.join();
        workers.clear();
        for (int i = 0; i < (int)ctx.size(); ++i) {
            if (i < (int)it.size() && it[i]) dgh_integrator_destroy(it[i]);
            if (i < (int)buf.size() && buf[i]) dgh_vec_free(ctx[i], buf[i]);
            if (ctx[i]) dgh_ctx_destroy(ctx[i]);
        }
        ctx.clear();
        it.clear();
        buf.clear();
    }
};

namespace {
thread_local std::string g_batch_create_error;
}

extern "C" {

int dgh_batch_create(const dgh_config *members, int count, dgh_batch **out) {
    if (!members || !out || count <= 0) return DGH_ERR_INVALID;
    *out = nullptr;
    auto *b = new dgh_batch;
    b->count = count;
    b->cfg.assign(members, members + count);
    b->status.assign(count, DGH_OK);
    b->group_of.assign(count, -1);
    b->errors.assign(count, std::string());
    for (int i = 0; i < count; ++i)
        if (b->cfg[i].method != DGH_METHOD_DG && b->cfg[i].method != DGH_METHOD_HDG) {
            g_batch_create_error = "batch member " + std::to_string(i) + ": method must be dg or hdg";
            delete b;
            return DGH_ERR_INVALID;
        }
    int rc = DGH_OK;
    for (int i = 0; i < count && rc == DGH_OK; ++i) {
        const dgh_config &c = b->cfg[i];
        dgh_ctx *ctx = nullptr;
        rc = dgh_ctx_create(&c, &ctx);
        if (rc != DGH_OK) {
            g_batch_create_error = "batch member " + std::to_string(i) + ": " + dgh_last_error(nullptr);
            break;
        }
        b->ctx.push_back(ctx);
        dgh_integrator *it = nullptr;
        rc = dgh_integrator_create(ctx, c.method, &it);
        if (rc != DGH_OK) {
            g_batch_create_error = "batch member " + std::to_string(i) + ": " + dgh_last_error(ctx);
            break;
        }
        b->it.push_back(it);
        int64_t s[8];
        double *p = nullptr;
        rc = dgh_sizes(ctx, s);
        if (rc == DGH_OK) rc = dgh_vec_alloc(ctx, s[0], &p);
        b->size.push_back(s[0]);
        if (rc != DGH_OK) {
            g_batch_create_error = "batch member " + std::to_string(i) + ": " + dgh_last_error(ctx);
            break;
        }
        b->buf.push_back(p);
    }
    if (rc != DGH_OK) {
        b->release();
        delete b;
        return rc;
    }
    for (int i = 0; i < count; ++i) b->workers.emplace_back([b, i] { b->worker(i); });
    *out = b;
    return DGH_OK;
}

int dgh_batch_destroy(dgh_batch *b) {
    if (!b) return DGH_ERR_INVALID;
    b->release();
    delete b;
    return DGH_OK;
}

const char *dgh_batch_error(const dgh_batch *b, int member) {
    if (!b) return g_batch_create_error.c_str();
    if (member < 0 || member >= b->count) return "";
    return b->errors[member].c_str();
}

int dgh_batch_member(dgh_batch *b, int member, dgh_ctx **ctx, dgh_integrator **it) {
    if (!b || member < 0 || member >= b->count) return DGH_ERR_INVALID;
    if (ctx) *ctx = b->ctx[member];
    if (it) *it = b->it[member];
    return DGH_OK;
}

int dgh_batch_stage_begin(dgh_batch *b, const double *const *host_states, double *dt, int *status) {
    if (!b) return DGH_ERR_INVALID;
    const int rc = b->run([&](int i) {
        dgh_ctx *c = b->ctx[i];
        int r = host_states && host_states[i] ? dgh_upload(c, b->buf[i], host_states[i], b->size[i])
                                              : dgh_initial(c, b->buf[i]);
        if (r != DGH_OK) {
            b->errors[i] = dgh_last_error(c);
            return r;
        }
        double step = 0;
        r = dgh_stage_begin(b->it[i], b->buf[i], &step);
        if (r != DGH_OK) b->errors[i] = dgh_integrator_error(b->it[i]);
        if (dt) dt[i] = step;
        return r;
    });
    if (status)
        for (int i = 0; i < b->count; ++i) status[i] = b->status[i];
    return rc;
}

int dgh_batch_lockstep(dgh_batch *b, int on) {
    if (!b) return DGH_ERR_INVALID;
    b->drop_groups();
    if (!on) return DGH_OK;
    // classes of members that can share a group; the others keep solving independently
    std::vector<std::vector<int>> classes;
    std::vector<const dgh_config *> key;
    for (int i = 0; i < b->count; ++i) {
        const dgh_config &c = b->cfg[i];
        const bool collocated = c.quadrature == 0 || c.quadrature <= c.degree + 1;
        if (c.method == DGH_METHOD_BOTH || c.dim == 1 || !collocated || c.preconditioner != 0) continue;
        int cls = -1;
        for (int q = 0; q < (int)key.size(); ++q)
            if (key[q]->method == c.method && key[q]->precision == c.precision && key[q]->restart == c.restart &&
                key[q]->device == c.device)
                cls = q;
        if (cls < 0) {
            cls = (int)key.size();
            key.push_back(&c);
            classes.emplace_back();
        }
        classes[cls].push_back(i);
    }
    for (const auto &members : classes) {
        std::vector<dgh_ctx *> ctxs;
        for (int i : members) ctxs.push_back(b->ctx[i]);
        dgh_lockstep *g = nullptr;
        const int op = b->cfg[members[0]].method == DGH_METHOD_HDG ? DGH_OP_HDG : DGH_OP_DG;
        const int rc = dgh_lockstep_create_op(ctxs.data(), (int)ctxs.size(), op, &g);
        if (rc != DGH_OK) {
            g_batch_create_error = dgh_lockstep_error();
            b->drop_groups();
            return rc;
        }
        for (int i : members) b->group_of[i] = (int)b->groups.size();
        b->groups.push_back(g);
        b->group_size.push_back((int)members.size());
    }
    return DGH_OK;
}

int dgh_batch_lockstep_report(const dgh_batch *b, int64_t out[4]) {
    if (!b || !out) return DGH_ERR_INVALID;
    for (int i = 0; i < 4; ++i) out[i] = 0;
    for (auto *g : b->groups) {
        int64_t r[4];
        const int rc = dgh_lockstep_report(g, r);
        if (rc != DGH_OK) return rc;
        for (int i = 0; i < 4; ++i) out[i] += r[i];
    }
    return DGH_OK;
}

int dgh_batch_newton_update(dgh_batch *b, dgh_update_stats *stats, int *status) {
    if (!b) return DGH_ERR_INVALID;
    for (size_t g = 0; g < b->groups.size(); ++g) {
        const int r = dgh_lockstep_begin(b->groups[g], b->group_size[g]);
        if (r != DGH_OK) return r;
    }
    const int rc = b->run([&](int i) {
        dgh_update_stats s{};
        const int r = dgh_newton_update(b->it[i], &s);
        if (r != DGH_OK) b->errors[i] = dgh_integrator_error(b->it[i]);
        // a DG member whose update ended before its GMRES solve leaves the lockstep session
        if (b->group_of[i] >= 0) dgh_lockstep_leave(b->groups[b->group_of[i]], b->ctx[i]);
        if (stats) stats[i] = s;
        return r;
    });
    if (status)
        for (int i = 0; i < b->count; ++i) status[i] = b->status[i];
    return rc;
}

int dgh_batch_download(dgh_batch *b, int member, double *host_state) {
    if (!b || member < 0 || member >= b->count || !host_state) return DGH_ERR_INVALID;
    return dgh_download(b->ctx[member], host_state, dgh_integrator_state(b->it[member]), b->size[member]);
}

}  // extern "C"
