// sm_server.cpp -- request loop over many shots of different grids on one
// device: admission by device memory, one handle and stream per running
// request, slices of steps fed round-robin so requests overlap on the GPU,
// latency percentiles.  No counterpart in the reference (one program per
// shot there); every request runs exactly the computation of a handle of its
// own, through the public C ABI of this library.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/seismod_gpu.h"
#include "sm_host.h"

namespace {

using Clock = std::chrono::steady_clock;

double secs(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

// host copy of one request
struct Req {
    uint64_t ticket = 0;
    int kind = 0;   // 0 e_iso, 1 a_iso_3d
    // e_iso
    sm_eiso_request e{};
    // a_iso_3d
    sm_a3d_request a{};
    std::vector<double> m[5];          // e_iso materials / a3d vp, rho
    std::vector<double> prof[3];       // e_iso d, dh, dH
    std::vector<std::vector<double>> coef;   // a3d: 18 arrays
    std::vector<const double *> coefp;
    std::vector<size_t> src_index, src_length, rec_index;
    std::vector<int> src_type, rec_comp;
    std::vector<double> src_fct, rec_t0, rec_dt;
    size_t nsteps = 0, nrec = 0, bytes = 0;
    double cells = 0;                  // cells updated per step
    // running state
    int state = SM_REQ_QUEUED;
    int error = SM_OK;
    std::string message;
    sm_eiso_t he = nullptr;
    sm_a3d_t ha = nullptr;
    cudaStream_t stream = nullptr;
    size_t enqueued = 0;
    std::deque<cudaEvent_t> slices;    // end of each queued slice
    Clock::time_point t_submit, t_admit, t_done;
    // result
    std::vector<double> traces;        // nrec x ld
    std::vector<size_t> counts;
    size_t ld = 0;
};

}  // namespace

struct sm_server {
    int device = 0;
    size_t budget = 0, used = 0, peak = 0;
    int max_active = 64, slice = 64, graph = 0;
    bool group = false;   // requests of one program and precision stepped together
                          // (sm_eiso_group_run, sm_a3d_group_run)
    std::mutex mu;
    std::condition_variable cv;        // request finished / new request
    std::deque<std::shared_ptr<Req>> queue;
    std::vector<std::shared_ptr<Req>> running;
    std::map<uint64_t, std::shared_ptr<Req>> all;
    uint64_t next = 1;
    bool stop = false;
    std::thread worker;
    // statistics
    size_t submitted = 0, completed = 0, failed = 0, max_running = 0;
    std::vector<double> lat, wait;
    double cells_done = 0;
    bool any_submit = false;
    Clock::time_point t_first, t_last;
};

namespace {

void finish(sm_server *s, Req &r, int rc, const char *msg) {
    // called with s->mu held
    r.t_done = Clock::now();
    if (rc == SM_OK) {
        r.state = SM_REQ_DONE;
        s->completed++;
        s->lat.push_back(secs(r.t_submit, r.t_done));
        s->cells_done += r.cells * (double)r.nsteps;
    } else {
        r.state = SM_REQ_FAILED;
        r.error = rc;
        r.message = msg ? msg : "";
        s->failed++;
    }
    s->t_last = r.t_done;
    s->cv.notify_all();
}

void release_device(Req &r) {
    for (cudaEvent_t e : r.slices) cudaEventDestroy(e);
    r.slices.clear();
    if (r.he) sm_eiso_destroy(r.he);
    if (r.ha) sm_a3d_destroy(r.ha);
    r.he = nullptr;
    r.ha = nullptr;
}

// create the handle of an admitted request (worker thread, s->mu not held)
int start(sm_server *s, Req &r) {
    int rc;
    void *st = nullptr;
    if (r.kind == 0) {
        const sm_eiso_request &q = r.e;
        rc = sm_eiso_create(s->device, q.nx, q.nz, q.npml, q.h, q.dt, q.la, q.mu, q.l2m, q.b,
                            q.bm, q.d, q.dh, q.dH, q.precision, 1, &r.he);
        if (!rc)
            rc = sm_eiso_set_sources(r.he, 0, q.nsrc, q.src_index, q.src_type, q.src_fct,
                                     q.src_length, q.src_stride, q.src_scale);
        if (!rc)
            rc = sm_eiso_set_receivers(r.he, 0, q.nrec, q.rec_index, q.rec_comp, q.rec_t0,
                                       q.rec_dt, q.nsteps);
        if (!rc && s->graph) rc = sm_eiso_set_graph(r.he, s->graph);
        if (!rc) rc = sm_eiso_stream(r.he, &st);
    } else {
        const sm_a3d_request &q = r.a;
        rc = sm_a3d_create(s->device, q.nx2, q.ny2, q.nz2, q.np, q.dx, q.dy, q.dz, q.dt, q.vp,
                           q.rho, q.coef, q.precision, &r.ha);
        if (!rc)
            rc = sm_a3d_set_sources(r.ha, q.nsrc, q.src_index, q.src_fct, q.src_length,
                                    q.src_stride, q.src_scale);
        if (!rc)
            rc = sm_a3d_set_receivers(r.ha, q.nrec, q.rec_index, q.rec_comp, q.rec_t0, q.rec_dt,
                                      q.nsteps);
        if (!rc && s->graph) rc = sm_a3d_set_graph(r.ha, s->graph);
        if (!rc) rc = sm_a3d_stream(r.ha, &st);
    }
    r.stream = static_cast<cudaStream_t>(st);
    return rc;
}

// queue one more slice of steps for a running request
int feed(sm_server *s, Req &r) {
    const size_t k = std::min<size_t>((size_t)s->slice, r.nsteps - r.enqueued);
    int rc = r.kind == 0 ? sm_eiso_run(r.he, k) : sm_a3d_run(r.ha, k);
    if (rc) return rc;
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(ev, r.stream) != cudaSuccess) {
        if (ev) cudaEventDestroy(ev);
        return sm_fail(SM_ECUDA, "server: event record failed");
    }
    r.slices.push_back(ev);
    r.enqueued += k;
    return SM_OK;
}

// grouped mode: every running request of one program and precision that
// wants a slice gets it from one sm_eiso_group_run / sm_a3d_group_run call
// (one launch per step over all of their grids); the slice is as long as the
// shortest remainder
int feed_group(sm_server *s, std::vector<Req *> &grp) {
    size_t k = (size_t)s->slice;
    for (Req *r : grp) k = std::min(k, r->nsteps - r->enqueued);
    if (grp[0]->kind == 0) {
        std::vector<sm_eiso_t> hs;
        for (Req *r : grp) hs.push_back(r->he);
        if (int rc = sm_eiso_group_run(hs.data(), (int)hs.size(), k)) return rc;
    } else {
        std::vector<sm_a3d_t> hs;
        for (Req *r : grp) hs.push_back(r->ha);
        if (int rc = sm_a3d_group_run(hs.data(), (int)hs.size(), k)) return rc;
    }
    for (Req *r : grp) {
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(ev, r->stream) != cudaSuccess) {
            if (ev) cudaEventDestroy(ev);
            return sm_fail(SM_ECUDA, "server: event record failed");
        }
        r->slices.push_back(ev);
        r->enqueued += k;
    }
    return SM_OK;
}

// copy a finished request's traces to the host
int collect(Req &r) {
    std::vector<size_t> cnt(r.nrec, 0);
    int rc = r.kind == 0 ? sm_eiso_read_traces(r.he, 0, 0, r.nrec, nullptr, 0, cnt.data())
                         : sm_a3d_read_traces(r.ha, 0, r.nrec, nullptr, 0, cnt.data());
    if (rc) return rc;
    size_t ld = 1;
    for (size_t c : cnt) ld = std::max(ld, c);
    r.ld = ld;
    r.traces.assign(r.nrec * ld, 0.0);
    r.counts = cnt;
    if (r.nrec == 0) return SM_OK;
    return r.kind == 0 ? sm_eiso_read_traces(r.he, 0, 0, r.nrec, r.traces.data(), ld, nullptr)
                       : sm_a3d_read_traces(r.ha, 0, r.nrec, r.traces.data(), ld, nullptr);
}

void work(sm_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        bool progress = false;
        // ---- admission, in arrival order ----
        std::vector<std::shared_ptr<Req>> admit;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
            while (!s->queue.empty() && (int)s->running.size() + (int)admit.size() < s->max_active &&
                   s->used + s->queue.front()->bytes <= s->budget) {
                std::shared_ptr<Req> r = s->queue.front();
                s->queue.pop_front();
                s->used += r->bytes;
                s->peak = std::max(s->peak, s->used);
                r->state = SM_REQ_RUNNING;
                r->t_admit = Clock::now();
                s->wait.push_back(secs(r->t_submit, r->t_admit));
                admit.push_back(r);
            }
        }
        for (auto &r : admit) {
            int rc = start(s, *r);
            std::lock_guard<std::mutex> lk(s->mu);
            if (rc) {
                release_device(*r);
                s->used -= r->bytes;
                finish(s, *r, rc, sm_last_error());
            } else {
                s->running.push_back(r);
                s->max_running = std::max(s->max_running, s->running.size());
            }
            progress = true;
        }
        // ---- feed and retire ----
        std::vector<std::shared_ptr<Req>> run;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            run = s->running;
        }
        std::map<Req *, int> grc;   // grouped feed failures
        if (s->group) {
            std::map<std::pair<int, int>, std::vector<Req *>> need;   // by program, precision
            for (auto &r : run) {
                while (!r->slices.empty() && cudaEventQuery(r->slices.front()) == cudaSuccess) {
                    cudaEventDestroy(r->slices.front());
                    r->slices.pop_front();
                    progress = true;
                }
                if (r->enqueued < r->nsteps && r->slices.size() < 2)
                    need[{r->kind, r->kind == 0 ? r->e.precision : r->a.precision}].push_back(r.get());
            }
            for (auto &g : need) {
                const int rc = feed_group(s, g.second);
                if (rc)
                    for (Req *r : g.second) grc[r] = rc;
                progress = true;
            }
        }
        for (auto &r : run) {
            int rc = SM_OK;
            auto gf = grc.find(r.get());
            if (gf != grc.end()) rc = gf->second;
            while (!r->slices.empty() && cudaEventQuery(r->slices.front()) == cudaSuccess) {
                cudaEventDestroy(r->slices.front());
                r->slices.pop_front();
                progress = true;
            }
            while (rc == SM_OK && !s->group && r->enqueued < r->nsteps &&
                   r->slices.size() < 2) {
                rc = feed(s, *r);
                progress = true;
            }
            const bool done = rc == SM_OK && r->enqueued >= r->nsteps && r->slices.empty();
            if (rc == SM_OK && !done) continue;
            if (done) rc = collect(*r);
            const char *msg = rc ? sm_last_error() : nullptr;
            std::string m = msg ? msg : "";
            release_device(*r);
            std::lock_guard<std::mutex> lk(s->mu);
            s->used -= r->bytes;
            s->running.erase(std::find(s->running.begin(), s->running.end(), r));
            finish(s, *r, rc, m.c_str());
            progress = true;
        }
        if (!progress) {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
            s->cv.wait_for(lk, std::chrono::microseconds(50));
        }
    }
    // shut down: finish what is queued on the device, then free it
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto &r : s->running) {
        if (r->stream) cudaStreamSynchronize(r->stream);
        release_device(*r);
        r->state = SM_REQ_FAILED;
        r->error = SM_ESTATE;
        r->message = "server stopped";
    }
    s->running.clear();
}

template <typename T>
std::vector<T> copy_of(const T *p, size_t n) {
    return p ? std::vector<T>(p, p + n) : std::vector<T>();
}

double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    // nearest-rank percentile
    size_t k = (size_t)std::ceil(q * (double)v.size());
    k = std::min(std::max<size_t>(k, 1), v.size());
    return v[k - 1];
}

int enqueue(sm_server *s, std::shared_ptr<Req> r, uint64_t *ticket) {
    if (r->bytes > s->budget)
        return sm_fail(SM_EBUSY, "server: request needs %zu bytes of device memory, budget %zu",
                       r->bytes, s->budget);
    std::lock_guard<std::mutex> lk(s->mu);
    r->ticket = s->next++;
    r->t_submit = Clock::now();
    if (!s->any_submit) {
        s->any_submit = true;
        s->t_first = r->t_submit;
    }
    s->submitted++;
    s->all[r->ticket] = r;
    s->queue.push_back(r);
    if (ticket) *ticket = r->ticket;
    s->cv.notify_all();
    return SM_OK;
}

std::shared_ptr<Req> find(sm_server *s, uint64_t t) {
    auto it = s->all.find(t);
    return it == s->all.end() ? nullptr : it->second;
}

}  // namespace

extern "C" int sm_server_create(int device, size_t hbm_budget, int max_active, int slice_steps,
                                int graph_steps, sm_server_t *out) {
    if (!out) return sm_fail(SM_EINVAL, "sm_server_create: out is NULL");
    *out = nullptr;
    if (graph_steps != 0 && graph_steps != 2 && graph_steps != 4 && graph_steps != 8 &&
        graph_steps != 16)
        return sm_fail(SM_EINVAL, "sm_server_create: graph_steps must be 0, 2, 4, 8 or 16");
    if (max_active < 0 || slice_steps < 0)
        return sm_fail(SM_EINVAL, "sm_server_create: negative limit");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return sm_fail(SM_EINVAL, "sm_server_create: no CUDA device %d", device);
    std::unique_ptr<sm_server> s(new (std::nothrow) sm_server());
    if (!s) return sm_fail(SM_ENOMEM, "sm_server_create: out of host memory");
    s->device = device;
    s->max_active = max_active ? max_active : 64;
    s->slice = slice_steps ? slice_steps : 64;
    s->graph = graph_steps;
    if (s->graph && s->slice % s->graph)
        return sm_fail(SM_EINVAL, "sm_server_create: slice_steps must be a multiple of graph_steps");
    if (hbm_budget) {
        s->budget = hbm_budget;
    } else {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        size_t fr = 0, tot = 0;
        cudaError_t e = cudaMemGetInfo(&fr, &tot);
        cudaSetDevice(prev);
        if (e != cudaSuccess) return sm_fail(SM_ECUDA, "cudaMemGetInfo: %s", cudaGetErrorString(e));
        const size_t reserve = (size_t)2 << 30;
        s->budget = fr > reserve ? fr - reserve : fr / 2;
    }
    s->worker = std::thread(work, s.get());
    *out = s.release();
    return SM_OK;
}

extern "C" int sm_server_submit_eiso(sm_server_t s, const sm_eiso_request *q, uint64_t *ticket) {
    if (!s || !q) return sm_fail(SM_EINVAL, "sm_server_submit_eiso: NULL");
    if (q->nx < 2 || q->nz < 2 || q->npml < 1 || !q->la || !q->mu || !q->l2m || !q->b || !q->bm ||
        !q->d || !q->dh || !q->dH || (q->nsrc && (!q->src_index || !q->src_type || !q->src_fct ||
                                                   !q->src_length)) ||
        (q->nrec && (!q->rec_index || !q->rec_comp || !q->rec_t0 || !q->rec_dt)))
        return sm_fail(SM_EINVAL, "sm_server_submit_eiso: incomplete request");
    auto r = std::make_shared<Req>();
    r->kind = 0;
    const size_t n = q->nx * q->nz;
    const double *src[5] = {q->la, q->mu, q->l2m, q->b, q->bm};
    for (int k = 0; k < 5; ++k) r->m[k] = copy_of(src[k], n);
    r->prof[0] = copy_of(q->d, q->npml);
    r->prof[1] = copy_of(q->dh, q->npml);
    r->prof[2] = copy_of(q->dH, q->npml);
    r->src_index = copy_of(q->src_index, q->nsrc);
    r->src_type = copy_of(q->src_type, q->nsrc);
    r->src_length = copy_of(q->src_length, q->nsrc);
    r->src_fct = copy_of(q->src_fct, q->nsrc * q->src_stride);
    r->rec_index = copy_of(q->rec_index, q->nrec);
    r->rec_comp = copy_of(q->rec_comp, q->nrec);
    r->rec_t0 = copy_of(q->rec_t0, q->nrec);
    r->rec_dt = copy_of(q->rec_dt, q->nrec);
    r->e = *q;
    r->e.la = r->m[0].data(); r->e.mu = r->m[1].data(); r->e.l2m = r->m[2].data();
    r->e.b = r->m[3].data(); r->e.bm = r->m[4].data();
    r->e.d = r->prof[0].data(); r->e.dh = r->prof[1].data(); r->e.dH = r->prof[2].data();
    r->e.src_index = r->src_index.data(); r->e.src_type = r->src_type.data();
    r->e.src_fct = r->src_fct.data(); r->e.src_length = r->src_length.data();
    r->e.rec_index = r->rec_index.data(); r->e.rec_comp = r->rec_comp.data();
    r->e.rec_t0 = r->rec_t0.data(); r->e.rec_dt = r->rec_dt.data();
    r->nsteps = q->nsteps;
    r->nrec = q->nrec;
    r->cells = (double)(q->nx + 2 * q->npml) * (double)(q->nz + 2 * q->npml);
    if (int rc = sm_eiso_device_bytes(q->nx, q->nz, q->npml, q->precision, 1, q->nrec, q->nsteps,
                                      &r->bytes))
        return rc;
    return enqueue(s, r, ticket);
}

extern "C" int sm_server_submit_a3d(sm_server_t s, const sm_a3d_request *q, uint64_t *ticket) {
    if (!s || !q) return sm_fail(SM_EINVAL, "sm_server_submit_a3d: NULL");
    if (q->nx2 < 3 || q->ny2 < 3 || q->nz2 < 3 || !q->vp || !q->rho || !q->coef ||
        (q->nsrc && (!q->src_index || !q->src_fct || !q->src_length)) ||
        (q->nrec && (!q->rec_index || !q->rec_comp || !q->rec_t0 || !q->rec_dt)))
        return sm_fail(SM_EINVAL, "sm_server_submit_a3d: incomplete request");
    auto r = std::make_shared<Req>();
    r->kind = 1;
    const size_t n = q->nx2 * q->ny2 * q->nz2;
    r->m[0] = copy_of(q->vp, n);
    r->m[1] = copy_of(q->rho, n);
    const size_t n2[3] = {q->nx2, q->ny2, q->nz2};
    r->coef.resize(18);
    r->coefp.resize(18);
    for (int k = 0; k < 18; ++k) {
        if (!q->coef[k]) return sm_fail(SM_EINVAL, "sm_server_submit_a3d: coef[%d] is NULL", k);
        const size_t len = k < 9 ? n2[k / 3] : n2[(k - 9) / 3] - 1;
        r->coef[k] = copy_of(q->coef[k], len);
        r->coefp[k] = r->coef[k].data();
    }
    r->src_index = copy_of(q->src_index, q->nsrc);
    r->src_length = copy_of(q->src_length, q->nsrc);
    r->src_fct = copy_of(q->src_fct, q->nsrc * q->src_stride);
    r->rec_index = copy_of(q->rec_index, q->nrec);
    r->rec_comp = copy_of(q->rec_comp, q->nrec);
    r->rec_t0 = copy_of(q->rec_t0, q->nrec);
    r->rec_dt = copy_of(q->rec_dt, q->nrec);
    r->a = *q;
    r->a.vp = r->m[0].data(); r->a.rho = r->m[1].data(); r->a.coef = r->coefp.data();
    r->a.src_index = r->src_index.data(); r->a.src_fct = r->src_fct.data();
    r->a.src_length = r->src_length.data();
    r->a.rec_index = r->rec_index.data(); r->a.rec_comp = r->rec_comp.data();
    r->a.rec_t0 = r->rec_t0.data(); r->a.rec_dt = r->rec_dt.data();
    r->nsteps = q->nsteps;
    r->nrec = q->nrec;
    r->cells = (double)n;
    if (int rc = sm_a3d_device_bytes(q->nx2, q->ny2, q->nz2, q->np, q->precision, q->nrec,
                                     q->nsteps, &r->bytes))
        return rc;
    return enqueue(s, r, ticket);
}

extern "C" int sm_server_wait(sm_server_t s, uint64_t ticket, double timeout_s) {
    if (!s) return sm_fail(SM_EINVAL, "sm_server_wait: NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    std::shared_ptr<Req> r = find(s, ticket);
    if (!r) return sm_fail(SM_ENOTFOUND, "sm_server_wait: unknown ticket %llu",
                           (unsigned long long)ticket);
    auto pred = [&] { return r->state == SM_REQ_DONE || r->state == SM_REQ_FAILED; };
    if (timeout_s < 0) {
        s->cv.wait(lk, pred);
    } else if (!s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
        return sm_fail(SM_ETIMEOUT, "sm_server_wait: request %llu not done",
                       (unsigned long long)ticket);
    }
    if (r->state == SM_REQ_FAILED) return sm_fail(r->error, "request %llu: %s",
                                                   (unsigned long long)ticket, r->message.c_str());
    return SM_OK;
}

extern "C" int sm_server_drain(sm_server_t s, double timeout_s) {
    if (!s) return sm_fail(SM_EINVAL, "sm_server_drain: NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] { return s->completed + s->failed == s->submitted; };
    if (timeout_s < 0) {
        s->cv.wait(lk, pred);
    } else if (!s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
        return sm_fail(SM_ETIMEOUT, "sm_server_drain: %zu requests not done",
                       s->submitted - s->completed - s->failed);
    }
    return SM_OK;
}

extern "C" int sm_server_status(sm_server_t s, uint64_t ticket, int *state, double *latency_s) {
    if (!s) return sm_fail(SM_EINVAL, "sm_server_status: NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    std::shared_ptr<Req> r = find(s, ticket);
    if (!r) return sm_fail(SM_ENOTFOUND, "sm_server_status: unknown ticket");
    if (state) *state = r->state;
    if (latency_s) *latency_s = r->state == SM_REQ_DONE ? secs(r->t_submit, r->t_done) : -1.0;
    return SM_OK;
}

extern "C" int sm_server_traces(sm_server_t s, uint64_t ticket, size_t rec0, size_t nrec,
                                double *out, size_t ld, size_t *counts) {
    if (!s) return sm_fail(SM_EINVAL, "sm_server_traces: NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    std::shared_ptr<Req> r = find(s, ticket);
    if (!r) return sm_fail(SM_ENOTFOUND, "sm_server_traces: unknown ticket");
    if (r->state != SM_REQ_DONE) return sm_fail(SM_ESTATE, "sm_server_traces: request not done");
    if (rec0 + nrec > r->nrec) return sm_fail(SM_EINVAL, "sm_server_traces: receiver range");
    for (size_t k = 0; k < nrec; ++k) {
        const size_t c = r->counts[rec0 + k];
        if (counts) counts[k] = c;
        if (!out) continue;
        if (ld < c) return sm_fail(SM_EINVAL, "sm_server_traces: ld smaller than sample count");
        std::memcpy(out + k * ld, r->traces.data() + (rec0 + k) * r->ld, c * sizeof(double));
    }
    return SM_OK;
}

extern "C" int sm_server_release(sm_server_t s, uint64_t ticket) {
    if (!s) return sm_fail(SM_EINVAL, "sm_server_release: NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    std::shared_ptr<Req> r = find(s, ticket);
    if (!r) return sm_fail(SM_ENOTFOUND, "sm_server_release: unknown ticket");
    if (r->state != SM_REQ_DONE && r->state != SM_REQ_FAILED)
        return sm_fail(SM_ESTATE, "sm_server_release: request still queued or running");
    s->all.erase(ticket);
    return SM_OK;
}

extern "C" int sm_server_get_stats(sm_server_t s, sm_server_stats *st) {
    if (!s || !st) return sm_fail(SM_EINVAL, "sm_server_get_stats: NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->running = s->running.size();
    st->queued = s->queue.size();
    st->latency_p50 = pct(s->lat, 0.50);
    st->latency_p99 = pct(s->lat, 0.99);
    double sum = 0, mx = 0;
    for (double x : s->lat) { sum += x; mx = std::max(mx, x); }
    st->latency_mean = s->lat.empty() ? 0.0 : sum / s->lat.size();
    st->latency_max = mx;
    st->wait_p50 = pct(s->wait, 0.50);
    st->wait_p99 = pct(s->wait, 0.99);
    st->busy_s = s->completed ? secs(s->t_first, s->t_last) : 0.0;
    st->shots_per_s = st->busy_s > 0 ? s->completed / st->busy_s : 0.0;
    st->gcell_per_s = st->busy_s > 0 ? s->cells_done / st->busy_s / 1e9 : 0.0;
    st->hbm_budget = s->budget;
    st->hbm_peak = s->peak;
    st->max_running = s->max_running;
    return SM_OK;
}

extern "C" int sm_server_set_group(sm_server_t s, int on) {
    if (!s) return sm_fail(SM_EINVAL, "sm_server_set_group: null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->submitted) return sm_fail(SM_ESTATE, "sm_server_set_group: requests already submitted");
    s->group = on != 0;
    return SM_OK;
}

extern "C" int sm_server_destroy(sm_server_t s) {
    if (!s) return SM_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    delete s;
    return SM_OK;
}

extern "C" int sm_server_struct_sizes(size_t *eiso_request, size_t *a3d_request, size_t *stats) {
    if (eiso_request) *eiso_request = sizeof(sm_eiso_request);
    if (a3d_request) *a3d_request = sizeof(sm_a3d_request);
    if (stats) *stats = sizeof(sm_server_stats);
    return SM_OK;
}
