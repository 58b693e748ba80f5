// Request server: continuous batching of single propagations on one GPU.
// Included at the end of propagator.cu (uses its bucket table, kernels and
// set-up functions).  No counterpart in the reference, whose drivers call
// MDPROP / LDPROP once per (JTOT, block, energy) in a loop
// (mol.driver.f:1181-1855, scctrl.f:173,185).
//
// * Systems are registered once: VL / IV tiles, EINT / CENT, the radial
//   tables and (MDPROP) the energy-independent 2HQ(C) table stay in device
//   memory for the server's lifetime.
// * A request is one propagation (system, ERED, initial Y).  Submitting copies
//   Y0; the caller's output buffers are filled when the request completes.
// * A scheduler thread retires finished batches and admits pending requests:
//   the N-bucket of the oldest pending request, then pending requests of that
//   bucket in arrival order, as many as the batch limit and the free part of
//   the HBM budget allow.  Each batch runs on its own stream slot, so batches
//   of different buckets (and later arrivals) overlap on the device; a batch
//   never waits for the others.  Per-batch memory comes from the
//   stream-ordered allocator and returns to it when the batch completes.
// * Results do not depend on the batch a request lands in: every kernel
//   propagates each job independently.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

struct mgpu_server {
    int iprop = 0, dev = 0;
    size_t budget = 0, in_use = 0;  // bytes of batch allocations
    int max_batch = 0;
    // registry
    int cap = 0, nsys = 0;
    SysDev *d_sys = nullptr;
    int *d_prep = nullptr;
    int *d_list = nullptr;  // d_list[s] = s
    std::vector<SysDev> hs;
    std::vector<int> sys_n, sys_nstep, sys_bucket, sys_nham;
    std::vector<void *> allocs;
    cudaStream_t reg = nullptr, reg_side = nullptr;
    cudaEvent_t reg_evf = nullptr, reg_evj = nullptr;
    // requests
    struct Req {
        int sys = 0;
        double ered = 0.0;
        std::vector<double> y0;
        double *y = nullptr;
        int *nodes = nullptr, *status = nullptr, *kfail = nullptr;
        double t[3] = {0, 0, 0};  // submitted, launched, completed
        int state = 0;            // 0 pending, 1 running, 2 done
        int rc = MGPU_OK;
    };
    std::unordered_map<long long, Req> reqs;
    std::deque<long long> pending;
    long long next_ticket = 1;
    struct Slot {
        cudaStream_t st = nullptr, side = nullptr;
        cudaEvent_t evf = nullptr, evj = nullptr, done = nullptr;
        bool busy = false;
        std::vector<long long> tickets;
        std::vector<size_t> yoff;
        std::vector<void *> dev;
        size_t bytes = 0, ydoubles = 0;
        char *pin = nullptr;
        size_t pin_cap = 0, pin_used = 0;
        double *y_pin = nullptr;
        int *out_pin = nullptr;
        cudaGraphExec_t graph = nullptr;
    };
    std::vector<Slot> slots;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;

    static double now()
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
    ~mgpu_server();
    void loop();
    bool retire();
    bool admit();
    int launch(Slot &sl, const std::vector<long long> &tickets, const std::vector<const Req *> &rq, int b, size_t bytes);
    size_t job_bytes(int b, int n) const;
};

// device bytes a batch of one bucket needs per job (Y, descriptors, outputs,
// large-N matrices and one round's scratch)
size_t mgpu_server::job_bytes(int b, int n) const
{
    size_t x = (size_t)n * n * 8 + sizeof(JobDev) + 3 * sizeof(int) + 64;
    if (kBuckets[b].kind == KIND_BIG) {
        const int ldj = iprop == MGPU_PROP_LDJ ? 2 : 1;
        const size_t td = matrix_elems(b), fr = (size_t)kBuckets[b].nt * big::MC * 32;
        x += ldj * td * 8 + 3 * (size_t)bucket_npad(b) * 8 + 3 * sizeof(int) + ldj * 2 * sizeof(big::MatDesc);
        x += ldj * ((size_t)big::NB * big::NB * 8 + big::NB * 8 + 4 * fr * 8);
    }
    return x;
}

static cudaError_t grow_pinned(mgpu_server::Slot &sl, size_t need)
{
    if (sl.pin_cap >= need) return cudaSuccess;
    if (sl.pin) cudaFreeHost(sl.pin);
    sl.pin = nullptr;
    sl.pin_cap = 0;
    size_t cap = std::max<size_t>(need, (size_t)8 << 20);
    cap = std::max(cap, need + need / 2);
    cudaError_t e = cudaHostAlloc((void **)&sl.pin, cap, cudaHostAllocDefault);
    if (e == cudaSuccess) sl.pin_cap = cap;
    return e;
}

// Launch one batch on a free slot.  Runs WITHOUT the mutex (CUDA calls can
// block): `rq` are the batch's requests, whose fields do not change after
// submission.  Slots belong to the scheduler thread.  Returns MGPU_OK or an
// error that fails the batch's requests.
int mgpu_server::launch(Slot &sl, const std::vector<long long> &tickets, const std::vector<const Req *> &rq, int b,
                        size_t bytes)
{
    cudaError_t e;
    const int M = (int)tickets.size();
    sl.tickets = tickets;
    sl.yoff.resize(M);
    size_t yd = 0;
    int nhmax = 0;
    std::vector<JobDev> jobs(M);
    for (int k = 0; k < M; ++k) {
        const Req &r = *rq[k];
        const int n = sys_n[r.sys];
        sl.yoff[k] = yd;
        jobs[k].sys = r.sys;
        jobs[k].out = k;
        jobs[k].ered = r.ered;
        jobs[k].yoff = (long long)yd;
        yd += (size_t)n * n;
        nhmax = std::max(nhmax, sys_nham[r.sys]);
    }
    sl.ydoubles = yd;
    // pinned: Y (in and out), JobDev, outputs, then an arena for descriptor uploads
    const size_t arena = (size_t)M * 4 * sizeof(big::MatDesc) + 4096;
    const size_t need = yd * 8 + (size_t)M * sizeof(JobDev) + 3 * (size_t)M * sizeof(int) + arena + 256;
    if ((e = grow_pinned(sl, need))) return set_err(MGPU_ERR_NOMEM, "pinned staging", e);
    sl.y_pin = (double *)sl.pin;
    JobDev *j_pin = (JobDev *)(sl.pin + yd * 8);
    sl.out_pin = (int *)(j_pin + M);
    sl.pin_used = (size_t)((char *)(sl.out_pin + 3 * M) - sl.pin);
    sl.pin_used = (sl.pin_used + 255) & ~(size_t)255;
    for (int k = 0; k < M; ++k) {
        const Req &r = *rq[k];
        memcpy(sl.y_pin + sl.yoff[k], r.y0.data(), r.y0.size() * 8);
        j_pin[k] = jobs[k];
    }
    sl.dev.clear();
    cudaStream_t st = sl.st;
    const AllocFn al = [&sl, st](void **q, size_t nb) {
        cudaError_t e2 = cudaMallocAsync(q, nb, st);
        if (e2 == cudaSuccess) sl.dev.push_back(*q);
        return e2;
    };
    const UploadFn up = [&sl, st](void *dst, const void *src, size_t nb) {
        if (sl.pin_used + nb > sl.pin_cap) return cudaErrorMemoryAllocation;
        char *p = sl.pin + sl.pin_used;
        memcpy(p, src, nb);
        sl.pin_used = (sl.pin_used + nb + 255) & ~(size_t)255;
        return cudaMemcpyAsync(dst, p, nb, cudaMemcpyHostToDevice, st);
    };
    double *y_dev = nullptr;
    JobDev *j_dev = nullptr;
    int *o_dev = nullptr;
    if ((e = alloc_n(al, &y_dev, yd)) || (e = alloc_n(al, &j_dev, (size_t)M)) || (e = alloc_n(al, &o_dev, 3 * (size_t)M)))
        return set_err(MGPU_ERR_NOMEM, "batch allocation", e);
    if ((e = cudaMemcpyAsync(y_dev, sl.y_pin, yd * 8, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(j_dev, j_pin, (size_t)M * sizeof(JobDev), cudaMemcpyHostToDevice, st)))
        return set_err(MGPU_ERR_CUDA, "batch upload", e);
    int *nodes = o_dev, *status = o_dev + M, *kfail = o_dev + 2 * M;
    if (kBuckets[b].kind == KIND_BIG) {
        BigBucket g;
        int mx = 0;
        for (const JobDev &jd : jobs) mx = std::max(mx, sys_nstep[jd.sys]);
        const int rc = setup_big(g, iprop, b, jobs.data(), j_dev, M, mx, {}, hs, sys_n, sys_nstep, d_prep, al, up);
        if (rc) return rc;
        e = run_big_prop(g, iprop, d_sys, y_dev, nodes, status, kfail, st, BigAux{sl.side, sl.evf, sl.evj});
        sl.graph = g.step_graph;  // destroyed when the batch retires
        if (e) return set_err(MGPU_ERR_CUDA, "large-N batch", e);
    } else {
        int use_vl = 0;
        const size_t smem = prop_smem(iprop, b, nhmax, &use_vl);
        if ((e = launch_prop(iprop, b, M, smem, use_vl, st, d_sys, j_dev, y_dev, nodes, status, kfail)))
            return set_err(MGPU_ERR_CUDA, "batch launch", e);
    }
    if ((e = cudaMemcpyAsync(sl.y_pin, y_dev, yd * 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(sl.out_pin, o_dev, 3 * (size_t)M * sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaEventRecord(sl.done, st)))
        return set_err(MGPU_ERR_CUDA, "batch download", e);
    sl.bytes = bytes;
    return MGPU_OK;
}

// Retire finished batches (called without the mutex; takes it to publish).
bool mgpu_server::retire()
{
    bool any = false;
    for (Slot &sl : slots) {
        if (!sl.busy) continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady) continue;
        {
            std::lock_guard<std::mutex> lk(mu);
            const double t = now();
            const int M = (int)sl.tickets.size();
            for (int k = 0; k < M; ++k) {
                auto it = reqs.find(sl.tickets[k]);
                if (it == reqs.end()) continue;
                Req &r = it->second;
                const int n = sys_n[r.sys];
                if (q == cudaSuccess) {
                    memcpy(r.y, sl.y_pin + sl.yoff[k], (size_t)n * n * 8);
                    *r.nodes = sl.out_pin[k];
                    *r.status = sl.out_pin[M + k];
                    *r.kfail = sl.out_pin[2 * M + k];
                } else {
                    r.rc = MGPU_ERR_CUDA;
                }
                r.state = 2;
                r.t[2] = t;
            }
            in_use -= sl.bytes;
        }
        for (void *p : sl.dev) cudaFreeAsync(p, sl.st);
        sl.dev.clear();
        if (sl.graph) cudaGraphExecDestroy(sl.graph);
        sl.graph = nullptr;
        sl.bytes = 0;
        sl.busy = false;
        sl.tickets.clear();
        any = true;
    }
    if (any) cv_done.notify_all();
    return any;
}

// Admit pending requests onto free slots (called without the mutex).
bool mgpu_server::admit()
{
    bool any = false;
    for (;;) {
        Slot *free_slot = nullptr;
        for (Slot &sl : slots)
            if (!sl.busy) {
                free_slot = &sl;
                break;
            }
        if (!free_slot) break;
        std::vector<long long> take;
        std::vector<const Req *> rq;
        int b = -1;
        size_t bytes = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            if (pending.empty()) break;
            b = sys_bucket[reqs[pending.front()].sys];
            for (auto it = pending.begin(); it != pending.end() && (int)take.size() < max_batch; ++it) {
                const Req &r = reqs[*it];
                if (sys_bucket[r.sys] != b) continue;
                const size_t jb = job_bytes(b, sys_n[r.sys]);
                if (in_use + bytes + jb > budget) break;
                take.push_back(*it);
                rq.push_back(&r);  // unordered_map nodes keep their address
                bytes += jb;
            }
            if (take.empty()) {
                if (in_use > 0) break;  // wait for memory to free up
                // the oldest request alone exceeds the budget
                Req &r = reqs[pending.front()];
                r.rc = MGPU_ERR_NOMEM;
                r.state = 2;
                r.t[2] = now();
                pending.pop_front();
                cv_done.notify_all();
                any = true;
                continue;
            }
            for (long long tk : take) pending.erase(std::find(pending.begin(), pending.end(), tk));
            in_use += bytes;  // reserved before launching
        }
        const int rc = launch(*free_slot, take, rq, b, bytes);
        {
            std::lock_guard<std::mutex> lk(mu);
            const double t = now();
            for (long long tk : take) {
                Req &r = reqs[tk];
                if (rc) {
                    r.rc = rc;
                    r.state = 2;
                    r.t[2] = t;
                } else {
                    r.state = 1;
                    r.t[1] = t;
                }
            }
            if (rc) in_use -= bytes;
        }
        if (rc) {
            // nothing of the batch is in flight: release what was allocated
            cudaStreamSynchronize(free_slot->st);
            cudaStreamSynchronize(free_slot->side);
            for (void *p : free_slot->dev) cudaFreeAsync(p, free_slot->st);
            free_slot->dev.clear();
            if (free_slot->graph) cudaGraphExecDestroy(free_slot->graph);
            free_slot->graph = nullptr;
            free_slot->bytes = 0;
            cv_done.notify_all();
        } else {
            free_slot->busy = true;
        }
        any = true;
    }
    return any;
}

void mgpu_server::loop()
{
    cudaSetDevice(dev);
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(mu);
            if (stop) break;
        }
        const bool r = retire();
        const bool a = admit();
        if (!r && !a) {
            std::unique_lock<std::mutex> lk(mu);
            if (stop) break;
            cv_work.wait_for(lk, std::chrono::microseconds(50));
        }
    }
}

mgpu_server::~mgpu_server()
{
    {
        std::lock_guard<std::mutex> lk(mu);
        stop = true;
    }
    cv_work.notify_all();
    if (th.joinable()) th.join();
    cudaSetDevice(dev);
    for (Slot &sl : slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        if (sl.side) cudaStreamSynchronize(sl.side);
        for (void *p : sl.dev) cudaFreeAsync(p, sl.st);
        if (sl.st) cudaStreamSynchronize(sl.st);
        if (sl.graph) cudaGraphExecDestroy(sl.graph);
        if (sl.pin) cudaFreeHost(sl.pin);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.evf) cudaEventDestroy(sl.evf);
        if (sl.evj) cudaEventDestroy(sl.evj);
        if (sl.side) cudaStreamDestroy(sl.side);
        if (sl.st) cudaStreamDestroy(sl.st);
    }
    if (reg) cudaStreamSynchronize(reg);
    for (void *p : allocs) cudaFree(p);
    if (reg_evf) cudaEventDestroy(reg_evf);
    if (reg_evj) cudaEventDestroy(reg_evj);
    if (reg_side) cudaStreamDestroy(reg_side);
    if (reg) cudaStreamDestroy(reg);
}

extern "C" {

int mgpu_server_create(mgpu_server **out, int iprop, size_t hbm_budget_bytes, int streams, int max_batch,
                       int max_systems)
{
    if (!out) return set_err(MGPU_ERR_ARG, "null server pointer");
    *out = nullptr;
    if (iprop != MGPU_PROP_LDMD && iprop != MGPU_PROP_LDJ) return set_err(MGPU_ERR_ARG, "IPROP must be 5 or 6");
    if (streams < 1 || streams > 64 || max_batch < 1 || max_batch > 65535 || max_systems < 1 || hbm_budget_bytes == 0)
        return set_err(MGPU_ERR_ARG, "streams 1..64, max_batch 1..65535, max_systems >= 1, budget > 0");
    mgpu_server *s = new (std::nothrow) mgpu_server();
    if (!s) return set_err(MGPU_ERR_NOMEM, "host allocation failed");
    s->iprop = iprop;
    s->budget = hbm_budget_bytes;
    s->max_batch = max_batch;
    s->cap = max_systems;
    // the scheduler reads these without the lock: they must never reallocate
    s->hs.reserve(max_systems);
    s->sys_n.reserve(max_systems);
    s->sys_nstep.reserve(max_systems);
    s->sys_bucket.reserve(max_systems);
    s->sys_nham.reserve(max_systems);
    cudaError_t e;
    int lo = 0, hi = 0;
    if ((e = cudaGetDevice(&s->dev)) || (e = cudaDeviceGetStreamPriorityRange(&lo, &hi))) {
        delete s;
        return set_err(MGPU_ERR_CUDA, "no CUDA device", e);
    }
    // keep freed batch memory in the device's stream-ordered pool
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->dev) == cudaSuccess) {
        uint64_t thr = (uint64_t)hbm_budget_bytes;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    std::vector<int> ids(max_systems);
    for (int i = 0; i < max_systems; ++i) ids[i] = i;
    const AllocFn al = [s](void **q, size_t nb) {
        cudaError_t e2 = cudaMalloc(q, nb);
        if (e2 == cudaSuccess) s->allocs.push_back(*q);
        return e2;
    };
    const UploadFn up = [](void *dst, const void *src, size_t nb) {
        return cudaMemcpy(dst, src, nb, cudaMemcpyHostToDevice);
    };
    if ((e = alloc_n(al, &s->d_sys, (size_t)max_systems)) || (e = alloc_n(al, &s->d_prep, 3 * (size_t)max_systems)) ||
        (e = put_n(al, up, &s->d_list, ids.data(), ids.size())) ||
        (e = cudaStreamCreateWithFlags(&s->reg, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithPriority(&s->reg_side, cudaStreamNonBlocking, hi)) ||
        (e = cudaEventCreateWithFlags(&s->reg_evf, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&s->reg_evj, cudaEventDisableTiming)) || (e = big_kernel_attributes())) {
        delete s;
        return set_err(MGPU_ERR_NOMEM, "server set-up", e);
    }
    s->slots.resize(streams);
    for (auto &sl : s->slots)
        if ((e = grow_pinned(sl, (size_t)32 << 20)) ||  // staging up front: allocating it later can wait on the GPU
            (e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking)) ||
            (e = cudaStreamCreateWithPriority(&sl.side, cudaStreamNonBlocking, hi)) ||
            (e = cudaEventCreateWithFlags(&sl.evf, cudaEventDisableTiming)) ||
            (e = cudaEventCreateWithFlags(&sl.evj, cudaEventDisableTiming)) ||
            (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming))) {
            delete s;
            return set_err(MGPU_ERR_CUDA, "server streams", e);
        }
    s->th = std::thread([s] { s->loop(); });
    *out = s;
    return MGPU_OK;
}

void mgpu_server_destroy(mgpu_server *s) { delete s; }

int mgpu_server_add_system(mgpu_server *s, const mgpu_coupling *c, const mgpu_grid *g, int *sys_id)
{
    if (!s || !sys_id) return set_err(MGPU_ERR_ARG, "null server or id");
    int rc = check_coupling(c, g, s->iprop);
    if (rc) return rc;
    cudaSetDevice(s->dev);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->nsys >= s->cap) return set_err(MGPU_ERR_UNSUPPORTED, "server system capacity reached");
    const int sid = s->nsys;
    const int b = bucket_for(c->n, s->iprop);
    const AllocFn al = [s](void **q, size_t nb) {
        cudaError_t e2 = cudaMalloc(q, nb);
        if (e2 == cudaSuccess) s->allocs.push_back(*q);
        return e2;
    };
    const UploadFn up = [s](void *dst, const void *src, size_t nb) {
        cudaError_t e2 = cudaMemcpyAsync(dst, src, nb, cudaMemcpyHostToDevice, s->reg);
        return e2 ? e2 : cudaStreamSynchronize(s->reg);
    };
    SysDev d;
    if ((rc = build_sysdev(*c, *g, s->iprop, b, d, al, up))) return rc;
    d.prep = s->d_prep + 3 * sid;
    cudaError_t e;
    if ((e = up(s->d_sys + sid, &d, sizeof d))) return set_err(MGPU_ERR_CUDA, "registering a system", e);
    s->hs.push_back(d);
    s->sys_n.push_back(c->n);
    s->sys_nstep.push_back(g->nstep);
    s->sys_bucket.push_back(b);
    s->sys_nham.push_back(c->nham);
    // counters, and for MDPROP the energy-independent 2HQ(C) table, once
    prep_reset_kernel<<<1, 128, 0, s->reg>>>(s->d_prep + 3 * sid, 1);
    if (s->iprop == MGPU_PROP_LDMD) {
        if (kBuckets[b].kind == KIND_BIG) {
            std::vector<void *> tmp;
            const AllocFn tal = [&tmp](void **q, size_t nb) {
                cudaError_t e2 = cudaMalloc(q, nb);
                if (e2 == cudaSuccess) tmp.push_back(*q);
                return e2;
            };
            BigBucket gb;
            rc = setup_big(gb, s->iprop, b, nullptr, nullptr, 0, 0, {sid}, s->hs, s->sys_n, s->sys_nstep, s->d_prep,
                           tal, up);
            if (!rc && (e = run_big_prep(gb, s->d_sys, s->sys_nstep, s->reg, BigAux{s->reg_side, s->reg_evf, s->reg_evj})))
                rc = set_err(MGPU_ERR_CUDA, "large-N preparation", e);
            cudaStreamSynchronize(s->reg);
            for (void *q : tmp) cudaFree(q);
            if (rc) return rc;
        } else if ((e = launch_prep(b, g->nstep, 1, s->reg, s->d_sys, s->d_list + sid))) {
            return set_err(MGPU_ERR_CUDA, "preparation", e);
        }
    }
    if ((e = cudaStreamSynchronize(s->reg))) return set_err(MGPU_ERR_CUDA, "registering a system", e);
    s->nsys = sid + 1;
    *sys_id = sid;
    return MGPU_OK;
}

int mgpu_submit(mgpu_server *s, int sys_id, double ered, const double *y0, double *y_out, int *nodes, int *status,
                int *kfail, long long *ticket)
{
    if (!s || !y0 || !y_out || !nodes || !status || !kfail || !ticket) return set_err(MGPU_ERR_ARG, "null argument");
    if (!std::isfinite(ered)) return set_err(MGPU_ERR_ARG, "ERED must be finite");
    std::lock_guard<std::mutex> lk(s->mu);
    if (sys_id < 0 || sys_id >= s->nsys) return set_err(MGPU_ERR_ARG, "unknown system id");
    const int n = s->sys_n[sys_id];
    mgpu_server::Req r;
    r.sys = sys_id;
    r.ered = ered;
    r.y0.assign(y0, y0 + (size_t)n * n);
    r.y = y_out;
    r.nodes = nodes;
    r.status = status;
    r.kfail = kfail;
    r.t[0] = mgpu_server::now();
    const long long tk = s->next_ticket++;
    s->reqs.emplace(tk, std::move(r));
    s->pending.push_back(tk);
    *ticket = tk;
    s->cv_work.notify_one();
    return MGPU_OK;
}

int mgpu_poll(mgpu_server *s, long long ticket)
{
    if (!s) return set_err(MGPU_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return -MGPU_ERR_ARG;
    return it->second.state == 2 ? 1 : 0;
}

int mgpu_wait(mgpu_server *s, long long ticket)
{
    if (!s) return set_err(MGPU_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_err(MGPU_ERR_ARG, "unknown ticket");
    s->cv_done.wait(lk, [&] { return it->second.state == 2; });
    return it->second.rc;
}

int mgpu_request_times(mgpu_server *s, long long ticket, double *t3)
{
    if (!s || !t3) return set_err(MGPU_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_err(MGPU_ERR_ARG, "unknown ticket");
    for (int i = 0; i < 3; ++i) t3[i] = it->second.t[i];
    return MGPU_OK;
}

int mgpu_release(mgpu_server *s, long long ticket)
{
    if (!s) return set_err(MGPU_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_err(MGPU_ERR_ARG, "unknown ticket");
    if (it->second.state != 2) return set_err(MGPU_ERR_ARG, "request still in flight");
    s->reqs.erase(it);
    return MGPU_OK;
}

int mgpu_server_in_flight(mgpu_server *s, int *batches, int *queued, size_t *bytes)
{
    if (!s) return set_err(MGPU_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    int nb = 0;
    for (const auto &sl : s->slots) nb += sl.busy ? 1 : 0;
    if (batches) *batches = nb;
    if (queued) *queued = (int)s->pending.size();
    if (bytes) *bytes = s->in_use;
    return MGPU_OK;
}

}  // extern "C"
