// lbf_server.cu -- batched solve server of the C ABI (lbf_server_*).
//
// The reference runs one box per process (LBFAST.f90 -> integrator_module.f90),
// so it has nothing like this; the server is what serving many small solves
// on one B200 needs.  A box of 32^3 fills 16 CTAs of the step kernel, about a
// tenth of the 148 SMs, so running such solves one at a time leaves the GPU
// mostly idle.  Here every resident solve keeps its fields in device memory
// and one launch of the batched step kernel advances ALL resident solves of a
// kernel class by one time step: the launch walks a work list of (solve,
// range of column-planes) items, one per CTA, whose per-solve parameters
// (pointers of the current and next time level, scales, physics) sit in a
// device array.  A chunk of steps is captured once as a CUDA graph and
// replayed until the set of resident solves changes.
//
// Admission is first in, first out against a device-memory budget: a solve's
// resident bytes are its two time levels of every field (see
// lbf_server_solve_bytes); a finished solve's fields are copied to host memory
// and its device memory is released at the end of the chunk in which it
// finished, which lets the next queued solves in.
//
// Each solve's arithmetic is the single-box kernel's (the same device
// function, step_body, with the same parameters), so a solve's result does not
// depend on the other resident solves, nor on the z segmentation the server
// picks for the batch.
#include <cuda_runtime.h>
#include <time.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lbfast_gpu.h"
#include "lbf_handle.h"
#include "lbf_internal.h"

namespace {

int sfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    lbf::record_error(buf);
    return code;
}

#define SRV_TRY(expr)                                                                                \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess) return sfail(LBF_E_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

double now_mono() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

struct Solve {
    long long id = 0;
    lbf_params p{};
    int dtype = LBF_F64;
    long long nsteps = 0;
    long long N = 0;
    std::vector<unsigned char> mom, phi;  // inputs until admission, results once done
    std::vector<int8_t> isf;
    lbf_handle* h = nullptr;
    int state = LBF_SOLVE_QUEUED;
    long long done = 0;
    long long bytes = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::string error;
};

struct ClassKey {
    int lat, ho, tc, obs, storage, tile;
    bool operator<(const ClassKey& o) const {
        if (lat != o.lat) return lat < o.lat;
        if (ho != o.ho) return ho < o.ho;
        if (tc != o.tc) return tc < o.tc;
        if (obs != o.obs) return obs < o.obs;
        if (storage != o.storage) return storage < o.storage;
        return tile < o.tile;
    }
};

// resident solves of one kernel class and the device arrays of their launch
struct Batch {
    lbf::BatchOps ops{};
    std::vector<Solve*> members;
    void* d_params[2] = {nullptr, nullptr};  // [parity][member] device-format step parameters
    size_t params_cap = 0;
    int4* d_work = nullptr;
    size_t work_cap = 0;
    int nwork = 0;
    std::vector<unsigned char> h_params[2];
    std::vector<int4> h_work;
};

// tile height of a solve's class: the one requested, else 8 rows.  A batch of
// small boxes has few 16-row columns to spread over the SMs (measured on the
// droplet ensemble: 4.9 solves/s with 8 rows, 4.1 with 16).
int solve_tile(const lbf_params& p) { return p.tile_y ? p.tile_y : 8; }

}  // namespace

struct lbf_server {
    lbf_server_config cfg{};
    cudaStream_t stream = nullptr;
    // uploads and set-up of newly admitted solves, which overlap the chunk of
    // steps running on `stream`
    cudaStream_t upload = nullptr;
    long long next_id = 1;
    std::map<long long, std::unique_ptr<Solve>> solves;
    std::deque<Solve*> queue;
    std::vector<Solve*> active;
    long long resident = 0;
    std::map<ClassKey, Batch> batches;
    bool dirty = true;
    int phase = 0;  // parity of the next step relative to the last rebuild
    cudaGraphExec_t graph = nullptr;
    int graph_phase = -1;
};

namespace {

void drop_graph(lbf_server* s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->graph_phase = -1;
}

void free_batch(Batch& b) {
    cudaFree(b.d_params[0]);
    cudaFree(b.d_params[1]);
    cudaFree(b.d_work);
    b.d_params[0] = b.d_params[1] = nullptr;
    b.d_work = nullptr;
    b.params_cap = b.work_cap = 0;
}

size_t host_bytes(int dtype) { return dtype == LBF_F64 ? 8 : 4; }

void release(lbf_server* s, Solve* v) {
    if (v->h) {
        lbf_destroy(v->h);
        v->h = nullptr;
        s->resident -= v->bytes;
    }
}

// first in, first out: stop at the first queued solve that does not fit
int admit(lbf_server* s) {
    while (!s->queue.empty()) {
        Solve* v = s->queue.front();
        if (s->cfg.max_active > 0 && (int)s->active.size() >= s->cfg.max_active) break;
        if (s->resident + v->bytes > s->cfg.mem_budget) break;
        s->queue.pop_front();
        lbf_handle* h = nullptr;
        int rc = lbf_create(&v->p, &h);
        if (rc == LBF_OK) rc = lbf_set_stream(h, s->upload);
        if (rc == LBF_OK && v->p.obstacles) rc = lbf_set_isfluid(h, v->isf.data());
        if (rc == LBF_OK)
            rc = lbf_set_fields(h, v->mom.data(), v->p.twocomponent ? v->phi.data() : nullptr, v->dtype);
        if (rc == LBF_OK) rc = lbf::handle_prime(h);
        // the solve's state is complete before it joins the steps on `stream`
        if (rc == LBF_OK && cudaStreamSynchronize(s->upload) != cudaSuccess)
            rc = sfail(LBF_E_CUDA, "solve set-up failed");
        if (rc == LBF_OK) rc = lbf_set_stream(h, s->stream);
        if (rc != LBF_OK) {
            char msg[512];
            lbf_last_error(msg, sizeof msg);
            v->error = msg;
            v->state = LBF_SOLVE_FAILED;
            v->t_done = now_mono();
            if (h) lbf_destroy(h);
            continue;
        }
        lbf::handle_release_staging(h);
        v->h = h;
        v->state = LBF_SOLVE_ACTIVE;
        v->t_admit = now_mono();
        std::vector<unsigned char>().swap(v->mom);
        std::vector<unsigned char>().swap(v->phi);
        std::vector<int8_t>().swap(v->isf);
        s->resident += v->bytes;
        s->active.push_back(v);
        s->dirty = true;
    }
    return LBF_OK;
}

// regroup the resident solves by kernel class and upload their launch tables
int rebuild(lbf_server* s) {
    drop_graph(s);
    for (auto& kv : s->batches) kv.second.members.clear();
    for (Solve* v : s->active) {
        ClassKey k{v->p.lattice, v->p.highorder, lbf::kernel_tc(v->p), v->p.obstacles ? 1 : 0, v->p.storage,
                   solve_tile(v->p)};
        Batch& b = s->batches[k];
        if (!b.ops.launch) {
            b.ops = lbf::batch_ops(k.storage, k.lat, k.ho, k.tc, k.obs, k.tile);
            if (!b.ops.launch) return sfail(LBF_E_UNSUPPORTED, "no batched kernel for this class");
            // sets the kernel's shared-memory attribute outside any graph capture
            SRV_TRY(b.ops.launch(nullptr, nullptr, 0, s->stream));
        }
        b.members.push_back(v);
    }
    for (auto it = s->batches.begin(); it != s->batches.end();) {
        if (it->second.members.empty()) {
            free_batch(it->second);
            it = s->batches.erase(it);
        } else {
            ++it;
        }
    }
    for (auto& kv : s->batches) {
        Batch& b = kv.second;
        std::stable_sort(b.members.begin(), b.members.end(), [](const Solve* a, const Solve* c) { return a->N > c->N; });
        const size_t pb = b.ops.params_bytes;
        const size_t n = b.members.size();
        b.h_params[0].assign(n * pb, 0);
        b.h_params[1].assign(n * pb, 0);
        b.h_work.clear();
        for (size_t i = 0; i < n; ++i) {
            lbf_handle* h = b.members[i]->h;
            lbf::StepArgs a;
            lbf::handle_step_args(h, a, h->dr);
            b.ops.fill(a, b.h_params[0].data() + i * pb);
            lbf_handle flipped = *h;
            flipped.cur = 1 - h->cur;
            lbf::handle_step_args(&flipped, a, h->dr);
            b.ops.fill(a, b.h_params[1].data() + i * pb);
        }
        // z segments per column: whole columns when the batch has at least one
        // wave of columns, else as many segments as still fit in one wave
        // (every segment start recomputes a few planes); one work item per
        // (member, segment, column), the columns of a segment consecutive so
        // that neighbouring columns run at the same planes and their halo
        // re-reads hit in L2
        long long cols = 0;
        for (Solve* v : b.members)
            cols += (long long)((v->p.lx + lbf::STEP_TILE_X - 1) / lbf::STEP_TILE_X) *
                    ((v->p.ly + b.ops.tile_y - 1) / b.ops.tile_y);
        const long long slots = lbf::resident_slots(b.ops.resident());
        const long long nseg = std::max<long long>(1, slots / std::max<long long>(cols, 1));
        for (size_t i = 0; i < n; ++i) {
            lbf_handle* h = b.members[i]->h;
            const int ncol = ((h->nx + lbf::STEP_TILE_X - 1) / lbf::STEP_TILE_X) *
                             ((h->ny + b.ops.tile_y - 1) / b.ops.tile_y);
            const int zseg = std::max((int)((h->nz + nseg - 1) / nseg), std::min(h->nz, 8));
            for (int z0 = 0; z0 < h->nz; z0 += zseg)
                for (int c = 0; c < ncol; ++c) {
                    const long long s0 = (long long)c * h->nz + z0;
                    b.h_work.push_back(make_int4((int)i, (int)s0, (int)(s0 + std::min(zseg, h->nz - z0)), 0));
                }
        }
        b.nwork = (int)b.h_work.size();
        if (b.params_cap < n * pb) {
            const size_t cap = std::max(n * pb, 2 * b.params_cap);
            cudaFree(b.d_params[0]);
            cudaFree(b.d_params[1]);
            b.d_params[0] = b.d_params[1] = nullptr;
            b.params_cap = 0;
            SRV_TRY(cudaMalloc(&b.d_params[0], cap));
            SRV_TRY(cudaMalloc(&b.d_params[1], cap));
            b.params_cap = cap;
        }
        if (b.work_cap < b.h_work.size()) {
            cudaFree(b.d_work);
            b.d_work = nullptr;
            b.work_cap = 0;
            const size_t cap = b.h_work.size();
            SRV_TRY(cudaMalloc(&b.d_work, cap * sizeof(int4)));
            b.work_cap = cap;
        }
        SRV_TRY(cudaMemcpyAsync(b.d_params[0], b.h_params[0].data(), n * pb, cudaMemcpyHostToDevice, s->stream));
        SRV_TRY(cudaMemcpyAsync(b.d_params[1], b.h_params[1].data(), n * pb, cudaMemcpyHostToDevice, s->stream));
        SRV_TRY(cudaMemcpyAsync(b.d_work, b.h_work.data(), b.h_work.size() * sizeof(int4), cudaMemcpyHostToDevice,
                                s->stream));
        // the host tables must outlive the asynchronous copies
        SRV_TRY(cudaStreamSynchronize(s->stream));
    }
    s->phase = 0;
    s->dirty = false;
    return LBF_OK;
}

// issue nsteps steps of every resident solve (directly, or into a capture)
int issue_steps(lbf_server* s, long long nsteps) {
    for (long long k = 0; k < nsteps; ++k) {
        for (auto& kv : s->batches) {
            Batch& b = kv.second;
            for (Solve* v : b.members) {
                int rc = lbf::handle_pre_step(v->h);
                if (rc) return rc;
            }
            SRV_TRY(b.ops.launch(b.d_params[s->phase], b.d_work, b.nwork, s->stream));
            for (Solve* v : b.members) {
                lbf::handle_advance(v->h, v->h->dr);
                int rc = lbf::handle_post_step(v->h);
                if (rc) return rc;
            }
        }
        s->phase ^= 1;
    }
    return LBF_OK;
}

// one chunk of nsteps (even) steps as a CUDA graph: captured when the resident
// set changed, replayed otherwise (the per-step work repeats with period two)
int graph_steps(lbf_server* s, long long nsteps) {
    if (s->graph && s->graph_phase == s->phase) {
        SRV_TRY(cudaGraphLaunch(s->graph, s->stream));
        for (Solve* v : s->active) v->h->step += nsteps;
        return LBF_OK;
    }
    drop_graph(s);
    const int phase0 = s->phase;
    SRV_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = issue_steps(s, nsteps);  // advances the host-side state as the graph will
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return sfail(LBF_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        s->graph = nullptr;
        return sfail(LBF_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    s->graph_phase = phase0;
    SRV_TRY(cudaGraphLaunch(s->graph, s->stream));
    return LBF_OK;
}

int retire(lbf_server* s) {
    std::vector<Solve*> keep;
    for (Solve* v : s->active) {
        if (v->done < v->nsteps) {
            keep.push_back(v);
            continue;
        }
        const size_t hb = host_bytes(v->dtype);
        v->mom.resize(10 * v->N * hb);
        if (v->p.twocomponent) v->phi.resize(v->N * hb);
        int rc = lbf_get_fields(v->h, v->mom.data(), v->p.twocomponent ? v->phi.data() : nullptr, nullptr, v->dtype);
        if (rc != LBF_OK) {
            char msg[512];
            lbf_last_error(msg, sizeof msg);
            v->error = msg;
            v->state = LBF_SOLVE_FAILED;
        } else {
            v->state = LBF_SOLVE_DONE;
        }
        release(s, v);
        v->t_done = now_mono();
        s->dirty = true;
    }
    s->active.swap(keep);
    return LBF_OK;
}

Solve* find(lbf_server* s, long long id) {
    auto it = s->solves.find(id);
    return it == s->solves.end() ? nullptr : it->second.get();
}

}  // namespace

extern "C" {

long long lbf_server_solve_bytes(const lbf_params* p) {
    if (!p) return -1;
    // fields of both time levels, the error flag and the reduction scratch
    return (long long)lbf::handle_bytes(p) + 64;
}

int lbf_server_create(const lbf_server_config* cfg, lbf_server** out) {
    if (!out) return sfail(LBF_E_ARG, "lbf_server_create: null argument");
    *out = nullptr;
    lbf_server* s = new (std::nothrow) lbf_server();
    if (!s) return sfail(LBF_E_NOMEM, "host allocation failed");
    if (cfg) s->cfg = *cfg;
    if (s->cfg.chunk <= 0) s->cfg.chunk = 32;
    if (s->cfg.chunk % 2) {
        delete s;
        return sfail(LBF_E_ARG, "chunk must be even");
    }
    if (!cfg) s->cfg.use_graph = 1;
    if (s->cfg.mem_budget <= 0) {
        size_t fr = 0, tot = 0;
        cudaError_t e = cudaMemGetInfo(&fr, &tot);
        if (e != cudaSuccess) {
            delete s;
            return sfail(LBF_E_CUDA, "cudaMemGetInfo: %s", cudaGetErrorString(e));
        }
        s->cfg.mem_budget = (long long)(0.8 * (double)fr);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return sfail(LBF_E_CUDA, "stream: %s", cudaGetErrorString(e));
    }
    *out = s;
    return LBF_OK;
}

int lbf_server_destroy(lbf_server* s) {
    if (!s) return sfail(LBF_E_ARG, "lbf_server_destroy: null server");
    cudaStreamSynchronize(s->stream);
    drop_graph(s);
    for (Solve* v : s->active) release(s, v);
    for (auto& kv : s->batches) free_batch(kv.second);
    cudaStreamDestroy(s->stream);
    cudaStreamDestroy(s->upload);
    delete s;
    return LBF_OK;
}

int lbf_server_submit(lbf_server* s, const lbf_params* p, const int8_t* isfluid, const void* mom10, const void* phi,
                      int dtype, long long nsteps, long long* id) {
    if (!s || !p || !mom10 || !id) return sfail(LBF_E_ARG, "lbf_server_submit: null argument");
    if (dtype != LBF_F32 && dtype != LBF_F64) return sfail(LBF_E_ARG, "dtype must be LBF_F32 or LBF_F64");
    if (nsteps < 0) return sfail(LBF_E_ARG, "nsteps < 0");
    if (p->twocomponent && !phi) return sfail(LBF_E_ARG, "two-component solve without phi");
    if (p->obstacles && !isfluid) return sfail(LBF_E_ARG, "obstacle solve without isfluid");
    if (p->lx < 1 || p->ly < 1 || p->lz < 1) return sfail(LBF_E_ARG, "box must be at least 1^3");
    auto v = std::make_unique<Solve>();
    v->p = *p;
    v->dtype = dtype;
    v->nsteps = nsteps;
    v->N = (long long)p->lx * p->ly * p->lz;
    v->bytes = lbf_server_solve_bytes(p);
    if (v->bytes > s->cfg.mem_budget)
        return sfail(LBF_E_NOMEM, "solve needs %lld device bytes, the budget is %lld", v->bytes, s->cfg.mem_budget);
    const size_t hb = host_bytes(dtype);
    const unsigned char* m = static_cast<const unsigned char*>(mom10);
    v->mom.assign(m, m + 10 * v->N * hb);
    if (p->twocomponent) {
        const unsigned char* f = static_cast<const unsigned char*>(phi);
        v->phi.assign(f, f + v->N * hb);
    }
    if (p->obstacles) v->isf.assign(isfluid, isfluid + v->N);
    v->id = s->next_id++;
    v->t_submit = now_mono();
    *id = v->id;
    s->queue.push_back(v.get());
    s->solves[v->id] = std::move(v);
    return LBF_OK;
}

int lbf_server_run(lbf_server* s, int max_chunks, int* active, int* queued) {
    if (!s) return sfail(LBF_E_ARG, "lbf_server_run: null server");
    int rc = LBF_OK;
    for (int c = 0; c < max_chunks && rc == LBF_OK; ++c) {
        if (c == 0) admit(s);
        if (s->active.empty()) break;
        if (s->dirty && (rc = rebuild(s))) break;
        long long L = s->cfg.chunk;
        bool steady = true;
        for (Solve* v : s->active) {
            L = std::min(L, v->nsteps - v->done);
            steady = steady && lbf::handle_steady(v->h);
        }
        if (L > 0) {
            if (!steady) L = 1;  // first step of a wetting solve: its per-step work is not periodic yet
            if (s->cfg.use_graph && L == s->cfg.chunk)
                rc = graph_steps(s, L);
            else
                rc = issue_steps(s, L);
            if (rc) break;
            for (Solve* v : s->active) v->done += L;
        }
        // solves that fit next to the resident ones are uploaded while the
        // chunk runs; they join at the next rebuild
        admit(s);
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) {
            rc = sfail(LBF_E_CUDA, "server step: %s", cudaGetErrorString(e));
            break;
        }
        rc = retire(s);
    }
    if (rc == LBF_OK) admit(s);
    if (active) *active = (int)s->active.size();
    if (queued) *queued = (int)s->queue.size();
    return rc;
}

int lbf_server_poll(lbf_server* s, long long id, lbf_solve_info* info) {
    if (!s || !info) return sfail(LBF_E_ARG, "lbf_server_poll: null argument");
    Solve* v = find(s, id);
    if (!v) return sfail(LBF_E_ARG, "unknown solve id %lld", id);
    info->state = v->state;
    info->steps_done = v->done;
    info->nsteps = v->nsteps;
    info->device_bytes = v->bytes;
    info->t_submit = v->t_submit;
    info->t_admit = v->t_admit;
    info->t_done = v->t_done;
    return LBF_OK;
}

int lbf_server_fetch(lbf_server* s, long long id, void* mom10, void* phi) {
    if (!s) return sfail(LBF_E_ARG, "lbf_server_fetch: null server");
    Solve* v = find(s, id);
    if (!v) return sfail(LBF_E_ARG, "unknown solve id %lld", id);
    if (v->state == LBF_SOLVE_FAILED) {
        std::string msg = v->error;
        s->solves.erase(id);
        return sfail(LBF_E_STATE, "solve %lld failed: %s", id, msg.c_str());
    }
    if (v->state != LBF_SOLVE_DONE) return sfail(LBF_E_STATE, "solve %lld is not done", id);
    if (mom10) std::memcpy(mom10, v->mom.data(), v->mom.size());
    if (phi && v->p.twocomponent) std::memcpy(phi, v->phi.data(), v->phi.size());
    s->solves.erase(id);
    return LBF_OK;
}

int lbf_server_cancel(lbf_server* s, long long id) {
    if (!s) return sfail(LBF_E_ARG, "lbf_server_cancel: null server");
    Solve* v = find(s, id);
    if (!v) return sfail(LBF_E_ARG, "unknown solve id %lld", id);
    if (v->state == LBF_SOLVE_QUEUED) {
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), v));
    } else if (v->state == LBF_SOLVE_ACTIVE) {
        SRV_TRY(cudaStreamSynchronize(s->stream));
        release(s, v);
        s->active.erase(std::find(s->active.begin(), s->active.end(), v));
        s->dirty = true;
    }
    s->solves.erase(id);
    return LBF_OK;
}

}  // extern "C"
