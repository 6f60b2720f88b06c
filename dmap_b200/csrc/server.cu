// The serving loop of include/dmap_b200.h (dmap_server_*): a worker thread
// that admits queued requests against a device-memory budget, packs the
// pieces of admitted ray requests of one scene and mode into one query per
// launch slot, runs render requests one batch of samples per slot turn, and
// refills each slot as soon as its launch finishes while the other slots'
// launches run. Host C++ over the CUDA runtime; the kernels are the query
// path's and the path tracer's.
#include "api_internal.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>
#include <unordered_set>

using namespace dmapi;
using Clock = std::chrono::steady_clock;

namespace
{

enum class Kind { Rays, Render };
enum class State { Queued, Active, Done };

struct Request
{
    uint64_t id = 0;
    Kind kind = Kind::Rays;
    dmap_scene *scene = nullptr;
    int mode = DMAP_MODE_CLOSEST;
    // ray requests
    const float *rays = nullptr;
    dmap_hit32 *hits = nullptr;
    int64_t n = 0, next = 0, answered = 0;
    bool pin_in = false, pin_out = false;
    // render requests
    dmap_render_desc desc{};
    float *rgb = nullptr;
    RenderJob *job = nullptr;
    cudaEvent_t ready = nullptr; // the job's buffers are cleared
    bool running = false;        // a batch of the job is in a slot
    int batches_done = 0;
    // bookkeeping
    size_t bytes = 0; // device bytes held while active
    State state = State::Queued;
    dmap_status status = DMAP_OK;
    Clock::time_point t_submit, t_done;
};

struct Piece
{
    Request *r;
    int64_t off, n, at; // rays [off, off + n) of r at [at, at + n) of the slot's batch
};

struct Slot
{
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    float *rays_d = nullptr, *rays_pin = nullptr;
    dmapdev::Hit32 *hits_d = nullptr, *hits_pin = nullptr;
    dmapk::WaveScratch wave;
    std::vector<Piece> pieces;
    Request *render = nullptr;
    bool busy = false, staged_out = false;
};

bool is_pinned(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

} // namespace

struct dmap_server
{
    dmap_context *ctx = nullptr;
    dmap_server_config cfg{};
    dmapk::QueryOpts q{};
    int64_t max_batch = 0;
    std::vector<Slot> slots;
    cudaStream_t setup = nullptr; // render jobs' allocation, clearing and graph capture

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queued;
    std::vector<Request *> active; // in admission (= arrival) order
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    uint64_t next_id = 1;
    bool stop = false;
    bool paused = false; // dmap_server_pause: queued requests wait, running ones finish
    std::thread worker;

    size_t held = 0, peak = 0, slot_bytes = 0;
    std::unordered_set<const dmap_asset *> resident;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, rays_done = 0, launches = 0;
    std::vector<double> lat_ms;
    int inflight = 0;
    double busy_s = 0.0;
    Clock::time_point busy_since, t_first;
    bool any = false;

    size_t asset_bytes_new(const dmap_scene *s) const
    {
        size_t b = 0;
        for (const dmap_asset *a : s->assets)
            if (!resident.count(a))
                b += a->bytes;
        return b;
    }

    void complete(Request *r, dmap_status st)
    {
        if (r->state != State::Active)
            return;
        r->status = st;
        r->state = State::Done;
        r->t_done = Clock::now();
        --r->scene->server_pending;
        if (st == DMAP_OK) {
            ++completed;
            lat_ms.push_back(ms_between(r->t_submit, r->t_done));
        } else {
            ++failed;
        }
        held -= r->bytes;
        active.erase(std::find(active.begin(), active.end(), r));
        cv_done.notify_all();
    }

    // Moves queued requests to active, in arrival order, while they fit.
    void admit()
    {
        const int cap = cfg.max_inflight > 0 ? cfg.max_inflight : 256;
        while (!queued.empty() && (int)active.size() < cap) {
            Request *r = queued.front();
            size_t need = r->bytes + asset_bytes_new(r->scene);
            if (cfg.hbm_budget_bytes && held + need > cfg.hbm_budget_bytes)
                break; // arrival order: later requests wait behind this one
            queued.pop_front();
            for (const dmap_asset *a : r->scene->assets)
                resident.insert(a);
            held += need;
            peak = std::max(peak, held);
            r->state = State::Active;
            active.push_back(r);
            if (r->kind == Kind::Render) {
                dmap_status st = render_begin(r->scene, &r->desc, &cfg.options, nullptr, setup, &r->job);
                if (st == DMAP_OK && (cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming) != cudaSuccess ||
                                      cudaEventRecord(r->ready, setup) != cudaSuccess)) {
                    render_free(r->job, setup);
                    r->job = nullptr;
                    st = DMAP_ERR_CUDA;
                }
                if (st != DMAP_OK)
                    complete(r, st);
            }
        }
    }

    // Queries a request has left to issue: its unsent rays, or a render's
    // unsent batches' share of its paths times two queries per vertex.
    static int64_t work_left(const Request *r)
    {
        if (r->kind == Kind::Rays)
            return r->n - r->next;
        const int64_t batches = render_batches(r->job), left = batches - render_enqueued(r->job);
        const int64_t paths = (int64_t)r->desc.camera.width * r->desc.camera.height * r->desc.spp;
        return batches > 0 ? paths * left / batches * 2 * r->desc.max_depth : 0;
    }

    // Puts admitted work into an idle slot: the oldest request's
    // (DMAP_SERVE_OLDEST) or the one with the least work left
    // (DMAP_SERVE_SHORTEST, the oldest of equals); false when there is none.
    bool fill(Slot &sl)
    {
        Request *first = nullptr;
        int64_t first_left = 0;
        for (Request *r : active) {
            if (!(r->kind == Kind::Rays ? r->next < r->n
                                        : (!r->running && r->job && render_enqueued(r->job) < render_batches(r->job))))
                continue;
            if (cfg.policy != DMAP_SERVE_SHORTEST) {
                first = r;
                break;
            }
            const int64_t left = work_left(r);
            if (!first || left < first_left) {
                first = r;
                first_left = left;
            }
        }
        if (!first)
            return false;
        cudaError_t e = cudaSuccess;
        if (first->kind == Kind::Render) {
            Request *r = first;
            if ((e = cudaStreamWaitEvent(sl.stream, r->ready, 0)) == cudaSuccess &&
                (e = render_enqueue_batch(r->job, sl.stream)) == cudaSuccess &&
                (e = cudaEventRecord(sl.done, sl.stream)) == cudaSuccess) {
                r->running = true;
                sl.render = r;
                sl.busy = true;
            }
        } else {
            // this request's scene and mode, every admitted request of them in order
            sl.pieces.clear();
            int64_t at = 0;
            bool all_pinned_out = true;
            for (Request *r : active) {
                if (at == max_batch)
                    break;
                if (r->kind != Kind::Rays || r->scene != first->scene || r->mode != first->mode || r->next >= r->n)
                    continue;
                int64_t k = std::min(r->n - r->next, max_batch - at);
                sl.pieces.push_back({r, r->next, k, at});
                r->next += k;
                at += k;
                all_pinned_out = all_pinned_out && r->pin_out;
            }
            // rays in
            bool staged_in = false;
            for (const Piece &p : sl.pieces) {
                if (p.r->pin_in) {
                    if (e == cudaSuccess)
                        e = cudaMemcpyAsync(sl.rays_d + 8 * p.at, p.r->rays + 8 * p.off, sizeof(float) * 8 * p.n,
                                            cudaMemcpyHostToDevice, sl.stream);
                } else {
                    std::memcpy(sl.rays_pin + 8 * p.at, p.r->rays + 8 * p.off, sizeof(float) * 8 * p.n);
                    staged_in = true;
                }
            }
            if (staged_in && e == cudaSuccess)
                for (const Piece &p : sl.pieces)
                    if (!p.r->pin_in && e == cudaSuccess)
                        e = cudaMemcpyAsync(sl.rays_d + 8 * p.at, sl.rays_pin + 8 * p.at, sizeof(float) * 8 * p.n,
                                            cudaMemcpyHostToDevice, sl.stream);
            // one query over the whole batch
            dmapk::QueryOpts qq = q;
            qq.mode = first->mode;
            qq.bvh_nodes = reinterpret_cast<const float4 *>(first->scene->bvh_nodes_dev);
            qq.bvh_tri = reinterpret_cast<const float4 *>(first->scene->bvh_tri_dev);
            qq.bvh_range = reinterpret_cast<const int4 *>(first->scene->bvh_range_dev);
            qq.inst_xf = first->scene->inst_dev;
            qq.bvh_n_nodes = first->scene->bvh_n_nodes;
            qq.ray_dtype = qq.hit_dtype = 0;
            apply_filter(first->scene, qq); // a filtered scene's batch runs the filter's passes
            dmap_scene *s = first->scene;
            if (e == cudaSuccess)
                e = dmapk::launch_walk32(s->tris32_dev, s->tris_dev, s->n_tri, s->assets_dev, sl.rays_d, at, qq,
                                         sl.hits_d, nullptr, ctx->status_dev, sl.wave, sl.stream);
            if (e == cudaSuccess)
                ctx->launches += dmapk::walk32_launches(qq);
            // hits out
            sl.staged_out = !all_pinned_out;
            if (e == cudaSuccess) {
                if (all_pinned_out) {
                    for (const Piece &p : sl.pieces)
                        if (e == cudaSuccess)
                            e = cudaMemcpyAsync(p.r->hits + p.off, sl.hits_d + p.at, sizeof(dmap_hit32) * p.n,
                                                cudaMemcpyDeviceToHost, sl.stream);
                } else {
                    e = cudaMemcpyAsync(sl.hits_pin, sl.hits_d, sizeof(dmap_hit32) * at, cudaMemcpyDeviceToHost,
                                        sl.stream);
                }
            }
            if (e == cudaSuccess)
                e = cudaEventRecord(sl.done, sl.stream);
            if (e == cudaSuccess) {
                sl.busy = true;
            } else {
                for (const Piece &p : sl.pieces)
                    if (p.r->state == State::Active)
                        complete(p.r, DMAP_ERR_CUDA);
                sl.pieces.clear();
            }
        }
        if (e != cudaSuccess) {
            if (first->state == State::Active)
                complete(first, DMAP_ERR_CUDA);
            return true;
        }
        ++launches;
        if (inflight++ == 0)
            busy_since = Clock::now();
        return true;
    }

    // A slot's launch is done: hand the results over.
    void retire(Slot &sl)
    {
        sl.busy = false;
        if (--inflight == 0)
            busy_s += std::chrono::duration<double>(Clock::now() - busy_since).count();
        if (sl.render) {
            Request *r = sl.render;
            sl.render = nullptr;
            r->running = false;
            if (++r->batches_done == render_batches(r->job)) {
                dmap_render_stats st{};
                dmap_status s = render_end(r->job, r->rgb, &st, nullptr, 0.0);
                render_free(r->job, setup);
                r->job = nullptr;
                cudaEventDestroy(r->ready);
                r->ready = nullptr;
                rays_done += st.extension_rays + st.shadow_rays;
                complete(r, s);
            }
            return;
        }
        for (const Piece &p : sl.pieces) {
            if (p.r->state != State::Active)
                continue; // failed in another slot
            if (sl.staged_out)
                std::memcpy(p.r->hits + p.off, sl.hits_pin + p.at, sizeof(dmap_hit32) * p.n);
            rays_done += p.n;
            p.r->answered += p.n;
            if (p.r->answered == p.r->n)
                complete(p.r, DMAP_OK);
        }
        sl.pieces.clear();
    }

    void run()
    {
        cudaSetDevice(ctx->device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            bool progressed = false;
            for (Slot &sl : slots)
                if (sl.busy && cudaEventQuery(sl.done) != cudaErrorNotReady) {
                    retire(sl);
                    progressed = true;
                }
            if (!paused)
                admit();
            for (Slot &sl : slots)
                if (!sl.busy && fill(sl))
                    progressed = true;
            bool busy = inflight > 0;
            if (stop && queued.empty() && active.empty() && !busy)
                break;
            if (progressed)
                continue;
            if (busy)
                cv_work.wait_for(lk, std::chrono::microseconds(100));
            else
                cv_work.wait(lk, [&] { return stop || (!paused && !queued.empty()); });
        }
    }

    dmap_status submit(std::unique_ptr<Request> r, uint64_t *id)
    {
        std::lock_guard<std::mutex> lk(mu);
        size_t need = r->bytes + slot_bytes;
        for (const dmap_asset *a : r->scene->assets)
            need += a->bytes;
        if (cfg.hbm_budget_bytes && need > cfg.hbm_budget_bytes)
            return DMAP_ERR_BUDGET;
        r->id = next_id++;
        r->t_submit = Clock::now();
        if (!any) {
            any = true;
            t_first = r->t_submit;
        }
        ++submitted;
        *id = r->id;
        ++r->scene->server_pending;
        queued.push_back(r.get());
        all[r->id] = std::move(r);
        cv_work.notify_one();
        return DMAP_OK;
    }
};

extern "C" {

dmap_status dmap_server_create(dmap_context *ctx, const dmap_server_config *cfg, dmap_server **out)
{
    if (!ctx || !cfg || !out)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_server_create: null argument");
    *out = nullptr;
    if (cfg->max_batch_rays < 0 || cfg->max_inflight < 0 || cfg->slots < 0 || cfg->slots > 8 ||
        (cfg->policy != DMAP_SERVE_OLDEST && cfg->policy != DMAP_SERVE_SHORTEST))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_server_create: bad configuration");
    auto S = std::make_unique<dmap_server>();
    S->ctx = ctx;
    S->cfg = *cfg;
    dmap_scene probe;
    probe.ctx = ctx;
    probe.all_f64 = false;
    dmap_status st = check_query(&probe, DMAP_F32, 0, &cfg->options, DMAP_F32, S->q);
    if (st != DMAP_OK)
        return st;
    if (S->q.precision != DMAP_PRECISION_F32)
        return fail(ctx, DMAP_ERR_UNSUPPORTED, "dmap_server_create: the server runs the FP32 query path");
    S->max_batch = cfg->max_batch_rays > 0 ? cfg->max_batch_rays : (4ll << 20);
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    DMAP_CUDA(ctx, cudaStreamCreateWithFlags(&S->setup, cudaStreamNonBlocking));
    int n_slots = cfg->slots > 0 ? cfg->slots : 2;
    S->slots.resize(n_slots);
    const size_t B = (size_t)S->max_batch;
    for (Slot &sl : S->slots) {
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaMalloc((void **)&sl.rays_d, sizeof(float) * 8 * B)) != cudaSuccess ||
            (e = cudaMalloc((void **)&sl.hits_d, sizeof(dmapdev::Hit32) * B)) != cudaSuccess ||
            (e = cudaHostAlloc((void **)&sl.rays_pin, sizeof(float) * 8 * B, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void **)&sl.hits_pin, sizeof(dmapdev::Hit32) * B, cudaHostAllocDefault)) !=
                cudaSuccess) {
            dmap_server_destroy(S.release());
            return cuda_fail(ctx, e, "dmap_server_create: slot buffers");
        }
        if ((st = wave_reserve(ctx, sl.wave, S->max_batch)) != DMAP_OK) {
            dmap_server_destroy(S.release());
            return st;
        }
        S->slot_bytes += B * (sizeof(float) * 8 + sizeof(dmapdev::Hit32)) + wave_bytes(S->max_batch);
    }
    S->held = S->peak = S->slot_bytes;
    if (cfg->hbm_budget_bytes && S->slot_bytes > cfg->hbm_budget_bytes) {
        dmap_server_destroy(S.release());
        return fail(ctx, DMAP_ERR_BUDGET, "dmap_server_create: the launch slots alone exceed the budget");
    }
    dmap_server *raw = S.release();
    raw->worker = std::thread([raw] { raw->run(); });
    *out = raw;
    return DMAP_OK;
}

void dmap_server_destroy(dmap_server *S)
{
    if (!S)
        return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        for (Request *r : S->queued) {
            r->state = State::Done;
            r->status = DMAP_ERR_CANCELLED;
            --r->scene->server_pending;
            ++S->cancelled;
        }
        S->queued.clear();
        S->cv_work.notify_all();
    }
    if (S->worker.joinable())
        S->worker.join();
    cudaSetDevice(S->ctx->device);
    for (Slot &sl : S->slots) {
        if (sl.stream)
            cudaStreamSynchronize(sl.stream);
        cudaFree(sl.rays_d);
        cudaFree(sl.hits_d);
        cudaFreeHost(sl.rays_pin);
        cudaFreeHost(sl.hits_pin);
        wave_release(sl.wave);
        if (sl.done)
            cudaEventDestroy(sl.done);
        if (sl.stream)
            cudaStreamDestroy(sl.stream);
    }
    if (S->setup) {
        cudaStreamSynchronize(S->setup);
        cudaStreamDestroy(S->setup);
    }
    delete S;
}

dmap_status dmap_server_submit_rays(dmap_server *S, dmap_scene *scene, const float *rays_host, int64_t n, int mode,
                                    dmap_hit32 *hits_host, uint64_t *id)
{
    if (!S || !scene || !id || n < 0 || (n > 0 && (!rays_host || !hits_host)) ||
        (mode != DMAP_MODE_CLOSEST && mode != DMAP_MODE_OCCLUDED) || scene->ctx != S->ctx)
        return DMAP_ERR_INVALID;
    auto r = std::make_unique<Request>();
    r->kind = Kind::Rays;
    r->scene = scene;
    r->mode = mode;
    r->rays = rays_host;
    r->hits = hits_host;
    r->n = n;
    r->pin_in = n > 0 && is_pinned(rays_host);
    r->pin_out = n > 0 && is_pinned(hits_host);
    if (n == 0) {
        std::lock_guard<std::mutex> lk(S->mu);
        r->id = S->next_id++;
        r->t_submit = r->t_done = Clock::now();
        r->state = State::Done;
        ++S->submitted;
        ++S->completed;
        S->lat_ms.push_back(0.0);
        *id = r->id;
        S->all[r->id] = std::move(r);
        return DMAP_OK;
    }
    return S->submit(std::move(r), id);
}

dmap_status dmap_server_submit_render(dmap_server *S, dmap_scene *scene, const dmap_render_desc *desc,
                                      float *rgb_host, uint64_t *id)
{
    if (!S || !scene || !desc || !rgb_host || !id || scene->ctx != S->ctx)
        return DMAP_ERR_INVALID;
    const dmap_camera &C = desc->camera;
    if (C.width <= 0 || C.height <= 0 || desc->spp <= 0 || desc->max_depth < 1)
        return DMAP_ERR_INVALID;
    auto r = std::make_unique<Request>();
    r->kind = Kind::Render;
    r->scene = scene;
    r->desc = *desc;
    r->rgb = rgb_host;
    r->bytes = render_device_bytes(desc, 0);
    return S->submit(std::move(r), id);
}

static Request *find_req(dmap_server *S, uint64_t id)
{
    auto it = S->all.find(id);
    return it == S->all.end() ? nullptr : it->second.get();
}

dmap_status dmap_server_poll(dmap_server *S, uint64_t id)
{
    if (!S)
        return DMAP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Request *r = find_req(S, id);
    if (!r)
        return DMAP_ERR_INVALID;
    return r->state == State::Done ? r->status : DMAP_ERR_NOT_READY;
}

dmap_status dmap_server_wait(dmap_server *S, uint64_t id, double timeout_s)
{
    if (!S)
        return DMAP_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    Request *r = find_req(S, id);
    if (!r)
        return DMAP_ERR_INVALID;
    auto done = [&] { return r->state == State::Done; };
    if (timeout_s < 0)
        S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
        return DMAP_ERR_NOT_READY;
    return r->status;
}

dmap_status dmap_server_pause(dmap_server *S, int paused)
{
    if (!S)
        return DMAP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    S->paused = paused != 0;
    S->cv_work.notify_all();
    return DMAP_OK;
}

dmap_status dmap_server_cancel(dmap_server *S, uint64_t id)
{
    if (!S)
        return DMAP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Request *r = find_req(S, id);
    if (!r)
        return DMAP_ERR_INVALID;
    if (r->state != State::Queued)
        return r->state == State::Done ? r->status : DMAP_ERR_NOT_READY;
    S->queued.erase(std::find(S->queued.begin(), S->queued.end(), r));
    r->state = State::Done;
    r->status = DMAP_ERR_CANCELLED;
    --r->scene->server_pending;
    ++S->cancelled;
    S->cv_done.notify_all();
    return DMAP_ERR_CANCELLED;
}

dmap_status dmap_server_latency(dmap_server *S, uint64_t id, double *ms)
{
    if (!S || !ms)
        return DMAP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Request *r = find_req(S, id);
    if (!r)
        return DMAP_ERR_INVALID;
    if (r->state != State::Done)
        return DMAP_ERR_NOT_READY;
    *ms = ms_between(r->t_submit, r->t_done);
    return r->status;
}

dmap_status dmap_server_drain(dmap_server *S, double timeout_s)
{
    if (!S)
        return DMAP_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto done = [&] { return S->queued.empty() && S->active.empty(); };
    if (timeout_s < 0)
        S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
        return DMAP_ERR_NOT_READY;
    return DMAP_OK;
}

dmap_status dmap_server_get_stats(dmap_server *S, dmap_server_stats *out)
{
    if (!S || !out)
        return DMAP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    dmap_server_stats st{};
    st.submitted = S->submitted;
    st.completed = S->completed;
    st.failed = S->failed;
    st.cancelled = S->cancelled;
    st.queued = (int64_t)S->queued.size();
    st.active = (int64_t)S->active.size();
    st.rays = S->rays_done;
    st.launches = S->launches;
    std::vector<double> l = S->lat_ms;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            // nearest rank
            size_t k = (size_t)std::ceil(p * (double)l.size());
            return l[std::min(l.size() - 1, k > 0 ? k - 1 : 0)];
        };
        st.p50_ms = pct(0.50);
        st.p99_ms = pct(0.99);
        double sum = 0.0;
        for (double x : l)
            sum += x;
        st.mean_ms = sum / (double)l.size();
        st.max_ms = l.back();
    }
    st.held_bytes = S->held;
    st.peak_bytes = S->peak;
    double busy = S->busy_s;
    if (S->inflight > 0)
        busy += std::chrono::duration<double>(Clock::now() - S->busy_since).count();
    st.busy_s = busy;
    st.wall_s = S->any ? std::chrono::duration<double>(Clock::now() - S->t_first).count() : 0.0;
    *out = st;
    return DMAP_OK;
}

} // extern "C"
