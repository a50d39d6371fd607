// serve.cu — continuous-batching request loop for reconstruction requests on one GPU.
//
// A request asks for simulate → signal → residual, the finite-difference derivatives and the
// gradient Jᴴ·r (Cartesian or spiral trajectory). The reference has no serving layer:
// its callers issue these operations one call at a time (src/simulate/fisp.cu, pssfp.cu,
// src/simulate/derivative.cu, src/trajectories/signal.cu, src/utils/residual.cu,
// src/jacobian/hermitian.cu). Here:
//
//  * admission: requests wait in arrival order; the worker admits the oldest ones into a batch
//    while their estimated device footprint (echoes, derivative echoes, signal, residual,
//    split-K partials, per-voxel tables, gradient) fits the memory budget and a batch slot is
//    free. Memory of finished batches and released results returns to the budget;
//  * continuous batching: each slot owns a stream; a batch is launched on a free slot as soon
//    as one exists, so requests that arrive while others run start at once and their kernels
//    overlap with the running batches on the device;
//  * a batch runs every simulation of its requests (the echoes, and the T1+Δ / T2+Δ copies for
//    the derivatives; with Δ = 0 one tangent pass per request gives exact derivatives instead) as
//    one SimulationBatch — persistent work-queue kernels and batched signal kernels — then per
//    request the derivative differences, the residual and Jᴴ·r;
//  * residency: sequences (with their device tables), trajectories and coil maps are device
//    objects the client keeps and reuses across requests; echoes and derivatives are kept in
//    an LRU cache by the request's echo_key, within its own byte budget;
//  * every kernel of a request is the one its one-request operation uses, on the same inputs,
//    so results are bit-identical alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <thread>
#include <unordered_map>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {
namespace kernels {
__global__ void add_difference_kernel(const float* __restrict__ src, float* __restrict__ dst, int64_t nvoxels,
                                      int field, float delta);
__global__ void finite_difference_kernel(const float2* __restrict__ e0, float2* __restrict__ e1, int64_t n,
                                         float inv_delta);
}  // namespace kernels

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

int readouts_of(const std::variant<FISPSequence, pSSFPSequence>& seq) {
    if (const auto* f = std::get_if<FISPSequence>(&seq)) return int(f->RF_train.size()) * f->undersampling_factor;
    return int(std::get<pSSFPSequence>(seq).RF_train.size());
}

const Trajectory& trajectory_of(const ServeRequest& r) {
    if (const auto* c = std::get_if<CartesianTrajectory>(&r.trajectory)) return *c;
    return std::get<SpiralTrajectory>(r.trajectory);
}

}  // namespace

struct ServeEngine::Impl {
    struct Ticket {
        ServeRequest request;
        size_t footprint = 0;      // working set while its batch runs
        size_t result_bytes = 0;   // residual + gradient, held until release
        Clock::time_point submitted, admitted, finished;
        bool done = false;
        bool failed = false;
        std::string error;
        ServeResult result;
    };
    struct CacheEntry {
        Array<cfloat, 2> echos, dT1, dT2;
        size_t bytes = 0;
        int users = 0;  // running batches reading it
        std::list<uint64_t>::iterator lru;
    };
    struct Running {
        std::vector<uint64_t> ids;
        std::unique_ptr<SimulationBatch> batch;
        std::vector<Array<float, 2>> perturbed;
        std::vector<Array<cfloat, 2>> echos, dT1, dT2;  // per request (views of batch or cache arrays)
        std::vector<Array<cfloat, 3>> signals, residuals;
        std::vector<Array<cfloat, 2>> gradients;
        std::vector<uint64_t> cache_reads;   // keys read from the cache
        std::vector<int> fresh;              // requests whose echoes were simulated here
        Array<float> objectives, partials;
        std::vector<int> partial_offset;
        cudaEvent_t done = nullptr;
        size_t footprint = 0;
        int id = 0;
    };
    struct Slot {
        cudaStream_t stream = nullptr;
        unsigned int* status = nullptr;  // this slot's device status word: its kernels' errors only
        std::unique_ptr<Running> running;
    };

    CompasContext ctx;
    ServeOptions opt;
    mutable std::mutex mu;
    std::condition_variable wake, finished;
    std::thread worker;
    bool stopping = false;
    uint64_t next_ticket = 1;
    std::map<uint64_t, std::shared_ptr<Ticket>> tickets;
    std::deque<uint64_t> pending;
    std::vector<Slot> slots;
    size_t used = 0;        // admitted working sets + unreleased results + cache
    size_t cache_used = 0;
    std::unordered_map<uint64_t, CacheEntry> cache;
    std::list<uint64_t> cache_lru;  // front = most recent
    int batches = 0;
    ServeStats st;
    std::vector<double> latencies;

    explicit Impl(const CompasContext& c, ServeOptions o) : ctx(c), opt(o) {}
    Impl(const Impl&) = delete;
    Impl& operator=(const Impl&) = delete;
    // the last engine handle is gone: finish the admitted and queued requests, stop the worker
    ~Impl() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
        }
        wake.notify_all();
        if (worker.joinable()) worker.join();
        tickets.clear();
        cache.clear();
        for (auto& s : slots) {
            if (s.stream) {
                cudaStreamSynchronize(s.stream);
                cudaStreamDestroy(s.stream);
            }
            if (s.status) cudaFree(s.status);
        }
    }

    size_t estimate(const ServeRequest& r) const;
    void loop();
    void launch(Slot& slot, std::vector<uint64_t> ids);
    void finalize(Slot& slot, bool ok, const std::string& error);
    void evict_for(size_t need);
    int running_batches() const {
        int n = 0;
        for (const auto& s : slots) n += s.running ? 1 : 0;
        return n;
    }
};

size_t ServeEngine::Impl::estimate(const ServeRequest& r) const {
    const int64_t V = r.parameters.nvoxels;
    const Trajectory& t = trajectory_of(r);
    const int64_t R = t.nreadouts, S = t.samples_per_readout, C = r.coil_sensitivities.size(0);
    const bool cart = std::holds_alternative<CartesianTrajectory>(r.trajectory);
    const int64_t echo = 8 * R * V, sig = 8 * C * R * S;
    int64_t bytes = echo * 3 + (opt.delta != 0.0f ? 2 * 36 * V : 0);  // echoes, derivative echoes, T1/T2+Δ copies
    bytes += 2 * sig;                                                  // signal, residual
    bytes += 40 * V + 8 * C * V;                                       // per-voxel tables, coil·w
    if (cart && signal_precision(opt.method) == Precision::SplitBF16) {
        const TcPlan p = tc_plan(ctx.device(), int(V), int(R), int(S), int(C), false);
        if (p.splits > 1) bytes += int64_t(p.splits) * sig;            // split-K partials of the signal
        bytes += tc_tables(int(V), int(R), int(S), int(C), false).bytes;  // E_k tables and packed A
    }
    bytes += 32 * V * 17;                                              // gradient and its split partials
    return size_t(bytes + bytes / 16 + (1 << 20));
}

void ServeEngine::Impl::evict_for(size_t need) {
    // drop least recently used cache entries nobody reads until `need` more bytes fit
    auto it = cache_lru.end();
    while (used + need > opt.memory_budget_bytes && it != cache_lru.begin()) {
        --it;
        auto e = cache.find(*it);
        if (e == cache.end() || e->second.users > 0) continue;
        used -= e->second.bytes;
        cache_used -= e->second.bytes;
        auto victim = it;
        it = std::next(it);
        cache.erase(e);
        cache_lru.erase(victim);
    }
}

void ServeEngine::Impl::launch(Slot& slot, std::vector<uint64_t> ids) {
    const int dev = ctx.device();
    const CompasContext sctx(dev, slot.stream, slot.status);
    auto run = std::make_unique<Running>();
    run->ids = ids;
    run->id = batches++;
    const size_t n = ids.size();
    run->echos.resize(n);
    run->dT1.resize(n);
    run->dT2.resize(n);
    run->signals.resize(n);
    run->residuals.resize(n);
    run->gradients.resize(n);
    std::vector<std::shared_ptr<Ticket>> ts;
    for (auto id : ids) ts.push_back(tickets.at(id));
    // sequence tables are built (once per sequence) on the device stream, which outlives the
    // slot streams, and are complete before any slot reads them
    for (const auto& t : ts) {
        const ServeRequest& r = t->request;
        if (const auto* f = std::get_if<FISPSequence>(&r.sequence)) (void)fisp_excite_table(ctx, *f);
        else (void)pssfp_args(ctx, r.parameters, 0, 0, std::get<pSSFPSequence>(r.sequence), nullptr, 0);
    }
    COMPAS_CUDA_CHECK(cudaStreamSynchronize(ctx.stream()));

    // simulation jobs: the echoes and, for gradients, the T1+Δ / T2+Δ echoes of every request
    // whose echoes are not resident
    std::vector<SimulationJob> jobs;
    std::vector<int> main_job(n, -1), d1_job(n, -1), d2_job(n, -1);
    DeviceGuard guard(dev);
    for (size_t i = 0; i < n; i++) {
        const ServeRequest& r = ts[i]->request;
        if (r.echo_key != 0) {
            auto e = cache.find(r.echo_key);
            if (e != cache.end()) {
                e->second.users++;
                run->cache_reads.push_back(r.echo_key);
                cache_lru.splice(cache_lru.begin(), cache_lru, e->second.lru);
                run->echos[i] = e->second.echos;
                run->dT1[i] = e->second.dT1;
                run->dT2[i] = e->second.dT2;
                ts[i]->result.echo_cache_hit = true;
                continue;
            }
        }
        run->fresh.push_back(int(i));
        SimulationJob job;
        job.parameters = r.parameters;
        job.sequence = r.sequence;
        if (const auto* c = std::get_if<CartesianTrajectory>(&r.trajectory)) job.trajectory = *c;
        else job.trajectory = std::get<SpiralTrajectory>(r.trajectory);
        job.coil_sensitivities = r.coil_sensitivities;
        job.tangents = opt.delta == 0.0f;  // exact derivatives from the simulation pass itself
        main_job[i] = int(jobs.size());
        jobs.push_back(job);
        if (!job.tangents) {  // derivative simulations at T1 + Δ and T2 + Δ
            const int V = r.parameters.nvoxels;
            for (int field = 0; field < 2; field++) {
                Array<float, 2> p({TissueParameterField::NUM_FIELDS, V}, dev, slot.stream);
                if (V > 0) {
                    kernels::add_difference_kernel<<<div_ceil(V, 256), 256, 0, slot.stream>>>(
                        r.parameters.data.data(), p.data(), V, field, opt.delta);
                    check_launch("add_difference_kernel");
                }
                SimulationJob d;
                d.parameters = TissueParameters(p, r.parameters.has_z, r.parameters.has_b0, r.parameters.has_b1);
                d.sequence = r.sequence;
                (field == 0 ? d1_job : d2_job)[i] = int(jobs.size());
                jobs.push_back(d);
                run->perturbed.push_back(p);
            }
        }
    }
    if (!jobs.empty()) {
        run->batch = std::make_unique<SimulationBatch>(sctx, jobs, opt.method);
        run->batch->run();
    }
    for (const auto& t : ts)
        if (t->request.inject_wait_timeout) {
            launch_wait_probe(sctx, 2000000);  // ~1 ms, then STATUS_WAIT_TIMEOUT in this slot's word
            break;
        }

    // per request: derivative differences, signal of resident echoes, residual, gradient
    run->objectives = Array<float>({int64_t(std::max<size_t>(n, 1))}, dev, slot.stream);
    int64_t np_total = 0;
    for (size_t i = 0; i < n; i++) {
        run->partial_offset.push_back(int(np_total));
        np_total += residual_partial_count(ts[i]->request.data.numel());
    }
    run->partials = Array<float>({std::max<int64_t>(np_total, 1)}, dev, slot.stream);
    const Precision prec = signal_precision(opt.method);
    for (size_t i = 0; i < n; i++) {
        const ServeRequest& r = ts[i]->request;
        const int V = r.parameters.nvoxels;
        const int C = int(r.coil_sensitivities.size(0));
        const float* pd = r.parameters.data.data();
        const int64_t ps = r.parameters.data.size(1);
        if (main_job[i] >= 0) {
            run->echos[i] = run->batch->echos(main_job[i]);
            run->signals[i] = run->batch->signal(main_job[i]);
            if (opt.delta == 0.0f) {
                run->dT1[i] = run->batch->derivative(main_job[i], 0);
                run->dT2[i] = run->batch->derivative(main_job[i], 1);
            } else if (d1_job[i] >= 0) {
                run->dT1[i] = run->batch->echos(d1_job[i]);
                run->dT2[i] = run->batch->echos(d2_job[i]);
                for (Array<cfloat, 2>* d : {&run->dT1[i], &run->dT2[i]}) {
                    const int64_t ne = d->numel();
                    if (ne == 0) continue;
                    kernels::finite_difference_kernel<<<int(std::min<int64_t>((ne + 255) / 256, 148 * 16)), 256, 0,
                                                        slot.stream>>>(
                        reinterpret_cast<const float2*>(run->echos[i].data()), reinterpret_cast<float2*>(d->data()),
                        ne, 1.0f / opt.delta);
                    check_launch("finite_difference_kernel");
                }
            }
        } else {
            run->signals[i] = magnetization_to_signal(sctx, run->echos[i], r.parameters, trajectory_of(r),
                                                      r.coil_sensitivities, opt.method);
        }
        const int64_t ns = r.data.numel();
        run->residuals[i] = Array<cfloat, 3>(r.data.sizes(), dev, slot.stream);
        const int np = residual_partial_count(ns);
        launch_residual(sctx, r.data.data(), run->signals[i].data(), ns, run->residuals[i].data(),
                        run->partials.data() + run->partial_offset[i], np, run->objectives.data() + i);
        run->gradients[i] = Array<cfloat, 2>({4, V}, dev, slot.stream);
        if (const auto* cart = std::get_if<CartesianTrajectory>(&r.trajectory)) {
            launch_jacobian_hermitian(sctx, pd, ps, V, run->echos[i].data(), run->dT1[i].data(), run->dT2[i].data(),
                                      r.coil_sensitivities.data(), C, run->residuals[i].data(), cartesian_geom(*cart),
                                      run->gradients[i].data(), prec);
        } else {
            const auto& sp = std::get<SpiralTrajectory>(r.trajectory);
            launch_jacobian_hermitian_spiral(sctx, pd, ps, V, run->echos[i].data(), run->dT1[i].data(),
                                             run->dT2[i].data(), r.coil_sensitivities.data(), C,
                                             run->residuals[i].data(), sp.nreadouts, sp.samples_per_readout,
                                             sp.delta_t, sp.k_start.data(), sp.delta_k.data(),
                                             run->gradients[i].data(), prec);
        }
    }
    COMPAS_CUDA_CHECK(cudaEventCreateWithFlags(&run->done, cudaEventDisableTiming));
    COMPAS_CUDA_CHECK(cudaEventRecord(run->done, slot.stream));
    for (size_t i = 0; i < n; i++) ts[i]->result.batch = run->id;
    slot.running = std::move(run);
}

void ServeEngine::Impl::finalize(Slot& slot, bool ok, const std::string& error) {
    Running& run = *slot.running;
    const auto now = Clock::now();
    std::vector<float> obj(run.ids.size(), 0.0f);
    std::string message = error;
    if (ok && !run.ids.empty()) {
        // the batch is complete and nothing follows it on the slot stream: these copies return at once
        unsigned int status = 0;
        unsigned int* word = slot.status;  // errors of this batch's kernels, and of no other batch
        cudaError_t e = cudaMemcpyAsync(obj.data(), run.objectives.data(), obj.size() * sizeof(float),
                                        cudaMemcpyDeviceToHost, slot.stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&status, word, sizeof(status), cudaMemcpyDeviceToHost, slot.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(slot.stream);
        if (e != cudaSuccess) {
            ok = false;
            (void)cudaGetLastError();
        } else if (status != 0) {
            ok = false;
            message = std::string("a kernel of the request's batch reported an error: ") + status_message(status);
            cudaMemsetAsync(word, 0, sizeof(unsigned int), slot.stream);
        }
    }
    for (size_t i = 0; i < run.ids.size(); i++) {
        auto& t = *tickets.at(run.ids[i]);
        t.finished = now;
        t.done = true;
        used -= t.footprint;
        if (!ok) {
            t.failed = true;
            t.error = message.empty() ? "a kernel of the request's batch reported an error" : message;
            st.failed++;
            continue;
        }
        // results outlive this slot's stream order: later reads and releases use the device stream
        ServeResult& res = t.result;
        res.residual = run.residuals[i];
        res.gradient = run.gradients[i];
        res.residual.set_stream(ctx.stream());
        res.gradient.set_stream(ctx.stream());
        res.objective = obj[i];
        res.queued_ms = ms_between(t.submitted, t.admitted);
        res.device_ms = ms_between(t.admitted, t.finished);
        res.latency_ms = ms_between(t.submitted, t.finished);
        t.result_bytes = size_t(res.residual.nbytes() + res.gradient.nbytes());
        used += t.result_bytes;
        latencies.push_back(res.latency_ms);
        st.completed++;
        if (res.echo_cache_hit) st.echo_cache_hits++;
    }
    for (auto key : run.cache_reads) {
        auto e = cache.find(key);
        if (e != cache.end()) e->second.users--;
    }
    // keep the freshly simulated echoes of keyed requests resident
    if (ok) {
        for (int i : run.fresh) {
            const ServeRequest& r = tickets.at(run.ids[size_t(i)])->request;
            if (r.echo_key == 0 || cache.count(r.echo_key)) continue;
            CacheEntry entry;
            entry.echos = run.echos[size_t(i)];
            entry.dT1 = run.dT1[size_t(i)];
            entry.dT2 = run.dT2[size_t(i)];
            entry.bytes = entry.echos.nbytes() + entry.dT1.nbytes() + entry.dT2.nbytes();
            if (entry.bytes > opt.echo_cache_bytes) continue;
            while (cache_used + entry.bytes > opt.echo_cache_bytes && !cache_lru.empty()) {
                auto victim = std::prev(cache_lru.end());
                auto ve = cache.find(*victim);
                if (ve->second.users > 0) break;
                used -= ve->second.bytes;
                cache_used -= ve->second.bytes;
                cache.erase(ve);
                cache_lru.erase(victim);
            }
            if (cache_used + entry.bytes > opt.echo_cache_bytes) continue;
            for (auto* a : {&entry.echos, &entry.dT1, &entry.dT2}) a->set_stream(ctx.stream());
            cache_lru.push_front(r.echo_key);
            entry.lru = cache_lru.begin();
            used += entry.bytes;
            cache_used += entry.bytes;
            cache.emplace(r.echo_key, std::move(entry));
        }
    }
    st.batches++;
    st.peak_bytes = std::max(st.peak_bytes, used);
    cudaEventDestroy(run.done);
    slot.running.reset();  // releases the batch's working set, stream-ordered on the slot stream
    finished.notify_all();
}

void ServeEngine::Impl::loop() {
    cudaSetDevice(ctx.device());
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        bool progressed = false;
        // retire finished batches
        for (auto& slot : slots) {
            if (!slot.running) continue;
            const cudaError_t q = cudaEventQuery(slot.running->done);
            if (q == cudaErrorNotReady) continue;
            std::string err;
            if (q != cudaSuccess) {
                err = cudaGetErrorString(q);
                (void)cudaGetLastError();
            }
            finalize(slot, q == cudaSuccess, err);
            progressed = true;
        }
        // admit the oldest requests into free slots
        for (auto& slot : slots) {
            if (slot.running || pending.empty()) continue;
            std::vector<uint64_t> ids;
            size_t need = 0;
            while (!pending.empty() && int(ids.size()) < opt.max_batch_requests) {
                auto& t = *tickets.at(pending.front());
                if (used + need + t.footprint > opt.memory_budget_bytes) evict_for(need + t.footprint);
                if (used + need + t.footprint > opt.memory_budget_bytes) break;
                need += t.footprint;
                ids.push_back(pending.front());
                pending.pop_front();
            }
            if (ids.empty()) {
                // nothing fits: fail a request larger than the whole budget once nothing runs
                auto& t = *tickets.at(pending.front());
                if (running_batches() == 0 && t.footprint > opt.memory_budget_bytes - std::min(used, opt.memory_budget_bytes)) {
                    t.done = t.failed = true;
                    t.error = "request needs more device memory than the serving budget";
                    t.finished = Clock::now();
                    st.failed++;
                    pending.pop_front();
                    finished.notify_all();
                    progressed = true;
                }
                break;
            }
            const auto now = Clock::now();
            for (auto id : ids) tickets.at(id)->admitted = now;
            used += need;
            st.peak_bytes = std::max(st.peak_bytes, used);
            try {
                launch(slot, ids);
                slot.running->footprint = need;
            } catch (const std::exception& e) {
                for (auto id : ids) {
                    auto& t = *tickets.at(id);
                    t.done = t.failed = true;
                    t.error = e.what();
                    t.finished = Clock::now();
                    used -= t.footprint;
                    st.failed++;
                }
                if (slot.running) {
                    if (slot.running->done) cudaEventDestroy(slot.running->done);
                    slot.running.reset();
                }
                cudaStreamSynchronize(slot.stream);
                (void)cudaGetLastError();
                finished.notify_all();
            }
            st.max_concurrent_batches = std::max(st.max_concurrent_batches, running_batches());
            progressed = true;
        }
        if (stopping && pending.empty() && running_batches() == 0) break;
        if (progressed) continue;
        if (running_batches() > 0) wake.wait_for(lk, std::chrono::microseconds(50));
        else wake.wait(lk);
    }
}

ServeEngine::ServeEngine(const CompasContext& ctx, ServeOptions options) :
    m_impl(std::make_shared<Impl>(ctx, options)) {
    Impl& im = *m_impl;
    if (options.max_inflight_batches < 1 || options.max_batch_requests < 1)
        COMPAS_ERROR("serving needs at least one batch slot and one request per batch");
    DeviceGuard guard(ctx.device());
    im.slots.resize(size_t(options.max_inflight_batches));
    for (auto& s : im.slots) {
        COMPAS_CUDA_CHECK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        COMPAS_CUDA_CHECK(cudaMalloc(&s.status, sizeof(unsigned int)));
        COMPAS_CUDA_CHECK(cudaMemset(s.status, 0, sizeof(unsigned int)));
    }
    im.worker = std::thread([&im] { im.loop(); });
}

ServeEngine::~ServeEngine() = default;

uint64_t ServeEngine::submit(ServeRequest request) {
    Impl& im = *m_impl;
    const Trajectory& t = trajectory_of(request);
    const int V = request.parameters.nvoxels;
    if (readouts_of(request.sequence) != t.nreadouts) COMPAS_ERROR("trajectory readouts do not match the sequence's echoes");
    COMPAS_CHECK(request.coil_sensitivities.size(1) == V);
    const int64_t C = request.coil_sensitivities.size(0);
    if (request.data.size(0) != C || request.data.size(1) != t.nreadouts || request.data.size(2) != t.samples_per_readout)
        COMPAS_ERROR("data must be [ncoils][nreadouts][samples_per_readout]");
    auto ticket = std::make_shared<Impl::Ticket>();
    ticket->footprint = im.estimate(request);
    ticket->request = std::move(request);
    ticket->submitted = Clock::now();
    uint64_t id;
    {
        std::lock_guard<std::mutex> lk(im.mu);
        if (im.stopping) COMPAS_ERROR("serving engine is shutting down");
        id = im.next_ticket++;
        im.tickets.emplace(id, std::move(ticket));
        im.pending.push_back(id);
    }
    im.wake.notify_all();
    return id;
}

bool ServeEngine::ready(uint64_t id) const {
    std::lock_guard<std::mutex> lk(m_impl->mu);
    auto it = m_impl->tickets.find(id);
    if (it == m_impl->tickets.end()) COMPAS_ERROR("unknown ticket");
    return it->second->done;
}

ServeResult ServeEngine::wait(uint64_t id) {
    Impl& im = *m_impl;
    std::unique_lock<std::mutex> lk(im.mu);
    auto it = im.tickets.find(id);
    if (it == im.tickets.end()) COMPAS_ERROR("unknown ticket");
    auto t = it->second;
    im.finished.wait(lk, [&] { return t->done; });
    if (t->failed) throw CompasException("request failed: " + t->error);
    return t->result;
}

void ServeEngine::release(uint64_t id) {
    Impl& im = *m_impl;
    std::lock_guard<std::mutex> lk(im.mu);
    auto it = im.tickets.find(id);
    if (it == im.tickets.end()) return;
    if (!it->second->done) COMPAS_ERROR("cannot release a request that has not completed");
    im.used -= it->second->result_bytes;
    im.tickets.erase(it);
    im.wake.notify_all();
}

void ServeEngine::drain() {
    Impl& im = *m_impl;
    std::unique_lock<std::mutex> lk(im.mu);
    im.finished.wait(lk, [&] {
        if (!im.pending.empty() || im.running_batches() > 0) return false;
        for (const auto& kv : im.tickets)
            if (!kv.second->done) return false;
        return true;
    });
}

ServeStats ServeEngine::stats() const {
    const Impl& im = *m_impl;
    std::lock_guard<std::mutex> lk(im.mu);
    ServeStats s = im.st;
    if (!im.latencies.empty()) {
        std::vector<double> v = im.latencies;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) {
            const double pos = q * double(v.size() - 1);
            const size_t lo = size_t(pos);
            const size_t hi = std::min(v.size() - 1, lo + 1);
            return v[lo] + (v[hi] - v[lo]) * (pos - double(lo));
        };
        s.p50_ms = pct(0.50);
        s.p99_ms = pct(0.99);
        s.max_ms = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        s.mean_ms = sum / double(v.size());
    }
    return s;
}

void ServeEngine::reset_stats() {
    Impl& im = *m_impl;
    std::lock_guard<std::mutex> lk(im.mu);
    im.st = ServeStats {};
    im.latencies.clear();
}

}  // namespace compas
