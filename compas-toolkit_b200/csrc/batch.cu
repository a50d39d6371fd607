// batch.cu — many independent simulate → signal jobs in a handful of launches.
//
// The reference runs one operation per call (src/simulate/fisp.cu:7-140, pssfp.cu:7-91,
// src/trajectories/signal.cu:13-356); a batch of small jobs then leaves most of the 148 SMs
// idle and pays one launch chain per job. Here a batch is planned once:
//
//  * simulation: jobs are grouped by kernel layout — the layout each job would get alone, so
//    the per-job bits do not depend on the batch (jobs with tangents in groups of their own, on
//    the tangent kernels). Every group is ONE persistent work-queue
//    launch: CTAs (as many as fit on the GPU) take (job, voxel tile) items through an atomic
//    counter; items are ordered longest job first so the last wave is short. FISP groups run on
//    the context's stream, pSSFP groups on a second stream, so the two families overlap (a
//    pSSFP CTA fits in the registers a FISP CTA leaves free on an SM);
//  * signal: after its family's simulation, the Cartesian signals of that family run as ONE
//    batched split-BF16 tensor-core launch (plus one batched prep and one batched split-K
//    sum), the spiral signals on the split-BF16 tensor-core kernel one launch per job (each job's
//    readouts × sample tiles fill the GPU), or with the FP32 method as one batched launch per coil
//    grouping. A flattened CTA index is
//    mapped to (job, tile) by a binary search over per-job CTA offsets; jobs are ordered by
//    decreasing work per CTA. The voxel split of each job is the one it gets alone;
//  * all device memory (echoes, signals, argument tables, split-K partials, per-voxel tables)
//    is allocated at construction, so run() only enqueues kernels and can be captured into a
//    CUDA graph.
#include <algorithm>
#include <numeric>
#include <tuple>

#include "common.cuh"
#include "compas/compas.h"
#include "job_args.cuh"
#include "kernels.h"

namespace compas {

namespace {

template<typename T>
Array<unsigned char> upload_table(const CompasContext& ctx, const std::vector<T>& v) {
    Array<unsigned char> out({int64_t(v.size() * sizeof(T))}, ctx.device(), ctx.stream());
    if (!v.empty()) {
        DeviceGuard guard(ctx.device());
        COMPAS_CUDA_CHECK(cudaMemcpyAsync(out.data(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                                          ctx.stream()));
    }
    return out;
}

template<typename T>
const T* as(const Array<unsigned char>& a) {
    return reinterpret_cast<const T*>(a.data());
}

// prefix offsets of per-job block counts: offsets[j] = Σ_{i<j} counts[i], plus the total
std::vector<int> prefix(const std::vector<int64_t>& counts, int64_t* total) {
    std::vector<int> off(counts.size() + 1, 0);
    int64_t acc = 0;
    for (size_t i = 0; i < counts.size(); i++) {
        off[i] = int(acc);
        acc += counts[i];
        if (acc > int64_t(INT32_MAX)) COMPAS_ERROR("batch too large for one launch");
    }
    off[counts.size()] = int(acc);
    *total = acc;
    return off;
}

}  // namespace

struct SimulationBatch::Impl {
    explicit Impl(const CompasContext& c) : ctx(c) {}
    Impl(const Impl&) = delete;
    Impl& operator=(const Impl&) = delete;

    CompasContext ctx;
    std::vector<SimulationJob> jobs;
    Precision prec = Precision::SplitBF16;
    std::vector<Array<cfloat, 2>> echos;
    std::vector<Array<cfloat, 2>> dT1, dT2;  // tangent jobs only (empty otherwise)
    std::vector<Array<cfloat, 3>> signals;
    Array<int> heads;  // one work-queue counter per simulation group
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;

    struct SimGroup {
        bool fisp;
        bool tangent;              // value and T1/T2 tangents (tangent layouts for FISP)
        int config, warps, cover;  // layout, warps (FISP), max_state / nz
        bool real = false;         // every job's RF is real (FISP: RF and slice-profile phases)
        Array<unsigned char> args;
        Array<unsigned char> items;
        int nitems = 0;
        int head = 0;
    };
    struct TcGroup {
        Array<unsigned char> args, prep_offsets, pack_offsets, cta_offsets, sums, sum_offsets;
        int njobs = 0, prep_blocks = 0, pack_blocks = 0, ctas = 0, nsums = 0, sum_blocks = 0;
        std::vector<Array<unsigned char>> scratch;  // per-voxel tables, packed A and partials
    };
    struct SpiralGroup {
        int coil_group;
        Array<unsigned char> args, cta_offsets;
        int njobs = 0, ctas = 0;
    };
    struct Family {
        std::vector<SimGroup> sims;
        TcGroup tc;
        std::vector<SpiralGroup> spirals;
        std::vector<int> simt_cartesian;  // jobs whose Cartesian signal runs on the FP32 kernels
        std::vector<int> tc_spiral;       // spiral jobs on the split-BF16 tensor-core kernel
        std::vector<int> empty_signals;   // jobs with no voxels: their signal is zero
    };
    Family families[2];  // 0: FISP (context stream), 1: pSSFP (side stream)

    ~Impl() {
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
    }

    void plan_simulation(Family& fam, bool fisp, const std::vector<int>& members);
    void plan_signal(Family& fam, const std::vector<int>& members);
    void enqueue(const Family& fam, cudaStream_t stream, int* head_base) const;
};

void SimulationBatch::Impl::plan_simulation(Family& fam, bool fisp, const std::vector<int>& members) {
    // group by the launch the job would get alone
    struct Key {
        int tangent, config, warps, cover, real;
        bool operator<(const Key& o) const {
            return std::tie(tangent, config, warps, cover, real) < std::tie(o.tangent, o.config, o.warps, o.cover, o.real);
        }
    };
    std::vector<std::pair<Key, int>> keyed;
    for (int j : members) {
        const auto& job = jobs[size_t(j)];
        if (job.parameters.nvoxels == 0) continue;
        const int tan = job.tangents ? 1 : 0;
        if (fisp) {
            const auto& seq = std::get<FISPSequence>(job.sequence);
            const int P = int(seq.sliceprofiles.size(0));
            const int V = job.parameters.nvoxels;
            FispLaunch D;
            if (tan) {
                D = tuned_fisp_tangent_launch(seq.max_state, V, P);
            } else {
                const FispLaunch L = tuned_fisp_launch(seq.max_state, V, P);
                D = L.config < 0 ? fisp_default_launch(seq.max_state, V, P) : L;
            }
            // jobs with real phases form their own groups, which a packed layout runs in its real-phase form
            const bool packed = tan ? fisp_tangent_config_packed(D.config) : fisp_config_packed(D.config);
            const int real = packed && fisp_sequence_real_phases(ctx, seq) ? 1 : 0;
            keyed.push_back({Key {tan, D.config, std::max(1, std::min(D.warps, 8)), seq.max_state, real}, j});
        } else {
            const auto& seq = std::get<pSSFPSequence>(job.sequence);
            const int nz = int(seq.z.size());
            const PssfpLaunch L = tuned_pssfp_launch(nz, job.parameters.nvoxels);
            const PssfpLaunch D = L.config < 0 ? pssfp_default_launch(nz, job.parameters.nvoxels) : L;
            // jobs with real RF form their own groups, which a packed layout runs in its real-RF form
            const int real = pssfp_config_packed(D.config) && pssfp_sequence_real_rf(ctx, seq) ? 1 : 0;
            keyed.push_back({Key {tan, D.config, 0, nz, real}, j});
        }
    }
    std::stable_sort(keyed.begin(), keyed.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t i = 0; i < keyed.size();) {
        size_t e = i;
        while (e < keyed.size() && !(keyed[i].first < keyed[e].first) && !(keyed[e].first < keyed[i].first)) e++;
        const Key key = keyed[i].first;
        // per job: argument block and tile count; order longest (per tile) first
        std::vector<int> js;
        for (size_t q = i; q < e; q++) js.push_back(keyed[q].second);
        auto cost = [&](int j) -> double {
            const auto& job = jobs[size_t(j)];
            if (fisp) {
                const auto& seq = std::get<FISPSequence>(job.sequence);
                return double(seq.RF_train.size()) * double(seq.sliceprofiles.size(0)) * seq.repetitions;
            }
            const auto& seq = std::get<pSSFPSequence>(job.sequence);
            return double(seq.RF_train.size()) * double(std::max<int64_t>(1, seq.gamma_dt_RF.size()));
        };
        std::stable_sort(js.begin(), js.end(), [&](int a, int b) { return cost(a) > cost(b); });
        SimGroup g;
        g.fisp = fisp;
        g.tangent = key.tangent != 0;
        g.config = key.config;
        g.warps = key.warps;
        g.cover = key.cover;
        g.real = key.real != 0;
        std::vector<int> items;
        if (fisp) {
            std::vector<kernels::FispArgs> args;
            const FispLaunch L {key.config, key.warps};
            const int vb = g.tangent ? fisp_tangent_tile_voxels(L) : fisp_tile_voxels(L);
            for (size_t q = 0; q < js.size(); q++) {
                const auto& job = jobs[size_t(js[q])];
                const auto& seq = std::get<FISPSequence>(job.sequence);
                const int V = job.parameters.nvoxels;
                args.push_back(fisp_args(ctx, job.parameters, 0, V, seq, echos[size_t(js[q])].data(), V));
                if (g.tangent) {
                    args.back().dT1 = reinterpret_cast<float2*>(dT1[size_t(js[q])].data());
                    args.back().dT2 = reinterpret_cast<float2*>(dT2[size_t(js[q])].data());
                }
                // items of fisp_queue_tiles_per_item tiles: the queue kernels run an item's
                // (tile, position) pairs in rounds of the CTA's warps
                const int tpi = kernels::fisp_queue_tiles_per_item(args.back().P, g.warps);
                for (int t = 0; t < div_ceil(V, vb); t += tpi) {
                    items.push_back(int(q));
                    items.push_back(t);
                }
            }
            g.args = upload_table(ctx, args);
        } else {
            std::vector<kernels::PssfpArgs> args;
            const int vb = pssfp_tile_voxels(PssfpLaunch {key.config});
            for (size_t q = 0; q < js.size(); q++) {
                const auto& job = jobs[size_t(js[q])];
                const auto& seq = std::get<pSSFPSequence>(job.sequence);
                const int V = job.parameters.nvoxels;
                args.push_back(pssfp_args(ctx, job.parameters, 0, V, seq, echos[size_t(js[q])].data(), V));
                if (g.tangent) {
                    args.back().dT1 = reinterpret_cast<float2*>(dT1[size_t(js[q])].data());
                    args.back().dT2 = reinterpret_cast<float2*>(dT2[size_t(js[q])].data());
                }
                for (int t = 0; t < div_ceil(V, vb); t++) {
                    items.push_back(int(q));
                    items.push_back(t);
                }
            }
            g.args = upload_table(ctx, args);
        }
        g.nitems = int(items.size() / 2);
        g.items = upload_table(ctx, items);
        fam.sims.push_back(std::move(g));
        i = e;
    }
}

void SimulationBatch::Impl::plan_signal(Family& fam, const std::vector<int>& members) {
    const int dev = ctx.device();
    std::vector<int> tc_jobs;
    std::vector<int> spiral_by_group[4];  // coil groupings 1, 2, 4, 8
    for (int j : members) {
        const auto& job = jobs[size_t(j)];
        if (std::holds_alternative<std::monostate>(job.trajectory)) continue;
        const int V = job.parameters.nvoxels;
        const int C = int(job.coil_sensitivities.size(0));
        if (C == 0 || signals[size_t(j)].size() == 0) continue;
        if (V == 0) {
            fam.empty_signals.push_back(j);
            continue;
        }
        if (std::holds_alternative<CartesianTrajectory>(job.trajectory)) {
            if (prec == Precision::SplitBF16 && tensor_cores_available(dev)) tc_jobs.push_back(j);
            else fam.simt_cartesian.push_back(j);
        } else if (prec == Precision::SplitBF16 && tensor_cores_available(dev)) {
            fam.tc_spiral.push_back(j);  // one tensor-core launch per job (each fills the GPU alone)
        } else {
            const int cg = spiral_coil_group(C);
            spiral_by_group[cg == 1 ? 0 : cg == 2 ? 1 : cg == 4 ? 2 : 3].push_back(j);
        }
    }

    // ---- Cartesian on tensor cores
    if (!tc_jobs.empty()) {
        struct Entry {
            int job;
            TcPlan plan;
        };
        std::vector<Entry> es;
        for (int j : tc_jobs) {
            const auto& job = jobs[size_t(j)];
            const auto& t = std::get<CartesianTrajectory>(job.trajectory);
            es.push_back({j, tc_plan(dev, job.parameters.nvoxels, t.nreadouts, t.samples_per_readout,
                                     int(job.coil_sensitivities.size(0)), false)});
        }
        std::stable_sort(es.begin(), es.end(), [](const Entry& a, const Entry& b) { return a.plan.vchunk > b.plan.vchunk; });
        TcGroup& g = fam.tc;
        std::vector<kernels::TcArgs> args;
        std::vector<int64_t> prep_counts, pack_counts, cta_counts, sum_counts;
        std::vector<kernels::PartialSum> sums;
        for (const auto& e : es) {
            const auto& job = jobs[size_t(e.job)];
            const auto& t = std::get<CartesianTrajectory>(job.trajectory);
            const int V = job.parameters.nvoxels, C = int(job.coil_sensitivities.size(0));
            kernels::TcArgs a = tc_signal_args(job.parameters.data.data(), job.parameters.data.size(1), V,
                                               echos[size_t(e.job)].data(), job.coil_sensitivities.data(), C,
                                               cartesian_geom(t));
            a.vchunk = e.plan.vchunk;
            a.status = ctx.status_word();
            const TcTables tables = tc_tables(V, t.nreadouts, t.samples_per_readout, C, false);
            Array<unsigned char> scratch({tables.bytes}, dev, ctx.stream());
            tc_assign_tables(a, tables, scratch.data());
            const int64_t n = int64_t(C) * t.nreadouts * t.samples_per_readout;
            float2* out = reinterpret_cast<float2*>(signals[size_t(e.job)].data());
            if (e.plan.splits > 1) {
                Array<unsigned char> partials({int64_t(e.plan.splits) * n * int64_t(sizeof(float2))}, dev, ctx.stream());
                a.out = reinterpret_cast<float2*>(partials.data());
                sums.push_back({a.out, out, n, e.plan.splits});
                sum_counts.push_back((n + 255) / 256);
                g.scratch.push_back(std::move(partials));
            } else {
                a.out = out;
            }
            g.scratch.push_back(std::move(scratch));
            args.push_back(a);
            prep_counts.push_back(div_ceil(V, 128));
            pack_counts.push_back(tc_pack_blocks(a.nr, t.nreadouts, a.apack_stages));
            cta_counts.push_back(e.plan.ctas);
        }
        int64_t total = 0;
        g.njobs = int(args.size());
        g.args = upload_table(ctx, args);
        g.prep_offsets = upload_table(ctx, prefix(prep_counts, &total));
        g.prep_blocks = int(total);
        g.pack_offsets = upload_table(ctx, prefix(pack_counts, &total));
        g.pack_blocks = int(total);
        g.cta_offsets = upload_table(ctx, prefix(cta_counts, &total));
        g.ctas = int(total);
        g.nsums = int(sums.size());
        g.sums = upload_table(ctx, sums);
        g.sum_offsets = upload_table(ctx, prefix(sum_counts, &total));
        g.sum_blocks = int(total);
    }

    // ---- spiral, one batched launch per coil grouping
    for (int gi = 0; gi < 4; gi++) {
        const int cg = 1 << gi;
        std::vector<int>& js = spiral_by_group[gi];
        if (js.empty()) continue;
        std::stable_sort(js.begin(), js.end(),
                         [&](int a, int b) { return jobs[size_t(a)].parameters.nvoxels > jobs[size_t(b)].parameters.nvoxels; });
        SpiralGroup g;
        g.coil_group = cg;
        std::vector<kernels::SpiralArgs> args;
        std::vector<int64_t> counts;
        for (int j : js) {
            const auto& job = jobs[size_t(j)];
            const auto& t = std::get<SpiralTrajectory>(job.trajectory);
            kernels::SpiralArgs a {};
            a.params = job.parameters.data.data();
            a.pstride = job.parameters.data.size(1);
            a.nvoxels = job.parameters.nvoxels;
            a.echo = reinterpret_cast<const float2*>(echos[size_t(j)].data());
            a.coils = reinterpret_cast<const float2*>(job.coil_sensitivities.data());
            a.R = t.nreadouts;
            a.S = t.samples_per_readout;
            a.C = int(job.coil_sensitivities.size(0));
            a.dt = t.delta_t;
            a.k_start = reinterpret_cast<const float2*>(t.k_start.data());
            a.delta_k = reinterpret_cast<const float2*>(t.delta_k.data());
            a.signal = reinterpret_cast<float2*>(signals[size_t(j)].data());
            args.push_back(a);
            counts.push_back(spiral_block_count(a.C, a.R, a.S));
        }
        int64_t total = 0;
        g.njobs = int(args.size());
        g.args = upload_table(ctx, args);
        g.cta_offsets = upload_table(ctx, prefix(counts, &total));
        g.ctas = int(total);
        fam.spirals.push_back(std::move(g));
    }
}

void SimulationBatch::Impl::enqueue(const Family& fam, cudaStream_t stream, int* head_base) const {
    const int dev = ctx.device();
    for (const auto& g : fam.sims) {
        if (g.fisp && g.tangent)
            launch_fisp_tangent_queue(stream, dev, FispLaunch {g.config, g.warps}, g.cover,
                                      as<kernels::FispArgs>(g.args), as<int2>(g.items), g.nitems, head_base + g.head,
                                      g.real);
        else if (g.fisp)
            launch_fisp_queue(stream, dev, FispLaunch {g.config, g.warps}, g.cover, as<kernels::FispArgs>(g.args),
                              as<int2>(g.items), g.nitems, head_base + g.head, g.real);
        else if (g.tangent)
            launch_pssfp_tangent_queue(stream, dev, PssfpLaunch {g.config}, g.cover, as<kernels::PssfpArgs>(g.args),
                                       as<int2>(g.items), g.nitems, head_base + g.head, g.real);
        else
            launch_pssfp_queue(stream, dev, PssfpLaunch {g.config}, g.cover, as<kernels::PssfpArgs>(g.args),
                               as<int2>(g.items), g.nitems, head_base + g.head, g.real);
    }
    for (int j : fam.empty_signals)
        COMPAS_CUDA_CHECK(cudaMemsetAsync(signals[size_t(j)].data(), 0, signals[size_t(j)].nbytes(), stream));
    const auto& tc = fam.tc;
    if (tc.njobs > 0) {
        launch_tc_batch(stream, dev, false, as<kernels::TcArgs>(tc.args), tc.njobs, as<int>(tc.prep_offsets),
                        tc.prep_blocks, as<int>(tc.pack_offsets), tc.pack_blocks, as<int>(tc.cta_offsets), tc.ctas);
        launch_sum_partials_batch(stream, dev, as<kernels::PartialSum>(tc.sums), as<int>(tc.sum_offsets), tc.nsums,
                                  tc.sum_blocks);
    }
    for (const auto& g : fam.spirals)
        launch_signal_spiral_batch(stream, dev, g.coil_group, as<kernels::SpiralArgs>(g.args), as<int>(g.cta_offsets),
                                   g.njobs, g.ctas);
    const CompasContext sctx(dev, stream, ctx.status_word());
    for (int j : fam.tc_spiral) {
        const auto& job = jobs[size_t(j)];
        const auto& t = std::get<SpiralTrajectory>(job.trajectory);
        launch_signal_spiral(sctx, job.parameters.data.data(), job.parameters.data.size(1), job.parameters.nvoxels,
                             echos[size_t(j)].data(), job.coil_sensitivities.data(),
                             int(job.coil_sensitivities.size(0)), t.nreadouts, t.samples_per_readout, t.delta_t,
                             t.k_start.data(), t.delta_k.data(), signals[size_t(j)].data(), Precision::SplitBF16);
    }
}

SimulationBatch::SimulationBatch(const CompasContext& ctx, std::vector<SimulationJob> jobs,
                                 SimulateSignalMethod method) :
    m_impl(std::make_shared<Impl>(ctx)) {
    Impl& im = *m_impl;
    im.jobs = std::move(jobs);
    im.prec = signal_precision(method);
    const int dev = ctx.device();
    DeviceGuard guard(dev);
    std::vector<int> members[2];
    for (size_t j = 0; j < im.jobs.size(); j++) {
        const auto& job = im.jobs[j];
        const int V = job.parameters.nvoxels;
        const bool fisp = std::holds_alternative<FISPSequence>(job.sequence);
        int nreadouts = 0;
        if (fisp) {
            const auto& seq = std::get<FISPSequence>(job.sequence);
            COMPAS_CHECK(seq.undersampling_factor >= 1);
            nreadouts = int(seq.RF_train.size()) * seq.undersampling_factor;
        } else {
            nreadouts = int(std::get<pSSFPSequence>(job.sequence).RF_train.size());
        }
        im.echos.emplace_back(std::array<int64_t, 2> {nreadouts, V}, dev, ctx.stream());
        if (job.tangents) {
            im.dT1.emplace_back(std::array<int64_t, 2> {nreadouts, V}, dev, ctx.stream());
            im.dT2.emplace_back(std::array<int64_t, 2> {nreadouts, V}, dev, ctx.stream());
        } else {
            im.dT1.emplace_back();
            im.dT2.emplace_back();
        }
        if (std::holds_alternative<std::monostate>(job.trajectory)) {
            im.signals.emplace_back();
        } else {
            const Trajectory& t = std::holds_alternative<CartesianTrajectory>(job.trajectory)
                                      ? static_cast<const Trajectory&>(std::get<CartesianTrajectory>(job.trajectory))
                                      : static_cast<const Trajectory&>(std::get<SpiralTrajectory>(job.trajectory));
            const int C = int(job.coil_sensitivities.size(0));
            if (t.nreadouts != nreadouts) COMPAS_ERROR("trajectory readouts do not match the sequence's echoes");
            COMPAS_CHECK(job.coil_sensitivities.size(1) == V);
            if (const auto* sp = std::get_if<SpiralTrajectory>(&job.trajectory))
                COMPAS_CHECK(sp->k_start.size() == t.nreadouts && sp->delta_k.size() == t.nreadouts);
            im.signals.emplace_back(std::array<int64_t, 3> {C, t.nreadouts, t.samples_per_readout}, dev, ctx.stream());
        }
        members[fisp ? 0 : 1].push_back(int(j));
    }
    for (int f = 0; f < 2; f++) {
        im.plan_simulation(im.families[f], f == 0, members[f]);
        im.plan_signal(im.families[f], members[f]);
    }
    int nheads = 0;
    for (auto& fam : im.families)
        for (auto& g : fam.sims) g.head = nheads++;
    im.heads = Array<int>({std::max(1, nheads)}, dev, ctx.stream());
    COMPAS_CUDA_CHECK(cudaStreamCreateWithFlags(&im.side, cudaStreamNonBlocking));
    COMPAS_CUDA_CHECK(cudaEventCreateWithFlags(&im.fork, cudaEventDisableTiming));
    COMPAS_CUDA_CHECK(cudaEventCreateWithFlags(&im.join, cudaEventDisableTiming));
    ctx.synchronize();  // argument tables uploaded, sequence tables built
}

void SimulationBatch::run() const {
    const Impl& im = *m_impl;
    const CompasContext& ctx = im.ctx;
    DeviceGuard guard(ctx.device());
    cudaStream_t main = ctx.stream();
    COMPAS_CUDA_CHECK(cudaMemsetAsync(im.heads.data(), 0, im.heads.nbytes(), main));
    COMPAS_CUDA_CHECK(cudaEventRecord(im.fork, main));
    COMPAS_CUDA_CHECK(cudaStreamWaitEvent(im.side, im.fork, 0));
    im.enqueue(im.families[0], main, im.heads.data());
    im.enqueue(im.families[1], im.side, im.heads.data());
    COMPAS_CUDA_CHECK(cudaEventRecord(im.join, im.side));
    COMPAS_CUDA_CHECK(cudaStreamWaitEvent(main, im.join, 0));
    // FP32 Cartesian signals (one launch chain per job, on the context's stream)
    for (const auto& fam : im.families) {
        for (int j : fam.simt_cartesian) {
            const auto& job = im.jobs[size_t(j)];
            const auto& t = std::get<CartesianTrajectory>(job.trajectory);
            launch_signal_cartesian(ctx, job.parameters.data.data(), job.parameters.data.size(1),
                                    job.parameters.nvoxels, im.echos[size_t(j)].data(),
                                    job.coil_sensitivities.data(), int(job.coil_sensitivities.size(0)),
                                    cartesian_geom(t), im.signals[size_t(j)].data(), Precision::FP32);
        }
    }
}

int SimulationBatch::size() const {
    return int(m_impl->jobs.size());
}

const Array<cfloat, 2>& SimulationBatch::echos(int job) const {
    if (job < 0 || job >= size()) COMPAS_ERROR("job index out of range");
    return m_impl->echos[size_t(job)];
}

const Array<cfloat, 3>& SimulationBatch::signal(int job) const {
    if (job < 0 || job >= size()) COMPAS_ERROR("job index out of range");
    return m_impl->signals[size_t(job)];
}

const Array<cfloat, 2>& SimulationBatch::derivative(int job, int field) const {
    if (job < 0 || job >= size()) COMPAS_ERROR("job index out of range");
    if (!m_impl->jobs[size_t(job)].tangents) COMPAS_ERROR("the job was not planned with tangents");
    if (field != 0 && field != 1) COMPAS_ERROR("derivatives are kept for T1 (0) and T2 (1)");
    return field == 0 ? m_impl->dT1[size_t(job)] : m_impl->dT2[size_t(job)];
}

}  // namespace compas
