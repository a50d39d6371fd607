// ref_sim.cpp — golden echoes from the reference's own simulation kernels, run on the CPU.
//
// TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile (target `ref`) into oracle/_ref/ref_sim with
// the reference's include and src trees on the include path (nothing of the reference is copied)
// and the host stand-ins of oracle/refshim (kmm views, CUDA built-ins). Each kernel runs as a
// one-thread launch per voxel:
//  * FISP: kernels::simulate_fisp<max_N, 1, 1> (src/simulate/fisp_kernels.cuh:225-241), one launch
//    per slice position accumulating into the transposed echoes as the host code does
//    (src/simulate/fisp.cu:35-48), then kernels::expand_undersampled_echos (:243-257);
//  * pSSFP: kernels::simulate_pssfp<1> (src/simulate/pssfp_kernels.cuh:111-129), one launch per z
//    position (the batch-of-1 path of src/simulate/pssfp.cu:16-41).
// The EPG operators (src/operators/epg.cuh) and the isochromat operators
// (src/operators/isochromat.cuh) are the reference's; the fast-math intrinsics are exact libm
// calls (oracle/refshim/cuda_host_shim.h). The signal, Jacobian, phase-encoding and residual
// kernels run the same way (one thread per output element or voxel) on seeded Cartesian and spiral
// cases. Prints inputs and outputs as JSON; tests/golden/make_golden.py stores them as
// tests/golden/ref_simulations.json.
#include <cstdio>
#include <random>
#include <vector>

#include "jacobian/product_kernels.cuh"
#include "simulate/fisp_kernels.cuh"
#include "simulate/pssfp_kernels.cuh"
#include "trajectories/phase_encoding_kernels.cuh"
#include "trajectories/signal_kernels.cuh"
#include "utils/residual_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

// ref_sim_hermitian.cpp (its own translation unit, as in the reference: hermitian_kernels.cuh and
// product_kernels.cuh both define kernels::compute_sample_decay)
void run_jacobian_hermitian_naive(int nv, int R, int S, int C, cfloat* jhv, cfloat* echos, cfloat* d1, cfloat* d2,
                                  float* params, const compas::CartesianTrajectoryView& traj, cfloat* coils,
                                  cfloat* u);

namespace {

std::mt19937_64 rng(20241204);

float uniform(float lo, float hi) {
    return std::uniform_real_distribution<float>(lo, hi)(rng);
}

float log_uniform(float lo, float hi) {
    return std::exp(uniform(std::log(lo), std::log(hi)));
}

// [9][nv]: T1 logU[0.1, 4] s, T2 logU[0.01, 0.5] s (< T1), B1 U[0.8, 1.2], B0 N(0, 20) Hz
// (voxel 0 exactly on resonance), rho, x, y, z
std::vector<float> tissue(int nv) {
    std::vector<float> p(9 * nv);
    std::normal_distribution<float> b0(0.0f, 20.0f);
    for (int v = 0; v < nv; v++) {
        float T1 = log_uniform(0.1f, 4.0f), T2;
        do {
            T2 = log_uniform(0.01f, 0.5f);
        } while (T2 >= T1);
        const float rho = uniform(0.5f, 1.0f), phi = uniform(0.0f, 6.2831853f);
        const float vals[9] = {T1, T2, uniform(0.8f, 1.2f), v == 0 ? 0.0f : b0(rng), rho * std::cos(phi),
                               rho * std::sin(phi), uniform(-0.1f, 0.1f), uniform(-0.1f, 0.1f),
                               uniform(-0.5f, 0.5f)};
        for (int f = 0; f < 9; f++) p[f * nv + v] = vals[f];
    }
    return p;
}

compas::TissueParametersView params_view(std::vector<float>& p, int nv) {
    compas::TissueParametersView view;
    view.parameters = host_view(p.data(), 9, nv);
    return view;
}

void print_floats(const char* key, const std::vector<float>& a, bool last = false) {
    std::printf("\"%s\": [", key);
    for (size_t i = 0; i < a.size(); i++) std::printf("%s%.9g", i ? ", " : "", a[i]);
    std::printf("]%s\n", last ? "" : ",");
}

void print_complex(const char* key, const std::vector<cfloat>& a, bool last = false) {
    std::printf("\"%s\": [", key);
    for (size_t i = 0; i < a.size(); i++) std::printf("%s%.9g, %.9g", i ? ", " : "", a[i].re, a[i].im);
    std::printf("]%s\n", last ? "" : ",");
}

struct FispCase {
    int nv, nTR, P, max_state, uf, reps;
    float TR, TE, TI, TW;
    bool inversion, wait_spoil;
};

template<int max_N>
void fisp_case(const FispCase& c, bool last) {
    std::vector<float> p = tissue(c.nv);
    std::vector<cfloat> rf(c.nTR), slices(c.P * c.nTR);
    for (auto& r : rf) r = compas::polar(uniform(5.0f, 80.0f), uniform(-0.3f, 0.3f));
    for (auto& s : slices) s = compas::polar(uniform(0.5f, 1.0f), uniform(-0.1f, 0.1f));

    compas::FISPSequenceView seq;
    seq.RF_train = host_view(rf.data(), c.nTR);
    seq.sliceprofiles = host_view(slices.data(), c.P, c.nTR);
    seq.TR = c.TR;
    seq.TE = c.TE;
    seq.TW = c.TW;
    seq.max_state = c.max_state;
    seq.TI = c.TI;
    seq.undersampling_factor = c.uf;
    seq.repetitions = c.reps;
    seq.inversion_prepulse = c.inversion;
    seq.wait_spoiling = c.wait_spoil;

    const int R = c.nTR * c.uf;
    std::vector<cfloat> transposed(size_t(c.nv) * c.nTR, cfloat(0)), echos(size_t(R) * c.nv, cfloat(0));
    auto tview = host_view(transposed.data(), c.nv, c.nTR);
    const auto pv = params_view(p, c.nv);
    // fisp.cu:35-48: one launch per slice position, the voxel's warp accumulating its samples
    for (int i = 0; i < c.P; i++) {
        for (int v = 0; v < c.nv; v++) {
            blockDim = {1, 1, 1};
            blockIdx = {0, unsigned(v), 0};
            threadIdx = {0, 0, 0};
            compas::kernels::simulate_fisp<max_N, 1, 1>(kmm::Range<int> {0, c.nv}, tview,
                                                        seq.sliceprofiles.drop_axis(i), pv, seq);
        }
    }
    auto eview = host_view(echos.data(), R, c.nv);
    for (int v = 0; v < c.nv; v++)
        for (int r = 0; r < R; r++) {
            blockDim = {1, 1, 1};
            blockIdx = {unsigned(v), unsigned(r), 0};
            threadIdx = {0, 0, 0};
            compas::kernels::expand_undersampled_echos(kmm::Range<int> {0, c.nv}, kmm::Range<int> {0, R}, c.uf,
                                                       eview, tview);
        }

    std::printf("{\"nv\": %d, \"nTR\": %d, \"P\": %d, \"max_state\": %d, \"uf\": %d, \"reps\": %d, ", c.nv, c.nTR,
                c.P, c.max_state, c.uf, c.reps);
    std::printf("\"TR\": %.9g, \"TE\": %.9g, \"TI\": %.9g, \"TW\": %.9g, \"inversion\": %d, \"wait_spoil\": %d,\n",
                c.TR, c.TE, c.TI, c.TW, int(c.inversion), int(c.wait_spoil));
    print_floats("params", p);
    print_complex("rf", rf);
    print_complex("slices", slices);
    print_complex("echos", echos, true);
    std::printf("}%s\n", last ? "" : ",");
}

struct PssfpCase {
    int nv, nTR, nRF, nz;
    float rf_lo, rf_hi;
};

void pssfp_case(const PssfpCase& c, bool last) {
    std::vector<float> p = tissue(c.nv);
    std::vector<cfloat> rf(c.nTR), g(c.nRF);
    std::vector<float> z(c.nz);
    for (auto& r : rf) r = compas::polar(uniform(c.rf_lo, c.rf_hi), uniform(-0.2f, 0.2f));
    // normalised Gaussian RF waveform scaled to 1 degree in total (hard-pulse samples)
    float total = 0.0f;
    for (int i = 0; i < c.nRF; i++) {
        const float t = (i - 0.5f * (c.nRF - 1)) / (0.25f * c.nRF);
        g[i] = cfloat(std::exp(-t * t), 0.0f);
        total += g[i].re;
    }
    for (auto& x : g) x = cfloat(x.re * (float(M_PI) / 180.0f) / total, 0.0f);
    for (int k = 0; k < c.nz; k++) z[k] = c.nz == 1 ? 0.0f : -1.0f + 2.0f * k / (c.nz - 1);

    compas::pSSFPSequenceView seq;
    seq.nTR = c.nTR;
    seq.RF_train = host_view(rf.data(), c.nTR);
    seq.TR = 5e-3f;
    seq.gamma_dt_RF = host_view(g.data(), c.nRF);
    seq.dt = {1e-4f, 1.5e-2f, 2.45e-3f};
    seq.gamma_dt_GRz = {0.4f, 0.0f, -0.2f};
    seq.z = host_view(z.data(), c.nz);

    std::vector<cfloat> echos(size_t(c.nTR) * c.nv, cfloat(0));
    auto eview = host_view(echos.data(), c.nTR, c.nv);
    const auto pv = params_view(p, c.nv);
    // pssfp.cu:16-41 with a batch size of 1: one launch per z position
    for (int iz = 0; iz < c.nz; iz++) {
        auto zsub = host_view(z.data() + iz, 1);
        for (int v = 0; v < c.nv; v++) {
            blockDim = {1, 1, 1};
            blockIdx = {unsigned(v), 0, 0};
            threadIdx = {0, 0, 0};
            compas::kernels::simulate_pssfp<1>(c.nv, eview, zsub, pv, seq);
        }
    }

    std::printf("{\"nv\": %d, \"nTR\": %d, \"nRF\": %d, \"nz\": %d, \"TR\": %.9g, ", c.nv, c.nTR, c.nRF, c.nz,
                seq.TR);
    std::printf("\"dt\": [%.9g, %.9g, %.9g], \"gamma_dt_GRz\": [%.9g, %.9g, %.9g],\n", seq.dt.ex, seq.dt.inv,
                seq.dt.pr, seq.gamma_dt_GRz.ex, seq.gamma_dt_GRz.inv, seq.gamma_dt_GRz.pr);
    print_floats("params", p);
    print_complex("rf", rf);
    print_complex("gamma_dt_RF", g);
    print_floats("z", z);
    print_complex("echos", echos, true);
    std::printf("}%s\n", last ? "" : ",");
}

std::vector<cfloat> random_complex(size_t n) {
    std::vector<cfloat> a(n);
    for (auto& x : a) x = cfloat(uniform(-1.0f, 1.0f), uniform(-1.0f, 1.0f));
    return a;
}

// one thread per launch over the grid (gx, gy, gz), as blockIdx with blockDim 1
template<typename F>
void launch_grid(int gx, int gy, int gz, F&& kernel) {
    for (int k = 0; k < gz; k++)
        for (int j = 0; j < gy; j++)
            for (int i = 0; i < gx; i++) {
                blockDim = {1, 1, 1};
                gridDim = {unsigned(gx), unsigned(gy), unsigned(gz)};
                blockIdx = {unsigned(i), unsigned(j), unsigned(k)};
                threadIdx = {0, 0, 0};
                kernel();
            }
}

// Cartesian trajectory: phase encoding (phase_encoding_kernels.cuh:10-25), the naive signal
// (signal_kernels.cuh:137-167), J·v (product_kernels.cuh:7-66) and Jᴴ·v
// (hermitian_kernels.cuh:30-92), the residual (residual_kernels.cuh, one-thread blocks)
void cartesian_case(int nv, int R, int S, int C) {
    std::vector<float> p = tissue(nv);
    const float fov = 0.2f, dk = 2.0f * float(M_PI) / fov, dt = 1e-5f;
    std::vector<cfloat> k_start(R);
    for (int r = 0; r < R; r++) k_start[r] = cfloat(-0.5f * S * dk, float(r % R - R / 2) * dk);
    auto echos = random_complex(size_t(R) * nv), d1 = random_complex(size_t(R) * nv),
         d2 = random_complex(size_t(R) * nv), coils = random_complex(size_t(C) * nv),
         v = random_complex(size_t(4) * nv), u = random_complex(size_t(C) * R * S),
         rhs = random_complex(size_t(C) * R * S);

    compas::CartesianTrajectoryView traj;
    traj.nreadouts = R;
    traj.samples_per_readout = S;
    traj.delta_t = dt;
    traj.k_start = host_view(k_start.data(), R);
    traj.delta_k = cfloat(dk, 0.0f);  // the C ABI takes a real Δk (julia-bindings/src/bindings.cpp:198-212)
    const auto pv = params_view(p, nv);
    auto ev = host_view(echos.data(), R, nv), d1v = host_view(d1.data(), R, nv), d2v = host_view(d2.data(), R, nv);
    auto cv = host_view(coils.data(), C, nv);

    std::vector<cfloat> ph(size_t(R) * nv), signal(size_t(C) * R * S), jv(size_t(C) * R * S), jhv(size_t(4) * nv);
    launch_grid(nv, R, 1, [&] {
        compas::kernels::phase_encoding(kmm::Bounds<2, int> {{0, nv}, {0, R}, {}}, host_view(ph.data(), R, nv), ev,
                                        pv, traj);
    });
    launch_grid(S, R, C, [&] {
        compas::kernels::sum_signal_cartesian_naive(kmm::Range<int> {0, nv}, host_view(signal.data(), C, R, S), ev,
                                                    pv, traj, cv);
    });
    for (int c = 0; c < C; c++)
        launch_grid(S, R, 1, [&] {
            compas::kernels::jacobian_product_naive(kmm::Range<int> {0, nv}, c, R, S, host_view(jv.data(), C, R, S),
                                                    ev, d1v, d2v, pv, traj, cv, host_view(v.data(), 4, nv));
        });
    run_jacobian_hermitian_naive(nv, R, S, C, jhv.data(), echos.data(), d1.data(), d2.data(), p.data(), traj,
                                 coils.data(), u.data());
    const int n = C * R * S;
    std::vector<cfloat> diff(n);
    std::vector<float> partial(1), objective(1);
    launch_grid(1, 1, 1, [&] {
        compas::kernels::calculate_elementwise_difference<1>(kmm::Range<int> {0, n}, signal.data(), rhs.data(),
                                                             diff.data(), host_view(partial.data(), 1));
    });
    launch_grid(1, 1, 1, [&] {
        compas::kernels::accumulate_partial_sums<1>(host_view(partial.data(), 1), host_view(objective.data(), 1));
    });

    std::printf("{\"nv\": %d, \"R\": %d, \"S\": %d, \"C\": %d, \"dt\": %.9g, \"dk\": %.9g,\n", nv, R, S, C, dt,
                dk);
    print_floats("params", p);
    print_complex("k_start", k_start);
    print_complex("echos", echos);
    print_complex("dT1", d1);
    print_complex("dT2", d2);
    print_complex("coils", coils);
    print_complex("v", v);
    print_complex("u", u);
    print_complex("rhs", rhs);
    print_complex("phase_encoded", ph);
    print_complex("signal", signal);
    print_complex("jv", jv);
    print_complex("jhv", jhv);
    print_complex("residual", diff);
    std::printf("\"objective\": %.9g}\n", objective[0]);
}

// spiral trajectory: prepare_readout_echos, prepare_sample_decay_spiral and sum_signal_spiral
// (signal_kernels.cuh:12-30, 93-105, 274-345) in the host code's order (signal.cu:197-236),
// with one-thread cooperative groups
void spiral_case(int nv, int R, int S, int C) {
    std::vector<float> p = tissue(nv);
    const float fov = 0.2f, dt = 4e-6f;
    std::vector<cfloat> k_start(R), delta_k(R);
    for (int r = 0; r < R; r++) {
        const float a = 2.0f * float(M_PI) * r / R;
        k_start[r] = cfloat(std::cos(a), std::sin(a)) * (2.0f * float(M_PI) / fov);
        delta_k[r] = cfloat(-std::sin(a), std::cos(a)) * (0.5f * float(M_PI) / fov);
    }
    auto echos = random_complex(size_t(R) * nv), coils = random_complex(size_t(C) * nv);
    compas::SpiralTrajectoryView traj;
    traj.nreadouts = R;
    traj.samples_per_readout = S;
    traj.delta_t = dt;
    traj.k_start = host_view(k_start.data(), R);
    traj.delta_k = host_view(delta_k.data(), R);
    const auto pv = params_view(p, nv);

    std::vector<cfloat> readout_echos(size_t(R) * nv), decay(size_t(R) * nv), signal(size_t(C) * R * S);
    launch_grid(nv, R, 1, [&] {
        compas::kernels::prepare_readout_echos(kmm::Range<int> {0, nv}, kmm::Range<int> {0, R},
                                               host_view(readout_echos.data(), R, nv),
                                               host_view(echos.data(), R, nv), pv, traj);
    });
    launch_grid(nv, R, 1, [&] {
        compas::kernels::prepare_sample_decay_spiral(host_view(decay.data(), R, nv), pv, traj);
    });
    launch_grid(S, R, C, [&] {
        compas::kernels::sum_signal_spiral<1, 1, 1, 1>(host_view(signal.data(), C, R, S),
                                                      host_view(decay.data(), R, nv),
                                                      host_view(readout_echos.data(), R, nv),
                                                      host_view(coils.data(), C, nv));
    });

    std::printf("{\"nv\": %d, \"R\": %d, \"S\": %d, \"C\": %d, \"dt\": %.9g,\n", nv, R, S, C, dt);
    print_floats("params", p);
    print_complex("k_start", k_start);
    print_complex("delta_k", delta_k);
    print_complex("echos", echos);
    print_complex("coils", coils);
    print_complex("signal", signal, true);
    std::printf("}\n");
}

}  // namespace

int main() {
    std::printf("{\"fisp\": [\n");
    fisp_case<32>({8, 50, 3, 8, 2, 2, 8.7e-3f, 4.35e-3f, 20e-3f, 30e-3f, true, true}, false);
    fisp_case<32>({6, 40, 2, 25, 1, 1, 8.7e-3f, 4.35e-3f, 25e-3f, 0.0f, true, true}, false);
    fisp_case<128>({5, 30, 2, 100, 1, 1, 6.0e-3f, 3.0e-3f, 15e-3f, 0.0f, true, true}, false);
    fisp_case<32>({6, 35, 2, 12, 1, 2, 8.7e-3f, 4.35e-3f, 20e-3f, 10e-3f, false, false}, true);
    std::printf("],\n\"pssfp\": [\n");
    pssfp_case({6, 30, 5, 7, 10.0f, 60.0f}, false);
    pssfp_case({5, 25, 15, 35, 10.0f, 60.0f}, false);
    pssfp_case({4, 20, 3, 9, 120.0f, 180.0f}, true);
    std::printf("],\n\"cartesian\": ");
    cartesian_case(12, 10, 8, 3);
    std::printf(",\n\"spiral\": ");
    spiral_case(10, 6, 12, 2);
    std::printf("}\n");
    return 0;
}
