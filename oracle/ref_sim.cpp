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
// calls (oracle/refshim/cuda_host_shim.h). Prints the inputs and echoes of seeded cases as JSON;
// tests/golden/make_golden.py stores them as tests/golden/ref_simulations.json.
#include <cstdio>
#include <random>
#include <vector>

#include "simulate/fisp_kernels.cuh"
#include "simulate/pssfp_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

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
    std::printf("]}\n");
    return 0;
}
