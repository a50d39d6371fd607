// tuning.cu — launch-layout selection for the simulation kernels.
//
// The FISP and pSSFP kernels are instantiated for several register layouts (states or
// isochromats per lane × lanes per voxel); the tensor-core contractions take a readout tile
// (Cartesian signal / J·v) and a split count. The choice is made, in order, from
//   1. an explicit override (compas_b200_set_*_launch, used by the autotuner while timing),
//   2. the autotuner's table (COMPAS_B200_TUNING file, one line per shape class:
//      "fisp <N> <voxel-bucket> <P-bucket> <config> <warps>",
//      "pssfp <nz> <voxel-bucket> <config>" or
//      "tc <kind> <readout-bucket> <voxel-bucket> <coil·sample-bucket> <tile> <splits>"), written by
//      compas_b200_autotune.py,
//   3. the built-in heuristic (fisp_default_launch / pssfp_default_launch / the plan functions of
//      the tensor-core launchers).
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>

#include "common.cuh"
#include "kernels.h"

namespace compas {

namespace {
std::atomic<int> g_fisp_cfg {-1}, g_fisp_warps {-1}, g_pssfp_cfg {-1}, g_fisp_tangent_cfg {-1};
constexpr int kTcKinds = int(TcKind::Count);
std::atomic<int> g_tc_tile[kTcKinds], g_tc_splits[kTcKinds];  // 0 = no override (static: zero-initialised)

struct Table {
    std::map<std::tuple<int, int, int>, std::pair<int, int>> fisp;  // (N, vbucket, pbucket) -> (cfg, warps)
    std::map<std::tuple<int, int>, int> pssfp;                        // (nz, vbucket) -> cfg
    std::map<std::tuple<int, int, int, int>, std::pair<int, int>> tc;  // (kind, rbucket, vbucket, csbucket) -> (tile, splits)
};

bool valid_tc_tile(int tile) {
    return tile == 0 || (tile >= 16 && tile <= 256 && tile % 16 == 0);
}

int bucket(int64_t n) {  // log2 bucket
    int b = 0;
    while (n > 1) {
        n >>= 1;
        b++;
    }
    return b;
}

const Table& table() {
    static Table t;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* path = std::getenv("COMPAS_B200_TUNING");
        if (!path || !*path) return;
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream s(line);
            std::string kind;
            s >> kind;
            if (kind == "fisp") {
                int N, vb, pb, cfg, w;
                if (s >> N >> vb >> pb >> cfg >> w) t.fisp[{N, vb, pb}] = {cfg, w};
            } else if (kind == "pssfp") {
                int nz, vb, cfg;
                if (s >> nz >> vb >> cfg) t.pssfp[{nz, vb}] = cfg;
            } else if (kind == "tc") {
                int k, rb, vb, cb, tile, splits;
                if (s >> k >> rb >> vb >> cb >> tile >> splits && k >= 0 && k < kTcKinds && valid_tc_tile(tile) &&
                    splits >= 0)
                    t.tc[{k, rb, vb, cb}] = {tile, splits};
            }
        }
    });
    return t;
}
}  // namespace

void set_fisp_override(int config, int warps) {
    if (config >= fisp_config_count()) COMPAS_ERROR("FISP layout index out of range");
    g_fisp_cfg = config;
    g_fisp_warps = warps;
}

void set_fisp_tangent_override(int config) {
    if (config >= fisp_tangent_config_count()) COMPAS_ERROR("FISP tangent layout index out of range");
    g_fisp_tangent_cfg = config;
}

// Tangent layout: the override when it covers N states, else the default; the warps per CTA are
// always the value kernel's, so the value sums the positions in the same order.
FispLaunch tuned_fisp_tangent_launch(int N, int64_t nvoxels, int P) {
    FispLaunch d = fisp_tangent_default_launch(N, nvoxels, P);
    const int cfg = g_fisp_tangent_cfg.load();
    int K = 0, G = 0;
    if (cfg >= 0 && fisp_tangent_config_info(cfg, &K, &G) && K * G >= N) d.config = cfg;
    return d;
}

void set_pssfp_override(int config) {
    if (config >= pssfp_config_count()) COMPAS_ERROR("pSSFP layout index out of range");
    g_pssfp_cfg = config;
}

FispLaunch tuned_fisp_launch(int N, int64_t nvoxels, int P) {
    FispLaunch d = fisp_default_launch(N, nvoxels, P);
    int cfg = g_fisp_cfg.load();
    if (cfg >= 0) {
        int K = 0, G = 0;
        fisp_config_info(cfg, &K, &G);
        if (K * G >= N) {
            int w = g_fisp_warps.load();
            return FispLaunch {cfg, w > 0 ? w : d.warps};
        }
    }
    const auto& t = table();
    auto it = t.fisp.find({N, bucket(nvoxels), bucket(P)});
    if (it != t.fisp.end()) {
        int K = 0, G = 0;
        if (fisp_config_info(it->second.first, &K, &G) && K * G >= N) return FispLaunch {it->second.first, it->second.second};
    }
    return d;
}

PssfpLaunch tuned_pssfp_launch(int nz, int64_t nvoxels) {
    int cfg = g_pssfp_cfg.load();
    if (cfg >= 0) {
        int ZT = 0, GZ = 0;
        pssfp_config_info(cfg, &ZT, &GZ);
        if (ZT * GZ >= nz) return PssfpLaunch {cfg};
    }
    const auto& t = table();
    auto it = t.pssfp.find({nz, bucket(nvoxels)});
    if (it != t.pssfp.end()) {
        int ZT = 0, GZ = 0;
        if (pssfp_config_info(it->second, &ZT, &GZ) && ZT * GZ >= nz) return PssfpLaunch {it->second};
    }
    return pssfp_default_launch(nz, nvoxels);
}

void set_tc_override(int kind, int tile, int splits) {
    if (kind < 0 || kind >= kTcKinds) COMPAS_ERROR("tensor-core contraction kind out of range");
    if (!valid_tc_tile(tile)) COMPAS_ERROR("tensor-core readout tile must be 0 or a multiple of 16 in [16, 256]");
    if (splits < 0) COMPAS_ERROR("tensor-core split count must be 0 (built-in) or positive");
    g_tc_tile[kind] = tile;
    g_tc_splits[kind] = splits;
}

TcTuning tuned_tc(TcKind kind, int R, int64_t nvoxels, int64_t coil_samples) {
    const int k = int(kind);
    TcTuning t;
    t.tile = g_tc_tile[k].load();
    t.splits = g_tc_splits[k].load();
    if (t.tile > 0 || t.splits > 0) return t;
    const auto& tab = table();
    auto it = tab.tc.find({k, bucket(R), bucket(nvoxels), bucket(coil_samples)});
    if (it != tab.tc.end()) {
        t.tile = it->second.first;
        t.splits = it->second.second;
    }
    return t;
}

TcTuning tc_launch_choice(int device, TcKind kind, int nvoxels, int R, int S, int C) {
    TcTuning t;
    switch (kind) {
    case TcKind::CartesianSignal:
    case TcKind::CartesianJacobian: {
        const TcPlan p = tc_plan(device, nvoxels, R, S, C, kind == TcKind::CartesianJacobian);
        t.tile = p.nr;
        t.splits = p.splits;
        break;
    }
    case TcKind::CartesianHermitian: t.splits = tc_hermitian_splits(device, nvoxels, R, S, C); break;
    case TcKind::SpiralSignal:
    case TcKind::SpiralJacobian:
        t.splits = tc_spiral_splits(device, nvoxels, R, S, C, kind == TcKind::SpiralJacobian);
        break;
    case TcKind::SpiralHermitian: t.splits = tc_spiral_hermitian_splits(device, nvoxels, R, S, C); break;
    default: COMPAS_ERROR("tensor-core contraction kind out of range");
    }
    return t;
}

}  // namespace compas
