// gg_run.cpp -- a C++ host for the B200 timestep: the reference's mode-4 run, driven through
// the C ABI of libgg_b200.so.
//
// It stands where ggLS.cpp's main (ggLS.cpp:27-84) and grainhdl::run_sim (grainhdl.cpp:
// 821-934) stand for a voxelised microstructure (MicrostructureGenMode 4): it reads the
// same parameters.xml tags (Settings.cpp:81-270), the same Container.raw and .uds files
// (grainhdl.cpp:404-578), builds the same initial comparison lists (the R-tree search of
// find_neighbors), runs NumberOfTimesteps + 1 loop iterations or until fewer than
// BreakupNumber grains remain, and prints the reference's per-analysis-step report.
//
//   gg_run parameters.xml [--mixed] [--stats file]
//
// --mixed selects GG_PRECISION_MIXED (FP32 storage, tensor-core convolution); the default
// is GG_PRECISION_FP64, bit-exact with the reference.  --stats writes one line per loop:
// loop, grains, live grains, the sum of the grains' volumes, ms of the step.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "gg_b200.h"

namespace {

// The text of <tag>...</tag> in the parameters file, or `fallback` when absent (the
// reference keeps the Settings default then, Settings.cpp:29-79, as the fallbacks below do).
std::string tag(const std::string& xml, const std::string& name, const std::string& fallback) {
    const std::string open = "<" + name + ">", close = "</" + name + ">";
    const size_t a = xml.find(open);
    if (a == std::string::npos) return fallback;
    const size_t b = xml.find(close, a + open.size());
    if (b == std::string::npos) return fallback;
    std::string v = xml.substr(a + open.size(), b - a - open.size());
    const size_t s = v.find_first_not_of(" \t\r\n"), e = v.find_last_not_of(" \t\r\n");
    return s == std::string::npos ? fallback : v.substr(s, e - s + 1);
}

std::string dir_of(const std::string& path) {
    const size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

std::string resolve(const std::string& dir, const std::string& file) {
    return (!file.empty() && file[0] == '/') ? file : dir + "/" + file;
}

struct Uds {
    int id_offset = 1, nx = 0, grains = 0;
    std::vector<int32_t> extents;   // grains x 6
    std::vector<int64_t> counts;    // grains
    std::vector<double> euler;      // grains x 3
    std::vector<double> stored;     // grains: the storedEnergy column
};

// read_voxelized_microstructure's header and rows (grainhdl.cpp:421-490).
Uds read_uds(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot read " + path);
    Uds u;
    std::string line;
    for (int i = 1; i <= 12 && std::getline(in, line); i++) {
        std::istringstream ls(line);
        std::string key;
        int v = 0;
        if (i == 2 && (ls >> key >> v)) u.id_offset = v;
        if (i == 6 && (ls >> key >> v)) u.nx = v;
        if (i == 9 && (ls >> key >> v)) u.grains = v;
    }
    if (u.nx <= 0 || u.grains <= 0) throw std::runtime_error("bad .uds header in " + path);
    u.extents.resize(6 * (size_t)u.grains);
    u.counts.resize(u.grains);
    u.euler.resize(3 * (size_t)u.grains);
    u.stored.resize(u.grains);
    for (int g = 0; g < u.grains; g++) {
        long long id, x, y, z, count;
        double e0, e1, e2, se;
        long long b[6];
        if (!(in >> id >> x >> y >> z >> e0 >> e1 >> e2 >> b[0] >> b[1] >> b[2] >> b[3] >> b[4] >> b[5] >> count >> se))
            throw std::runtime_error("truncated .uds row " + std::to_string(g + 1) + " in " + path);
        for (int q = 0; q < 6; q++) u.extents[6 * (size_t)g + q] = (int32_t)b[q];
        u.counts[g] = count;
        u.euler[3 * (size_t)g] = e0;
        u.euler[3 * (size_t)g + 1] = e1;
        u.euler[3 * (size_t)g + 2] = e2;
        u.stored[g] = se;
    }
    return u;
}

void check(gg_ctx* ctx, int rc, const char* what) {
    if (rc < 0) throw std::runtime_error(std::string(what) + ": " + gg_last_error(ctx));
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s parameters.xml [--mixed] [--stats file]\n", argv[0]);
        return 2;
    }
    gg_ctx* ctx = nullptr;
    try {
        const std::string params_path = argv[1];
        bool mixed = false;
        std::string stats_path;
        for (int i = 2; i < argc; i++) {
            if (!std::strcmp(argv[i], "--mixed")) mixed = true;
            else if (!std::strcmp(argv[i], "--stats") && i + 1 < argc) stats_path = argv[++i];
        }
        std::ifstream pf(params_path);
        if (!pf) throw std::runtime_error("cannot read " + params_path);
        std::stringstream ss;
        ss << pf.rdbuf();
        const std::string xml = ss.str();
        if (std::atoi(tag(xml, "MicrostructureGenMode", "4").c_str()) != 4)
            throw std::runtime_error("only MicrostructureGenMode 4 (voxelised input) is read by this host");
        const std::string dir = dir_of(params_path);
        const Uds uds = read_uds(resolve(dir, tag(xml, "AdditionalFilename", "")));
        const int N = uds.nx, G = uds.grains;
        std::vector<uint32_t> labels((size_t)N * N * N);
        {
            const std::string raw = resolve(dir, tag(xml, "ReadFromFilename", ""));
            FILE* f = std::fopen(raw.c_str(), "rb");
            if (!f) throw std::runtime_error("cannot read " + raw);
            const size_t got = std::fread(labels.data(), sizeof(uint32_t), labels.size(), f);
            std::fclose(f);
            if (got != labels.size()) throw std::runtime_error("short container file " + raw);
            for (auto& v : labels) v -= (uint32_t)(uds.id_offset - 1);
        }
        const auto num = [&](const char* name, const char* fallback) { return std::atof(tag(xml, name, fallback).c_str()); };
        gg_params p = {};
        p.domain_size = N;
        p.border = (int32_t)num("DomainBorderSize", "0");
        p.time_step = num("TimeStepSize", "0.2");
        p.n_grains = G;
        p.precision = mixed ? GG_PRECISION_MIXED : GG_PRECISION_FP64;
        p.disable_correction = (int32_t)num("DisableConvolutionCorrection", "0");
        p.unique_gb_energies = (int32_t)num("UniqueGBEnergies", "0");
        p.mobility_model = (int32_t)num("UseMobilityFactor", "0");
        p.use_stored_energy = (int32_t)num("UseStoredElasticEnergy", "0");
        p.triple_line_drag = num("TripleLineDrag", "0");
        p.grid_coarsening = (int32_t)num("GridCoarsement", "0");
        p.coarsening_gradient = num("GridCoarsementGradient", "0.95");
        p.device = 0;
        check(ctx, gg_create(&p, &ctx), "gg_create");
        check(ctx, gg_load_state(ctx, labels.data(), uds.extents.data(), uds.counts.data()), "gg_load_state");
        check(ctx, gg_set_orientations(ctx, uds.euler.data()), "gg_set_orientations");
        // m_StoredElasticEnergy = DislocEnPerM * storedEnergy / HAGB_Energy * Physical_Domain_Size (box.cpp:232-233)
        const double disloc = num("DislocEnPerM", "0"), hagb = num("HAGB_Energy", "0"),
                     phys = num("Physical_Domain_Size", "0");
        std::vector<double> see(G);
        for (int g = 0; g < G; g++) see[g] = hagb != 0 ? disloc * uds.stored[g] / hagb * phys : 0.0;
        check(ctx, gg_set_stored_energy(ctx, see.data()), "gg_set_stored_energy");
        check(ctx, gg_rtree_lists(ctx), "gg_rtree_lists");

        const int steps = (int)num("NumberOfTimesteps", "0"), breakup = (int)num("BreakupNumber", "0");
        const int analysis = std::max(1, (int)num("AnalysisTimestep", "0"));
        FILE* stats = stats_path.empty() ? nullptr : std::fopen(stats_path.c_str(), "w");
        std::vector<double> volume(G + 1);
        std::vector<uint8_t> exists(G + 1);
        const auto t0 = std::chrono::steady_clock::now();
        for (int loop = 0; loop <= steps; loop++) {  // grainhdl.cpp:837
            gg_step_stats st{};
            check(ctx, gg_step(ctx, &st), "gg_step");
            if (stats) {
                check(ctx, gg_get_grain_stats(ctx, exists.data(), volume.data(), nullptr, nullptr, nullptr),
                      "gg_get_grain_stats");
                double total = 0;
                for (int g = 1; g <= G; g++)
                    if (exists[g]) total += volume[g];
                std::fprintf(stats, "%d\t%d\t%d\t%.17g\t%.4f\n", st.loop, st.grain_count, st.live_grains, total,
                             st.ms_total);
            }
            if (loop % analysis == 0) {
                std::printf("Timestep %d complete:\n", loop);
                std::printf("Number of grains remaining in the Network :%d\n", st.grain_count);
            }
            if (st.grain_count < breakup) {  // grainhdl.cpp:911-917
                std::printf("Network has coarsened such that only %d grains remain\n", st.grain_count);
                break;
            }
        }
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("Elapsed seconds for simulation: %.3f\n", secs);
        if (stats) std::fclose(stats);
        gg_destroy(ctx);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "gg_run: %s\n", e.what());
        if (ctx) gg_destroy(ctx);
        return 1;
    }
}
