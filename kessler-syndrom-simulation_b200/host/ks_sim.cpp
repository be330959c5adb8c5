// ks_sim: the reference CLI's screened step loop (src/main.cpp:346-407) on
// the B200 engine, with the same inputs and the same output files.
//
//   ks_sim [catalogue] [duration_h] [dt_s] [options]
//     --conj-km X          conjunction threshold, km (default 5)
//     --radius-scale S     multiplies every collision radius (default 1)
//     --min-vrel V         minimum encounter speed, m/s (default 10)
//     --split              split precision (FP32 J2 / lunar terms, FP32 pair gate)
//     --steps-per-graph K  steps captured per CUDA graph (default 32)
//     --out DIR            output directory (default output)
//     --device D           CUDA device (default 0)
//
// Reads the reference's pipe-separated catalogue format (fields 0, 1, 2, 4, 5,
// 11-16; sizes from the RCS class, src/core/orbital.cpp:136-170) and the
// common epoch of its header (src/core/orbital.cpp:172-188). Writes
// DIR/conjunctions.csv and DIR/final_state.csv in the reference's formats
// (src/main.cpp:264-266, 395-400; src/core/orbital.cpp:190-197), so the files
// can be diffed against the reference's.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "kessler_b200.hpp"

namespace {

constexpr double kDefaultEpochJd = 2461253.916666667;  // src/core/orbital.hpp:30

struct CatalogObject {
    int id = 0;
    std::string name;
    double size_m = 0.8;
    double s[6] = {0, 0, 0, 0, 0, 0};
};

std::string trim(const std::string& s) {
    const size_t b = s.find_first_not_of(" \t\r\n"), e = s.find_last_not_of(" \t\r\n");
    return b == std::string::npos ? "" : s.substr(b, e - b + 1);
}

// Pipe-separated rows; '#' lines are the header. Size from the radar cross
// section class: SMALL 0.2 m, LARGE 4 m, anything else 0.8 m.
std::vector<CatalogObject> load_catalog(const std::string& path, int* dropped) {
    std::ifstream in(path);
    std::vector<CatalogObject> out;
    if (!in) return out;
    std::string line;
    int bad = 0;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::vector<std::string> f;
        std::stringstream ss(line);
        std::string tok;
        while (std::getline(ss, tok, '|')) f.push_back(trim(tok));
        if (f.size() < 17) {
            ++bad;
            continue;
        }
        try {
            CatalogObject o;
            o.id = std::stoi(f[0]);
            o.name = f[1];
            o.size_m = f[5] == "SMALL" ? 0.2 : f[5] == "LARGE" ? 4.0 : 0.8;
            for (int q = 0; q < 6; ++q) o.s[q] = std::stod(f[11 + q]);
            out.push_back(o);
        } catch (...) {
            ++bad;
        }
    }
    if (dropped) *dropped = bad;
    return out;
}

// Civil date (UTC) to Julian date, Meeus, Astronomical Algorithms ch. 7.
double to_jd(int y, int m, double day) {
    if (m <= 2) {
        y -= 1;
        m += 12;
    }
    const int A = y / 100;
    const int B = 2 - A + A / 4;
    return std::floor(365.25 * (y + 4716)) + std::floor(30.6001 * (m + 1)) + day + B - 1524.5;
}

// Epoch from a header line "...epoch commun) : YYYY-MM-DDTHH:MM:SS..." (the
// reference's exporter writes it; src/core/orbital.cpp:178-184).
double read_epoch_jd(const std::string& path) {
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] != '#') break;
        const size_t pos = line.find("epoch commun) :");
        if (pos == std::string::npos) continue;
        int y, mo, d, h, mi, s;
        if (std::sscanf(line.c_str() + pos, "epoch commun) : %d-%d-%dT%d:%d:%d", &y, &mo, &d, &h, &mi, &s) == 6)
            return to_jd(y, mo, d + (h + mi / 60.0 + s / 3600.0) / 24.0);
    }
    return kDefaultEpochJd;
}

std::string csv_quote(const std::string& s) {
    std::string out = "\"";
    for (char c : s) out += (c == '"') ? std::string("\"\"") : std::string(1, c);
    return out + "\"";
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    kessler_b200::ScreeningConfig cfg;
    bool split = false;
    int spg = 32, device = 0;
    std::string out_dir = "output";
    for (int k = 1; k < argc; ++k) {
        const std::string a = argv[k];
        if (a == "--conj-km" && k + 1 < argc) cfg.threshold_km = std::atof(argv[++k]);
        else if (a == "--radius-scale" && k + 1 < argc) cfg.radius_scale = std::atof(argv[++k]);
        else if (a == "--min-vrel" && k + 1 < argc) cfg.min_encounter_speed_km_s = std::atof(argv[++k]) * 1e-3;
        else if (a == "--split") split = true;
        else if (a == "--steps-per-graph" && k + 1 < argc) spg = std::atoi(argv[++k]);
        else if (a == "--out" && k + 1 < argc) out_dir = argv[++k];
        else if (a == "--device" && k + 1 < argc) device = std::atoi(argv[++k]);
        else if (a.rfind("--", 0) == 0) {
            std::cerr << "unknown option " << a << "\n";
            return 1;
        } else pos.push_back(a);
    }
    const std::string path = pos.size() > 0 ? pos[0] : "data/satellites_20260801_1000Z.txt";
    const double duration = (pos.size() > 1 ? std::atof(pos[1].c_str()) : 24.0) * 3600.0;
    const double dt = pos.size() > 2 ? std::atof(pos[2].c_str()) : 10.0;

    int dropped = 0;
    const std::vector<CatalogObject> objs = load_catalog(path, &dropped);
    if (objs.empty()) {
        std::cerr << "no object loaded from " << path << "\n";
        return 1;
    }
    if (dropped) std::cerr << dropped << " malformed lines skipped\n";
    const double epoch = read_epoch_jd(path);
    const size_t n = objs.size();
    std::vector<double> states(6 * n), size_m(n);
    for (size_t i = 0; i < n; ++i) {
        std::copy(objs[i].s, objs[i].s + 6, &states[6 * i]);
        size_m[i] = objs[i].size_m;
    }
    const long steps = static_cast<long>(std::ceil(duration / dt));

    try {
        kessler_b200::DeviceSimulation sim(device);
        std::cout << n << " objects, " << duration / 3600.0 << " h, dt " << dt << " s, " << steps << " steps on "
                  << sim.context().device_name() << (split ? " (split precision)" : " (FP64)") << "\n";
        sim.set_precision(split ? KS_PRECISION_SPLIT : KS_PRECISION_FP64);
        sim.set_steps_per_graph(spg);
        sim.set_clock(epoch, 0.0, dt);
        sim.set_screening(true, cfg);
        sim.set_population(states, size_m);

        std::filesystem::create_directories(out_dir);
        std::ofstream conj_out(out_dir + "/conjunctions.csv");
        conj_out << "t_s,id1,id2,name1,name2,miss_km,v_rel_km_s,collision\n";
        conj_out << std::setprecision(10);
        long long n_conj = 0, n_coll = 0, candidates = 0, below[4] = {0, 0, 0, 0};
        const double bins[4] = {0.1, 1.0, 2.0, 5.0};
        double closest = 1e30;
        int ci = -1, cj = -1;
        double tc = 0;
        const auto t0 = std::chrono::steady_clock::now();
        const long chunk = std::max<long>(spg, 1) * 32;
        for (long done = 0; done < steps;) {
            const long k = std::min(chunk, steps - done);
            sim.advance(k);
            done += k;
            for (const ks_conjunction& c : sim.take_conjunctions()) {
                const CatalogObject& a = objs[c.i];
                const CatalogObject& b = objs[c.j];
                conj_out << c.t << ',' << a.id << ',' << b.id << ',' << csv_quote(a.name) << ',' << csv_quote(b.name)
                         << ',' << c.miss_km << ',' << c.v_rel_km_s << ',' << (c.collision ? 1 : 0) << '\n';
                ++n_conj;
                n_coll += c.collision ? 1 : 0;
                for (int q = 0; q < 4; ++q) below[q] += c.miss_km < bins[q] ? 1 : 0;
                if (c.miss_km < closest) {
                    closest = c.miss_km;
                    ci = c.i;
                    cj = c.j;
                    tc = c.t;
                }
            }
            for (const ks_step_stats& st : sim.take_step_stats()) candidates += st.candidate_pairs;
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

        std::vector<double> fs;
        std::vector<uint8_t> fa;
        sim.get_population(fs, fa);
        std::ofstream snap(out_dir + "/final_state.csv");
        snap << "# t = " << sim.time() << " s apres l'epoch\nid,x_km,y_km,z_km,vx,vy,vz,alive\n";
        snap.precision(9);
        for (size_t i = 0; i < n; ++i) {
            snap << objs[i].id;
            for (int q = 0; q < 6; ++q) snap << ',' << fs[6 * i + q];
            snap << ',' << (fa[i] ? 1 : 0) << '\n';
        }

        std::cout << "conjunctions below " << cfg.threshold_km << " km: " << n_conj << " (collisions " << n_coll
                  << ")\n";
        for (int q = 0; q < 4; ++q)
            if (bins[q] <= cfg.threshold_km) std::cout << "  below " << bins[q] << " km: " << below[q] << "\n";
        if (ci >= 0)
            std::cout << "closest: " << closest * 1000.0 << " m between " << objs[ci].name << " (" << objs[ci].id
                      << ") and " << objs[cj].name << " (" << objs[cj].id << ") at t = " << tc / 3600.0 << " h\n";
        std::cout << "candidate pairs per step: " << candidates / std::max(1L, steps) << "\n";
        std::cout << "wall " << wall << " s, " << static_cast<double>(n) * steps / wall << " object-steps/s\n";
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 2;
    }
    return 0;
}
