// ks_sim: the reference CLI's screened step loop (src/main.cpp:346-407) on
// the B200 engine, with the same inputs and the same output files.
//
//   ks_sim [catalogue] [duration_h] [dt_s] [out_every_s] [ids] [options]
//     out_every_s          write DIR/snapshot_<k>.csv every out_every_s seconds (0 = final state only)
//     ids                  comma-separated ids: instead of snapshots, their positions go to
//                          DIR/trajectories.csv and the Moon's to DIR/moon.csv (every out_every_s,
//                          default 60 s)
//     --conj-km X          conjunction threshold, km (default 5)
//     --radius-scale S     multiplies every collision radius (default 1)
//     --min-vrel V         minimum encounter speed, m/s (default 10)
//     --breakup            collisions fragment their objects (NASA SBM)
//     --lc L               smallest fragment followed, m (default 0.1)
//     --masses FILE        catalogue mass table (default config/masses.csv)
//     --seed N             seed of the fragment draws (default 1)
//     --impact NORAD       forced impact of a fictitious projectile on that object (implies --breakup)
//     --impact-mass KG     projectile mass (default 10)
//     --impact-vrel KMS    impact speed (default 10)
//     --impact-at H        time of the impact, hours (default 0)
//     --split              split precision (FP32 J2 / lunar terms, FP32 pair gate)
//     --steps-per-graph K  steps captured per CUDA graph (default 32)
//     --out DIR            output directory (default output)
//     --device D           CUDA device (default 0)
//   (--screen, --gpu and --threads N are accepted for compatibility: the loop
//   always screens, on the GPU.)
//
// Reads the reference's pipe-separated catalogue format (fields 0, 1, 2, 4, 5,
// 11-16; sizes from the RCS class, src/core/orbital.cpp:136-170) and the
// common epoch of its header (src/core/orbital.cpp:172-188). Writes
// DIR/conjunctions.csv and DIR/final_state.csv in the reference's formats
// (src/main.cpp:264-266, 395-400; src/core/orbital.cpp:190-197), with
// fragmentation DIR/breakups.csv and DIR/population.csv (src/main.cpp:283-333),
// and the periodic snapshots or trajectories of src/main.cpp:185-235, 437-447,
// so the files can be diffed against the reference's.
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

constexpr int kFragmentIdBase = 10000000;  // src/core/orbital.hpp:65

struct CatalogObject {
    int id = 0;
    std::string name, type, rcs;
    double size_m = 0.8;
    double s[6] = {0, 0, 0, 0, 0, 0};
};

// Catalogue masses by radar cross-section class (SMALL, MEDIUM, LARGE, other)
// and object type (PAYLOAD, DEBRIS, ROCKET BODY, other): the defaults and CSV
// format ("rcs,type,mass_kg") of the reference's MassTable
// (src/core/breakup.cpp:47-102).
class MassTable {
public:
    double kg[4][4] = {{5.0, 0.5, 50.0, 1.0}, {50.0, 5.0, 300.0, 10.0}, {500.0, 50.0, 2000.0, 100.0},
                       {100.0, 5.0, 500.0, 10.0}};

    static int rcs_row(const std::string& rcs) {
        return rcs == "SMALL" ? 0 : rcs == "MEDIUM" ? 1 : rcs == "LARGE" ? 2 : 3;
    }
    static int type_col(const std::string& type) {
        return type == "PAYLOAD" ? 0 : type == "DEBRIS" ? 1 : type == "ROCKET BODY" ? 2 : 3;
    }
    bool load(const std::string& path, std::string* error) {
        std::ifstream in(path);
        if (!in) {
            *error = "cannot open " + path;
            return false;
        }
        static const char* kTypes[4] = {"PAYLOAD", "DEBRIS", "ROCKET BODY", "UNKNOWN"};
        std::string line;
        int lineno = 0;
        while (std::getline(in, line)) {
            ++lineno;
            if (!line.empty() && line.back() == '\r') line.pop_back();
            if (line.empty() || line[0] == '#' || line.rfind("rcs,", 0) == 0) continue;
            std::stringstream ss(line);
            std::string rcs, type, mass;
            std::getline(ss, rcs, ',');
            std::getline(ss, type, ',');
            std::getline(ss, mass, ',');
            int col = -1;
            for (int k = 0; k < 4; ++k)
                if (type == kTypes[k]) col = k;
            const bool rcs_ok = rcs == "SMALL" || rcs == "MEDIUM" || rcs == "LARGE" || rcs == "NONE";
            const double v = std::atof(mass.c_str());
            if (col < 0 || !rcs_ok || v <= 0) {
                *error = path + ", line " + std::to_string(lineno) + " invalid: " + line;
                return false;
            }
            kg[rcs_row(rcs)][col] = v;
        }
        return true;
    }
    double mass_for(const CatalogObject& o) const { return kg[rcs_row(o.rcs)][type_col(o.type)]; }
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
            o.type = f[2];
            o.rcs = f[5];
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
    bool split = false, breakup = false, conj_explicit = false;
    int spg = 32, device = 0;
    double lc_m = 0.10, impact_mass = 10.0, impact_vrel = 10.0, impact_at_h = 0.0;
    uint64_t seed = 1;
    int impact_id = -1;
    std::string out_dir = "output", masses_path = "config/masses.csv";
    for (int k = 1; k < argc; ++k) {
        const std::string a = argv[k];
        if (a == "--conj-km" && k + 1 < argc) {
            cfg.threshold_km = std::atof(argv[++k]);
            conj_explicit = true;
        } else if (a == "--radius-scale" && k + 1 < argc) cfg.radius_scale = std::atof(argv[++k]);
        else if (a == "--min-vrel" && k + 1 < argc) cfg.min_encounter_speed_km_s = std::atof(argv[++k]) * 1e-3;
        else if (a == "--breakup") breakup = true;
        else if (a == "--lc" && k + 1 < argc) lc_m = std::atof(argv[++k]);
        else if (a == "--masses" && k + 1 < argc) masses_path = argv[++k];
        else if (a == "--seed" && k + 1 < argc) seed = std::strtoull(argv[++k], nullptr, 10);
        else if (a == "--impact" && k + 1 < argc) {
            impact_id = std::atoi(argv[++k]);
            breakup = true;
        } else if (a == "--impact-mass" && k + 1 < argc) impact_mass = std::atof(argv[++k]);
        else if (a == "--impact-vrel" && k + 1 < argc) impact_vrel = std::atof(argv[++k]);
        else if (a == "--impact-at" && k + 1 < argc) impact_at_h = std::atof(argv[++k]);
        else if (a == "--split") split = true;
        else if (a == "--steps-per-graph" && k + 1 < argc) spg = std::atoi(argv[++k]);
        else if (a == "--out" && k + 1 < argc) out_dir = argv[++k];
        else if (a == "--device" && k + 1 < argc) device = std::atoi(argv[++k]);
        else if (a == "--threads" && k + 1 < argc) ++k;
        else if (a == "--screen" || a == "--gpu") continue;
        else if (a.rfind("--", 0) == 0) {
            std::cerr << "unknown option " << a << "\n";
            return 1;
        } else pos.push_back(a);
    }
    const std::string path = pos.size() > 0 ? pos[0] : "data/satellites_20260801_1000Z.txt";
    const double duration = (pos.size() > 1 ? std::atof(pos[1].c_str()) : 24.0) * 3600.0;
    const double dt = pos.size() > 2 ? std::atof(pos[2].c_str()) : 10.0;
    const double out_every = pos.size() > 3 ? std::atof(pos[3].c_str()) : 0.0;
    std::vector<int> track_ids;
    if (pos.size() > 4) {
        std::stringstream ss(pos[4]);
        std::string tok;
        while (std::getline(ss, tok, ',')) track_ids.push_back(std::atoi(tok.c_str()));
    }

    int dropped = 0;
    const std::vector<CatalogObject> objs = load_catalog(path, &dropped);
    if (objs.empty()) {
        std::cerr << "no object loaded from " << path << "\n";
        return 1;
    }
    if (dropped) std::cerr << dropped << " malformed lines skipped\n";
    const double epoch = read_epoch_jd(path);
    const size_t n = objs.size();
    std::vector<double> states(6 * n), size_m(n), mass_kg(n);
    MassTable masses;
    if (std::filesystem::exists(masses_path)) {
        std::string err;
        if (!masses.load(masses_path, &err)) {
            std::cerr << "mass table: " << err << "\n";
            return 1;
        }
    } else if (breakup) {
        std::cout << masses_path << " absent: default masses\n";
    }
    for (size_t i = 0; i < n; ++i) {
        std::copy(objs[i].s, objs[i].s + 6, &states[6 * i]);
        size_m[i] = objs[i].size_m;
        mass_kg[i] = masses.mass_for(objs[i]);
    }
    int64_t impact_index = -1;
    if (impact_id >= 0) {
        for (size_t i = 0; i < n; ++i)
            if (objs[i].id == impact_id) impact_index = static_cast<int64_t>(i);
        if (impact_index < 0) {
            std::cerr << "--impact: no object " << impact_id << " in the catalogue\n";
            return 1;
        }
    }
    if (breakup && !conj_explicit) {
        // Only collisions matter: the threshold is the largest possible radius sum (src/main.cpp:251-260).
        double max_size = 0;
        for (double v : size_m) max_size = std::max(max_size, v);
        cfg.threshold_km = max_size * 1e-3 * cfg.radius_scale;
    }
    const long steps = static_cast<long>(std::ceil(duration / dt));
    long next_out = out_every > 0 ? static_cast<long>(out_every / dt) : 0;
    std::vector<size_t> tracked;
    for (size_t i = 0; i < n; ++i)
        if (std::find(track_ids.begin(), track_ids.end(), objs[i].id) != track_ids.end()) tracked.push_back(i);
    if (!track_ids.empty() && next_out == 0) next_out = std::max(1L, static_cast<long>(60.0 / dt));

    // Object names and ids, extended as fragments appear (src/core/breakup.cpp:295-303).
    std::vector<int> ids(n);
    std::vector<std::string> names(n);
    for (size_t i = 0; i < n; ++i) {
        ids[i] = objs[i].id;
        names[i] = objs[i].name;
    }

    try {
        kessler_b200::DeviceSimulation sim(device);
        std::cout << n << " objects, " << duration / 3600.0 << " h, dt " << dt << " s, " << steps << " steps on "
                  << sim.context().device_name() << (split ? " (split precision)" : " (FP64)") << "\n";
        sim.set_precision(split ? KS_PRECISION_SPLIT : KS_PRECISION_FP64);
        sim.set_steps_per_graph(spg);
        sim.set_clock(epoch, 0.0, dt);
        sim.set_screening(true, cfg);
        sim.set_population(states, size_m);
        if (breakup) {
            sim.set_masses(mass_kg);
            sim.set_breakup(true, lc_m, 40.0, seed);
        }

        std::filesystem::create_directories(out_dir);
        if (next_out > 0 && track_ids.empty()) {
            // Snapshots of an earlier run would mix with this one's (src/main.cpp:207-219).
            std::error_code ec;
            for (const auto& e : std::filesystem::directory_iterator(out_dir, ec)) {
                const std::string fn = e.path().filename().string();
                if (fn.rfind("snapshot_", 0) == 0 && e.path().extension() == ".csv") std::filesystem::remove(e.path(), ec);
            }
        }
        std::ofstream traj, moon_out;
        if (!track_ids.empty()) {
            traj.open(out_dir + "/trajectories.csv");
            traj << "t_s,id,name,x_km,y_km,z_km\n";
            moon_out.open(out_dir + "/moon.csv");
            moon_out << "t_s,x_km,y_km,z_km\n";
        }
        std::vector<double> snap_states;
        std::vector<uint8_t> snap_alive;
        long snap_index = 0;
        // Positions of the tracked objects and of the Moon (src/main.cpp:222-233).
        auto record = [&](double t, const std::vector<double>& st) {
            for (size_t i : tracked)
                traj << t << ',' << ids[i] << ',' << names[i] << ',' << st[6 * i] << ',' << st[6 * i + 1] << ','
                     << st[6 * i + 2] << '\n';
            double m[3];
            ks_moon_position(epoch + t / 86400.0, m);
            moon_out << t << ',' << m[0] << ',' << m[1] << ',' << m[2] << '\n';
        };
        auto write_states = [&](const std::string& file, double t, const std::vector<double>& st,
                                const std::vector<uint8_t>& al) {
            std::ofstream snap(file);
            snap << "# t = " << t << " s apres l'epoch\nid,x_km,y_km,z_km,vx,vy,vz,alive\n";
            snap.precision(9);
            for (size_t i = 0; i < al.size(); ++i) {
                snap << ids[i];
                for (int q = 0; q < 6; ++q) snap << ',' << st[6 * i + q];
                snap << ',' << (al[i] ? 1 : 0) << '\n';
            }
        };
        if (!tracked.empty()) record(0.0, states);
        std::ofstream conj_out(out_dir + "/conjunctions.csv");
        conj_out << "t_s,id1,id2,name1,name2,miss_km,v_rel_km_s,collision\n";
        conj_out << std::setprecision(10);
        std::ofstream breakup_out, pop_out;
        long long n_breakups = 0, n_catastrophic = 0, n_fragments = 0;
        if (breakup) {
            breakup_out.open(out_dir + "/breakups.csv");
            breakup_out << "t_s,event,target_id,target_name,projectile_id,projectile_name,"
                           "catastrophic,v_rel_km_s,energy_j_per_g,target_mass_kg,"
                           "projectile_mass_kg,sbm_mass_kg,expected_fragments,fragments,"
                           "fragments_mass_kg,escaped\n";
            breakup_out << std::setprecision(8);
            pop_out.open(out_dir + "/population.csv");
            pop_out << "t_s,t_days,alive,alive_catalog,alive_fragments,breakups,catastrophic,fragments_created\n";
        }
        auto take_events = [&]() {
            for (const ks_breakup_event& ev : sim.take_breakups()) {
                for (int k = 0; k < ev.fragments; ++k) {
                    ids.push_back(kFragmentIdBase + static_cast<int>(ids.size() - n));
                    names.push_back("FRAG " + std::to_string(ev.id) + "-" + std::to_string(k));
                }
                auto id_of = [&](int64_t idx) { return idx >= 0 ? std::to_string(ids[idx]) : std::string(); };
                auto name_of = [&](int64_t idx) { return idx >= 0 ? names[idx] : std::string("PROJECTILE"); };
                breakup_out << ev.t << ',' << ev.id << ',' << id_of(ev.target) << ',' << csv_quote(name_of(ev.target))
                            << ',' << id_of(ev.projectile) << ',' << csv_quote(name_of(ev.projectile)) << ','
                            << ev.catastrophic << ',' << ev.v_rel_km_s << ',' << ev.energy_j_per_g << ','
                            << ev.target_mass_kg << ',' << ev.projectile_mass_kg << ',' << ev.sbm_mass_kg << ','
                            << ev.expected_fragments << ',' << ev.fragments << ',' << ev.fragments_mass_kg << ','
                            << ev.escaped << '\n';
                ++n_breakups;
                n_catastrophic += ev.catastrophic ? 1 : 0;
                n_fragments += ev.fragments;
            }
        };
        auto log_population = [&]() {
            std::vector<double> fs;
            std::vector<uint8_t> fa;
            sim.get_population(fs, fa);
            const std::vector<int32_t> ev = sim.events_of_objects();
            long alive = 0, alive_frag = 0;
            for (size_t i = 0; i < fa.size(); ++i)
                if (fa[i]) {
                    ++alive;
                    alive_frag += ev[i] >= 0 ? 1 : 0;
                }
            const double t = sim.time();
            pop_out << t << ',' << t / 86400.0 << ',' << alive << ',' << alive - alive_frag << ',' << alive_frag << ','
                    << n_breakups << ',' << n_catastrophic << ',' << n_fragments << std::endl;
        };

        long long n_conj = 0, n_coll = 0, candidates = 0, below[4] = {0, 0, 0, 0};
        const double bins[4] = {0.1, 1.0, 2.0, 5.0};
        double closest = 1e30;
        int64_t ci = -1, cj = -1;
        double tc = 0;
        if (breakup) log_population();

        // Segments end where the host acts between steps: the forced impact
        // (at the first step starting at or after its time) and, with
        // fragmentation, each hour boundary (population log). The clock is
        // stepped exactly as Simulation::step steps it (t += dt).
        std::vector<double> t_before(static_cast<size_t>(steps) + 1);
        t_before[0] = 0.0;
        for (long k = 0; k < steps; ++k) t_before[static_cast<size_t>(k) + 1] = t_before[static_cast<size_t>(k)] + dt;
        long impact_step = -1;
        if (impact_index >= 0)
            for (long k = 0; k < steps; ++k)
                if (t_before[static_cast<size_t>(k)] >= impact_at_h * 3600.0) {
                    impact_step = k;
                    break;
                }
        const auto t0 = std::chrono::steady_clock::now();
        const long chunk = std::max<long>(spg, 1) * 32;
        long last_hour = 0;
        for (long done = 0; done < steps;) {
            if (done == impact_step) {
                sim.impact(impact_index, impact_mass, impact_vrel);
                take_events();
            }
            long k = std::min(chunk, steps - done);
            if (impact_step > done) k = std::min(k, impact_step - done);
            if (breakup)
                for (long q = done + 1; q <= done + k; ++q)
                    if (static_cast<long>(t_before[static_cast<size_t>(q)] / 3600.0) > last_hour) {
                        k = q - done;
                        break;
                    }
            if (next_out > 0) k = std::min(k, next_out - done % next_out);
            sim.advance(k);
            done += k;
            take_events();
            for (const ks_conjunction& c : sim.take_conjunctions()) {
                conj_out << c.t << ',' << ids[c.i] << ',' << ids[c.j] << ',' << csv_quote(names[c.i]) << ','
                         << csv_quote(names[c.j]) << ',' << c.miss_km << ',' << c.v_rel_km_s << ','
                         << (c.collision ? 1 : 0) << '\n';
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
            if (breakup && static_cast<long>(t_before[static_cast<size_t>(done)] / 3600.0) > last_hour) {
                last_hour = static_cast<long>(t_before[static_cast<size_t>(done)] / 3600.0);
                log_population();
            }
            if (next_out > 0 && done % next_out == 0) {
                sim.get_population(snap_states, snap_alive);
                if (!tracked.empty()) record(sim.time(), snap_states);
                else
                    write_states(out_dir + "/snapshot_" + std::to_string(snap_index++) + ".csv", sim.time(),
                                 snap_states, snap_alive);
            }
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

        std::vector<double> fs;
        std::vector<uint8_t> fa;
        sim.get_population(fs, fa);
        write_states(out_dir + "/final_state.csv", sim.time(), fs, fa);

        std::cout << "conjunctions below " << cfg.threshold_km << " km: " << n_conj << " (collisions " << n_coll
                  << ")\n";
        for (int q = 0; q < 4; ++q)
            if (bins[q] <= cfg.threshold_km) std::cout << "  below " << bins[q] << " km: " << below[q] << "\n";
        if (ci >= 0)
            std::cout << "closest: " << closest * 1000.0 << " m between " << names[ci] << " (" << ids[ci] << ") and "
                      << names[cj] << " (" << ids[cj] << ") at t = " << tc / 3600.0 << " h\n";
        if (breakup)
            std::cout << "breakups: " << n_breakups << " (" << n_catastrophic << " catastrophic), fragments created "
                      << n_fragments << "\n";
        std::cout << "candidate pairs per step: " << candidates / std::max(1L, steps) << "\n";
        std::cout << "wall " << wall << " s, " << static_cast<double>(n) * steps / wall << " object-steps/s\n";
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 2;
    }
    return 0;
}
