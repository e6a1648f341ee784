// The whole `rrgsim <work_dir>` run: params.json -> ICs -> integration -> dump/ and data/.
//
// Mirrors main() (solver/app/src/rrgsim.cu:12-62) and integrate()
// (solver/app/src/rrgsim_integration.cu:19-146): the same output tree, the same save cadence
// (a save when the accumulated time reaches next_save), the same snapshot format and the same
// CSV tables (solver/app/src/rrgsim_conservation.cu). Steps between two saves run as one fused,
// graph-replayed call.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <set>
#include <string>
#include <vector>

#include "host_io.h"
#include "rrg.h"

namespace fs = std::filesystem;

namespace {

// Plain logger: <work>/logs/rrgsim_<timestamp>.log plus stderr for info and above.
struct Log {
    FILE* f = nullptr;
    bool quiet = false;
    void open(const fs::path& dir) {
        std::error_code ec;
        fs::create_directories(dir, ec);
        char ts[64];
        std::time_t t = std::time(nullptr);
        std::strftime(ts, sizeof(ts), "%Y-%m-%d_%H-%M-%S", std::localtime(&t));
        f = std::fopen((dir / (std::string("rrgsim_") + ts + ".log")).c_str(), "ab");
        quiet = std::getenv("RRGSIM_QUIET") != nullptr;
    }
    void write(const char* level, const char* fmt, va_list ap) {
        char buf[2048];
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        if (f) {
            std::fprintf(f, "[%s] %s\n", level, buf);
            std::fflush(f);
        }
        if (!quiet && level[0] != 'd') std::fprintf(stderr, "[%s] %s\n", level, buf);
    }
    ~Log() {
        if (f) std::fclose(f);
    }
};
Log g_log;

void log_info(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    g_log.write("info", fmt, ap);
    va_end(ap);
}
void log_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    g_log.write("error", fmt, ap);
    va_end(ap);
}

// IOHandler::append_table (solver/lib/rrgsim_io/src/io_handler.cpp:71-105): a header line of
// tags joined by ", " when the table is first written in this run, then one row of values in
// fixed notation with the given precision.
struct Table {
    const char* tag;
    double value;
    int precision;
};

struct CsvWriter {
    fs::path data_dir;
    std::set<std::string> filled;
    bool keep_existing = false;  // a resumed run appends to the tables its first part wrote
    void append(const std::string& tag, const std::vector<Table>& items,
                const std::string& subdir = std::string()) {
        fs::path dir = subdir.empty() ? data_dir : data_dir / subdir;
        std::error_code ec;
        fs::create_directories(dir, ec);
        const fs::path path = dir / (tag + ".csv");
        const bool first = filled.insert(tag).second && !(keep_existing && fs::exists(path));
        FILE* f = std::fopen(path.c_str(), first ? "wb" : "ab");
        if (!f) throw std::runtime_error("cannot write " + path.string());
        if (first) {
            for (size_t i = 0; i < items.size(); ++i)
                std::fprintf(f, i + 1 < items.size() ? "%s, " : "%s\n", items[i].tag);
        }
        for (size_t i = 0; i < items.size(); ++i)
            std::fprintf(f, i + 1 < items.size() ? "%.*f, " : "%.*f\n", items[i].precision,
                         items[i].value);
        std::fclose(f);
    }
};

double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// print_conservation(info0, info): rrgsim_conservation.cu:9-98, 263-278
void save_conservation(CsvWriter& csv, const rrg_conservation& c0, const rrg_conservation& c) {
    const int p20 = 20, p15 = 15;
    const double ang_z_rel = c.angular[2] / c0.angular[2] - 1.;
    csv.append("delta_ang_z", {{"t", c.time, 8},
                               {"ang_z", c.angular[2], p20},
                               {"ang_z_rel_signed", ang_z_rel, p20},
                               {"ang_z_rel", std::fabs(ang_z_rel), p20}});
    const double an = norm3(c.angular), an0 = norm3(c0.angular);
    const double an_rel = an / an0 - 1.;
    csv.append("delta_ang_norm", {{"t", c.time, 8},
                                  {"ang_norm", an, p20},
                                  {"ang_norm_rel_signed", an_rel, p20},
                                  {"ang_norm_rel", std::fabs(an_rel), p20}});
    const double pn = norm3(c.momentum), pn0 = norm3(c0.momentum);
    const double p_rel = pn / pn0 - 1.;
    csv.append("delta_momentum", {{"t", c.time, p20},
                                  {"momentum_norm", pn, p20},
                                  {"momentum_diff", pn - pn0, p20},
                                  {"momentum_rel_signed", p_rel, p20},
                                  {"momentum_rel", std::fabs(p_rel), p20}});
    const double E = c.Ek + c.Ep, E0 = c0.Ek + c0.Ep;
    const double E_rel = E / E0 - 1.;
    csv.append("delta_energy", {{"t", c.time, 8},
                                {"E", E, p15},
                                {"E_rel_signed", E_rel, p15},
                                {"E_rel", std::fabs(E_rel), p15},
                                {"Ek", c.Ek, p15},
                                {"Ep", c.Ep, p15}});
    log_info("conservation t=%.6f E=%.15f (rel %.3e) |P|=%.15f |L|=%.15f", c.time, E, E_rel, pn,
             an);
}

// print_sample_particle: rrgsim_conservation.cu:334-359
void save_sample(CsvWriter& csv, const std::vector<double>& pos, const std::vector<double>& vel,
                 const std::vector<double>& acc, const std::vector<double>& grav) {
    if (pos.empty()) return;
    csv.append("sample_particle", {{"i", 0, 8},
                                   {"x", pos[0], 8},
                                   {"y", pos[1], 8},
                                   {"z", pos[2], 8},
                                   {"vx", vel[0], 8},
                                   {"vy", vel[1], 8},
                                   {"vz", vel[2], 8},
                                   {"grav", grav[0], 8},
                                   {"ax", acc[0], 8},
                                   {"ay", acc[1], 8},
                                   {"az", acc[2], 8}});
}

// print_{acc,grav,mass}_projection: rrgsim_conservation.cu:360-424
void save_grid_profiles(CsvWriter& csv, rrg_ctx* ctx, const rrg_grid_info& g, double time) {
    const size_t NX = static_cast<size_t>(g.nx);
    const size_t nc = NX * NX * NX;
    std::vector<double> mass(nc), grav(nc), acc(3 * nc);
    if (rrg_get_grid(ctx, mass.data(), grav.data(), acc.data()) != RRG_OK)
        throw std::runtime_error(rrg_last_error(ctx));
    auto AT = [&](size_t x, size_t y, size_t z) { return x + y * NX + z * NX * NX; };
    char name[128];
    std::snprintf(name, sizeof(name), "a_grid_center_%.08f", time);
    for (size_t xi = 0; xi < NX; ++xi) {
        const size_t c = AT(xi, NX / 2, NX / 2);
        csv.append(name, {{"x", g.domain_min + g.dx * xi, 8},
                          {"ax", acc[3 * c], 8},
                          {"ay", acc[3 * c + 1], 8},
                          {"az", acc[3 * c + 2], 8}},
                   "a_grid");
    }
    std::snprintf(name, sizeof(name), "grav_axis_center_%.10f", time);
    for (size_t i = 0; i < NX; ++i)
        csv.append(name, {{"r", g.domain_min + g.dx * i, 8},
                          {"gx", grav[AT(i, NX / 2, NX / 2)], 8},
                          {"gy", grav[AT(NX / 2, i, NX / 2)], 8},
                          {"gz", grav[AT(NX / 2, NX / 2, i)], 8}},
                   "grav_grid");
    std::snprintf(name, sizeof(name), "mass_axis_center_%.10f", time);
    for (size_t i = 0; i < NX; ++i)
        csv.append(name, {{"r", g.domain_min + g.dx * i, 8},
                          {"mx", mass[AT(i, NX / 2, NX / 2)], 8},
                          {"my", mass[AT(NX / 2, i, NX / 2)], 8},
                          {"mz", mass[AT(NX / 2, NX / 2, i)], 8}},
                   "mass_grid");
}

// check_bounds: rrgsim_conservation.cu:280-332 (logged, not fatal)
void check_bounds(const std::vector<double>& pos, const rrg_grid_info& g) {
    if (pos.empty()) return;
    double lo[3] = {pos[0], pos[1], pos[2]}, hi[3] = {pos[0], pos[1], pos[2]};
    for (size_t i = 0; i < pos.size() / 3; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], pos[3 * i + k]);
            hi[k] = std::max(hi[k], pos[3 * i + k]);
        }
    const char* ax = "XYZ";
    for (int k = 0; k < 3; ++k) {
        if (lo[k] < g.domain_min)
            log_error("%c min bounds violation! Particle %c: %g; domain_min: %g", ax[k], ax[k],
                      lo[k], g.domain_min);
        if (hi[k] > g.domain_max)
            log_error("%c max bounds violation! Particle %c: %g; domain_max: %g", ax[k], ax[k],
                      hi[k], g.domain_max);
    }
}

// The reference opens the IC path as given (relative to the process directory) and the sample
// writes it Windows-style ("ini\\S.txt"). Here '\' becomes '/', and a relative path is tried
// against the work directory first, then the process directory.
std::string resolve_ic(const fs::path& work, const std::string& raw) {
    std::string p = raw;
    for (char& ch : p)
        if (ch == '\\') ch = '/';
    fs::path fp(p);
    if (fp.is_absolute()) return fp.string();
    if (fs::exists(work / fp)) return (work / fp).string();
    return fp.string();
}

struct CtxGuard {
    rrg_ctx* c = nullptr;
    ~CtxGuard() {
        if (c) rrg_destroy(c);
    }
};

#define RUN_CHECK(call)                                                                       \
    do {                                                                                      \
        const rrg_status s_ = (call);                                                         \
        if (s_ != RRG_OK) {                                                                   \
            log_error("%s failed: %s", #call, rrg_last_error(guard.c));                       \
            rrg::set_thread_error(std::string(#call) + ": " + rrg_last_error(guard.c));       \
            return s_;                                                                        \
        }                                                                                     \
    } while (0)

// The base conservation of a run (its t = 0 state) beside the dumps, so that a resumed run
// reports the same relative drifts: 9 float64 (time, Ek, Ep, P[3], L[3]).
bool write_base(const fs::path& dump_dir, const rrg_conservation& c) {
    FILE* f = std::fopen((dump_dir / "C0.bin").c_str(), "wb");
    if (!f) return false;
    const double v[9] = {c.time, c.Ek, c.Ep, c.momentum[0], c.momentum[1], c.momentum[2],
                         c.angular[0], c.angular[1], c.angular[2]};
    const bool ok = std::fwrite(v, 8, 9, f) == 9;
    return (std::fclose(f) == 0) && ok;
}

bool read_base(const fs::path& dump_dir, rrg_conservation& c) {
    FILE* f = std::fopen((dump_dir / "C0.bin").c_str(), "rb");
    if (!f) return false;
    double v[9];
    const bool ok = std::fread(v, 8, 9, f) == 9;
    std::fclose(f);
    if (!ok) return false;
    c.time = v[0];
    c.Ek = v[1];
    c.Ep = v[2];
    for (int k = 0; k < 3; ++k) {
        c.momentum[k] = v[3 + k];
        c.angular[k] = v[6 + k];
    }
    return true;
}

rrg_status run_impl(const char* work_dir, int device, int precision, bool resume,
                    uint64_t resume_iter) {
    if (!work_dir) return RRG_ERR_INVALID;
    const fs::path work(work_dir);
    g_log.open(work / "logs");
    CsvWriter csv;
    csv.data_dir = work / "data";
    csv.keep_existing = resume;
    if (!resume) {
        std::error_code ec;
        fs::remove_all(csv.data_dir, ec);  // IOHandler::setup wipes data/ (io_handler.cpp:14)
    }
    const fs::path dump_dir = work / "dump";
    auto dump_name = [&](const char* prefix, uint64_t it) {
        char name[64];
        std::snprintf(name, sizeof(name), "%s_%5llu.bin", prefix,
                      static_cast<unsigned long long>(it));
        return (dump_dir / name).string();
    };
    CtxGuard guard;
    try {
        rrg_parsed_params pp;
        const std::string params_path = (work / "params.json").string();
        if (rrg_parse_params_json(params_path.c_str(), &pp) != RRG_OK) {
            log_error("Error: %s", rrg_last_error(nullptr));
            return RRG_ERR_IO;
        }
        log_info("Params json parsed successfully (%s wave model)",
                 pp.sim.use_wave_model ? "use" : "don't use");

        // read_simple_particles_data: star component then dark component
        struct Comp {
            const char* file;
            double mass, soft;
        } comps[2] = {{pp.ini.ini_file_star, pp.ini.mass_star, pp.ini.soft_star},
                      {pp.ini.ini_file_dark, pp.ini.mass_dark, pp.ini.soft_dark}};
        int64_t total = 0;
        std::string paths[2];
        for (int k = 0; k < 2; ++k) {
            if (!comps[k].file[0]) continue;
            paths[k] = resolve_ic(work, comps[k].file);
            int64_t nh = 0;
            if (rrg_ic_header_count(paths[k].c_str(), &nh) != RRG_OK) {
                log_error("Error: %s", rrg_last_error(nullptr));
                return RRG_ERR_IO;
            }
            total += nh;
        }
        if (total <= 0) {
            log_error("Error: no particles (no IC file given)");
            rrg::set_thread_error("no particles (no IC file given)");
            return RRG_ERR_INVALID;
        }
        std::vector<double> pos(3 * total), vel(3 * total), mass(total), soft2(total);
        int64_t have = 0;
        for (int k = 0; k < 2; ++k) {
            if (paths[k].empty()) continue;
            int64_t got = 0;
            if (rrg_read_ic_component(paths[k].c_str(), comps[k].mass, comps[k].soft, have, total,
                                      pos.data(), vel.data(), mass.data(), soft2.data(),
                                      &got) != RRG_OK) {
                log_error("Error: %s", rrg_last_error(nullptr));
                return RRG_ERR_IO;
            }
            have += got;
        }
        log_info("%lld particles loaded", static_cast<long long>(have));

        double time0 = 0.0;
        if (resume) {
            // read_particles_dump (io_particles_bin.cu:39-77): positions, velocities and time;
            // masses and softening stay those of the ICs
            const std::string sp = dump_name("S", resume_iter);
            int64_t nd = 0;
            if (rrg_read_dump(sp.c_str(), have, &nd, &time0, pos.data(), vel.data()) != RRG_OK) {
                log_error("Error: %s", rrg_last_error(nullptr));
                return RRG_ERR_IO;
            }
            if (nd != have) {
                log_error("Error: %s holds %lld particles, the ICs %lld", sp.c_str(),
                          static_cast<long long>(nd), static_cast<long long>(have));
                rrg::set_thread_error("dump and ICs differ in particle count");
                return RRG_ERR_INVALID;
            }
            log_info("resuming from %s (t = %.10f)", sp.c_str(), time0);
        }

        RUN_CHECK(rrg_create(device, precision, &guard.c));
        RUN_CHECK(rrg_load_particles(guard.c, have, pos.data(), vel.data(), mass.data(),
                                     soft2.data()));
        if (pp.has_grid) {
            RUN_CHECK(rrg_init_grid(guard.c, &pp.grid));
            check_bounds(pos, pp.grid);
        }
        if (pp.has_wave) RUN_CHECK(rrg_set_wave_params(guard.c, &pp.wave));
        RUN_CHECK(rrg_solver_init(guard.c, &pp.sim));
        const bool wave = pp.sim.use_wave_model != 0;
        const size_t ncells =
            pp.has_grid ? static_cast<size_t>(pp.grid.nx) * pp.grid.nx * pp.grid.nx : 0;
        if (resume) {
            if (wave) {
                std::vector<double> cur(ncells), prev(ncells);
                const std::string wp = dump_name("W", resume_iter);
                if (rrg_read_wave_state(wp.c_str(), pp.grid.nx, nullptr, cur.data(),
                                        prev.data()) != RRG_OK) {
                    log_error("Error: %s", rrg_last_error(nullptr));
                    return RRG_ERR_IO;
                }
                RUN_CHECK(rrg_set_wave_state(guard.c, cur.data(), prev.data()));
            }
            RUN_CHECK(rrg_solver_resume(guard.c));
        } else {
            RUN_CHECK(rrg_solver_precalc(guard.c));
        }
        RUN_CHECK(rrg_solver_sync(guard.c));

        {
            std::error_code ec;
            fs::create_directories(dump_dir, ec);
        }
        const int64_t n = have;
        std::vector<double> acc(3 * n), grav(n);
        rrg_conservation c0;
        RUN_CHECK(rrg_get_particles(guard.c, pos.data(), vel.data(), acc.data(), grav.data()));
        if (resume && read_base(dump_dir, c0)) {
            log_info("base conservation from C0.bin: Ek=%.15f Ep=%.15f", c0.Ek, c0.Ep);
        } else {
            RUN_CHECK(rrg_calc_conservation(guard.c, &c0));
            c0.time = time0;
            log_info("base conservation: Ek=%.15f Ep=%.15f", c0.Ek, c0.Ep);
            if (!write_base(dump_dir, c0)) log_error("cannot write %s/C0.bin", dump_dir.c_str());
        }
        if (!resume) {
            save_sample(csv, pos, vel, acc, grav);
            if (pp.has_grid) save_grid_profiles(csv, guard.c, pp.grid, 0.0);
        }

        const double dt = pp.sim.dt_dynamics;
        uint64_t iteration = resume ? resume_iter : 0;
        double time = time0;
        // the save cadence up to `time`, accumulated as the first part of the run did (one
        // save, and one dt_save increment, per save interval)
        double next_save = 0.0 + pp.sim.dt_save;
        uint64_t saves_without_dump = 0;
        while (resume && time >= next_save && pp.sim.dt_save > 0) {
            next_save += pp.sim.dt_save;
            ++saves_without_dump;
        }
        std::vector<double> wcur(wave ? ncells : 0), wprev(wave ? ncells : 0);
        while (time < pp.sim.time_max) {
            // steps until the next save or the end, accumulated exactly as the reference does
            int k = 0;
            double t = time;
            do {
                ++k;
                t += dt;
            } while (t < next_save && t < pp.sim.time_max && k < (1 << 20));
            RUN_CHECK(rrg_solver_calc_steps(guard.c, k));
            iteration += static_cast<uint64_t>(k);
            time = t;
            if (time >= next_save) {
                log_info("Simulation time: %.5f / %.5f (iter: %llu)", time, pp.sim.time_max,
                         static_cast<unsigned long long>(iteration));
                RUN_CHECK(rrg_solver_sync(guard.c));
                RUN_CHECK(rrg_get_particles(guard.c, pos.data(), vel.data(), acc.data(),
                                            grav.data()));
                rrg_conservation c;
                RUN_CHECK(rrg_calc_conservation(guard.c, &c));
                c.time = time;
                save_sample(csv, pos, vel, acc, grav);
                save_conservation(csv, c0, c);
                if (pp.has_grid) {
                    check_bounds(pos, pp.grid);
                    save_grid_profiles(csv, guard.c, pp.grid, time);
                }
                next_save += pp.sim.dt_save;
                ++saves_without_dump;
                if (saves_without_dump < pp.sim.saves_without_dump) {
                    if (rrg_write_dump(dump_dir.c_str(), iteration, time, n, pos.data(),
                                       vel.data()) != RRG_OK)
                        log_error("%s", rrg_last_error(nullptr));
                    if (wave) {
                        // the wave levels beside the snapshot, for an exact resume
                        RUN_CHECK(rrg_get_wave_state(guard.c, wcur.data(), wprev.data()));
                        if (rrg_write_wave_state(dump_dir.c_str(), iteration, time, pp.grid.nx,
                                                 wcur.data(), wprev.data()) != RRG_OK)
                            log_error("%s", rrg_last_error(nullptr));
                    }
                }
            }
        }
        log_info("integration completed (%llu iterations)",
                 static_cast<unsigned long long>(iteration));
    } catch (const std::exception& e) {
        log_error("Exception: %s", e.what());
        rrg::set_thread_error(e.what());
        return RRG_ERR_IO;
    }
    return RRG_OK;
}

}  // namespace

extern "C" RRG_API rrg_status rrg_run(const char* work_dir, int device, int precision) {
    return run_impl(work_dir, device, precision, false, 0);
}

extern "C" RRG_API rrg_status rrg_run_resume(const char* work_dir, uint64_t iteration,
                                             int device, int precision) {
    return run_impl(work_dir, device, precision, true, iteration);
}
