// Host I/O of the rrgsim boundary: params.json, IC text files, snapshot dumps, and the
// synthetic initial-condition generators. No GPU code here.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "host_io.h"
#include "rrg.h"

namespace rrg {

static thread_local std::string t_io_error;
const char* io_error() { return t_io_error.c_str(); }
static rrg_status io_fail(rrg_status s, const std::string& m) {
    t_io_error = m;
    set_thread_error(m);
    return s;
}

// ---------------------------------------------------------------------------------------------
// Minimal JSON reader (objects, arrays, strings, numbers, true/false/null).
// ---------------------------------------------------------------------------------------------
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;
    const Json* find(const std::string& k) const {
        for (auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

namespace {

struct JsonParser {
    const std::string& s;
    size_t i = 0;
    explicit JsonParser(const std::string& src) : s(src) {}
    [[noreturn]] void fail(const std::string& what) {
        throw std::runtime_error("JSON parse error at offset " + std::to_string(i) + ": " + what);
    }
    void ws() {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
    }
    bool lit(const char* w) {
        const size_t n = std::strlen(w);
        if (s.compare(i, n, w) == 0) {
            i += n;
            return true;
        }
        return false;
    }
    Json value() {
        ws();
        if (i >= s.size()) fail("unexpected end");
        Json v;
        const char c = s[i];
        if (c == '{') {
            v.kind = Json::Object;
            ++i;
            ws();
            if (i < s.size() && s[i] == '}') {
                ++i;
                return v;
            }
            for (;;) {
                ws();
                if (i >= s.size() || s[i] != '"') fail("expected key");
                std::string k = string();
                ws();
                if (i >= s.size() || s[i] != ':') fail("expected ':'");
                ++i;
                v.obj.emplace_back(k, value());
                ws();
                if (i < s.size() && s[i] == ',') {
                    ++i;
                    continue;
                }
                if (i < s.size() && s[i] == '}') {
                    ++i;
                    break;
                }
                fail("expected ',' or '}'");
            }
        } else if (c == '[') {
            v.kind = Json::Array;
            ++i;
            ws();
            if (i < s.size() && s[i] == ']') {
                ++i;
                return v;
            }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (i < s.size() && s[i] == ',') {
                    ++i;
                    continue;
                }
                if (i < s.size() && s[i] == ']') {
                    ++i;
                    break;
                }
                fail("expected ',' or ']'");
            }
        } else if (c == '"') {
            v.kind = Json::String;
            v.str = string();
        } else if (lit("true")) {
            v.kind = Json::Bool;
            v.b = true;
        } else if (lit("false")) {
            v.kind = Json::Bool;
            v.b = false;
        } else if (lit("null")) {
            v.kind = Json::Null;
        } else {
            const char* b = s.c_str() + i;
            char* e = nullptr;
            errno = 0;
            const double d = std::strtod(b, &e);
            if (e == b) fail("unexpected character");
            v.kind = Json::Number;
            v.num = d;
            i += static_cast<size_t>(e - b);
        }
        return v;
    }
    std::string string() {
        std::string out;
        ++i;  // opening quote
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\') {
                if (i >= s.size()) fail("bad escape");
                const char e = s[i++];
                switch (e) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        if (i + 4 > s.size()) fail("bad \\u escape");
                        const unsigned cp = std::stoul(s.substr(i, 4), nullptr, 16);
                        i += 4;
                        if (cp < 0x80) out += static_cast<char>(cp);
                        else if (cp < 0x800) {
                            out += static_cast<char>(0xC0 | (cp >> 6));
                            out += static_cast<char>(0x80 | (cp & 0x3F));
                        } else {
                            out += static_cast<char>(0xE0 | (cp >> 12));
                            out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
                            out += static_cast<char>(0x80 | (cp & 0x3F));
                        }
                        break;
                    }
                    default: fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        if (i >= s.size()) fail("unterminated string");
        ++i;
        return out;
    }
};

double need_num(const Json& o, const char* key, const char* section) {
    const Json* v = o.find(key);
    if (!v) throw std::runtime_error(std::string("missing key '") + key + "' in " + section);
    if (v->kind != Json::Number)
        throw std::runtime_error(std::string("key '") + key + "' in " + section +
                                 " must be a number");
    return v->num;
}

bool opt_num(const Json& o, const char* key, const char* section, double* out) {
    const Json* v = o.find(key);
    if (!v) return false;
    if (v->kind != Json::Number)
        throw std::runtime_error(std::string("key '") + key + "' in " + section +
                                 " must be a number");
    *out = v->num;
    return true;
}

void opt_path(const Json& o, const char* key, char* dst, size_t cap) {
    dst[0] = '\0';
    const Json* v = o.find(key);
    if (!v || v->kind == Json::Null) return;
    if (v->kind != Json::String)
        throw std::runtime_error(std::string("key '") + key + "' must be a string or null");
    if (v->str.size() + 1 > cap) throw std::runtime_error(std::string("path too long: ") + key);
    std::memcpy(dst, v->str.c_str(), v->str.size() + 1);
}

}  // namespace

Json parse_json_text(const std::string& text) {
    JsonParser p(text);
    Json v = p.value();
    p.ws();
    if (p.i != text.size()) p.fail("trailing characters");
    return v;
}

void grid_from_values(int nx, double dx, double bc_frac, rrg_grid_info* g) {
    // io_json.cpp:28-40
    g->nx = nx;
    g->dx = dx;
    g->domain_l = g->dx * g->nx;
    g->sim_l = (1. - bc_frac) * g->domain_l;
    g->bc_l = 0.5 * bc_frac * g->domain_l;
    g->domain_max = 0.5 * g->domain_l;
    g->domain_min = -0.5 * g->domain_l;
}

}  // namespace rrg

using namespace rrg;

extern "C" {

RRG_API rrg_status rrg_parse_params_json(const char* path, rrg_parsed_params* out) {
    if (!path || !out) return io_fail(RRG_ERR_INVALID, "rrg_parse_params_json: NULL argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return io_fail(RRG_ERR_IO, std::string("Expected params json: '") + path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    try {
        const Json j = parse_json_text(ss.str());
        if (j.kind != Json::Object) throw std::runtime_error("params json must be an object");
        std::memset(out, 0, sizeof(*out));
        // grid_params (optional), io_json.cpp:28-40
        if (const Json* g = j.find("grid_params")) {
            const double nx = need_num(*g, "nx", "grid_params");
            const double dx = need_num(*g, "dx", "grid_params");
            const double bc = need_num(*g, "bc_frac", "grid_params");
            grid_from_values(static_cast<int>(nx), dx, bc, &out->grid);
            out->has_grid = 1;
        }
        // sim_params (mandatory), io_json.cpp:13-21
        const Json* s = j.find("sim_params");
        if (!s) throw std::runtime_error("No sim_params section");
        out->sim.time_max = need_num(*s, "time_max", "sim_params");
        out->sim.dt_save = need_num(*s, "dt_save", "sim_params");
        out->sim.dt_dynamics = need_num(*s, "dt_dynamics", "sim_params");
        out->sim.saves_without_dump = UINT64_MAX;
        double swd;
        if (opt_num(*s, "saves_without_dump", "sim_params", &swd))
            out->sim.saves_without_dump = static_cast<uint64_t>(swd);
        // ini_params (mandatory), io_json.cpp:115-131
        const Json* ini = j.find("ini_params");
        if (!ini) throw std::runtime_error("No ini_params section");
        out->ini.mass_star = need_num(*ini, "mass_star", "ini_params");
        out->ini.mass_dark = need_num(*ini, "mass_dark", "ini_params");
        out->ini.soft_star = need_num(*ini, "soft_star", "ini_params");
        out->ini.soft_dark = need_num(*ini, "soft_dark", "ini_params");
        opt_path(*ini, "ini_file_star", out->ini.ini_file_star, sizeof(out->ini.ini_file_star));
        opt_path(*ini, "ini_file_dark", out->ini.ini_file_dark, sizeof(out->ini.ini_file_dark));
        // wave_params (optional), io_json.cpp:53-99, defaults as there
        if (const Json* w = j.find("wave_params")) {
            out->wave.diss_base = need_num(*w, "diss_base", "wave_params");
            out->wave.diss_extra = need_num(*w, "diss_extra", "wave_params");
            out->wave.wave_speed = need_num(*w, "wave_speed", "wave_params");
            double v;
            out->wave.setup_iterations =
                opt_num(*w, "setup_iterations", "wave_params", &v) ? static_cast<int>(v) : 30000;
            out->wave.iterations =
                opt_num(*w, "iterations", "wave_params", &v) ? static_cast<int>(v) : 3000;
            out->wave.tolerance = opt_num(*w, "tolerance", "wave_params", &v) ? v : 1.E-6;
            out->wave.print_step =
                opt_num(*w, "print_step", "wave_params", &v) ? static_cast<int>(v) : 500;
            out->wave.steady_check_step =
                opt_num(*w, "steady_check_step", "wave_params", &v) ? static_cast<int>(v) : 30;
            out->wave.steady_hold_steps =
                opt_num(*w, "steady_hold_steps", "wave_params", &v) ? static_cast<int>(v) : 3;
            out->has_wave = 1;
        }
        // validate_dependent_fields, io_json.cpp:170-186
        if (out->has_grid && out->has_wave) {
            out->sim.use_wave_model = 1;
            const double dx = out->grid.dx;
            const double c = out->wave.wave_speed;
            constexpr double DIM = 3;
            out->wave.dt = 0.5 * dx / (c * std::sqrt(DIM));
        }
    } catch (const std::exception& e) {
        return io_fail(RRG_ERR_IO, std::string("Params json parsing failed: ") + e.what());
    }
    return RRG_OK;
}

// Tokenising reader of the IC text format (header "N t", rows "x y z vx vy vz").
RRG_API rrg_status rrg_ic_header_count(const char* path, int64_t* n) {
    if (!path || !n) return io_fail(RRG_ERR_INVALID, "rrg_ic_header_count: NULL argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(RRG_ERR_IO, std::string("cannot open IC file '") + path + "'");
    double hn = 0, ht = 0;
    const int got = std::fscanf(f, "%lf %lf", &hn, &ht);
    std::fclose(f);
    if (got != 2 || !(hn >= 0) || hn != std::floor(hn))
        return io_fail(RRG_ERR_IO, std::string("Failed to read ini header in '") + path + "'");
    *n = static_cast<int64_t>(hn);
    return RRG_OK;
}

RRG_API rrg_status rrg_read_ic_component(const char* path, double component_mass,
                                         double component_soft, int64_t n_before,
                                         int64_t capacity, double* pos, double* vel,
                                         double* mass, double* soft2, int64_t* n_read) {
    if (!path || !pos || !vel || !mass || !soft2)
        return io_fail(RRG_ERR_INVALID, "rrg_read_ic_component: NULL argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return io_fail(RRG_ERR_IO, std::string("cannot open IC file '") + path + "'");
    std::string line;
    // header
    int64_t ini_n = -1;
    while (std::getline(f, line)) {
        const char* b = line.c_str();
        char* e = nullptr;
        const double hn = std::strtod(b, &e);
        if (e == b) {
            bool blank = true;
            for (char ch : line)
                if (!std::isspace(static_cast<unsigned char>(ch))) blank = false;
            if (blank) continue;
            return io_fail(RRG_ERR_IO, "Failed to read ini header");
        }
        if (!(hn >= 0) || hn != std::floor(hn)) return io_fail(RRG_ERR_IO, "Failed to read ini header");
        ini_n = static_cast<int64_t>(hn);
        break;
    }
    if (ini_n < 0) return io_fail(RRG_ERR_IO, "Failed to read ini header");
    const int64_t total = n_before + ini_n;
    if (total > capacity)
        return io_fail(RRG_ERR_INVALID, "IC arrays too small for the header's particle count");
    const double pm = component_mass / static_cast<double>(total);  // io_particles_csv.cpp:37
    const double ps = component_soft * component_soft;
    int64_t k = 0;
    while (std::getline(f, line)) {
        const char* b = line.c_str();
        double v[6];
        int got = 0;
        while (got < 6) {
            char* e = nullptr;
            const double d = std::strtod(b, &e);
            if (e == b) break;
            v[got++] = d;
            b = e;
        }
        if (got == 0) {
            bool blank = true;
            for (char ch : line)
                if (!std::isspace(static_cast<unsigned char>(ch))) blank = false;
            if (blank) continue;
        }
        if (got < 6) {
            return io_fail(RRG_ERR_IO, "IC row " + std::to_string(k + 1) +
                                           " has fewer than 6 numbers");
        }
        if (k >= ini_n) {
            k++;
            continue;  // counted for the mismatch message
        }
        const int64_t i = n_before + k;
        for (int a = 0; a < 3; ++a) {
            pos[3 * i + a] = v[a];
            vel[3 * i + a] = v[3 + a];
        }
        mass[i] = pm;
        soft2[i] = ps;
        ++k;
    }
    if (k != ini_n)
        return io_fail(RRG_ERR_IO, "Rows header/file mismatch (" + std::to_string(total) + "/" +
                                       std::to_string(n_before + k) + ")");
    if (n_read) *n_read = ini_n;
    return RRG_OK;
}

RRG_API rrg_status rrg_write_ic_text(const char* path, int64_t n, double t, const double* pos,
                                     const double* vel) {
    if (!path || n < 0 || (n > 0 && (!pos || !vel)))
        return io_fail(RRG_ERR_INVALID, "rrg_write_ic_text: bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(RRG_ERR_IO, std::string("cannot write '") + path + "'");
    std::fprintf(f, "%lld %.6f\n", static_cast<long long>(n), t);
    for (int64_t i = 0; i < n; ++i)
        std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", pos[3 * i], pos[3 * i + 1],
                     pos[3 * i + 2], vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    const bool ok = std::fclose(f) == 0;
    return ok ? RRG_OK : io_fail(RRG_ERR_IO, std::string("write failed: ") + path);
}

RRG_API rrg_status rrg_write_dump(const char* dump_dir, uint64_t iter, double time, int64_t n,
                                  const double* pos, const double* vel) {
    if (!dump_dir || n < 0 || (n > 0 && (!pos || !vel)))
        return io_fail(RRG_ERR_INVALID, "rrg_write_dump: bad argument");
    char name[64];
    std::snprintf(name, sizeof(name), "S_%5llu.bin", static_cast<unsigned long long>(iter));
    const std::string path = std::string(dump_dir) + "/" + name;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return io_fail(RRG_ERR_IO, "Can't write particles dump: cannot open " + path);
    const uint64_t N = static_cast<uint64_t>(n);
    bool ok = std::fwrite(&N, 8, 1, f) == 1 && std::fwrite(&time, 8, 1, f) == 1;
    if (n > 0) {
        ok = ok && std::fwrite(pos, 8, 3 * static_cast<size_t>(n), f) == 3 * static_cast<size_t>(n);
        ok = ok && std::fwrite(vel, 8, 3 * static_cast<size_t>(n), f) == 3 * static_cast<size_t>(n);
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RRG_OK : io_fail(RRG_ERR_IO, "Can't write particles dump: short write to " + path);
}

RRG_API rrg_status rrg_read_dump(const char* path, int64_t capacity, int64_t* n, double* time,
                                 double* pos, double* vel) {
    if (!path || !n) return io_fail(RRG_ERR_INVALID, "rrg_read_dump: NULL argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(RRG_ERR_IO, std::string("Can't read particles dump: ") + path);
    uint64_t N = 0;
    double t = 0;
    bool ok = std::fread(&N, 8, 1, f) == 1 && std::fread(&t, 8, 1, f) == 1;
    if (ok && pos && vel) {
        if (static_cast<int64_t>(N) > capacity) {
            std::fclose(f);
            return io_fail(RRG_ERR_INVALID, "rrg_read_dump: arrays too small");
        }
        ok = std::fread(pos, 8, 3 * N, f) == 3 * N && std::fread(vel, 8, 3 * N, f) == 3 * N;
    }
    std::fclose(f);
    if (!ok) return io_fail(RRG_ERR_IO, std::string("Can't read particles dump: truncated ") + path);
    *n = static_cast<int64_t>(N);
    if (time) *time = t;
    return RRG_OK;
}

// Wave state beside a snapshot: W_{iter:>5d}.bin = uint64 nx; float64 time;
// float64 phi_cur[nx^3]; float64 phi_prev[nx^3] (x fastest).
RRG_API rrg_status rrg_write_wave_state(const char* dump_dir, uint64_t iter, double time,
                                        int32_t nx, const double* phi_cur,
                                        const double* phi_prev) {
    if (!dump_dir || nx < 1 || !phi_cur || !phi_prev)
        return io_fail(RRG_ERR_INVALID, "rrg_write_wave_state: bad argument");
    char name[64];
    std::snprintf(name, sizeof(name), "W_%5llu.bin", static_cast<unsigned long long>(iter));
    const std::string path = std::string(dump_dir) + "/" + name;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return io_fail(RRG_ERR_IO, "Can't write wave state: cannot open " + path);
    const uint64_t N = static_cast<uint64_t>(nx);
    const size_t nc = static_cast<size_t>(nx) * nx * nx;
    bool ok = std::fwrite(&N, 8, 1, f) == 1 && std::fwrite(&time, 8, 1, f) == 1 &&
              std::fwrite(phi_cur, 8, nc, f) == nc && std::fwrite(phi_prev, 8, nc, f) == nc;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RRG_OK : io_fail(RRG_ERR_IO, "Can't write wave state: short write to " + path);
}

RRG_API rrg_status rrg_read_wave_state(const char* path, int32_t nx, double* time,
                                       double* phi_cur, double* phi_prev) {
    if (!path || nx < 1 || !phi_cur || !phi_prev)
        return io_fail(RRG_ERR_INVALID, "rrg_read_wave_state: bad argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(RRG_ERR_IO, std::string("Can't read wave state: ") + path);
    uint64_t N = 0;
    double t = 0;
    bool ok = std::fread(&N, 8, 1, f) == 1 && std::fread(&t, 8, 1, f) == 1;
    if (ok && N != static_cast<uint64_t>(nx)) {
        std::fclose(f);
        return io_fail(RRG_ERR_INVALID, std::string("wave state grid size differs: ") + path);
    }
    const size_t nc = static_cast<size_t>(nx) * nx * nx;
    ok = ok && std::fread(phi_cur, 8, nc, f) == nc && std::fread(phi_prev, 8, nc, f) == nc;
    std::fclose(f);
    if (!ok) return io_fail(RRG_ERR_IO, std::string("Can't read wave state: truncated ") + path);
    if (time) *time = t;
    return RRG_OK;
}

}  // extern "C"

// ================================================================================================
// Synthetic initial conditions
// ================================================================================================
namespace {

// xoshiro256** seeded through SplitMix64 (Blackman & Vigna).
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (auto& v : s) {
            z += 0x9e3779b97f4a7c15ULL;
            uint64_t x = z;
            x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
            x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
            v = x ^ (x >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }   // [0, 1)
    double uniform_open() { return (static_cast<double>(next() >> 11) + 0.5) * 0x1.0p-53; }
    double normal() {
        const double u1 = uniform_open(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
    void iso(double r, double* out) {
        const double cz = 2.0 * uniform() - 1.0;
        const double ph = 2.0 * M_PI * uniform();
        const double sz = std::sqrt(std::max(0.0, 1.0 - cz * cz));
        out[0] = r * sz * std::cos(ph);
        out[1] = r * sz * std::sin(ph);
        out[2] = r * cz;
    }
};

// Enclosed mass of an exponential disk in the spherical approximation: M (1 - (1 + x) e^-x).
double disk_menc(double M, double Rd, double R) {
    const double x = R / Rd;
    return M * (1.0 - (1.0 + x) * std::exp(-x));
}

}  // namespace

extern "C" {

RRG_API rrg_status rrg_generate_plummer(uint64_t seed, int64_t n, double total_mass,
                                        double scale_radius, double r_max, double* pos,
                                        double* vel) {
    if (n < 0 || (n > 0 && (!pos || !vel)) || !(scale_radius > 0) || !(total_mass >= 0) ||
        !(r_max > 0))
        return io_fail(RRG_ERR_INVALID, "rrg_generate_plummer: bad argument");
    Rng rng(seed);
    const double a = scale_radius, G = 1.0;
    for (int64_t i = 0; i < n; ++i) {
        double r;
        do {  // Aarseth, Henon & Wielen (1974): M(<r)/M = X -> r = a / sqrt(X^-2/3 - 1)
            const double X = rng.uniform_open();
            r = a / std::sqrt(std::pow(X, -2.0 / 3.0) - 1.0);
        } while (!(r <= r_max));
        rng.iso(r, pos + 3 * i);
        // speed: q = v / v_esc with density g(q) ~ q^2 (1 - q^2)^(7/2), von Neumann rejection
        double q;
        for (;;) {
            q = rng.uniform();
            const double y = 0.1 * rng.uniform();
            if (y < q * q * std::pow(1.0 - q * q, 3.5)) break;
        }
        const double vesc = std::sqrt(2.0 * G * total_mass / std::sqrt(r * r + a * a));
        rng.iso(q * vesc, vel + 3 * i);
    }
    return RRG_OK;
}

RRG_API rrg_status rrg_generate_exp_disk(uint64_t seed, int64_t n, double disk_mass,
                                         double scale_length, double z0, double r_max,
                                         double z_max, double disp_frac, double bulge_mass,
                                         double bulge_a, double* pos, double* vel) {
    if (n < 0 || (n > 0 && (!pos || !vel)) || !(scale_length > 0) || !(z0 > 0) ||
        !(r_max > 0) || !(z_max > 0) || !(disp_frac >= 0))
        return io_fail(RRG_ERR_INVALID, "rrg_generate_exp_disk: bad argument");
    Rng rng(seed);
    const double Rd = scale_length, G = 1.0;
    const double fmax = 1.0 - (1.0 + r_max / Rd) * std::exp(-r_max / Rd);
    for (int64_t i = 0; i < n; ++i) {
        // R from M(<R)/M = u (truncated at r_max): solve 1 - (1 + x) e^-x = u by bisection
        const double u = rng.uniform() * fmax;
        double lo = 0.0, hi = r_max / Rd;
        for (int it = 0; it < 80; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (1.0 - (1.0 + mid) * std::exp(-mid) < u) lo = mid;
            else hi = mid;
        }
        const double R = 0.5 * (lo + hi) * Rd;
        const double ph = 2.0 * M_PI * rng.uniform();
        double z;
        do {  // sech^2(z / z0): CDF (1 + tanh(z / z0)) / 2
            const double w = rng.uniform_open();
            z = z0 * std::atanh(2.0 * w - 1.0);
        } while (!(std::fabs(z) < z_max));
        const double c = std::cos(ph), s = std::sin(ph);
        pos[3 * i] = R * c;
        pos[3 * i + 1] = R * s;
        pos[3 * i + 2] = z;
        double menc = disk_menc(disk_mass, Rd, R);
        if (bulge_mass > 0 && bulge_a > 0) menc += bulge_mass * R * R * R /
                                                   std::pow(R * R + bulge_a * bulge_a, 1.5);
        const double vc = R > 0 ? std::sqrt(G * menc / R) : 0.0;
        const double sig = disp_frac * vc;
        vel[3 * i] = -vc * s + sig * rng.normal();
        vel[3 * i + 1] = vc * c + sig * rng.normal();
        vel[3 * i + 2] = sig * rng.normal();
    }
    return RRG_OK;
}

}  // extern "C"
