// negftrans_main.cpp -- the driver of src/main.f90 over the B200 engine.
//
// Reads INPUT (the &INPUT namelist, main.f90:52-54, 90-92) and POTENTIAL
// (main.f90:156-160) from the working directory, converts units
// (main.f90:184-205), builds the k-mesh, basis and V table, runs the parts
// that are switched on through libnegfgpu.so, and writes TRANSMISSION,
// DENSITY and LDOS in the reference's formats ('(2G17.8)', '(3I5)'/'(4I5)' +
// '(5G17.8)', main.f90:570-601) plus an OUTPUT log.  With --check it only
// parses and validates, and prints the parsed deck as JSON (no GPU needed).
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "negf_gpu.h"

namespace {
constexpr double HARTREE = 27.211386245988;       // global.f90:24
constexpr double K_B = 8.617333262e-5 / HARTREE;  // global.f90:26
constexpr double A_0 = 0.529177210903;            // global.f90:27
constexpr double PI = 3.141592653589793;          // global.f90:28

// &INPUT with the defaults of main.f90:26-50
struct Deck {
    bool if_density = false, if_transmission = false, if_LDOS = false;
    double V_L = 0, V_R = 0, MU = 5.568, ETA = 1e-5, TEMPERATURE = 20, LX = 0, LY = 0, LZ = 0;
    double ENCUT = 100, GAP = 6, VDS = 0;
    double TRANSMISSION_GRID[3] = {0, 0, 0}, LDOS_ENERGY_GRID[3] = {0, 0, 0};
    int LDOS_GRID[3] = {-10, -10, -10};
    int NGX = 0, NGY = 0, NKX = 0, NKY = 0, N_circle = 40, N_line_per_eV = 500;
    // Engine key with no reference counterpart: effective mass m*/m_e (the
    // reference's kinetic term is |k+G|^2/2, i.e. m* = 1).
    double EMASS = 1;
    // Engine key with no reference counterpart: NEQ = .true. accepts VDS != 0
    // (rejected by main.f90:129-132) and computes the biased density with
    // mu_L = MU + VDS/2, mu_R = MU - VDS/2 (negf_density_neq).
    bool NEQ = false;
};

// Folds EMASS = m* into the energy scale: E' = m* E, V' = m* V, eta' = m* eta,
// T' = m* T, ENCUT' = m* ENCUT (and N_line_per_eV' = N_line_per_eV / m*), the
// m* = 1 problem with the same tau and density; G' = G / m*.
void fold_emass(Deck &d) {
    const double m = d.EMASS;
    if (m == 1) return;
    d.V_L *= m; d.V_R *= m; d.MU *= m; d.ETA *= m; d.TEMPERATURE *= m; d.ENCUT *= m; d.VDS *= m;
    d.TRANSMISSION_GRID[0] *= m; d.TRANSMISSION_GRID[1] *= m;
    d.LDOS_ENERGY_GRID[0] *= m; d.LDOS_ENERGY_GRID[1] *= m;
    d.N_line_per_eV = (int)std::floor(d.N_line_per_eV / m + 0.5);
}

std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// A Fortran real: accepts d/D exponents.
bool parse_real(std::string t, double *v) {
    for (auto &c : t)
        if (c == 'd' || c == 'D') c = 'e';
    char *end = nullptr;
    *v = std::strtod(t.c_str(), &end);
    return end && *end == 0 && !t.empty();
}

bool parse_logical(const std::string &t0, bool *b) {
    std::string t = lower(t0);
    if (!t.empty() && t[0] == '.') t = t.substr(1);
    if (t.empty()) return false;
    if (t[0] == 't') { *b = true; return true; }
    if (t[0] == 'f') { *b = false; return true; }
    return false;
}

// Values of one namelist item, with r*v repeats expanded.
std::vector<std::string> expand(const std::vector<std::string> &vals) {
    std::vector<std::string> out;
    for (const auto &v : vals) {
        const auto star = v.find('*');
        if (star != std::string::npos) {
            const int r = std::atoi(v.substr(0, star).c_str());
            for (int i = 0; i < r; ++i) out.push_back(v.substr(star + 1));
        } else {
            out.push_back(v);
        }
    }
    return out;
}

// Reads the &INPUT group (case-insensitive keys; comma, blank or newline
// separators; "!" comments; "/" ends the group).
bool read_namelist(const std::string &path, Deck &d, std::string &err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open " + path; return false; }
    std::string text, line;
    while (std::getline(f, line)) {
        const auto bang = line.find('!');
        if (bang != std::string::npos) line = line.substr(0, bang);
        text += line + "\n";
    }
    std::string lt = lower(text);
    auto start = lt.find("&input");
    if (start == std::string::npos) { err = "no &INPUT group"; return false; }
    start += 6;
    auto stop = lt.find('/', start);
    if (stop == std::string::npos) { err = "&INPUT group not terminated by /"; return false; }
    std::string body = text.substr(start, stop - start);
    for (auto &c : body)
        if (c == ',' || c == '\n' || c == '\r' || c == '\t') c = ' ';
    // split "KEY = v v v" groups: a token followed by '=' starts an item
    std::string spaced;
    for (char c : body) {
        if (c == '=') spaced += " = ";
        else spaced += c;
    }
    std::istringstream ss(spaced);
    std::vector<std::string> tok;
    for (std::string t; ss >> t;) tok.push_back(t);
    std::map<std::string, std::vector<std::string>> items;
    std::string key;
    for (size_t i = 0; i < tok.size(); ++i) {
        if (i + 1 < tok.size() && tok[i + 1] == "=") {
            key = lower(tok[i]);
            items[key].clear();
            ++i;
        } else if (!key.empty()) {
            items[key].push_back(tok[i]);
        } else {
            err = "value without a name: " + tok[i];
            return false;
        }
    }
    for (auto &kv : items) {
        const std::string &k = kv.first;
        const auto v = expand(kv.second);
        auto real1 = [&](double *dst) {
            if (v.empty() || !parse_real(v[0], dst)) { err = "bad value for " + k; return false; }
            return true;
        };
        auto int1 = [&](int *dst) {
            double x;
            if (v.empty() || !parse_real(v[0], &x)) { err = "bad value for " + k; return false; }
            *dst = (int)x;
            return true;
        };
        auto realn = [&](double *dst, int n) {
            for (int i = 0; i < n && i < (int)v.size(); ++i)
                if (!parse_real(v[i], dst + i)) { err = "bad value for " + k; return false; }
            return true;
        };
        auto intn = [&](int *dst, int n) {
            for (int i = 0; i < n && i < (int)v.size(); ++i) {
                double x;
                if (!parse_real(v[i], &x)) { err = "bad value for " + k; return false; }
                dst[i] = (int)x;
            }
            return true;
        };
        auto log1 = [&](bool *dst) {
            if (v.empty() || !parse_logical(v[0], dst)) { err = "bad value for " + k; return false; }
            return true;
        };
        bool ok = true;
        if (k == "if_density") ok = log1(&d.if_density);
        else if (k == "if_transmission") ok = log1(&d.if_transmission);
        else if (k == "if_ldos") ok = log1(&d.if_LDOS);
        else if (k == "v_l") ok = real1(&d.V_L);
        else if (k == "v_r") ok = real1(&d.V_R);
        else if (k == "mu") ok = real1(&d.MU);
        else if (k == "eta") ok = real1(&d.ETA);
        else if (k == "temperature") ok = real1(&d.TEMPERATURE);
        else if (k == "lx") ok = real1(&d.LX);
        else if (k == "ly") ok = real1(&d.LY);
        else if (k == "lz") ok = real1(&d.LZ);
        else if (k == "encut") ok = real1(&d.ENCUT);
        else if (k == "gap") ok = real1(&d.GAP);
        else if (k == "vds") ok = real1(&d.VDS);
        else if (k == "transmission_grid") ok = realn(d.TRANSMISSION_GRID, 3);
        else if (k == "ldos_energy_grid") ok = realn(d.LDOS_ENERGY_GRID, 3);
        else if (k == "ldos_grid") ok = intn(d.LDOS_GRID, 3);
        else if (k == "ngx") ok = int1(&d.NGX);
        else if (k == "ngy") ok = int1(&d.NGY);
        else if (k == "nkx") ok = int1(&d.NKX);
        else if (k == "nky") ok = int1(&d.NKY);
        else if (k == "n_circle") ok = int1(&d.N_circle);
        else if (k == "n_line_per_ev") ok = int1(&d.N_line_per_eV);
        else if (k == "emass") ok = real1(&d.EMASS);
        else if (k == "neq") ok = log1(&d.NEQ);
        else { err = "unknown namelist item " + k; return false; }
        if (!ok) return false;
    }
    return true;
}

// POTENTIAL: "N_x N_y N_z" then N_x*N_y*N_z values, x fastest (main.f90:156-160).
bool read_potential(const std::string &path, int dims[3], std::vector<double> &v, std::string &err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open " + path; return false; }
    std::vector<std::string> tok;
    for (std::string t; f >> t;) {
        for (auto &c : t)
            if (c == ',') c = ' ';
        std::istringstream s2(t);
        for (std::string u; s2 >> u;) tok.push_back(u);
    }
    if (tok.size() < 3) { err = "POTENTIAL too short"; return false; }
    for (int a = 0; a < 3; ++a) dims[a] = std::atoi(tok[a].c_str());
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    v.clear();
    v.reserve(n);
    for (size_t i = 3; i < tok.size() && v.size() < n; ++i) {
        const auto star = tok[i].find('*');
        double x;
        if (star != std::string::npos) {
            const int r = std::atoi(tok[i].substr(0, star).c_str());
            if (!parse_real(tok[i].substr(star + 1), &x)) { err = "bad POTENTIAL value " + tok[i]; return false; }
            for (int q = 0; q < r; ++q) v.push_back(x);
        } else {
            if (!parse_real(tok[i], &x)) { err = "bad POTENTIAL value " + tok[i]; return false; }
            v.push_back(x);
        }
    }
    if (v.size() != n) { err = "POTENTIAL has fewer values than N_x*N_y*N_z"; return false; }
    return true;
}

// Fortran Gw.d output editing (w=17, d=8 here): F editing with d-k decimals
// and 4 trailing blanks when 0.1 <= |x| < 10^d after rounding to d digits,
// E editing (0.dddddddE+xx) otherwise.
std::string gfmt(double x, int w = 17, int d = 8) {
    char buf[64];
    if (x == 0.0) {
        std::snprintf(buf, sizeof buf, "%*.*f%4s", w - 4, d - 1, 0.0, "");
        return buf;
    }
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, x);
    const int e10 = std::atoi(std::strchr(buf, 'e') + 1);
    const int k = e10 + 1;  // 10^(k-1) <= |x| < 10^k after rounding
    if (k >= 0 && k <= d) {
        std::snprintf(buf, sizeof buf, "%*.*f%4s", w - 4, d - k, x, "");
        return buf;
    }
    // mantissa 0.d1..d8, exponent k
    char mant[32];
    std::snprintf(mant, sizeof mant, "%.*e", d - 1, std::fabs(x));
    std::string digits;
    for (char c : std::string(mant))
        if (std::isdigit((unsigned char)c)) digits += c;
        else if (c == 'e') break;
    char ex[16];
    if (std::abs(k) <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", k < 0 ? '-' : '+', std::abs(k));
    else std::snprintf(ex, sizeof ex, "%c%03d", k < 0 ? '-' : '+', std::abs(k));
    std::string s = std::string(x < 0 ? "-" : "") + "0." + digits.substr(0, d) + ex;
    if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
    return s;
}

void write_g(FILE *f, const std::vector<double> &v, int per_line) {
    for (size_t i = 0; i < v.size(); ++i) {
        std::fputs(gfmt(v[i]).c_str(), f);
        if ((i + 1) % per_line == 0 || i + 1 == v.size()) std::fputc('\n', f);
    }
}

void banner(FILE *o, const char *word) {
    std::fprintf(o, " ********************\n *                  *\n *      %-12s*\n *                  *\n ********************\n",
                 word);
}

int nint(double x) { return (int)std::floor(x + 0.5); }

}  // namespace

int main(int argc, char **argv) {
    if (argc > 1 && std::strcmp(argv[1], "--gfmt") == 0) {  // the G17.8 writer, for tests
        for (int i = 2; i < argc; ++i) std::printf("[%s]\n", gfmt(std::strtod(argv[i], nullptr)).c_str());
        return 0;
    }
    const bool check_only = argc > 1 && std::strcmp(argv[1], "--check") == 0;
    const int device = std::getenv("NEGF_DEVICE") ? std::atoi(std::getenv("NEGF_DEVICE")) : 0;
    const auto t0 = std::chrono::steady_clock::now();
    FILE *out = std::fopen("OUTPUT", "w");
    if (!out) { std::fprintf(stderr, "cannot write OUTPUT\n"); return 2; }
    std::fprintf(out, " NEGF transport on the B200 engine (%s)\n Read in INPUT...\n", negf_version());
    Deck d;
    std::string err;
    if (!read_namelist("INPUT", d, err)) {
        std::fprintf(out, " ERROR: %s\n", err.c_str());
        banner(out, "EXIT");
        std::fclose(out);
        std::fprintf(stderr, "INPUT: %s\n", err.c_str());
        return 1;
    }
    const double emass = d.EMASS;
    if (!(emass > 0)) {
        std::fprintf(out, " ERROR: EMASS must be positive\n");
        banner(out, "EXIT");
        std::fclose(out);
        return 1;
    }
    fold_emass(d);
    // NGX, NGY (main.f90:94-100; the NGX test reads LY as the reference does)
    const double s = std::sqrt(d.ENCUT / HARTREE / 2);
    if (d.NGX <= (int)std::ceil((d.LY / A_0) / PI * s * 2)) d.NGX = (int)std::ceil((d.LX / A_0) / PI * s * 2) + 1;
    if (d.NGY <= (int)std::ceil((d.LY / A_0) / PI * s * 2)) d.NGY = (int)std::ceil((d.LY / A_0) / PI * s * 2) + 1;
    // checks of main.f90:102-132
    std::vector<std::string> bad;
    if (d.LX == 0 || d.LY == 0 || d.LZ == 0) bad.push_back("ERROR: LX, LY, LZ must be specified in INPUT");
    if (d.NKX == 0 || d.NKY == 0) bad.push_back("ERROR: NKX, NKY must be specified in INPUT");
    if (!(d.if_density || d.if_transmission || d.if_LDOS))
        bad.push_back("ERROR: At least one of (if_xxxxx) be .true.   Nothing to do...");
    if (d.if_transmission && d.TRANSMISSION_GRID[2] == 0)
        bad.push_back("ERROR: TRANSMISSION_GRID must be specified for (if_transmission = .true.)");
    if (d.if_LDOS && d.LDOS_ENERGY_GRID[2] == 0)
        bad.push_back("ERROR: LDOS_ENERGY_GRID must be specified for (if_LDOS = .true.)");
    if (d.if_LDOS && (d.LDOS_GRID[0] < -1 || d.LDOS_GRID[1] < -1 || d.LDOS_GRID[2] < -1))
        bad.push_back("ERROR: LDOS_GRID must be specified for (if_LDOS = .true.)");
    if (d.VDS != 0 && !d.NEQ)
        bad.push_back("ERROR: VDS must be zero in this version, please upgrade to higher version.");
    std::fprintf(out, " Checking Parameters...\n");
    for (auto &b : bad) std::fprintf(out, " %s\n", b.c_str());
    if (!bad.empty()) {
        banner(out, "EXIT");
        std::fclose(out);
        return 1;
    }
    std::fprintf(out, " -success-\n ----------\n Read in POTENTIAL...\n");
    int dims[3];
    std::vector<double> V;
    if (!read_potential("POTENTIAL", dims, V, err)) {
        std::fprintf(out, " ERROR: %s\n", err.c_str());
        banner(out, "EXIT");
        std::fclose(out);
        std::fprintf(stderr, "POTENTIAL: %s\n", err.c_str());
        return 1;
    }
    const int Nx = dims[0], Ny = dims[1], Nz = dims[2];
    if (Nx % 2 || Ny % 2) {  // main.f90:163-174
        std::fprintf(out, " ERROR: The number of grid point in x & y direction must be even number\n");
        banner(out, "EXIT");
        std::fclose(out);
        return 1;
    }
    std::fprintf(out, " -success-\n The size of POTENTIAL is: %d %d %d\n ----------\n", Nx, Ny, Nz);
    // units, main.f90:184-205
    const double aV_L = d.V_L / HARTREE, aV_R = d.V_R / HARTREE, aMU = d.MU / HARTREE, aETA = d.ETA;
    const double aLX = d.LX / A_0, aLY = d.LY / A_0, aLZ = d.LZ / A_0, aENCUT = d.ENCUT / HARTREE;
    const double aGAP = d.GAP * K_B * d.TEMPERATURE;
    double min_v = 1e300;
    for (auto &x : V) {
        x = x * emass / HARTREE;
        min_v = std::min(min_v, x);
    }
    std::vector<double> kpt(3 * (size_t)d.NKX * d.NKY);
    negf_kmesh(d.NKX, d.NKY, aLX, aLY, kpt.data());
    int32_t N = 0;
    negf_basis_size(aENCUT, aLX, aLY, &N);
    std::vector<int32_t> nxg(N), nyg(N);
    negf_basis(aENCUT, aLX, aLY, N, nxg.data(), nyg.data());
    std::fprintf(out, " Number of K-point grid is: %d\n Layout the Grid...\n Grid size in x, y direction is: N = %d\n"
                      " Grid size in z direction is: N_z = %d\n NGX, NGY = %d %d\n ----------\n",
                 d.NKX * d.NKY, N, Nz, d.NGX, d.NGY);
    if (check_only) {
        std::printf("{\"N\": %d, \"Nz\": %d, \"Nx\": %d, \"Ny\": %d, \"NGX\": %d, \"NGY\": %d, \"nk\": %d, "
                    "\"if_density\": %d, \"if_transmission\": %d, \"if_LDOS\": %d, \"ETA\": %.17g, \"ENCUT\": %.17g, "
                    "\"LX\": %.17g, \"LY\": %.17g, \"LZ\": %.17g, \"TRANSMISSION_GRID\": [%.17g, %.17g, %.17g], "
                    "\"LDOS_GRID\": [%d, %d, %d], \"N_circle\": %d, \"N_line_per_eV\": %d, \"min_V\": %.17g, "
                    "\"V_sum\": %.17g, \"MU\": %.17g, \"TEMPERATURE\": %.17g, \"EMASS\": %.17g, \"NEQ\": %d, "
                    "\"VDS\": %.17g}\n",
                    N, Nz, Nx, Ny, d.NGX, d.NGY, d.NKX * d.NKY, d.if_density, d.if_transmission, d.if_LDOS, d.ETA,
                    d.ENCUT, d.LX, d.LY, d.LZ, d.TRANSMISSION_GRID[0], d.TRANSMISSION_GRID[1],
                    d.TRANSMISSION_GRID[2], d.LDOS_GRID[0], d.LDOS_GRID[1], d.LDOS_GRID[2], d.N_circle,
                    d.N_line_per_eV, min_v, [&] { double t = 0; for (double x : V) t += x; return t; }(), d.MU,
                    d.TEMPERATURE, emass, (int)d.NEQ, d.VDS);
        std::fclose(out);
        return 0;
    }
    // V table (LocalPotential_RealToPlanewave + main.f90:239-247)
    std::vector<double> vhat(2 * (size_t)(2 * d.NGX + 1) * (2 * d.NGY + 1) * Nz);
    if (negf_vhat(V.data(), Nx, Ny, Nz, d.NGX, d.NGY, vhat.data()) != NEGF_OK) {
        std::fprintf(out, " ERROR: 'The size of V_reciprocal minus one' should not be larger than 'the size of V_real'\n");
        banner(out, "EXIT");
        std::fclose(out);
        return 1;
    }
    negf_problem p{N, Nz, d.NGX, d.NGY, nxg.data(), nyg.data(), vhat.data(), aLX, aLY, aLZ, aV_L, aV_R, aETA,
                   d.NKX * d.NKY, kpt.data(), 0};
    // engine option outside the reference's namelist: NEGF_LEAD_MODEL=1 selects the
    // exact lattice surface Green's function of the leads
    if (const char *lm = std::getenv("NEGF_LEAD_MODEL")) p.lead_model = std::atoi(lm);
    negf_ctx *ctx = nullptr;
    int rc = negf_ctx_create(&p, device, &ctx);
    if (rc) {
        std::fprintf(out, " ERROR: negf_ctx_create failed (%d)\n", rc);
        banner(out, "EXIT");
        std::fclose(out);
        return 1;
    }
    negf_stats st{};
    double t_dens = 0, t_trans = 0, t_ldos = 0;
    std::vector<double> density, tau, ldos;
    int ldos_m[4] = {0, 0, 0, 0};
    if (d.if_density && d.NEQ) {
        // biased density: Gauss-Legendre semicircle (N_circle nodes) and a real-axis
        // window [min(mu) - GAP, max(mu) + GAP] with N_line_per_eV nodes per eV
        const double aVDS = d.VDS / HARTREE;
        const int n_window = std::max(1, nint(d.N_line_per_eV * ((2 * aGAP + std::fabs(aVDS)) * HARTREE)));
        std::fprintf(out, " Density calculation start (bias VDS = %s eV)...\n Number of energy points for integration: %d\n",
                     gfmt(d.VDS / emass).c_str(), d.N_circle + n_window);
        density.assign((size_t)Nx * Ny * Nz, 0.0);
        std::vector<double> dm(2 * (size_t)N * N * Nz);
        const auto a = std::chrono::steady_clock::now();
        rc = negf_density_neq(ctx, d.N_circle, n_window, min_v, aMU + aVDS / 2, aMU - aVDS / 2, aGAP, d.TEMPERATURE,
                              dm.data(), &st);
        if (rc >= 0) {
            const int r2 = negf_dm_real(ctx, dm.data(), Nx, Ny, (double)Nz / (d.LX * d.LY * d.LZ), density.data());
            if (r2 < 0) rc = r2;
        }
        t_dens = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        if (rc < 0) { std::fprintf(out, " ERROR: density failed (%d)\n", rc); negf_ctx_destroy(ctx); std::fclose(out); return 1; }
        if (rc > 0) std::fprintf(out, " WARNING: zero pivot in %d contour jobs (first job %d)\n", st.n_singular, st.first_bad_job);
        std::fprintf(out, " Density calculation DONE\n ----------\n");
    } else if (d.if_density) {
        const int n_line = nint(d.N_line_per_eV * ((2 * aGAP) * HARTREE));  // main.f90:261
        std::fprintf(out, " Density calculation start...\n Number of energy points for integration: %d\n", d.N_circle + n_line);
        density.assign((size_t)Nx * Ny * Nz, 0.0);
        const auto a = std::chrono::steady_clock::now();
        rc = negf_density_real(ctx, d.N_circle, n_line, min_v, aMU, aGAP, d.TEMPERATURE, Nx, Ny,
                               (double)Nz / (d.LX * d.LY * d.LZ), density.data(), nullptr, &st);
        t_dens = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        if (rc < 0) { std::fprintf(out, " ERROR: density failed (%d)\n", rc); negf_ctx_destroy(ctx); std::fclose(out); return 1; }
        if (rc > 0) std::fprintf(out, " WARNING: zero pivot in %d contour jobs (first job %d)\n", st.n_singular, st.first_bad_job);
        std::fprintf(out, " Density calculation DONE\n ----------\n");
    }
    if (d.if_transmission) {
        const int nE = nint(d.TRANSMISSION_GRID[2]);  // main.f90:369-375
        std::vector<double> E(nE);
        const double e1 = d.TRANSMISSION_GRID[0] / HARTREE, e2 = d.TRANSMISSION_GRID[1] / HARTREE;
        for (int i = 0; i < nE; ++i) E[i] = e1 + (e2 - e1) * i / nE;
        tau.assign(nE, 0.0);
        std::fprintf(out, " Transmission calculation start...\n Number of energy grid points: %d\n", nE);
        const auto a = std::chrono::steady_clock::now();
        rc = negf_transmission(ctx, E.data(), nE, NEGF_FP64, tau.data(), &st);
        t_trans = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        if (rc < 0) { std::fprintf(out, " ERROR: transmission failed (%d)\n", rc); negf_ctx_destroy(ctx); std::fclose(out); return 1; }
        if (rc > 0) std::fprintf(out, " WARNING: zero pivot in %d jobs (first job %d)\n", st.n_singular, st.first_bad_job);
        std::fprintf(out, " Transmission calculation DONE\n ----------\n");
        FILE *f = std::fopen("TRANSMISSION", "w");
        std::fprintf(f, " #   Energy (eV)    Transmission_coefficient\n");
        for (int i = 0; i < nE; ++i) std::fprintf(f, "%s%s\n", gfmt(E[i] * HARTREE / emass).c_str(), gfmt(tau[i]).c_str());
        std::fclose(f);
    }
    if (d.if_LDOS) {
        const int nE = nint(d.LDOS_ENERGY_GRID[2]);
        ldos_m[0] = d.LDOS_GRID[0] == 0 ? Nx : 1;
        ldos_m[1] = d.LDOS_GRID[1] == 0 ? Ny : 1;
        ldos_m[2] = d.LDOS_GRID[2] == 0 ? Nz : 1;
        ldos_m[3] = nE;
        ldos.assign((size_t)ldos_m[0] * ldos_m[1] * ldos_m[2] * nE, 0.0);
        const double dxyz[3] = {d.LX / Nx, d.LY / Ny, d.LZ / Nz};
        std::fprintf(out, " LDOS calculation start...\n Number of energy grid points: %d\n", nE);
        const auto a = std::chrono::steady_clock::now();
        rc = negf_ldos(ctx, d.LDOS_ENERGY_GRID[0] / HARTREE, d.LDOS_ENERGY_GRID[1] / HARTREE, nE, d.LDOS_GRID, Nx, Ny,
                       dxyz, (double)Nz / (d.LX * d.LY * d.LZ) / HARTREE * emass, ldos.data(), &st);
        t_ldos = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        if (rc < 0) { std::fprintf(out, " ERROR: LDOS failed (%d)\n", rc); negf_ctx_destroy(ctx); std::fclose(out); return 1; }
        std::fprintf(out, " LDOS calculation DONE\n ----------\n");
    }
    negf_ctx_destroy(ctx);
    std::fprintf(out, "\n ===== ALL NEGF calculation DONE =====\n\n");
    if (d.if_density) {
        double tot = 0;
        for (double x : density) tot += x;
        std::fprintf(out, " Total charge is: %s\n Writing DENSITY...\n",
                     gfmt(tot * (d.LX * d.LY * d.LZ) / ((double)Nx * Ny * Nz)).c_str());
        FILE *f = std::fopen("DENSITY", "w");
        std::fprintf(f, "%5d%5d%5d\n", Nx, Ny, Nz);
        write_g(f, density, 5);
        std::fclose(f);
    }
    if (d.if_transmission) std::fprintf(out, " Writing TRANSMISSION...\n");
    if (d.if_LDOS) {
        std::fprintf(out, " Writing LDOS...\n");
        FILE *f = std::fopen("LDOS", "w");
        std::fprintf(f, "%5d%5d%5d%5d\n", ldos_m[0], ldos_m[1], ldos_m[2], ldos_m[3]);
        write_g(f, ldos, 5);
        std::fclose(f);
    }
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::fprintf(out, " Wall time (Total): %.3f s\n ├── Wall time (Density): %.3f s\n ├── Wall time (Transmission): %.3f s\n"
                      " └── Wall time (LDOS): %.3f s\n",
                 total, t_dens, t_trans, t_ldos);
    banner(out, "DONE");
    std::fclose(out);
    return 0;
}
