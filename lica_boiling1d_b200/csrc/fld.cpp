// fld###### restart files of the 1-D column (host code, no GPU).
//
// Writer: WRITEFIELD (1d.f:1121-1232), record by record with its FORMATs 1001-1016.
// Reader: PREFLD (1d.f:972-1098), then the start-up steps that follow a read in MAIN:
// LVSINIT's read branch (two_phase.f:148-205: ALPHI_EXT = 0, band values from the lists,
// ALPHI_BC, CAL_PSIF(1, N_MAX)), GRID_COUPLING(1) (1d.f:138), VOL_TOT_IPHS = VOL_TOT_ORI
// (1d.f:146-151), IRESET (1d.f:175-178) and the DO loop's restart at M = 1 (1d.f:195).
//
// The column is the reference's 1-D case (grid.in: N1 = N2 = 2, N3 = n + 1; N1F = N2F = 3,
// N3F = 2n + 1).  Every field is the same on its (I, J) replicas: the writer repeats the
// column value over them, the reader takes the replica I = J = 1.  U and V are zero in a
// column and are written as zeros and skipped on reading.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lica_gpu.h"

void lica_set_last_error(const char* what, const char* msg, const char* file, int line);

namespace {

constexpr int kMMax = 11;  // M_MAX, 1dmodulesX.f:21: band layers
constexpr int kGL = 2;     // phi / layer index of refined cell k = -2

// ---------------------------------------------------------------------------------------
// Output edit descriptors (Fortran 2008 10.7.2.3.2 ES, 10.7.2.2 I)

// ESw.d: one nonzero leading digit, d decimals, exponent "E+zz" (|e| <= 99) or "+zzz"
// (99 < |e| <= 999), right-justified in w; a value that does not fit prints w asterisks.
std::string ed_es(double x, int w, int d) {
    std::string s;
    if (std::isnan(x)) {
        s = "NaN";
    } else if (std::isinf(x)) {
        s = (w >= 9) ? (x < 0 ? "-Infinity" : "Infinity") : (x < 0 ? "-Inf" : "Inf");
    } else {
        char b[64];
        std::snprintf(b, sizeof b, "%.*E", d, x);
        s = b;
        const size_t e = s.find('E');
        const int ex = std::atoi(s.c_str() + e + 1);
        if (ex > 99 || ex < -99) s.erase(e, 1);
    }
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}

std::string ed_i(long long v, int w) {
    const std::string s = std::to_string(v);
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}

// One WRITE statement of `count` like items under a FORMAT of `per` repeated descriptors:
// records of `per` items (format reversion); an empty list writes one empty record.
template <class F>
void put_list(std::string& out, size_t count, size_t per, F item) {
    if (count == 0) {
        out += '\n';
        return;
    }
    for (size_t i = 0; i < count; ++i) {
        out += item(i);
        if ((i + 1) % per == 0 || i + 1 == count) out += '\n';
    }
}

// ---------------------------------------------------------------------------------------
// Input (Fortran 2008 10.7.2: BLANK = 'NULL' and PAD = 'YES', the OPEN defaults)

struct Desc {
    bool real;
    int w, d;
};

struct Value {
    long long i = 0;
    double r = 0.0;
};

struct Reader {
    std::vector<std::string> lines;
    size_t next = 0;
    std::string err;

    // Iw: blanks ignored, an all-blank field is zero.
    static bool parse_int(const std::string& f, long long& v) {
        std::string s;
        for (char c : f)
            if (c != ' ' && c != '\t') s += c;
        v = 0;
        if (s.empty()) return true;
        size_t i = 0;
        bool neg = false;
        if (s[0] == '+' || s[0] == '-') {
            neg = s[0] == '-';
            i = 1;
        }
        if (i == s.size()) return false;
        unsigned long long a = 0;
        for (; i < s.size(); ++i) {
            if (!std::isdigit((unsigned char)s[i])) return false;
            a = a * 10 + (unsigned long long)(s[i] - '0');
            if (a > (1ull << 62)) return false;
        }
        v = neg ? -(long long)a : (long long)a;
        return true;
    }

    // Ew.d / ESw.d input: [sign] digits [. digits] [exponent], the exponent "E|D|Q [sign]
    // digits" or "sign digits"; without a decimal point the rightmost d digits are the
    // fraction; blanks ignored (an all-blank field is zero); NaN and Inf / Infinity.
    static bool parse_real(const std::string& f, int d, double& v) {
        std::string s;
        for (char c : f)
            if (c != ' ' && c != '\t') s += c;
        v = 0.0;
        if (s.empty()) return true;
        size_t i = 0;
        bool neg = false;
        if (s[0] == '+' || s[0] == '-') {
            neg = s[0] == '-';
            i = 1;
        }
        std::string u;
        for (size_t q = i; q < s.size(); ++q) u += (char)std::toupper((unsigned char)s[q]);
        if (u == "INF" || u == "INFINITY") {
            v = neg ? -INFINITY : INFINITY;
            return true;
        }
        if (u.rfind("NAN", 0) == 0 && (u.size() == 3 || (u[3] == '(' && u.back() == ')'))) {
            v = NAN;
            return true;
        }
        std::string digits;
        long point = -1;
        for (; i < s.size() && (std::isdigit((unsigned char)s[i]) || s[i] == '.'); ++i) {
            if (s[i] == '.') {
                if (point >= 0) return false;
                point = (long)digits.size();
            } else {
                digits += s[i];
            }
        }
        if (digits.empty()) return false;
        long ex = 0;
        if (i < s.size()) {
            const char c = (char)std::toupper((unsigned char)s[i]);
            if (c == 'E' || c == 'D' || c == 'Q') ++i;
            else if (c != '+' && c != '-') return false;
            bool eneg = false;
            if (i < s.size() && (s[i] == '+' || s[i] == '-')) eneg = s[i++] == '-';
            if (i == s.size()) return false;
            for (; i < s.size(); ++i) {
                if (!std::isdigit((unsigned char)s[i])) return false;
                if (ex < 100000) ex = ex * 10 + (s[i] - '0');
            }
            if (eneg) ex = -ex;
        }
        const long frac = (point < 0) ? d : (long)digits.size() - point;
        const std::string t = (neg ? "-" : "") + digits + "E" + std::to_string(ex - frac);
        errno = 0;
        char* end = nullptr;
        v = std::strtod(t.c_str(), &end);
        if (end != t.c_str() + t.size()) return false;
        return !std::isinf(v);
    }

    // One READ statement of `count` items: each record supplies the fields of `fmt` in
    // order; when they are used up and items remain, the next record starts the FORMAT
    // again.  A READ takes at least one record; a record shorter than its fields reads as
    // blanks.
    bool read(const std::vector<Desc>& fmt, size_t count, std::vector<Value>& out, const char* what) {
        out.assign(count, Value{});
        size_t item = 0;
        do {
            if (next >= lines.size()) {
                err = std::string("end of file in ") + what;
                return false;
            }
            const std::string& rec = lines[next++];
            size_t col = 0;
            for (size_t q = 0; q < fmt.size() && item < count; ++q, ++item) {
                std::string f = col < rec.size() ? rec.substr(col, fmt[q].w) : std::string();
                col += fmt[q].w;
                const bool ok = fmt[q].real ? parse_real(f, fmt[q].d, out[item].r) : parse_int(f, out[item].i);
                if (!ok) {
                    err = std::string("bad field '") + f + "' in " + what + " (line " + std::to_string(next) + ")";
                    return false;
                }
            }
        } while (item < count);
        return true;
    }
};

const std::vector<Desc> F1001 = {{false, 8, 0}, {false, 8, 0}, {false, 8, 0}};                   // 3I8
const std::vector<Desc> F1002 = {{false, 8, 0}, {false, 8, 0}, {true, 20, 12}, {true, 20, 12}};   // 2I8,2ES20.12
const std::vector<Desc> F1003 = {{false, 8, 0}, {false, 8, 0}, {false, 8, 0}, {false, 8, 0},
                                 {true, 20, 12}};                                                 // 4I8,1ES20.12
const std::vector<Desc> F1004 = {{true, 20, 12}};                                                 // 1ES20.12
const std::vector<Desc> F1005(5, Desc{true, 20, 12});                                             // 5ES20.12
const std::vector<Desc> F1006(3, Desc{true, 20, 12});                                             // 3ES20.12
const std::vector<Desc> F1007(4, Desc{false, 8, 0});                                              // 4I8
const std::vector<Desc> F1012(6, Desc{true, 20, 12});                                             // 6ES20.12
const std::vector<Desc> F1013 = {{false, 8, 0}, {false, 8, 0}};                                   // 2I8
const std::vector<Desc> F1014(8, Desc{true, 20, 12});                                             // 8ES20.12
const std::vector<Desc> F1015(8, Desc{false, 8, 0});                                              // 8I8
const std::vector<Desc> F1016 = {{false, 8, 0}, {false, 8, 0}, {false, 8, 0}, {true, 20, 12}};    // 3I8,1ES20.12

int fail(int code, const std::string& msg, int line) {
    lica_set_last_error("fld", msg.c_str(), __FILE__, line);
    return code;
}

bool load_lines(const char* path, std::vector<std::string>& lines, std::string& err) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        err = std::string("cannot open ") + path + ": " + std::strerror(errno);
        return false;
    }
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
    const bool bad = std::ferror(fp) != 0;
    std::fclose(fp);
    if (bad) {
        err = std::string("read error on ") + path;
        return false;
    }
    lines.clear();
    size_t a = 0;
    while (a < text.size()) {
        size_t b = text.find('\n', a);
        if (b == std::string::npos) b = text.size();
        std::string l = text.substr(a, b - a);
        if (!l.empty() && l.back() == '\r') l.pop_back();
        lines.push_back(std::move(l));
        a = b + 1;
    }
    return true;
}

// ---------------------------------------------------------------------------------------
// Start-up after a read, 1-D column (phi and layer indexed [k + kGL], k = -2..nf+4)

// ALPHI_BC (two_phase.f:462-642), z part: linear extension by SDZF from the end cells,
// then the periodic copy that runs for IPZ /= 1 (two_phase.f:624-634, N3F_BD = 2).
void alphi_bc(double* phi, int nf, double hf) {
    auto P = [&](int k) -> double& { return phi[k + kGL]; };
    const double a1 = P(1);
    if (std::fabs(a1) < 1e-8) {
        P(0) = 0.0;
        P(-1) = 0.0;
        P(-2) = 0.0;
    } else if (a1 > 0.0) {
        P(0) = a1 + hf;
        P(-1) = P(0) + hf;
        P(-2) = P(-1) + hf;
    } else if (a1 < 0.0) {
        P(0) = a1 - hf;
        P(-1) = P(0) - hf;
        P(-2) = P(-1) - hf;
    }
    const double an = P(nf);
    if (std::fabs(an) < 1e-8) {
        for (int q = 1; q <= 4; ++q) P(nf + q) = 0.0;
    } else if (an > 0.0) {
        P(nf + 1) = an + hf;
        for (int q = 2; q <= 4; ++q) P(nf + q) = P(nf + q - 1) + hf;
    } else if (an < 0.0) {
        P(nf + 1) = an - hf;
        for (int q = 2; q <= 4; ++q) P(nf + q) = P(nf + q - 1) - hf;
    }
    for (int k = 0; k <= 2; ++k) {
        P(-k) = P(nf - k);
        P(nf + 1 + k) = P(1 + k);
    }
}

// CAL_PSIF(1, N_MAX) (two_phase.f:2503-2560, 2711-2722): CAL_PSIF_MTP(1, N_MAX)
// (two_phase.f:2835-3060) -- the sub-cell fraction on every band cell (x and y
// differences vanish in a column), its 1e-5 snap, the fill of the other cells from the
// sign changes of phi scanned from the top -- then the global snap.  psif[k], k = 1..nf.
void cal_psif(const double* phi, const int* layer, int nf, double* psif) {
    auto P = [&](int k) { return phi[k + kGL]; };
    std::vector<double> ps(nf + 2, 0.0);
    std::vector<char> band(nf + 2, 0);
    for (int k = 1; k <= nf; ++k) {
        const int m = layer[k + kGL];
        if (m < 1 || m > kMMax) continue;
        const double e1 = 0.5 * std::fabs(P(k + 1) - P(k - 1));
        double t;
        if (e1 > 1e-8) {
            const double f1 = std::max(0.5 * (e1 + 0.0 + 0.0) - std::fabs(P(k)), 0.0);
            t = f1 / e1;
        } else {
            t = (P(k) != 0.0) ? 0.0 : 0.5;
        }
        double v = (P(k) <= 0.0) ? t : 1.0 - t;
        if (v < 1e-5) v = 0.0;
        else if (v > 0.99999) v = 1.0;
        ps[k] = v;
        band[k] = 1;
    }
    std::vector<int> kc;
    for (int k = nf; k >= 1; --k)
        if (P(k) * P(k + 1) < 0.0) kc.push_back(k);
    if (kc.empty()) {
        for (int k = 1; k <= nf; ++k)
            if (!band[k]) ps[k] = 1.0;
    } else {
        for (size_t l = 0; l < kc.size(); ++l) {
            const double t = (P(kc[l]) < 0.0) ? 0.0 : 1.0;
            const int k0 = (l == 0) ? ((std::fabs(ps[1] - 0.5) < 0.5) ? 2 : 1) : kc[l - 1];
            for (int k = k0; k <= kc[l]; ++k)
                if (!band[k]) ps[k] = t;
        }
        const int kl = kc.back();
        const double t = (P(kl + 1) < 0.0) ? 0.0 : 1.0;
        for (int k = kl + 1; k <= nf; ++k)
            if (!band[k]) ps[k] = t;
    }
    psif[0] = 0.0;
    psif[nf + 1] = 0.0;
    for (int k = 1; k <= nf; ++k) {
        double v = ps[k];
        if (v < 1e-5) v = 0.0;
        else if (v > 0.99999) v = 1.0;
        psif[k] = v;
    }
}

double zp(double h, int n, int k) {
    if (k <= 0) return 0.0;
    if (k >= n + 1) return n * h;
    return (k - 1) * h + 0.5 * h;
}

// The refined-cell box mean of INTER_PSI (two_phase.f:5123-5538) over [z1, z2] and
// refined cells k1..k2, once per (II, JJ) replica; an index outside 1..nf reads the end.
double box_mean(const double* f, int nf, int k1, int k2, double z1, double z2, double hf) {
    const double ssdzf = 1.0 / hf;
    double sum = 0.0, volf = 0.0;
    for (int rep = 0; rep < 4; ++rep)
        for (int kk = k1; kk <= k2; ++kk) {
            const double v = f[kk < 1 ? 1 : (kk > nf ? nf : kk)];
            const double za = (kk - 1) * hf, zb = kk * hf;
            if (za <= z1 && zb >= z2) {
                sum = sum + v;
                volf = volf + 1.0;
                break;
            } else if (za < z1 && zb > z1) {
                sum = sum + v * (zb - z1) * ssdzf;
                volf = volf + (zb - z1) * ssdzf;
            } else if (za >= z1 && zb <= z2) {
                sum = sum + v;
                volf = volf + 1.0;
            } else if (za < z2 && zb > z2) {
                sum = sum + v * (z2 - za) * ssdzf;
                volf = volf + (z2 - za) * ssdzf;
            } else if (za >= z2) {
                break;
            }
        }
    return sum / volf;
}

// GRID_COUPLING(1) (two_phase.f:4863-5118) on every flow cell: PSI_ZN over [ZP(k-1),
// ZP(k)], PSI_CN over [Z(k), Z(k+1)], the 1e-3 / 0.999 snaps, PSI_CN's end copies.
void grid_coupling1(int n, double L, const double* psif, double* psi_cn, double* psi_zn) {
    const int nf = 2 * n;
    const double h = L / n, hf = L / nf;
    for (int k = 0; k <= n + 1; ++k) {
        psi_cn[k] = 0.0;
        psi_zn[k] = 0.0;
    }
    for (int k = 2; k <= n; ++k)
        psi_zn[k] = box_mean(psif, nf, 2 * k - 2, 2 * k - 1, zp(h, n, k - 1), zp(h, n, k), hf);
    for (int k = 1; k <= n; ++k) {
        if (psi_zn[k] < 1e-3) psi_zn[k] = 0.0;
        else if (psi_zn[k] > 0.999) psi_zn[k] = 1.0;
    }
    for (int k = 1; k <= n; ++k) psi_cn[k] = box_mean(psif, nf, 2 * k - 1, 2 * k, (k - 1) * h, k * h, hf);
    for (int k = 1; k <= n; ++k) {
        if (psi_cn[k] < 1e-3) psi_cn[k] = 0.0;
        else if (psi_cn[k] > 0.999) psi_cn[k] = 1.0;
    }
    psi_cn[0] = psi_cn[1];
    psi_cn[n + 1] = psi_cn[n];
}

bool state_ok(const lica_col_state* st) {
    return st && st->w && st->p && st->t && st->psi_cn && st->psi_zn && st->phi && st->layer && st->psif &&
           st->wo && st->mflvs && st->sfgas && st->sfgas2 && st->imask && st->scal && st->stats;
}

}  // namespace

extern "C" {

int lica_fld_name(int64_t ihist, char* out, int32_t cap) {
    if (!out || cap < 10) return LICA_BAD_ARG;
    // the reference's digit arithmetic (1d.f:1155-1163): char(48 + digit) for six places
    long long r = ihist;
    const long long p[6] = {100000, 10000, 1000, 100, 10, 1};
    std::memcpy(out, "fld", 3);
    for (int q = 0; q < 6; ++q) {
        const long long dgt = r / p[q];
        r -= dgt * p[q];
        if (dgt < 0 || dgt > 9) return fail(LICA_BAD_ARG, "IHIST outside 0..999999 has no fld###### name", __LINE__);
        out[3 + q] = (char)('0' + dgt);
    }
    out[9] = '\0';
    return LICA_OK;
}

int lica_col_fld_write(const char* path, int32_t n, const lica_col_props* props, const lica_col_state* st,
                       const lica_fld_info* info) {
    if (!path || n < 1 || !props || !state_ok(st) || !info)
        return fail(LICA_BAD_ARG, "lica_col_fld_write: null argument or n < 1", __LINE__);
    const long long N1 = 2, N2 = 2, N3 = (long long)n + 1, N1M = 1, N2M = 1, N3M = n;
    const int nf = 2 * n;
    std::string o;
    o.reserve((size_t)(30 * N3 + 64) * 21);
    auto es = [](double x) { return ed_es(x, 20, 12); };
    auto i8 = [](long long v) { return ed_i(v, 8); };
    o += i8(N1) + i8(N2) + i8(N3) + '\n';                                                            // 1001
    o += i8(info->ihist) + i8((long long)st->scal[2]) + es(st->scal[1]) + es(st->scal[0]) + '\n';     // 1002
    o += i8(info->ips) + i8(info->ipx) + i8(info->ipy) + i8(info->ipz) + es(props->prm) + '\n';       // 1003
    o += es(info->qvol_ori) + '\n';                                                                  // 1004
    put_list(o, (size_t)(N1 * (N2 + 1) * (N3 + 1)), 5, [&](size_t) { return es(0.0); });             // U
    put_list(o, (size_t)((N1 + 1) * N2 * (N3 + 1)), 5, [&](size_t) { return es(0.0); });             // V
    const size_t rw = (size_t)((N1 + 1) * (N2 + 1));
    put_list(o, rw * (size_t)N3, 5, [&](size_t i) { return es(st->w[1 + i / rw]); });                  // W
    put_list(o, (size_t)(N1M * N2M * N3M), 5, [&](size_t i) { return es(st->p[1 + i]); });             // P
    o += i8(3) + i8(3) + i8(2LL * n + 1) + '\n';                                                      // 1011
    o += es(props->denr) + es(props->visr) + es(props->fr) + es(props->weber) + es(info->fk) + es(props->re) +
         '\n';                                                                                       // 1012
    o += i8(1) + i8(kMMax) + '\n';                                                                    // 1013
    put_list(o, 1, 8, [&](size_t) { return es(st->scal[3]); });                                      // 1014
    std::vector<std::vector<int>> band(kMMax + 1);
    for (int k = -2; k <= nf + 4; ++k) {
        const int m = st->layer[k + kGL];
        if (m >= 1 && m <= kMMax) band[m].push_back(k);
        else if (m != 0) return fail(LICA_BAD_ARG, "lica_col_fld_write: layer outside 0..11", __LINE__);
    }
    put_list(o, kMMax, 8, [&](size_t q) { return i8(4LL * (long long)band[q + 1].size()); });        // 1015
    for (int m = 1; m <= kMMax; ++m)
        for (int k : band[m])
            for (int j = 1; j <= 2; ++j)
                for (int i = 1; i <= 2; ++i) o += i8(i) + i8(j) + i8(k) + es(st->phi[k + kGL]) + '\n';  // 1016
    o += i8(info->contact) + '\n';                                                                    // 1007
    o += i8(info->contact_old) + '\n';
    o += es(info->contact_start) + '\n';                                                              // 1005
    o += es(info->contact_time) + '\n';
    o += i8(info->lvson) + '\n';
    o += es(info->t_con) + '\n';
    if (info->ips == 1) {
        o += es(props->prm) + es(props->scr) + es(props->tcr) + '\n';                                 // 1006
        const size_t rt = (size_t)((N1 + 1) * (N2 + 1));
        put_list(o, rt * (size_t)(N3 + 1), 5, [&](size_t i) { return es(st->t[i / rt]); });           // T
    }
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(LICA_ERR_IO, std::string("cannot create ") + path + ": " + std::strerror(errno), __LINE__);
    const size_t put = std::fwrite(o.data(), 1, o.size(), fp);
    const int closed = std::fclose(fp);
    if (put != o.size() || closed != 0) return fail(LICA_ERR_IO, std::string("write error on ") + path, __LINE__);
    return LICA_OK;
}

int lica_col_fld_dims(const char* path, int32_t* n) {
    if (!path || !n) return fail(LICA_BAD_ARG, "lica_col_fld_dims: null argument", __LINE__);
    Reader R;
    if (!load_lines(path, R.lines, R.err)) return fail(LICA_ERR_IO, R.err, __LINE__);
    std::vector<Value> v;
    if (!R.read(F1001, 3, v, "N1,N2,N3")) return fail(LICA_ERR_IO, R.err, __LINE__);
    if (v[0].i != 2 || v[1].i != 2 || v[2].i < 2 || v[2].i > (1LL << 30))
        return fail(LICA_BAD_ARG,
                    "not a 1-D column: N1,N2,N3 = " + std::to_string(v[0].i) + "," + std::to_string(v[1].i) + "," +
                        std::to_string(v[2].i) + " (a column has N1 = N2 = 2)",
                    __LINE__);
    *n = (int32_t)(v[2].i - 1);
    return LICA_OK;
}

int lica_col_fld_read(const char* path, int32_t n, double length, const lica_col_props* props,
                      const lica_fld_options* opt, lica_col_state* st, lica_fld_info* info) {
    if (!path || n < 1 || !(length > 0.0) || !props || !opt || !state_ok(st) || !info)
        return fail(LICA_BAD_ARG, "lica_col_fld_read: null argument, n < 1 or length <= 0", __LINE__);
    Reader R;
    if (!load_lines(path, R.lines, R.err)) return fail(LICA_ERR_IO, R.err, __LINE__);
    std::vector<Value> v;
#define FLD_READ(fmt, count, what) \
    if (!R.read(fmt, (size_t)(count), v, what)) return fail(LICA_ERR_IO, R.err, __LINE__)
    FLD_READ(F1001, 3, "N1,N2,N3");
    const long long N1 = v[0].i, N2 = v[1].i, N3 = v[2].i;
    if (N1 != 2 || N2 != 2 || N3 != (long long)n + 1)
        return fail(LICA_BAD_ARG,
                    "N1,N2,N3 = " + std::to_string(N1) + "," + std::to_string(N2) + "," + std::to_string(N3) +
                        " is not the column 2,2," + std::to_string(n + 1),
                    __LINE__);
    const int nf = 2 * n;
    *info = lica_fld_info{};
    FLD_READ(F1002, 4, "IHIST,M,TIME,DT_O");
    info->ihist = v[0].i;
    info->m = v[1].i;
    info->time = v[2].r;
    info->dt = v[3].r;
    FLD_READ(F1003, 5, "IPSS,IIPX,IIPY,IIPZ,PRAA");
    info->ips = (int32_t)v[0].i;
    info->ipx = (int32_t)v[1].i;
    info->ipy = (int32_t)v[2].i;
    info->ipz = (int32_t)v[3].i;
    info->pra = v[4].r;
    FLD_READ(F1004, 1, "QVOL_ORI");
    info->qvol_ori = v[0].r;
    FLD_READ(F1005, N1 * (N2 + 1) * (N3 + 1), "U");
    FLD_READ(F1005, (N1 + 1) * N2 * (N3 + 1), "V");
    FLD_READ(F1005, (N1 + 1) * (N2 + 1) * N3, "W");
    for (int k = 0; k <= n + 1; ++k) st->w[k] = 0.0;
    for (long long k = 1; k <= N3; ++k) st->w[k] = v[(size_t)((k - 1) * (N1 + 1) * (N2 + 1) + 1 * (N1 + 1) + 1)].r;
    FLD_READ(F1005, n, "P");
    for (int k = 0; k <= n + 1; ++k) st->p[k] = (k >= 1 && k <= n) ? v[k - 1].r : 0.0;
    FLD_READ(F1001, 3, "N1F,N2F,N3F");
    if (v[0].i != 3 || v[1].i != 3 || v[2].i != 2LL * n + 1)
        return fail(LICA_BAD_ARG,
                    "N1F,N2F,N3F = " + std::to_string(v[0].i) + "," + std::to_string(v[1].i) + "," +
                        std::to_string(v[2].i) + " is not the column's refined grid 3,3," + std::to_string(nf + 1),
                    __LINE__);
    FLD_READ(F1012, 6, "DENR,VISR,FR,SURF_J,FK,RE_AIR");
    info->denr = v[0].r;
    info->visr = v[1].r;
    info->fr = v[2].r;
    info->surf_j = v[3].r;
    info->fk = v[4].r;
    info->re_air = v[5].r;
    FLD_READ(F1013, 2, "NLVS,N_MAX");
    const long long nlvs = v[0].i, nmax = v[1].i;
    if (nlvs != 1 || nmax < 0 || nmax > kMMax)
        return fail(LICA_BAD_ARG,
                    "NLVS,N_MAX = " + std::to_string(nlvs) + "," + std::to_string(nmax) +
                        ": a column holds one level set of at most 11 band layers",
                    __LINE__);
    info->n_max = (int32_t)nmax;
    FLD_READ(F1014, 1, "VOL_TOT_ORI");
    info->vol_tot_ori = v[0].r;
    FLD_READ(F1015, nmax, "NUMA");
    std::vector<long long> numa(nmax + 1, 0);
    for (long long m = 1; m <= nmax; ++m) {
        numa[m] = v[m - 1].i;
        if (numa[m] < 0 || numa[m] > 4LL * (nf + 7))
            return fail(LICA_BAD_ARG, "NUMA(" + std::to_string(m) + ") = " + std::to_string(numa[m]) +
                                          " is more than the column's refined cells", __LINE__);
    }
    for (int q = 0; q < nf + 7; ++q) {
        st->phi[q] = 0.0;
        st->layer[q] = 0;
    }
    std::vector<char> seen11(nf + 7, 0);
    for (long long m = 1; m <= nmax; ++m)
        for (long long c = 0; c < numa[m]; ++c) {
            FLD_READ(F1016, 4, "I,J,K,ALPHI");
            const long long i = v[0].i, j = v[1].i, k = v[2].i;
            if (i < 1 || i > 2 || j < 1 || j > 2 || k < -2 || k > nf + 4)
                return fail(LICA_BAD_ARG,
                            "band cell (" + std::to_string(i) + "," + std::to_string(j) + "," + std::to_string(k) +
                                ") outside the refined column",
                            __LINE__);
            int& lay = st->layer[k + kGL];
            if (lay != 0 && lay != (int)m)
                return fail(LICA_BAD_ARG, "refined cell K = " + std::to_string(k) + " listed in two band layers",
                            __LINE__);
            lay = (int)m;
            if (i == 1 && j == 1) {
                st->phi[k + kGL] = v[3].r;
                seen11[k + kGL] = 1;
            }
        }
    for (int q = 0; q < nf + 7; ++q)
        if (st->layer[q] != 0 && !seen11[q])
            return fail(LICA_BAD_ARG, "band cell K = " + std::to_string(q - kGL) + " has no I = J = 1 entry",
                        __LINE__);
    FLD_READ(F1007, 1, "CONTACT");
    info->contact = (int32_t)v[0].i;
    FLD_READ(F1007, 1, "CONTACT_OLD");
    info->contact_old = (int32_t)v[0].i;
    FLD_READ(F1005, 1, "CONTACT_START");
    info->contact_start = v[0].r;
    FLD_READ(F1005, 1, "CONTACT_TIME");
    info->contact_time = v[0].r;
    FLD_READ(F1007, 1, "LVSON");
    info->lvson = (int32_t)v[0].i;
    FLD_READ(F1005, 1, "T_CON");
    info->t_con = v[0].r;
    // IPS = 1 in the column: T follows when the file says IPSS = 1, else MAKEFLD_TEMP's T = 0
    for (int k = 0; k <= n + 1; ++k) st->t[k] = 0.0;
    if (info->ips == 1) {
        FLD_READ(F1006, 3, "PRM,SCR,TCR");
        info->prm = v[0].r;
        info->scr = v[1].r;
        info->tcr = v[2].r;
        FLD_READ(F1005, (N1 + 1) * (N2 + 1) * (N3 + 1), "T");
        for (long long k = 0; k <= N3; ++k) st->t[k] = v[(size_t)(k * (N1 + 1) * (N2 + 1) + 1 * (N1 + 1) + 1)].r;
    }
#undef FLD_READ
    if (opt->ipzero == 1)
        for (int k = 0; k <= n + 1; ++k) st->p[k] = 0.0;
    // LVSINIT, read branch: ALPHI_BC, then CAL_PSIF(1, N_MAX) with N_MAX = M_MAX (1d.f:137)
    alphi_bc(st->phi, nf, length / nf);
    cal_psif(st->phi, st->layer, nf, st->psif);
    grid_coupling1(n, length, st->psif, st->psi_cn, st->psi_zn);
    for (int k = 0; k <= n + 1; ++k) {
        st->wo[k] = 0.0;
        st->imask[k] = 0;
    }
    for (int q = 0; q < nf + 7; ++q) st->mflvs[q] = 0.0;
    for (int k = 0; k <= nf + 1; ++k) {
        st->sfgas[k] = 0.0;
        st->sfgas2[k] = 0.0;
    }
    st->scal[0] = (opt->idtold == 1) ? info->dt : props->dt0;
    st->scal[1] = (opt->ireset == 1) ? 0.0 : info->time;
    st->scal[2] = 0.0;
    st->scal[3] = info->vol_tot_ori;
    st->scal[4] = info->vol_tot_ori;
    for (int q = 0; q < 8; ++q) st->stats[q] = 0.0;
    return LICA_OK;
}

}  // extern "C"
