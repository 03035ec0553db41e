// Input stage: basis.in namelist, nadvibs.in list-directed coefficients, term compiler.
//
// Formats follow the reference exactly because they are the drop-in boundary:
//  * basis.in  : &NADVIBS namelist, keys/defaults of Source/secondary.f90:835-846;
//  * nadvibs.in: list-directed records of Source/top.f90:122-135;
//  * monomial order within an order d: Source/top.f90:153-168 (first index fastest,
//    k1 >= k2 >= ... >= kd);
//  * merge of identical monomials across blocks and the 1/prod(omega^(p/2)) scaling:
//    Source/top.f90:170-231.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "nvb_internal.h"

namespace nvb {

std::string read_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) fail(NVB_ERR_IO, "cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

int64_t numut(int64_t n, int64_t d) {
    // C(n+d-1, d), Source/function.f90:253-258
    long double r = 1;
    for (int64_t i = 1; i <= d; ++i) r = r * (long double)(n - 1 + i) / (long double)i;
    return (int64_t)std::llround((double)r);
}

std::vector<std::vector<int>> monomials(int nmodes, int order) {
    std::vector<std::vector<int>> out;
    std::vector<int> dig(order, 1);
    dig[0] = 0;
    int64_t cnt = numut(nmodes, order);
    for (int64_t k = 0; k < cnt; ++k) {
        dig[0] += 1;
        for (int l = 0; l + 1 < order; ++l)
            if (dig[l] > nmodes) {
                dig[l] = 1;
                dig[l + 1] += 1;
            }
        for (int l = order - 2; l >= 0; --l)
            if (dig[l] < dig[l + 1]) dig[l] = dig[l + 1];
        out.push_back(dig);
    }
    return out;
}

int64_t npot_of(const nvb_params &p) {
    int64_t per = 0;
    for (int64_t d = 1; d <= p.ordr; ++d) per += numut(p.nmodes, d);
    return per * (p.nstates * (p.nstates + 1) / 2);
}

// ------------------------------------------------------------------ namelist
static std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

static double to_real(const std::string &tok) {
    std::string t = tok;
    for (auto &c : t)
        if (c == 'd' || c == 'D') c = 'e';
    char *end = nullptr;
    double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0') fail(NVB_ERR_IO, "bad number '" + tok + "'");
    return v;
}

static int64_t to_int(const std::string &tok) {
    double v = to_real(tok);
    if (v != std::floor(v)) fail(NVB_ERR_IO, "expected an integer, got '" + tok + "'");
    return (int64_t)v;
}

void parse_basis_text(const std::string &text, nvb_params &p) {
    // strip comments, find the group
    std::string body;
    {
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) {
            auto pos = line.find('!');
            if (pos != std::string::npos) line = line.substr(0, pos);
            body += line + "\n";
        }
    }
    std::string lb = lower(body);
    auto st = lb.find("&nadvibs");
    size_t skip = 8;
    if (st == std::string::npos) {
        st = lb.find("$nadvibs");
        if (st == std::string::npos) fail(NVB_ERR_IO, "basis.in: no &NADVIBS namelist group");
    }
    size_t en = std::string::npos;
    for (size_t i = st + skip; i < lb.size(); ++i) {
        if (lb[i] == '/') { en = i; break; }
        if (lb.compare(i, 4, "&end") == 0 || lb.compare(i, 4, "$end") == 0) { en = i; break; }
    }
    if (en == std::string::npos) fail(NVB_ERR_IO, "basis.in: unterminated &NADVIBS group");
    std::string g = body.substr(st + skip, en - st - skip);
    // tokens: split on whitespace/commas, '=' as its own token
    std::vector<std::string> tok;
    std::string cur;
    auto flush = [&]() { if (!cur.empty()) { tok.push_back(cur); cur.clear(); } };
    for (char c : g) {
        if (std::isspace((unsigned char)c) || c == ',') flush();
        else if (c == '=') { flush(); tok.push_back("="); }
        else cur += c;
    }
    flush();
    // join "name (idx)" written with a space
    std::vector<std::string> t2;
    for (size_t i = 0; i < tok.size(); ++i) {
        if (!t2.empty() && tok[i].size() && tok[i][0] == '(' && i + 1 < tok.size() && tok[i + 1] == "=")
            t2.back() += tok[i];
        else t2.push_back(tok[i]);
    }
    tok.swap(t2);
    int64_t npirr_seen = 0;
    // defaults, Source/secondary.f90:835-843 (npirr(1)=nmodes with the default nmodes=1)
    size_t i = 0;
    while (i < tok.size()) {
        if (i + 1 >= tok.size() || tok[i + 1] != "=") fail(NVB_ERR_IO, "basis.in: expected name= near '" + tok[i] + "'");
        std::string name = lower(tok[i]);
        int64_t idx = 1;
        auto lp = name.find('(');
        if (lp != std::string::npos) {
            auto rp = name.find(')', lp);
            if (rp == std::string::npos) fail(NVB_ERR_IO, "basis.in: bad subscript in " + name);
            idx = to_int(name.substr(lp + 1, rp - lp - 1));
            name = name.substr(0, lp);
        }
        i += 2;
        std::vector<std::string> vals;
        while (i < tok.size() && !(i + 1 < tok.size() && tok[i + 1] == "=")) {
            const std::string &v = tok[i];
            auto star = v.find('*');
            if (star != std::string::npos) {
                int64_t r = to_int(v.substr(0, star));
                for (int64_t k = 0; k < r; ++k) vals.push_back(v.substr(star + 1));
            } else vals.push_back(v);
            ++i;
        }
        if (vals.empty()) fail(NVB_ERR_IO, "basis.in: no value for " + name);
        auto arr_i = [&](int64_t *a, int64_t n) {
            if (idx < 1 || idx - 1 + (int64_t)vals.size() > n) fail(NVB_ERR_IO, "basis.in: too many values for " + name);
            for (size_t k = 0; k < vals.size(); ++k) a[idx - 1 + k] = to_int(vals[k]);
        };
        if (name == "niter") p.niter = to_int(vals[0]);
        else if (name == "natoms") p.natoms = to_int(vals[0]);
        else if (name == "nmodes") p.nmodes = to_int(vals[0]);
        else if (name == "nstates") p.nstates = to_int(vals[0]);
        else if (name == "ordr") p.ordr = to_int(vals[0]);
        else if (name == "restart") p.restart = to_int(vals[0]);
        else if (name == "bconv") p.bconv = to_int(vals[0]);
        else if (name == "idroots") p.idroots = to_int(vals[0]);
        else if (name == "soroots") p.soroots = to_int(vals[0]);
        else if (name == "reorthog") p.reorthog = to_int(vals[0]);
        else if (name == "chkorthog") p.chkorthog = to_int(vals[0]);
        else if (name == "nseg") p.nseg = to_int(vals[0]);
        else if (name == "shiftref") p.shiftref = to_int(vals[0]);
        else if (name == "nirreps") p.nirreps = to_int(vals[0]);
        else if (name == "ztoler") p.ztoler = to_real(vals[0]);
        else if (name == "maxdisk") p.maxdisk = to_real(vals[0]);
        else if (name == "basis") arr_i(p.basis, 100);
        else if (name == "initstate") arr_i(p.initstate, 100);
        else if (name == "npirr") { arr_i(p.npirr, 10); npirr_seen = 1; }
        else if (name == "weights") {
            if (idx < 1 || idx - 1 + (int64_t)vals.size() > 10) fail(NVB_ERR_IO, "basis.in: too many weights");
            for (size_t k = 0; k < vals.size(); ++k) p.weights[idx - 1 + k] = to_real(vals[k]);
        } else fail(NVB_ERR_IO, "basis.in: unknown key '" + name + "'");
    }
    (void)npirr_seen;
    // symmetry conflict resets (Source/secondary.f90:847-851)
    int64_t s = 0;
    for (int k = 0; k < 10; ++k) s += p.npirr[k];
    if (s != p.nmodes) {
        p.nirreps = 1;
        p.npirr[0] = p.nmodes;
    }
    p.idroots = std::llabs(p.idroots);
    p.soroots = std::llabs(p.soroots);
}

// ------------------------------------------------------------------ nadvibs.in
namespace {
struct ListReader {
    std::vector<std::string> lines;
    size_t pos = 0;
    explicit ListReader(const std::string &text) {
        std::istringstream in(text);
        std::string l;
        while (std::getline(in, l)) {
            if (!l.empty() && l.back() == '\r') l.pop_back();
            lines.push_back(l);
        }
    }
    void skip(const char *what) {
        if (pos >= lines.size()) fail(NVB_ERR_IO, std::string("nadvibs.in: end of file before ") + what);
        ++pos;
    }
    void values(int64_t n, std::vector<double> &out, const char *what) {
        int64_t got = 0;
        while (got < n) {
            if (pos >= lines.size())
                fail(NVB_ERR_IO, std::string("nadvibs.in: end of file reading ") + what + " (wanted " +
                                     std::to_string(n) + ", got " + std::to_string(got) + ")");
            std::string l = lines[pos++];
            std::string cur;
            std::vector<std::string> tk;
            for (char c : l) {
                if (std::isspace((unsigned char)c) || c == ',') {
                    if (!cur.empty()) { tk.push_back(cur); cur.clear(); }
                } else cur += c;
            }
            if (!cur.empty()) tk.push_back(cur);
            for (auto &t : tk) {
                if (got >= n) break;
                if (t[0] == '/') return;
                auto star = t.find('*');
                if (star != std::string::npos) {
                    int64_t r = to_int(t.substr(0, star));
                    double v = to_real(t.substr(star + 1));
                    for (int64_t k = 0; k < r && got < n; ++k, ++got) out.push_back(v);
                } else {
                    out.push_back(to_real(t));
                    ++got;
                }
            }
        }
    }
};
}  // namespace

void parse_nadvibs_text(const std::string &text, const nvb_params &p, std::vector<double> &omega,
                        std::vector<double> &concoef, std::vector<double> &pot, std::vector<double> *displaced) {
    ListReader rd(text);
    const int64_t nstblks = p.nstates * (p.nstates + 1) / 2;
    omega.clear(); concoef.clear(); pot.clear();
    rd.skip("frequencies");
    rd.values(p.nmodes, omega, "frequencies");
    for (int64_t b = 0; b < nstblks; ++b) {
        rd.skip("block constant");
        rd.values(1, concoef, "block constant");
        for (int64_t d = 1; d <= p.ordr; ++d) {
            rd.skip("expansion coefficients");
            rd.values(numut(p.nmodes, d), pot, "expansion coefficients");
        }
    }
    // the initial state's frequencies, displacement and Duschinsky matrix (Source/top.f90:130-134)
    if (displaced && p.shiftref != 0) {
        displaced->clear();
        rd.skip("initial-state frequencies");
        rd.values(p.nmodes, *displaced, "initial-state frequencies");
        rd.skip("displacement");
        rd.values(p.nmodes, *displaced, "displacement");
        rd.skip("Duschinsky matrix");
        rd.values(p.nmodes * p.nmodes, *displaced, "Duschinsky matrix");
    }
}

void set_displaced(System &sys, const double *bomega, const double *dvec, const double *tmat) {
    const int M = sys.M;
    for (int i = 0; i < M; ++i)
        if (!(bomega[i] > 0.0) || !std::isfinite(bomega[i]) || !std::isfinite(dvec[i]))
            fail(NVB_ERR_ARG, "initial-state frequencies must be positive and displacements finite");
    for (int i = 0; i < M * M; ++i)
        if (!std::isfinite(tmat[i])) fail(NVB_ERR_ARG, "non-finite Duschinsky matrix");
    sys.bomega.assign(bomega, bomega + M);
    sys.dvec.assign(dvec, dvec + M);
    sys.tmat.assign(tmat, tmat + (size_t)M * M);
    sys.neworigin = true;
}

// ------------------------------------------------------------------ term compiler
void build_system(System &sys, const nvb_params &p, const double *omega, const double *concoef,
                  const double *pot) {
    if (p.nstates < 1 || p.nstates > MAX_STATES) fail(NVB_ERR_ARG, "nstates must be in 1..10");
    if (p.nmodes < 1 || p.nmodes > MAX_MODES) fail(NVB_ERR_ARG, "nmodes must be in 1..64");
    if (p.ordr < 1 || p.ordr > MAX_ORDER) fail(NVB_ERR_ARG, "ordr must be in 1..4 (<m|x^p|n> is tabulated to p=4)");
    sys.prm = p;
    sys.S = (int)p.nstates;
    sys.M = (int)p.nmodes;
    sys.ordr = (int)p.ordr;
    sys.nfunc.assign(p.basis, p.basis + p.nmodes);
    sys.dimen = 1;
    for (auto nf : sys.nfunc) {
        if (nf < 1 || nf > 255) fail(NVB_ERR_ARG, "basis values must be in 1..255");
        if (sys.dimen > (int64_t(1) << 40) / nf) fail(NVB_ERR_ARG, "basis product too large");
        sys.dimen *= nf;
    }
    if (sys.dimen * sys.S > (int64_t(1) << 40)) fail(NVB_ERR_ARG, "vector too large");
    sys.shft.assign(sys.M, 1);
    for (int k = 0; k < sys.M; ++k)
        for (int j = k + 1; j < sys.M; ++j) sys.shft[k] *= sys.nfunc[j];
    // symmetry blocks of the modes (npirr, Source/secondary.f90:396-405) and the initial state:
    // only its first excited mode counts (Source/top.f90:326-334)
    sys.irrep.assign(sys.M, 0);
    {
        int m = 0;
        for (int l = 0; l < 10 && m < sys.M; ++l)
            for (int64_t c = 0; c < p.npirr[l] && m < sys.M; ++c) sys.irrep[m++] = l;
    }
    sys.istate.assign(sys.M, 0);
    for (int i = 0; i < sys.M; ++i)
        if (p.initstate[i] > 0) {
            if (p.initstate[i] > 100) fail(NVB_ERR_ARG, "initstate above 100 quanta");
            sys.istate[i] = p.initstate[i];
            break;
        }
    sys.omega.assign(omega, omega + sys.M);
    for (double w : sys.omega)
        if (!(w > 0.0) || !std::isfinite(w)) fail(NVB_ERR_ARG, "frequencies must be positive and finite");
    const int nb = sys.nstblks();
    sys.concoef.assign(concoef, concoef + nb);
    const int64_t npot = npot_of(p);
    sys.potterms.assign(pot, pot + npot);
    for (double v : sys.potterms)
        if (!std::isfinite(v)) fail(NVB_ERR_ARG, "non-finite expansion coefficient");
    for (double v : sys.concoef)
        if (!std::isfinite(v)) fail(NVB_ERR_ARG, "non-finite constant coefficient");
    sys.pot_offset.assign((size_t)nb * sys.ordr, 0);
    {
        int64_t off = 0;
        for (int b = 0; b < nb; ++b)
            for (int d = 1; d <= sys.ordr; ++d) {
                sys.pot_offset[(size_t)b * sys.ordr + d - 1] = off;
                off += numut(sys.M, d);
            }
    }
    // block k (0-based) -> (i, j), i >= j, k = i(i-1)/2 + j - 1 (Source/top.f90:79-85)
    std::vector<std::pair<int, int>> cp(nb);
    for (int i = 1; i <= sys.S; ++i)
        for (int j = 1; j <= i; ++j) cp[i * (i - 1) / 2 + j - 1] = {i - 1, j - 1};
    struct Tmp {
        std::vector<int> modes, pows, blocks;
        std::vector<double> vals;
        std::vector<int64_t> src;
    };
    std::vector<std::vector<Tmp>> grp(sys.ordr + 1);
    std::vector<std::map<std::vector<int>, size_t>> index(sys.ordr + 1);
    std::vector<std::vector<std::vector<int>>> mons(sys.ordr + 1);
    for (int d = 1; d <= sys.ordr; ++d) mons[d] = monomials(sys.M, d);
    for (int b = 0; b < nb; ++b)
        for (int d = 1; d <= sys.ordr; ++d) {
            const int64_t off = sys.pot_offset[(size_t)b * sys.ordr + d - 1];
            for (size_t k = 0; k < mons[d].size(); ++k) {
                const double v = sys.potterms[off + k];
                if (!(std::fabs(v) >= p.ztoler)) continue;
                const auto &dig = mons[d][k];
                std::vector<int> uniq, cnt;
                for (int m : dig) {
                    auto it = std::find(uniq.begin(), uniq.end(), m);
                    if (it == uniq.end()) { uniq.push_back(m); cnt.push_back(1); }
                    else cnt[it - uniq.begin()] += 1;
                }
                const int c = (int)uniq.size();
                std::vector<int> key(uniq);
                key.insert(key.end(), cnt.begin(), cnt.end());
                auto f = index[c].find(key);
                if (f == index[c].end()) {
                    index[c][key] = grp[c].size();
                    grp[c].push_back(Tmp{uniq, cnt, {b}, {v}, {off + (int64_t)k}});
                } else {
                    auto &t = grp[c][f->second];
                    t.blocks.push_back(b);
                    t.vals.push_back(v);
                    t.src.push_back(off + (int64_t)k);
                }
            }
        }
    sys.terms.clear();
    for (int c = 1; c <= sys.ordr; ++c)
        for (auto &t : grp[c]) {
            Term T;
            T.nm = c;
            double dval = 1.0;
            for (int l = 0; l < c; ++l) {
                T.mode[l] = t.modes[l] - 1;
                T.pow[l] = t.pows[l];
                dval = dval / std::sqrt(std::pow(sys.omega[T.mode[l]], (double)T.pow[l]));
            }
            for (size_t q = 0; q < t.blocks.size(); ++q) {
                auto [r, col] = cp[t.blocks[q]];
                T.pairs.push_back({r, col, t.vals[q] * dval});
                T.src.push_back(t.src[q]);
                if (r != col) {
                    T.pairs.push_back({col, r, t.vals[q] * dval});
                    T.src.push_back(t.src[q]);
                }
            }
            sys.terms.push_back(std::move(T));
        }
}

}  // namespace nvb
