// Text outputs in the reference's formats (output.dat header and eigenvalue table).
// The layouts are the drop-in boundary (extract.py:27-42 parses the eigenvalue table), so
// they follow the reference's FORMAT statements (Source/top.f90:248-342, 1051-1113).
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "handle.h"

namespace nvb {

std::string fstr(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return buf;
}

// Fortran Iw: right-justified, asterisks when it does not fit.
std::string fI(int64_t v, int w) {
    std::string s = std::to_string(v);
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}

// Fortran Fw.d
std::string fF(double v, int w, int d) {
    if (!std::isfinite(v)) return std::string(w, '*');
    std::string s = fstr("%.*f", d, v);
    if ((int)s.size() > w) {
        // Fortran drops the leading zero of |v| < 1 before giving up
        if (s.rfind("0.", 0) == 0) s = s.substr(1);
        else if (s.rfind("-0.", 0) == 0) s = "-" + s.substr(2);
        if ((int)s.size() > w) return std::string(w, '*');
    }
    return std::string(w - s.size(), ' ') + s;
}

// Fortran ESw.d: d.dddE+xx; a three-digit exponent drops the letter (d.ddd+xxx).
std::string fES(double v, int w, int d) {
    if (!std::isfinite(v)) return std::string(w, '*');
    std::string s = fstr("%.*E", d, v);
    auto pos = s.find('E');
    int ex = std::atoi(s.c_str() + pos + 1);
    if (std::abs(ex) >= 100) s = s.substr(0, pos) + (ex < 0 ? "-" : "+") + std::to_string(std::abs(ex));
    if ((int)s.size() > w) return std::string(w, '*');
    return std::string(w - s.size(), ' ') + s;
}

static std::string timestamp_line() {
    std::time_t t = std::time(nullptr);
    std::tm tm{};
    localtime_r(&t, &tm);
    static const char *mon[] = {"January", "February", "March", "April", "May", "June", "July",
                                "August", "September", "October", "November", "December"};
    int h = tm.tm_hour;
    const char *ampm = h < 12 ? "AM" : (h == 12 ? "Noon" : "PM");
    int h12 = h % 12 == 0 ? 12 : h % 12;
    return fstr("%2d %s %4d %2d:%02d:%02d.000 %s", tm.tm_mday, mon[tm.tm_mon], tm.tm_year + 1900, h12, tm.tm_min,
                tm.tm_sec, ampm);
}

// print_basis, Source/top.f90:248-342 (memory estimate and GA distribution omitted: one
// device, no Global Arrays).
void write_header(nvb_handle *h, const char *path) {
    FILE *f = std::fopen(path, "w");
    if (!f) fail(NVB_ERR_IO, std::string("cannot write ") + path);
    const auto &p = h->sys.prm;
    const auto &sys = h->sys;
    std::fprintf(f, "NadVibS: nonadiabatic vibronic spectrum simulation package\n");
    std::fprintf(f, "Originate from NADVIBS.X by Michael Schuurman 2007\n\n");
    std::fprintf(f, "%s\n", timestamp_line().c_str());
    std::fprintf(f, "Calculation begins.\n\n");
    std::fprintf(f, "Input parameters read from basis.in:\n");
    std::fprintf(f, "------------------------------------\n");
    std::fprintf(f, "  Number of atoms:                              %s\n", fI(p.natoms, 10).c_str());
    std::fprintf(f, "  Number of electronic states:                  %s\n", fI(p.nstates, 10).c_str());
    std::fprintf(f, "  Order of the expansion:                       %s\n", fI(p.ordr, 10).c_str());
    std::fprintf(f, "  Number of vibrational modes:                  %s\n", fI(p.nmodes, 10).c_str());
    std::fprintf(f, "  Number of irreducible representations         %s\n", fI(p.nirreps, 10).c_str());
    std::string irr;
    for (int64_t i = 0; i < p.nirreps && i < 10; ++i) irr += fI(p.npirr[i], 3);
    std::fprintf(f, "  Number of modes per irrep:                         %s\n", irr.c_str());
    std::fprintf(f, "  Number of Lanczos iterations:                 %s\n", fI(p.niter, 10).c_str());
    std::fprintf(f, "  Number of processors used in execution:       %s\n", fI(1, 10).c_str());
    std::fprintf(f, "  Zero tolerance for potential coeffs.:         %s\n", fES(p.ztoler, 10, 0).c_str());
    std::fprintf(f, "  Compute spin-orbit parameters for first N roots:   %s\n", fI(p.soroots, 5).c_str());
    const bool orthog = p.reorthog > 0, exact = p.reorthog > 1;
    std::fprintf(f, "  Perform lanczos vector re-orthogonalization:       %s\n", orthog ? "    T" : "    F");
    if (orthog) {
        std::fprintf(f, "    - exact dot products for vector orthog.:         %s\n", exact ? "    T" : "    F");
        if (!exact) std::fprintf(f, "    - compute exact orthog. every X iterations: %s\n", fI(p.chkorthog, 10).c_str());
    }
    for (int i = 0; i < sys.S; ++i)
        std::fprintf(f, "  Initial weight of reference state %s:              %s\n", fI(i + 1, 2).c_str(),
                     fF(p.weights[i], 5, 2).c_str());
    std::fprintf(f, "  Convergence criteria for eigenvalues (bji):     %s\n", fES(std::pow(10.0, -(double)p.bconv), 8, 0).c_str());
    std::fprintf(f, "  Number of Segements per Lanczos Vector:        %s\n", fI(p.nseg, 10).c_str());
    std::fprintf(f, "  Dimensionality of a single State Vector:%s\n", fI(sys.dimen, 16).c_str());
    std::fprintf(f, "  Total Dimensionality of H matrix:       %s\n", fI(sys.dimen * sys.S, 16).c_str());
    std::fprintf(f, "  Machine precision for this architecture:%s\n", fES(std::ldexp(1.0, -53), 16, 6).c_str());
    // terms per block and order (Source/top.f90:292-311)
    const int nb = sys.nstblks();
    std::vector<int64_t> ntot((size_t)nb * sys.ordr, 0);
    for (const auto &t : sys.terms) {
        int pord = 0;
        for (int l = 0; l < t.nm; ++l) pord += t.pow[l];
        for (const auto &pr : t.pairs) {
            if (pr.a < pr.b) continue;  // count each block once
            const int blk = (pr.a + 1) * pr.a / 2 + pr.b;
            ntot[(size_t)blk * sys.ordr + pord - 1] += 1;
        }
    }
    std::fprintf(f, " \n  Number of Potential Terms per Block -----------\n \n");
    std::string hdr = "  ORDER:    ";
    for (int i = 1; i <= sys.ordr; ++i) hdr += "    " + fI(i, 2) + "   ";
    std::fprintf(f, "%s\n", hdr.c_str());
    for (int b = 0; b < nb; ++b) {
        std::string row = "  Block " + fI(b + 1, 3) + ":";
        for (int d = 0; d < sys.ordr; ++d) row += fI(ntot[(size_t)b * sys.ordr + d], 6) + "   ";
        std::fprintf(f, "%s\n", row.c_str());
    }
    std::fprintf(f, " \n  Basis set specification:\n");
    std::fprintf(f, "    mode  # func.    omega\n");
    for (int i = 0; i < sys.M; ++i)
        std::fprintf(f, "    %s%s%s\n", fI(i + 1, 3).c_str(), fI(sys.nfunc[i], 7).c_str(),
                     fF(sys.omega[i] * AU2WAVE, 12, 3).c_str());
    std::fprintf(f, " \n \n  Initial state specification:\n");
    std::fprintf(f, "    mode  # quanta   omega\n");
    // only the first excited mode of initstate is kept (Source/top.f90:330-335)
    bool seen = false;
    for (int i = 0; i < sys.M; ++i) {
        int64_t q = p.initstate[i];
        if (q > 0 && !seen) seen = true;
        else q = 0;
        std::fprintf(f, "    %s%s%s\n", fI(i + 1, 3).c_str(), fI(q, 7).c_str(), fF(sys.omega[i] * AU2WAVE, 12, 3).c_str());
    }
    std::fprintf(f, " \n");
    std::fclose(f);
}

// compute_eigenvalues, Source/top.f90:1051-1113.
void write_eigenvalues(nvb_handle *h, const char *path, double seconds) {
    const int64_t n = h->iters;
    if (n < 1) fail(NVB_ERR_STATE, "no Lanczos iterations to diagonalise");
    std::vector<double> E(n), V((size_t)n * n);
    tridiag_eigen(n, h->alpha.data() + 1, h->beta.data() + 1, E.data(), V.data());
    std::vector<double> bji(n), inten(n);
    for (int64_t i = 0; i < n; ++i) {
        bji[i] = std::fabs(h->beta[n] * V[(size_t)i * n + n - 1]);
        inten[i] = V[(size_t)i * n] * V[(size_t)i * n];
    }
    const double bjiconv = std::pow(10.0, -(double)h->sys.prm.bconv);
    const double thresh = 0.0;
    std::vector<int64_t> good{0};
    for (int64_t i = 1; i < n; ++i) {
        if (bji[i] < bjiconv) {
            const int64_t g = good.back();
            if (AU2WAVE * std::fabs(E[i] - E[g]) < thresh) {  // merge of near roots; off with thresh=0
                inten[g] += inten[i];
                if (bji[i] < bji[g]) { inten[i] = inten[g]; good.back() = i; }
            } else good.push_back(i);
        }
    }
    double zpve = 0.0;
    for (double w : h->sys.omega) zpve += w * 0.5;
    double fac = 0.0;
    for (auto g : good)
        if (inten[g] > fac) fac = inten[g];
    FILE *f = std::fopen(path, "a");
    if (!f) fail(NVB_ERR_IO, std::string("cannot append to ") + path);
    std::fprintf(f, "\nCOMPUTED EIGENVALUES \n------------------------------\n\n");
    std::fprintf(f, "  ZPVE from nadvibs.in (reference state): %s cm-1\n", fF(zpve * AU2WAVE, 12, 4).c_str());
    std::fprintf(f, "  FIRST eigenvalue:                       %s cm-1\n", fF(E[good[0]] * AU2WAVE, 12, 4).c_str());
    std::fprintf(f, "  Intensity Factor (MAX Intensity):       %s\n", fF(fac, 12, 8).c_str());
    std::fprintf(f, " \n  Root  Index  Convergence     E(cm-1)        E(eV)     Intensity\n");
    for (size_t k = 0; k < good.size(); ++k) {
        const int64_t g = good[k];
        std::fprintf(f, "%s%s%s%s%s%s\n", fI((int64_t)k + 1, 6).c_str(), fI(g + 1, 7).c_str(), fES(bji[g], 13, 4).c_str(),
                     fF((E[g] - E[good[0]]) * AU2WAVE, 15, 5).c_str(), fF((E[g] - E[0]) * AU2EV, 12, 5).c_str(),
                     fF(fac > 0 ? inten[g] / fac : 0.0, 12, 7).c_str());
    }
    std::fprintf(f, " \n   All requested eigenvalues computed.\n");
    std::fprintf(f, "  Time Required: %s secs.\n", fF(seconds, 14, 5).c_str());
    std::fclose(f);
}

}  // namespace nvb
