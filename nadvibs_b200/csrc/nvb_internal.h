// Internal declarations of libnadvibs_gpu.so (host side).
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/nadvibs.h"

namespace nvb {

constexpr double AU2WAVE = 219474.6313705;  // Source/progdata.f90:7
constexpr double AU2EV = 27.211384523;      // Source/progdata.f90:8
constexpr int MAX_ORDER = 4;    // <m|x^p|n> is tabulated for p <= 4 (Source/function.f90:196-248)
constexpr int MAX_STATES = 10;  // weights(10) in the namelist
constexpr int MAX_MODES = 64;

struct Error {
    int code;
    std::string msg;
};
[[noreturn]] void fail(int code, const std::string &msg);
void set_error(const std::string &msg);

// One state-pair coupling of a monomial: y_a += coef * M x_b.
struct Pair {
    int a, b;     // 0-based states
    double coef;  // scaled by 1/prod(omega^(p/2)) (Source/top.f90:216)
};

// A merged monomial prod_l x_{mode[l]}^{pow[l]} with its block pairs, in the reference's
// term order (grouped by the number of distinct modes, Source/top.f90:199-231).
struct Term {
    int nm = 0;
    int mode[MAX_ORDER] = {0, 0, 0, 0};  // 0-based, decreasing
    int pow[MAX_ORDER] = {0, 0, 0, 0};
    std::vector<Pair> pairs;
    // index of each (block, order, monomial) coefficient feeding this term
    std::vector<int64_t> src;  // potterms index per pair (both orders of a block share it)
};

// The input of the stage: namelist + coefficients, and the merged term table.
struct System {
    nvb_params prm{};
    int S = 0, M = 0, ordr = 0;
    std::vector<int64_t> nfunc;       // [M]
    std::vector<int64_t> shft;        // [M], last mode fastest
    int64_t dimen = 0;
    std::vector<double> omega;        // [M] hartree
    std::vector<double> concoef;      // [nstblks]
    std::vector<double> potterms;     // file layout [block][order][monomial]
    std::vector<int64_t> pot_offset;  // [nstblks*ordr] start of each (block, order)
    std::vector<Term> terms;
    // displaced / Duschinsky seed (shiftref != 0, Source/secondary.f90:372-726)
    bool neworigin = false;
    std::vector<double> bomega, dvec, tmat;  // initial-state frequencies, displacement, T (column-major)
    std::vector<int> irrep;                  // symmetry block of every mode (npirr)
    std::vector<int64_t> istate;             // initial-state quanta, at most one mode excited
    int nstblks() const { return S * (S + 1) / 2; }
};

// Parsing / term compilation (input.cpp)
void parse_basis_text(const std::string &text, nvb_params &p);
void parse_nadvibs_text(const std::string &text, const nvb_params &p, std::vector<double> &omega,
                        std::vector<double> &concoef, std::vector<double> &pot,
                        std::vector<double> *displaced = nullptr);  // bomega | dvec | tmat when shiftref != 0
void set_displaced(System &sys, const double *bomega, const double *dvec, const double *tmat);
std::string read_file(const std::string &path);
int64_t numut(int64_t n, int64_t d);
std::vector<std::vector<int>> monomials(int nmodes, int order);  // file order, 1-based digits
void build_system(System &sys, const nvb_params &p, const double *omega, const double *concoef,
                  const double *pot);
int64_t npot_of(const nvb_params &p);

// Spectrum post-step (spectrum.cu)
void convolve_lines(const double *c, const double *h, int64_t n, const double *grid, int64_t ng, double width,
                    int64_t shape, double *out);

// Tridiagonal eigensolver (tridiag.cpp)
void tridiag_eigen(int64_t n, const double *diag, const double *codiag, double *eig, double *vect);

}  // namespace nvb
