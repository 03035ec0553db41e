// Device-side description of the Hamiltonian (built once per handle from the term table).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "nvb_internal.h"

namespace nvb {

constexpr int MAXS = MAX_STATES;
constexpr int ETAB_J = 5;  // |shift| 0..4

// One (term, nonzero shift) combination: y_a += C_ab * prod_l E(p_l, n_l, s_l) * x_b(n+s).
struct DevStep {
    int nm;
    int mode[MAX_ORDER];
    int sig[MAX_ORDER];
    int etab[MAX_ORDER];  // element table row of (power, |shift|); element = E[etab + min(n, n+s)]
    long long stride;     // sum_l s_l * shft(mode_l)
    int term;             // index into the per-term coefficient blocks
    int pad;
};

// A term whose shifts are all zero-able (all powers even): its zero shift is part of the
// diagonal block, applied in the diagonal section (Source/top.f90:731-751).
struct DevDiag {
    int nm;
    int mode[MAX_ORDER];
    int etab[MAX_ORDER];
    int term;
};

struct Plan {
    int S = 0, M = 0, nmax = 0;
    int nsteps = 0, ndiag = 0, nterms = 0;
    long long dimen = 0;
    // host copies
    std::vector<DevStep> h_steps;
    std::vector<DevDiag> h_diag;
    std::vector<double> h_coef;       // [nterms][S][S] dense coupling matrix per term
    std::vector<unsigned long long> h_mask;  // [nterms][2] bit a*S+b set when pair (a,b) exists
    std::vector<double> h_const;      // [S][S] diagonal-section constants (after dblks rules)
    std::vector<int> h_dpair;         // [S][S] 1 when the (a,b) entry of the diagonal block is applied
    std::vector<double> h_etab;       // element table [(p-1)*5+j][nmax]
    std::vector<int> h_nfunc;
    std::vector<long long> h_shft;
    std::vector<double> h_omega;
    // device copies
    DevStep *d_steps = nullptr;
    DevDiag *d_diag = nullptr;
    double *d_coef = nullptr;
    float *d_coef_f = nullptr;
    unsigned long long *d_mask = nullptr;
    double *d_const = nullptr;
    float *d_const_f = nullptr;
    int *d_dpair = nullptr;
    double *d_etab = nullptr;
    float *d_etab_f = nullptr;
    int *d_nfunc = nullptr;
    long long *d_shft = nullptr;
    double *d_omega = nullptr;
    float *d_omega_f = nullptr;
};

void plan_build(Plan &pl, const System &sys, int quirk_cubic, int quirk_lower);
void plan_upload(Plan &pl);
void plan_free(Plan &pl);
double hoelem(int p, int a, int b, int quirk_cubic);

// y = scale * H x; when alpha_part != nullptr also per-block partials of <scale*x, y> (FP64)
// into alpha_part[gridDim.x].  Returns the number of blocks used (for the partial sums).
template <typename T>
int hv_launch(const Plan &pl, const T *x, T *y, const double *scale_dev, double *alpha_part, cudaStream_t st,
              int kernel);
int hv_max_blocks(const Plan &pl, int kernel);

}  // namespace nvb
