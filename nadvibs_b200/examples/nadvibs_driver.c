/* C driver of the Lanczos stage through the C ABI: the sequence of Source/main.f90:61-79.
 *   nadvibs_driver <workdir> [niter]
 * reads <workdir>/basis.in and nadvibs.in, writes output.dat, restart.log, nadvibs.35.0. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nadvibs.h"

static int check(int rc, const char *what) {
    if (rc != NVB_OK) {
        fprintf(stderr, "%s failed (%d): %s\n", what, rc, nvb_last_error());
        exit(1);
    }
    return rc;
}

int main(int argc, char **argv) {
    const char *dir = argc > 1 ? argv[1] : ".";
    char basis[4096], pot[4096], out[4096];
    snprintf(basis, sizeof basis, "%s/basis.in", dir);
    snprintf(pot, sizeof pot, "%s/nadvibs.in", dir);
    snprintf(out, sizeof out, "%s/output.dat", dir);
    nvb_params p;
    check(nvb_read_basis(basis, &p), "nvb_read_basis");
    int64_t niter = argc > 2 ? atoll(argv[2]) : p.niter;
    nvb_options o;
    nvb_options_default(&o);
    nvb_handle *h = NULL;
    check(nvb_create_from_files(basis, pot, &o, &h), "nvb_create_from_files");
    check(nvb_write_header(h, out), "nvb_write_header");
    check(nvb_seed(h, NULL), "nvb_seed");
    double *alpha = malloc(sizeof(double) * (size_t)niter), *beta = malloc(sizeof(double) * (size_t)(niter + 1));
    check(nvb_lanczos(h, niter, alpha, beta), "nvb_lanczos");
    check(nvb_save_restart(h, dir, dir), "nvb_save_restart");
    check(nvb_write_eigenvalues(h, out), "nvb_write_eigenvalues");
    printf("alpha(1) = %.17e  beta(%lld) = %.17e\n", alpha[0], (long long)niter, beta[niter]);
    free(alpha);
    free(beta);
    check(nvb_destroy(h), "nvb_destroy");
    return 0;
}
