/* A plain C caller of libsdot_b200.so: what a C or C++ program (or a cgo / JNI shim) writes against
 * include/sdot_b200.h, with no Python in the process.
 *
 *   c_caller            -> one 2D solve of 2000 uniform seeds (targets 1/n, mass_rtol 1e-8), then prints
 *                          "solve <status> <max |m n - 1|> <launches>"; without a device it prints
 *                          "context <code> <message>" and exits 0 (the library has no CPU fallback).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sdot_b200.h"

int main(void) {
    if (sdot_abi_version() != SDOT_ABI_VERSION) {
        printf("abi %d\n", (int)sdot_abi_version());
        return 1;
    }
    sdot_context ctx;
    sdot_status st;
    memset(&st, 0, sizeof(st));
    int32_t code = sdot_context_create(0, 0, &ctx, &st);
    if (code != SDOT_OK) {
        printf("context %d %s\n", (int)code, st.message);
        return 0;
    }
    const int64_t n = 2000;
    double *pos = malloc(sizeof(double) * 2 * n), *w = calloc(n, sizeof(double)), *m = calloc(n, sizeof(double));
    unsigned long long s = 12345;
    for (int64_t i = 0; i < 2 * n; ++i) {            /* a 64-bit LCG: the seeds need no quality, only spread */
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        pos[i] = (double)(s >> 11) / 9007199254740992.0;
    }
    sdot_solve_desc d;
    memset(&d, 0, sizeof(d));
    d.diagram.dim = 2;
    d.diagram.n = n;
    d.diagram.positions = pos;
    d.diagram.box_hi[0] = d.diagram.box_hi[1] = 1.0;
    d.diagram.density.kind = SDOT_DENSITY_UNIFORM;
    d.diagram.density.value = 1.0;
    d.diagram.memory = SDOT_HOST;
    d.options[SDOT_OPT_TOL_REL] = 1e-8;
    d.options[SDOT_OPT_MAXIT] = 100;
    d.options[SDOT_OPT_MAX_BACKTRACKS] = 60;
    d.options[SDOT_OPT_T_MIN] = 1e-10;
    d.options[SDOT_OPT_MULT_OK] = 4;
    d.options[SDOT_OPT_RESIDUAL] = 1;
    d.options[SDOT_OPT_POWER] = 0.5;
    d.options[SDOT_OPT_SWITCH] = 2;
    d.options[SDOT_OPT_LIN_TOL] = 1e-6;
    d.options[SDOT_OPT_LIN_MAXIT] = 20000;
    d.options[SDOT_OPT_CONTINUATION] = 1;
    d.options[SDOT_OPT_CONV_THRESHOLD] = 1e-2;
    d.options[SDOT_OPT_CONV_RATIO] = sqrt(2.0);
    d.options[SDOT_OPT_LIN_METHOD] = 1;
    d.options[SDOT_OPT_AGG_MARGIN] = 4;
    sdot_solve_out o;
    memset(&o, 0, sizeof(o));
    o.weights = w;
    o.masses = m;
    code = sdot_solve(ctx, &d, &o, &st);
    double worst = 0;
    for (int64_t i = 0; i < n; ++i) worst = fmax(worst, fabs(m[i] * (double)n - 1.0));
    printf("solve %d %d %.3e %llu\n", (int)code, (int)o.stats[0], worst, (unsigned long long)sdot_context_kernel_launches(ctx));
    sdot_context_destroy(ctx);
    free(pos);
    free(w);
    free(m);
    return code == SDOT_OK ? 0 : 2;
}
