/*
 * A driver in the shape of the reference's examples/synthetic_dmle_test.c
 * (lines 136-285 and 404-494), written against include/exageostat_b200.h
 * only: synthetic field, derivative-free MLE from the lower bounds, kriging
 * of held-out points, the Fisher matrix and MLOE / MMOM.  It shows that a C
 * caller of the reference API compiles and links against the library
 * unchanged.  The reference draws the N(0,1) vector with LAPACKE_dlarnv,
 * which is not part of this library: with a fifth argument the driver reads
 * that vector from a file (one value per line, readObsFile), as a caller
 * holding the reference's draws would; without it the draws come from a
 * Box-Muller transform of rand().  Prints one line "key=value ..." (the
 * log-likelihood at theta0, checksums of z and of the predictions, theta-hat,
 * the MSE, ...) and exits 0 on success.
 *
 *   synthetic_dmle N dts nZmiss seed [nrand_file]
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "exageostat_b200.h"

output results; /* the driver owns it, as examples/examples.c:24 */

static void normals(double *out, int n)
{
    for (int i = 0; i < n; i += 2) {
        const double u1 = (rand() + 1.0) / ((double)RAND_MAX + 2.0), u2 = rand() / ((double)RAND_MAX + 1.0);
        const double r = sqrt(-2.0 * log(u1));
        out[i] = r * cos(6.283185307179586 * u2);
        if (i + 1 < n) out[i + 1] = r * sin(6.283185307179586 * u2);
    }
}

int main(int argc, char **argv)
{
    int N = argc > 1 ? atoi(argv[1]) : 1600, dts = argc > 2 ? atoi(argv[2]) : 320;
    int nZmiss = argc > 3 ? atoi(argv[3]) : 100, seed = argc > 4 ? atoi(argv[4]) : 0;
    int ncores = 1, gpus = 1, lts = 0;
    const int nZobs = N - nZmiss;
    MLE_data data = {0};
    data.computation = "exact";
    data.kernel_fun = "univariate_matern_stationary";
    data.dm = "ed";
    data.precision = 0;
    data.recovery_file = "";
    data.checkpoint_file = "";

    exageostat_init(&ncores, &gpus, &dts, &lts);
    location *l = GenerateXYLoc(N, seed);
    data.l1 = *l;
    double *Nrand;
    if (argc > 5) {
        Nrand = readObsFile(argv[5], N);
        if (!Nrand) {
            fprintf(stderr, "reading %s: %s\n", argv[5], exageostat_last_error());
            return 1;
        }
    } else {
        Nrand = malloc(N * sizeof(double));
        normals(Nrand, N);
    }

    EXAGEOSTAT_dmle_Call(&data, ncores, gpus, dts, 1, 1, N, nZobs, nZmiss);
    double theta0[3] = {1.0, 0.1, 0.5};
    MLE_zvg(&data, Nrand, theta0, N, dts, 0, 1, 1);
    double *z = malloc(N * sizeof(double));
    MLE_get_zobs(&data, z, N);
    double zsum = 0, zsq = 0;
    for (int i = 0; i < N; ++i) {
        zsum += z[i];
        zsq += z[i] * z[i];
    }
    free(z);
    const double loglik0 = MLE_alg(3, theta0, NULL, &data);

    double lb[3] = {0.01, 0.01, 0.01}, ub[3] = {5, 5, 5}, x[3] = {0.01, 0.01, 0.01}, fmax = 0;
    const int evals = exageostat_b200_bobyqa(3, x, lb, ub, 0.0, 0.0, 1e-9, 0, MLE_alg, &data, &fmax);
    if (evals <= 0 || !isfinite(fmax)) {
        fprintf(stderr, "MLE failed: %s\n", exageostat_last_error());
        return 1;
    }

    double *Zobs = malloc(nZobs * sizeof(double)), *Zact = malloc(nZmiss * sizeof(double));
    double *Zmiss = malloc(nZmiss * sizeof(double));
    prediction_init(&data, nZmiss, nZobs, dts, 1, 1, 1);
    pick_random_points(&data, Zobs, Zact, nZmiss, nZobs, N);
    const double mse = EXAGEOSTAT_dmle_Predict_Tile(&data, x, nZmiss, nZobs, Zobs, Zact, Zmiss, N);
    prediction_finalize(&data);
    double pred_sum = 0;
    for (int i = 0; i < nZmiss; ++i) pred_sum += Zmiss[i];

    double *finv = EXAGEOSTAT_Fisher_Tile(&data, N, x, dts, 1, 1);
    if (!finv) {
        fprintf(stderr, "Fisher failed: %s\n", exageostat_last_error());
        return 1;
    }

    mloe_mmom_init(&data, nZmiss, nZobs, dts, 1, 1);
    EXAGEOSTAT_dmle_mloe_mmom_Tile(&data, theta0, x, nZmiss, nZobs, N);
    mloe_mmom_finalize(&data);

    printf("evals=%d loglik0=%.17g zsum=%.17g zsq=%.17g loglik=%.17g theta=%.17g,%.17g,%.17g mse=%.17g "
           "pred_sum=%.17g fisher_inv_diag=%.6e,%.6e,%.6e mloe=%.8f mmom=%.8f\n",
           evals, loglik0, zsum, zsq, fmax, x[0], x[1], x[2], mse, pred_sum, finv[0], finv[4], finv[8], data.mloe,
           data.mmom);
    const int ok = mse >= 0 && isfinite(data.mloe) && isfinite(data.mmom) && finv[0] > 0 && finv[4] > 0 &&
                   finv[8] > 0 && results.fisher_00 == finv[0] && results.mloe == data.mloe;
    free(finv);
    free(Zmiss);
    free(Zact);
    free(Zobs);
    free(Nrand);
    MLE_Finalize(&data);
    exageostat_finalize();
    return ok ? 0 : 1;
}
