/*
 * Host-side synthetic-data helpers of the reference driver workflow
 * (misc/compute/MLE_misc.c).  They consume the libc rand() stream in the
 * reference's order, so a driver that calls GenerateXYLoc(N, seed) and later
 * pick_random_points() sees the same locations and the same hold-out split.
 * Also the real-data flat-file readers of the reference's CSV drivers
 * (misc/compute/flat_file.c, countlines in misc/compute/MLE_misc.c).
 */
#include <math.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/exageostat_b200.h"

/* MLE_misc.c:753-761 */
extern "C" double uniform_distribution(double rangeLow, double rangeHigh)
{
    const double u = (double)rand() / (double)(1.0 + RAND_MAX);
    const double range = rangeHigh - rangeLow;
    return u * range + rangeLow;
}

/* Morton codes on 16-bit quantised coordinates (MLE_misc.c:225-296). */
static uint32_t xg_spread16(uint32_t v)
{
    v &= 0x0000ffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

static uint32_t xg_compact16(uint32_t v)
{
    v &= 0x55555555u;
    v = (v | (v >> 1)) & 0x33333333u;
    v = (v | (v >> 2)) & 0x0f0f0f0fu;
    v = (v | (v >> 4)) & 0x00ff00ffu;
    v = (v | (v >> 8)) & 0x0000ffffu;
    return v;
}

/* MLE_misc.c:297-319: sort by Morton code of (round(x * 65535), round(y *
 * 65535)) and replace the coordinates by their quantised values. */
static void xg_zsort_quantise(int n, double *x, double *y)
{
    std::vector<uint32_t> code((size_t)n);
    for (int i = 0; i < n; ++i) {
        const uint16_t qx = (uint16_t)(x[i] * (double)UINT16_MAX + .5);
        const uint16_t qy = (uint16_t)(y[i] * (double)UINT16_MAX + .5);
        code[i] = (xg_spread16(qy) << 1) + xg_spread16(qx);
    }
    std::sort(code.begin(), code.end());
    for (int i = 0; i < n; ++i) {
        x[i] = (double)(uint16_t)xg_compact16(code[i]) / (double)UINT16_MAX;
        y[i] = (double)(uint16_t)xg_compact16(code[i] >> 1) / (double)UINT16_MAX;
    }
}

/* MLE_misc.c:763-792 */
extern "C" location *GenerateXYLoc(int n, int seed)
{
    srand((unsigned)seed);
    location *loc = (location *)malloc(sizeof(location));
    loc->x = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    loc->y = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    loc->z = NULL;
    const int side = (int)ceil(sqrt((double)n));
    int idx = 0;
    for (int i = 0; i < side && idx < n; ++i)
        for (int j = 0; j < side && idx < n; ++j) {
            const double gx = (double)(i + 1);
            const double gy = (double)(j + 1);
            loc->x[idx] = (gx - 0.5 + uniform_distribution(-0.4, 0.4)) / side;
            loc->y[idx] = (gy - 0.5 + uniform_distribution(-0.4, 0.4)) / side;
            ++idx;
        }
    xg_zsort_quantise(n, loc->x, loc->y);
    return loc;
}

/* MLE_misc.c:1238-1259 */
extern "C" void shuffle(double *array, location *locations, size_t n)
{
    if (n <= 1) return;
    for (size_t i = 0; i < n - 1; ++i) {
        const size_t j = i + (size_t)rand() / (RAND_MAX / (n - i) + 1);
        std::swap(array[i], array[j]);
        std::swap(locations->x[i], locations->x[j]);
        std::swap(locations->y[i], locations->y[j]);
    }
}

/* MLE_misc.c:405-441: MSD binary radix sort over interleaved bits, highest
 * bit first, dimension ndim-1 first within a bit; the partition order
 * (zeros ascending from lo, ones descending from hi) is kept so equal keys
 * land where the reference puts them. */
static void xg_radix(const uint32_t *keys, int count, int ndim, int *order, int *tmp, int sdim, int sbit, int lo,
                     int hi)
{
    int lo_last = lo, hi_last = hi;
    const uint32_t *k = keys + (size_t)sdim * count;
    const uint32_t mask = 1u << sbit;
    for (int i = lo; i <= hi; ++i) {
        if ((k[order[i]] & mask) == 0)
            tmp[lo_last++] = order[i];
        else
            tmp[hi_last--] = order[i];
    }
    for (int i = lo; i <= hi; ++i) order[i] = tmp[i];
    int nd = sdim - 1, nb = sbit;
    if (sdim == 0) {
        if (sbit == 0) return;
        nd = ndim - 1;
        nb = sbit - 1;
    }
    if (lo_last - lo > 1) xg_radix(keys, count, ndim, order, tmp, nd, nb, lo, lo_last - 1);
    if (hi - hi_last > 1) xg_radix(keys, count, ndim, order, tmp, nd, nb, hi_last + 1, hi);
}

/* MLE_misc.c:453-534 */
extern "C" int locations_obs_zsort_inplace(int n, location *locations, double *z)
{
    if (n <= 0) return 0;
    const int ndim = 2;
    const double *coord[2] = {locations->x, locations->y};
    double lo[2], hi[2];
    for (int d = 0; d < ndim; ++d) {
        lo[d] = hi[d] = coord[d][0];
        for (int j = 1; j < n; ++j) {
            if (lo[d] > coord[d][j])
                lo[d] = coord[d][j];
            else if (hi[d] < coord[d][j])
                hi[d] = coord[d][j];
        }
    }
    std::vector<uint32_t> keys((size_t)ndim * n);
    for (int d = 0; d < ndim; ++d) {
        const double range = hi[d] - lo[d];
        for (int j = 0; j < n; ++j) keys[(size_t)d * n + j] = (uint32_t)((coord[d][j] - lo[d]) / range * UINT32_MAX);
    }
    std::vector<int> order((size_t)n), tmp((size_t)n);
    for (int j = 0; j < n; ++j) order[j] = j;
    xg_radix(keys.data(), n, ndim, order.data(), tmp.data(), ndim - 1, 31, 0, n - 1);
    std::vector<double> nx((size_t)n), ny((size_t)n), nz((size_t)n);
    for (int j = 0; j < n; ++j) {
        nx[j] = locations->x[order[j]];
        ny[j] = locations->y[order[j]];
        nz[j] = z[order[j]];
    }
    memcpy(locations->x, nx.data(), sizeof(double) * n);
    memcpy(locations->y, ny.data(), sizeof(double) * n);
    memcpy(z, nz.data(), sizeof(double) * n);
    return 0;
}

/* MLE_misc.c:1700-1741: z comes from MLE_get_zobs (the synthetic field);
 * data->lmiss.{x,y} and data->lobs.{x,y} point into two malloc'd N-arrays
 * (lobs = lmiss + nZmiss), as in the reference. */
extern "C" void pick_random_points(MLE_data *data, double *Zobs, double *Zactual, int nZmiss, int nZobs, int N)
{
    std::vector<double> Z((size_t)N);
    location l;
    l.x = (double *)malloc(sizeof(double) * (size_t)N);
    l.y = (double *)malloc(sizeof(double) * (size_t)N);
    l.z = NULL;
    MLE_get_zobs(data, Z.data(), N);
    for (int i = 0; i < N; ++i) {
        l.x[i] = data->l1.x[i];
        l.y[i] = data->l1.y[i];
    }
    shuffle(Z.data(), &l, (size_t)N);
    for (int i = 0; i < nZobs; ++i) Zobs[i] = Z[nZmiss + i];
    for (int i = 0; i < nZmiss; ++i) Zactual[i] = Z[i];
    data->lmiss.x = l.x;
    data->lmiss.y = l.y;
    data->lmiss.z = NULL;
    data->lobs.x = &l.x[nZmiss];
    data->lobs.y = &l.y[nZmiss];
    data->lobs.z = NULL;
    locations_obs_zsort_inplace(nZobs, &data->lobs, Zobs);
    locations_obs_zsort_inplace(nZmiss, &data->lmiss, Zactual);
}

/* MLE_misc.c:1261-1285: shuffle of the two variables of a bivariate field
 * and their locations with one draw per step, as shuffle does. */
extern "C" void shuffle2(double *array, double *array2, location *locations, size_t n)
{
    if (n <= 1) return;
    for (size_t i = 0; i < n - 1; ++i) {
        const size_t j = i + (size_t)rand() / (RAND_MAX / (n - i) + 1);
        std::swap(array[i], array[j]);
        std::swap(array2[i], array2[j]);
        std::swap(locations->x[i], locations->x[j]);
        std::swap(locations->y[i], locations->y[j]);
    }
}

/* MLE_misc.c:1744-1810: the bivariate hold-out.  N is the matrix dimension (2
 * x locations); nZmiss and nZobs count locations.  z is split into its two
 * variables, locations and both variables are shuffled together, and the
 * first nZmiss locations are missing; Zactual and Zobs interleave the two
 * variables again.  No Morton re-sort (the reference has it commented out). */
extern "C" void pick_random_points2(MLE_data *data, double *Zobs, double *Zactual, int nZmiss, int nZobs, int N)
{
    const int nloc = N / 2;
    std::vector<double> Z((size_t)N), Z1((size_t)nloc), Z2((size_t)nloc);
    location l;
    l.x = (double *)malloc(sizeof(double) * (size_t)nloc);
    l.y = (double *)malloc(sizeof(double) * (size_t)nloc);
    l.z = NULL;
    MLE_get_zobs(data, Z.data(), N);
    for (int i = 0; i < nloc; ++i) {
        Z1[i] = Z[2 * (size_t)i];
        Z2[i] = Z[2 * (size_t)i + 1];
        l.x[i] = data->l1.x[i];
        l.y[i] = data->l1.y[i];
    }
    shuffle2(Z1.data(), Z2.data(), &l, (size_t)nloc);
    for (int i = 0; i < nZmiss; ++i) {
        Zactual[2 * i] = Z1[i];
        Zactual[2 * i + 1] = Z2[i];
    }
    for (int i = 0; i < nZobs; ++i) {
        Zobs[2 * i] = Z1[nZmiss + i];
        Zobs[2 * i + 1] = Z2[nZmiss + i];
    }
    data->lmiss.x = l.x;
    data->lmiss.y = l.y;
    data->lmiss.z = NULL;
    data->lobs.x = &l.x[nZmiss];
    data->lobs.y = &l.y[nZmiss];
    data->lobs.z = NULL;
}

/* ------------------------------------------------------------------------- */
/* real-data flat files (misc/compute/flat_file.c, misc/compute/MLE_misc.c)  */
/* ------------------------------------------------------------------------- */

/* MLE_misc.c:965-985: the number of '\n' characters in the file (so a last
 * line without a newline is not counted), 0 if it cannot be opened. */
extern "C" int countlines(char *filename)
{
    FILE *fp = fopen(filename, "r");
    if (!fp) {
        fprintf(stderr, "cannot open locations file\n");
        return 0;
    }
    int lines = 0, ch;
    while ((ch = fgetc(fp)) != EOF)
        if (ch == '\n') ++lines;
    fclose(fp);
    return lines;
}

/* Reads n rows of nf comma-separated numbers (the field values the
 * reference's strtok + atof loop takes, flat_file.c:38-45) into cols[0..nf).
 * Blank lines are skipped.  Unlike the reference, which writes past the n
 * entries it allocated when the file is longer and dereferences NULL on a
 * short line, reading stops after n rows and a short, missing or malformed
 * row is an error.  Returns 0, or -1 with a message. */
static int xg_read_rows(const char *path, int n, int nf, double **cols, const char *who)
{
    FILE *fp = fopen(path, "r");
    if (!fp) {
        fprintf(stderr, "%s: cannot open %s\n", who, path);
        return -1;
    }
    char *line = nullptr;
    size_t cap = 0;
    int row = 0, lineno = 0, rc = 0;
    while (row < n && getline(&line, &cap, fp) != -1) {
        ++lineno;
        const char *p = line;
        while (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n') ++p;
        if (!*p) continue;
        for (int f = 0; f < nf; ++f) {
            char *end = nullptr;
            const double v = strtod(p, &end);
            if (end == p) {
                fprintf(stderr, "%s: %s line %d: expected %d comma-separated numbers\n", who, path, lineno, nf);
                rc = -1;
                break;
            }
            cols[f][row] = v;
            p = end;
            if (f + 1 < nf) {
                while (*p == ' ' || *p == '\t') ++p;
                if (*p != ',') {
                    fprintf(stderr, "%s: %s line %d: expected %d comma-separated numbers\n", who, path, lineno, nf);
                    rc = -1;
                    break;
                }
                ++p;
            }
        }
        if (rc) break;
        ++row;
    }
    free(line);
    fclose(fp);
    if (!rc && row < n) {
        fprintf(stderr, "%s: %s holds %d rows, %d requested\n", who, path, row, n);
        rc = -1;
    }
    return rc;
}

static location *xg_read_locations(char *path, int n, int dims, const char *who)
{
    if (n <= 0) {
        fprintf(stderr, "%s: n = %d\n", who, n);
        return nullptr;
    }
    location *l = (location *)calloc(1, sizeof(location));
    double *cols[3] = {nullptr, nullptr, nullptr};
    for (int f = 0; f < dims && l; ++f) cols[f] = (double *)malloc((size_t)n * sizeof(double));
    bool ok = l != nullptr;
    for (int f = 0; f < dims; ++f) ok = ok && cols[f] != nullptr;
    if (ok && xg_read_rows(path, n, dims, cols, who) == 0) {
        l->x = cols[0];
        l->y = cols[1];
        l->z = cols[2];
        return l;
    }
    for (int f = 0; f < dims; ++f) free(cols[f]);
    free(l);
    return nullptr;
}

/* flat_file.c:23-64: n two-column rows "x,y" -> a malloc'd location (z = NULL). */
extern "C" location *readLocsFile(char *locs_file, int n) { return xg_read_locations(locs_file, n, 2, "readLocsFile"); }

/* flat_file.c:68-111: n rows "x,y,z". */
extern "C" location *readLocsFile3d(char *locs_file, int n)
{
    return xg_read_locations(locs_file, n, 3, "readLocsFile3d");
}

static double *xg_read_column(char *path, int n, const char *who)
{
    if (n <= 0) {
        fprintf(stderr, "%s: n = %d\n", who, n);
        return nullptr;
    }
    double *v = (double *)malloc((size_t)n * sizeof(double));
    if (v && xg_read_rows(path, n, 1, &v, who) == 0) return v;
    free(v);
    return nullptr;
}

/* flat_file.c:115-142: one value per line. */
extern "C" double *readObsFile(char *obsfile, int n) { return xg_read_column(obsfile, n, "readObsFile"); }

/* flat_file.c:146-171: one time value per line (space-time data). */
extern "C" double *readTimeFile(char *timefile, int n) { return xg_read_column(timefile, n, "readTimeFile"); }
