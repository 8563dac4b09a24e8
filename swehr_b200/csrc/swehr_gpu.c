/*
 * swehr_gpu.c -- command-line host of libswehr that reads and writes what
 * SWEHR.c's main() reads and writes, so an existing run directory works
 * unchanged:
 *
 *   inputs  (SWEHR.c:468-522, 223-227)  input.txt (14 values), rain.txt,
 *           particlesizein.txt, particlepercentin.txt, topoin.txt (i-major)
 *   console (SWEHR.c:524-535, 695-696, 718, 1413, 1681, 1702)
 *   movies  (SWEHR.c:1679-1698) topomovie.txt depthmovie.txt
 *           velocitymovie.txt cmovie.txt Mmovie.txt: one frame each time t
 *           reaches the next print time (every max(1, tend/1000) s)
 *   results (SWEHR.c:1705-1761) topoout.txt depth.txt uh.txt vh.txt ch.txt
 *           m.txt c.txt vel.txt maxvel.txt maxdepth.txt (rows j, columns i,
 *           %10.10lf), stage.txt (24 columns, %lf), saveflow.txt (18, %lf)
 *
 * The solver loop runs on the GPU through the C ABI of include/swehr.h; the
 * host only steers it to the print times and formats the results.  After a
 * CFL error the reference still finishes the step, records its stage row and
 * movie frame and writes every result file; so does this host.
 *
 *   swehr_gpu [-C dir] [--mixed] [--no-movies] [--dump] [--budget]
 *             [--inflow 0|1] [--bndry a,b,c,d] [--max-steps N]
 *
 * --dump also writes swehr_dump.txt: every state field in %.17g (the format
 * the reference build under oracle/ writes), for bit-level comparisons.
 * Exit status: 0 on a completed run (CFL error included, as the reference),
 * 2 for missing or malformed input files, 3 for a library error.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "swehr.h"

static void die(int code, const char *what, const char *detail)
{
    fprintf(stderr, "swehr_gpu: %s%s%s\n", what, detail ? ": " : "", detail ? detail : "");
    exit(code);
}

static double *read_values(const char *path, long n)
{
    FILE *f = fopen(path, "r");
    if (!f) die(2, "cannot open", path);
    double *v = (double *)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    if (!v) die(3, "out of host memory", path);
    for (long k = 0; k < n; k++)
        if (fscanf(f, "%lf", &v[k]) != 1) {
            fclose(f);
            die(2, "too few values in", path);
        }
    fclose(f);
    return v;
}

static void check(int st, const char *what)
{
    if (st != SWEHR_OK && st != SWEHR_CFL_ERROR && st != SWEHR_NAN) {
        fprintf(stderr, "swehr_gpu: %s: %s (%s)\n", what, swehr_status_str(st), swehr_last_error());
        exit(3);
    }
}

/* one nx*ny field in the reference's text layout: rows j, columns i */
static void write_grid(FILE *f, const double *a, int nx, int ny)
{
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            fprintf(f, i != nx - 1 ? "%10.10lf\t" : "%10.10lf\n", a[(size_t)i * ny + j]);
}

static void read_field(swehr_ctx *c, int field, int k, double *dst)
{
    check(swehr_read_field(c, field, k, dst), "swehr_read_field");
}

static void write_file(const char *name, swehr_ctx *c, int field, int k, double *buf, int nx, int ny)
{
    FILE *f = fopen(name, "w");
    if (!f) die(3, "cannot write", name);
    read_field(c, field, k, buf);
    write_grid(f, buf, nx, ny);
    fclose(f);
}

static void dump_state(swehr_ctx *c, const swehr_params *p, int64_t steps, double t, double *buf,
                       const double *stage, const double *saveflow, int64_t rows)
{
    FILE *f = fopen("swehr_dump.txt", "w");
    if (!f) die(3, "cannot write", "swehr_dump.txt");
    const size_t N = (size_t)p->nx * p->ny;
    fprintf(f, "%d %d %d %ld %.17g\n", p->nx, p->ny, p->sclass, (long)steps, t);
    const int fixed[] = {SWEHR_FIELD_H, SWEHR_FIELD_HU, SWEHR_FIELD_HV, SWEHR_FIELD_Z, SWEHR_FIELD_VINF,
                         SWEHR_FIELD_TOTM, SWEHR_FIELD_DEP, SWEHR_FIELD_TOTSED, SWEHR_FIELD_MAXVEL,
                         SWEHR_FIELD_MAXDEPTH};
    for (size_t m = 0; m < sizeof fixed / sizeof fixed[0]; m++) {
        read_field(c, fixed[m], 0, buf);
        for (size_t q = 0; q < N; q++) fprintf(f, "%.17g\n", buf[q]);
    }
    const int per_class[] = {SWEHR_FIELD_U, SWEHR_FIELD_M, SWEHR_FIELD_SED};
    for (int m = 0; m < 3; m++)
        for (int k = 1; k <= p->sclass; k++) {
            read_field(c, per_class[m], k, buf);
            for (size_t q = 0; q < N; q++) fprintf(f, "%.17g\n", buf[q]);
        }
    fprintf(f, "%ld\n", (long)rows);
    for (int64_t r = 0; r < rows; r++)
        for (int q = 0; q < 24; q++) fprintf(f, "%.17g\n", stage[r * 24 + q]);
    for (int64_t r = 0; r < rows; r++)
        for (int q = 0; q < 18; q++) fprintf(f, "%.17g\n", saveflow[r * 18 + q]);
    fclose(f);
}

int main(int argc, char **argv)
{
    const char *dir = NULL;
    int precision = SWEHR_FP64, movies = 1, dump = 0, budget = 0, inflow = -1, bndry_set = 0;
    int bndry[4] = {0, 0, 0, 0};
    long long max_steps = -1;
    for (int a = 1; a < argc; a++) {
        if (!strcmp(argv[a], "-C") && a + 1 < argc) dir = argv[++a];
        else if (!strcmp(argv[a], "--mixed")) precision = SWEHR_MIXED;
        else if (!strcmp(argv[a], "--no-movies")) movies = 0;
        else if (!strcmp(argv[a], "--dump")) dump = 1;
        else if (!strcmp(argv[a], "--budget")) budget = 1;
        else if (!strcmp(argv[a], "--inflow") && a + 1 < argc) inflow = atoi(argv[++a]) ? 1 : 0;
        else if (!strcmp(argv[a], "--bndry") && a + 1 < argc) {
            if (sscanf(argv[++a], "%d,%d,%d,%d", &bndry[0], &bndry[1], &bndry[2], &bndry[3]) != 4)
                die(2, "--bndry wants four comma-separated 0/1 values", NULL);
            bndry_set = 1;
        } else if (!strcmp(argv[a], "--max-steps") && a + 1 < argc) max_steps = atoll(argv[++a]);
        else {
            fprintf(stderr,
                    "usage: swehr_gpu [-C dir] [--mixed] [--no-movies] [--dump] [--budget] [--inflow 0|1]\n"
                    "                 [--bndry a,b,c,d] [--max-steps N]\n");
            return 2;
        }
    }
    if (dir && chdir(dir) != 0) die(2, "cannot enter", dir);

    /* input.txt: nx ny dx F manning0 tend a ad h0 mtstar0 rnum rint sclass J (SWEHR.c:474-505) */
    double *in = read_values("input.txt", 14);
    swehr_params p;
    swehr_params_default(&p);
    p.nx = (int)in[0]; p.ny = (int)in[1]; p.dx = in[2]; p.F = in[3]; p.manning0 = in[4]; p.tend = in[5];
    p.a = in[6]; p.ad = in[7]; p.h0 = in[8]; p.mtstar0 = in[9]; p.rnum = (int)in[10]; p.rint = in[11];
    p.sclass = (int)in[12]; p.J = in[13];
    free(in);
    if (inflow >= 0) p.inflow = inflow;
    if (bndry_set)
        for (int k = 0; k < 4; k++) p.bndry[k] = bndry[k];
    p.budget = budget;
    if (p.nx < 1 || p.ny < 1 || p.rnum < 1 || p.sclass < 1 || p.sclass > SWEHR_MAX_CLASSES)
        die(2, "input.txt: nx, ny, rnum >= 1 and sclass in 1..16 required", NULL);
    const int nx = p.nx, ny = p.ny, S = p.sclass;
    double *rain = read_values("rain.txt", p.rnum);
    double *ds = read_values("particlesizein.txt", S);
    double *pf = read_values("particlepercentin.txt", S);
    double *topo = read_values("topoin.txt", (long)nx * ny);

    printf("Grid Size (Spacing): %d x %d (%lf)\n", nx, ny, p.dx);
    printf("Number of conserved variables: %d\n", 3 + S);
    printf("Number of particle size classes: %d\n", S);
    printf("H-R Parameters: \n");
    printf("a0: %lf\n", p.a);
    printf("ad0: %lf\n", p.ad);
    printf("F: %lf\n", p.F);
    printf("J: %lf\n", p.J);
    printf("h0: %lf\n", p.h0);
    printf("mtstar0: %lf\n", p.mtstar0);
    printf("b: %lf\n", p.b);
    {
        /* lowest cell of the first row (SWEHR.c:684-696) */
        int outlet = 1;
        double elev = 99999;
        for (int i = 1; i <= nx; i++)
            if (topo[(size_t)(i - 1) * ny] < elev) { elev = topo[(size_t)(i - 1) * ny]; outlet = i; }
        printf("Basin Outlet Pixel: %d\n", outlet);
        printf("Basin Outlet Elevation (m): %lf\n", elev);
        for (int k = 0; k < 6; k++) {
            const int xi = p.xpoint[k] < nx ? p.xpoint[k] : nx, yj = p.ypoint[k] < ny ? p.ypoint[k] : ny;
            printf("Point %d at (%d,%d) has elevation %lf\n", k + 1, xi, yj, topo[(size_t)(xi - 1) * ny + (yj - 1)]);
        }
    }

    swehr_inputs inputs = {topo, rain, ds, pf, NULL, NULL};
    swehr_ctx *ctx = NULL;
    check(swehr_create(&p, &inputs, precision, &ctx), "swehr_create");

    const size_t N = (size_t)nx * ny;
    double *buf = (double *)malloc(N * sizeof(double));
    if (!buf) die(3, "out of host memory", NULL);
    FILE *fm[5] = {NULL, NULL, NULL, NULL, NULL};
    const char *mnames[5] = {"topomovie.txt", "depthmovie.txt", "velocitymovie.txt", "cmovie.txt", "Mmovie.txt"};
    const int mfields[5] = {SWEHR_FIELD_Z, SWEHR_FIELD_H, SWEHR_FIELD_VEL, SWEHR_FIELD_TOTSED, SWEHR_FIELD_TOTM};
    for (int m = 0; m < 5; m++) {   /* the reference creates them whether or not frames follow */
        fm[m] = fopen(mnames[m], "w");
        if (!fm[m]) die(3, "cannot write", mnames[m]);
    }

    const double printint = fmax(1, p.tend / 1000);
    double printinterval = printint;
    const time_t t0 = time(NULL);
    swehr_progress pr;
    memset(&pr, 0, sizeof pr);
    double t = 0;
    int64_t steps = 0;
    int st = SWEHR_OK;
    while (t < p.tend) {
        long long left = max_steps < 0 ? -1 : max_steps - steps;
        if (left == 0) break;
        if (!movies) {
            st = swehr_advance(ctx, INFINITY, left, &pr);
        } else if (t >= printinterval) {
            st = swehr_advance(ctx, INFINITY, 1, &pr);   /* a lagging print time: one step, one frame */
        } else {
            st = swehr_advance(ctx, printinterval, left, &pr);
        }
        check(st, "swehr_advance");
        if (pr.steps == steps && st == SWEHR_OK) break;   /* nothing left to do */
        t = pr.t;
        steps = pr.steps;
        if (st == SWEHR_CFL_ERROR) printf("!!! CFL Error at t=%lf\n", pr.t_step);
        if (movies && t >= printinterval) {
            printf("%lf\t %lf\t %lf\t %lf\n", t, pr.courant, pr.dt, pr.rain);
            printinterval += printint;
            for (int m = 0; m < 5; m++) {
                read_field(ctx, mfields[m], 0, buf);
                write_grid(fm[m], buf, nx, ny);
            }
        }
        if (st != SWEHR_OK) break;
    }
    printf("Elapsed wall clock time: %ld\n", (long)(time(NULL) - t0));
    for (int m = 0; m < 5; m++) fclose(fm[m]);

    write_file("topoout.txt", ctx, SWEHR_FIELD_Z, 0, buf, nx, ny);
    write_file("depth.txt", ctx, SWEHR_FIELD_H, 0, buf, nx, ny);
    write_file("uh.txt", ctx, SWEHR_FIELD_HU, 0, buf, nx, ny);
    write_file("vh.txt", ctx, SWEHR_FIELD_HV, 0, buf, nx, ny);
    write_file("ch.txt", ctx, SWEHR_FIELD_U, 1, buf, nx, ny);
    write_file("m.txt", ctx, SWEHR_FIELD_TOTM, 0, buf, nx, ny);
    write_file("c.txt", ctx, SWEHR_FIELD_TOTSED, 0, buf, nx, ny);
    write_file("vel.txt", ctx, SWEHR_FIELD_VEL, 0, buf, nx, ny);
    write_file("maxvel.txt", ctx, SWEHR_FIELD_MAXVEL, 0, buf, nx, ny);
    write_file("maxdepth.txt", ctx, SWEHR_FIELD_MAXDEPTH, 0, buf, nx, ny);

    /* stage rows: at most one per stageint of simulated time (plus a CFL row) */
    double cap_d = p.stageint > 0 ? p.tend / p.stageint + 8 : 8;
    if (!(cap_d < 100008)) cap_d = 100008;
    const int64_t cap = (int64_t)cap_d;
    double *stage = (double *)malloc((size_t)cap * 24 * sizeof(double));
    double *saveflow = (double *)malloc((size_t)cap * 18 * sizeof(double));
    if (!stage || !saveflow) die(3, "out of host memory", NULL);
    int64_t rows = 0;
    check(swehr_read_series(ctx, stage, saveflow, cap, &rows), "swehr_read_series");
    FILE *f9 = fopen("stage.txt", "w"), *f12 = fopen("saveflow.txt", "w");
    if (!f9 || !f12) die(3, "cannot write", "stage.txt / saveflow.txt");
    for (int64_t r = 0; r < rows; r++)
        for (int q = 0; q < 24; q++) fprintf(f9, q != 23 ? "%lf\t" : "%lf\n", stage[r * 24 + q]);
    for (int64_t r = 0; r < rows; r++)
        for (int q = 0; q < 18; q++) fprintf(f12, q != 17 ? "%lf\t" : "%lf\n", saveflow[r * 18 + q]);
    fclose(f9);
    fclose(f12);

    if (dump) dump_state(ctx, &p, steps, t, buf, stage, saveflow, rows);
    if (budget) {
        swehr_budget b;
        check(swehr_get_budget(ctx, &b), "swehr_get_budget");
        printf("Water budget: now %.17g init %.17g rain %.17g outflow %.17g residual %.3e\n", b.water_now,
               b.water_init, b.rain_in, b.outflow, b.water_residual);
        for (int k = 0; k < S; k++)
            printf("Sediment budget class %d: now %.17g detached %.17g outflow %.17g residual %.3e\n", k + 1,
                   b.sed_now[k], b.detach[k], b.sed_outflow[k], b.sed_residual[k]);
    }
    swehr_destroy(ctx);
    free(stage); free(saveflow); free(buf); free(topo); free(rain); free(ds); free(pf);
    return 0;
}
