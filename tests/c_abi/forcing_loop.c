/*
 * forcing_loop.c — a host written in C against include/hydist_b200.h alone: the set-up of
 * a straight channel reach, the running loop that feeds new boundary tables every step and
 * reads the water level after every step through the host mirror, then the reference's
 * time loop (hyd_run) to a later time with an output callback, and the water budget.
 * Built and run by tests/test_c_abi.py; prints "forcing_loop ok" and exits 0 on success.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hydist_b200.h"

#define CHECK(call)                                                                  \
    do {                                                                             \
        int rc_ = (call);                                                            \
        if (rc_ != HYD_OK) {                                                         \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, hyd_last_error());   \
            exit(1);                                                                 \
        }                                                                            \
    } while (0)

enum { N = 160, M = 40, BANK = 5, HOURS = 3 };
#define TOTAL_TIME (HOURS + 3)

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct Outputs {
    int calls;
    double last_t;
    double zmax;
};

/* hyd_run's output callback: read the level field the way the reference's host appends
 * u, v, z to its lists at every output time */
static int on_output(hyd_handle h, double t, void* user) {
    struct Outputs* o = (struct Outputs*)user;
    static double z[(N + 3) * (M + 3)];
    if (hyd_get_field(h, "z", z, (size_t)(N + 3) * (M + 3)) != HYD_OK) return 1;
    o->calls++;
    o->last_t = t;
    o->zmax = -1e300;
    for (int i = 2; i <= N; i++)
        for (int j = 2; j <= M; j++)
            if (z[i * (M + 3) + j] > o->zmax) o->zmax = z[i * (M + 3) + j];
    return 0;
}

int main(void) {
    const size_t cells = (size_t)(N + 3) * (M + 3);
    HydCaseParams p;
    hyd_params_default(&p);
    p.dX = p.dY = 5.0;
    p.dT = 2.0;
    p.sediment_start = p.bed_change_start = 1e12; /* hydraulics only */
    hyd_params_derive(&p);

    /* the channel: depth 3 m + 1e-4 x along i, dry banks of BANK cells at +2 m; the
       (N, M) map edge-padded to (N+3) x (M+3) as the reference pads its input maps */
    double* f[10];
    for (int k = 0; k < 10; k++) f[k] = (double*)calloc(cells, sizeof(double));
    double *h = f[0], *n = f[1], *visc = f[2];
    for (int i = 0; i < N + 3; i++)
        for (int j = 0; j < M + 3; j++) {
            const int a = clampi(i - 1, 0, N - 1), b = clampi(j - 1, 0, M - 1);
            const int bank = b < BANK || b >= M - BANK;
            h[i * (M + 3) + j] = bank ? -2.0 : 3.0 + 1e-4 * a * p.dX;
            n[i * (M + 3) + j] = 0.025;
            visc[i * (M + 3) + j] = 1e-6;
        }
    const char* names[10] = {"h", "hsnham", "VISCOIDX", "Fw", "Tsxw", "Tsyw", "u", "v", "z", "FS"};

    hyd_handle sim = NULL;
    CHECK(hyd_create(&p, N, M, 0, &sim));
    for (int k = 0; k < 10; k++) CHECK(hyd_set_field(sim, names[k], f[k], cells));

    /* discharge in at the left edge, stage 0 at the right edge, walls elsewhere */
    int btype[4 * HYD_SEGMENT_LIMIT];
    memset(btype, 0, sizeof btype);
    btype[HYD_EDGE_LEFT * HYD_SEGMENT_LIMIT] = 2;
    btype[HYD_EDGE_RIGHT * HYD_SEGMENT_LIMIT] = 1;
    static double tab[4][TOTAL_TIME], cc[4][TOTAL_TIME];
    for (int t = 0; t < TOTAL_TIME; t++) tab[HYD_EDGE_LEFT][t] = 60.0;
    const double* tables[4] = {tab[0], tab[1], tab[2], tab[3]};
    const double* ccs[4] = {cc[0], cc[1], cc[2], cc[3]};
    const int nseg[4] = {1, 1, 1, 1};
    CHECK(hyd_set_boundary(sim, btype, tables, ccs, nseg, TOTAL_TIME));
    CHECK(hyd_init(sim, 0.0));

    /* the running loop: new forcing in before every step, the level out after it */
    const double* view = NULL;
    size_t moved = 0, moved_total = 0;
    CHECK(hyd_mirror_open(sim, "z"));
    for (int k = 0; k < 200; k++) {
        for (int t = 0; t < TOTAL_TIME; t++) tab[HYD_EDGE_LEFT][t] = 60.0 + 0.05 * k;
        CHECK(hyd_update_boundary(sim, tables, ccs));
        CHECK(hyd_step(sim, 1, 0, NULL));
        CHECK(hyd_mirror_update_async(sim, &view, &moved));
        moved_total += moved;
    }
    CHECK(hyd_wait_fields(sim));
    double* z = (double*)malloc(cells * sizeof(double));
    CHECK(hyd_get_field(sim, "z", z, cells));
    if (memcmp(z, view, cells * sizeof(double)) != 0) {
        fprintf(stderr, "the mirror's last copy differs from hyd_get_field\n");
        return 1;
    }
    CHECK(hyd_mirror_close(sim));

    /* the reference's time loop to 2 h with an output every 10 min */
    double vol0[5], b0[HYD_BUDGET_SLOTS];
    CHECK(hyd_mass_balance(sim, vol0, 5));
    CHECK(hyd_mass_budget(sim, b0, HYD_BUDGET_SLOTS));
    struct Outputs out = {0, 0.0, 0.0};
    double t = 0;
    CHECK(hyd_run(sim, 7200.0, 600.0, on_output, &out, &t));
    if (t != 7200.0 || out.calls != 12 || out.last_t != 7200.0 || !(out.zmax > 0)) {
        fprintf(stderr, "hyd_run: t %.1f, %d outputs, last at %.1f, zmax %g\n", t, out.calls, out.last_t, out.zmax);
        return 1;
    }
    double vol1[5], b1[HYD_BUDGET_SLOTS];
    CHECK(hyd_mass_balance(sim, vol1, 5));
    CHECK(hyd_mass_budget(sim, b1, HYD_BUDGET_SLOTS));
    const double dv = vol1[0] - vol0[0];
    const double pred = (b1[0] - b0[0]) + (b1[3] - b0[3]) - (b1[4] - b0[4]) + (b1[5] - b0[5]) + (b1[10] - b0[10]) -
                        (b1[11] - b0[11]);
    const double rel = fabs(dv - pred) / vol1[0];
    if (!(rel <= 1e-10) || vol1[4] != 0) {
        fprintf(stderr, "water budget: dV %.6e, budget %.6e, rel %.3e, non-finite %g\n", dv, pred, rel, vol1[4]);
        return 1;
    }
    CHECK(hyd_destroy(sim));
    printf("forcing_loop ok: t = %.0f s, %d outputs, z max %.4f m, %zu level bytes copied in 200 steps, "
           "budget closure %.2e\n", t, out.calls, out.zmax, moved_total, rel);
    for (int k = 0; k < 10; k++) free(f[k]);
    free(z);
    return 0;
}
