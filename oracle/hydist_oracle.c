/*
 * hydist_oracle.c — CPU oracle for the GPU-hydist ADI hot path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline).  The product
 * library never links or calls this file.
 *
 * Each function restates one reference kernel (file:line given beside it) as loop
 * nests over the threads the reference launches.  Two execution rules decide the
 * reference's intra-kernel races; both are what a converged warp does and what
 * the reference's own kernels do when executed thread by thread in launch order
 * (the CPU emulation build of oracle/ref_harness.cpp):
 *   (1) a later statement of the kernel body overwrites an earlier one, even when
 *       different threads execute them (the segment end-row overrides of
 *       _calculate_matrix_coeff, UVZSolver_multithread.cu:469-592);
 *   (2) within one kernel, a thread for a smaller line index runs before a
 *       larger one (the last-cell velocity of the extract kernels reads the
 *       freshly written neighbour, UVZSolver_multithread.cu:659,720).
 * Kernels launched with 32 redundant threads per line run once per line.
 * Arithmetic is written in the reference's operand order and compiled without
 * FMA contraction, so that it is bit-identical to the reference compiled the
 * same way.
 *
 * The scratch arrays of Array_Pointers (constant.cuh:22-29) are persistent and
 * indexed exactly as in the reference, because the reference reads stale scratch
 * in a few degenerate cases (single-cell segments on an open edge).
 */
#include "hydist_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SEGL HYD_SEGMENT_LIMIT
#define PI_REF 3.14159265359 /* constant.cuh:3 */
#define EPS_REF 1e-16        /* UVZSolver_multithread.cu:12 */
#define BED_LIMIT 0.1        /* the library's fed-back bed change limit, a fraction of the depth */
#define BED_CAP 0.05         /* and in metres */

struct OraSim {
    HydCaseParams P;
    int N, M, W;
    size_t nf;
    double *h, *hsnham, *VISCOIDX, *Fw, *Tsxw, *Tsyw, *u, *v, *z, *t_u, *t_v, *t_z, *Htdu, *Htdv,
        *H_moi, *htaiz, *htaiz_bd, *Kx1, *Ky1, *FS, *tFS, *VTH, *Kx, *Ky, *Qbx, *Qby, *dH;
    double *h0, *dHc; /* morphodynamic feedback: h = h0 + dH, dH's Kahan compensation */
    double* dHinc;    /* feedback: the update's unfiltered bed change (NaN where none) */
    int* khouot;
    int *daui, *cuoii, *moci, *dauj, *cuoij, *mocj;
    double *ubt, *ubp, *vbt, *vbd, *hi;
    double hmax_u, hmax_d, hmax_l, hmax_r;
    int bienQ[4];
    int boundary_type[4 * SEGL];
    double *bc[4], *cc[4];
    int total_time;
    /* Array_Pointers scratch */
    double *a1, *b1, *c1, *d1, *a2, *c2, *d2, *f1, *f2, *f3, *f5;
    double *AA, *BB, *CC, *DD, *x, *Ap, *Bp, *ep;
    int* SN;
    /* derived device helpers (constant.cuh:126-133) */
    double windx, windy, ufr, dxr, wss;
    double t;
    int start_idx, end_idx; /* Engine.py loop variables that reach BedLoad (Engine.py:366) */
    int overflow;
    /* water account (ora_water_enable): caller-owned sums, the half-step's old levels and
       the mask and depths before the reset */
    double* water;
    double *w_zold, *w_H;
    int* w_kh;
    void* mem[96];
    int nmem;
};

/* ------------------------------------------------------------------ memory */

static void* ora_alloc(OraSim* s, size_t count, size_t elem, size_t guard) {
    char* base = (char*)calloc(count + 2 * guard, elem);
    if (!base) return NULL;
    s->mem[s->nmem++] = base;
    return base + guard * elem;
}

void ora_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void ora_derived_constants(const HydCaseParams* p, double* out) {
    /* constant.cuh:126-133 */
    out[0] = 0.0013 * (0.00075 + 0.000067 * fabs(p->Wind)) * fabs(p->Wind) * p->Wind *
             cos(p->huonggio * (PI_REF / 180));
    out[1] = 0.0013 * (0.00075 + 0.000067 * fabs(p->Wind)) * fabs(p->Wind) * p->Wind *
             sin(p->huonggio * (PI_REF / 180));
    out[2] = 0.25 * pow((p->Sx - 1) * p->g, 8.0 / 15.0) * pow(p->dm, 9.0 / 15.0) *
             pow(p->muy, -1.0 / 15.0);
    out[3] = p->dm * pow(p->g * (p->Sx - 1) / p->muy * p->muy, (1.0 / 3.0));
    out[4] = 10 * p->muy / p->dm *
             (sqrt(1 + 0.01 * (p->Sx - 1) * 9.81 * pow(p->dm, 3) / pow(p->muy, 2)) - 1);
}

OraSim* ora_create(const HydCaseParams* p, int N, int M) {
    if (N < 4 || M < 4) return NULL;
    OraSim* s = (OraSim*)calloc(1, sizeof(OraSim));
    if (!s) return NULL;
    s->P = *p;
    s->N = N;
    s->M = M;
    s->W = M + 3;
    s->nf = (size_t)(N + 3) * (M + 3);
    const size_t nf = s->nf;
    const size_t G = 4 * (size_t)(M + 3) + 64; /* guard: the reference reads a few cells outside */
    double** fields[] = {&s->h,     &s->hsnham, &s->VISCOIDX, &s->Fw,    &s->Tsxw,     &s->Tsyw,
                         &s->u,     &s->v,      &s->z,        &s->t_u,   &s->t_v,      &s->t_z,
                         &s->Htdu,  &s->Htdv,   &s->H_moi,    &s->htaiz, &s->htaiz_bd, &s->Kx1,
                         &s->Ky1,   &s->FS,     &s->tFS,      &s->VTH,   &s->Kx,       &s->Ky,
                         &s->Qbx,   &s->Qby,    &s->dH,       &s->h0,    &s->dHc,      &s->dHinc};
    for (size_t k = 0; k < sizeof(fields) / sizeof(fields[0]); k++) {
        *fields[k] = (double*)ora_alloc(s, nf, sizeof(double), G);
        if (!*fields[k]) goto fail;
    }
    s->khouot = (int*)ora_alloc(s, nf, sizeof(int), G);
    s->daui = (int*)ora_alloc(s, (size_t)(N + 2) * SEGL, sizeof(int), 2 * SEGL);
    s->cuoii = (int*)ora_alloc(s, (size_t)(N + 2) * SEGL, sizeof(int), 2 * SEGL);
    s->moci = (int*)ora_alloc(s, (size_t)(N + 2), sizeof(int), 8);
    s->dauj = (int*)ora_alloc(s, (size_t)(M + 2) * SEGL, sizeof(int), 2 * SEGL);
    s->cuoij = (int*)ora_alloc(s, (size_t)(M + 2) * SEGL, sizeof(int), 2 * SEGL);
    s->mocj = (int*)ora_alloc(s, (size_t)(M + 2), sizeof(int), 8);
    s->ubt = (double*)ora_alloc(s, (size_t)(M + 2), sizeof(double), 8);
    s->ubp = (double*)ora_alloc(s, (size_t)(M + 2), sizeof(double), 8);
    s->vbt = (double*)ora_alloc(s, (size_t)(N + 2), sizeof(double), 8);
    s->vbd = (double*)ora_alloc(s, (size_t)(N + 2), sizeof(double), 8);
    /* the reference sizes hi as float32 (Global_Variables.py:113) but writes doubles;
       it is sized for the doubles the kernels write */
    s->hi = (double*)ora_alloc(s, (size_t)(2 * (N + 3) + 2 * (M + 3)), sizeof(double), 8);
    {
        const size_t L = (size_t)(N > M ? N : M) + 3;
        const size_t s1 = L * L; /* a1..f5: line * (L-1) + cell */
        size_t s2 = L * (2 * L + 1);
        if (s2 < nf) s2 = nf; /* AA/BB double as the smoothing buffers */
        const size_t G2 = 4 * L + 64;
        double** sc1[] = {&s->a1, &s->b1, &s->c1, &s->d1, &s->a2, &s->c2,
                          &s->d2, &s->f1, &s->f2, &s->f3, &s->f5};
        for (size_t k = 0; k < sizeof(sc1) / sizeof(sc1[0]); k++) {
            *sc1[k] = (double*)ora_alloc(s, s1, sizeof(double), G2);
            if (!*sc1[k]) goto fail;
        }
        double** sc2[] = {&s->AA, &s->BB, &s->CC, &s->DD, &s->x, &s->Ap, &s->Bp, &s->ep};
        for (size_t k = 0; k < sizeof(sc2) / sizeof(sc2[0]); k++) {
            *sc2[k] = (double*)ora_alloc(s, s2 + 2 * L, sizeof(double), G2);
            if (!*sc2[k]) goto fail;
        }
        s->SN = (int*)ora_alloc(s, L * SEGL, sizeof(int), 2 * SEGL);
    }
    if (!s->khouot || !s->daui || !s->cuoii || !s->moci || !s->dauj || !s->cuoij || !s->mocj ||
        !s->ubt || !s->ubp || !s->vbt || !s->vbd || !s->hi || !s->SN)
        goto fail;
    {
        double dc[5];
        ora_derived_constants(&s->P, dc);
        s->windx = dc[0];
        s->windy = dc[1];
        s->ufr = dc[2];
        s->dxr = dc[3];
        s->wss = dc[4];
    }
    return s;
fail:
    ora_destroy(s);
    return NULL;
}

void ora_destroy(OraSim* s) {
    if (!s) return;
    for (int k = 0; k < s->nmem; k++) free(s->mem[k]);
    for (int e = 0; e < 4; e++) {
        free(s->bc[e]);
        free(s->cc[e]);
    }
    free(s);
}

void* ora_field(OraSim* s, const char* name, int* is_int, size_t* count) {
    const int N = s->N, M = s->M;
    *is_int = 0;
    *count = s->nf;
    struct {
        const char* n;
        double* p;
    } dtab[] = {{"h", s->h},         {"hsnham", s->hsnham}, {"VISCOIDX", s->VISCOIDX},
                {"Fw", s->Fw},       {"Tsxw", s->Tsxw},     {"Tsyw", s->Tsyw},
                {"u", s->u},         {"v", s->v},           {"z", s->z},
                {"t_u", s->t_u},     {"t_v", s->t_v},       {"t_z", s->t_z},
                {"Htdu", s->Htdu},   {"Htdv", s->Htdv},     {"H_moi", s->H_moi},
                {"htaiz", s->htaiz}, {"htaiz_bd", s->htaiz_bd}, {"Kx1", s->Kx1},
                {"Ky1", s->Ky1},     {"FS", s->FS},         {"tFS", s->tFS},
                {"VTH", s->VTH},     {"Kx", s->Kx},         {"Ky", s->Ky},
                {"Qbx", s->Qbx},     {"Qby", s->Qby},       {"dH", s->dH}};
    for (size_t k = 0; k < sizeof(dtab) / sizeof(dtab[0]); k++)
        if (!strcmp(name, dtab[k].n)) return dtab[k].p;
    if (!strcmp(name, "khouot")) {
        *is_int = 1;
        return s->khouot;
    }
    *is_int = 1;
    if (!strcmp(name, "daui")) { *count = (size_t)(N + 2) * SEGL; return s->daui; }
    if (!strcmp(name, "cuoii")) { *count = (size_t)(N + 2) * SEGL; return s->cuoii; }
    if (!strcmp(name, "moci")) { *count = (size_t)(N + 2); return s->moci; }
    if (!strcmp(name, "dauj")) { *count = (size_t)(M + 2) * SEGL; return s->dauj; }
    if (!strcmp(name, "cuoij")) { *count = (size_t)(M + 2) * SEGL; return s->cuoij; }
    if (!strcmp(name, "mocj")) { *count = (size_t)(M + 2); return s->mocj; }
    *is_int = 0;
    if (!strcmp(name, "ubt")) { *count = (size_t)(M + 2); return s->ubt; }
    if (!strcmp(name, "ubp")) { *count = (size_t)(M + 2); return s->ubp; }
    if (!strcmp(name, "vbt")) { *count = (size_t)(N + 2); return s->vbt; }
    if (!strcmp(name, "vbd")) { *count = (size_t)(N + 2); return s->vbd; }
    if (!strcmp(name, "hi")) { *count = (size_t)(2 * (N + 3) + 2 * (M + 3)); return s->hi; }
    return NULL;
}

int ora_set_boundary(OraSim* s, const int* boundary_type, const double* const* tables,
                     const double* const* cc, const int* nseg, int total_time) {
    if (total_time < 2) return -1;
    memcpy(s->boundary_type, boundary_type, sizeof(int) * 4 * SEGL);
    /* bienQ[e] = 1 when any segment of edge e is a discharge edge (Global_Variables.py:56-66) */
    for (int e = 0; e < 4; e++) {
        s->bienQ[e] = 0;
        for (int k = 0; k < SEGL; k++)
            if (boundary_type[e * SEGL + k] == 2) s->bienQ[e] = 1;
        free(s->bc[e]);
        free(s->cc[e]);
        int ns = nseg[e] > 0 ? nseg[e] : 1;
        s->bc[e] = (double*)calloc((size_t)ns * total_time + 2, sizeof(double));
        s->cc[e] = (double*)calloc((size_t)ns * total_time + 2, sizeof(double));
        if (!s->bc[e] || !s->cc[e]) return -1;
        if (nseg[e] > 0) {
            memcpy(s->bc[e], tables[e], sizeof(double) * (size_t)nseg[e] * total_time);
            memcpy(s->cc[e], cc[e], sizeof(double) * (size_t)nseg[e] * total_time);
        }
    }
    s->total_time = total_time;
    return 0;
}

double ora_time(const OraSim* s) { return s->t; }

void ora_set_time(OraSim* s, double t) { s->t = t; }

void ora_set_hmax(OraSim* s, const double* hmax4) {
    s->hmax_u = hmax4[0];
    s->hmax_d = hmax4[1];
    s->hmax_l = hmax4[2];
    s->hmax_r = hmax4[3];
}

/* ------------------------------------------------------- segment lookups */

/* locate_segment_v (constant.cuh:135-154): segment of row `row` holding column `col`.
 * Returns -1 when no segment holds it (the reference falls off the end there and the
 * callers then only test first/last, which stay 0). */
static int loc_seg_v(const OraSim* s, int row, int col, int* first, int* last, int* br1,
                     int* br2) {
    const int W = s->W, M = s->M;
    const double* h = s->h;
    for (int k = 0; k < s->moci[row]; k++) {
        const int f = s->daui[row * SEGL + k], l = s->cuoii[row * SEGL + k];
        if (f <= col && col <= l) {
            *first = f;
            *last = l;
            if (f > 2 || (f == 2 && (h[row * W + f - 1] + h[(row - 1) * W + f - 1]) * 0.5 ==
                                        s->P.NANGDAY))
                *br1 = 1;
            if (l < M || (l == M && (h[row * W + l] + h[(row - 1) * W + l]) * 0.5 == s->P.NANGDAY))
                *br2 = 1;
            return k;
        }
    }
    return -1;
}

/* locate_segment_u (constant.cuh:156-178): segment of column `col` holding row `row`. */
static int loc_seg_u(const OraSim* s, int row, int col, int* first, int* last, int* br1,
                     int* br2) {
    const int W = s->W, N = s->N;
    const double* h = s->h;
    for (int k = 0; k < s->mocj[col]; k++) {
        const int f = s->dauj[col * SEGL + k], l = s->cuoij[col * SEGL + k];
        if (f <= row && row <= l) {
            *first = f;
            *last = l;
            if (f > 2 || (f == 2 && (h[1 * W + col] + h[1 * W + col - 1]) * 0.5 == s->P.NANGDAY))
                *br1 = 1;
            if (l < N || (l == N && (h[N * W + col] + h[N * W + col - 1]) * 0.5 == s->P.NANGDAY))
                *br2 = 1;
            return k;
        }
    }
    return -1;
}

/* ------------------------------------------------------ one-time set-up */

/* Onetime_init (support_funcs.cu:20-58) */
static void k_onetime_init(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const HydCaseParams* P = &s->P;
    const double* h = s->h;
    for (int i0 = 0; i0 < N + 3; i0++)
        for (int j0 = 0; j0 < M + 3; j0++) {
            s->khouot[i0 * W] = 2;
            s->khouot[j0] = 2;
            const int i = i0 + 1, j = j0 + 1;
            const size_t ij = (size_t)i * W + j;
            if (ij < s->nf) s->khouot[ij] = 2; /* the reference also writes one row past the end */
            if (i > N + 1 || j > M + 1) continue;
            if ((h[(i - 1) * W + j - 1] + h[(i - 1) * W + j] + h[i * W + j - 1] + h[i * W + j]) * 0.25 >
                P->NANGDAY) {
                s->khouot[ij] = 0;
                s->H_moi[ij] = 0;
            }
            if (i > N || j > M) continue;
            s->htaiz[ij] =
                (h[(i - 1) * W + j - 1] + h[(i - 1) * W + j] + h[i * W + j - 1] + h[i * W + j]) * 0.25;
            s->htaiz_bd[ij] = s->htaiz[ij];
            if (h[i * W + j - 1] + h[i * W + j] != 0)
                s->Kx1[ij] = P->g * pow((h[i * W + j - 1] + h[i * W + j]) * 0.5, -2 * P->mu_mn) *
                             pow((s->hsnham[i * W + j - 1] + s->hsnham[i * W + j]) * 0.5, 2);
            if (h[(i - 1) * W + j] + h[i * W + j] != 0)
                s->Ky1[ij] = P->g * pow((h[(i - 1) * W + j] + h[i * W + j]) * 0.5, -2 * P->mu_mn) *
                             pow((s->hsnham[(i - 1) * W + j] + s->hsnham[i * W + j]) * 0.5, 2);
        }
}

/* Interpolate_FS_ng (support_funcs.cu:189-208) */
static void interp_fs_ng(OraSim* s, int location, int offset, int sign) {
    const int M = s->M, W = s->W, N = s->N;
    const double dT = s->P.dT, dX = s->P.dX;
    for (int j = 1; j < M; j++) {
        if (s->t_u[location * W + j] > 0) {
            const double deltaX = (s->u[location * W + j] + s->t_u[location * W + j]) * 0.25 * dT;
            const int i = (int)(offset + sign * (deltaX / dX));
            const int i_deltaX = (int)nearbyint(deltaX);
            const int i_dX = (int)nearbyint(dX);
            if (i < 0 || i + 1 > N + 2) continue; /* outside the grid in the reference too */
            s->FS[location * W + j] = s->FS[i * W + j] + sign * (s->FS[(i + 1) * W + j] - s->FS[i * W + j]) *
                                                            (deltaX / dX - i_deltaX / i_dX);
        }
    }
}

/* Interpolate_FS_d (support_funcs.cu:210-229); the row bound is M as in the reference */
static void interp_fs_d(OraSim* s, int location, int offset, int sign) {
    const int M = s->M, W = s->W, N = s->N;
    const double dT = s->P.dT, dY = s->P.dY;
    for (int i = 1; i < M && i <= N + 2; i++) {
        if (s->t_v[i * W + location] > 0) {
            const double deltaY = (s->v[i * W + location] + s->t_v[i * W + location]) * 0.25 * dT;
            const int j = (int)(offset + sign * (deltaY / dY));
            const int j_deltaY = (int)nearbyint(deltaY);
            const int j_dY = (int)nearbyint(dY);
            if (j < 0 || j + 1 > M + 2) continue;
            s->FS[i * W + location] = s->FS[i * W + j + 1] + (s->FS[i * W + j + 1] - s->FS[i * W + j]) *
                                                                 (deltaY / dY - j_deltaY / j_dY);
        }
    }
}

/* Wet-segment scan of one line (support_funcs.cu:252-279, 303-330). */
static int scan_line(OraSim* s, const int* kh, int stride, int L, int* dau, int* cuoi) {
    int nseg = 0, start = 2, end = 0;
    while (start < L) {
        if (kh[start * stride] != 0) {
            while (kh[start * stride] && start < L) start++;
        }
        if (start + 1 == L) start = L;
        if (kh[start * stride] == 0 && start + 1 < L) {
            if (nseg >= SEGL) {
                s->overflow = 1;
                return nseg;
            }
            dau[nseg] = start;
            end = start;
            while (kh[end * stride] == 0 && end < L) end++;
            if (kh[end * stride] != 0 && end <= L) {
                cuoi[nseg] = end - 1;
                start = end;
                nseg++;
            } else {
                cuoi[nseg] = L;
                start = L;
                nseg++;
            }
        }
    }
    return nseg;
}

/* Find_Calculation_limits_Horizontal (support_funcs.cu:230-280): rows 2..N,
 * with the edge interpolation of FS done by the blocks of rows 2 and N. */
static void k_limits_horizontal(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    interp_fs_ng(s, 2, 2, 1);
    interp_fs_ng(s, N, N - 1, -1);
#pragma omp parallel for schedule(static)
    for (int i = 2; i <= N; i++)
        s->moci[i] = scan_line(s, s->khouot + (size_t)i * W, 1, M, s->daui + i * SEGL, s->cuoii + i * SEGL);
}

/* Find_Calculation_limits_Vertical (support_funcs.cu:283-335) */
static void k_limits_vertical(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    interp_fs_d(s, M, M - 1, -1);
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= M; j++)
        s->mocj[j] = scan_line(s, s->khouot + j, W, N, s->dauj + j * SEGL, s->cuoij + j * SEGL);
}

/* Htuongdoi (support_funcs.cu:338-354) */
static void k_htuongdoi(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const double *h = s->h, *z = s->z;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; i++)
        for (int j = 1; j <= M; j++) {
            s->Htdu[i * W + j] = (h[i * W + j - 1] + h[i * W + j] + z[(i + 1) * W + j] + z[i * W + j]) * 0.5;
            s->Htdv[i * W + j] = (h[(i - 1) * W + j] + h[i * W + j] + z[i * W + j + 1] + z[i * W + j]) * 0.5;
        }
}

/* preprocess_data (support_funcs.cu:433-542): Q-edge conveyance weights hi and hmax_* */
static void k_preprocess(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const double *h = s->h, NANGDAY = s->P.NANGDAY, dX = s->P.dX, ros = s->P.ros;
    double* hi = s->hi;
    for (int k = 0; k < s->mocj[M]; k++) {
        double sum = 0;
        for (int i = s->dauj[M * SEGL + k]; i <= s->cuoij[M * SEGL + k]; i++) {
            hi[i] = (h[i * W + M] + h[(i - 1) * W + M]) / 2.0 - NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = s->dauj[M * SEGL + k]; i <= s->cuoij[M * SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * dX);
    }
    hi += N + 3;
    for (int k = 0; k < s->mocj[2]; k++) {
        double sum = 0;
        for (int i = s->dauj[2 * SEGL + k]; i <= s->cuoij[2 * SEGL + k]; i++) {
            hi[i] = (h[i * W + 1] + h[(i - 1) * W + 1]) / 2.0 - NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = s->dauj[2 * SEGL + k]; i <= s->cuoij[2 * SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * dX);
    }
    hi += N + 3;
    for (int k = 0; k < s->moci[2]; k++) {
        double sum = 0;
        for (int i = s->daui[2 * SEGL + k]; i <= s->cuoii[2 * SEGL + k]; i++) {
            hi[i] = (h[1 * W + i] + h[1 * W + i - 1]) / 2.0 - NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = s->daui[2 * SEGL + k]; i <= s->cuoii[2 * SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * dX);
    }
    hi += M + 3;
    for (int k = 0; k < s->moci[N]; k++) {
        double sum = 0;
        for (int i = s->daui[N * SEGL + k]; i <= s->cuoii[N * SEGL + k]; i++) {
            hi[i] = (h[N * W + i] + h[N * W + i - 1]) / 2.0 - NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = s->daui[N * SEGL + k]; i <= s->cuoii[N * SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * dX);
    }
    const double* hb = s->htaiz_bd;
    s->hmax_u = hb[2 * W + M];
    s->hmax_d = hb[2 * W + 2];
    for (int i = 3; i < N; i++) {
        if (hb[i * W + M] > s->hmax_u) s->hmax_u = hb[i * W + M];
        if (hb[i * W + 2] > s->hmax_d) s->hmax_d = hb[i * W + 2];
    }
    s->hmax_l = hb[2 * W + 2];
    s->hmax_r = hb[N * W + 2];
    for (int i = 3; i < M; i++) {
        if (hb[2 * W + i] > s->hmax_l) s->hmax_l = hb[2 * W + i];
        if (hb[N * W + i] > s->hmax_r) s->hmax_r = hb[N * W + i];
    }
    if (s->hmax_u != 0) s->hmax_u = 1.0 / (ros * s->hmax_u);
    if (s->hmax_d != 0) s->hmax_d = 1.0 / (ros * s->hmax_d);
    if (s->hmax_l != 0) s->hmax_l = 1.0 / (ros * s->hmax_l);
    if (s->hmax_r != 0) s->hmax_r = 1.0 / (ros * s->hmax_r);
}

/* Morphodynamic feedback set-up (no reference counterpart): h0 = h - dH, no compensation. */
static void bed_feedback_reset(OraSim* s) {
    for (size_t q = 0; q < s->nf; q++) {
        s->h0[q] = s->h[q] - s->dH[q];
        s->dHc[q] = 0.0;
    }
}

/* rep.py:126-131 with pick_up: the mask loaded from the pick-up files replaces the one
 * Onetime_init derives, before the segment scans, Htuongdoi and preprocess_data. */
void ora_init_pickup(OraSim* s, double t_start) {
    const size_t n = (size_t)(s->N + 3) * (s->M + 3);
    int* keep = (int*)malloc(n * sizeof(int));
    memcpy(keep, s->khouot, n * sizeof(int));
    k_onetime_init(s);
    memcpy(s->khouot, keep, n * sizeof(int));
    free(keep);
    k_limits_horizontal(s);
    k_limits_vertical(s);
    k_htuongdoi(s);
    k_preprocess(s);
    bed_feedback_reset(s);
    s->t = t_start;
}

void ora_init(OraSim* s, double t_start) {
    k_onetime_init(s);
    k_limits_horizontal(s);
    k_limits_vertical(s);
    k_htuongdoi(s);
    k_preprocess(s);
    bed_feedback_reset(s);
    s->t = t_start;
}

/* ------------------------------------------------------ boundary values */

/* Boundary_value + FS_boundary for one edge and one thread index i
 * (support_funcs.cu:544-617). */
static void bnd_edge(OraSim* s, int i, double t, int isU, int location, int location_ext,
                     const int* btype, const double* hi_e, double* barr, const double* bcv,
                     const double* ccv, double hmax, const int* moc, const int* dau, const int* cuoi) {
    const int W = s->W, tt = s->total_time;
    {
        const int t1 = (int)(t / 3600);
        const double t2 = (t - (3600.0 * t1)) / 3600.0;
        int seg_no = -1;
        if (moc[location] > 0 && dau[location * SEGL] <= i && i <= cuoi[location * SEGL]) seg_no = 0;
        if (seg_no != -1) {
            const double value = bcv[seg_no * tt + t1] * (1.0 - t2) + bcv[seg_no * tt + t1 + 1] * t2;
            if (btype[seg_no] == 2) {
                barr[i] = value * hi_e[i];
            } else if (isU) {
                s->t_z[location * W + i] = value;
                s->t_z[location_ext * W + i] = value;
            } else {
                s->t_z[i * W + location] = value;
                s->t_z[i * W + location_ext] = value;
            }
        }
    }
    {
        const int t1 = (int)(t / 3600);
        const double t2 = (t - (3600.0 * t1)) / 3600.0;
        int seg_no = -1;
        if (moc[location] > 0 && dau[location * SEGL] <= i && i <= cuoi[location * SEGL]) seg_no = 0;
        if (seg_no == -1 || btype[seg_no] != 2) return;
        const int ii = isU ? location : i, jj = isU ? i : location;
        const double value = ccv[seg_no * tt + t1] * (1.0 - t2) + ccv[seg_no * tt + t1 + 1] * t2;
        s->FS[ii * W + jj] = value * s->htaiz_bd[ii * W + jj] * hmax;
    }
}

/* Update_Boundary_Value (support_funcs.cu:622-668) */
static void k_boundary(OraSim* s, double t) {
    const int N = s->N, M = s->M;
    const int imax = N > M ? N : M;
    double* hi_up = s->hi;
    double* hi_down = hi_up + (N + 3);
    double* hi_left = hi_down + (N + 3);
    double* hi_right = hi_left + (M + 3);
    for (int i = 2; i <= imax; i++) {
        bnd_edge(s, i, t, 0, M, M + 1, s->boundary_type + 0 * SEGL, hi_up, s->vbt, s->bc[0], s->cc[0],
                 s->hmax_u, s->mocj, s->dauj, s->cuoij);
        bnd_edge(s, i, t, 0, 2, 1, s->boundary_type + 1 * SEGL, hi_down, s->vbd, s->bc[1], s->cc[1],
                 s->hmax_d, s->mocj, s->dauj, s->cuoij);
        bnd_edge(s, i, t, 1, 2, 1, s->boundary_type + 2 * SEGL, hi_left, s->ubt, s->bc[2], s->cc[2],
                 s->hmax_l, s->moci, s->daui, s->cuoii);
        bnd_edge(s, i, t, 1, N, N + 1, s->boundary_type + 3 * SEGL, hi_right, s->ubp, s->bc[3],
                 s->cc[3], s->hmax_r, s->moci, s->daui, s->cuoii);
    }
}

/* Channel-mode analytic seiche boundaries (support_funcs.cu:356-429, Engine.py:29-43).
 * Engine.py passes m_offset = 5 as the kernels' segment_limit parameter, so the segment
 * tables are indexed with a stride of 5 there; bienQ is read through a bool*, i.e. byte e
 * of the int32 array. */
static void k_boundary_channel(OraSim* s, double t) {
    const int N = s->N, M = s->M, W = s->W;
    const int sl = 5;
    const double dX = s->P.dX, dY = s->P.dY;
    const unsigned char* bq = (const unsigned char*)s->bienQ;
    for (int i = s->dauj[M * sl]; i <= s->cuoij[M * sl] && i < s->dauj[M * sl] + N; i++) {
        s->t_z[i * W + M] = 0.01 * cos(2 * PI_REF / 27.750 * t) * cos(2 * (PI_REF / 100) * (100 - dY / 2));
        s->t_z[i * W + M + 1] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * (100 + dY / 2));
    }
    for (int i = s->dauj[2 * sl]; i <= s->cuoij[2 * sl] && i < s->dauj[2 * sl] + N; i++) {
        if (bq[1]) s->vbd[i] = 0;
        else {
            s->t_z[i * W + 2] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * dY / 2);
            s->t_z[i * W + 1] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * (-dY) / 2);
        }
    }
    for (int i = s->daui[2 * sl]; i <= s->cuoii[2 * sl] && i < s->daui[2 * sl] + M; i++) {
        if (bq[2]) s->ubt[i] = 0;
        else {
            s->t_z[2 * W + i] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * dX / 2);
            s->t_z[1 * W + i] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * (-dX) / 2);
        }
    }
    for (int i = s->daui[2 * sl]; i <= s->cuoii[N * sl] && i < s->daui[2 * sl] + M; i++) {
        if (bq[3]) s->ubp[i] = 0;
        else {
            s->t_z[N * W + i] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * (100 - dX / 2));
            s->t_z[(N + 1) * W + i] = 0.01 * cos(2 * PI_REF / 27.75 * t) * cos(2 * (PI_REF / 100) * (100 + dX / 2));
        }
    }
}

/* ------------------------------------------------------------- tridiag */

void ora_tridiag(int sn, const double* AA, const double* BB, const double* CC, const double* DD,
                 double* x, double* Ap, double* Bp, double* ep) {
    /* tridiag (UVZSolver_multithread.cu:203-228) */
    if (sn == 0) {
        x[0] = DD[0] / BB[0];
        return;
    }
    Ap[0] = -CC[0] / BB[0];
    Bp[0] = DD[0] / BB[0];
    for (int i = 1; i < sn; i++) {
        ep[i] = AA[i] * Ap[i - 1] + BB[i];
        Ap[i] = -CC[i] / ep[i];
        Bp[i] = (DD[i] - (AA[i] * Bp[i - 1])) / ep[i];
    }
    x[sn] = (DD[sn] - (AA[sn] * Bp[sn - 1])) / (BB[sn] + (AA[sn] * Ap[sn - 1]));
    for (int i = sn - 1; i >= 0; i--) x[i] = Bp[i] + (Ap[i] * x[i + 1]);
}

static void solve_at(OraSim* s, size_t pos, int sn) {
    ora_tridiag(sn, s->AA + pos, s->BB + pos, s->CC + pos, s->DD + pos, s->x + pos, s->Ap + pos,
                s->Bp + pos, s->ep + pos);
}

/* ------------------------------------------------- hydrodynamic sweeps */

/* _calculate_abcd (UVZSolver_multithread.cu:409-466) for one segment of one line;
 * `sw` = support_array_width, `line` = line index.  The __syncthreads at line 436
 * orders every thread's general row before the edge overrides. */
static void seg_abcd(OraSim* s, int line, int sw, int first, int last, double f4, int br1, int br2) {
    double *a1 = s->a1 + (size_t)line * sw, *b1 = s->b1 + (size_t)line * sw,
           *c1 = s->c1 + (size_t)line * sw, *d1 = s->d1 + (size_t)line * sw;
    const double *a2 = s->a2 + (size_t)line * sw, *c2 = s->c2 + (size_t)line * sw,
                 *d2 = s->d2 + (size_t)line * sw, *f1 = s->f1 + (size_t)line * sw,
                 *f2 = s->f2 + (size_t)line * sw, *f3 = s->f3 + (size_t)line * sw,
                 *f5 = s->f5 + (size_t)line * sw;
    if (last - 1 > first) {
        for (int j = first; j <= last; j++) {
            a1[j] = f4 - f1[j] / a2[j];
            c1[j] = -f4 - (f3[j] / c2[j + 1]);
            b1[j] = f2[j] - (f1[j] * c2[j] / a2[j]) - (f3[j] * a2[j + 1] / c2[j + 1]);
            d1[j] = f5[j] - (f1[j] * d2[j] / a2[j]) - (f3[j] * d2[j + 1] / c2[j + 1]);
        }
        if (br1) {
            a1[first] = f4;
            b1[first] = f2[first] - (f3[first] * a2[first + 1] / c2[first + 1]);
            c1[first] = -f4 - (f3[first] / c2[first + 1]);
            d1[first] = f5[first] - (f3[first] * d2[first + 1] / c2[first + 1]);
        }
        if (br2) {
            a1[last - 1] = f4 - f1[last - 1] / a2[last - 1];
            b1[last - 1] = f2[last - 1] - (f1[last - 1] * c2[last - 1] / a2[last - 1]);
            c1[last - 1] = -f4;
            d1[last - 1] = f5[last - 1] - (f1[last - 1] * d2[last - 1] / a2[last - 1]);
        }
    } else {
        a1[first] = f4;
        b1[first] = f2[first];
        d1[first] = f5[first];
        c1[first] = -f4;
    }
}

/* _calculate_matrix_coeff + bienrandau + bienlongdau (UVZSolver_multithread.cu:264-292,
 * 469-593) for one segment; returns sn (also stored in SN). */
static int seg_matrix(OraSim* s, int line, int sw, int tw, int first, int last, int seg_no, int br1,
                      int br2, double ubt_or_vbd, double ubp_or_vbt, double TZ_r, double TZ_l,
                      int dkBienQ_1, int dkBienQ_2, int dkfr) {
    const double *a1 = s->a1 + (size_t)line * sw, *b1 = s->b1 + (size_t)line * sw,
                 *c1 = s->c1 + (size_t)line * sw, *d1 = s->d1 + (size_t)line * sw,
                 *a2 = s->a2 + (size_t)line * sw, *c2 = s->c2 + (size_t)line * sw,
                 *d2 = s->d2 + (size_t)line * sw;
    double *AA = s->AA + (size_t)line * tw, *BB = s->BB + (size_t)line * tw,
           *CC = s->CC + (size_t)line * tw, *DD = s->DD + (size_t)line * tw;
    const int offset = first * 2;
    int sn = 2 * (last - first);
#define BIENRANDAU(j)                  \
    do {                               \
        AA[(j) * 2] = a2[j];           \
        AA[(j) * 2 + 1] = a1[j];       \
        BB[(j) * 2] = 1;               \
        BB[(j) * 2 + 1] = b1[j];       \
        CC[(j) * 2] = c2[j];           \
        CC[(j) * 2 + 1] = c1[j];       \
        DD[(j) * 2] = d2[j];           \
        DD[(j) * 2 + 1] = d1[j];       \
    } while (0)
#define BIENLONGDAU(j)                 \
    do {                               \
        AA[(j) * 2] = a1[j];           \
        AA[(j) * 2 + 1] = a2[(j) + 1]; \
        BB[(j) * 2] = b1[j];           \
        BB[(j) * 2 + 1] = 1;           \
        CC[(j) * 2] = c1[j];           \
        CC[(j) * 2 + 1] = c2[(j) + 1]; \
        DD[(j) * 2] = d1[j];           \
        DD[(j) * 2 + 1] = d2[(j) + 1]; \
    } while (0)
    if (br1) {
        for (int j = first; j <= last; j++) BIENRANDAU(j);
        DD[offset] = d2[first];
        if (!br2) {
            if (dkBienQ_2 && last == dkfr) {
                AA[sn + offset] = a2[last];
                BB[sn + offset] = 1;
                DD[sn + offset] = d2[last] - c2[last] * ubp_or_vbt;
            } else {
                sn--;
                AA[sn + offset] = a1[last - 1];
                BB[sn + offset] = b1[last - 1];
                DD[sn + offset] = d1[last - 1] - c1[last - 1] * TZ_r;
            }
        } else {
            AA[sn + offset] = a2[last];
            BB[sn + offset] = 1;
            DD[sn + offset] = d2[last];
        }
    } else {
        int isBienran;
        if (dkBienQ_1 && first == 2) {
            for (int j = first; j <= last; j++) BIENRANDAU(j);
            DD[offset] = d2[first] - a2[first] * ubt_or_vbd;
            isBienran = 1;
        } else {
            for (int j = first; j <= last; j++) BIENLONGDAU(j);
            BB[offset] = b1[first];
            CC[offset] = c1[first];
            DD[offset] = d1[first] - a1[first] * TZ_l;
            isBienran = 0;
        }
        if (!br2) {
            if (dkBienQ_1 && last == dkfr) {
                if (!isBienran) sn--;
                AA[sn + offset] = a2[last];
                BB[sn + offset] = 1;
                DD[sn + offset] = d2[last] - c2[last] * ubp_or_vbt;
            } else {
                sn--;
                if (!isBienran) sn -= 1;
                AA[sn + offset] = a1[last - 1];
                BB[sn + offset] = b1[last - 1];
                DD[sn + offset] = d1[last - 1] - c1[last - 1] * TZ_r;
            }
        } else {
            if (!isBienran) sn--;
            AA[sn + offset] = a2[last];
            BB[sn + offset] = 1;
            DD[sn + offset] = d2[last];
        }
    }
#undef BIENRANDAU
#undef BIENLONGDAU
    s->SN[line * SEGL + seg_no] = sn;
    return sn;
}

/* UZ sweep of one column line j: UZSolver_calculate_preindex, _abcd, _matrix_coeff,
 * tridiagSolver(jumpstep 2) and UZSolver_extract_solution
 * (UVZSolver_multithread.cu:881-943, 352-407, 231-262, 668-723). */
static void uz_line(OraSim* s, int j) {
    const int N = s->N, M = s->M, W = s->W;
    const int sw = N + 2, tw = 2 * N + 1;
    const HydCaseParams* P = &s->P;
    const double *u = s->u, *v = s->v, *z = s->z, *Htdu = s->Htdu, *Htdv = s->Htdv,
                 *VISC = s->VISCOIDX, *Tsxw = s->Tsxw, *H_moi = s->H_moi, *Kx1 = s->Kx1;
    const double dT = P->dT, dXbp = P->dXbp, dY2 = P->dY2, dYbp = P->dYbp, H_TINH = P->H_TINH;
    const int nseg = s->mocj[j];
    int fa[SEGL], la[SEGL], b1a[SEGL], b2a[SEGL];
    for (int k = 0; k < nseg; k++) {
        fa[k] = s->dauj[j * SEGL + k];
        la[k] = s->cuoij[j * SEGL + k];
        int f = 0, l = 0;
        b1a[k] = b2a[k] = 0;
        loc_seg_u(s, fa[k], j, &f, &l, &b1a[k], &b2a[k]);
    }
    double *a2 = s->a2 + (size_t)j * sw, *c2 = s->c2 + (size_t)j * sw, *d2 = s->d2 + (size_t)j * sw,
           *f1 = s->f1 + (size_t)j * sw, *f2 = s->f2 + (size_t)j * sw, *f3 = s->f3 + (size_t)j * sw,
           *f5 = s->f5 + (size_t)j * sw;
    /* _uzSolver_calculate_preindex (UVZSolver_multithread.cu:352-407) */
    for (int k = 0; k < nseg; k++)
        for (int i = fa[k]; i <= la[k]; i++) {
            double p = 0.0, q = 0.0;
            const double vtb = (v[i * W + j - 1] + v[i * W + j] + v[(i + 1) * W + j - 1] + v[(i + 1) * W + j]) * 0.25;
            f1[i] = P->dTchia2dX * u[i * W + j] + VISC[i * W + j] * dT / dXbp;
            f2[i] = -(2 + Kx1[i * W + j] * dT * sqrt(u[i * W + j] * u[i * W + j] + vtb * vtb) / Htdu[i * W + j] +
                      (2 * dT * VISC[i * W + j]) / dXbp);
            f3[i] = dT * VISC[i * W + j] / dXbp - P->dTchia2dX * u[i * W + j];
            if (H_moi[i * W + j - 1] <= H_TINH) {
                if (vtb < 0) {
                    p = vtb * (-3 * u[i * W + j] + 4 * u[i * W + j + 1] - u[i * W + j + 2]) / dY2;
                    q = (u[i * W + j] - 2 * u[i * W + j + 1] + u[i * W + j + 2]) / dYbp;
                }
            } else {
                if (H_moi[i * W + j + 1] <= H_TINH) {
                    if ((H_moi[i * W + j - 2] > H_TINH) && (vtb > 0)) {
                        p = vtb * (3 * u[i * W + j] - 4 * u[i * W + j - 1] + u[i * W + j - 2]) / dY2;
                        q = (u[i * W + j] - 2 * u[i * W + j - 1] + u[i * W + j - 2]) / dYbp;
                    }
                } else {
                    p = vtb * (u[i * W + j + 1] - u[i * W + j - 1]) / dY2;
                    q = (u[i * W + j + 1] - 2 * u[i * W + j] + u[i * W + j - 1]) / dYbp;
                }
            }
            f5[i] = -2 * u[i * W + j] + dT * p - dT * P->CORIOLIS_FORCE * vtb - dT * VISC[i * W + j] * q -
                    dT * (s->windx - Tsxw[i * W + j]) / Htdu[i * W + j];
            c2[i] = P->dTchia2dX * Htdu[i * W + j];
            a2[i] = -P->dTchia2dX * Htdu[(i - 1) * W + j];
            d2[i] = z[i * W + j] - P->dTchia2dY * (Htdv[i * W + j] * v[i * W + j] - Htdv[i * W + j - 1] * v[i * W + j - 1]);
        }
    const double f4 = 2 * P->g * P->dTchia2dX;
    for (int k = 0; k < nseg; k++) seg_abcd(s, j, sw, fa[k], la[k], f4, b1a[k], b2a[k]);
    int sns[SEGL];
    for (int k = 0; k < nseg; k++)
        sns[k] = seg_matrix(s, j, sw, tw, fa[k], la[k], k, b1a[k], b2a[k], s->ubt[j], s->ubp[j],
                            s->t_z[la[k] * W + j], s->t_z[fa[k] * W + j], s->bienQ[2], s->bienQ[3], N);
    /* tridiagSolver (UVZSolver_multithread.cu:231-262), jumpstep 2 */
    for (int k = 0; k < nseg; k++) solve_at(s, (size_t)j * tw + fa[k] * 2, s->SN[j * SEGL + k]);
    (void)sns;
    /* _uzSolver_extract_solution (UVZSolver_multithread.cu:668-723) */
    const double* xl = s->x + (size_t)j * tw;
    double *t_z = s->t_z, *t_u = s->t_u;
    for (int k = 0; k < nseg; k++) {
        const int first = fa[k], last = la[k], sn = s->SN[j * SEGL + k];
        for (int i = first; i <= last; i++) {
            if (i < last) {
                if (b1a[k]) {
                    t_z[i * W + j] = xl[2 * i];
                    t_u[i * W + j] = xl[2 * i + 1];
                    t_u[(first - 1) * W + j] = 0;
                } else if (s->bienQ[2] && first == 2) {
                    t_z[i * W + j] = xl[2 * i];
                    t_u[i * W + j] = xl[2 * i + 1];
                    t_u[(first - 1) * W + j] = s->ubt[j];
                } else {
                    if (i == first) {
                        t_u[first * W + j] = xl[first * 2];
                        t_u[(first - 1) * W + j] =
                            (d2[first] - t_z[first * W + j] - c2[first] * t_u[first * W + j]) / a2[first];
                    } else if (i < last) {
                        t_z[i * W + j] = xl[2 * i - 1];
                        t_u[i * W + j] = xl[2 * i];
                    }
                }
            } else {
                if (b2a[k]) {
                    t_u[last * W + j] = 0;
                    t_z[last * W + j] = xl[first * 2 + sn];
                } else if (s->bienQ[3] && last == N) {
                    t_u[last * W + j] = s->ubp[j];
                    t_z[last * W + j] = xl[first * 2 + sn];
                } else {
                    t_u[last * W + j] =
                        (d2[last] - a2[last] * t_u[(last - 1) * W + j] - t_z[last * W + j]) / c2[last];
                }
            }
        }
    }
    (void)M;
}

/* VZ sweep of one row line i: VZSolver_* kernels (UVZSolver_multithread.cu:818-879, 295-350,
 * 231-262, 595-665). */
static void vz_line(OraSim* s, int i) {
    const int M = s->M, W = s->W;
    const int sw = M + 2, tw = 2 * M + 1;
    const HydCaseParams* P = &s->P;
    const double *u = s->u, *v = s->v, *z = s->z, *Htdu = s->Htdu, *Htdv = s->Htdv,
                 *VISC = s->VISCOIDX, *Tsyw = s->Tsyw, *H_moi = s->H_moi, *Ky1 = s->Ky1;
    const double dT = P->dT, dYbp = P->dYbp, dX2 = P->dX2, dXbp = P->dXbp, H_TINH = P->H_TINH;
    const int nseg = s->moci[i];
    int fa[SEGL], la[SEGL], b1a[SEGL], b2a[SEGL];
    for (int k = 0; k < nseg; k++) {
        fa[k] = s->daui[i * SEGL + k];
        la[k] = s->cuoii[i * SEGL + k];
        int f = 0, l = 0;
        b1a[k] = b2a[k] = 0;
        loc_seg_v(s, i, fa[k], &f, &l, &b1a[k], &b2a[k]);
    }
    double *a2 = s->a2 + (size_t)i * sw, *c2 = s->c2 + (size_t)i * sw, *d2 = s->d2 + (size_t)i * sw,
           *f1 = s->f1 + (size_t)i * sw, *f2 = s->f2 + (size_t)i * sw, *f3 = s->f3 + (size_t)i * sw,
           *f5 = s->f5 + (size_t)i * sw;
    /* _vzSolver_calculate_preindex (UVZSolver_multithread.cu:295-350) */
    for (int k = 0; k < nseg; k++)
        for (int j = fa[k]; j <= la[k]; j++) {
            double p = 0.0, q = 0.0;
            const double utb = (u[(i - 1) * W + j] + u[i * W + j] + u[(i - 1) * W + j + 1] + u[i * W + j + 1]) * 0.25;
            f1[j] = P->dTchia2dY * v[i * W + j] + VISC[i * W + j] * dT / dYbp;
            f2[j] = -(2 + Ky1[i * W + j] * dT * sqrt(v[i * W + j] * v[i * W + j] + utb * utb) / Htdv[i * W + j] +
                      (2 * dT * VISC[i * W + j]) / dYbp);
            f3[j] = dT * VISC[i * W + j] / dYbp - P->dTchia2dY * v[i * W + j];
            if (H_moi[(i - 1) * W + j] <= H_TINH) {
                if (utb < 0) {
                    q = utb * (-3 * v[i * W + j] + 4 * v[(i + 1) * W + j] - v[(i + 2) * W + j]) / dX2;
                    p = (v[i * W + j] - 2 * v[(i + 1) * W + j] + v[(i + 2) * W + j]) / dXbp;
                }
            } else {
                if (H_moi[(i + 1) * W + j] <= H_TINH) {
                    if ((H_moi[(i - 2) * W + j] > H_TINH) && (utb > 0)) {
                        q = utb * (3 * v[i * W + j] - 4 * v[(i - 1) * W + j] + v[(i - 2) * W + j]) / dX2;
                        p = (v[i * W + j] - 2 * v[(i - 1) * W + j] + v[(i - 2) * W + j]) / dXbp;
                    }
                } else {
                    q = utb * (v[(i + 1) * W + j] - v[(i - 1) * W + j]) / dX2;
                    p = (v[(i + 1) * W + j] - 2 * v[i * W + j] + v[(i - 1) * W + j]) / dXbp;
                }
            }
            f5[j] = -2 * v[i * W + j] + dT * q + dT * P->CORIOLIS_FORCE * utb - dT * VISC[i * W + j] * p -
                    dT * (s->windy - Tsyw[i * W + j]) / Htdv[i * W + j];
            c2[j] = P->dTchia2dY * Htdv[i * W + j];
            a2[j] = -P->dTchia2dY * Htdv[i * W + j - 1];
            d2[j] = z[i * W + j] - P->dTchia2dX * (Htdu[i * W + j] * u[i * W + j] - Htdu[(i - 1) * W + j] * u[(i - 1) * W + j]);
        }
    const double f4 = 2 * P->g * P->dTchia2dY;
    for (int k = 0; k < nseg; k++) seg_abcd(s, i, sw, fa[k], la[k], f4, b1a[k], b2a[k]);
    for (int k = 0; k < nseg; k++)
        seg_matrix(s, i, sw, tw, fa[k], la[k], k, b1a[k], b2a[k], s->vbd[i], s->vbt[i],
                   s->t_z[i * W + la[k]], s->t_z[i * W + fa[k]], s->bienQ[1], s->bienQ[0], M);
    for (int k = 0; k < nseg; k++) solve_at(s, (size_t)i * tw + fa[k] * 2, s->SN[i * SEGL + k]);
    const double* xl = s->x + (size_t)i * tw;
    double *t_z = s->t_z, *t_v = s->t_v;
    for (int k = 0; k < nseg; k++) {
        const int first = fa[k], last = la[k], sn = s->SN[i * SEGL + k];
        for (int j = first; j <= last; j++) {
            if (j < last) {
                if (b1a[k]) {
                    t_z[i * W + j] = xl[2 * j];
                    t_v[i * W + j] = xl[2 * j + 1];
                    t_v[i * W + first - 1] = 0;
                } else if (s->bienQ[1] && first == 2) {
                    t_z[i * W + j] = xl[2 * j];
                    t_v[i * W + j] = xl[2 * j + 1];
                    t_v[i * W + first - 1] = s->vbd[i];
                } else {
                    if (j == first) {
                        t_v[i * W + first] = xl[2 * first];
                        t_v[i * W + first - 1] =
                            (d2[first] - t_z[i * W + first] - c2[first] * t_v[i * W + first]) / a2[first];
                    } else {
                        t_z[i * W + j] = xl[2 * j - 1];
                        t_v[i * W + j] = xl[2 * j];
                    }
                }
            } else {
                if (b2a[k]) {
                    t_v[i * W + last] = 0;
                    t_z[i * W + last] = xl[first * 2 + sn];
                } else if (s->bienQ[0] && last == M) {
                    t_v[i * W + last] = s->vbt[i];
                    t_z[i * W + last] = xl[2 * first + sn];
                } else {
                    t_v[i * W + last] =
                        (d2[last] - a2[last] * t_v[i * W + last - 1] - t_z[i * W + last]) / c2[last];
                }
            }
        }
    }
}

static void k_uz_sweep(OraSim* s, int startidx, int endidx) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = startidx; j <= endidx; j++) uz_line(s, j);
}

static void k_vz_sweep(OraSim* s, int startidx, int endidx) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = startidx; i <= endidx; i++) vz_line(s, i);
}

/* Normalize + update_buffer (support_funcs.cu:682-729): 5-point smoothing of t_u
 * (isU, buffer AA) or t_v (buffer BB). */
static void k_normalize(OraSim* s, int isU) {
    const int N = s->N, M = s->M, W = s->W;
    const double coeff = s->P.heso;
    double* val = isU ? s->t_u : s->t_v;
    double* tmp = isU ? s->AA : s->BB;
    const int close_d = isU ? W : 1, far_d = isU ? 1 : W;
    const int* kh = s->khouot;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N + 3; i++)
        for (int j = 0; j < M + 3; j++) {
            const int gp = i * W + j;
            tmp[gp] = val[gp];
            if (i > N || j > M || i < 2 || j < 2) continue;
            if (val[gp] != 0) {
                int count = 2;
                double nb = val[gp - close_d] + val[gp + close_d];
                if (kh[gp - far_d] == 0) {
                    nb += val[gp - far_d];
                    count++;
                }
                if (kh[gp + far_d] == 0) {
                    nb += val[gp + far_d];
                    count++;
                }
                tmp[gp] = tmp[gp] * coeff + (1 - coeff) * nb / count;
            }
        }
#pragma omp parallel for schedule(static)
    for (int i = 2; i <= N; i++)
        for (int j = 2; j <= M; j++) val[i * W + j] = tmp[i * W + j];
}

/* solveV / vSolver (UVZSolver_multithread.cu:1055-1071, 727-768) */
static void k_solve_v(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const HydCaseParams* P = &s->P;
    const double *u = s->u, *v = s->v, *z = s->z, *t_u = s->t_u, *Ky1 = s->Ky1, *Htdv = s->Htdv,
                 *H_moi = s->H_moi, *VISC = s->VISCOIDX, *Tsyw = s->Tsyw;
    double* t_v = s->t_v;
    const double dY2 = P->dY2, dX2 = P->dX2, dXbp = P->dXbp, dYbp = P->dYbp, H_TINH = P->H_TINH;
#pragma omp parallel for schedule(static)
    for (int row = 2; row <= N; row++)
        for (int col = 2; col <= M; col++) {
            int first = 0, last = 0, b1 = 0, b2 = 0;
            loc_seg_v(s, row, col, &first, &last, &b1, &b2);
            if ((first >= last) || (col >= last) || (col < first)) continue;
            const int o = W;
            double p, q, tmp;
            q = 0;
            p = 0;
            tmp = 0;
            const double utb = (u[(row - 1) * o + col] + u[row * o + col] + u[(row - 1) * o + col + 1] + u[row * o + col + 1]) * 0.25;
            const double t_utb = (t_u[(row - 1) * o + col] + t_u[row * o + col] + t_u[(row - 1) * o + col + 1] + t_u[row * o + col + 1]) * 0.25;
            p = (v[row * o + col + 1] - v[row * o + col - 1]) / dY2;
            p = P->HaiChiadT + p + Ky1[row * o + col] * sqrt(utb * utb + v[row * o + col] * v[row * o + col]) / Htdv[row * o + col];
            if (H_moi[(row - 1) * o + col] <= H_TINH) {
                if (utb < 0) {
                    q = t_utb * (-3 * v[row * o + col] + 4 * v[(row + 1) * o + col] - v[(row + 2) * o + col]) / dX2;
                    tmp = (v[row * o + col] - 2 * v[(row + 1) * o + col] + v[(row + 2) * o + col]) / dXbp;
                }
            } else {
                if (H_moi[(row + 1) * o + col] <= H_TINH) {
                    if ((H_moi[(row - 2) * o + col] > H_TINH) && (utb > 0)) {
                        q = t_utb * (3 * v[row * o + col] - 4 * v[(row - 1) * o + col] + v[(row - 2) * o + col]) / dX2;
                        tmp = (v[row * o + col] - 2 * v[(row - 1) * o + col] + v[(row - 2) * o + col]) / dXbp;
                    }
                } else {
                    q = t_utb * (v[(row + 1) * o + col] - v[(row - 1) * o + col]) / dX2;
                    tmp = (v[(row + 1) * o + col] - 2 * v[row * o + col] + v[(row - 1) * o + col]) / dXbp;
                }
            }
            q = P->HaiChiadT * v[row * o + col] - q - P->CORIOLIS_FORCE * t_utb;
            q = (q - P->g * (z[row * o + col + 1] - z[row * o + col]) / P->dY +
                 VISC[row * o + col] * (tmp + (v[row * o + col + 1] - 2 * v[row * o + col] + v[row * o + col - 1]) / dYbp)) +
                (s->windy - Tsyw[row * o + col]) / Htdv[row * o + col];
            t_v[row * o + col] = q / p;
        }
}

/* solveU / uSolver (UVZSolver_multithread.cu:947-968, 773-815) */
static void k_solve_u(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const HydCaseParams* P = &s->P;
    const double *u = s->u, *v = s->v, *z = s->z, *t_v = s->t_v, *Kx1 = s->Kx1, *Htdu = s->Htdu,
                 *H_moi = s->H_moi, *VISC = s->VISCOIDX, *Tsxw = s->Tsxw;
    double* t_u = s->t_u;
    const double dY2 = P->dY2, dX2 = P->dX2, dXbp = P->dXbp, dYbp = P->dYbp, H_TINH = P->H_TINH;
#pragma omp parallel for schedule(static)
    for (int row = 1; row <= N; row++)
        for (int col = 2; col <= M; col++) {
            int first = 0, last = 0, b1 = 0, b2 = 0;
            loc_seg_u(s, row, col, &first, &last, &b1, &b2);
            if (first > last || row < first - 1 || row >= last) continue;
            const int o = W;
            double p, q, tmp;
            p = 0;
            q = 0;
            tmp = 0;
            const double vtb = (v[row * o + col - 1] + v[row * o + col] + v[(row + 1) * o + col - 1] + v[(row + 1) * o + col]) * 0.25;
            const double t_vtb = (t_v[row * o + col - 1] + t_v[row * o + col] + t_v[(row + 1) * o + col - 1] + t_v[(row + 1) * o + col]) * 0.25;
            p = (u[(row + 1) * o + col] - u[(row - 1) * o + col]) / dX2;
            p = (P->HaiChiadT + p + Kx1[row * o + col] * sqrt(vtb * vtb + u[row * o + col] * u[row * o + col]) / Htdu[row * o + col]);
            if (H_moi[row * o + col - 1] <= H_TINH) {
                if (vtb < 0) {
                    q = t_vtb * (-3 * u[row * o + col] + 4 * u[row * o + col + 1] - u[row * o + col + 2]) / dY2;
                    tmp = (u[row * o + col] - 2 * u[row * o + col + 1] + u[row * o + col + 2]) / dYbp;
                }
            } else {
                if (H_moi[row * o + col + 1] <= H_TINH) {
                    if ((H_moi[row * o + col - 2] > H_TINH) && (vtb > 0)) {
                        q = t_vtb * (3 * u[row * o + col] - 4 * u[row * o + col - 1] + u[row * o + col - 2]) / dY2;
                        tmp = (u[row * o + col] - 2 * u[row * o + col - 1] + u[row * o + col - 2]) / dYbp;
                    }
                } else {
                    q = t_vtb * (u[row * o + col + 1] - u[row * o + col - 1]) / dY2;
                    tmp = (u[row * o + col + 1] - 2 * u[row * o + col] + u[row * o + col - 1]) / dYbp;
                }
            }
            q = P->HaiChiadT * u[row * o + col] - q + P->CORIOLIS_FORCE * t_vtb;
            q = (q - P->g * (z[(row + 1) * o + col] - z[row * o + col]) / P->dX +
                 VISC[row * o + col] * (tmp + (u[(row + 1) * o + col] - 2 * u[row * o + col] + u[(row - 1) * o + col]) / dXbp)) +
                (s->windx - Tsxw[row * o + col]) / Htdu[row * o + col];
            t_u[row * o + col] = q / p;
        }
}

/* update_margin_elem_V (UVZSolver_multithread.cu:1008-1052), rows 2..N */
static void k_margin_v(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const double* h = s->h;
    const double NANGDAY = s->P.NANGDAY;
    double* t_v = s->t_v;
#pragma omp parallel for schedule(static)
    for (int i = 2; i <= N; i++)
        for (int k = 0; k < s->moci[i]; k++) {
            int b1 = 0, b2 = 0;
            const int first = s->daui[i * SEGL + k], last = s->cuoii[i * SEGL + k];
            if ((first > 2) || ((first == 2) && (fabs((h[i * W + first - 1] + h[(i - 1) * W + first - 1]) * 0.5 - NANGDAY) < EPS_REF)))
                b1 = 1;
            if ((last < M) || ((last == M) && (fabs((h[i * W + last] + h[(i - 1) * W + last]) * 0.5 - NANGDAY) < EPS_REF)))
                b2 = 1;
            if (b1) t_v[i * W + first - 1] = 0;
            else t_v[i * W + first - 1] = 2 * t_v[i * W + first] - t_v[i * W + first + 1];
            if (b2) t_v[i * W + last] = 0;
            else t_v[i * W + last] = 2 * t_v[i * W + last - 1] - t_v[i * W + last - 2];
        }
}

/* update_margin_elem_U (UVZSolver_multithread.cu:970-1006), columns 2..M */
static void k_margin_u(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const double* h = s->h;
    const double NANGDAY = s->P.NANGDAY;
    double* t_u = s->t_u;
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= M; j++)
        for (int k = 0; k < s->mocj[j]; k++) {
            const int first = s->dauj[j * SEGL + k], last = s->cuoij[j * SEGL + k];
            int b1 = 0, b2 = 0;
            if ((first > 2) || ((first == 2) && ((fabs(h[1 * W + j] + h[1 * W + j - 1]) * 0.5 - NANGDAY) < EPS_REF)))
                b1 = 1;
            if ((last < N) || ((last == N) && (fabs((h[N * W + j] + h[N * W + j - 1]) * 0.5 - NANGDAY) < EPS_REF)))
                b2 = 1;
            if (b1) t_u[(first - 1) * W + j] = 0;
            else t_u[(first - 1) * W + j] = 2 * t_u[first * W + j] - t_u[(first + 1) * W + j];
            if (b2) t_u[last * W + j] = 0;
            else t_u[last * W + j] = 2 * t_u[(last - 1) * W + j] - t_u[(last - 2) * W + j];
        }
}

/* update_h_moi (support_funcs.cu:60-73) */
static void k_update_h_moi(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; i++)
        for (int j = 1; j <= M; j++) {
            const int gp = i * W + j;
            if (s->khouot[gp] == 0) s->H_moi[gp] = s->htaiz[gp] + s->t_z[gp];
        }
}

/* Reset_states_horizontal (support_funcs.cu:75-129): rows 1..N, each a sequential scan */
static void k_reset_horizontal(OraSim* s) {
    const int N = s->N, M = s->M, o = s->W;
    const double H_TINH = s->P.H_TINH;
    double *H_moi = s->H_moi, *htaiz = s->htaiz, *z = s->z, *t_z = s->t_z, *t_u = s->t_u, *t_v = s->t_v, *FS = s->FS;
    int* khouot = s->khouot;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; i++) {
        for (int j = 2; j <= M; j++) {
            if (t_z[i * o + j] > z[i * o + j]) {
                if (khouot[i * o + j - 1] == 1) {
                    t_z[i * o + j - 1] = t_z[i * o + j];
                    H_moi[i * o + j - 1] = htaiz[i * o + j - 1] + t_z[i * o + j];
                    khouot[i * o + j - 1] = 0;
                    FS[i * o + j - 1] = FS[i * o + j];
                }
                if (khouot[i * o + j + 1] == 1) {
                    t_z[i * o + j + 1] = t_z[i * o + j];
                    H_moi[i * o + j + 1] = htaiz[i * o + j + 1] + t_z[i * o + j];
                    khouot[i * o + j + 1] = 0;
                    FS[i * o + j + 1] = FS[i * o + j];
                }
            }
        }
        for (int j = 2; j <= M; j++) {
            if ((khouot[i * o + j] == 0) && (H_moi[i * o + j] <= H_TINH)) {
                t_u[(i - 1) * o + j] = 0;
                t_u[i * o + j] = 0;
                t_v[i * o + j - 1] = 0;
                t_v[i * o + j] = 0;
                khouot[i * o + j] = 1;
                FS[i * o + j] = 0;
            }
        }
    }
}

/* Reset_states_vertical (support_funcs.cu:134-186): columns 1..M */
static void k_reset_vertical(OraSim* s) {
    const int N = s->N, M = s->M, o = s->W;
    const double H_TINH = s->P.H_TINH;
    double *H_moi = s->H_moi, *htaiz = s->htaiz, *z = s->z, *t_z = s->t_z, *t_u = s->t_u, *t_v = s->t_v, *FS = s->FS;
    int* khouot = s->khouot;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= M; j++) {
        for (int i = 2; i <= N; i++) {
            if (t_z[i * o + j] > z[i * o + j]) {
                if (khouot[(i - 1) * o + j] == 1) {
                    t_z[(i - 1) * o + j] = t_z[i * o + j];
                    H_moi[(i - 1) * o + j] = htaiz[(i - 1) * o + j] + t_z[i * o + j];
                    khouot[(i - 1) * o + j] = 0;
                    FS[(i - 1) * o + j] = FS[i * o + j];
                }
                if (khouot[(i + 1) * o + j] == 1) {
                    t_z[(i + 1) * o + j] = t_z[i * o + j];
                    H_moi[(i + 1) * o + j] = htaiz[(i + 1) * o + j] + t_z[i * o + j];
                    khouot[(i + 1) * o + j] = 0;
                    FS[(i + 1) * o + j] = FS[i * o + j];
                }
            }
        }
        for (int i = 2; i <= N; i++) {
            if ((khouot[i * o + j] == 0) && (H_moi[i * o + j] <= H_TINH)) {
                t_u[(i - 1) * o + j] = 0;
                t_u[i * o + j] = 0;
                t_v[i * o + j - 1] = 0;
                t_v[i * o + j] = 0;
                khouot[i * o + j] = 1;
                FS[i * o + j] = 0;
            }
        }
    }
}

/* update_uvz (support_funcs.cu:671-680).  Engine.py:90 passes two arguments fewer than
 * the kernel declares, so its kenhhepd/kenhhepng parameters never hold the host's flags
 * and the velocities are copied unmasked. */
static void k_update_uvz(OraSim* s) {
    const int N = s->N, M = s->M, o = s->W;
    const int kd = 0, kn = 0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= N; i++)
        for (int j = 0; j <= M; j++) {
            s->z[i * o + j] = s->t_z[i * o + j];
            s->u[i * o + j] = s->t_u[i * o + j] * (1 - kd);
            s->v[i * o + j] = s->t_v[i * o + j] * (1 - kn);
        }
}

/* ------------------------------------------------------------ sediment */

/* source_chs (Sediment_Transport.cu:12-49) */
static double source_chs(const HydCaseParams* P, double wsm, double Zf, double fs, double fw, double vth,
                         double h_moi) {
    double toee = P->Toe;
    const double todd = P->Tod;
    double S = 0;
    double Pd, beta, Cb;
    const double tob = P->ro * fw * (vth * vth);
    if (h_moi > P->ghtoe) toee = P->Toe * (1 + P->hstoe * ((h_moi - P->ghtoe)));
    if (tob > toee) S = P->Mbochat / P->ros * (tob - toee) / toee;
    else {
        if (tob < todd) {
            Pd = 1 - (tob / todd);
            beta = 1 + (Zf / (1.25 + 4.75 * pow(Pd, 2.5)));
            Cb = beta * fs;
            S = -wsm * Cb * Pd;
        }
    }
    return S;
}

/* source_nchs (Sediment_Transport.cu:52-60) */
static double source_nchs(const HydCaseParams* P, double wsm, double Zf, double Dxr, double Ufr, double Uf,
                          double h_moi, double fs) {
    double S = 0;
    const double gamac = 0.434 + 5.975 * Zf + 2.888 * Zf * Zf;
    const double Tx = fmax(0.0, (Uf * Uf - Ufr * Ufr) / (Ufr * Ufr));
    const double Cac = 0.015 * P->dm * pow(Tx, 1.5) * pow(Dxr, (-0.3)) / (0.05 * h_moi);
    S = wsm * (Cac - gamac * fs);
    return S;
}

/* Find_VTH (Sediment_Transport.cu:541-568) */
static void k_find_vth(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
#pragma omp parallel for schedule(static)
    for (int i = 2; i <= N; i++)
        for (int j = 2; j <= M; j++) {
            const int pos = i * W + j;
            if ((s->htaiz[pos] > s->P.NANGDAY) && (s->H_moi[pos] > s->P.H_TINH)) {
                const double ut = (s->t_u[pos] + s->t_u[pos - W]) * 0.5;
                const double vt = (s->t_v[pos] + s->t_v[pos - 1]) * 0.5;
                s->VTH[pos] = sqrt(ut * ut + vt * vt);
            } else
                s->VTH[pos] = 0;
        }
}

/* hesoK (Sediment_Transport.cu:508-539) */
static void k_hesok(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const double g = s->P.g, Ks = s->P.Ks;
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= N; i++)
        for (int j = 0; j <= M; j++) {
            double Cz = 0;
            const int pos = i * W + j;
            if (s->Htdu[pos] > 0) {
                Cz = 18 * log(12 * s->Htdu[pos] / Ks);
                s->Kx[pos] = 5.93 * sqrt(g) * (s->h[pos - 1] + s->h[pos]) * 0.25 * fabs(s->t_u[pos]) / Cz;
                s->Kx[pos] = fmin(100.0, fmax(5.0, s->Kx[pos]));
            }
            if (s->Htdv[pos] > 0) {
                Cz = 18 * log(12 * s->Htdv[pos] / Ks);
                s->Ky[pos] = 5.93 * sqrt(g) * (s->h[pos - W] + s->h[pos]) * 0.25 * fabs(s->t_v[pos]) / Cz;
                s->Ky[pos] = fmin(100.0, fmax(5.0, s->Ky[pos]));
            }
        }
}

/* Scan_FSj + _FSj_calculate__mactrix_coeff (Sediment_Transport.cu:594-606, 205-302):
 * column line j, interior cells first+1..last-1 of each segment. */
static void fsj_coeff(OraSim* s, int j, double t, double s_start) {
    const int N = s->N, W = s->W;
    const HydCaseParams* P = &s->P;
    const double *FS = s->FS, *H_moi = s->H_moi, *t_u = s->t_u, *t_v = s->t_v, *VTH = s->VTH,
                 *Htdu = s->Htdu, *Htdv = s->Htdv, *Fw = s->Fw, *Kx = s->Kx, *Ky = s->Ky;
    const int tw = N + 3;
    double *AA = s->AA + (size_t)j * tw, *BB = s->BB + (size_t)j * tw, *CC = s->CC + (size_t)j * tw,
           *DD = s->DD + (size_t)j * tw;
    const double H_TINH = P->H_TINH, dX2 = P->dX2, dXbp = P->dXbp, dY2 = P->dY2, dYbp = P->dYbp;
    for (int k = 0; k < s->mocj[j]; k++) {
        int first = 0, last = 0, br1 = 0, br2 = 0;
        loc_seg_u(s, s->dauj[j * SEGL + k], j, &first, &last, &br1, &br2);
        for (int i = first + 1; i <= last - 1; i++) {
            const int pos = i * W + j;
            const double c = 18 * log(12 * H_moi[pos] / P->Ks);
            const double Uf = sqrt(P->g) * fabs(VTH[pos]) / c;
            const double wsm = s->wss * pow((1 - FS[pos]), 4);
            double Zf = 0;
            double S = 0;
            const double gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
            if (FS[pos] > 0.00001) Zf = wsm / (0.4 * (Uf + 2 * wsm));
            if (P->ketdinh) S = source_chs(P, wsm, Zf, FS[pos], Fw[pos], VTH[pos], H_moi[pos]);
            else S = source_nchs(P, wsm, Zf, s->dxr, s->ufr, Uf, H_moi[pos], FS[pos]);
            if (t < s_start) S = 0;
            AA[i] = -gamav * 0.5 * (t_u[pos] + t_u[pos - W]) / dX2 - Htdu[pos - W] * Kx[pos - W] / (H_moi[pos] * (dXbp));
            CC[i] = gamav * 0.5 * (t_u[pos] + t_u[pos - W]) / dX2 - Htdu[pos] * Kx[pos] / (H_moi[pos] * (dXbp));
            BB[i] = P->HaiChiadT + (Htdu[pos] * Kx[pos] + Htdu[pos - W] * Kx[pos - W]) / (H_moi[pos] * (dXbp));
            double p, q;
            p = q = 0;
            if ((H_moi[pos - 1] > H_TINH) && (H_moi[pos + 2] > H_TINH)) p = (FS[pos + 1] - FS[pos]);
            if ((H_moi[pos - 2] > H_TINH) && (H_moi[pos + 1] > H_TINH)) q = (FS[pos] - FS[pos - 1]);
            p = (1 / (H_moi[pos] * dYbp)) * (Htdv[pos] * Ky[pos] * p - Htdv[pos - 1] * Ky[pos - 1] * q);
            if ((H_moi[pos - 2] > H_TINH) && (H_moi[pos + 2] > H_TINH)) {
                q = (FS[pos + 1] - FS[pos - 1]) / dY2;
                q = (t_v[pos] + t_v[pos - 1]) * 0.5 * q * gamav;
            } else
                q = 0;
            DD[i] = FS[pos] / (P->dT * 0.5) - q + p + (S / H_moi[pos]);
            if (i == first + 1) {
                if ((br1) || (t_u[first * W + j] == 0)) BB[i] += AA[i];
                else DD[i] -= AA[i] * FS[first * W + j];
            }
            if (i == last - 1) {
                if ((br2) && (t_u[last * W + j] == 0)) BB[i] += CC[i];
                else DD[i] -= CC[i] * FS[last * W + j];
                s->SN[j * SEGL + k] = last - first - 2;
            }
        }
    }
}

/* Scan_FSi + _FSi_calculate__mactrix_coeff (Sediment_Transport.cu:570-580, 62-165): row line i */
static void fsi_coeff(OraSim* s, int i, double t, double s_start) {
    const int M = s->M, W = s->W;
    const HydCaseParams* P = &s->P;
    const double *FS = s->FS, *H_moi = s->H_moi, *t_u = s->t_u, *t_v = s->t_v, *VTH = s->VTH,
                 *Htdu = s->Htdu, *Htdv = s->Htdv, *Fw = s->Fw, *Kx = s->Kx, *Ky = s->Ky;
    const int tw = M + 3;
    double *AA = s->AA + (size_t)i * tw, *BB = s->BB + (size_t)i * tw, *CC = s->CC + (size_t)i * tw,
           *DD = s->DD + (size_t)i * tw;
    const double H_TINH = P->H_TINH, dX2 = P->dX2, dXbp = P->dXbp, dY2 = P->dY2, dYbp = P->dYbp;
    const int width = W;
    for (int k = 0; k < s->moci[i]; k++) {
        int first = 0, last = 0, br1 = 0, br2 = 0;
        loc_seg_v(s, i, s->daui[i * SEGL + k], &first, &last, &br1, &br2);
        for (int j = first + 1; j <= last - 1; j++) {
            const int pos = i * W + j;
            const double c = 18 * log(12 * H_moi[pos] / P->Ks);
            const double Uf = sqrt(P->g) * fabs(VTH[pos]) / c;
            const double wsm = s->wss * pow((1 - FS[pos]), 4);
            double Zf = 0;
            if (FS[pos] > 0.00001) Zf = wsm / (0.4 * (Uf + 2 * wsm));
            double S;
            if (P->ketdinh) S = source_chs(P, wsm, Zf, FS[pos], Fw[pos], VTH[pos], H_moi[pos]);
            else S = source_nchs(P, wsm, Zf, s->dxr, s->ufr, Uf, H_moi[pos], FS[pos]);
            if (t < s_start) S = 0;
            const double gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
            AA[j] = -gamav * 0.5 * (t_v[pos - 1] + t_v[pos]) / dY2 - Htdv[pos - 1] * Ky[pos - 1] / (H_moi[pos] * dYbp);
            CC[j] = gamav * 0.5 * (t_v[pos - 1] + t_v[pos]) / dY2 - Htdv[pos] * Ky[pos] / (H_moi[pos] * dYbp);
            BB[j] = P->HaiChiadT + (Htdv[pos] * Ky[pos] + Htdv[pos - 1] * Ky[pos - 1]) / (H_moi[pos] * dYbp);
            double p, q;
            p = 0;
            q = 0;
            if ((H_moi[pos + 2 * width] > H_TINH) && (H_moi[pos - width] > H_TINH)) p = (FS[pos + width] - FS[pos]);
            if (H_moi[pos - 2 * width] > H_TINH && H_moi[pos + width] > H_TINH) q = (FS[pos] - FS[pos - width]);
            p = (1 / (H_moi[pos] * dXbp)) * (Htdu[pos] * Kx[pos] * p - Htdu[pos - width] * Kx[pos - width] * q);
            if (H_moi[pos + 2 * width] > H_TINH && H_moi[pos - 2 * width] > H_TINH) {
                q = (FS[pos + width] - FS[pos - width]) / dX2;
                q = (t_u[pos] + t_u[pos - width]) * 0.5 * q * gamav;
            } else
                q = 0;
            DD[j] = FS[pos] / (P->dT * 0.5) - q + p + (S / H_moi[pos]);
            if (j == first + 1) {
                if ((br1) || (t_v[i * width + first] == 0)) BB[j] = BB[j] + AA[j];
                else DD[j] = DD[j] - AA[j] * FS[i * width + first];
            }
            if (j == last - 1) {
                if ((br2) || (t_v[i * width + last] == 0)) BB[j] = BB[j] + CC[j];
                else DD[j] = DD[j] - CC[j] * FS[i * width + last];
                s->SN[i * SEGL + k] = last - first - 2;
            }
        }
    }
}

/* FSj_extract_solution (Sediment_Transport.cu:608-617, 305-338) */
static void fsj_extract(OraSim* s, int j) {
    const int N = s->N, W = s->W;
    const double* x = s->x + (size_t)j * (N + 3);
    for (int k = 0; k < s->mocj[j]; k++) {
        int first = 0, last = 0, br1 = 0, br2 = 0;
        loc_seg_u(s, s->dauj[j * SEGL + k], j, &first, &last, &br1, &br2);
        for (int i = first + 1; i <= last - 1; i++) {
            const int pos = i * W + j;
            s->tFS[pos] = x[i];
            if (x[i] < 0) s->tFS[pos] = s->P.NDnen;
            if (i == first + 1) {
                if ((br1) || (s->t_u[pos - W] == 0)) s->tFS[first * W + j] = s->tFS[pos];
                else s->tFS[first * W + j] = s->FS[first * W + j];
            }
            if (i == last - 1) {
                if ((br2) || (s->t_u[pos + W] == 0)) s->tFS[last * W + j] = s->tFS[pos];
                else s->tFS[last * W + j] = s->FS[last * W + j];
            }
        }
    }
}

/* FSi_extract_solution (Sediment_Transport.cu:581-591, 168-202) */
static void fsi_extract(OraSim* s, int i) {
    const int M = s->M, W = s->W;
    double* x = s->x + (size_t)i * (M + 3);
    for (int k = 0; k < s->moci[i]; k++) {
        int first = 0, last = 0, br1 = 0, br2 = 0;
        loc_seg_v(s, i, s->daui[i * SEGL + k], &first, &last, &br1, &br2);
        for (int j = first + 1; j <= last - 1; j++) {
            const int pos = i * W + j;
            if (x[j] < 0) x[j] = s->P.NDnen;
            s->tFS[pos] = x[j];
            if (j == first + 1) {
                if ((br1) || (s->t_v[i * W + first] == 0)) s->tFS[i * W + first] = s->tFS[pos];
                else s->tFS[i * W + first] = s->FS[i * W + first];
            }
            if (j == last - 1) {
                if ((br2) || (s->t_v[i * W + last] == 0)) s->tFS[i * W + last] = s->tFS[pos];
                else s->tFS[i * W + last] = s->FS[i * W + last];
            }
        }
    }
}

/* FS tridiagonal solves of one sweep (tridiagSolver with jumpstep 1).  Segments too
 * short to have an interior row run on whatever SN holds, exactly like the reference;
 * their results are never read.  Those run first and serially, so that the solves
 * whose results are read are the last writers of their rows. */
static void fs_solves(OraSim* s, int isU, int startidx, int endidx) {
    const int width = isU ? s->N + 3 : s->M + 3;
    const int* moc = isU ? s->mocj : s->moci;
    const int* dau = isU ? s->dauj : s->daui;
    const int* cuoi = isU ? s->cuoij : s->cuoii;
    for (int line = startidx; line <= endidx; line++)
        for (int k = 0; k < moc[line]; k++)
            if (cuoi[line * SEGL + k] - dau[line * SEGL + k] < 2)
                solve_at(s, (size_t)line * width + dau[line * SEGL + k] + 1, s->SN[line * SEGL + k]);
#pragma omp parallel for schedule(dynamic, 4)
    for (int line = startidx; line <= endidx; line++)
        for (int k = 0; k < moc[line]; k++)
            if (cuoi[line * SEGL + k] - dau[line * SEGL + k] >= 2)
                solve_at(s, (size_t)line * width + dau[line * SEGL + k] + 1, s->SN[line * SEGL + k]);
}

/* Update_FS (Sediment_Transport.cu:620-629) */
static void k_update_fs(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= N; i++)
        for (int j = 1; j <= M; j++) s->FS[i * W + j] = s->tFS[i * W + j];
}

static void sediment_fsj(OraSim* s, double t, double s_start) {
    const int M = s->M;
    /* Engine.py:219-239 */
    k_find_vth(s);
    k_hesok(s);
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 3; j <= M - 1; j++) fsj_coeff(s, j, t, s_start);
    fs_solves(s, 1, 3, M - 1);
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 3; j <= M - 1; j++) fsj_extract(s, j);
    k_update_fs(s);
}

static void sediment_fsi(OraSim* s, double t, double s_start) {
    const int N = s->N;
    /* Engine.py:339-361 */
    k_find_vth(s);
    k_hesok(s);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 3; i <= N - 1; i++) fsi_coeff(s, i, t, s_start);
    fs_solves(s, 0, 3, N - 1);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 3; i <= N - 1; i++) fsi_extract(s, i);
    k_update_fs(s);
}

/* Calculate_Qb (Sediment_Transport.cu:341-414).  With the library's bed_feedback option
 * (no reference counterpart) the flux is evaluated where VTH > 0 instead of VTH == 0
 * (quirk Q3). */
static void k_calculate_qb(OraSim* s) {
    const int N = s->N, M = s->M, width = s->W;
    const HydCaseParams* P = &s->P;
    double *Qbx = s->Qbx, *Qby = s->Qby;
#pragma omp parallel for schedule(static)
    for (int i = 2; i <= N; i++)
        for (int j = 2; j <= M; j++) {
            double Tob;
            double Toee = P->Toe;
            double Tx = 0;
            const int pos = i * width + j;
            if ((P->bed_feedback ? s->VTH[pos] > 0 : !s->VTH[pos]) && (s->khouot[pos] == 0)) {
                Tob = P->ro * s->Fw[pos] * (s->VTH[pos] * s->VTH[pos]);
                if (s->H_moi[pos] > P->ghtoe) Toee = P->Toe * (1 + P->hstoe * ((s->H_moi[pos] - P->ghtoe)));
                if (Tob > Toee) Tx = Tob / Toee - 1;
                Qbx[pos] = 0.053 * pow((P->Sx - 1) * P->g, 0.5) * pow(P->dm, 1.5) * pow(Tx, 2.1) * pow(s->dxr, -0.3) *
                           (s->t_u[pos] + s->t_u[pos - width]) * 0.5 / s->VTH[pos];
                Qby[pos] = 0.053 * pow((P->Sx - 1) * P->g, 0.5) * pow(P->dm, 1.5) * pow(Tx, 2.1) * pow(s->dxr, -0.3) *
                           (s->t_v[pos] + s->t_v[pos - 1]) * 0.5 / s->VTH[pos];
            } else {
                Qbx[pos] = 0;
                Qby[pos] = 0;
            }
        }
    /* edge copies, in launch order (the unbraced statements at 394-398 run for every i) */
    for (int i = 2; i <= N; i++)
        for (int j = 2; j <= M; j++) {
            const int pos = i * width + j;
            if (i == 2) {
                Qbx[pos - width] = Qbx[pos];
                Qby[pos - width] = Qby[pos];
            }
            if (i == N) {
                Qbx[pos + width] = Qbx[pos];
                Qby[pos + width] = Qby[pos];
            }
            if (j == 2) {
                Qbx[pos - 1] = Qbx[pos];
                Qby[pos - 1] = Qby[pos];
                if (i == 2) Qbx[1 * width + 1] = Qbx[pos];
                Qby[1 * width + 1] = Qby[pos];
                if (i == N) Qbx[(N + 1) * width + 1] = Qbx[pos];
                Qby[(N + 1) * width + 1] = Qby[pos];
            }
            if (j == M) {
                Qbx[pos + 1] = Qbx[pos];
                Qby[pos + 1] = Qby[pos];
                if (i == 2) {
                    Qbx[1 * width + M + 1] = Qbx[pos];
                    Qby[1 * width + M + 1] = Qby[pos];
                }
                if (i == N) {
                    Qbx[(N + 1) * width + M + 1] = Qbx[pos];
                    Qby[(N + 1) * width + M + 1] = Qby[pos];
                }
            }
        }
}

/* BedLoad + _bed_load (Sediment_Transport.cu:630-639, 416-506): rows startidx..endidx-1.
 * With the library's bed_feedback option (no reference counterpart): the upwind test reads
 * t_u[pos] > 0 (quirk Q4) and the update's raw bed change, morfac * bed_period / (1 - Dorong)
 * * rate (0 if not finite), is stored in dHinc (NaN at the cells not computed) for
 * bed_feedback_apply. */
static void k_bedload(OraSim* s, int startidx, int endidx) {
    const int N = s->N, M = s->M, width = s->W;
    const HydCaseParams* P = &s->P;
    const double *FS = s->FS, *H_moi = s->H_moi, *t_u = s->t_u, *t_v = s->t_v, *VTH = s->VTH,
                 *Htdu = s->Htdu, *Htdv = s->Htdv, *Fw = s->Fw, *Kx = s->Kx, *Ky = s->Ky, *Qbx = s->Qbx,
                 *Qby = s->Qby;
    const int* khouot = s->khouot;
    const double dX2 = P->dX2, dY2 = P->dY2, dXbp = P->dXbp, dYbp = P->dYbp;
    if (P->bed_feedback) {
        for (int i = startidx; i < endidx; i++)
            for (int j = 2; j <= M; j++) s->dHinc[i * width + j] = NAN;
    }
#pragma omp parallel for schedule(static)
    for (int i = startidx; i < endidx; i++)
        for (int j = 2; j <= M + 2; j++) {
            int first = 0, last = 0, br1 = 0, br2 = 0;
            loc_seg_v(s, i, j, &first, &last, &br1, &br2);
            if (last - first < 2 || j < first || j > last) continue;
            const int pos = i * width + j;
            double p, q;
            p = q = 0;
            if (khouot[pos - width] == 1) {
                if (t_u[pos] < 0) p = (-3 * Qbx[pos] + 4 * Qbx[pos + width] - Qbx[pos + 2 * width]) / dX2;
            } else {
                if (khouot[pos + width] == 1) {
                    if (P->bed_feedback ? t_u[pos] > 0 : t_u[pos > 0] != 0)
                        p = (3 * Qbx[pos] - 4 * Qbx[pos - width] + Qbx[pos - 2 * width]) / dX2;
                } else
                    p = (Qbx[pos + width] - Qbx[pos - width]) / dX2;
            }
            if (khouot[pos - 1] == 1) {
                if (t_v[pos] < 0) q = (-3 * Qby[pos] + 4 * Qby[pos + 1] - Qby[pos + 2]) / dY2;
            } else {
                if (khouot[pos + 1] == 1) {
                    if (t_v[pos] > 0) q = (3 * Qby[pos] - 4 * Qby[pos - 1] + Qby[pos - 2]) / dY2;
                } else
                    q = (Qby[pos + 1] - Qby[pos - 1]) / dY2;
            }
            double tH = p + q;
            p = FS[pos + width] - FS[pos];
            if ((khouot[pos + 2 * width] == 1 || khouot[pos - width] == 1) && (i < N)) p = 0;
            q = FS[pos] - FS[pos - width];
            if ((i > 2) && (khouot[pos - 2 * width] == 1 || khouot[pos + width] == 1)) q = 0;
            p = 1 / dXbp * (Htdu[pos] * Kx[pos] * p - Htdu[pos - width] * Kx[pos - width] * q);
            tH = tH + p;
            p = FS[pos + 1] - FS[pos];
            if (((last < M) && (khouot[pos - 1] == 1 || khouot[pos + 2] == 1)) || (last == M && (khouot[pos - 1] == 1)))
                p = 0;
            q = FS[pos] - FS[pos - 1];
            if (((first > 2) && (khouot[pos - 2] == 1 || khouot[pos + 1] == 1)) || (first == 2 && khouot[pos + 1] == 1))
                q = 0;
            p = 1 / (dYbp) * (Htdv[pos] * Ky[pos] * p - Htdv[pos - 1] * Ky[pos - 1] * q);
            tH = tH + p;
            const double c = 18 * log(12 * H_moi[pos] / P->Ks);
            const double Uf = sqrt(P->g) * fabs(VTH[pos]) / c;
            const double wsm = s->wss * pow((1 - FS[pos]), 4);
            double Zf = 0;
            double S = 0;
            if (FS[pos] > 0.0) Zf = wsm / (0.4 * (Uf + 2 * wsm));
            if (P->ketdinh) S = source_chs(P, wsm, Zf, FS[pos], Fw[pos], VTH[pos], H_moi[pos]);
            else S = source_nchs(P, wsm, Zf, s->dxr, s->ufr, Uf, H_moi[pos], FS[pos]);
            if (!P->bed_feedback) {
                s->dH[pos] += P->dT / (1 - P->Dorong) * (S + tH);
                continue;
            }
            if (j <= M) {
                const double period = P->bed_period > 0 ? P->bed_period : P->bed_change_start;
                double x = P->morfac * period / (1 - P->Dorong) * (S + tH);
                if (!isfinite(x)) x = 0.0;
                s->dHinc[pos] = x;
            }
        }
}

/* The fed-back bed change of one update (no reference counterpart).  The explicit Exner
 * rate from central bed-load and diffusion differences carries a grid-scale (2 dx)
 * oscillation, which a morphological step of many minutes turns into a checkerboard bed
 * that the hydraulics do not survive; so the raw change is filtered by the 3 x 3 binomial
 * kernel (weights 1 2 1 x 1 2 1, renormalised over the computed neighbours in rows
 * startidx..endidx-1, columns 2..M), which removes the 2 dx mode exactly and keeps smooth
 * changes, then limited to BED_LIMIT of the depth and BED_CAP metres, added to dH as a
 * Kahan sum and applied to the bed, h = h0 + dH.  Cells within bed_fixed cells of the
 * grid's edges, and cells with less than bed_min_depth of water, keep their bed. */
static void bed_feedback_apply(OraSim* s, int startidx, int endidx) {
    const int N = s->N, M = s->M, width = s->W;
    const int F = s->P.bed_fixed > 0 ? s->P.bed_fixed : 0;
    const double* inc = s->dHinc;
#pragma omp parallel for schedule(static)
    for (int i = startidx; i < endidx; i++)
        for (int j = 2; j <= M; j++) {
            const int pos = i * width + j;
            if (i < 2 + F || i > N - F || j < 2 + F || j > M - F) continue;
            if (s->H_moi[pos] < s->P.bed_min_depth) continue;
            if (!isfinite(inc[pos])) continue;
            double num = 0.0, den = 0.0;
            for (int di = -1; di <= 1; di++) {
                const int ii = i + di;
                if (ii < startidx || ii >= endidx) continue;
                for (int dj = -1; dj <= 1; dj++) {
                    const int jj = j + dj;
                    if (jj < 2 || jj > M) continue;
                    const double v = inc[ii * width + jj];
                    if (!isfinite(v)) continue;
                    const double w = (di == 0 ? 2.0 : 1.0) * (dj == 0 ? 2.0 : 1.0);
                    num += w * v;
                    den += w;
                }
            }
            double x = num / den;
            const double lim = fmin(BED_LIMIT * s->H_moi[pos], BED_CAP);
            x = fmin(fmax(x, -lim), lim);
            const double y = x - s->dHc[pos];
            const double sum = s->dH[pos] + y;
            s->dHc[pos] = (sum - s->dH[pos]) - y;
            s->dH[pos] = sum;
            s->h[pos] = s->h0[pos] + sum;
        }
}

/* After a fed-back bed change (no reference counterpart): what the set-up derived from h
 * re-derived for the new bed: htaiz, htaiz_bd, Kx1, Ky1 (the set-up's formula; a face depth
 * below datum that is not positive, where the set-up's pow has no real value, taken as H_TINH)
 * (Onetime_init,
 * support_funcs.cu:20-58), H_moi of the wet cells (update_h_moi, 60-73), Htuongdoi and
 * preprocess_data. */
static void bed_feedback_derive(OraSim* s) {
    const int N = s->N, M = s->M, W = s->W;
    const HydCaseParams* P = &s->P;
    const double* h = s->h;
    for (int i = 1; i <= N; i++)
        for (int j = 1; j <= M; j++) {
            const size_t ij = (size_t)i * W + j;
            s->htaiz[ij] = (h[(i - 1) * W + j - 1] + h[(i - 1) * W + j] + h[i * W + j - 1] + h[i * W + j]) * 0.25;
            s->htaiz_bd[ij] = s->htaiz[ij];
            if (h[i * W + j - 1] + h[i * W + j] != 0) {
                const double d = (h[i * W + j - 1] + h[i * W + j]) * 0.5;
                s->Kx1[ij] = P->g * pow(d > 0 ? d : P->H_TINH, -2 * P->mu_mn) *
                             pow((s->hsnham[i * W + j - 1] + s->hsnham[i * W + j]) * 0.5, 2);
            }
            if (h[(i - 1) * W + j] + h[i * W + j] != 0) {
                const double d = (h[(i - 1) * W + j] + h[i * W + j]) * 0.5;
                s->Ky1[ij] = P->g * pow(d > 0 ? d : P->H_TINH, -2 * P->mu_mn) *
                             pow((s->hsnham[(i - 1) * W + j] + s->hsnham[i * W + j]) * 0.5, 2);
            }
            if (s->khouot[ij] == 0) s->H_moi[ij] = s->htaiz[ij] + s->z[ij];
        }
    k_htuongdoi(s);
    k_preprocess(s);
}

/* ---------------------------------------------------------- time loop */

static int g_trace = 0;
void ora_set_trace(int on) { g_trace = on; }

/* Debug aid: report the first non-finite value of the main fields after a phase. */
static void trace(const OraSim* s, const char* phase) {
    if (!g_trace) return;
    const char* names[] = {"t_z", "t_u", "t_v", "z", "u", "v", "H_moi", "FS", "tFS"};
    const double* arrs[] = {s->t_z, s->t_u, s->t_v, s->z, s->u, s->v, s->H_moi, s->FS, s->tFS};
    for (int k = 0; k < 9; k++)
        for (size_t q = 0; q < s->nf; q++)
            if (!isfinite(arrs[k][q])) {
                fprintf(stderr, "t=%g after %s: %s[%zu,%zu] = %g\n", s->t, phase, names[k], q / s->W,
                        q % s->W, arrs[k][q]);
                return;
            }
}
#define TRACE(name) trace(s, name)

/* One iteration of the while loop of Engine.hydraulic_Calculation (Engine.py:144-366). */
/* ------------------------------------------------------------ water account
 * The terms of the library's water budget (hyd_mass_budget) restated on the oracle's step,
 * so that their definitions can be checked against the volume of the oracle's own fields:
 * water[0] volume in through the domain's edge faces, water[1] opened, water[2] closed,
 * water[3] lost to wet cells a sweep leaves unsolved (flux into them, less the stage level
 * the boundary puts on them), water[4] edge faces taken from a one-cell segment's
 * continuity (count).  m^3, accumulated over the steps.  No reference counterpart. */
static int in_seg(const OraSim* s, int isU, int i, int j, int* f, int* l) {
    if (isU) {
        for (int k = 0; k < s->mocj[j]; k++)
            if (s->dauj[j * SEGL + k] <= i && i <= s->cuoij[j * SEGL + k]) {
                *f = s->dauj[j * SEGL + k];
                *l = s->cuoij[j * SEGL + k];
                return 1;
            }
    } else {
        for (int k = 0; k < s->moci[i]; k++)
            if (s->daui[i * SEGL + k] <= j && j <= s->cuoii[i * SEGL + k]) {
                *f = s->daui[i * SEGL + k];
                *l = s->cuoii[i * SEGL + k];
                return 1;
            }
    }
    return 0;
}

static void water_sweep(OraSim* s, int isU) {
    const int N = s->N, M = s->M, W = s->W;
    const double dX = s->P.dX, dY = s->P.dY, h = s->P.dT * 0.5;
    const double* xu = isU ? s->t_u : s->u;
    const double* yv = isU ? s->v : s->t_v;
    const double* zo = s->w_zold;
    double edge = 0.0, leak = 0.0;
    for (int e = 0; e < 4; e++) {
        const int n = e >= 2 ? M : N;
        for (int k = 2; k <= n; k++) {
            int i, j, fp;
            double sgn;
            if (e == 0) { i = k; j = M; fp = i * W + M; sgn = -1.0; }
            else if (e == 1) { i = k; j = 2; fp = i * W + 1; sgn = 1.0; }
            else if (e == 2) { i = 2; j = k; fp = W + j; sgn = 1.0; }
            else { i = N; j = k; fp = N * W + j; sgn = -1.0; }
            const int c = i * W + j;
            int f, l;
            if (s->khouot[c] != 0 || !in_seg(s, isU, i, j, &f, &l)) continue;
            if (f == l && (isU ? e == 2 : e == 1)) {
                const double west = h * dY * s->Htdu[c - W] * xu[c - W], east = -h * dY * s->Htdu[c] * xu[c];
                const double south = h * dX * s->Htdv[c - 1] * yv[c - 1], north = -h * dX * s->Htdv[c] * yv[c];
                const double dv = (s->t_z[c] - zo[c]) * dX * dY;
                edge += e == 2 ? dv - (east + south + north) : dv - (west + east + north);
                s->water[4] += 1;
            } else {
                const double q = e >= 2 ? s->Htdu[fp] * xu[fp] * dY : s->Htdv[fp] * yv[fp] * dX;
                edge += sgn * q * h;
            }
        }
    }
    for (int i = isU ? N - 1 : 2; i <= N; i++)
        for (int j = isU ? 2 : M - 1; j <= M; j++) {
            const int c = i * W + j;
            int f, l;
            if (s->khouot[c] != 0) continue;
            if (!in_seg(s, isU, i, j, &f, &l)) {
                leak -= (s->t_z[c] - zo[c]) * dX * dY;
                continue;
            }
            double q = 0.0;
            if (isU) {
                if (j + 1 <= M && s->khouot[c + 1] == 0 && !in_seg(s, 1, i, j + 1, &f, &l)) q += s->Htdv[c] * s->v[c];
                if (j - 1 >= 2 && s->khouot[c - 1] == 0 && !in_seg(s, 1, i, j - 1, &f, &l))
                    q -= s->Htdv[c - 1] * s->v[c - 1];
                leak += q * dX * h;
            } else {
                if (i + 1 <= N && s->khouot[c + W] == 0 && !in_seg(s, 0, i + 1, j, &f, &l)) q += s->Htdu[c] * s->u[c];
                if (i - 1 >= 2 && s->khouot[c - W] == 0 && !in_seg(s, 0, i - 1, j, &f, &l))
                    q -= s->Htdu[c - W] * s->u[c - W];
                leak += q * dY * h;
            }
        }
    s->water[0] += edge;
    s->water[3] += leak;
}

static void water_reset(OraSim* s, int after) {
    const int N = s->N, M = s->M, W = s->W;
    const double area = s->P.dX * s->P.dY;
    if (!after) {
        memcpy(s->w_kh, s->khouot, sizeof(int) * s->nf);
        memcpy(s->w_H, s->H_moi, sizeof(double) * s->nf);
        return;
    }
    for (int i = 2; i <= N; i++)
        for (int j = 2; j <= M; j++) {
            const int c = i * W + j;
            if (s->w_kh[c] != 0 && s->khouot[c] == 0) s->water[1] += s->H_moi[c] * area;
            if (s->w_kh[c] == 0 && s->khouot[c] != 0) s->water[2] += s->w_H[c] * area;
        }
}

void ora_water_enable(OraSim* s, double* acc) {
    s->water = acc;
    if (acc && !s->w_zold) {
        s->w_zold = (double*)ora_alloc(s, s->nf, sizeof(double), 0);
        s->w_H = (double*)ora_alloc(s, s->nf, sizeof(double), 0);
        s->w_kh = (int*)ora_alloc(s, s->nf, sizeof(int), 0);
    }
}

static void full_step(OraSim* s) {
    const int N = s->N, M = s->M;
    const HydCaseParams* P = &s->P;
    const int channel = P->kenhhepd || P->kenhhepng;
    double t = s->t;
    /* ---- half-step 1: implicit along i (columns), explicit v ---- */
    t = t + P->dT * 0.5;
    if (channel)
        k_boundary_channel(s, t);
    else
        k_boundary(s, t);
    TRACE("k_boundary");
    int start_idx = 2, end_idx = M;
    if (channel && P->kenhhepd == 1) {
        start_idx = 3;
        end_idx = M - 1;
    }
    if (s->water) memcpy(s->w_zold, s->z, sizeof(double) * s->nf);
    k_uz_sweep(s, start_idx, end_idx); TRACE("k_uz_sweep");
    if (s->water) water_sweep(s, 1);
    k_normalize(s, 1); TRACE("normalize_u");
    k_solve_v(s); TRACE("k_solve_v");
    k_margin_v(s); TRACE("k_margin_v");
    k_normalize(s, 0); TRACE("normalize_v");
    k_update_h_moi(s); TRACE("k_update_h_moi");
    if (s->water) water_reset(s, 0);
    k_reset_horizontal(s); TRACE("k_reset_horizontal");
    if (s->water) water_reset(s, 1);
    k_update_uvz(s); TRACE("k_update_uvz");
    k_limits_horizontal(s);
    k_limits_vertical(s); TRACE("k_limits_vertical");
    k_htuongdoi(s); TRACE("k_htuongdoi");
    if (t >= P->sediment_start) {
        start_idx = 3;
        end_idx = M - 1;
        sediment_fsj(s, t, P->bed_change_start); TRACE("sediment_fsj");
    }
    /* ---- half-step 2: implicit along j (rows), explicit u ---- */
    t = t + P->dT * 0.5;
    if (channel)
        k_boundary_channel(s, t);
    else
        k_boundary(s, t);
    TRACE("k_boundary");
    start_idx = 2;
    end_idx = N;
    if (channel && P->kenhhepng == 1) {
        start_idx = 3;
        end_idx = N;
    }
    if (s->water) memcpy(s->w_zold, s->z, sizeof(double) * s->nf);
    k_vz_sweep(s, start_idx, end_idx); TRACE("k_vz_sweep");
    if (s->water) water_sweep(s, 0);
    k_normalize(s, 0); TRACE("normalize_v");
    k_solve_u(s); TRACE("k_solve_u");
    k_margin_u(s); TRACE("k_margin_u");
    k_normalize(s, 1); TRACE("normalize_u");
    k_update_h_moi(s); TRACE("k_update_h_moi");
    if (s->water) water_reset(s, 0);
    k_reset_vertical(s); TRACE("k_reset_vertical");
    if (s->water) water_reset(s, 1);
    k_update_uvz(s); TRACE("k_update_uvz");
    k_limits_horizontal(s);
    k_limits_vertical(s); TRACE("k_limits_vertical");
    k_htuongdoi(s); TRACE("k_htuongdoi");
    if (t >= P->sediment_start) {
        start_idx = 3;
        end_idx = N - 1;
        sediment_fsi(s, t, P->bed_change_start); TRACE("sediment_fsi");
    }
    /* Engine.py:364: int(t) % bed_change_start == 0 and t integral; with the library's
       bed_period, every bed_period s from bed_change_start on */
    {
        const double it = (double)(long long)t;
        const int bed = P->bed_period > 0
                            ? (t - it == 0 && t >= P->bed_change_start && fmod(it, P->bed_period) == 0)
                            : (fmod(it, P->bed_change_start) == 0 && t - it == 0);
        if (bed) {
            k_calculate_qb(s);
            k_bedload(s, start_idx, end_idx);
            if (P->bed_feedback) {
                bed_feedback_apply(s, start_idx, end_idx);
                bed_feedback_derive(s);
            }
        }
    }
    s->start_idx = start_idx;
    s->end_idx = end_idx;
    s->t = t;
}

void ora_step(OraSim* s, int nsteps) {
    for (int n = 0; n < nsteps; n++) full_step(s);
}
