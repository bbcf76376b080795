/*
 * ref_harness.cpp — runs the reference's own kernel sources, unmodified, launch for
 * launch as rep.py:gpu_init (rep.py:58-139) and Engine.hydraulic_Calculation
 * (Engine.py:144-366) launch them.
 *
 * TEST INFRASTRUCTURE ONLY.  PyCUDA and Python 2 are not available offline, so this
 * C++ host replaces them.  The recipe (oracle/Makefile) compiles this file together
 * with support_funcs.cu, UVZSolver_multithread.cu and Sediment_Transport.cu from the
 * reference tree, in two builds, both written to oracle/_ref/:
 *   - HYDREF_CPU: g++ with oracle/cuda_emu.h, executed on the CPU (no GPU needed);
 *   - default:    nvcc for sm_100a, executed on the GPU (reference timing arm).
 *
 * Deviations from the reference host, each one forced by undefined behaviour there:
 *   - locate_segment_v/_u (constant.cuh:135-178) fall off the end without a return
 *     value when no segment holds the cell; this harness supplies versions that
 *     return -1 there and behave identically otherwise.
 *   - hi is allocated as doubles (the reference allocates float32 and writes doubles,
 *     Global_Variables.py:113, support_funcs.cu:451-511).
 *   - every buffer is zero-filled and padded, so the few reads and writes the
 *     reference makes just outside an array land in padding.
 *   - update_uvz receives 0 for its kenhhepd/kenhhepng parameters: Engine.py:90
 *     passes two arguments fewer than the kernel declares (support_funcs.cu:671),
 *     so those parameters are never the flags the host meant.
 */
#ifdef HYDREF_CPU
#include "cuda_emu.h"
emu_uint3 threadIdx, blockIdx;
dim3 blockDim, gridDim;
#else
#include <cuda_runtime.h>
#endif

#include <cstdint>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/hydist_b200.h"

/* constant.cuh with its two segment lookups set aside, then this harness's versions */
#define locate_segment_v hydref_unused_locate_segment_v
#define locate_segment_u hydref_unused_locate_segment_u
#include "constant.cuh"
#undef locate_segment_v
#undef locate_segment_u

__device__ int locate_segment_v(int N, int M, bool* bienran1, bool* bienran2, int* first, int* last,
                                int row, int col, int* daui, int* cuoii, int* moci, DOUBLE* h) {
    (void)N;
    const int nk = moci[row];
    for (int k = 0; k < nk; k++) {
        const int a = daui[row * segment_limit + k];
        const int b = cuoii[row * segment_limit + k];
        if (a > col || col > b) continue;
        *first = a;
        *last = b;
        const int w = M + 3;
        if (a > 2 || (a == 2 && (h[row * w + a - 1] + h[(row - 1) * w + a - 1]) * 0.5 == NANGDAY))
            *bienran1 = true;
        if (b < M || (b == M && (h[row * w + b] + h[(row - 1) * w + b]) * 0.5 == NANGDAY))
            *bienran2 = true;
        return k;
    }
    return -1;
}

__device__ int locate_segment_u(int N, int M, bool* bienran1, bool* bienran2, int* first, int* last,
                                int row, int col, int* dauj, int* cuoij, int* mocj, DOUBLE* h) {
    const int nk = mocj[col];
    for (int k = 0; k < nk; k++) {
        const int a = dauj[col * segment_limit + k];
        const int b = cuoij[col * segment_limit + k];
        if (a > row || row > b) continue;
        *first = a;
        *last = b;
        const int w = M + 3;
        if (a > 2 || (a == 2 && (h[1 * w + col] + h[1 * w + col - 1]) * 0.5 == NANGDAY)) *bienran1 = true;
        if (b < N || (b == N && (h[N * w + col] + h[N * w + col - 1]) * 0.5 == NANGDAY)) *bienran2 = true;
        return k;
    }
    return -1;
}

#include "support_funcs.cu"
#include "UVZSolver_multithread.cu"
#include "Sediment_Transport.cu"

/* ------------------------------------------------------------------ host side */

#ifdef HYDREF_CPU
#define LAUNCH(kern, g, b, ...) emu_launch(g, b, [&]() { kern(__VA_ARGS__); })
#define SYNC() ((void)0)
/* kernels the reference runs with 32 identical threads per line */
#define RED32 dim3(1, 1, 1)
#define RED32Y dim3(1, 1, 1)
#define SETC(sym, val)            \
    do {                          \
        sym = (val);              \
    } while (0)
#else
#define LAUNCH(kern, g, b, ...)                        \
    do {                                               \
        kern<<<(g), (b)>>>(__VA_ARGS__);               \
        ref_check(cudaGetLastError(), #kern);          \
    } while (0)
#define SYNC() ref_check(cudaDeviceSynchronize(), "synchronize")
#define RED32 dim3(32, 1, 1)
#define RED32Y dim3(1, 32, 1)
#define SETC(sym, val)                                               \
    do {                                                             \
        decltype(sym) v_ = (val);                                    \
        ref_check(cudaMemcpyToSymbol(sym, &v_, sizeof(v_)), #sym);   \
    } while (0)
#endif

namespace {

int g_err = 0;
char g_msg[256];

#ifndef HYDREF_CPU
void ref_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess && !g_err) {
        g_err = 1;
        snprintf(g_msg, sizeof g_msg, "%s: %s", what, cudaGetErrorString(e));
    }
}
#endif

struct RefSim {
    int N, M;
    HydCaseParams P;
    Argument_Pointers host_arg;   /* pointer image, as PointersStruct packs it */
    Array_Pointers host_arr;
    Argument_Pointers* arg;       /* device (or host, CPU build) copy */
    Array_Pointers* arr;
    std::vector<void*> blocks;
    int total_time;
    double t;
    size_t nf;
    double last_ms;
};

void* ref_alloc(RefSim* s, size_t bytes, size_t guard) {
    const size_t total = bytes + 2 * guard;
#ifdef HYDREF_CPU
    char* p = (char*)calloc(total, 1);
    if (!p) return nullptr;
#else
    char* p = nullptr;
    if (cudaMalloc(&p, total) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, total);
#endif
    s->blocks.push_back(p);
    return p + guard;
}

void ref_copy_in(void* dst, const void* src, size_t bytes) {
#ifdef HYDREF_CPU
    memcpy(dst, src, bytes);
#else
    ref_check(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "copy in");
#endif
}

void ref_copy_out(void* dst, const void* src, size_t bytes) {
#ifdef HYDREF_CPU
    memcpy(dst, src, bytes);
#else
    ref_check(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "copy out");
#endif
}

void set_constants(const HydCaseParams& P) {
    SETC(dX, P.dX);
    SETC(dY, P.dY);
    SETC(dT, P.dT);
    SETC(dXbp, P.dXbp);
    SETC(dX2, P.dX2);
    SETC(dYbp, P.dYbp);
    SETC(dY2, P.dY2);
    SETC(dTchia2dX, P.dTchia2dX);
    SETC(dTchia2dY, P.dTchia2dY);
    SETC(QuyDoiTime, P.QuyDoiTime);
    SETC(QuyDoiPi, P.QuyDoiPi);
    SETC(HaiChiadT, P.HaiChiadT);
    SETC(NANGDAY, P.NANGDAY);
    SETC(H_TINH, P.H_TINH);
    SETC(Wind, P.Wind);
    SETC(huonggio, P.huonggio);
    SETC(Zbandau, P.Zbandau);
    SETC(heso, P.heso);
    SETC(mu_mn, P.mu_mn);
    SETC(NDnen, P.NDnen);
    SETC(NDbphai, P.NDbphai);
    SETC(NDbtrai, P.NDbtrai);
    SETC(NDbtren, P.NDbtren);
    SETC(NDbduoi, P.NDbduoi);
    SETC(Tod, P.Tod);
    SETC(Toe, P.Toe);
    SETC(hstoe, P.hstoe);
    SETC(ghtoe, P.ghtoe);
    SETC(Mbochat, P.Mbochat);
    SETC(ro, P.ro);
    SETC(ros, P.ros);
    SETC(dm, P.dm);
    SETC(d90, P.d90);
    SETC(muy, P.muy);
    SETC(Dorong, P.Dorong);
    SETC(Sx, P.Sx);
    SETC(sohn, P.sohn);
    SETC(soha, P.soha);
    SETC(sohn1, P.sohn1);
    SETC(CORIOLIS_FORCE, P.CORIOLIS_FORCE);
    SETC(g, P.g);
    SETC(Ks, P.Ks);
}

struct FieldRef {
    const char* name;
    size_t off;  /* offset of the member in Argument_Pointers */
    int is_int;
    int kind;    /* 0 grid field, 1 row table (N+2)*20, 2 col table (M+2)*20, 3 N+2, 4 M+2, 5 hi */
};

#define FR(n, k, isint) {#n, offsetof(Argument_Pointers, n), isint, k}
const FieldRef kFields[] = {
    FR(h, 0, 0),       FR(u, 0, 0),      FR(v, 0, 0),     FR(z, 0, 0),        FR(t_u, 0, 0),
    FR(t_v, 0, 0),     FR(t_z, 0, 0),    FR(Htdu, 0, 0),  FR(Htdv, 0, 0),     FR(H_moi, 0, 0),
    FR(htaiz, 0, 0),   FR(htaiz_bd, 0, 0), FR(hsnham, 0, 0), FR(VISCOIDX, 0, 0), FR(Kx1, 0, 0),
    FR(Ky1, 0, 0),     FR(Tsyw, 0, 0),   FR(Tsxw, 0, 0),  FR(FS, 0, 0),       FR(tFS, 0, 0),
    FR(VTH, 0, 0),     FR(Kx, 0, 0),     FR(Ky, 0, 0),    FR(Fw, 0, 0),       FR(Qbx, 0, 0),
    FR(Qby, 0, 0),     FR(dH, 0, 0),     FR(khouot, 0, 1), FR(daui, 1, 1),    FR(cuoii, 1, 1),
    FR(moci, 3, 1),    FR(dauj, 2, 1),   FR(cuoij, 2, 1), FR(mocj, 4, 1),     FR(ubt, 4, 0),
    FR(ubp, 4, 0),     FR(vbt, 3, 0),    FR(vbd, 3, 0),   FR(hi, 5, 0),
};
#undef FR

size_t kind_count(const RefSim* s, int kind) {
    switch (kind) {
        case 0: return s->nf;
        case 1: return (size_t)(s->N + 2) * HYD_SEGMENT_LIMIT;
        case 2: return (size_t)(s->M + 2) * HYD_SEGMENT_LIMIT;
        case 3: return (size_t)(s->N + 2);
        case 4: return (size_t)(s->M + 2);
        default: return (size_t)(2 * (s->N + 3) + 2 * (s->M + 3));
    }
}

const FieldRef* find_field(const char* name) {
    if (!strcmp(name, "VISCOINDX")) name = "VISCOIDX";
    for (const FieldRef& f : kFields)
        if (!strcmp(f.name, name)) return &f;
    return nullptr;
}

void* member_ptr(RefSim* s, const FieldRef* f) {
    return *(void**)((char*)&s->host_arg + f->off);
}

void upload_structs(RefSim* s) {
#ifdef HYDREF_CPU
    *s->arg = s->host_arg;
    *s->arr = s->host_arr;
#else
    ref_copy_in(s->arg, &s->host_arg, sizeof(Argument_Pointers));
    ref_copy_in(s->arr, &s->host_arr, sizeof(Array_Pointers));
#endif
}

inline unsigned cdiv(unsigned a, unsigned b) { return (a + b - 1) / b; }

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err ? g_msg : ""; }

int ref_is_gpu(void) {
#ifdef HYDREF_CPU
    return 0;
#else
    return 1;
#endif
}

void* ref_create(const HydCaseParams* p, int N, int M) {
    g_err = 0;
    RefSim* s = new RefSim();
    s->N = N;
    s->M = M;
    s->P = *p;
    s->t = 0;
    s->total_time = 0;
    s->last_ms = 0;
    s->nf = (size_t)(N + 3) * (M + 3);
    const size_t L = (size_t)(N > M ? N : M) + 3;
    const size_t W = (size_t)M + 3;
    /* padding: Interpolate_FS_d walks rows up to M (support_funcs.cu:219); Normalize may
       overrun a row by up to a block when M+3 > 1024 (Engine.py:63-64) */
    const size_t fguard = ((size_t)(M > N ? M - N : 0) + 8) * W * 8 + 8192 * 8;
    Argument_Pointers& a = s->host_arg;
    memset(&a, 0, sizeof a);
    a.M = M;
    a.N = N;
    for (const FieldRef& f : kFields) {
        const size_t n = kind_count(s, f.kind);
        void* ptr = ref_alloc(s, n * (f.is_int ? 4 : 8), f.kind == 0 ? fguard : 64 * 8 + 8 * L * 8);
        if (!ptr) {
            delete s;
            return nullptr;
        }
        *(void**)((char*)&a + f.off) = ptr;
    }
    a.bienQ = (int*)ref_alloc(s, 4 * sizeof(int), 64);
    a.boundary_type = (int*)ref_alloc(s, 4 * HYD_SEGMENT_LIMIT * sizeof(int), 64);
    /* Array_Pointers scratch; sized for the largest index any sweep or the smoothing
       buffer reaches (Pointers.py:47-81 allocates less for N != M) */
    size_t s2 = L * (2 * L + 1);
    if (s2 < s->nf) s2 = s->nf;
    const size_t sguard = (8 * L + 8192) * 8;
    double** sc1[] = {&s->host_arr.a1, &s->host_arr.b1, &s->host_arr.c1, &s->host_arr.d1,
                      &s->host_arr.a2, &s->host_arr.c2, &s->host_arr.d2, &s->host_arr.f1,
                      &s->host_arr.f2, &s->host_arr.f3, &s->host_arr.f5};
    for (double** q : sc1) *q = (double*)ref_alloc(s, L * L * 8, sguard);
    double** sc2[] = {&s->host_arr.AA, &s->host_arr.BB, &s->host_arr.CC, &s->host_arr.DD,
                      &s->host_arr.x,  &s->host_arr.Ap, &s->host_arr.Bp, &s->host_arr.ep};
    for (double** q : sc2) *q = (double*)ref_alloc(s, (s2 + 2 * L) * 8, sguard);
    s->host_arr.SN = (int*)ref_alloc(s, L * HYD_SEGMENT_LIMIT * 4, 64 * 4 + 8 * L * 4);
#ifdef HYDREF_CPU
    s->arg = new Argument_Pointers;
    s->arr = new Array_Pointers;
#else
    s->arg = (Argument_Pointers*)ref_alloc(s, sizeof(Argument_Pointers), 256);
    s->arr = (Array_Pointers*)ref_alloc(s, sizeof(Array_Pointers), 256);
#endif
    upload_structs(s);
    set_constants(s->P);
    if (g_err) return nullptr;
    return s;
}

void ref_destroy(void* h) {
    RefSim* s = (RefSim*)h;
    if (!s) return;
#ifdef HYDREF_CPU
    for (void* p : s->blocks) free(p);
    delete s->arg;
    delete s->arr;
#else
    for (void* p : s->blocks) cudaFree(p);
#endif
    delete s;
}

int ref_set_field(void* h, const char* name, const void* host, size_t count) {
    RefSim* s = (RefSim*)h;
    const FieldRef* f = find_field(name);
    if (!f || count != kind_count(s, f->kind)) return -1;
    ref_copy_in(member_ptr(s, f), host, count * (f->is_int ? 4 : 8));
    return g_err ? -2 : 0;
}

int ref_get_field(void* h, const char* name, void* host, size_t count) {
    RefSim* s = (RefSim*)h;
    const FieldRef* f = find_field(name);
    if (!f || count != kind_count(s, f->kind)) return -1;
#ifndef HYDREF_CPU
    SYNC();
#endif
    ref_copy_out(host, member_ptr(s, f), count * (f->is_int ? 4 : 8));
    return g_err ? -2 : 0;
}

int ref_set_boundary(void* h, const int* btype, const double* const* tables, const double* const* cc,
                     const int* nseg, int total_time) {
    RefSim* s = (RefSim*)h;
    if (total_time < 2) return -1;
    int bienQ[4];
    for (int e = 0; e < 4; e++) {
        bienQ[e] = 0;
        for (int k = 0; k < HYD_SEGMENT_LIMIT; k++)
            if (btype[e * HYD_SEGMENT_LIMIT + k] == 2) bienQ[e] = 1;
    }
    ref_copy_in(s->host_arg.bienQ, bienQ, sizeof bienQ);
    ref_copy_in(s->host_arg.boundary_type, btype, 4 * HYD_SEGMENT_LIMIT * sizeof(int));
    double** dst_bc[4] = {&s->host_arg.bc_up, &s->host_arg.bc_down, &s->host_arg.bc_left, &s->host_arg.bc_right};
    double** dst_cc[4] = {&s->host_arg.CC_u, &s->host_arg.CC_d, &s->host_arg.CC_l, &s->host_arg.CC_r};
    for (int e = 0; e < 4; e++) {
        const size_t n = (size_t)(nseg[e] > 0 ? nseg[e] : 1) * total_time + 2;
        *dst_bc[e] = (double*)ref_alloc(s, n * 8, 64 * 8);
        *dst_cc[e] = (double*)ref_alloc(s, n * 8, 64 * 8);
        if (!*dst_bc[e] || !*dst_cc[e]) return -3;
        if (nseg[e] > 0) {
            ref_copy_in(*dst_bc[e], tables[e], (size_t)nseg[e] * total_time * 8);
            ref_copy_in(*dst_cc[e], cc[e], (size_t)nseg[e] * total_time * 8);
        }
    }
    s->total_time = total_time;
    upload_structs(s);
    return g_err ? -2 : 0;
}

/* rep.py:126-139 */
int ref_init(void* h, double t_start) {
    RefSim* s = (RefSim*)h;
    const int N = s->N, M = s->M;
    Argument_Pointers* arg = s->arg;
    const dim3 b2((unsigned)(M + 3 < 32 ? M + 3 : 32), 1, 1);
    const dim3 g2((unsigned)((M + 3) / (M + 3 < 32 ? M + 3 : 32) + 1), (unsigned)(N + 3), 1);
    LAUNCH(Onetime_init, g2, b2, arg);
    SYNC();
    LAUNCH(Find_Calculation_limits_Horizontal, dim3(1, N, 1), RED32, arg);
    LAUNCH(Find_Calculation_limits_Vertical, dim3(1, M, 1), RED32, arg);
    LAUNCH(Htuongdoi, g2, b2, arg);
    SYNC();
    LAUNCH(preprocess_data, dim3(1, 1, 1), RED32, arg);
    SYNC();
    s->t = t_start;
    return g_err ? -2 : 0;
}

/* rep.py:126-131 with pick_up: Onetime_init, then the pick-up mask copied to the device
 * (load_intial_condition's toDevice), then the scans, Htuongdoi and preprocess_data. */
int ref_init_pickup(void* h, double t_start, const int* mask) {
    RefSim* s = (RefSim*)h;
    const int N = s->N, M = s->M;
    Argument_Pointers* arg = s->arg;
    const dim3 b2((unsigned)(M + 3 < 32 ? M + 3 : 32), 1, 1);
    const dim3 g2((unsigned)((M + 3) / (M + 3 < 32 ? M + 3 : 32) + 1), (unsigned)(N + 3), 1);
    LAUNCH(Onetime_init, g2, b2, arg);
    SYNC();
    ref_copy_in(s->host_arg.khouot, mask, sizeof(int) * (size_t)(N + 3) * (M + 3));
    LAUNCH(Find_Calculation_limits_Horizontal, dim3(1, N, 1), RED32, arg);
    LAUNCH(Find_Calculation_limits_Vertical, dim3(1, M, 1), RED32, arg);
    LAUNCH(Htuongdoi, g2, b2, arg);
    SYNC();
    LAUNCH(preprocess_data, dim3(1, 1, 1), RED32, arg);
    SYNC();
    s->t = t_start;
    return g_err ? -2 : 0;
}

/* Engine.py:144-366, nsteps iterations of the while loop */
int ref_step(void* h, int nsteps) {
    RefSim* s = (RefSim*)h;
    const int N = s->N, M = s->M;
    const unsigned M1 = (unsigned)M + 3, N1 = (unsigned)N + 3;
    Argument_Pointers* arg = s->arg;
    Array_Pointers* arr = s->arr;
    const Argument_Pointers& ha = s->host_arg;
    const HydCaseParams& P = s->P;
    const bool channel = P.kenhhepd || P.kenhhepng;
    const bool ketdinh = P.ketdinh != 0;
    const double bed_change_start = P.bed_change_start;
    const dim3 block_2d(M1 < 1024 ? M1 : 1024, 1, 1);
    const dim3 grid_2d(cdiv(M1, M1 < 1024 ? M1 : 1024), N1, 1);
    const int total_time = s->total_time;
#ifndef HYDREF_CPU
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
#endif
    auto boundary_at = [&](double t) {
        if (channel) {
            /* Engine.py:30-43; the kernels take bool* bienQ (support_funcs.cu:356) */
            const int m_offset = 5;
            bool* bq = (bool*)ha.bienQ;
            const unsigned bn = (unsigned)(N < 1024 ? N : 1024), bm = (unsigned)(M < 1024 ? M : 1024);
            LAUNCH(boundary_up, dim3(N / bn, 1, 1), dim3(bn, 1, 1), t, m_offset, M, N, bq, ha.t_z, ha.daui, ha.cuoii, ha.dauj, ha.cuoij, ha.vbt, ha.vbd, ha.ubt, ha.ubp);
            LAUNCH(boundary_down, dim3(N / bn, 1, 1), dim3(bn, 1, 1), t, m_offset, M, N, bq, ha.t_z, ha.daui, ha.cuoii, ha.dauj, ha.cuoij, ha.vbt, ha.vbd, ha.ubt, ha.ubp);
            LAUNCH(boundary_left, dim3(M / bm, 1, 1), dim3(bm, 1, 1), t, m_offset, M, N, bq, ha.t_z, ha.daui, ha.cuoii, ha.dauj, ha.cuoij, ha.vbt, ha.vbd, ha.ubt, ha.ubp);
            LAUNCH(boundary_right, dim3(M / bm, 1, 1), dim3(bm, 1, 1), t, m_offset, M, N, bq, ha.t_z, ha.daui, ha.cuoii, ha.dauj, ha.cuoij, ha.vbt, ha.vbd, ha.ubt, ha.ubp);
            SYNC();
        } else {
            LAUNCH(Update_Boundary_Value, dim3(1, (unsigned)((M > N ? M : N) / 1024 + 1), 1), dim3(1, 1024, 1), t, total_time, arg);
        }
    };
    double t = s->t;
    for (int step = 0; step < nsteps; step++) {
        t = t + P.dT * 0.5;
        boundary_at(t);
        SYNC();
        int start_idx = 2, end_idx = M;
        bool isU = true;
        int jump_step = 2;
        if (channel && P.kenhhepd == 1) {
            start_idx = 3;
            end_idx = M - 1;
        }
        dim3 block_size(1, 1024, 1);
        dim3 grid_size(M1, cdiv((unsigned)N, 1024), 1);
        LAUNCH(UZSolver_calculate_preindex, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(UZSolver_calculate_abcd, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(UZSolver_calculate_matrix_coeff, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(tridiagSolver, dim3(1, M - 1, 1), RED32, false, isU, start_idx, end_idx, jump_step, 2 * N + 1, arg, arr);
        SYNC();
        LAUNCH(UZSolver_extract_solution, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(Normalize, grid_2d, block_2d, 1.0, arg, arr);
        SYNC();
        LAUNCH(update_buffer, grid_2d, block_2d, true, arg, arr);
        SYNC();
        LAUNCH(solveV, grid_2d, block_2d, t, 2, N, arg);
        SYNC();
        LAUNCH(update_margin_elem_V, dim3(1, N, 1), RED32, t, 2, N, arg);
        LAUNCH(Normalize, grid_2d, block_2d, 0.0, arg, arr);
        SYNC();
        LAUNCH(update_buffer, grid_2d, block_2d, false, arg, arr);
        SYNC();
        LAUNCH(update_h_moi, grid_2d, block_2d, arg);
        SYNC();
        LAUNCH(Reset_states_horizontal, dim3(1, N, 1), RED32, arg);
        SYNC();
        LAUNCH(update_uvz, grid_2d, block_2d, M, N, ha.u, ha.v, ha.z, ha.t_u, ha.t_v, ha.t_z, (DOUBLE*)nullptr, (DOUBLE*)nullptr, 0, 0);
        SYNC();
        LAUNCH(Find_Calculation_limits_Horizontal, dim3(1, N, 1), RED32, arg);
        LAUNCH(Find_Calculation_limits_Vertical, dim3(1, M, 1), RED32, arg);
        LAUNCH(Htuongdoi, grid_2d, block_2d, arg);
        SYNC();
        if (t >= P.sediment_start) {
            LAUNCH(Find_VTH, grid_2d, block_2d, arg);
            LAUNCH(hesoK, grid_2d, block_2d, arg);
            SYNC();
            start_idx = 3;
            end_idx = M - 1;
            LAUNCH(Scan_FSj, grid_size, block_size, t, bed_change_start, ketdinh, start_idx, end_idx, arg, arr);
            SYNC();
            jump_step = 1;
            LAUNCH(tridiagSolver, dim3(1, M - 1, 1), RED32, true, isU, start_idx, end_idx, jump_step, N + 3, arg, arr);
            SYNC();
            LAUNCH(FSj_extract_solution, grid_size, block_size, ketdinh, start_idx, end_idx, arg, arr);
            SYNC();
            LAUNCH(Update_FS, grid_2d, block_2d, arg);
        }
        /* ---- second half-step ---- */
        t = t + P.dT * 0.5;
        boundary_at(t);
        SYNC();
        block_size = dim3(1024, 1, 1);
        grid_size = dim3(cdiv((unsigned)M, 1024), (unsigned)N, 1);
        start_idx = 2;
        end_idx = N;
        jump_step = 2;
        isU = false;
        if (channel && P.kenhhepng == 1) {
            start_idx = 3;
            end_idx = N;
        }
        LAUNCH(VZSolver_calculate_preindex, grid_size, block_size, t, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(VZSolver_calculate_abcd, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(VZSolver_calculate_matrix_coeff, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(tridiagSolver, dim3(1, N - 1, 1), RED32, false, isU, start_idx, end_idx, jump_step, 2 * M + 1, arg, arr);
        SYNC();
        LAUNCH(VZSolver_extract_solution, grid_size, block_size, start_idx, end_idx, arg, arr);
        SYNC();
        LAUNCH(Normalize, grid_2d, block_2d, 0.0, arg, arr);
        SYNC();
        LAUNCH(update_buffer, grid_2d, block_2d, false, arg, arr);
        SYNC();
        LAUNCH(solveU, grid_2d, block_2d, t, 2, M, arg);
        SYNC();
        LAUNCH(update_margin_elem_U, dim3(1, M, 1), RED32, 2, M, arg);
        SYNC();
        LAUNCH(Normalize, grid_2d, block_2d, 1.0, arg, arr);
        SYNC();
        LAUNCH(update_buffer, grid_2d, block_2d, true, arg, arr);
        SYNC();
        LAUNCH(update_h_moi, grid_2d, block_2d, arg);
        SYNC();
        LAUNCH(Reset_states_vertical, dim3(M, 1, 1), RED32Y, arg);
        SYNC();
        LAUNCH(update_uvz, grid_2d, block_2d, M, N, ha.u, ha.v, ha.z, ha.t_u, ha.t_v, ha.t_z, (DOUBLE*)nullptr, (DOUBLE*)nullptr, 0, 0);
        SYNC();
        LAUNCH(Find_Calculation_limits_Horizontal, dim3(1, N, 1), RED32, arg);
        LAUNCH(Find_Calculation_limits_Vertical, dim3(1, M, 1), RED32, arg);
        SYNC();
        LAUNCH(Htuongdoi, grid_2d, block_2d, arg);
        SYNC();
        if (t >= P.sediment_start) {
            LAUNCH(Find_VTH, grid_2d, block_2d, arg);
            LAUNCH(hesoK, grid_2d, block_2d, arg);
            SYNC();
            start_idx = 3;
            end_idx = N - 1;
            LAUNCH(Scan_FSi, grid_size, block_size, t, bed_change_start, ketdinh, start_idx, end_idx, arg, arr);
            SYNC();
            jump_step = 1;
            LAUNCH(tridiagSolver, dim3(1, N - 3, 1), RED32, true, isU, start_idx, end_idx, jump_step, M + 3, arg, arr);
            SYNC();
            LAUNCH(FSi_extract_solution, grid_size, block_size, ketdinh, start_idx, end_idx, arg, arr);
            SYNC();
            LAUNCH(Update_FS, grid_2d, block_2d, arg);
            SYNC();
        }
        {
            const double it = (double)(long long)t;
            if (fmod(it, bed_change_start) == 0 && t - it == 0) {
                LAUNCH(Calculate_Qb, grid_2d, block_2d, ketdinh, arg, arr);
                LAUNCH(BedLoad, grid_2d, block_2d, t, ketdinh, start_idx, end_idx, arg, arr);
            }
        }
        if (g_err) break;
    }
#ifndef HYDREF_CPU
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    s->last_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
#endif
    s->t = t;
    return g_err ? -2 : 0;
}

double ref_time(void* h) { return ((RefSim*)h)->t; }
double ref_last_ms(void* h) { return ((RefSim*)h)->last_ms; }

}  // extern "C"
