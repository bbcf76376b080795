// k_grid.cu — the non-implicit parts of the ADI step: boundary values, smoothing,
// explicit momentum, wet/dry resets, state update, face depths, wet-segment scans,
// edge concentration interpolation, sediment coefficients and the Exner update.
//
// Each kernel restates one or more reference kernels (file:line beside it).  Kernels
// the reference runs as one thread (or 32 identical threads) per line with a serial
// loop are mapped to one CTA or warp per line; where the loop carries a dependence
// (the wet/dry opening cascade) only the iterations that can act run serially.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <type_traits>

#include "hydist_dev.cuh"

namespace {

constexpr double kPiRef = 3.14159265359;  // constant.cuh:3
constexpr double kEpsRef = 1e-16;         // UVZSolver_multithread.cu:12
constexpr int kSpanHalo = 4;              // extended-span margin, cells
constexpr double kBedLimit = 0.1;         // fed-back bed change per update: at most this fraction of the depth
constexpr double kBedCap = 0.05;          // and at most this many metres

inline dim3 grid2d(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y); }

// ---------------------------------------------------------------- one-time set-up

// Onetime_init (support_funcs.cu:20-58)
__global__ void k_onetime_init(DevGrid g, DevParams p) {
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = blockIdx.y * blockDim.y + threadIdx.y;
    const int N = g.N, M = g.M, P = g.P;
    if (i0 >= N + 3 || j0 >= M + 3) return;
    g.khouot[i0 * P] = 2;
    g.khouot[j0] = 2;
    const int i = i0 + 1, j = j0 + 1;
    if (i <= N + 2 && j <= M + 2) g.khouot[i * P + j] = 2;
    if (i > N + 1 || j > M + 1) return;
    const double* h = g.h;
    if ((h[(i - 1) * P + j - 1] + h[(i - 1) * P + j] + h[i * P + j - 1] + h[i * P + j]) * 0.25 > p.NANGDAY) {
        g.khouot[i * P + j] = 0;
        g.H_moi[i * P + j] = 0;
    }
    if (i > N || j > M) return;
    const double ht = (h[(i - 1) * P + j - 1] + h[(i - 1) * P + j] + h[i * P + j - 1] + h[i * P + j]) * 0.25;
    g.htaiz[i * P + j] = ht;
    g.htaiz_bd[i * P + j] = ht;
    if (h[i * P + j - 1] + h[i * P + j] != 0)
        g.Kx1[i * P + j] = p.g * pow((h[i * P + j - 1] + h[i * P + j]) * 0.5, -2 * p.mu_mn) *
                           pow((g.hsnham[i * P + j - 1] + g.hsnham[i * P + j]) * 0.5, 2);
    if (h[(i - 1) * P + j] + h[i * P + j] != 0)
        g.Ky1[i * P + j] = p.g * pow((h[(i - 1) * P + j] + h[i * P + j]) * 0.5, -2 * p.mu_mn) *
                           pow((g.hsnham[(i - 1) * P + j] + g.hsnham[i * P + j]) * 0.5, 2);
}

// preprocess_data (support_funcs.cu:433-542): discharge-edge conveyance weights hi and
// the edge concentration scales hmax.  One thread; runs once.
__global__ void k_preprocess(DevGrid g, DevParams p) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int N = g.N, M = g.M, P = g.P;
    const double* h = g.h;
    double* hi = g.hi;
    for (int k = 0; k < g.mocj[M]; k++) {
        double sum = 0;
        for (int i = g.dauj[M * HYD_SEGL + k]; i <= g.cuoij[M * HYD_SEGL + k]; i++) {
            hi[i] = (h[i * P + M] + h[(i - 1) * P + M]) / 2.0 - p.NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = g.dauj[M * HYD_SEGL + k]; i <= g.cuoij[M * HYD_SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * p.dX);
    }
    hi += N + 3;
    for (int k = 0; k < g.mocj[2]; k++) {
        double sum = 0;
        for (int i = g.dauj[2 * HYD_SEGL + k]; i <= g.cuoij[2 * HYD_SEGL + k]; i++) {
            hi[i] = (h[i * P + 1] + h[(i - 1) * P + 1]) / 2.0 - p.NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = g.dauj[2 * HYD_SEGL + k]; i <= g.cuoij[2 * HYD_SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * p.dX);
    }
    hi += N + 3;
    for (int k = 0; k < g.moci[2]; k++) {
        double sum = 0;
        for (int i = g.daui[2 * HYD_SEGL + k]; i <= g.cuoii[2 * HYD_SEGL + k]; i++) {
            hi[i] = (h[1 * P + i] + h[1 * P + i - 1]) / 2.0 - p.NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = g.daui[2 * HYD_SEGL + k]; i <= g.cuoii[2 * HYD_SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * p.dX);
    }
    hi += M + 3;
    for (int k = 0; k < g.moci[N]; k++) {
        double sum = 0;
        for (int i = g.daui[N * HYD_SEGL + k]; i <= g.cuoii[N * HYD_SEGL + k]; i++) {
            hi[i] = (h[N * P + i] + h[N * P + i - 1]) / 2.0 - p.NANGDAY;
            sum += pow(hi[i], 5.0 / 3.0);
        }
        for (int i = g.daui[N * HYD_SEGL + k]; i <= g.cuoii[N * HYD_SEGL + k]; i++)
            hi[i] = pow(hi[i], 2.0 / 3.0) / (sum * p.dX);
    }
    const double* hb = g.htaiz_bd;
    double hu = hb[2 * P + M], hd = hb[2 * P + 2];
    for (int i = 3; i < N; i++) {
        if (hb[i * P + M] > hu) hu = hb[i * P + M];
        if (hb[i * P + 2] > hd) hd = hb[i * P + 2];
    }
    double hl = hb[2 * P + 2], hr = hb[N * P + 2];
    for (int i = 3; i < M; i++) {
        if (hb[2 * P + i] > hl) hl = hb[2 * P + i];
        if (hb[N * P + i] > hr) hr = hb[N * P + i];
    }
    if (hu != 0) hu = 1.0 / (p.ros * hu);
    if (hd != 0) hd = 1.0 / (p.ros * hd);
    if (hl != 0) hl = 1.0 / (p.ros * hl);
    if (hr != 0) hr = 1.0 / (p.ros * hr);
    g.hmax[0] = hu;
    g.hmax[1] = hd;
    g.hmax[2] = hl;
    g.hmax[3] = hr;
}

// ------------------------------------------------------------------ step clock

// Advances the device copy of the simulation time by one full step exactly as the host
// loop does (Engine.py:146,260: t = t + dT * 0.5, twice), so that a captured step can be
// replayed without baking the time into kernel arguments.

// --------------------------------------------------------------- boundary values

// Boundary_value + FS_boundary for one edge at index i (support_funcs.cu:544-617), split
// into the computation (BndRec) and the writes it makes (bnd_apply).
struct BndRec {
    int kind;  // 0 nothing, 1 discharge edge (velocity table + FS), 2 level edge (two levels)
    double value, fsv;
};

struct EdgeArgs {
    int isU, location, location_ext;
    const int* btype;
    const double *hi_e, *bcv, *ccv;
    double* barr;
    double hmax;
    const int *moc, *dau, *cuoi;
};

// Edges in the order up (column M), down (column 2), left (row 2), right (row N).
__device__ __forceinline__ EdgeArgs edge_args(const DevGrid& g, int e) {
    const int N = g.N, M = g.M;
    const double* hi_up = g.hi;
    const double* hi_down = hi_up + (N + 3);
    const double* hi_left = hi_down + (N + 3);
    const double* hi_right = hi_left + (M + 3);
    if (e == 0) return {0, M, M + 1, g.btype + 0 * HYD_SEGL, hi_up, g.bc[0], g.cc[0], g.vbt, g.hmax[0], g.mocj, g.dauj, g.cuoij};
    if (e == 1) return {0, 2, 1, g.btype + 1 * HYD_SEGL, hi_down, g.bc[1], g.cc[1], g.vbd, g.hmax[1], g.mocj, g.dauj, g.cuoij};
    if (e == 2) return {1, 2, 1, g.btype + 2 * HYD_SEGL, hi_left, g.bc[2], g.cc[2], g.ubt, g.hmax[2], g.moci, g.daui, g.cuoii};
    return {1, N, N + 1, g.btype + 3 * HYD_SEGL, hi_right, g.bc[3], g.cc[3], g.ubp, g.hmax[3], g.moci, g.daui, g.cuoii};
}

// What an edge applies at time t, the same for every index of the edge: the open segment
// (the edge line's first wet segment, [lo, hi]; empty when the line has none), its kind
// and the table values interpolated at t.
struct BndSeg {
    int lo, hi, kind;
    double value, cv;
};

__device__ __forceinline__ BndSeg bnd_segment(const DevGrid& g, const EdgeArgs& a, double t) {
    BndSeg s{1, 0, 0, 0.0, 0.0};
    if (a.moc[a.location] <= 0) return s;
    const int tt = g.total_time;
    const int t1 = (int)(t / 3600);
    const double t2 = (t - (3600.0 * t1)) / 3600.0;
    const int seg_no = 0;
    s.lo = a.dau[a.location * HYD_SEGL];
    s.hi = a.cuoi[a.location * HYD_SEGL];
    s.value = a.bcv[seg_no * tt + t1] * (1.0 - t2) + a.bcv[seg_no * tt + t1 + 1] * t2;
    if (a.btype[seg_no] == 2) {
        s.kind = 1;
        s.cv = a.ccv[seg_no * tt + t1] * (1.0 - t2) + a.ccv[seg_no * tt + t1 + 1] * t2;
    } else {
        s.kind = 2;
    }
    return s;
}

// The record of index i of the edge (the body of Boundary_value / FS_boundary for one
// thread, support_funcs.cu:544-617).
__device__ __forceinline__ BndRec bnd_at(const DevGrid& g, const EdgeArgs& a, const BndSeg& s, int i) {
    BndRec r{0, 0.0, 0.0};
    if (i < s.lo || i > s.hi) return r;
    r.kind = s.kind;
    if (s.kind == 1) {
        r.value = s.value * a.hi_e[i];
        const int ii = a.isU ? a.location : i, jj = a.isU ? i : a.location;
        r.fsv = s.cv * g.htaiz_bd[ii * g.P + jj] * a.hmax;
    } else {
        r.value = s.value;
    }
    return r;
}

// writes: kBndHydro (discharge-edge velocities, stage-edge levels), kBndFS (inflow
// concentrations), or both.
constexpr int kBndHydro = 1, kBndFS = 2, kBndAll = 3;

__device__ void bnd_apply(const DevGrid& g, const EdgeArgs& a, const BndRec& r, int i, int writes) {
    const int P = g.P;
    if (r.kind == 1) {
        if (writes & kBndHydro) a.barr[i] = r.value;
        const int ii = a.isU ? a.location : i, jj = a.isU ? i : a.location;
        if (writes & kBndFS) g.FS[ii * P + jj] = r.fsv;
    } else if (r.kind == 2 && (writes & kBndHydro)) {
        if (a.isU) {
            g.t_z[a.location * P + i] = r.value;
            g.t_z[a.location_ext * P + i] = r.value;
        } else {
            g.t_z[i * P + a.location] = r.value;
            g.t_z[i * P + a.location_ext] = r.value;
        }
    }
}

// Update_Boundary_Value (support_funcs.cu:622-668).  The reference applies the edges in
// the order up, down, left, right (the order a converged warp applies them); two edges
// only meet at the corner indices (2 and N of the up/down edges, 2 and M of left/right).
// Here the four edges run at once, each in a quarter of the CTA (blockDim a multiple of
// 128), holding back their corner writes; thread 0 then applies those in the reference's
// order, and again the (N, 2) write of the down edge and, when N > M, the (N, M) write of
// the up edge, which threads past the first warp repeat in the reference.  `writes`
// selects the arrays written (the same order applies within each array), so the
// concentration part can run after work that the velocity/level part need not wait for.
__device__ void boundary_body(const DevGrid& g, double t, int writes = kBndAll) {
    __shared__ BndRec s_rec[4][2];
    const int N = g.N, M = g.M;
    const int imax = N > M ? N : M;
    const int Q = blockDim.x / 4, e = threadIdx.x / Q, r = threadIdx.x % Q;
    if (e < 4) {
        const EdgeArgs a = edge_args(g, e);
        const int far = a.isU ? M : N;
        const BndSeg sg = bnd_segment(g, a, t);
        // four indices at a time: their loads issue before any of their stores
        constexpr int U = 4;
        for (int i0 = 2 + r; i0 <= imax; i0 += U * Q) {
            BndRec rec[U];
#pragma unroll
            for (int u = 0; u < U; u++) rec[u] = bnd_at(g, a, sg, i0 + u * Q);
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 + u * Q;
                if (i > imax) break;
                if (i == 2) s_rec[e][0] = rec[u];
                else if (i == far) s_rec[e][1] = rec[u];
                else bnd_apply(g, a, rec[u], i, writes);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; k++) {
            const EdgeArgs a = edge_args(g, k);
            bnd_apply(g, a, s_rec[k][0], 2, writes);
            bnd_apply(g, a, s_rec[k][1], a.isU ? M : N, writes);
        }
        bnd_apply(g, edge_args(g, 1), s_rec[1][1], N, writes);
        if (N > M) bnd_apply(g, edge_args(g, 0), s_rec[0][1], N, writes);
    }
}


// Channel-mode analytic seiche boundaries (support_funcs.cu:356-429, Engine.py:30-43).
// Engine.py passes m_offset = 5 as the kernels' segment_limit parameter, so the segment
// tables are read with a stride of 5; bienQ is read through a bool pointer, i.e. byte e
// of the int32 array.  Each edge covers at most N (up/down) or M (left/right) indices,
// the extent of the reference's launch.
__device__ void boundary_channel_body(const DevGrid& g, const DevParams& p, double t) {
    const int N = g.N, M = g.M, P = g.P;
    const int sl = 5;
    const unsigned char* bq = (const unsigned char*)g.bienQ;
    for (int e = 0; e < 4; e++) {
        int lo, hi;
        if (e == 0) { lo = g.dauj[M * sl]; hi = g.cuoij[M * sl]; }
        else if (e == 1) { lo = g.dauj[2 * sl]; hi = g.cuoij[2 * sl]; }
        else if (e == 2) { lo = g.daui[2 * sl]; hi = g.cuoii[2 * sl]; }
        else { lo = g.daui[2 * sl]; hi = g.cuoii[N * sl]; }
        const int span = e < 2 ? N : M;
        if (hi > lo + span - 1) hi = lo + span - 1;
        // the indices address rows/columns 0..N+2 / 0..M+2 only
        const int cap = e < 2 ? N + 2 : M + 2;
        if (hi > cap) hi = cap;
        for (int i = lo + threadIdx.x; i <= hi; i += blockDim.x) {
            if (e == 0) {
                g.t_z[i * P + M] = 0.01 * cos(2 * kPiRef / 27.750 * t) * cos(2 * (kPiRef / 100) * (100 - p.dY / 2));
                g.t_z[i * P + M + 1] = 0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * (100 + p.dY / 2));
            } else if (e == 1) {
                if (bq[1]) g.vbd[i] = 0;
                else {
                    g.t_z[i * P + 2] = 0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * p.dY / 2);
                    g.t_z[i * P + 1] = 0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * (-p.dY) / 2);
                }
            } else if (e == 2) {
                if (bq[2]) g.ubt[i] = 0;
                else {
                    g.t_z[2 * P + i] = 0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * p.dX / 2);
                    g.t_z[1 * P + i] = 0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * (-p.dX) / 2);
                }
            } else {
                if (bq[3]) g.ubp[i] = 0;
                else {
                    g.t_z[N * P + i] = 0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * (100 - p.dX / 2));
                    g.t_z[(N + 1) * P + i] =
                        0.01 * cos(2 * kPiRef / 27.75 * t) * cos(2 * (kPiRef / 100) * (100 + p.dX / 2));
                }
            }
        }
        __syncthreads();
    }
}


// The coefficient kernels below and the explicit momentum are templates on the arithmetic
// type R: double for the FP64 form (the reference's operation order term by term), float for
// the mixed form.  Every operand is read in FP64 and taken to R at its use; water-level
// differences are taken in FP64 first (z is a datum plus small changes); the wet/dry tests
// compare the stored FP64 depths, so both forms take the same branches.

// Continuity and momentum coefficients of one wet cell of a UZ line (column j, cell i):
// a2, c2, d2 (_uzSolver_calculate_preindex, UVZSolver_multithread.cu:402-406) and f1, f2,
// f3, f5 (352-400).  Cell-local, so they are computed for every wet cell by a row-major
// kernel and stored column-major for the column sweep.  Mixed form (R = float): the rows
// of the level increment z' - z, i.e. d2 - z and f5 - f4 (z_i - z_i+1), f4 = 2 g dT / 2dX.
template <class R>
__device__ __forceinline__ void uz_cell_coeffs(const DevGrid& g, const DevParams& p, int pos, R& a2, R& c2, R& d2,
                                               R& f1, R& f2, R& f3, R& f5) {
    constexpr bool MIX = sizeof(R) == sizeof(float);
    const int P = g.P;
    auto L = [](const double* a, int q) { return R(a[q]); };
    const R dTx = R(p.dTchia2dX), dTy = R(p.dTchia2dY), dT = R(p.dT), dXbp = R(p.dXbp), dY2 = R(p.dY2),
            dYbp = R(p.dYbp);
    c2 = dTx * L(g.Htdu, pos);
    a2 = -dTx * L(g.Htdu, pos - P);
    const R ydiv = dTy * (L(g.Htdv, pos) * L(g.v, pos) - L(g.Htdv, pos - 1) * L(g.v, pos - 1));
    d2 = MIX ? -ydiv : R(g.z[pos]) - ydiv;
    R pp = 0.0, qq = 0.0;
    const double* u = g.u;
    const double* H = g.H_moi;
    const R u0 = L(u, pos);
    const R vtb = (L(g.v, pos - 1) + L(g.v, pos) + L(g.v, pos + P - 1) + L(g.v, pos + P)) * R(0.25);
    f1 = dTx * u0 + L(g.VISC, pos) * dT / dXbp;
    f2 = -(2 + L(g.Kx1, pos) * dT * sqrt(u0 * u0 + vtb * vtb) / L(g.Htdu, pos) + (2 * dT * L(g.VISC, pos)) / dXbp);
    f3 = dT * L(g.VISC, pos) / dXbp - dTx * u0;
    // the neighbours the branches below take, loaded before the depth tests that choose
    // among them (one memory round trip; interior cells have two cells either side)
    const R um1 = L(u, pos - 1), up1 = L(u, pos + 1), um2 = L(u, pos - 2), up2 = L(u, pos + 2);
    const double Hm1 = H[pos - 1], Hp1 = H[pos + 1], Hm2 = H[pos - 2];
    if (Hm1 <= p.H_TINH) {
        if (vtb < 0) {
            pp = vtb * (-3 * u0 + 4 * up1 - up2) / dY2;
            qq = (u0 - 2 * up1 + up2) / dYbp;
        }
    } else {
        if (Hp1 <= p.H_TINH) {
            if ((Hm2 > p.H_TINH) && (vtb > 0)) {
                pp = vtb * (3 * u0 - 4 * um1 + um2) / dY2;
                qq = (u0 - 2 * um1 + um2) / dYbp;
            }
        } else {
            pp = vtb * (up1 - um1) / dY2;
            qq = (up1 - 2 * u0 + um1) / dYbp;
        }
    }
    f5 = -2 * u0 + dT * pp - dT * R(p.CORIOLIS_FORCE) * vtb - dT * L(g.VISC, pos) * qq -
         dT * (R(p.windx) - L(g.Tsxw, pos)) / L(g.Htdu, pos);
    if (MIX) f5 -= R(2 * p.g * p.dTchia2dX) * R(g.z[pos] - g.z[pos + P]);
}

// Momentum and continuity coefficients of a VZ cell (preindex, _calculate_abcd:
// UVZSolver_multithread.cu:345-349, 409-466 for the v direction): the terms the VZ sweep
// combines into its rows, precomputed row-major so that the sweep's row building is loads.
// Mixed form as uz_cell_coeffs, with f4 = 2 g dT / 2dY and z_j+1.
template <class R>
__device__ __forceinline__ void vz_cell_coeffs(const DevGrid& g, const DevParams& p, int pos, R& a2, R& c2, R& d2,
                                               R& f1, R& f2, R& f3, R& f5) {
    constexpr bool MIX = sizeof(R) == sizeof(float);
    const int P = g.P;
    auto L = [](const double* a, int q) { return R(a[q]); };
    const R dTx = R(p.dTchia2dX), dTy = R(p.dTchia2dY), dT = R(p.dT), dX2 = R(p.dX2), dXbp = R(p.dXbp),
            dYbp = R(p.dYbp);
    c2 = dTy * L(g.Htdv, pos);
    a2 = -dTy * L(g.Htdv, pos - 1);
    const R xdiv = dTx * (L(g.Htdu, pos) * L(g.u, pos) - L(g.Htdu, pos - P) * L(g.u, pos - P));
    d2 = MIX ? -xdiv : R(g.z[pos]) - xdiv;
    const double* v = g.v;
    const double* H = g.H_moi;
    R pp = 0.0, qq = 0.0;
    const R v0 = L(v, pos);
    const R utb = (L(g.u, pos - P) + L(g.u, pos) + L(g.u, pos - P + 1) + L(g.u, pos + 1)) * R(0.25);
    f1 = dTy * v0 + L(g.VISC, pos) * dT / dYbp;
    f2 = -(2 + L(g.Ky1, pos) * dT * sqrt(v0 * v0 + utb * utb) / L(g.Htdv, pos) + (2 * dT * L(g.VISC, pos)) / dYbp);
    f3 = dT * L(g.VISC, pos) / dYbp - dTy * v0;
    // as in uz_cell_coeffs: the branches' neighbours loaded first
    const R vm1 = L(v, pos - P), vp1 = L(v, pos + P), vm2 = L(v, pos - 2 * P), vp2 = L(v, pos + 2 * P);
    const double Hm1 = H[pos - P], Hp1 = H[pos + P], Hm2 = H[pos - 2 * P];
    if (Hm1 <= p.H_TINH) {
        if (utb < 0) {
            qq = utb * (-3 * v0 + 4 * vp1 - vp2) / dX2;
            pp = (v0 - 2 * vp1 + vp2) / dXbp;
        }
    } else {
        if (Hp1 <= p.H_TINH) {
            if ((Hm2 > p.H_TINH) && (utb > 0)) {
                qq = utb * (3 * v0 - 4 * vm1 + vm2) / dX2;
                pp = (v0 - 2 * vm1 + vm2) / dXbp;
            }
        } else {
            qq = utb * (vp1 - vm1) / dX2;
            pp = (vp1 - 2 * v0 + vm1) / dXbp;
        }
    }
    f5 = -2 * v0 + dT * qq + dT * R(p.CORIOLIS_FORCE) * utb - dT * L(g.VISC, pos) * pp -
         dT * (R(p.windy) - L(g.Tsyw, pos)) / L(g.Htdv, pos);
    if (MIX) f5 -= R(2 * p.g * p.dTchia2dY) * R(g.z[pos] - g.z[pos + 1]);
}

// The first launch of each half-step.  KIND 0 (half-step 1): UZ coefficients of every wet
// interior cell written column-major (g.colT arrays 0..6: a2 c2 d2 f1 f2 f3 f5), and in
// the last CTA the clock advance and the boundary values of the half-step.  KIND 1
// (half-step 2): VZ coefficients written row-major (g.rowC arrays 0..6), and in the last
// CTA the half-step's boundary values (`writes`).  The coefficients read none of what the
// boundary writes (edge levels, edge velocity arrays, inflow concentrations).  One warp
// per row of the grid over the row's span of cells that can be wet; small CTAs, so that
// the stores spread over many SMs; TILE (large grids, g.tile_cols) stores KIND 0 through a
// shared-memory tile (colmajor_tile), 8 rows of a column at a time.  The variants are
// separate kernels: the tile's shared memory would otherwise shrink the L1 share of the
// small grids' launches, whose stencil loads it serves.
// bx, gx: the CTA's index among the launch's CTAs of this grid and their count (blockIdx.x
// and gridDim.x of a launch for one grid; a member's share of a batched launch).
template <int KIND, int TILE, class R>
__device__ __forceinline__ void coef_bnd_body(const DevGrid& g, const DevParams& p, int writes, int bx, int gx) {
    // CTA 0 takes the clock and the boundary (a chain of dependent loads, started first
    // so that it runs beside the coefficient CTAs instead of after them); the others the
    // coefficients
    if (bx == 0) {
        __shared__ double s_t;
        if (threadIdx.x == 0) {
            if (KIND == 0) {  // k_clock
                const double t1 = g.clock[2] + p.dT * 0.5;
                const double t2 = t1 + p.dT * 0.5;
                g.clock[0] = t1;
                g.clock[1] = t2;
                g.clock[2] = t2;
                s_t = t1;
            } else {
                s_t = g.clock[1];
            }
        }
        __syncthreads();
        if (p.channel) boundary_channel_body(g, p, s_t);
        else boundary_body(g, s_t, writes);
        return;
    }
    bx -= 1;
    if constexpr (KIND == 0 && TILE) {
        R* const dst[7] = {colTr<R>(g, 0), colTr<R>(g, 1), colTr<R>(g, 2), colTr<R>(g, 3),
                           colTr<R>(g, 4), colTr<R>(g, 5), colTr<R>(g, 6)};
        colmajor_tile<7>(
            g, 2 + kTileRows * bx, g.N, 2, g.M,
            [&](int i, int j, R* v) {
                const int pos = i * g.P + j;
                if (g.khouot[pos] != 0) return false;
                uz_cell_coeffs<R>(g, p, pos, v[0], v[1], v[2], v[3], v[4], v[5], v[6]);
                return true;
            },
            dst);
        return;
    }
    // rows 2..N, one warp per row (several warps per row measured slower on config 4:
    // 46 -> 50 us), lanes striding over the row's cells
    const int i = 2 + ((bx * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i > g.N) return;
    const int lo = max(g.rlo[i], 2), hi = min(g.rhi[i], g.M);
    for (int j = lo + lane; j <= hi; j += 32) {
        const int pos = i * g.P + j;
        if (g.khouot[pos] != 0) continue;
        R a2, c2, d2, f1, f2, f3, f5;
        if (KIND == 0) {
            uz_cell_coeffs<R>(g, p, pos, a2, c2, d2, f1, f2, f3, f5);
            const size_t t = (size_t)j * g.LT + i;
            colTr<R>(g, 0)[t] = a2;
            colTr<R>(g, 1)[t] = c2;
            colTr<R>(g, 2)[t] = d2;
            colTr<R>(g, 3)[t] = f1;
            colTr<R>(g, 4)[t] = f2;
            colTr<R>(g, 5)[t] = f3;
            colTr<R>(g, 6)[t] = f5;
        } else {
            vz_cell_coeffs<R>(g, p, pos, a2, c2, d2, f1, f2, f3, f5);
            rowCr<R>(g, 0)[pos] = a2;
            rowCr<R>(g, 1)[pos] = c2;
            rowCr<R>(g, 2)[pos] = d2;
            rowCr<R>(g, 3)[pos] = f1;
            rowCr<R>(g, 4)[pos] = f2;
            rowCr<R>(g, 5)[pos] = f3;
            rowCr<R>(g, 6)[pos] = f5;
        }
    }
}

template <int KIND, int TILE, class R>
__global__ void __launch_bounds__(256) k_coef_bnd(DevGrid g, DevParams p, int writes) {
    coef_bnd_body<KIND, TILE, R>(g, p, writes, blockIdx.x, gridDim.x);
}
template <int KIND, int TILE, class R>
__global__ void __launch_bounds__(256) k_coef_bnd_b(BatchRef br, int writes) {
    const BatchMember bm(br);
    coef_bnd_body<KIND, TILE, R>(bm.g, bm.p, writes, bm.bx, bm.gx);
}

// ------------------------------------------------------------------- smoothing

// Normalize + update_buffer (support_funcs.cu:682-729): out = 5-point smoothed velocity on
// the interior, a copy elsewhere.  isU smooths t_u (neighbours along i, wet check along j).
// A nonzero velocity outside the row's extended span is reported in *g.span_wide (the
// spans then cannot bound the smoothing).
__device__ __forceinline__ void smooth_cell(const DevGrid& g, const DevParams& p, int isU, double* __restrict__ out,
                                            int i, int j, bool check_span) {
    const int N = g.N, M = g.M, P = g.P;
    if (i >= N + 3 || j >= M + 3) return;
    const double* val = isU ? g.t_u : g.t_v;
    const int gp = i * P + j;
    const bool inner = !(i > N || j > M || i < 2 || j < 2);
    const int close_d = isU ? P : 1, far_d = isU ? 1 : P;
    // every load first (one memory round trip): the cell, its four neighbours and the
    // mask of the two across the smoothing direction
    const double v0 = val[gp];
    double vcm = 0.0, vcp = 0.0, vfm = 0.0, vfp = 0.0;
    int kfm = 1, kfp = 1;
    if (inner) {
        vcm = val[gp - close_d];
        vcp = val[gp + close_d];
        vfm = val[gp - far_d];
        vfp = val[gp + far_d];
        kfm = g.khouot[gp - far_d];
        kfp = g.khouot[gp + far_d];
    }
    double r = v0;
    if (check_span && v0 != 0 && (j < g.elo[i] || j > g.ehi[i])) *g.span_wide = 1;
    if (inner && v0 != 0) {
        int count = 2;
        double nb = vcm + vcp;
        if (kfm == 0) {
            nb += vfm;
            count++;
        }
        if (kfp == 0) {
            nb += vfp;
            count++;
        }
        r = v0 * p.heso + (1 - p.heso) * nb / count;
    }
    out[gp] = r;
}

// The column-major reset byte of cell (i, j) for the column resets that follow (k_reset
// columns): mask | (t_z > z, rows 2..N) << 2 | (wet with H <= H_TINH, rows 2..N) << 3,
// after update_h_moi (support_funcs.cu:60-73) on the wet cells of 1..N x 1..M.
__device__ __forceinline__ void reset_byte_cell(const DevGrid& g, const DevParams& p, int i, int j) {
    if (i >= g.N + 3 || j >= g.M + 3) return;
    const int gp = i * g.P + j;
    const int kv = g.khouot[gp];
    const double tz = g.t_z[gp], zc = g.z[gp], ht = g.htaiz[gp];  // loads first
    unsigned b = (unsigned)kv;
    if (i >= 2 && i <= g.N && tz > zc) b |= 4u;
    if (kv == 0 && i >= 1 && i <= g.N && j >= 1 && j <= g.M) {
        const double hv = ht + tz;
        g.H_moi[gp] = hv;
        if (i >= 2 && hv <= p.H_TINH) b |= 8u;
    }
    g.colB[(size_t)j * g.LT + i] = (unsigned char)b;
}

// Row-lane mapping of the extended-span kernels: g.wpr warps per row, so that a row's
// span is covered in one pass.  Thread -> row i0 + (warp / wpr), first cell offset
// (warp % wpr) * 32 + lane, stride wpr * 32.
struct RowLane {
    int i, off, stride;
    __device__ __forceinline__ RowLane(const DevGrid& g, int i0, int bx) {
        const int gw = (bx * blockDim.x + threadIdx.x) >> 5;
        i = i0 + gw / g.wpr;
        off = (gw % g.wpr) * 32 + (threadIdx.x & 31);
        stride = g.wpr * 32;
    }
};

// The open-edge part of the water budget for one half-step, by kEdgeCtas CTAs for edge e
// (0 up: faces j = M, 1 down: faces j = 1, 2 left: faces i = 1, 3 right: faces i = N), run
// right after the half-step's sweep.  A sweep's continuity row of cell (i, j) reads
//   z' = z - dT/(2 dX) (Htdu[i,j] u[i,j] - Htdu[i-1,j] u[i-1,j])
//          - dT/(2 dY) (Htdv[i,j] v[i,j] - Htdv[i,j-1] v[i,j-1])
// (_uzSolver/_vzSolver_calculate_preindex, UVZSolver_multithread.cu:345-349, 402-406),
// with the implicit component new (t_u in the UZ sweep, t_v in the VZ sweep) and the other
// as it stood; summed over the cells the sweep solved, the inner faces cancel and the
// volume change is the flux through the domain's edge faces.  So for every edge cell the
// sweep solved (the cell lies in a segment of the sweep's lines) its edge face's volume
// flux over the half-step, dT/2 x face depth x velocity x face width, signed into the
// domain, is added to the edge's inflow or outflow.  CTA c of the edge takes the cells
// k = 2 + c blockDim + t (stride kEdgeCtas blockDim) and writes its partial sums; the last
// CTA to finish adds the kEdgeCtas partials in CTA order to the edge's Kahan sums, so the
// result does not depend on the CTAs' order.
// half1: the UZ sweep (x faces t_u, y faces v); otherwise the VZ sweep (x faces u, y faces
// t_v).
// The volume a one-cell segment's continuity row took in through the edge face of edge e
// (0 up: north face, 1 down: south, 2 left: west, 3 right: east) of cell (i, j): the
// cell's level change less what its other three faces carried.  Extracting a one-cell
// segment never writes the velocity of the face before it (_uzSolver/_vzSolver_extract_
// solution, UVZSolver_multithread.cu:595-723: the branch that sets it runs for cells
// before the last one), so where the segment starts on the edge that face keeps an older
// velocity while the row used the boundary's; the face's own product would miss the
// difference.  (A run starting at a line's last two cells is not a segment, so the far
// edge has no such cell.)
__device__ __forceinline__ double single_cell_edge_inflow(const DevGrid& g, const DevParams& p, int half1, int i, int j,
                                                          int e) {
    const int P = g.P, c = i * P + j;
    const double* xu = half1 ? g.t_u : g.u;
    const double* yv = half1 ? g.v : g.t_v;
    const double h = p.dT * 0.5;
    const double west = h * p.dY * g.Htdu[c - P] * xu[c - P], east = -h * p.dY * g.Htdu[c] * xu[c];
    const double south = h * p.dX * g.Htdv[c - 1] * yv[c - 1], north = -h * p.dX * g.Htdv[c] * yv[c];
    const double dv = (g.t_z[c] - g.z[c]) * p.dX * p.dY;
    if (e == 0) return dv - (west + east + south);
    if (e == 1) return dv - (west + east + north);
    if (e == 2) return dv - (east + south + north);
    return dv - (west + south + north);
}

__device__ void edge_budget(const DevGrid& g, const DevParams& p, int half1, int e, int c) {
    __shared__ double s_in[32], s_out[32];
    __shared__ int s_last;
    const int N = g.N, M = g.M, P = g.P;
    const int n = e >= 2 ? M : N;  // edge cells j = 2..M (left/right) or i = 2..N (up/down)
    double vin = 0.0, vout = 0.0;
    for (int k = 2 + c * blockDim.x + threadIdx.x; k <= n; k += kEdgeCtas * blockDim.x) {
        int i, j, fp;
        double sgn;
        if (e == 0) { i = k; j = M; fp = i * P + M; sgn = -1.0; }
        else if (e == 1) { i = k; j = 2; fp = i * P + 1; sgn = 1.0; }
        else if (e == 2) { i = 2; j = k; fp = 1 * P + j; sgn = 1.0; }
        else { i = N; j = k; fp = N * P + j; sgn = -1.0; }
        if (g.khouot[i * P + j] != 0) continue;
        int f, l;
        const int seg = half1 ? find_seg_u(g, i, j, f, l) : find_seg_v(g, i, j, f, l);
        if (seg < 0) continue;
        double q;
        if (e >= 2) q = g.Htdu[fp] * (half1 ? g.t_u[fp] : g.u[fp]) * p.dY;
        else q = g.Htdv[fp] * (half1 ? g.v[fp] : g.t_v[fp]) * p.dX;
        // the face before a one-cell segment that starts on the edge (the sweep's own
        // direction: left edge for the UZ sweep's columns, down edge for the VZ sweep's rows)
        const bool stale = f == l && (half1 ? e == 2 : e == 1);
        const double vol = stale ? single_cell_edge_inflow(g, p, half1, i, j, e) : sgn * q * (p.dT * 0.5);
        if (vol > 0) vin += vol;
        else vout -= vol;
    }
    for (int o = 16; o > 0; o >>= 1) {
        vin += __shfl_down_sync(0xffffffffu, vin, o);
        vout += __shfl_down_sync(0xffffffffu, vout, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_in[w] = vin;
        s_out[w] = vout;
    }
    __syncthreads();
    double* B = g.budget;
    unsigned* count = reinterpret_cast<unsigned*>(B + kBudCount) + e;
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
            a += s_in[q];
            b += s_out[q];
        }
        B[kBudPart + 2 * (e * kEdgeCtas + c)] = a;
        B[kBudPart + 2 * (e * kEdgeCtas + c) + 1] = b;
        __threadfence();
        s_last = atomicAdd(count, 1u) == (unsigned)(kEdgeCtas - 1);
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    const volatile double* V = B;
    double a = 0.0, b = 0.0;
    for (int q = 0; q < kEdgeCtas; q++) {
        a += V[kBudPart + 2 * (e * kEdgeCtas + q)];
        b += V[kBudPart + 2 * (e * kEdgeCtas + q) + 1];
    }
    auto kahan = [&](int sum, int comp, double x) {
        const double y = x - B[comp];
        const double t = B[sum] + y;
        B[comp] = (t - B[sum]) - y;
        B[sum] = t;
    };
    kahan(kBudNet + e, kBudNetC + e, a - b);
    kahan(kBudIn + e, kBudInC + e, a);
    kahan(kBudOut + e, kBudOutC + e, b);
    *count = 0u;  // ready for the next half-step (stream order separates the launches)
}

// The water a half-step's continuity rows move between a cell the sweep solved and a wet
// cell it did not, for cell (i, j) of [2,N] x [2,M] (m^3, out of the solved cells
// positive).  The segment scan skips a wet run that starts at the line's last two cells
// (Find_Calculation_limits, support_funcs.cu:230-335), so a wet cell of rows N-1..N (the
// UZ sweep's columns) or of columns M-1..M (the VZ sweep's rows) can lie in no segment;
// its neighbours across the sweep still carry their face flux to it (the explicit v in the
// UZ half-step, u in the VZ half-step), which the unsolved cell does not receive.  (The
// same faces towards a dry or land cell carry no flux: the velocities there are zero.)
// Such an unsolved cell may also lie on an edge whose stage the boundary imposes; the
// level change that puts on it is returned for it (as water gained, a negative loss).
// Faces on the domain's edges are edge_budget's.
__device__ __forceinline__ double leak_cell(const DevGrid& g, const DevParams& p, int isU, int i, int j) {
    const int N = g.N, M = g.M, P = g.P;
    if (i < 2 || i > N || j < 2 || j > M) return 0.0;
    if (isU ? i < N - 1 : j < M - 1) return 0.0;
    const int gp = i * P + j;
    if (g.khouot[gp] != 0) return 0.0;
    int f, l;
    double q = 0.0;
    // a wet cell the sweep does not solve keeps its level unless the boundary set it
    // (Update_Boundary_Value writes the stage of the edge's first segment into t_z,
    // support_funcs.cu:622-668, whether or not the cell lies in a segment of this sweep):
    // that level change adds water no face carried, entered here as a negative loss
    const double imposed = -(g.t_z[gp] - g.z[gp]) * p.dX * p.dY;
    if (isU) {
        if (find_seg_u(g, i, j, f, l) < 0) return imposed;
        if (j + 1 <= M && g.khouot[gp + 1] == 0 && find_seg_u(g, i, j + 1, f, l) < 0) q += g.Htdv[gp] * g.v[gp];
        if (j - 1 >= 2 && g.khouot[gp - 1] == 0 && find_seg_u(g, i, j - 1, f, l) < 0)
            q -= g.Htdv[gp - 1] * g.v[gp - 1];
        return q * p.dX * (p.dT * 0.5);
    }
    if (find_seg_v(g, i, j, f, l) < 0) return imposed;
    if (i + 1 <= N && g.khouot[gp + P] == 0 && find_seg_v(g, i + 1, j, f, l) < 0) q += g.Htdu[gp] * g.u[gp];
    if (i - 1 >= 2 && g.khouot[gp - P] == 0 && find_seg_v(g, i - 1, j, f, l) < 0) q -= g.Htdu[gp - P] * g.u[gp - P];
    return q * p.dY * (p.dT * 0.5);
}

// A warp's leak sum added to the budget (one atomic per warp that has one).

__device__ __forceinline__ void add_leak(const DevGrid& g, double q) {
    for (int o = 16; o > 0; o >>= 1) q += __shfl_down_sync(0xffffffffu, q, o);
    if ((threadIdx.x & 31) == 0 && q != 0.0) atomicAdd(&g.budget[kBudLeak], q);
}

// The leak term over the whole grid (after a whole-grid smoothing pass).
__global__ void k_leak_full(DevGrid g, DevParams p, int isU) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    add_leak(g, (i < g.N + 3 && j < g.M + 3) ? leak_cell(g, p, isU, i, j) : 0.0);
}

// The edge budget alone (after a whole-grid smoothing pass): kEdgeCtas CTAs per edge.
__global__ void k_edge_budget(DevGrid g, DevParams p, int half1) {
    edge_budget(g, p, half1, blockIdx.x / kEdgeCtas, blockIdx.x % kEdgeCtas);
}

// The open-edge budget and the leak term of one half-step (isU: the UZ sweep's) as a launch
// of its own, on a stream beside the smoothing and the explicit momentum that follow the
// sweep (it reads the swept velocity, the other component, the face depths, the mask and
// the sweep's segments, none of which those launches write; the resets that change the
// mask wait for it): kBudCtas edge CTAs, then CTAs over the cells of the last two rows
// (UZ) or columns (VZ), the only cells leak_cell counts.
__global__ void k_budget_half(DevGrid g, DevParams p, int isU) {
    if ((int)blockIdx.x < kBudCtas) {
        edge_budget(g, p, isU, blockIdx.x / kEdgeCtas, blockIdx.x % kEdgeCtas);
        return;
    }
    const int t = (blockIdx.x - kBudCtas) * blockDim.x + threadIdx.x;
    double q = 0.0;
    if (isU) {  // rows N-1, N; columns 2..M
        const int n = g.M - 1;
        if (t < 2 * n) q = leak_cell(g, p, 1, g.N - 1 + t / n, 2 + t % n);
    } else {  // columns M-1, M; rows 2..N
        const int n = g.N - 1;
        if (t < 2 * n) q = leak_cell(g, p, 0, 2 + t % n, g.M - 1 + t / n);
    }
    add_leak(g, q);  // every lane of the warp takes part
}

// BYTES: also write the column reset bytes (the smoothing of u right before the column
// resets; H_moi is not read in between).
template <int BYTES>
__global__ void k_smooth(DevGrid g, DevParams p, int isU, double* __restrict__ out) {
    const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    smooth_cell(g, p, isU, out, i, j, true);
    if (BYTES) reset_byte_cell(g, p, i, j);
}

// FSB: one more CTA (the first) applies the concentration part of the second half-step's
// boundary (kBndFS), when the velocity/level part ran before the first half-step's
// sediment sweep had finished.
// BUD: kBudCtas more CTAs (the first) add the half-step's open-edge volumes to the budget
// (edge_budget; the smoothing of the swept velocity, isU = the UZ sweep's half-step); the
// smoothing warps add the flows to wet cells in no segment (leak_cell).
template <int BYTES, int FSB, int BUD>
__device__ __forceinline__ void smooth_span_body(const DevGrid& g, const DevParams& p, int isU,
                                                 double* __restrict__ out, int bx, int gx) {
    // the budget and boundary CTAs (chains of dependent loads) first, beside the smoothing
    if (BUD) {
        if (bx < 4 * kEdgeCtas) {
            edge_budget(g, p, isU, bx / kEdgeCtas, bx % kEdgeCtas);
            return;
        }
        bx -= kBudCtas;
    }
    if (FSB) {
        if (bx == 0) {
            boundary_body(g, g.clock[1], kBndFS);
            return;
        }
        bx -= 1;
    }
    const RowLane rl(g, 0, bx);
    const int i = rl.i;
    double leak = 0.0;
    if (i <= g.N + 2) {
        for (int j = g.elo[i] + rl.off; j <= g.ehi[i]; j += rl.stride) {
            smooth_cell(g, p, isU, out, i, j, false);
            if (BYTES) reset_byte_cell(g, p, i, j);
            if (BUD) leak += leak_cell(g, p, isU, i, j);
        }
    }
    if (BUD) add_leak(g, leak);  // every lane of the warp takes part
}

template <int BYTES, int FSB, int BUD>
__global__ void k_smooth_span(DevGrid g, DevParams p, int isU, double* __restrict__ out) {
    smooth_span_body<BYTES, FSB, BUD>(g, p, isU, out, blockIdx.x, gridDim.x);
}
// outs[m]: member m's output array
template <int BYTES, int FSB, int BUD>
__global__ void k_smooth_span_b(BatchRef br, int isU, double* const* outs) {
    const BatchMember bm(br);
    smooth_span_body<BYTES, FSB, BUD>(bm.g, bm.p, isU, outs[bm.m], bm.bx, bm.gx);
}

// ----------------------------------------------------------- explicit momentum

// vSolver (UVZSolver_multithread.cu:727-768) for one cell in the arithmetic type R: the new
// v velocity.
template <class R>
__device__ __forceinline__ R ev_cell(const DevGrid& g, const DevParams& p, int row, int col) {
    const int o = g.P;
    const double *u = g.u, *v = g.v, *z = g.z, *t_u = g.t_u, *H = g.H_moi;
    auto L = [](const double* a, int q) { return R(a[q]); };
    R pp, q, tmp;
    q = 0;
    pp = 0;
    tmp = 0;
    const R v0 = L(v, row * o + col);
    const R utb = (L(u, (row - 1) * o + col) + L(u, row * o + col) + L(u, (row - 1) * o + col + 1) + L(u, row * o + col + 1)) * R(0.25);
    const R t_utb = (L(t_u, (row - 1) * o + col) + L(t_u, row * o + col) + L(t_u, (row - 1) * o + col + 1) + L(t_u, row * o + col + 1)) * R(0.25);
    pp = (L(v, row * o + col + 1) - L(v, row * o + col - 1)) / R(p.dY2);
    pp = R(p.HaiChiadT) + pp + L(g.Ky1, row * o + col) * sqrt(utb * utb + v0 * v0) / L(g.Htdv, row * o + col);
    // the neighbours the branches take, loaded before the depth tests (one round trip)
    const R vm1 = L(v, (row - 1) * o + col), vp1 = L(v, (row + 1) * o + col), vm2 = L(v, (row - 2) * o + col),
            vp2 = L(v, (row + 2) * o + col);
    const double Hm1 = H[(row - 1) * o + col], Hp1 = H[(row + 1) * o + col], Hm2 = H[(row - 2) * o + col];
    if (Hm1 <= p.H_TINH) {
        if (utb < 0) {
            q = t_utb * (-3 * v0 + 4 * vp1 - vp2) / R(p.dX2);
            tmp = (v0 - 2 * vp1 + vp2) / R(p.dXbp);
        }
    } else {
        if (Hp1 <= p.H_TINH) {
            if ((Hm2 > p.H_TINH) && (utb > 0)) {
                q = t_utb * (3 * v0 - 4 * vm1 + vm2) / R(p.dX2);
                tmp = (v0 - 2 * vm1 + vm2) / R(p.dXbp);
            }
        } else {
            q = t_utb * (vp1 - vm1) / R(p.dX2);
            tmp = (vp1 - 2 * v0 + vm1) / R(p.dXbp);
        }
    }
    q = R(p.HaiChiadT) * v0 - q - R(p.CORIOLIS_FORCE) * t_utb;
    q = (q - R(p.g) * R(z[row * o + col + 1] - z[row * o + col]) / R(p.dY) +
         L(g.VISC, row * o + col) * (tmp + (L(v, row * o + col + 1) - 2 * v0 + L(v, row * o + col - 1)) / R(p.dYbp))) +
        (R(p.windy) - L(g.Tsyw, row * o + col)) / L(g.Htdv, row * o + col);
    return q / pp;
}

// solveV/vSolver (UVZSolver_multithread.cu:1055-1071, 727-768) on row i, then
// update_margin_elem_V (1008-1052) for the same row.
template <class R>
__device__ __forceinline__ void explicit_v_body(const DevGrid& g, const DevParams& p, int bx) {
    extern __shared__ double sv[];  // the row's t_v over [k0, k1]
    __shared__ int s_b1[HYD_SEGL], s_b2[HYD_SEGL], s_first[HYD_SEGL], s_last[HYD_SEGL], s_off[HYD_SEGL + 1];
    const int row = 2 + bx;
    const int P = g.P, M = g.M;
    const int nseg = g.moci[row];
    if (nseg == 0) return;
    // cells read or written: two before the first segment to one past the last
    const int k0 = max(g.daui[row * HYD_SEGL] - 2, 0);
    const int k1 = min(g.cuoii[row * HYD_SEGL + nseg - 1] + 1, M + 2);
    if (k1 - k0 + 1 > g.sv_cap) {  // cannot happen while the spans hold (see refresh_widths)
        if (threadIdx.x == 0) flag_status(g, HYD_ST_STAGE_RANGE);
        return;
    }
    for (int j = k0 + threadIdx.x; j <= k1; j += blockDim.x) sv[j - k0] = g.t_v[row * P + j];
    if ((int)threadIdx.x < nseg) {
        const int i = row, W = P, k = threadIdx.x;
        const int first = g.daui[i * HYD_SEGL + k], last = g.cuoii[i * HYD_SEGL + k];
        const double* h = g.h;
        s_first[k] = first;
        s_last[k] = last;
        s_b1[k] = (first > 2) || ((first == 2) && (fabs((h[i * W + first - 1] + h[(i - 1) * W + first - 1]) * 0.5 - p.NANGDAY) < kEpsRef));
        s_b2[k] = (last < M) || ((last == M) && (fabs((h[i * W + last] + h[(i - 1) * W + last]) * 0.5 - p.NANGDAY) < kEpsRef));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int off = 0;
        for (int q = 0; q < nseg; q++) {
            s_off[q] = off;
            off += max(s_last[q] - s_first[q], 0);
        }
        s_off[nseg] = off;
    }
    __syncthreads();
    // every cell first..last-1 of every segment, packed segment after segment
    for (int c = threadIdx.x; c < s_off[nseg]; c += blockDim.x) {
        int k = 0;
        while (k + 1 < nseg && s_off[k + 1] <= c) k++;
        const int col = s_first[k] + (c - s_off[k]);
        const double tv = ev_cell<R>(g, p, row, col);
        g.t_v[row * P + col] = tv;
        sv[col - k0] = tv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // segment ends in order, on the staged row (update_margin_elem_V)
        double* t_v = g.t_v + row * P;
        for (int k = 0; k < nseg; k++) {
            const int first = s_first[k], last = s_last[k];
            const double a = s_b1[k] ? 0.0 : 2 * sv[first - k0] - sv[first + 1 - k0];
            sv[first - 1 - k0] = a;
            t_v[first - 1] = a;
            const double b = s_b2[k] ? 0.0 : 2 * sv[last - 1 - k0] - sv[last - 2 - k0];
            sv[last - k0] = b;
            t_v[last] = b;
        }
    }
    __syncthreads();  // keep the other warps resident while thread 0 works
}

template <class R>
__global__ void k_explicit_v(DevGrid g, DevParams p) {
    explicit_v_body<R>(g, p, blockIdx.x);
}
template <class R>
__global__ void k_explicit_v_b(BatchRef br) {
    const BatchMember bm(br);
    explicit_v_body<R>(bm.g, bm.p, bm.bx);
}

// uSolver (UVZSolver_multithread.cu:773-815) for one cell in the arithmetic type R: the new
// u velocity.  Cell-local, so it is computed for every wet cell by a row-major kernel and
// stored column-major.
template <class R>
__device__ __forceinline__ R eu_cell(const DevGrid& g, const DevParams& p, int row, int col) {
    const int P = g.P;
    const double *u = g.u, *v = g.v, *z = g.z, *t_v = g.t_v, *H = g.H_moi;
    auto L = [](const double* a, int q) { return R(a[q]); };
    const int o = P;
    R pp, q, tmp;
    pp = 0;
    q = 0;
    tmp = 0;
    const R u0 = L(u, row * o + col);
    const R vtb = (L(v, row * o + col - 1) + L(v, row * o + col) + L(v, (row + 1) * o + col - 1) + L(v, (row + 1) * o + col)) * R(0.25);
    const R t_vtb = (L(t_v, row * o + col - 1) + L(t_v, row * o + col) + L(t_v, (row + 1) * o + col - 1) + L(t_v, (row + 1) * o + col)) * R(0.25);
    pp = (L(u, (row + 1) * o + col) - L(u, (row - 1) * o + col)) / R(p.dX2);
    pp = (R(p.HaiChiadT) + pp + L(g.Kx1, row * o + col) * sqrt(vtb * vtb + u0 * u0) / L(g.Htdu, row * o + col));
    // as in ev_cell: the branches' neighbours loaded first
    const R um1 = L(u, row * o + col - 1), up1 = L(u, row * o + col + 1), um2 = L(u, row * o + col - 2),
            up2 = L(u, row * o + col + 2);
    const double Hm1 = H[row * o + col - 1], Hp1 = H[row * o + col + 1], Hm2 = H[row * o + col - 2];
    if (Hm1 <= p.H_TINH) {
        if (vtb < 0) {
            q = t_vtb * (-3 * u0 + 4 * up1 - up2) / R(p.dY2);
            tmp = (u0 - 2 * up1 + up2) / R(p.dYbp);
        }
    } else {
        if (Hp1 <= p.H_TINH) {
            if ((Hm2 > p.H_TINH) && (vtb > 0)) {
                q = t_vtb * (3 * u0 - 4 * um1 + um2) / R(p.dY2);
                tmp = (u0 - 2 * um1 + um2) / R(p.dYbp);
            }
        } else {
            q = t_vtb * (up1 - um1) / R(p.dY2);
            tmp = (up1 - 2 * u0 + um1) / R(p.dYbp);
        }
    }
    q = R(p.HaiChiadT) * u0 - q + R(p.CORIOLIS_FORCE) * t_vtb;
    q = (q - R(p.g) * R(z[(row + 1) * o + col] - z[row * o + col]) / R(p.dX) +
         L(g.VISC, row * o + col) * (tmp + (L(u, (row + 1) * o + col) - 2 * u0 + L(u, (row - 1) * o + col)) / R(p.dXbp))) +
        (R(p.windx) - L(g.Tsxw, row * o + col)) / L(g.Htdu, row * o + col);
    return q / pp;
}

// The column-major slot of the explicit_u values: not one of the FSj coefficients' slots
// (0..3), which the FSj sweep may still be reading while the next half-step runs.
constexpr int kEuSlot = 4;

// explicit_u values of every wet cell of rows 2..N-1, columns 2..M, one warp per row over
// the row's span; written column-major (g.colT array kEuSlot), with TILE through a tile.
template <int TILE, class R>
__device__ __forceinline__ void coef_eu_body(const DevGrid& g, const DevParams& p, int bx) {
    if constexpr (!TILE) {
        const int i = 2 + ((bx * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
        if (i > g.N - 1) return;
        const int lo = max(g.rlo[i], 2), hi = min(g.rhi[i], g.M);
        for (int j = lo + lane; j <= hi; j += 32) {
            if (g.khouot[i * g.P + j] != 0) continue;
            colTr<R>(g, kEuSlot)[(size_t)j * g.LT + i] = eu_cell<R>(g, p, i, j);
        }
    } else {
        R* const dst[1] = {colTr<R>(g, kEuSlot)};
        colmajor_tile<1>(
            g, 2 + kTileRows * bx, g.N - 1, 2, g.M,
            [&](int i, int j, R* v) {
                if (g.khouot[i * g.P + j] != 0) return false;
                v[0] = eu_cell<R>(g, p, i, j);
                return true;
            },
            dst);
    }
}

template <int TILE, class R>
__global__ void __launch_bounds__(256) k_coef_eu(DevGrid g, DevParams p) {
    coef_eu_body<TILE, R>(g, p, blockIdx.x);
}
template <int TILE, class R>
__global__ void __launch_bounds__(256) k_coef_eu_b(BatchRef br) {
    const BatchMember bm(br);
    coef_eu_body<TILE, R>(bm.g, bm.p, bm.bx);
}

// solveU/uSolver (UVZSolver_multithread.cu:947-968, 773-815) on column j from the values
// k_coef_eu stored, then update_margin_elem_U (970-1006).
template <class R>
__device__ __forceinline__ void explicit_u_body(const DevGrid& g, const DevParams& p, int bx) {
    extern __shared__ double su[];  // the column's t_u over [k0, k1]
    __shared__ int s_b1[HYD_SEGL], s_b2[HYD_SEGL], s_first[HYD_SEGL], s_last[HYD_SEGL], s_off[HYD_SEGL + 1];
    const int col = 2 + bx;
    const int P = g.P, N = g.N;
    const int nseg = g.mocj[col];
    if (nseg == 0) return;
    const int k0 = max(g.dauj[col * HYD_SEGL] - 2, 0);
    const int k1 = min(g.cuoij[col * HYD_SEGL + nseg - 1] + 1, N + 2);
    if (k1 - k0 + 1 > g.su_cap) {  // cannot happen while the spans hold (see refresh_widths)
        if (threadIdx.x == 0) flag_status(g, HYD_ST_STAGE_RANGE);
        return;
    }
    for (int i = k0 + threadIdx.x; i <= k1; i += blockDim.x) su[i - k0] = g.t_u[i * P + col];
    if ((int)threadIdx.x < nseg) {
        const int j = col, W = P, k = threadIdx.x;
        const int first = g.dauj[j * HYD_SEGL + k], last = g.cuoij[j * HYD_SEGL + k];
        const double* h = g.h;
        s_first[k] = first;
        s_last[k] = last;
        s_b1[k] = (first > 2) || ((first == 2) && ((fabs(h[1 * W + j] + h[1 * W + j - 1]) * 0.5 - p.NANGDAY) < kEpsRef));
        s_b2[k] = (last < N) || ((last == N) && (fabs((h[N * W + j] + h[N * W + j - 1]) * 0.5 - p.NANGDAY) < kEpsRef));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int off = 0;
        for (int q = 0; q < nseg; q++) {
            s_off[q] = off;
            off += max(s_last[q] - s_first[q], 0);
        }
        s_off[nseg] = off;
    }
    __syncthreads();
    // every cell first..last-1 of every segment, packed segment after segment
    for (int c = threadIdx.x; c < s_off[nseg]; c += blockDim.x) {
        {
            int k = 0;
            while (k + 1 < nseg && s_off[k + 1] <= c) k++;
            const int row = s_first[k] + (c - s_off[k]);
            const double tu = colTr<R>(g, kEuSlot)[(size_t)col * g.LT + row];  // k_coef_eu
            g.t_u[row * P + col] = tu;
            su[row - k0] = tu;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // segment ends in order, on the staged column (update_margin_elem_U)
        for (int k = 0; k < nseg; k++) {
            const int first = s_first[k], last = s_last[k];
            const double a = s_b1[k] ? 0.0 : 2 * su[first - k0] - su[first + 1 - k0];
            su[first - 1 - k0] = a;
            g.t_u[(first - 1) * P + col] = a;
            const double b = s_b2[k] ? 0.0 : 2 * su[last - 1 - k0] - su[last - 2 - k0];
            su[last - k0] = b;
            g.t_u[last * P + col] = b;
        }
    }
    __syncthreads();  // keep the other warps resident while thread 0 works
}

template <class R>
__global__ void k_explicit_u(DevGrid g, DevParams p) {
    explicit_u_body<R>(g, p, blockIdx.x);
}
template <class R>
__global__ void k_explicit_u_b(BatchRef br) {
    const BatchMember bm(br);
    explicit_u_body<R>(bm.g, bm.p, bm.bx);
}

// --------------------------------------------------------------- wet/dry resets

// Mark line `line` of the other direction for a segment rescan (once).
__device__ __forceinline__ void mark_dirty(int* flags, int* list, unsigned* ctr, int line) {
    if (atomicExch(&flags[line], 1) == 0) list[atomicAdd(ctr, 1u)] = line;
}

struct WetBytes;
struct WetGlobal;

// The wet flags of cells a..b packed into 32-cell words by one warp: bit t of
// words[w - w0] is cell origin + 32 w + t (cells outside [a, b] give 0), w = w0..w1.
// Generic form: one cell per lane and word, origin 2.
template <class Wet>
__device__ __forceinline__ void pack_wet_words(const Wet& wet, int a, int b, int origin, unsigned* words, int w0,
                                               int w1) {
    const int lane = threadIdx.x & 31;
    for (int w = w0; w <= w1; w++) {
        const int k = origin + 32 * w + lane;
        const bool z = (k >= a && k <= b) ? wet(k) : false;
        const unsigned bits = __ballot_sync(0xffffffffu, z);
        if (lane == 0) words[w - w0] = bits;
    }
}

// Column-major mask bytes (origin 0): 16 consecutive bytes per lane (one 16-byte load),
// 512 cells per pass, so that a 4096-cell column takes 8 dependent loads instead of 128.
// Lanes 2m and 2m+1 hold the two halves of word (base >> 5) + m.  A column starts on a
// 32-byte boundary and holds LT >= N + 3 bytes, LT a multiple of 32, so a lane's load at
// c <= b <= N (c a multiple of 16) ends within the column.
__device__ __forceinline__ void pack_wet_bytes(const unsigned char* col, int a, int b, unsigned* words, int w0,
                                               int w1) {
    const int lane = threadIdx.x & 31;
    for (int base = w0 * 32; base <= w1 * 32 + 31; base += 512) {
        const int c = base + lane * 16;
        unsigned m = 0;
        if (c <= b) {
            const uint4 q = *reinterpret_cast<const uint4*>(col + c);
            const unsigned v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int t = 0; t < 16; t++) {
                const int k = c + t;
                if (((v[t >> 2] >> (8 * (t & 3))) & 3u) == 0u && k >= a && k <= b) m |= 1u << t;
            }
        }
        const unsigned hi = __shfl_down_sync(0xffffffffu, m, 1);
        const int w = (base >> 5) + (lane >> 1);
        if ((lane & 1) == 0 && w <= w1) words[w - w0] = m | (hi << 16);
    }
}

// A row of the int mask (origin 0): 4 consecutive cells per lane (one 16-byte load), 128
// cells per pass; lanes 8m..8m+7 make word (base >> 5) + m.  A row starts on a 128-byte
// boundary (the pitch is a multiple of 32 cells) and holds pitch >= M + 3 cells, so a
// lane's load at c <= b <= M (c a multiple of 4) ends within the row.
__device__ __forceinline__ void pack_wet_ints(const int* row, int a, int b, unsigned* words, int w0, int w1) {
    const int lane = threadIdx.x & 31;
    for (int base = w0 * 32; base <= w1 * 32 + 31; base += 128) {
        const int c = base + lane * 4;
        unsigned m = 0;
        if (c <= b) {
            const int4 q = *reinterpret_cast<const int4*>(row + c);
            if (q.x == 0 && c >= a && c <= b) m |= 1u;
            if (q.y == 0 && c + 1 >= a && c + 1 <= b) m |= 2u;
            if (q.z == 0 && c + 2 >= a && c + 2 <= b) m |= 4u;
            if (q.w == 0 && c + 3 >= a && c + 3 <= b) m |= 8u;
        }
        m <<= 4 * (lane & 7);
        m |= __shfl_xor_sync(0xffffffffu, m, 1);
        m |= __shfl_xor_sync(0xffffffffu, m, 2);
        m |= __shfl_xor_sync(0xffffffffu, m, 4);
        const int w = (base >> 5) + (lane >> 3);
        if ((lane & 7) == 0 && w <= w1) words[w - w0] = m;
    }
}

// Wet-segment scan of one line by one warp (Find_Calculation_limits_Horizontal/Vertical,
// support_funcs.cu:230-335).  The serial while-loop there yields the maximal runs of
// khouot == 0 within [2, L] in order, except runs starting at L-1 or L, which it skips.
// Cells a..b are tested with wet(k); every other cell is dry.  The warp packs the wet
// flags into 32-cell words (words: (b - a) / 32 + 2 entries of shared memory; mask bytes
// and mask rows with wide loads), then lane 0 walks the run starts and ends word by word.
template <class Wet>
__device__ void warp_scan_line(const DevGrid& g, Wet wet, int a, int b, int L, unsigned* words, int* dau, int* cuoi,
                               int* moc) {
    const int lane = threadIdx.x & 31;
    if (a < 2) a = 2;
    if (b > L) b = L;
    int origin = 2;
    if constexpr (std::is_same<Wet, WetBytes>::value) origin = 0;
    if constexpr (std::is_same<Wet, WetGlobal>::value) origin = wet.along == 1 ? 0 : 2;
    const int w0 = (a - origin) >> 5, w1 = (b - origin) >> 5;
    if (b >= a) {
        if constexpr (std::is_same<Wet, WetBytes>::value) {
            pack_wet_bytes(wet.col, a, b, words, w0, w1);
        } else if constexpr (std::is_same<Wet, WetGlobal>::value) {
            if (wet.along == 1) pack_wet_ints(wet.kh + wet.base, a, b, words, w0, w1);
            else pack_wet_words(wet, a, b, origin, words, w0, w1);
        } else {
            pack_wet_words(wet, a, b, origin, words, w0, w1);
        }
    }
    __syncwarp();
    if (lane == 0) {
        int nseg = 0;
        int open_start = -1;
        for (int w = w0; b >= a && w <= w1; w++) {
            const unsigned cur = words[w - w0];
            const unsigned prev = w > w0 ? words[w - w0 - 1] : 0u;
            const unsigned next = w < w1 ? words[w - w0 + 1] : 0u;
            unsigned starts = cur & ~((cur << 1) | (prev >> 31));
            unsigned ends = cur & ~((cur >> 1) | (next << 31));
            const int c0 = origin + 32 * w;
            // events in position order; a run's start precedes or equals its end
            while (starts | ends) {
                if (open_start < 0) {
                    if (!starts) break;
                    open_start = c0 + __ffs(starts) - 1;
                    starts &= starts - 1;
                } else {
                    if (!ends) break;  // the run continues into the next word
                    const int e = c0 + __ffs(ends) - 1;
                    ends &= ends - 1;
                    if (open_start <= L - 2) {
                        if (nseg < HYD_SEGL) {
                            dau[nseg] = open_start;
                            cuoi[nseg] = e;
                        } else {
                            flag_status(g, HYD_ST_SEG_OVERFLOW);
                        }
                        nseg++;
                    }
                    open_start = -1;
                }
            }
        }
        *moc = nseg < HYD_SEGL ? nseg : HYD_SEGL;
    }
    __syncwarp();
}

struct WetShared {  // staged mask: cell k at kh[k - k0]
    const signed char* kh;
    int k0;
    __device__ bool operator()(int k) const { return kh[k - k0] == 0; }
};

struct WetGlobal {  // mask in HBM: cell k at kh[base + k * along]
    const int* kh;
    int base, along;
    __device__ bool operator()(int k) const { return kh[base + k * along] == 0; }
};

// A column's mask from its column-major reset bytes (g.colB, low two bits): one coalesced
// byte per cell instead of one 32-byte sector per 4-byte mask value of the pitched grid.
// The resets keep those bits equal to the mask (they write the byte of every cell they
// open or close; the smoothing pass before the column resets rewrites every byte).
// warp_scan_line packs these bytes 16 at a time (pack_wet_bytes).
struct WetBytes {
    const unsigned char* col;
};

// Words of each k_reset bitset: one bit per cell of a line.
__host__ __device__ __forceinline__ int reset_words(int L) { return (L + 3) / 32 + 2; }

// update_h_moi (support_funcs.cu:60-73) and Reset_states_horizontal/_vertical
// (support_funcs.cu:75-186) for one line.  ROWS: line = row i (1..N), cells j (2..M);
// otherwise line = column j (1..M), cells i (2..N).
// Cells whose mask is 2 never change (only 0 <-> 1 transitions exist), so each line is
// staged in shared memory over its span [lo, hi] of cells that are not 2, widened by one
// cell: nothing outside can act or be acted on.
// The opening pass is a serial scan in the reference.  Iteration k acts when t_z[k] >
// z[k] and a neighbour's mask is 1; the only value it passes on is through the cell k+1
// it opens, whose t_z it sets, so iteration k+1 then tests that value (a cascade through
// a run of 1s).  Every other iteration sees the t_z, z and mask 1s of the start of the
// pass.  So the CTA tests t_z[k] > z[k] and the mask-1 neighbours for all cells at once
// (bitsets), and one thread runs only the cells that pass, in increasing order, each
// with its cascade.  The closing pass closes the cells that are wet after the opening
// pass with H <= H_TINH: the cells wet from the start (their H is update_h_moi's) and
// the cells just opened (H stored with the opening), known as a bitset too.
// Rows stage the mask, t_z and z of the row (coalesced) and apply update_h_moi here.
// Columns read the column-major byte the preceding smoothing pass wrote per cell (mask,
// t_z > z, wet with H <= H_TINH; it also applied update_h_moi), so a column is one
// coalesced byte read instead of strided loads.
// A line only changes its own cells, so its segments are rescanned here when a cell
// changed (or when `force`); every changed cell marks its line of the other direction
// for the rescan that follows.
// blockDim.x is a multiple of 32: each warp pass covers whole 32-cell words.
template <int ROWS>
__device__ __forceinline__ void reset_body(const DevGrid& g, const DevParams& p, int force, int bx) {
    extern __shared__ unsigned char rsm[];
    __shared__ int s_changed;
    const int line = 1 + bx;
    const int P = g.P;
    const int L = ROWS ? g.M : g.N;  // last cell index of the line
    const int along = ROWS ? 1 : P;
    const int base = ROWS ? line * P : line;
    const int lo = ROWS ? g.rlo[line] : g.clo[line];
    const int hi = ROWS ? g.rhi[line] : g.chi[line];
    int* dau = ROWS ? g.daui + line * HYD_SEGL : g.dauj + line * HYD_SEGL;
    int* cuoi = ROWS ? g.cuoii + line * HYD_SEGL : g.cuoij + line * HYD_SEGL;
    int* moc = ROWS ? g.moci + line : g.mocj + line;
    if (hi < lo) {  // no cell of the line can ever be wet
        if (force && line >= 2 && threadIdx.x == 0) *moc = 0;
        return;
    }
    int* oflags = ROWS ? g.dirty_c : g.dirty_r;
    int* olist = ROWS ? g.dlist_c : g.dlist_r;
    unsigned* octr = g.dctr + (ROWS ? 1 : 0);
    const int k0 = lo - 1 > 0 ? lo - 1 : 0;
    const int k1 = hi + 1 < L + 2 ? hi + 1 : L + 2;
    const int nwords = reset_words(L);
    signed char* khs = (signed char*)rsm;                       // khs[k - k0], k in [k0, k1]
    unsigned* c0w = (unsigned*)(rsm + ((L + 3 + 15) & ~15));    // t_z > z bits, then scan words
    unsigned* evw = c0w + nwords;                               // cells the opening pass runs
    unsigned* clw = evw + nwords;                               // cells the closing pass closes
    auto khv = [&](int k) -> int { return (k >= k0 && k <= k1) ? khs[k - k0] : 2; };
    double *H = g.H_moi, *t_z = g.t_z, *FS = g.FS;
    const double* z = g.z;
    int* kh = g.khouot;
    const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_changed = 0;
    // staging: the mask and the bits of every cell of [k0, k1]
    for (int kb0 = k0; kb0 <= k1; kb0 += T) {  // uniform over the CTA
        const int k = kb0 + tid;
        const bool in = k <= k1;
        bool c0 = false, cl = false;
        if constexpr (ROWS) {
            if (in) {
                const int gp = base + k;
                const int kv = kh[gp];
                khs[k - k0] = (signed char)kv;
                const double tz = t_z[gp];
                c0 = k >= 2 && k <= L && tz > z[gp];
                if (k >= 1 && k <= L && kv == 0) {
                    const double hv = g.htaiz[gp] + tz;
                    H[gp] = hv;
                    cl = k >= 2 && hv <= p.H_TINH;
                }
            }
        } else {
            const unsigned b = in ? g.colB[(size_t)line * g.LT + k] : 2u;
            if (in) khs[k - k0] = (signed char)(b & 3u);
            c0 = (b >> 2) & 1u;
            cl = (b >> 3) & 1u;
        }
        const unsigned c0b = __ballot_sync(0xffffffffu, c0), clb = __ballot_sync(0xffffffffu, cl);
        const int q = (kb0 - k0 + warp * 32) >> 5;
        if (lane == 0 && kb0 + warp * 32 <= k1) {
            c0w[q] = c0b;
            clw[q] = clb;
        }
    }
    __syncthreads();
    // the cells the opening pass runs: t_z > z with a neighbour whose mask is 1
    const int nq = (k1 - k0) / 32 + 1;
    int anyev = 0;
    for (int q = warp; q < nq; q += T >> 5) {
        const int k = k0 + q * 32 + lane;
        const bool ev = ((c0w[q] >> lane) & 1u) && (khv(k - 1) == 1 || khv(k + 1) == 1);
        const unsigned bits = __ballot_sync(0xffffffffu, ev);
        if (lane == 0) evw[q] = bits;
        anyev |= bits != 0;
    }
    // opening pass (loop 1), serial over those cells
    // interior cells opened / closed here change the domain's water volume (the budget)
    const bool interior_line = line >= 2 && line <= (ROWS ? g.N : g.M);
    double opened = 0.0;
    if (__syncthreads_or(anyev) && warp == 0) {
        const int kb = k1 < L ? k1 : L;
        int done = -1;
        auto open = [&](int kk, double tzv, double fsv) {
            const int gq = base + kk * along;
            const double hv = g.htaiz[gq] + tzv;
            t_z[gq] = tzv;
            H[gq] = hv;
            kh[gq] = 0;
            g.colB[ROWS ? (size_t)kk * g.LT + line : (size_t)line * g.LT + kk] = 0;  // mask bits of the byte
            khs[kk - k0] = 0;
            FS[gq] = fsv;
            if (kk >= 2 && kk <= L && hv <= p.H_TINH) clw[(kk - k0) >> 5] |= 1u << ((kk - k0) & 31);
            if (interior_line && kk >= 2 && kk <= L) opened += hv;
            s_changed = 1;
            mark_dirty(oflags, olist, octr, kk);
        };
        for (int q0 = 0; q0 < nq; q0 += 32) {
            const unsigned wl = q0 + lane < nq ? evw[q0 + lane] : 0u;
            unsigned nz = __ballot_sync(0xffffffffu, wl != 0);
            if (lane == 0) {
                while (nz) {
                    const int q = q0 + __ffs(nz) - 1;
                    nz &= nz - 1;
                    unsigned w = evw[q];
                    while (w) {
                        int m = k0 + q * 32 + __ffs(w) - 1;
                        w &= w - 1;
                        if (m <= done) continue;  // already run inside a cascade
                        const double tzv = t_z[base + m * along], fsv = FS[base + m * along];
                        bool act = true;
                        for (;;) {
                            done = m;
                            if (!act) break;
                            bool right = false;
                            if (khv(m - 1) == 1) open(m - 1, tzv, fsv);
                            if (khv(m + 1) == 1) {
                                open(m + 1, tzv, fsv);
                                right = true;
                            }
                            if (!right || m + 1 > kb) break;
                            m++;  // the opened cell now holds tzv
                            act = tzv > z[base + m * along];
                        }
                    }
                }
            }
            __syncwarp();
        }
    }
    if (opened != 0.0) atomicAdd(&g.budget[kBudOpen], opened);
    __syncthreads();
    // closing pass (loop 2): independent per cell
    double closed = 0.0;
    for (int q = warp; q < nq; q += T >> 5) {
        if (!((clw[q] >> lane) & 1u)) continue;
        const int k = k0 + q * 32 + lane;
        const int gp = base + k * along;
        if (interior_line) closed += H[gp];
        g.t_u[gp - P] = 0;
        g.t_u[gp] = 0;
        g.t_v[gp - 1] = 0;
        g.t_v[gp] = 0;
        kh[gp] = 1;
        g.colB[ROWS ? (size_t)k * g.LT + line : (size_t)line * g.LT + k] = 1;
        khs[k - k0] = 1;
        FS[gp] = 0;
        s_changed = 1;
        mark_dirty(oflags, olist, octr, k);
    }
    if (closed != 0.0) atomicAdd(&g.budget[kBudClose], closed);
    __syncthreads();
    if (tid < 32 && line >= 2 && (s_changed || force))
        warp_scan_line(g, WetShared{khs, k0}, lo, hi, L, c0w, dau, cuoi, moc);
    __syncthreads();  // keep the other warps resident while warp 0 scans
}

template <int ROWS>
__global__ void k_reset(DevGrid g, DevParams p, int force) {
    reset_body<ROWS>(g, p, force, blockIdx.x);
}
template <int ROWS>
__global__ void k_reset_b(BatchRef br, int force) {
    const BatchMember bm(br);
    reset_body<ROWS>(bm.g, bm.p, force, bm.bx);
}

// Column-major mask bytes of the whole grid (the cells outside the extended spans keep
// them: their mask is 2 for good).
__global__ void k_reset_bytes_init(DevGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.N + 3 || j >= g.M + 3) return;
    g.colB[(size_t)j * g.LT + i] = (unsigned char)g.khouot[i * g.P + j];
}

// Spans of the cells whose mask is not 2: rows [rlo, rhi], columns [clo, chi] (the
// bounds start at INT_MAX / -1).
__global__ void k_spans(DevGrid g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.N + 2 || j > g.M + 2) return;
    if (g.khouot[i * g.P + j] != 2) {
        atomicMin(&g.rlo[i], j);
        atomicMax(&g.rhi[i], j);
        atomicMin(&g.clo[j], i);
        atomicMax(&g.chi[j], i);
    }
}

// Extended span of row i: every cell within H cells (rows and columns) of a cell whose
// mask is not 2.  Velocities, levels and depths only change within one cell of those
// cells and the elementwise kernels read one cell around, so outside the extended spans
// they reproduce what is there.
__global__ void k_ext_spans(DevGrid g, int H) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > g.N + 2) return;
    int lo = 0x7fffffff, hi = -1;
    for (int r = i - H; r <= i + H; r++) {
        if (r < 0 || r > g.N + 2 || g.rhi[r] < g.rlo[r]) continue;
        lo = min(lo, g.rlo[r] - H);
        hi = max(hi, g.rhi[r] + H);
    }
    if (hi < lo) {
        // nothing within H rows can change: an empty span of small bounds (the row
        // kernels start at elo plus a lane offset, which must not overflow)
        g.elo[i] = 1;
        g.ehi[i] = 0;
        return;
    }
    g.elo[i] = max(lo, 0);
    g.ehi[i] = min(hi, g.M + 2);
}

// After a full-grid pass found a velocity outside the extended spans: spans = whole rows.
__global__ void k_widen_spans(DevGrid g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > g.N + 2 || !*g.span_wide) return;
    g.elo[i] = 0;
    g.ehi[i] = g.M + 2;
}

// *flag = 1 if a and b differ at a cell of [i0, i1] x [j0, j1] outside the extended span
// of its row (where the span-limited kernels would not bring them together).
__global__ void k_outside_diff(DevGrid g, const double* a, const double* b, int i0, int i1, int j0, int j1,
                               int* flag) {
    const int j = j0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int i = i0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > i1 || j > j1) return;
    if (j >= g.elo[i] && j <= g.ehi[i]) return;
    const int pos = i * g.P + j;
    if (a[pos] != b[pos] && !(a[pos] != a[pos] && b[pos] != b[pos])) *flag = 1;
}

// List every row (ROWS) or column of the grid for a segment rescan.
template <int ROWS>
__global__ void k_mark_all(DevGrid g) {
    const int n = ROWS ? g.N + 3 : g.M + 3;
    int* flags = ROWS ? g.dirty_r : g.dirty_c;
    int* list = ROWS ? g.dlist_r : g.dlist_c;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        flags[k] = 1;
        list[k] = k;
    }
    if (k == 0) g.dctr[ROWS ? 0 : 1] = n;
}

// --------------------------------------------------- state update and face depths

// update_uvz (support_funcs.cu:671-680) and Htuongdoi (338-354) in one pass.  The
// kernel's kenhhepd/kenhhepng parameters never receive the host's flags (Engine.py:90
// passes two arguments fewer than it declares), so velocities are copied unmasked.
__device__ __forceinline__ void post_cell(const DevGrid& g, int with_uvz, int i, int j) {
    const int N = g.N, M = g.M, P = g.P;
    if (i > N || j > M) return;
    const int gp = i * P + j;
    if (with_uvz) {
        g.z[gp] = g.t_z[gp];
        g.u[gp] = g.t_u[gp];
        g.v[gp] = g.t_v[gp];
    }
    if (i < 1 || j < 1) return;
    const double* zs = with_uvz ? g.t_z : g.z;
    const double z_ij = zs[gp];
    const double z_ip = (with_uvz && i + 1 <= N) ? g.t_z[gp + P] : g.z[gp + P];
    const double z_jp = (with_uvz && j + 1 <= M) ? g.t_z[gp + 1] : g.z[gp + 1];
    const double* h = g.h;
    g.Htdu[gp] = (h[gp - 1] + h[gp] + z_ip + z_ij) * 0.5;
    g.Htdv[gp] = (h[gp - P] + h[gp] + z_jp + z_ij) * 0.5;
}

__global__ void k_post(DevGrid g, int with_uvz) {
    post_cell(g, with_uvz, blockIdx.y * blockDim.y + threadIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void k_post_span(DevGrid g) {
    const RowLane rl(g, 0, blockIdx.x);
    const int i = rl.i;
    if (i > g.N) return;
    for (int j = g.elo[i] + rl.off; j <= g.ehi[i]; j += rl.stride) post_cell(g, 1, i, j);
}

// ------------------------------------------------------------- wet-segment scans

template <int AFTER_UPDATE>
__device__ void fs_edges_part(const DevGrid& g, const DevParams& p, int part, int parts);

// Rescan of the listed rows (ROWS) or columns: a line is listed when one of its cells
// changed since its segments were last scanned, and a line whose mask did not change
// keeps segments equal to a fresh scan.  Warp w of the scanning CTAs takes listed lines
// w, w + W, ...; CTA `edges` (or none, -1) runs the edge concentration interpolation of
// the same reference kernels.  The last CTA to finish empties the list.
template <int ROWS>
__global__ void k_scan_dirty(DevGrid g, DevParams p, int edges) {
    extern __shared__ unsigned swords[];
    if ((int)blockIdx.x == edges) {
        fs_edges_part<1>(g, p, 0, 1);
    } else {
        const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int scanning = gridDim.x - (edges >= 0 ? 1 : 0);
        const int n = *(volatile unsigned*)&g.dctr[ROWS ? 0 : 1];
        const int L = ROWS ? g.M : g.N;
        const int Lines = ROWS ? g.N : g.M;
        const int nwords = (L + 63) / 32 + 1;
        unsigned* words = swords + warp * nwords;
        int* flags = ROWS ? g.dirty_r : g.dirty_c;
        const int* list = ROWS ? g.dlist_r : g.dlist_c;
        for (int k = blockIdx.x * warps + warp; k < n; k += scanning * warps) {
            const int line = list[k];
            if (lane == 0) flags[line] = 0;
            if (line < 2 || line > Lines) continue;
            const int lo = ROWS ? g.rlo[line] : g.clo[line];
            const int hi = ROWS ? g.rhi[line] : g.chi[line];
            const WetGlobal wet{g.khouot, ROWS ? line * g.P : line, ROWS ? 1 : g.P};
            if (ROWS) warp_scan_line(g, wet, lo, hi, L, words, g.daui + line * HYD_SEGL, g.cuoii + line * HYD_SEGL, g.moci + line);
            else warp_scan_line(g, wet, lo, hi, L, words, g.dauj + line * HYD_SEGL, g.cuoij + line * HYD_SEGL, g.mocj + line);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned* done = &g.dctr[ROWS ? 2 : 3];
        if (atomicAdd(done, 1u) == gridDim.x - 1) {
            g.dctr[ROWS ? 0 : 1] = 0;
            *done = 0;
            __threadfence();
        }
    }
}

// Interpolate_FS_ng / Interpolate_FS_d (support_funcs.cu:189-229), run by the row-2,
// row-N and column-M blocks of the scans in the reference: row 2, then row N, then column
// M.  One item is one index of one of the three passes: pass 0 (row 2) and pass 1 (row N)
// at column j, pass 2 (column M) at row i.
// AFTER_UPDATE = 0: run concurrently with the state update, so u and v (which the update
// sets to t_u and t_v on i <= N, j <= M) are read as t_u and t_v there.
// CG: FS read through L2 only (values other CTAs of the launch wrote).
template <int AFTER_UPDATE, int CG>
__device__ __forceinline__ void fs_edge_item(const DevGrid& g, const DevParams& p, int pass, int idx) {
    const double* uu = AFTER_UPDATE ? g.u : g.t_u;
    const int N = g.N, M = g.M, P = g.P;
    auto fs = [&](size_t q) { return CG ? __ldcg(g.FS + q) : g.FS[q]; };
    if (pass < 2) {
        const int j = idx;
        const int location = pass == 0 ? 2 : N, offset = pass == 0 ? 2 : N - 1, sign = pass == 0 ? 1 : -1;
        if (g.t_u[location * P + j] > 0) {
            const double deltaX = (uu[location * P + j] + g.t_u[location * P + j]) * 0.25 * p.dT;
            const int i = (int)(offset + sign * (deltaX / p.dX));
            const int i_deltaX = __double2int_rn(deltaX);
            if (i < 0 || i + 1 > N + 2) {
                flag_status(g, HYD_ST_INTERP_RANGE);
                return;
            }
            // the two row passes run side by side: a pass reading the other's edge row
            // would see it in either state
            if (pass == 0 ? i + 1 >= N : i <= 2) flag_status(g, HYD_ST_EDGE_REACH);
            const int i_dX = __double2int_rn(p.dX);
            g.FS[location * P + j] =
                fs((size_t)i * P + j) + sign * (fs((size_t)(i + 1) * P + j) - fs((size_t)i * P + j)) *
                                            (deltaX / p.dX - i_deltaX / i_dX);
        }
    } else {
        const int i = idx;
        const int location = M, offset = M - 1, sign = -1;
        if (g.t_v[i * P + location] > 0) {
            const double vv = (AFTER_UPDATE || i > N) ? g.v[i * P + location] : g.t_v[i * P + location];
            const double deltaY = (vv + g.t_v[i * P + location]) * 0.25 * p.dT;
            const int j = (int)(offset + sign * (deltaY / p.dY));
            const int j_deltaY = __double2int_rn(deltaY);
            if (j < 0 || j + 1 > M + 2) {
                flag_status(g, HYD_ST_INTERP_RANGE);
                return;
            }
            const int j_dY = __double2int_rn(p.dY);
            g.FS[i * P + location] = fs((size_t)i * P + j + 1) + (fs((size_t)i * P + j + 1) - fs((size_t)i * P + j)) *
                                                                    (deltaY / p.dY - j_deltaY / j_dY);
        }
    }
}

// The edge interpolation by `parts` CTAs (this one is `part`).  Items are independent but
// for the column pass at rows 2 and N, which reads the row passes' results in row 2 and
// row N: every other item runs first, spread over the CTAs; the last CTA to finish them
// (counter g.dctr[4], reset by that CTA) then runs those two.
template <int AFTER_UPDATE>
__device__ void fs_edges_part(const DevGrid& g, const DevParams& p, int part, int parts) {
    const int N = g.N, M = g.M;
    const int nrow = M - 1;                       // j = 1 .. M-1
    const int ncol = min(M - 1, N + 2);           // i = 1 .. ncol
    const int K = 2 * nrow + ncol;
    for (int k = part * blockDim.x + threadIdx.x; k < K; k += parts * blockDim.x) {
        if (k < 2 * nrow) {
            fs_edge_item<AFTER_UPDATE, 0>(g, p, k < nrow ? 0 : 1, 1 + (k < nrow ? k : k - nrow));
        } else {
            const int i = 1 + k - 2 * nrow;
            if (i != 2 && i != N) fs_edge_item<AFTER_UPDATE, 0>(g, p, 2, i);
        }
    }
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&g.dctr[4], 1u) == (unsigned)parts - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0 && 2 <= ncol) fs_edge_item<AFTER_UPDATE, 1>(g, p, 2, 2);
    if (threadIdx.x == 32 && N <= ncol && N != 2) fs_edge_item<AFTER_UPDATE, 1>(g, p, 2, N);
    if (threadIdx.x == 0) g.dctr[4] = 0;
}

// --------------------------------------------------------------------- sediment

// The FSi row terms of a wet cell that depend on the cell alone
// (_FSi_calculate__mactrix_coeff, Sediment_Transport.cu:62-165): gamav (evaluated after
// Zf) and the source S, gated by t < bed_change_start, over the depth; into rowC arrays 0
// and 1 (in the arithmetic type R) for the FSi sweep that follows.  vth: the cell's new VTH.
template <class R>
__device__ __forceinline__ void fsi_cell_terms(const DevGrid& g, const DevParams& p, int pos, R vth, double t) {
    const double* FS = g.FS;
    const R H = R(g.H_moi[pos]);
    const R FSp = R(FS[pos]);
    const R c = 18 * log(12 * H / R(p.Ks));
    const R Uf = sqrt(R(p.g)) * fabs(vth) / c;
    const R fq = 1 - FSp;
    const R wsm = R(p.wss) * ((fq * fq) * (fq * fq));  // wss (1 - FS)^4
    R Zf = 0;
    R S;
    if (FS[pos] > 0.00001) Zf = wsm / (R(0.4) * (Uf + 2 * wsm));
    if (p.ketdinh) S = source_chs<R>(p, wsm, Zf, FSp, R(g.Fw[pos]), vth, H);
    else S = source_nchs<R>(p, wsm, Zf, Uf, H, FSp);
    if (t < p.bed_change_start) S = 0;
    rowCr<R>(g, 0)[pos] = R(0.98) - R(0.198) * Zf + R(0.032) * Zf * Zf;
    rowCr<R>(g, 1)[pos] = S / H;
}

// Find_VTH (Sediment_Transport.cu:541-568) and hesoK (508-539) for cell (i, j), in the
// arithmetic type R; FSI: also the FSi terms of the cell when it is wet.
template <int FSI, class R>
__device__ __forceinline__ void vth_cell(const DevGrid& g, const DevParams& p, int i, int j) {
    const int N = g.N, M = g.M, P = g.P;
    if (i > N || j > M) return;
    const int pos = i * P + j;
    if (i >= 2 && j >= 2) {
        R vth = 0;
        if ((g.htaiz[pos] > p.NANGDAY) && (g.H_moi[pos] > p.H_TINH)) {
            const R ut = (R(g.t_u[pos]) + R(g.t_u[pos - P])) * R(0.5);
            const R vt = (R(g.t_v[pos]) + R(g.t_v[pos - 1])) * R(0.5);
            vth = sqrt(ut * ut + vt * vt);
        }
        g.VTH[pos] = vth;
        if (FSI && i >= 3 && i < N && j <= M && g.khouot[pos] == 0) fsi_cell_terms<R>(g, p, pos, vth, g.clock[1]);
    }
    const R sg = sqrt(R(p.g));
    if (g.Htdu[pos] > 0 && pos >= 1) {
        const R Cz = 18 * log(12 * R(g.Htdu[pos]) / R(p.Ks));
        const R kx = R(5.93) * sg * (R(g.h[pos - 1]) + R(g.h[pos])) * R(0.25) * fabs(R(g.t_u[pos])) / Cz;
        g.Kx[pos] = rmin(R(100.0), rmax(R(5.0), kx));
    }
    if (g.Htdv[pos] > 0 && pos >= P) {
        const R Cz = 18 * log(12 * R(g.Htdv[pos]) / R(p.Ks));
        const R ky = R(5.93) * sg * (R(g.h[pos - P]) + R(g.h[pos])) * R(0.25) * fabs(R(g.t_v[pos])) / Cz;
        g.Ky[pos] = rmin(R(100.0), rmax(R(5.0), ky));
    }
}

template <int FSI, class R>
__global__ void k_vth_hesok(DevGrid g, DevParams p) {
    vth_cell<FSI, R>(g, p, blockIdx.y * blockDim.y + threadIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

template <int FSI, class R>
__global__ void k_vth_span(DevGrid g, DevParams p) {
    const RowLane rl(g, 0, blockIdx.x);
    const int i = rl.i;
    if (i > g.N) return;
    for (int j = g.elo[i] + rl.off; j <= g.ehi[i]; j += rl.stride) vth_cell<FSI, R>(g, p, i, j);
}

// post_cell (with the state update) followed by vth_cell, for one cell of the extended
// spans, with every load of the cell issued before its first store: the stores to z, u,
// v, Htdu and Htdv would otherwise keep the compiler from hoisting the later loads (the
// arrays may alias for all it knows), and a cell would take three memory round trips
// instead of one.  Row and column 0 take the two calls as they are.  The values, and
// the order of their operations, are those of the two calls.
template <int VTH, int FSI, class R>
__device__ __forceinline__ void post_vth_cell(const DevGrid& g, const DevParams& p, int i, int j) {
    const int N = g.N, M = g.M, P = g.P;
    if (i > N || j > M) return;
    if (i < 1 || j < 1) {
        post_cell(g, 1, i, j);
        if (VTH) vth_cell<FSI, R>(g, p, i, j);
        return;
    }
    const int gp = i * P + j;
    const double tz = g.t_z[gp], tu = g.t_u[gp], tv = g.t_v[gp];
    const double z_ip = i + 1 <= N ? g.t_z[gp + P] : g.z[gp + P];
    const double z_jp = j + 1 <= M ? g.t_z[gp + 1] : g.z[gp + 1];
    const double hw = g.h[gp - 1], hc = g.h[gp], hs = g.h[gp - P];
    double htz = 0.0, Hm = 0.0, tu_s = 0.0, tv_w = 0.0;
    int kh = 1;
    if (VTH) {
        htz = g.htaiz[gp];
        Hm = g.H_moi[gp];
        tu_s = g.t_u[gp - P];
        tv_w = g.t_v[gp - 1];
        if (FSI) kh = g.khouot[gp];
    }
    g.z[gp] = tz;
    g.u[gp] = tu;
    g.v[gp] = tv;
    const double htdu = (hw + hc + z_ip + tz) * 0.5;
    const double htdv = (hs + hc + z_jp + tz) * 0.5;
    g.Htdu[gp] = htdu;
    g.Htdv[gp] = htdv;
    if (!VTH) return;
    if (i >= 2 && j >= 2) {
        R vth = 0;
        if ((htz > p.NANGDAY) && (Hm > p.H_TINH)) {
            const R ut = (R(tu) + R(tu_s)) * R(0.5);
            const R vt = (R(tv) + R(tv_w)) * R(0.5);
            vth = sqrt(ut * ut + vt * vt);
        }
        g.VTH[gp] = vth;
        if (FSI && i >= 3 && i < N && kh == 0) fsi_cell_terms<R>(g, p, gp, vth, g.clock[1]);
    }
    const R sg = sqrt(R(p.g));
    if (htdu > 0) {
        const R Cz = 18 * log(12 * R(htdu) / R(p.Ks));
        const R kx = R(5.93) * sg * (R(hw) + R(hc)) * R(0.25) * fabs(R(tu)) / Cz;
        g.Kx[gp] = rmin(R(100.0), rmax(R(5.0), kx));
    }
    if (htdv > 0) {
        const R Cz = 18 * log(12 * R(htdv) / R(p.Ks));
        const R ky = R(5.93) * sg * (R(hs) + R(hc)) * R(0.25) * fabs(R(tv)) / Cz;
        g.Ky[gp] = rmin(R(100.0), rmax(R(5.0), ky));
    }
}

// After a half-step's reset, in one launch: the state update (update_uvz + Htuongdoi)
// and, when VTH, Find_VTH + hesoK on the extended spans (nbp CTAs, one warp per row; both
// only read the cell's own new Htdu/Htdv); the rescan of the changed lines of the other
// direction (nbs CTAs); and the edge concentration interpolation (kEdgeParts CTAs,
// reading t_u / t_v where the reference reads u / v after the update).  None of the
// three writes what another reads.
constexpr int kEdgeParts = 8;
template <int ROWS, int VTH, class R>
__device__ __forceinline__ void post_fused_body(const DevGrid& g, const DevParams& p, int nbp, int nbs, int bx,
                                                int gx) {
    extern __shared__ unsigned swords[];
    // CTAs [0, kEdgeParts) the edge interpolation and [kEdgeParts, kEdgeParts + nbs) the
    // rescans (chains of dependent loads, started first so that they run beside the state
    // update), then the nbp state-update CTAs
    const int b = bx;
    if (b < kEdgeParts) {
        fs_edges_part<0>(g, p, b, kEdgeParts);
        return;
    }
    if (b >= kEdgeParts + nbs) {
        const RowLane rl(g, 0, b - kEdgeParts - nbs);
        const int i = rl.i;
        if (i > g.N) return;
        // rows: the second half-step, with the FSi terms
        for (int j = g.elo[i] + rl.off; j <= g.ehi[i]; j += rl.stride) post_vth_cell<VTH, ROWS, R>(g, p, i, j);
        return;
    }
    const int sb = b - kEdgeParts;
    {
        const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int n = *(volatile unsigned*)&g.dctr[ROWS ? 0 : 1];
        const int L = ROWS ? g.M : g.N;
        const int Lines = ROWS ? g.N : g.M;
        const int nwords = (L + 63) / 32 + 1;
        unsigned* words = swords + warp * nwords;
        int* flags = ROWS ? g.dirty_r : g.dirty_c;
        const int* list = ROWS ? g.dlist_r : g.dlist_c;
        for (int k = sb * warps + warp; k < n; k += nbs * warps) {
            const int line = list[k];
            if (lane == 0) flags[line] = 0;
            if (line < 2 || line > Lines) continue;
            const int lo = ROWS ? g.rlo[line] : g.clo[line];
            const int hi = ROWS ? g.rhi[line] : g.chi[line];
            if (ROWS) {
                const WetGlobal wet{g.khouot, line * g.P, 1};
                warp_scan_line(g, wet, lo, hi, L, words, g.daui + line * HYD_SEGL, g.cuoii + line * HYD_SEGL, g.moci + line);
            } else {
                const WetBytes wet{g.colB + (size_t)line * g.LT};
                warp_scan_line(g, wet, lo, hi, L, words, g.dauj + line * HYD_SEGL, g.cuoij + line * HYD_SEGL, g.mocj + line);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the last rescanning CTA empties the list
        __threadfence();
        unsigned* done = &g.dctr[ROWS ? 2 : 3];
        if (atomicAdd(done, 1u) == (unsigned)nbs - 1) {
            g.dctr[ROWS ? 0 : 1] = 0;
            *done = 0;
            __threadfence();
        }
    }
}

template <int ROWS, int VTH, class R>
__global__ void k_post_fused(DevGrid g, DevParams p, int nbp, int nbs) {
    post_fused_body<ROWS, VTH, R>(g, p, nbp, nbs, blockIdx.x, gridDim.x);
}
template <int ROWS, int VTH, class R>
__global__ void k_post_fused_b(BatchRef br) {
    const BatchMember bm(br);
    const int nbp = row_warp_ctas(bm.g, bm.g.N + 1);
    post_fused_body<ROWS, VTH, R>(bm.g, bm.p, nbp, bm.gx - nbp - kEdgeParts, bm.bx, bm.gx);
}

// Update_FS (Sediment_Transport.cu:620-629)
__global__ void k_update_fs(DevGrid g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.N || j > g.M) return;
    g.FS[i * g.P + j] = g.tFS[i * g.P + j];
}

// Update_FS over the extended spans, plus rows 2 and N and column M in full (the edge
// interpolation writes FS there): CTAs [0, nb) take the rows other than 2 and N, the
// last two CTAs rows 2 and N.
__device__ __forceinline__ void update_fs_span_body(const DevGrid& g, int nb, int bx) {
    const int N = g.N, M = g.M, P = g.P;
    if (bx >= nb) {
        const int i = bx == nb ? 2 : N;
        for (int j = 1 + threadIdx.x; j <= M; j += blockDim.x) g.FS[i * P + j] = g.tFS[i * P + j];
        return;
    }
    const RowLane rl(g, 1, bx);
    const int i = rl.i;
    if (i > N || i == 2 || i == N) return;
    const int lo = g.elo[i] > 1 ? g.elo[i] : 1, hi = g.ehi[i] < M ? g.ehi[i] : M;
    for (int j = lo + rl.off; j <= hi; j += rl.stride) g.FS[i * P + j] = g.tFS[i * P + j];
    if (rl.off == 0 && (M < lo || M > hi)) g.FS[i * P + M] = g.tFS[i * P + M];
}

__global__ void k_update_fs_span(DevGrid g, int nb) { update_fs_span_body(g, nb, blockIdx.x); }
__global__ void k_update_fs_span_b(BatchRef br) {
    const BatchMember bm(br);
    update_fs_span_body(bm.g, row_warp_ctas(bm.g, bm.g.N), bm.bx);
}

// Calculate_Qb (Sediment_Transport.cu:341-414): bed-load flux, then the edge copies.
// FB (morphodynamic feedback, no reference counterpart): the flux is evaluated where the
// speed is positive, the formula's evident intent; the reference evaluates it only where
// VTH == 0 (quirk Q3, reproduced with FB = 0), dividing by that zero.
template <int FB>
__global__ void k_qb(DevGrid g, DevParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 2;
    const int N = g.N, M = g.M, P = g.P;
    if (i > N || j > M) return;
    const int pos = i * P + j;
    double Tob, Toee = p.Toe, Tx = 0;
    double qx = 0, qy = 0;
    if ((FB ? g.VTH[pos] > 0 : !g.VTH[pos]) && (g.khouot[pos] == 0)) {
        Tob = p.ro * g.Fw[pos] * (g.VTH[pos] * g.VTH[pos]);
        if (g.H_moi[pos] > p.ghtoe) Toee = p.Toe * (1 + p.hstoe * ((g.H_moi[pos] - p.ghtoe)));
        if (Tob > Toee) Tx = Tob / Toee - 1;
        qx = 0.053 * pow((p.Sx - 1) * p.g, 0.5) * pow(p.dm, 1.5) * pow(Tx, 2.1) * p.dxr_m03 *
             (g.t_u[pos] + g.t_u[pos - P]) * 0.5 / g.VTH[pos];
        qy = 0.053 * pow((p.Sx - 1) * p.g, 0.5) * pow(p.dm, 1.5) * pow(Tx, 2.1) * p.dxr_m03 *
             (g.t_v[pos] + g.t_v[pos - 1]) * 0.5 / g.VTH[pos];
    }
    double *Qbx = g.Qbx, *Qby = g.Qby;
    Qbx[pos] = qx;
    Qby[pos] = qy;
    if (i == 2) {
        Qbx[pos - P] = qx;
        Qby[pos - P] = qy;
    }
    if (i == N) {
        Qbx[pos + P] = qx;
        Qby[pos + P] = qy;
    }
    if (j == 2) {
        Qbx[pos - 1] = qx;
        Qby[pos - 1] = qy;
        if (i == 2) Qbx[1 * P + 1] = qx;
        // every (i, 2) thread writes these two in the reference; the last in launch order is i = N
        if (i == N) {
            Qby[1 * P + 1] = qy;
            Qbx[(N + 1) * P + 1] = qx;
            Qby[(N + 1) * P + 1] = qy;
        }
    }
    if (j == M) {
        Qbx[pos + 1] = qx;
        Qby[pos + 1] = qy;
        if (i == 2) {
            Qbx[1 * P + M + 1] = qx;
            Qby[1 * P + M + 1] = qy;
        }
        if (i == N) {
            Qbx[(N + 1) * P + M + 1] = qx;
            Qby[(N + 1) * P + M + 1] = qy;
        }
    }
}

// BedLoad/_bed_load (Sediment_Transport.cu:630-639, 416-506): Exner increment into dH
// on rows startidx..endidx-1.  FB (morphodynamic feedback, no reference counterpart): the
// increment covers the Exner period times the morphological factor, is added to dH as a
// Kahan sum (dHc) and applied to the bed, h = h0 + dH; the upwind test the reference
// writes as t_u[pos > 0] (quirk Q4, reproduced with FB = 0) reads t_u[pos] > 0.
template <int FB>
__global__ void k_bedload(DevGrid g, DevParams p, int startidx, int endidx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
    const int N = g.N, M = g.M, width = g.P;
    if (i >= endidx || j > M) return;
    if (FB) g.dHinc[i * width + j] = __longlong_as_double(0x7ff8000000000000LL);  // not computed
    int first = 0, last = 0;
    find_seg_v(g, i, j, first, last);
    if (last - first < 2 || j < first || j > last) return;
    const int pos = i * width + j;
    const int* kh = g.khouot;
    const double *Qbx = g.Qbx, *Qby = g.Qby, *FS = g.FS;
    double pp = 0, q = 0;
    if (kh[pos - width] == 1) {
        if (g.t_u[pos] < 0) pp = (-3 * Qbx[pos] + 4 * Qbx[pos + width] - Qbx[pos + 2 * width]) / p.dX2;
    } else {
        if (kh[pos + width] == 1) {
            if (FB ? g.t_u[pos] > 0 : g.t_u[1] != 0)
                pp = (3 * Qbx[pos] - 4 * Qbx[pos - width] + Qbx[pos - 2 * width]) / p.dX2;
        } else
            pp = (Qbx[pos + width] - Qbx[pos - width]) / p.dX2;
    }
    if (kh[pos - 1] == 1) {
        if (g.t_v[pos] < 0) q = (-3 * Qby[pos] + 4 * Qby[pos + 1] - Qby[pos + 2]) / p.dY2;
    } else {
        if (kh[pos + 1] == 1) {
            if (g.t_v[pos] > 0) q = (3 * Qby[pos] - 4 * Qby[pos - 1] + Qby[pos - 2]) / p.dY2;
        } else
            q = (Qby[pos + 1] - Qby[pos - 1]) / p.dY2;
    }
    double tH = pp + q;
    pp = FS[pos + width] - FS[pos];
    if ((kh[pos + 2 * width] == 1 || kh[pos - width] == 1) && (i < N)) pp = 0;
    q = FS[pos] - FS[pos - width];
    if ((i > 2) && (kh[pos - 2 * width] == 1 || kh[pos + width] == 1)) q = 0;
    pp = 1 / p.dXbp * (g.Htdu[pos] * g.Kx[pos] * pp - g.Htdu[pos - width] * g.Kx[pos - width] * q);
    tH = tH + pp;
    pp = FS[pos + 1] - FS[pos];
    if (((last < M) && (kh[pos - 1] == 1 || kh[pos + 2] == 1)) || (last == M && (kh[pos - 1] == 1))) pp = 0;
    q = FS[pos] - FS[pos - 1];
    if (((first > 2) && (kh[pos - 2] == 1 || kh[pos + 1] == 1)) || (first == 2 && kh[pos + 1] == 1)) q = 0;
    pp = 1 / (p.dYbp) * (g.Htdv[pos] * g.Ky[pos] * pp - g.Htdv[pos - 1] * g.Ky[pos - 1] * q);
    tH = tH + pp;
    const double c = 18 * log(12 * g.H_moi[pos] / p.Ks);
    const double Uf = sqrt(p.g) * fabs(g.VTH[pos]) / c;
    const double fq = 1 - FS[pos];
    const double wsm = p.wss * ((fq * fq) * (fq * fq));  // wss (1 - FS)^4
    double Zf = 0, S = 0;
    if (FS[pos] > 0.0) Zf = wsm / (0.4 * (Uf + 2 * wsm));
    if (p.ketdinh) S = source_chs(p, wsm, Zf, FS[pos], g.Fw[pos], g.VTH[pos], g.H_moi[pos]);
    else S = source_nchs(p, wsm, Zf, Uf, g.H_moi[pos], FS[pos]);
    if (!FB) {
        g.dH[pos] += p.dT / (1 - p.Dorong) * (S + tH);
        return;
    }
    // the period's raw change, filtered and applied by k_bed_apply
    double x = p.morfac * p.bed_period / (1 - p.Dorong) * (S + tH);
    if (!isfinite(x)) x = 0.0;
    g.dHinc[pos] = x;
}

// The fed-back bed change of one update.  The explicit Exner rate from central bed-load and
// diffusion differences carries a grid-scale (2 dx) oscillation, which a morphological step
// of many minutes turns into a checkerboard bed that the hydraulics do not survive; so the
// raw change is filtered by the 3 x 3 binomial kernel (weights 1 2 1 x 1 2 1, renormalised
// over the computed neighbours in rows startidx..endidx-1, columns 2..M), which removes the
// 2 dx mode exactly and keeps smooth changes, then limited to kBedLimit of the water depth
// and kBedCap metres (the step stays small against the depth it acts on), added to dH as a
// Kahan sum and applied to the bed, h = h0 + dH.  Cells within bed_fixed cells of the
// grid's edges (the inlet and outlet sections of the open boundaries) and cells with less
// than bed_min_depth of water (a threshold depth for the bed change, as morphodynamic
// models keep: the banks' wet/dry fringe would otherwise break into patches) keep their
// bed.  Indexing as k_bedload.
__global__ void k_bed_apply(DevGrid g, DevParams p, int startidx, int endidx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
    const int N = g.N, M = g.M, width = g.P;
    if (i >= endidx || j > M) return;
    const int F = p.bed_fixed;
    if (i < 2 + F || i > N - F || j < 2 + F || j > M - F) return;
    if (g.H_moi[i * width + j] < p.bed_min_depth) return;
    const int pos = i * width + j;
    const double* __restrict__ inc = g.dHinc;
    if (!isfinite(inc[pos])) return;
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
    const double lim = fmin(kBedLimit * g.H_moi[pos], kBedCap);
    x = fmin(fmax(x, -lim), lim);
    const double y = x - g.dHc[pos];
    const double sum = g.dH[pos] + y;
    g.dHc[pos] = (sum - g.dH[pos]) - y;
    g.dH[pos] = sum;
    g.h[pos] = g.h0[pos] + sum;
}

// After a fed-back bed change: what the set-up derived from h, re-derived for the new bed
// (Onetime_init, support_funcs.cu:20-58: htaiz, htaiz_bd, Kx1, Ky1; update_h_moi 60-73 on
// the wet cells; Htuongdoi 338-354), and the water the bed moved into or out of the wet
// interior cells' depths added to the budget.  Indexing as k_onetime_init.
__global__ void k_bed_derive(DevGrid g, DevParams p) {
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = blockIdx.y * blockDim.y + threadIdx.y;
    const int N = g.N, M = g.M, P = g.P;
    const int i = i0 + 1, j = j0 + 1;
    double dv = 0.0;
    if (i <= N && j <= M) {
        const double* h = g.h;
        const int pos = i * P + j;
        const double ht = (h[(i - 1) * P + j - 1] + h[(i - 1) * P + j] + h[pos - 1] + h[pos]) * 0.25;
        const double old = g.htaiz[pos];
        g.htaiz[pos] = ht;
        g.htaiz_bd[pos] = ht;
        // the set-up's formula; a face depth below datum that is not positive (a raised bed),
        // where its pow has no real value, is taken as H_TINH.  Clamping every face depth to
        // H_TINH instead would change the friction of the shallow faces that the set-up gave
        // a depth between 0 and H_TINH at the first update, unbalancing the flow there.
        if (h[pos - 1] + h[pos] != 0) {
            const double d = (h[pos - 1] + h[pos]) * 0.5;
            g.Kx1[pos] = p.g * pow(d > 0 ? d : p.H_TINH, -2 * p.mu_mn) * pow((g.hsnham[pos - 1] + g.hsnham[pos]) * 0.5, 2);
        }
        if (h[pos - P] + h[pos] != 0) {
            const double d = (h[pos - P] + h[pos]) * 0.5;
            g.Ky1[pos] = p.g * pow(d > 0 ? d : p.H_TINH, -2 * p.mu_mn) * pow((g.hsnham[pos - P] + g.hsnham[pos]) * 0.5, 2);
        }
        if (g.khouot[pos] == 0) {
            g.H_moi[pos] = ht + g.z[pos];
            if (i >= 2 && j >= 2) dv = ht - old;
        }
        post_cell(g, 0, i, j);
    }
    for (int o = 16; o > 0; o >>= 1) dv += __shfl_down_sync(0xffffffffu, dv, o);
    if ((threadIdx.x & 31) == 0 && dv != 0.0) atomicAdd(&g.budget[kBudBed], dv);
}

// ------------------------------------------------------- quasi-steady support

// hyd_add_levels, pass 1: the increments of cell (i0 + r, j0 + c) (element r ld + c of each
// array) added to z, u, v and their swept copies on the wet interior cells, H_moi = htaiz +
// z (update_h_moi, support_funcs.cu:60-73); a cell whose new depth would not exceed H_TINH
// keeps its level.  The water added goes to the budget's kBudJump slot (depth units).
__global__ void k_add_levels(DevGrid g, DevParams p, const float* __restrict__ du, const float* __restrict__ dv,
                             const float* __restrict__ dz, int i0, int j0, int rows, int cols, long long ld) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    double dvol = 0.0;
    const int i = i0 + r, j = j0 + c;
    if (r < rows && c < cols && i >= 2 && i <= g.N && j >= 2 && j <= g.M) {
        const int pos = i * g.P + j;
        const long long q = (long long)r * ld + c;
        if (g.khouot[pos] == 0) {
            const double zn = g.z[pos] + (double)dz[q];
            if (g.htaiz[pos] + zn > p.H_TINH) {
                dvol = zn - g.z[pos];
                g.z[pos] = zn;
                g.t_z[pos] = zn;
                g.H_moi[pos] = g.htaiz[pos] + zn;
            }
            const double un = g.u[pos] + (double)du[q], vn = g.v[pos] + (double)dv[q];
            g.u[pos] = un;
            g.t_u[pos] = un;
            g.v[pos] = vn;
            g.t_v[pos] = vn;
        }
    }
    for (int o = 16; o > 0; o >>= 1) dvol += __shfl_down_sync(0xffffffffu, dvol, o);
    if ((threadIdx.x & 31) == 0 && dvol != 0.0) atomicAdd(&g.budget[kBudJump], dvol);
}

// hyd_add_levels, pass 2: Htuongdoi (support_funcs.cu:338-354) over the rectangle grown by
// one cell, for the new levels.
__global__ void k_add_levels_faces(DevGrid g, int i0, int j0, int rows, int cols) {
    const int i = i0 - 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int j = j0 - 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 1 || j < 1 || i > i0 + rows || j > j0 + cols) return;
    post_cell(g, 0, i, j);
}

// hyd_steady_residual: sums over the wet cells of 2..N x 2..M of (u - u0)^2 + (v - v0)^2,
// u^2 + v^2, (z - z0)^2 and H_moi^2, per CTA; with snapshot, the cell's u, v, z are copied
// to u0, v0, z0 after they are read.
__global__ void k_resid_partial(DevGrid g, double* __restrict__ u0, double* __restrict__ v0, double* __restrict__ z0,
                                int snapshot, double* __restrict__ part) {
    __shared__ double sh[4][256];
    const int tid = threadIdx.x;
    double a = 0, b = 0, c = 0, d = 0;
    const int W = g.M - 1;
    const long long ncell = (long long)(g.N - 1) * W;
    for (long long q = (long long)blockIdx.x * blockDim.x + tid; q < ncell; q += (long long)gridDim.x * blockDim.x) {
        const int i = 2 + (int)(q / W), j = 2 + (int)(q % W);
        const int gp = i * g.P + j;
        if (g.khouot[gp] != 0) continue;
        const double u = g.u[gp], v = g.v[gp], z = g.z[gp], H = g.H_moi[gp];
        const double du = u - u0[gp], dv = v - v0[gp], dz = z - z0[gp];
        a += du * du + dv * dv;
        b += u * u + v * v;
        c += dz * dz;
        d += H * H;
        if (snapshot) {
            u0[gp] = u;
            v0[gp] = v;
            z0[gp] = z;
        }
    }
    sh[0][tid] = a;
    sh[1][tid] = b;
    sh[2][tid] = c;
    sh[3][tid] = d;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (tid < w)
            for (int k = 0; k < 4; k++) sh[k][tid] += sh[k][tid + w];
        __syncthreads();
    }
    if (tid == 0)
        for (int k = 0; k < 4; k++) part[blockIdx.x * 4 + k] = sh[k][0];
}

__global__ void k_resid_final(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double acc[4] = {0, 0, 0, 0};
    for (int b = 0; b < nblocks; b++)
        for (int k = 0; k < 4; k++) acc[k] += part[b * 4 + k];
    for (int k = 0; k < 4; k++) out[k] = acc[k];
}

// Feedback set-up: h0 = h - dH (so that h = h0 + dH holds now), no compensation yet.
__global__ void k_bed_reset(DevGrid g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.N + 3 || j >= g.M + 3) return;
    const int pos = i * g.P + j;
    g.h0[pos] = g.h[pos] - g.dH[pos];
    g.dHc[pos] = 0.0;
}

}  // namespace

// Pitched (N+3) x pitch rows into a packed (N+3) x (M+3) array (a field snapshot for an
// asynchronous host read).
__global__ void k_pack_rows(const double* __restrict__ src, int pitch, double* __restrict__ dst, int rows,
                            int cols) {
    const long long n = (long long)rows * cols;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q / cols), c = (int)(q - (long long)r * cols);
        dst[q] = src[(long long)r * pitch + c];
    }
}

// ------------------------------------------------------------------ host wrappers

namespace {
constexpr int kScanThreads = 256;
size_t scan_smem(const DevGrid& g) {
    const int L = g.N > g.M ? g.N : g.M;
    return sizeof(unsigned) * (kScanThreads / 32) * ((L + 63) / 32 + 1);
}
// dynamic shared memory of k_reset: the line's mask bytes and two bitsets / scan words
size_t reset_smem(int L) { return ((L + 3 + 15) & ~15) + 3 * sizeof(unsigned) * reset_words(L); }
int scan_grid() {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm < 1) nsm = 1;
    }
    return nsm;
}
void scan_dirty(const DevGrid& g, const DevParams& p, int rows, int with_edges, cudaStream_t s) {
    const int nb = scan_grid();
    const int edges = with_edges ? nb : -1;
    if (rows) k_scan_dirty<1><<<nb + (with_edges ? 1 : 0), kScanThreads, scan_smem(g), s>>>(g, p, edges);
    else k_scan_dirty<0><<<nb + (with_edges ? 1 : 0), kScanThreads, scan_smem(g), s>>>(g, p, edges);
}
}  // namespace

// Allow `f` `bytes` of dynamic shared memory on the current device.
cudaError_t allow_smem(const void* f, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Opt the kernels that stage a line in shared memory into the dynamic shared memory
// this grid needs.
cudaError_t grid_setup(int N, int M) {
    DevGrid g{};
    g.N = N;
    g.M = M;
    cudaError_t e;
    if ((e = allow_smem((const void*)k_scan_dirty<1>, scan_smem(g))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_scan_dirty<0>, scan_smem(g))) != cudaSuccess) return e;
    const void* fused[] = {(const void*)k_post_fused<0, 0, double>, (const void*)k_post_fused<0, 1, double>,
                           (const void*)k_post_fused<1, 0, double>, (const void*)k_post_fused<1, 1, double>,
                           (const void*)k_post_fused<0, 0, float>,  (const void*)k_post_fused<0, 1, float>,
                           (const void*)k_post_fused<1, 0, float>,  (const void*)k_post_fused<1, 1, float>};
    for (const void* f : fused)
        if ((e = allow_smem(f, scan_smem(g))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_u<double>, sizeof(double) * (N + 3))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_v<double>, sizeof(double) * (M + 3))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_u<float>, sizeof(double) * (N + 3))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_v<float>, sizeof(double) * (M + 3))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_reset<1>, reset_smem(M))) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_reset<0>, reset_smem(N))) != cudaSuccess) return e;
    return cudaSuccess;
}

// Spans of the never-dry-forever cells of every line, from the current mask.
void launch_spans(const DevGrid& g, cudaStream_t s) {
    cudaMemsetAsync(g.rlo, 0x7f, sizeof(int) * (g.N + 3), s);
    cudaMemsetAsync(g.rhi, 0xff, sizeof(int) * (g.N + 3), s);
    cudaMemsetAsync(g.clo, 0x7f, sizeof(int) * (g.M + 3), s);
    cudaMemsetAsync(g.chi, 0xff, sizeof(int) * (g.M + 3), s);
    cudaMemsetAsync(g.span_wide, 0, sizeof(int), s);
    const dim3 b(32, 8);
    k_spans<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g);
    k_ext_spans<<<(g.N + 3 + 127) / 128, 128, 0, s>>>(g, kSpanHalo);
    k_reset_bytes_init<<<grid2d(g.N + 3, g.M + 3, b), b, 0, s>>>(g);
    hyd_kernel_launches_add(3);
}

void launch_widen_spans(const DevGrid& g, cudaStream_t s) {
    k_widen_spans<<<(g.N + 3 + 127) / 128, 128, 0, s>>>(g);
    hyd_kernel_launches_add(1);
}

int outside_differs(const DevGrid& g, const double* a, const double* b, int i0, int i1, int j0, int j1, int* dflag,
                    cudaStream_t s) {
    int h = 0;
    if (cudaMemsetAsync(dflag, 0, sizeof(int), s) != cudaSuccess) return -1;
    const dim3 bl(32, 8);
    k_outside_diff<<<grid2d(j1 - j0 + 1, i1 - i0 + 1, bl), bl, 0, s>>>(g, a, b, i0, i1, j0, j1, dflag);
    hyd_kernel_launches_add(1);
    if (cudaMemcpyAsync(&h, dflag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    return h;
}

// Empty the rescan lists.
void clear_rescan_lists(const DevGrid& g, cudaStream_t s) {
    cudaMemsetAsync(g.dirty_r, 0, sizeof(int) * (g.N + 3), s);
    cudaMemsetAsync(g.dirty_c, 0, sizeof(int) * (g.M + 3), s);
    cudaMemsetAsync(g.dctr, 0, 5 * sizeof(unsigned), s);
}

// List every column for the rescan after the next row resets.
void launch_mark_all_cols(const DevGrid& g, cudaStream_t s) {
    k_mark_all<0><<<(g.M + 3 + 255) / 256, 256, 0, s>>>(g);
    hyd_kernel_launches_add(1);
}

// keep_mask: when not null, a saved mask (pitched like khouot) copied over the one
// Onetime_init derives, before the scans (the pick-up order of rep.py:126-131).
void launch_init_kernels(const DevGrid& g, const DevParams& p, const int* keep_mask, cudaStream_t s) {
    const dim3 b(32, 8);
    k_onetime_init<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p);
    hyd_kernel_launches_add(1);
    if (keep_mask)
        cudaMemcpyAsync(g.khouot, keep_mask, sizeof(int) * (size_t)(g.N + 3) * g.P, cudaMemcpyDeviceToDevice, s);
    launch_spans(g, s);
    clear_rescan_lists(g, s);
    k_mark_all<1><<<(g.N + 3 + 255) / 256, 256, 0, s>>>(g);
    k_mark_all<0><<<(g.M + 3 + 255) / 256, 256, 0, s>>>(g);
    scan_dirty(g, p, 1, 1, s);
    scan_dirty(g, p, 0, 0, s);
    k_post<<<grid2d(g.M + 1, g.N + 1, b), b, 0, s>>>(g, 0);
    k_preprocess<<<1, 32, 0, s>>>(g, p);
    hyd_kernel_launches_add(6);
}


void launch_coef_bnd(const DevGrid& g, const DevParams& p, int half, int writes, cudaStream_t s) {
    // the tiled form: kTileRows rows per CTA; the row form: one warp per row (the same count)
    const int nb = ((g.N - 1) * 32 + 255) / 256 + 1;
    const int nbr = nb;
    if (p.mixed) {
        if (half == 1) k_coef_bnd<1, 0, float><<<nbr, 256, 0, s>>>(g, p, writes);
        else if (g.tile_cols) k_coef_bnd<0, 1, float><<<nb, 256, 0, s>>>(g, p, writes);
        else k_coef_bnd<0, 0, float><<<nbr, 256, 0, s>>>(g, p, writes);
    } else {
        if (half == 1) k_coef_bnd<1, 0, double><<<nbr, 256, 0, s>>>(g, p, writes);
        else if (g.tile_cols) k_coef_bnd<0, 1, double><<<nb, 256, 0, s>>>(g, p, writes);
        else k_coef_bnd<0, 0, double><<<nbr, 256, 0, s>>>(g, p, writes);
    }
    hyd_kernel_launches_add(1);
}

// Elementwise kernels: the whole grid (`full`), or one warp per row over its extended span.
static int row_warps_blocks(const DevGrid& g, int rows) { return row_warp_ctas(g, rows); }

void launch_smooth(const DevGrid& g, const DevParams& p, int isU, double* out, int full, int bytes, int fs_bnd,
                   int budget, cudaStream_t s) {
    const dim3 b(32, 8);
    if (full) {  // callers pass fs_bnd = 0 with full passes
        if (bytes) k_smooth<1><<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p, isU, out);
        else k_smooth<0><<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p, isU, out);
        if (budget) {  // the smoothing reads the swept velocity and writes elsewhere
            k_edge_budget<<<kBudCtas, 256, 0, s>>>(g, p, isU);
            k_leak_full<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p, isU);
            hyd_kernel_launches_add(2);
        }
    } else {
        const int nb = row_warps_blocks(g, g.N + 3);
        if (bytes && fs_bnd) k_smooth_span<1, 1, 0><<<nb + 1, 256, 0, s>>>(g, p, isU, out);
        else if (bytes) k_smooth_span<1, 0, 0><<<nb, 256, 0, s>>>(g, p, isU, out);
        else if (budget) k_smooth_span<0, 0, 1><<<nb + kBudCtas, 256, 0, s>>>(g, p, isU, out);
        else k_smooth_span<0, 0, 0><<<nb, 256, 0, s>>>(g, p, isU, out);
    }
    hyd_kernel_launches_add(1);
}

void launch_budget_half(const DevGrid& g, const DevParams& p, int isU, cudaStream_t s) {
    const int n = isU ? g.M - 1 : g.N - 1;
    k_budget_half<<<kBudCtas + (2 * n + 255) / 256, 256, 0, s>>>(g, p, isU);
    hyd_kernel_launches_add(1);
}

// The line kernels below take `threads` per CTA (a multiple of 32, at least 64), chosen
// by the caller from the longest span of the direction.
void launch_explicit_v(const DevGrid& g, const DevParams& p, int threads, cudaStream_t s) {
    if (p.mixed) k_explicit_v<float><<<g.N - 1, threads, sizeof(double) * g.sv_cap, s>>>(g, p);
    else k_explicit_v<double><<<g.N - 1, threads, sizeof(double) * g.sv_cap, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_coef_eu(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    const int nb = ((g.N - 2) * 32 + 255) / 256;
    if (p.mixed) {
        if (g.tile_cols) k_coef_eu<1, float><<<nb, 256, 0, s>>>(g, p);
        else k_coef_eu<0, float><<<nb, 256, 0, s>>>(g, p);
    } else {
        if (g.tile_cols) k_coef_eu<1, double><<<nb, 256, 0, s>>>(g, p);
        else k_coef_eu<0, double><<<nb, 256, 0, s>>>(g, p);
    }
    hyd_kernel_launches_add(1);
}

void launch_explicit_u(const DevGrid& g, const DevParams& p, int threads, cudaStream_t s) {
    if (p.mixed) k_explicit_u<float><<<g.M - 1, threads, sizeof(double) * g.su_cap, s>>>(g, p);
    else k_explicit_u<double><<<g.M - 1, threads, sizeof(double) * g.su_cap, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_reset_rows(const DevGrid& g, const DevParams& p, int force, int threads, cudaStream_t s) {
    k_reset<1><<<g.N, threads, reset_smem(g.M), s>>>(g, p, force);
    hyd_kernel_launches_add(1);
}

void launch_reset_cols(const DevGrid& g, const DevParams& p, int force, int threads, cudaStream_t s) {
    k_reset<0><<<g.M, threads, reset_smem(g.N), s>>>(g, p, force);
    hyd_kernel_launches_add(1);
}

void launch_post(const DevGrid& g, const DevParams& p, int full, cudaStream_t s) {
    const dim3 b(32, 8);
    if (full) k_post<<<grid2d(g.M + 1, g.N + 1, b), b, 0, s>>>(g, 1);
    else k_post_span<<<row_warps_blocks(g, g.N + 1), 256, 0, s>>>(g);
    hyd_kernel_launches_add(1);
}

// After the row resets the changed columns are rescanned (and vice versa); the same
// launch carries the edge concentration interpolation.
void launch_scan_cols(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    scan_dirty(g, p, 0, 1, s);
    hyd_kernel_launches_add(1);
}

void launch_scan_rows(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    scan_dirty(g, p, 1, 1, s);
    hyd_kernel_launches_add(1);
}

// The fused update / rescan / interpolation launch (k_post_fused); rows: which direction
// is rescanned.
void launch_post_fused(const DevGrid& g, const DevParams& p, int rows, int vth, cudaStream_t s) {
    const int nbp = row_warps_blocks(g, g.N + 1), nbs = 32;
    const int grid = nbp + nbs + kEdgeParts;
    const size_t sm = scan_smem(g);
    if (!vth) {  // no sediment terms: the FP64 kernel in both forms
        if (rows) k_post_fused<1, 0, double><<<grid, 256, sm, s>>>(g, p, nbp, nbs);
        else k_post_fused<0, 0, double><<<grid, 256, sm, s>>>(g, p, nbp, nbs);
    } else if (p.mixed) {
        if (rows) k_post_fused<1, 1, float><<<grid, 256, sm, s>>>(g, p, nbp, nbs);
        else k_post_fused<0, 1, float><<<grid, 256, sm, s>>>(g, p, nbp, nbs);
    } else {
        if (rows) k_post_fused<1, 1, double><<<grid, 256, sm, s>>>(g, p, nbp, nbs);
        else k_post_fused<0, 1, double><<<grid, 256, sm, s>>>(g, p, nbp, nbs);
    }
    hyd_kernel_launches_add(1);
}

void launch_vth_hesok(const DevGrid& g, const DevParams& p, int full, int fsi, cudaStream_t s) {
    const dim3 b(32, 8);
    if (full) {
        const dim3 gr = grid2d(g.M + 1, g.N + 1, b);
        if (p.mixed) {
            if (fsi) k_vth_hesok<1, float><<<gr, b, 0, s>>>(g, p);
            else k_vth_hesok<0, float><<<gr, b, 0, s>>>(g, p);
        } else {
            if (fsi) k_vth_hesok<1, double><<<gr, b, 0, s>>>(g, p);
            else k_vth_hesok<0, double><<<gr, b, 0, s>>>(g, p);
        }
    } else {
        const int nb = row_warps_blocks(g, g.N + 1);
        if (p.mixed) {
            if (fsi) k_vth_span<1, float><<<nb, 256, 0, s>>>(g, p);
            else k_vth_span<0, float><<<nb, 256, 0, s>>>(g, p);
        } else {
            if (fsi) k_vth_span<1, double><<<nb, 256, 0, s>>>(g, p);
            else k_vth_span<0, double><<<nb, 256, 0, s>>>(g, p);
        }
    }
    hyd_kernel_launches_add(1);
}

void launch_update_fs(const DevGrid& g, int full, cudaStream_t s) {
    const dim3 b(32, 8);
    if (full) k_update_fs<<<grid2d(g.M, g.N, b), b, 0, s>>>(g);
    else {
        const int nb = row_warps_blocks(g, g.N);
        k_update_fs_span<<<nb + 2, 256, 0, s>>>(g, nb);
    }
    hyd_kernel_launches_add(1);
}

void launch_bed(const DevGrid& g, const DevParams& p, int startidx, int endidx, cudaStream_t s) {
    const dim3 b(32, 8);
    if (!p.bed_feedback) {
        k_qb<0><<<grid2d(g.M - 1, g.N - 1, b), b, 0, s>>>(g, p);
        if (endidx > startidx) k_bedload<0><<<grid2d(g.M - 1, endidx - startidx, b), b, 0, s>>>(g, p, startidx, endidx);
        hyd_kernel_launches_add(2);
        return;
    }
    k_qb<1><<<grid2d(g.M - 1, g.N - 1, b), b, 0, s>>>(g, p);
    if (endidx > startidx) {
        k_bedload<1><<<grid2d(g.M - 1, endidx - startidx, b), b, 0, s>>>(g, p, startidx, endidx);
        k_bed_apply<<<grid2d(g.M - 1, endidx - startidx, b), b, 0, s>>>(g, p, startidx, endidx);
        hyd_kernel_launches_add(2);
    }
    k_bed_derive<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p);
    k_preprocess<<<1, 32, 0, s>>>(g, p);
    hyd_kernel_launches_add(3);
}

void launch_bed_reset(const DevGrid& g, cudaStream_t s) {
    const dim3 b(32, 8);
    k_bed_reset<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g);
    hyd_kernel_launches_add(1);
}

void launch_add_levels(const DevGrid& g, const DevParams& p, const float* du, const float* dv, const float* dz,
                       int i0, int j0, int rows, int cols, long long ld, cudaStream_t s) {
    const dim3 b(32, 8);
    k_add_levels<<<grid2d(cols, rows, b), b, 0, s>>>(g, p, du, dv, dz, i0, j0, rows, cols, ld);
    k_add_levels_faces<<<grid2d(cols + 2, rows + 2, b), b, 0, s>>>(g, i0, j0, rows, cols);
    hyd_kernel_launches_add(2);
}

void launch_steady_residual(const DevGrid& g, double* u0, double* v0, double* z0, int snapshot, double* part,
                            int nblocks, double* out, cudaStream_t s) {
    k_resid_partial<<<nblocks, 256, 0, s>>>(g, u0, v0, z0, snapshot, part);
    k_resid_final<<<1, 32, 0, s>>>(part, nblocks, out);
    hyd_kernel_launches_add(2);
}

// Up to kPutDoubles values carried in the launch's parameters into dst[0..n): a small
// upload in order with the stream's kernels that takes no copy engine (those may be busy
// with a device-to-host copy of an earlier step).
struct PutDoubles {
    double v[kPutDoubles];
};
__global__ void k_put_doubles(double* __restrict__ dst, int n, PutDoubles pl) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = pl.v[i];
}

int launch_put_doubles(double* dst, const double* src, int n, cudaStream_t s) {
    if (n < 0 || n > kPutDoubles) return 0;
    PutDoubles pl;
    memcpy(pl.v, src, sizeof(double) * n);
    k_put_doubles<<<1, 256, 0, s>>>(dst, n, pl);
    hyd_kernel_launches_add(1);
    return 1;
}

void launch_pack_rows(const double* src, int pitch, double* dst, int rows, int cols, cudaStream_t s) {
    k_pack_rows<<<4 * 148, 256, 0, s>>>(src, pitch, dst, rows, cols);
    hyd_kernel_launches_add(1);
}

// ------------------------------------------------------------- batched launches
// One launch for every member of a batch: `ctas` CTAs, member m's share starting at
// br.bstart[m] (the CTAs its own launch would have), each CTA working for one member.

void launch_coef_bnd_batch(const BatchRef& br, int ctas, int half, int writes, int mixed, cudaStream_t s) {
    if (mixed) {
        if (half == 1) k_coef_bnd_b<1, 0, float><<<ctas, 256, 0, s>>>(br, writes);
        else k_coef_bnd_b<0, 0, float><<<ctas, 256, 0, s>>>(br, writes);
    } else {
        if (half == 1) k_coef_bnd_b<1, 0, double><<<ctas, 256, 0, s>>>(br, writes);
        else k_coef_bnd_b<0, 0, double><<<ctas, 256, 0, s>>>(br, writes);
    }
    hyd_kernel_launches_add(1);
}

void launch_smooth_batch(const BatchRef& br, int ctas, int isU, double* const* outs, int bytes, int fs_bnd, int budget,
                         cudaStream_t s) {
    if (bytes && fs_bnd) k_smooth_span_b<1, 1, 0><<<ctas, 256, 0, s>>>(br, isU, outs);
    else if (bytes) k_smooth_span_b<1, 0, 0><<<ctas, 256, 0, s>>>(br, isU, outs);
    else if (budget) k_smooth_span_b<0, 0, 1><<<ctas, 256, 0, s>>>(br, isU, outs);
    else k_smooth_span_b<0, 0, 0><<<ctas, 256, 0, s>>>(br, isU, outs);
    hyd_kernel_launches_add(1);
}

void launch_explicit_v_batch(const BatchRef& br, int ctas, int threads, size_t smem, int mixed, cudaStream_t s) {
    if (mixed) k_explicit_v_b<float><<<ctas, threads, smem, s>>>(br);
    else k_explicit_v_b<double><<<ctas, threads, smem, s>>>(br);
    hyd_kernel_launches_add(1);
}

void launch_coef_eu_batch(const BatchRef& br, int ctas, int mixed, cudaStream_t s) {
    if (mixed) k_coef_eu_b<0, float><<<ctas, 256, 0, s>>>(br);
    else k_coef_eu_b<0, double><<<ctas, 256, 0, s>>>(br);
    hyd_kernel_launches_add(1);
}

void launch_explicit_u_batch(const BatchRef& br, int ctas, int threads, size_t smem, int mixed, cudaStream_t s) {
    if (mixed) k_explicit_u_b<float><<<ctas, threads, smem, s>>>(br);
    else k_explicit_u_b<double><<<ctas, threads, smem, s>>>(br);
    hyd_kernel_launches_add(1);
}

void launch_reset_batch(const BatchRef& br, int ctas, int rows, int threads, size_t smem, cudaStream_t s) {
    if (rows) k_reset_b<1><<<ctas, threads, smem, s>>>(br, 0);
    else k_reset_b<0><<<ctas, threads, smem, s>>>(br, 0);
    hyd_kernel_launches_add(1);
}

void launch_post_fused_batch(const BatchRef& br, int ctas, int rows, int vth, int mixed, size_t smem, cudaStream_t s) {
    if (!vth) {
        if (rows) k_post_fused_b<1, 0, double><<<ctas, 256, smem, s>>>(br);
        else k_post_fused_b<0, 0, double><<<ctas, 256, smem, s>>>(br);
    } else if (mixed) {
        if (rows) k_post_fused_b<1, 1, float><<<ctas, 256, smem, s>>>(br);
        else k_post_fused_b<0, 1, float><<<ctas, 256, smem, s>>>(br);
    } else {
        if (rows) k_post_fused_b<1, 1, double><<<ctas, 256, smem, s>>>(br);
        else k_post_fused_b<0, 1, double><<<ctas, 256, smem, s>>>(br);
    }
    hyd_kernel_launches_add(1);
}

void launch_update_fs_batch(const BatchRef& br, int ctas, cudaStream_t s) {
    k_update_fs_span_b<<<ctas, 256, 0, s>>>(br);
    hyd_kernel_launches_add(1);
}

// Opt the batched kernels that stage a line in shared memory into `bytes` of it (the
// largest any member needs).
cudaError_t batch_grid_setup(size_t smem_ev, size_t smem_eu, size_t smem_rr, size_t smem_rc, size_t smem_pf) {
    cudaError_t e;
    const void* pf[] = {(const void*)k_post_fused_b<0, 0, double>, (const void*)k_post_fused_b<0, 1, double>,
                        (const void*)k_post_fused_b<1, 0, double>, (const void*)k_post_fused_b<1, 1, double>,
                        (const void*)k_post_fused_b<0, 1, float>, (const void*)k_post_fused_b<1, 1, float>};
    for (const void* f : pf)
        if ((e = allow_smem(f, smem_pf)) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_v_b<double>, smem_ev)) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_v_b<float>, smem_ev)) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_u_b<double>, smem_eu)) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_explicit_u_b<float>, smem_eu)) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_reset_b<1>, smem_rr)) != cudaSuccess) return e;
    if ((e = allow_smem((const void*)k_reset_b<0>, smem_rc)) != cudaSuccess) return e;
    return cudaSuccess;
}

// Shared memory the line kernels of one grid need (k_explicit_v / _u, k_reset rows /
// columns, k_post_fused).
void line_smem(int N, int M, size_t* ev, size_t* eu, size_t* rr, size_t* rc, size_t* pf) {
    DevGrid g{};
    g.N = N;
    g.M = M;
    *ev = sizeof(double) * (M + 3);
    *eu = sizeof(double) * (N + 3);
    *rr = reset_smem(M);
    *rc = reset_smem(N);
    *pf = scan_smem(g);
}
