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

#include "hydist_dev.cuh"

namespace {

constexpr double kPiRef = 3.14159265359;  // constant.cuh:3
constexpr double kEpsRef = 1e-16;         // UVZSolver_multithread.cu:12

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

// --------------------------------------------------------------- boundary values

// Boundary_value + FS_boundary for one edge at index i (support_funcs.cu:544-617)
__device__ void bnd_edge(const DevGrid& g, int i, double t, int isU, int location, int location_ext,
                         const int* btype, const double* hi_e, double* barr, const double* bcv, const double* ccv,
                         double hmax, const int* moc, const int* dau, const int* cuoi) {
    const int P = g.P, tt = g.total_time;
    const int t1 = (int)(t / 3600);
    const double t2 = (t - (3600.0 * t1)) / 3600.0;
    int seg_no = -1;
    if (moc[location] > 0 && dau[location * HYD_SEGL] <= i && i <= cuoi[location * HYD_SEGL]) seg_no = 0;
    if (seg_no == -1) return;
    const double value = bcv[seg_no * tt + t1] * (1.0 - t2) + bcv[seg_no * tt + t1 + 1] * t2;
    if (btype[seg_no] == 2) {
        barr[i] = value * hi_e[i];
    } else if (isU) {
        g.t_z[location * P + i] = value;
        g.t_z[location_ext * P + i] = value;
    } else {
        g.t_z[i * P + location] = value;
        g.t_z[i * P + location_ext] = value;
    }
    if (btype[seg_no] != 2) return;
    const int ii = isU ? location : i, jj = isU ? i : location;
    const double cv = ccv[seg_no * tt + t1] * (1.0 - t2) + ccv[seg_no * tt + t1 + 1] * t2;
    g.FS[ii * P + jj] = cv * g.htaiz_bd[ii * P + jj] * hmax;
}

// Update_Boundary_Value (support_funcs.cu:622-668); edges in the order up, down, left,
// right, each completed before the next (the order a converged warp applies them).
__global__ void k_boundary(DevGrid g, DevParams p, double t) {
    const int N = g.N, M = g.M;
    const int imax = N > M ? N : M;
    const double* hi_up = g.hi;
    const double* hi_down = hi_up + (N + 3);
    const double* hi_left = hi_down + (N + 3);
    const double* hi_right = hi_left + (M + 3);
    for (int e = 0; e < 4; e++) {
        for (int i = 2 + threadIdx.x; i <= imax; i += blockDim.x) {
            if (e == 0)
                bnd_edge(g, i, t, 0, M, M + 1, g.btype + 0 * HYD_SEGL, hi_up, g.vbt, g.bc[0], g.cc[0], g.hmax[0], g.mocj,
                         g.dauj, g.cuoij);
            else if (e == 1)
                bnd_edge(g, i, t, 0, 2, 1, g.btype + 1 * HYD_SEGL, hi_down, g.vbd, g.bc[1], g.cc[1], g.hmax[1], g.mocj,
                         g.dauj, g.cuoij);
            else if (e == 2)
                bnd_edge(g, i, t, 1, 2, 1, g.btype + 2 * HYD_SEGL, hi_left, g.ubt, g.bc[2], g.cc[2], g.hmax[2], g.moci,
                         g.daui, g.cuoii);
            else
                bnd_edge(g, i, t, 1, N, N + 1, g.btype + 3 * HYD_SEGL, hi_right, g.ubp, g.bc[3], g.cc[3], g.hmax[3],
                         g.moci, g.daui, g.cuoii);
        }
        __syncthreads();
    }
}

// Channel-mode analytic seiche boundaries (support_funcs.cu:356-429, Engine.py:30-43).
// Engine.py passes m_offset = 5 as the kernels' segment_limit parameter, so the segment
// tables are read with a stride of 5; bienQ is read through a bool pointer, i.e. byte e
// of the int32 array.  Each edge covers at most N (up/down) or M (left/right) indices,
// the extent of the reference's launch.
__global__ void k_boundary_channel(DevGrid g, DevParams p, double t) {
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

// ------------------------------------------------------------------- smoothing

// Normalize + update_buffer (support_funcs.cu:682-729): out = 5-point smoothed velocity on
// the interior, a copy elsewhere.  isU smooths t_u (neighbours along i, wet check along j).
__global__ void k_smooth(DevGrid g, DevParams p, int isU, double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int N = g.N, M = g.M, P = g.P;
    if (i >= N + 3 || j >= M + 3) return;
    const double* val = isU ? g.t_u : g.t_v;
    const int gp = i * P + j;
    const double v0 = val[gp];
    double r = v0;
    if (!(i > N || j > M || i < 2 || j < 2) && v0 != 0) {
        const int close_d = isU ? P : 1, far_d = isU ? 1 : P;
        int count = 2;
        double nb = val[gp - close_d] + val[gp + close_d];
        if (g.khouot[gp - far_d] == 0) {
            nb += val[gp - far_d];
            count++;
        }
        if (g.khouot[gp + far_d] == 0) {
            nb += val[gp + far_d];
            count++;
        }
        r = v0 * p.heso + (1 - p.heso) * nb / count;
    }
    out[gp] = r;
}

// ----------------------------------------------------------- explicit momentum

// solveV/vSolver (UVZSolver_multithread.cu:1055-1071, 727-768) on row i, then
// update_margin_elem_V (1008-1052) for the same row.
__global__ void k_explicit_v(DevGrid g, DevParams p) {
    const int row = 2 + blockIdx.x;
    const int P = g.P, M = g.M;
    const int nseg = g.moci[row];
    const double *u = g.u, *v = g.v, *z = g.z, *t_u = g.t_u, *H = g.H_moi;
    for (int k = 0; k < nseg; k++) {
        const int first = g.daui[row * HYD_SEGL + k], last = g.cuoii[row * HYD_SEGL + k];
        if (first >= last) continue;
        for (int col = first + threadIdx.x; col < last; col += blockDim.x) {
            const int o = P;
            double pp, q, tmp;
            q = 0;
            pp = 0;
            tmp = 0;
            const double utb = (u[(row - 1) * o + col] + u[row * o + col] + u[(row - 1) * o + col + 1] + u[row * o + col + 1]) * 0.25;
            const double t_utb = (t_u[(row - 1) * o + col] + t_u[row * o + col] + t_u[(row - 1) * o + col + 1] + t_u[row * o + col + 1]) * 0.25;
            pp = (v[row * o + col + 1] - v[row * o + col - 1]) / p.dY2;
            pp = p.HaiChiadT + pp + g.Ky1[row * o + col] * sqrt(utb * utb + v[row * o + col] * v[row * o + col]) / g.Htdv[row * o + col];
            if (H[(row - 1) * o + col] <= p.H_TINH) {
                if (utb < 0) {
                    q = t_utb * (-3 * v[row * o + col] + 4 * v[(row + 1) * o + col] - v[(row + 2) * o + col]) / p.dX2;
                    tmp = (v[row * o + col] - 2 * v[(row + 1) * o + col] + v[(row + 2) * o + col]) / p.dXbp;
                }
            } else {
                if (H[(row + 1) * o + col] <= p.H_TINH) {
                    if ((H[(row - 2) * o + col] > p.H_TINH) && (utb > 0)) {
                        q = t_utb * (3 * v[row * o + col] - 4 * v[(row - 1) * o + col] + v[(row - 2) * o + col]) / p.dX2;
                        tmp = (v[row * o + col] - 2 * v[(row - 1) * o + col] + v[(row - 2) * o + col]) / p.dXbp;
                    }
                } else {
                    q = t_utb * (v[(row + 1) * o + col] - v[(row - 1) * o + col]) / p.dX2;
                    tmp = (v[(row + 1) * o + col] - 2 * v[row * o + col] + v[(row - 1) * o + col]) / p.dXbp;
                }
            }
            q = p.HaiChiadT * v[row * o + col] - q - p.CORIOLIS_FORCE * t_utb;
            q = (q - p.g * (z[row * o + col + 1] - z[row * o + col]) / p.dY +
                 g.VISC[row * o + col] * (tmp + (v[row * o + col + 1] - 2 * v[row * o + col] + v[row * o + col - 1]) / p.dYbp)) +
                (p.windy - g.Tsyw[row * o + col]) / g.Htdv[row * o + col];
            g.t_v[row * o + col] = q / pp;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double* t_v = g.t_v;
        const double* h = g.h;
        const int i = row, W = P;
        for (int k = 0; k < nseg; k++) {
            const int first = g.daui[i * HYD_SEGL + k], last = g.cuoii[i * HYD_SEGL + k];
            const bool b1 = (first > 2) || ((first == 2) && (fabs((h[i * W + first - 1] + h[(i - 1) * W + first - 1]) * 0.5 - p.NANGDAY) < kEpsRef));
            const bool b2 = (last < M) || ((last == M) && (fabs((h[i * W + last] + h[(i - 1) * W + last]) * 0.5 - p.NANGDAY) < kEpsRef));
            if (b1) t_v[i * W + first - 1] = 0;
            else t_v[i * W + first - 1] = 2 * t_v[i * W + first] - t_v[i * W + first + 1];
            if (b2) t_v[i * W + last] = 0;
            else t_v[i * W + last] = 2 * t_v[i * W + last - 1] - t_v[i * W + last - 2];
        }
    }
}

// solveU/uSolver (UVZSolver_multithread.cu:947-968, 773-815) on column j, then
// update_margin_elem_U (970-1006).
__global__ void k_explicit_u(DevGrid g, DevParams p) {
    const int col = 2 + blockIdx.x;
    const int P = g.P, N = g.N;
    const int nseg = g.mocj[col];
    const double *u = g.u, *v = g.v, *z = g.z, *t_v = g.t_v, *H = g.H_moi;
    for (int k = 0; k < nseg; k++) {
        const int first = g.dauj[col * HYD_SEGL + k], last = g.cuoij[col * HYD_SEGL + k];
        for (int row = first + threadIdx.x; row < last; row += blockDim.x) {
            const int o = P;
            double pp, q, tmp;
            pp = 0;
            q = 0;
            tmp = 0;
            const double vtb = (v[row * o + col - 1] + v[row * o + col] + v[(row + 1) * o + col - 1] + v[(row + 1) * o + col]) * 0.25;
            const double t_vtb = (t_v[row * o + col - 1] + t_v[row * o + col] + t_v[(row + 1) * o + col - 1] + t_v[(row + 1) * o + col]) * 0.25;
            pp = (u[(row + 1) * o + col] - u[(row - 1) * o + col]) / p.dX2;
            pp = (p.HaiChiadT + pp + g.Kx1[row * o + col] * sqrt(vtb * vtb + u[row * o + col] * u[row * o + col]) / g.Htdu[row * o + col]);
            if (H[row * o + col - 1] <= p.H_TINH) {
                if (vtb < 0) {
                    q = t_vtb * (-3 * u[row * o + col] + 4 * u[row * o + col + 1] - u[row * o + col + 2]) / p.dY2;
                    tmp = (u[row * o + col] - 2 * u[row * o + col + 1] + u[row * o + col + 2]) / p.dYbp;
                }
            } else {
                if (H[row * o + col + 1] <= p.H_TINH) {
                    if ((H[row * o + col - 2] > p.H_TINH) && (vtb > 0)) {
                        q = t_vtb * (3 * u[row * o + col] - 4 * u[row * o + col - 1] + u[row * o + col - 2]) / p.dY2;
                        tmp = (u[row * o + col] - 2 * u[row * o + col - 1] + u[row * o + col - 2]) / p.dYbp;
                    }
                } else {
                    q = t_vtb * (u[row * o + col + 1] - u[row * o + col - 1]) / p.dY2;
                    tmp = (u[row * o + col + 1] - 2 * u[row * o + col] + u[row * o + col - 1]) / p.dYbp;
                }
            }
            q = p.HaiChiadT * u[row * o + col] - q + p.CORIOLIS_FORCE * t_vtb;
            q = (q - p.g * (z[(row + 1) * o + col] - z[row * o + col]) / p.dX +
                 g.VISC[row * o + col] * (tmp + (u[(row + 1) * o + col] - 2 * u[row * o + col] + u[(row - 1) * o + col]) / p.dXbp)) +
                (p.windx - g.Tsxw[row * o + col]) / g.Htdu[row * o + col];
            g.t_u[row * o + col] = q / pp;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double* t_u = g.t_u;
        const double* h = g.h;
        const int j = col, W = P;
        for (int k = 0; k < nseg; k++) {
            const int first = g.dauj[j * HYD_SEGL + k], last = g.cuoij[j * HYD_SEGL + k];
            const bool b1 = (first > 2) || ((first == 2) && ((fabs(h[1 * W + j] + h[1 * W + j - 1]) * 0.5 - p.NANGDAY) < kEpsRef));
            const bool b2 = (last < N) || ((last == N) && (fabs((h[N * W + j] + h[N * W + j - 1]) * 0.5 - p.NANGDAY) < kEpsRef));
            if (b1) t_u[(first - 1) * W + j] = 0;
            else t_u[(first - 1) * W + j] = 2 * t_u[first * W + j] - t_u[(first + 1) * W + j];
            if (b2) t_u[last * W + j] = 0;
            else t_u[last * W + j] = 2 * t_u[(last - 1) * W + j] - t_u[(last - 2) * W + j];
        }
    }
}

// --------------------------------------------------------------- wet/dry resets

// update_h_moi (support_funcs.cu:60-73) and Reset_states_horizontal/_vertical
// (support_funcs.cu:75-186) for one line.  ROWS: line = row i (1..N), cells j (2..M);
// otherwise line = column j (1..M), cells i (2..N).  The opening pass is a serial
// scan in the reference; an iteration can only act next to a cell whose mask is 1
// at the start of the pass, so warp 0 ballots those candidates and lane 0 runs them
// in increasing order.
template <int ROWS>
__global__ void k_reset(DevGrid g, DevParams p) {
    const int line = 1 + blockIdx.x;
    const int P = g.P;
    const int L = ROWS ? g.M : g.N;           // last cell index of the line
    const int along = ROWS ? 1 : P;
    const int base = ROWS ? line * P : line;
    double *H = g.H_moi, *t_z = g.t_z, *FS = g.FS;
    int* kh = g.khouot;
    // update_h_moi for this line (cells 1..L)
    for (int k = 1 + threadIdx.x; k <= L; k += blockDim.x) {
        const int gp = base + k * along;
        if (kh[gp] == 0) H[gp] = g.htaiz[gp] + t_z[gp];
    }
    __syncthreads();
    // opening pass (loop 1)
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int c0 = 2; c0 <= L; c0 += 32) {
            const int k = c0 + lane;
            bool cand = false;
            if (k <= L) cand = (kh[base + (k - 1) * along] == 1) || (kh[base + (k + 1) * along] == 1);
            unsigned mask = __ballot_sync(0xffffffffu, cand);
            if (lane == 0) {
                while (mask) {
                    const int b = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const int kk = c0 + b;
                    const int gp = base + kk * along;
                    if (t_z[gp] > g.z[gp]) {
                        const int gm = gp - along, gq = gp + along;
                        if (kh[gm] == 1) {
                            t_z[gm] = t_z[gp];
                            H[gm] = g.htaiz[gm] + t_z[gp];
                            kh[gm] = 0;
                            FS[gm] = FS[gp];
                        }
                        if (kh[gq] == 1) {
                            t_z[gq] = t_z[gp];
                            H[gq] = g.htaiz[gq] + t_z[gp];
                            kh[gq] = 0;
                            FS[gq] = FS[gp];
                        }
                    }
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // closing pass (loop 2): independent per cell
    for (int k = 2 + threadIdx.x; k <= L; k += blockDim.x) {
        const int gp = base + k * along;
        if (kh[gp] == 0 && H[gp] <= p.H_TINH) {
            g.t_u[gp - P] = 0;
            g.t_u[gp] = 0;
            g.t_v[gp - 1] = 0;
            g.t_v[gp] = 0;
            kh[gp] = 1;
            FS[gp] = 0;
        }
    }
}

// --------------------------------------------------- state update and face depths

// update_uvz (support_funcs.cu:671-680) and Htuongdoi (338-354) in one pass.  The
// kernel's kenhhepd/kenhhepng parameters never receive the host's flags (Engine.py:90
// passes two arguments fewer than it declares), so velocities are copied unmasked.
__global__ void k_post(DevGrid g, int with_uvz) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
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

// ------------------------------------------------------------- wet-segment scans

// Find_Calculation_limits_Horizontal/Vertical (support_funcs.cu:230-335).  The serial
// while-loop there yields the maximal runs of khouot == 0 within [2, L] in order,
// except runs starting at L-1 or L, which it skips; one warp per line finds the run
// starts and ends with ballots.  Blocks [0, N-1) scan rows 2..N, the rest columns 2..M.
__global__ void k_scan(DevGrid g) {
    const int lane = threadIdx.x;
    const int N = g.N, M = g.M, P = g.P;
    int line, L, along, base;
    int *dau, *cuoi, *moc;
    if ((int)blockIdx.x < N - 1) {
        line = 2 + blockIdx.x;
        L = M;
        along = 1;
        base = line * P;
        dau = g.daui + line * HYD_SEGL;
        cuoi = g.cuoii + line * HYD_SEGL;
        moc = g.moci + line;
    } else {
        line = 2 + (blockIdx.x - (N - 1));
        L = N;
        along = P;
        base = line;
        dau = g.dauj + line * HYD_SEGL;
        cuoi = g.cuoij + line * HYD_SEGL;
        moc = g.mocj + line;
    }
    const int* kh = g.khouot;
    int nseg = 0;       // uniform across the warp
    int open_start = -1;
    for (int c0 = 2; c0 <= L; c0 += 32) {
        const int k = c0 + lane;
        bool isz = false, prevz = false, nextz = false;
        if (k <= L) {
            isz = kh[base + k * along] == 0;
            prevz = (k > 2) && kh[base + (k - 1) * along] == 0;
            nextz = (k < L) && kh[base + (k + 1) * along] == 0;
        }
        unsigned starts = __ballot_sync(0xffffffffu, isz && !prevz);
        unsigned ends = __ballot_sync(0xffffffffu, isz && !nextz);
        // walk events in position order; a run's start precedes or equals its end
        while (starts | ends) {
            const int bs = starts ? __ffs(starts) - 1 : 64;
            const int be = ends ? __ffs(ends) - 1 : 64;
            if (open_start < 0) {
                // next event must be a start
                if (!starts) break;
                open_start = c0 + bs;
                starts &= starts - 1;
            } else {
                if (!ends) break;  // the run continues into the next chunk
                const int e = c0 + be;
                ends &= ends - 1;
                if (open_start <= L - 2) {
                    if (nseg < HYD_SEGL) {
                        if (lane == 0) {
                            dau[nseg] = open_start;
                            cuoi[nseg] = e;
                        }
                    } else if (lane == 0) {
                        flag_status(g, HYD_ST_SEG_OVERFLOW);
                    }
                    nseg++;
                }
                open_start = -1;
            }
        }
    }
    if (lane == 0) *moc = nseg < HYD_SEGL ? nseg : HYD_SEGL;
}

// Interpolate_FS_ng / Interpolate_FS_d (support_funcs.cu:189-229), run by the row-2,
// row-N and column-M blocks of the scans in the reference.  Rows first (row 2, then
// row N), then the column.
__global__ void k_fs_edges(DevGrid g, DevParams p) {
    const int N = g.N, M = g.M, P = g.P;
    const int i_dX = __double2int_rn(p.dX);
    const int j_dY = __double2int_rn(p.dY);
    for (int pass = 0; pass < 2; pass++) {
        const int location = pass == 0 ? 2 : N, offset = pass == 0 ? 2 : N - 1, sign = pass == 0 ? 1 : -1;
        for (int j = 1 + threadIdx.x; j < M; j += blockDim.x) {
            if (g.t_u[location * P + j] > 0) {
                const double deltaX = (g.u[location * P + j] + g.t_u[location * P + j]) * 0.25 * p.dT;
                const int i = (int)(offset + sign * (deltaX / p.dX));
                const int i_deltaX = __double2int_rn(deltaX);
                if (i < 0 || i + 1 > N + 2) {
                    flag_status(g, HYD_ST_INTERP_RANGE);
                    continue;
                }
                g.FS[location * P + j] = g.FS[i * P + j] + sign * (g.FS[(i + 1) * P + j] - g.FS[i * P + j]) *
                                                               (deltaX / p.dX - i_deltaX / i_dX);
            }
        }
        __syncthreads();
    }
    {
        const int location = M, offset = M - 1, sign = -1;
        for (int i = 1 + threadIdx.x; i < M && i <= N + 2; i += blockDim.x) {
            if (g.t_v[i * P + location] > 0) {
                const double deltaY = (g.v[i * P + location] + g.t_v[i * P + location]) * 0.25 * p.dT;
                const int j = (int)(offset + sign * (deltaY / p.dY));
                const int j_deltaY = __double2int_rn(deltaY);
                if (j < 0 || j + 1 > M + 2) {
                    flag_status(g, HYD_ST_INTERP_RANGE);
                    continue;
                }
                g.FS[i * P + location] = g.FS[i * P + j + 1] + (g.FS[i * P + j + 1] - g.FS[i * P + j]) *
                                                                   (deltaY / p.dY - j_deltaY / j_dY);
            }
        }
    }
}

// --------------------------------------------------------------------- sediment

// Find_VTH (Sediment_Transport.cu:541-568) and hesoK (508-539) in one pass
__global__ void k_vth_hesok(DevGrid g, DevParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int N = g.N, M = g.M, P = g.P;
    if (i > N || j > M) return;
    const int pos = i * P + j;
    if (i >= 2 && j >= 2) {
        if ((g.htaiz[pos] > p.NANGDAY) && (g.H_moi[pos] > p.H_TINH)) {
            const double ut = (g.t_u[pos] + g.t_u[pos - P]) * 0.5;
            const double vt = (g.t_v[pos] + g.t_v[pos - 1]) * 0.5;
            g.VTH[pos] = sqrt(ut * ut + vt * vt);
        } else
            g.VTH[pos] = 0;
    }
    const double sg = sqrt(p.g);
    if (g.Htdu[pos] > 0 && pos >= 1) {
        const double Cz = 18 * log(12 * g.Htdu[pos] / p.Ks);
        const double kx = 5.93 * sg * (g.h[pos - 1] + g.h[pos]) * 0.25 * fabs(g.t_u[pos]) / Cz;
        g.Kx[pos] = fmin(100.0, fmax(5.0, kx));
    }
    if (g.Htdv[pos] > 0 && pos >= P) {
        const double Cz = 18 * log(12 * g.Htdv[pos] / p.Ks);
        const double ky = 5.93 * sg * (g.h[pos - P] + g.h[pos]) * 0.25 * fabs(g.t_v[pos]) / Cz;
        g.Ky[pos] = fmin(100.0, fmax(5.0, ky));
    }
}

// Update_FS (Sediment_Transport.cu:620-629)
__global__ void k_update_fs(DevGrid g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.N || j > g.M) return;
    g.FS[i * g.P + j] = g.tFS[i * g.P + j];
}

// Calculate_Qb (Sediment_Transport.cu:341-414): bed-load flux, then the edge copies
__global__ void k_qb(DevGrid g, DevParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 2;
    const int N = g.N, M = g.M, P = g.P;
    if (i > N || j > M) return;
    const int pos = i * P + j;
    double Tob, Toee = p.Toe, Tx = 0;
    double qx = 0, qy = 0;
    if ((!g.VTH[pos]) && (g.khouot[pos] == 0)) {
        Tob = p.ro * g.Fw[pos] * (g.VTH[pos] * g.VTH[pos]);
        if (g.H_moi[pos] > p.ghtoe) Toee = p.Toe * (1 + p.hstoe * ((g.H_moi[pos] - p.ghtoe)));
        if (Tob > Toee) Tx = Tob / Toee - 1;
        qx = 0.053 * pow((p.Sx - 1) * p.g, 0.5) * pow(p.dm, 1.5) * pow(Tx, 2.1) * pow(p.dxr, -0.3) *
             (g.t_u[pos] + g.t_u[pos - P]) * 0.5 / g.VTH[pos];
        qy = 0.053 * pow((p.Sx - 1) * p.g, 0.5) * pow(p.dm, 1.5) * pow(Tx, 2.1) * pow(p.dxr, -0.3) *
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

__device__ __forceinline__ double source_chs_g(const DevParams& p, double wsm, double Zf, double fs, double fw,
                                               double vth, double h_moi) {
    double toee = p.Toe;
    double S = 0;
    const double tob = p.ro * fw * (vth * vth);
    if (h_moi > p.ghtoe) toee = p.Toe * (1 + p.hstoe * ((h_moi - p.ghtoe)));
    if (tob > toee) S = p.Mbochat / p.ros * (tob - toee) / toee;
    else if (tob < p.Tod) {
        const double Pd = 1 - (tob / p.Tod);
        const double beta = 1 + (Zf / (1.25 + 4.75 * pow(Pd, 2.5)));
        const double Cb = beta * fs;
        S = -wsm * Cb * Pd;
    }
    return S;
}

// BedLoad/_bed_load (Sediment_Transport.cu:630-639, 416-506): Exner increment into dH
// on rows startidx..endidx-1.
__global__ void k_bedload(DevGrid g, DevParams p, int startidx, int endidx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
    const int N = g.N, M = g.M, width = g.P;
    if (i >= endidx || j > M) return;
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
            if (g.t_u[1]) pp = (3 * Qbx[pos] - 4 * Qbx[pos - width] + Qbx[pos - 2 * width]) / p.dX2;
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
    const double wsm = p.wss * pow((1 - FS[pos]), 4);
    double Zf = 0, S = 0;
    if (FS[pos] > 0.0) Zf = wsm / (0.4 * (Uf + 2 * wsm));
    if (p.ketdinh) S = source_chs_g(p, wsm, Zf, FS[pos], g.Fw[pos], g.VTH[pos], g.H_moi[pos]);
    else {
        const double gamac = 0.434 + 5.975 * Zf + 2.888 * Zf * Zf;
        const double Tx = fmax(0.0, (Uf * Uf - p.ufr * p.ufr) / (p.ufr * p.ufr));
        const double Cac = 0.015 * p.dm * pow(Tx, 1.5) * pow(p.dxr, (-0.3)) / (0.05 * g.H_moi[pos]);
        S = wsm * (Cac - gamac * FS[pos]);
    }
    g.dH[pos] += p.dT / (1 - p.Dorong) * (S + tH);
}

}  // namespace

// ------------------------------------------------------------------ host wrappers

void launch_init_kernels(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    const dim3 b(32, 8);
    k_onetime_init<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p);
    k_fs_edges<<<1, 512, 0, s>>>(g, p);
    k_scan<<<(g.N - 1) + (g.M - 1), 32, 0, s>>>(g);
    k_post<<<grid2d(g.M + 1, g.N + 1, b), b, 0, s>>>(g, 0);
    k_preprocess<<<1, 32, 0, s>>>(g, p);
    hyd_kernel_launches_add(5);
}

void launch_boundary(const DevGrid& g, const DevParams& p, double t, cudaStream_t s) {
    if (p.channel) k_boundary_channel<<<1, 256, 0, s>>>(g, p, t);
    else k_boundary<<<1, 1024, 0, s>>>(g, p, t);
    hyd_kernel_launches_add(1);
}

void launch_smooth(const DevGrid& g, const DevParams& p, int isU, double* out, cudaStream_t s) {
    const dim3 b(32, 8);
    k_smooth<<<grid2d(g.M + 3, g.N + 3, b), b, 0, s>>>(g, p, isU, out);
    hyd_kernel_launches_add(1);
}

void launch_explicit_v(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    k_explicit_v<<<g.N - 1, 128, 0, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_explicit_u(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    k_explicit_u<<<g.M - 1, 128, 0, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_reset_rows(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    k_reset<1><<<g.N, 128, 0, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_reset_cols(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    k_reset<0><<<g.M, 128, 0, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_post(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    const dim3 b(32, 8);
    k_post<<<grid2d(g.M + 1, g.N + 1, b), b, 0, s>>>(g, 1);
    hyd_kernel_launches_add(1);
}

void launch_scan_fs_edges(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    k_fs_edges<<<1, 512, 0, s>>>(g, p);
    k_scan<<<(g.N - 1) + (g.M - 1), 32, 0, s>>>(g);
    hyd_kernel_launches_add(2);
}

void launch_vth_hesok(const DevGrid& g, const DevParams& p, cudaStream_t s) {
    const dim3 b(32, 8);
    k_vth_hesok<<<grid2d(g.M + 1, g.N + 1, b), b, 0, s>>>(g, p);
    hyd_kernel_launches_add(1);
}

void launch_update_fs(const DevGrid& g, cudaStream_t s) {
    const dim3 b(32, 8);
    k_update_fs<<<grid2d(g.M, g.N, b), b, 0, s>>>(g);
    hyd_kernel_launches_add(1);
}

void launch_bed(const DevGrid& g, const DevParams& p, int startidx, int endidx, cudaStream_t s) {
    const dim3 b(32, 8);
    k_qb<<<grid2d(g.M - 1, g.N - 1, b), b, 0, s>>>(g, p);
    if (endidx > startidx) k_bedload<<<grid2d(g.M - 1, endidx - startidx, b), b, 0, s>>>(g, p, startidx, endidx);
    hyd_kernel_launches_add(2);
}
