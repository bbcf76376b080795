// k_sweep.cu — fused implicit line sweeps of the ADI step.
//
// One CTA per grid line does what the reference spreads over five kernels and global
// scratch (UZSolver_calculate_preindex/_abcd/_matrix_coeff, tridiagSolver,
// UZSolver_extract_solution, UVZSolver_multithread.cu:881-943 and the VZ twins
// 818-879; Scan_FS*/tridiagSolver/FS*_extract_solution, Sediment_Transport.cu:570-617):
//   A  continuity coefficients a2, c2, d2 of every wet cell            -> shared memory
//   B  momentum coefficients and the interleaved tridiagonal rows       -> shared memory
//   C  the line's tridiagonal system, solved in shared memory by a
//      partitioned method: each thread eliminates its chunk of rows,
//      the 2T interface unknowns are solved by parallel cyclic reduction,
//      and each thread substitutes back into its chunk (replaces the
//      reference's serial Thomas sweep, UVZSolver_multithread.cu:203-228)
//   D  the solution scattered to t_z / t_u (t_v) with the reference's
//      boundary-case formulas.
// All wet segments of a line are solved as one system: the rows of a segment
// are decoupled from their neighbours and every row outside a segment is an
// identity row.  Each line's fields are read from HBM once.
#include <cuda_runtime.h>

#include <cmath>

#include "hydist_dev.cuh"

namespace {

constexpr int kRedBuf = 2 * 4;  // two buffers of (A, B, C, D)

// Partitioned tridiagonal solve of rows [0, T*m) held in shared memory.
// Row r: A[r] x[r-1] + B[r] x[r] + C[r] x[r+1] = D[r]; A[0] and C[last] are ignored.
// Thread t owns rows [t*m, t*m+m), m >= 3.  On return B[r] holds x[r].
template <int T>
__device__ void solve_partitioned(double* A, double* B, double* C, double* D, int m, double* red) {
    const int t = threadIdx.x;
    const int s = t * m, e = s + m - 1;
    // downward elimination inside the chunk: x_i + c'_i x_{i+1} + a'_i x_s = d'_i
    {
        int i = s + 1;
        double den = B[i];
        double cp = C[i] / den, dp = D[i] / den, ap = A[i] / den;
        A[i] = ap;
        C[i] = cp;
        D[i] = dp;
        for (i = s + 2; i <= e; i++) {
            const double ai = A[i];
            den = B[i] - ai * cp;
            cp = C[i] / den;
            dp = (D[i] - ai * dp) / den;
            ap = -(ai * ap) / den;
            A[i] = ap;
            C[i] = cp;
            D[i] = dp;
        }
    }
    // upward: x_i = d''_i - a''_i x_s - c''_i x_e for s < i < e
    {
        double an = A[e - 1], cn = C[e - 1], dn = D[e - 1];
        for (int i = e - 2; i >= s + 1; i--) {
            const double ci = C[i];
            dn = D[i] - ci * dn;
            an = A[i] - ci * an;
            cn = -ci * cn;
            A[i] = an;
            C[i] = cn;
            D[i] = dn;
        }
    }
    // reduced system on the 2T interface unknowns (x_s, x_e of every chunk)
    constexpr int n = 2 * T;
    double* rA = red;
    double* rB = red + n;
    double* rC = red + 2 * n;
    double* rD = red + 3 * n;
    {
        const double as = A[s], bs = B[s], cs = C[s], ds = D[s];
        if (m >= 3) {
            rA[2 * t] = as;
            rB[2 * t] = bs - cs * A[s + 1];
            rC[2 * t] = -cs * C[s + 1];
            rD[2 * t] = ds - cs * D[s + 1];
        }
        rA[2 * t + 1] = A[e];
        rB[2 * t + 1] = 1.0;
        rC[2 * t + 1] = C[e];
        rD[2 * t + 1] = D[e];
    }
    __syncthreads();
    // parallel cyclic reduction, ping-pong between the two buffers
    double* cur = red;
    double* nxt = red + 4 * n;
    for (int d = 1; d < n; d <<= 1) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = 2 * t + q;
            const double* cA = cur;
            const double* cB = cur + n;
            const double* cC = cur + 2 * n;
            const double* cD = cur + 3 * n;
            double nA = 0.0, nB = cB[r], nC = 0.0, nD = cD[r];
            const int lo = r - d, hi = r + d;
            if (lo >= 0) {
                const double k1 = cA[r] / cB[lo];
                nA = -cA[lo] * k1;
                nB -= cC[lo] * k1;
                nD -= cD[lo] * k1;
            }
            if (hi < n) {
                const double k2 = cC[r] / cB[hi];
                nC = -cC[hi] * k2;
                nB -= cA[hi] * k2;
                nD -= cD[hi] * k2;
            }
            nxt[r] = nA;
            nxt[n + r] = nB;
            nxt[2 * n + r] = nC;
            nxt[3 * n + r] = nD;
        }
        __syncthreads();
        double* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    const double xs = cur[3 * n + 2 * t] / cur[n + 2 * t];
    const double xe = cur[3 * n + 2 * t + 1] / cur[n + 2 * t + 1];
    for (int i = s + 1; i < e; i++) B[i] = D[i] - A[i] * xs - C[i] * xe;
    B[s] = xs;
    B[e] = xe;
    __syncthreads();
}

// Serial Thomas per line by thread 0, in the reference's operation order
// (tridiag, UVZSolver_multithread.cu:203-228) applied to the whole decoupled line.
__device__ void solve_thomas(double* A, double* B, double* C, double* D, int rows) {
    if (threadIdx.x == 0) {
        // forward: store Ap in C, Bp in D
        double Ap = -C[0] / B[0], Bp = D[0] / B[0];
        C[0] = Ap;
        D[0] = Bp;
        for (int i = 1; i < rows; i++) {
            const double ep = A[i] * Ap + B[i];
            Ap = -C[i] / ep;
            Bp = (D[i] - (A[i] * Bp)) / ep;
            C[i] = Ap;
            D[i] = Bp;
        }
        double x = D[rows - 1];
        B[rows - 1] = x;
        for (int i = rows - 2; i >= 0; i--) {
            x = D[i] + (C[i] * x);
            B[i] = x;
        }
    }
    __syncthreads();
}

struct SegInfo {
    int first[HYD_SEGL], last[HYD_SEGL];
    int br1[HYD_SEGL], br2[HYD_SEGL];
    int typeR[HYD_SEGL];  // rows start with continuity (bienrandau) instead of momentum (bienlongdau)
    int sn[HYD_SEGL];
    double tzl[HYD_SEGL], tzr[HYD_SEGL];
    int nseg;
};

// Hydrodynamic sweep.  DIR 0: UZ, line = column j, cells i (t_u, ubt/ubp, bienQ[2]/[3]).
//                      DIR 1: VZ, line = row i, cells j (t_v, vbd/vbt, bienQ[1]/[0]).
template <int DIR, int T, int SOLVER>
__global__ void __launch_bounds__(T) k_hydro_sweep(DevGrid g, DevParams p, int startidx, int m) {
    extern __shared__ double smem[];
    __shared__ SegInfo sg;
    const int line = startidx + blockIdx.x;
    const int N = g.N, M = g.M, P = g.P;
    const int L = DIR == 0 ? N : M;
    const int Lc = L + 3;
    const int Rpad = T * m;
    double* A = smem;
    double* B = A + Rpad;
    double* C = B + Rpad;
    double* D = C + Rpad;
    double* a2 = D + Rpad;
    double* c2 = a2 + Lc;
    double* d2 = c2 + Lc;
    double* red = d2 + Lc;
    const int tid = threadIdx.x;
    // cell k of this line -> linear position; stride across the line for the cross neighbour
    const int along = DIR == 0 ? P : 1;  // offset to the next cell of the line
    const int cross = DIR == 0 ? 1 : P;  // offset to the neighbouring line
    const int base = DIR == 0 ? line : line * P;
    double* tvel = DIR == 0 ? g.t_u : g.t_v;
    const double bq_first = DIR == 0 ? g.ubt[line] : g.vbd[line];  // ubt_or_vbd
    const double bq_last = DIR == 0 ? g.ubp[line] : g.vbt[line];   // ubp_or_vbt
    const int Q1 = DIR == 0 ? g.bienQ[2] : g.bienQ[1];             // dkBienQ_1
    const int Q2 = DIR == 0 ? g.bienQ[3] : g.bienQ[0];             // dkBienQ_2

    if (tid == 0) {
        const int n = DIR == 0 ? g.mocj[line] : g.moci[line];
        sg.nseg = n;
    }
    for (int r = tid; r < Rpad; r += T) {
        A[r] = 0.0;
        B[r] = 1.0;
        C[r] = 0.0;
        D[r] = 0.0;
    }
    __syncthreads();
    const int nseg = sg.nseg;
    if (tid < nseg) {
        const int f = DIR == 0 ? g.dauj[line * HYD_SEGL + tid] : g.daui[line * HYD_SEGL + tid];
        const int l = DIR == 0 ? g.cuoij[line * HYD_SEGL + tid] : g.cuoii[line * HYD_SEGL + tid];
        int b1, b2;
        if (DIR == 0) seg_flags_u(g, p, line, f, l, b1, b2);
        else seg_flags_v(g, p, line, f, l, b1, b2);
        sg.first[tid] = f;
        sg.last[tid] = l;
        sg.br1[tid] = b1;
        sg.br2[tid] = b2;
        sg.typeR[tid] = b1 || (Q1 && f == 2);
        sg.tzl[tid] = g.t_z[base + f * along];
        sg.tzr[tid] = g.t_z[base + l * along];
    }
    __syncthreads();

    // ---- A: continuity coefficients (preindex, UVZSolver_multithread.cu:402-406 / 345-349)
    for (int sI = 0; sI < nseg; sI++) {
        const int f = sg.first[sI], l = sg.last[sI];
        for (int k = f + tid; k <= l; k += T) {
            const int pos = base + k * along;
            if (DIR == 0) {
                c2[k] = p.dTchia2dX * g.Htdu[pos];
                a2[k] = -p.dTchia2dX * g.Htdu[pos - P];
                d2[k] = g.z[pos] - p.dTchia2dY * (g.Htdv[pos] * g.v[pos] - g.Htdv[pos - 1] * g.v[pos - 1]);
            } else {
                c2[k] = p.dTchia2dY * g.Htdv[pos];
                a2[k] = -p.dTchia2dY * g.Htdv[pos - 1];
                d2[k] = g.z[pos] - p.dTchia2dX * (g.Htdu[pos] * g.u[pos] - g.Htdu[pos - P] * g.u[pos - P]);
            }
        }
    }
    __syncthreads();

    // ---- B1: momentum rows (preindex f1..f5, _calculate_abcd 409-466) and the interleaved rows
    const double f4 = DIR == 0 ? 2 * p.g * p.dTchia2dX : 2 * p.g * p.dTchia2dY;
    for (int sI = 0; sI < nseg; sI++) {
        const int f = sg.first[sI], l = sg.last[sI];
        const int Ls = l - f;
        const int tR = sg.typeR[sI];
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        for (int k = f + tid; k <= l; k += T) {
            if (tR) {
                A[2 * k] = a2[k];
                B[2 * k] = 1.0;
                C[2 * k] = c2[k];
                D[2 * k] = d2[k];
            }
            if (k == l) continue;
            if (Ls <= 1 && k != f) continue;
            const int pos = base + k * along;
            double f1, f2, f3, f5;
            {
                double pp = 0.0, qq = 0.0;
                if (DIR == 0) {
                    const double* u = g.u;
                    const double* H = g.H_moi;
                    const double vtb = (g.v[pos - 1] + g.v[pos] + g.v[pos + P - 1] + g.v[pos + P]) * 0.25;
                    f1 = p.dTchia2dX * u[pos] + g.VISC[pos] * p.dT / p.dXbp;
                    f2 = -(2 + g.Kx1[pos] * p.dT * sqrt(u[pos] * u[pos] + vtb * vtb) / g.Htdu[pos] +
                           (2 * p.dT * g.VISC[pos]) / p.dXbp);
                    f3 = p.dT * g.VISC[pos] / p.dXbp - p.dTchia2dX * u[pos];
                    if (H[pos - 1] <= p.H_TINH) {
                        if (vtb < 0) {
                            pp = vtb * (-3 * u[pos] + 4 * u[pos + 1] - u[pos + 2]) / p.dY2;
                            qq = (u[pos] - 2 * u[pos + 1] + u[pos + 2]) / p.dYbp;
                        }
                    } else {
                        if (H[pos + 1] <= p.H_TINH) {
                            if ((H[pos - 2] > p.H_TINH) && (vtb > 0)) {
                                pp = vtb * (3 * u[pos] - 4 * u[pos - 1] + u[pos - 2]) / p.dY2;
                                qq = (u[pos] - 2 * u[pos - 1] + u[pos - 2]) / p.dYbp;
                            }
                        } else {
                            pp = vtb * (u[pos + 1] - u[pos - 1]) / p.dY2;
                            qq = (u[pos + 1] - 2 * u[pos] + u[pos - 1]) / p.dYbp;
                        }
                    }
                    f5 = -2 * u[pos] + p.dT * pp - p.dT * p.CORIOLIS_FORCE * vtb - p.dT * g.VISC[pos] * qq -
                         p.dT * (p.windx - g.Tsxw[pos]) / g.Htdu[pos];
                } else {
                    const double* v = g.v;
                    const double* H = g.H_moi;
                    const double utb = (g.u[pos - P] + g.u[pos] + g.u[pos - P + 1] + g.u[pos + 1]) * 0.25;
                    f1 = p.dTchia2dY * v[pos] + g.VISC[pos] * p.dT / p.dYbp;
                    f2 = -(2 + g.Ky1[pos] * p.dT * sqrt(v[pos] * v[pos] + utb * utb) / g.Htdv[pos] +
                           (2 * p.dT * g.VISC[pos]) / p.dYbp);
                    f3 = p.dT * g.VISC[pos] / p.dYbp - p.dTchia2dY * v[pos];
                    if (H[pos - P] <= p.H_TINH) {
                        if (utb < 0) {
                            qq = utb * (-3 * v[pos] + 4 * v[pos + P] - v[pos + 2 * P]) / p.dX2;
                            pp = (v[pos] - 2 * v[pos + P] + v[pos + 2 * P]) / p.dXbp;
                        }
                    } else {
                        if (H[pos + P] <= p.H_TINH) {
                            if ((H[pos - 2 * P] > p.H_TINH) && (utb > 0)) {
                                qq = utb * (3 * v[pos] - 4 * v[pos - P] + v[pos - 2 * P]) / p.dX2;
                                pp = (v[pos] - 2 * v[pos - P] + v[pos - 2 * P]) / p.dXbp;
                            }
                        } else {
                            qq = utb * (v[pos + P] - v[pos - P]) / p.dX2;
                            pp = (v[pos + P] - 2 * v[pos] + v[pos - P]) / p.dXbp;
                        }
                    }
                    f5 = -2 * v[pos] + p.dT * qq + p.dT * p.CORIOLIS_FORCE * utb - p.dT * g.VISC[pos] * pp -
                         p.dT * (p.windy - g.Tsyw[pos]) / g.Htdv[pos];
                }
            }
            double ra, rb, rc, rd;
            if (Ls >= 2) {
                if (k == f && b1f) {
                    ra = f4;
                    rb = f2 - (f3 * a2[f + 1] / c2[f + 1]);
                    rc = -f4 - (f3 / c2[f + 1]);
                    rd = f5 - (f3 * d2[f + 1] / c2[f + 1]);
                } else if (k == l - 1 && b2f) {
                    ra = f4 - f1 / a2[k];
                    rb = f2 - (f1 * c2[k] / a2[k]);
                    rc = -f4;
                    rd = f5 - (f1 * d2[k] / a2[k]);
                } else {
                    ra = f4 - f1 / a2[k];
                    rc = -f4 - (f3 / c2[k + 1]);
                    rb = f2 - (f1 * c2[k] / a2[k]) - (f3 * a2[k + 1] / c2[k + 1]);
                    rd = f5 - (f1 * d2[k] / a2[k]) - (f3 * d2[k + 1] / c2[k + 1]);
                }
            } else {
                ra = f4;
                rb = f2;
                rd = f5;
                rc = -f4;
            }
            const int r = tR ? 2 * k + 1 : 2 * k;
            A[r] = ra;
            B[r] = rb;
            C[r] = rc;
            D[r] = rd;
            if (!tR) {
                A[2 * k + 1] = a2[k + 1];
                B[2 * k + 1] = 1.0;
                C[2 * k + 1] = c2[k + 1];
                D[2 * k + 1] = d2[k + 1];
            }
        }
    }
    __syncthreads();

    // ---- B2: segment end rows (_calculate_matrix_coeff 469-592) and decoupling
    if (tid < nseg) {
        const int f = sg.first[tid], l = sg.last[tid];
        const int Ls = l - f;
        const int b1f = sg.br1[tid], b2f = sg.br2[tid], tR = sg.typeR[tid];
        int sn;
        int lastKind;  // 0 wall (row kept), 1 discharge end (DD -= CC*bq_last), 2 stage end (DD -= CC*TZ_r)
        const int qEnd = Q1 && l == (DIR == 0 ? N : M);
        if (b1f) {
            if (!b2f) {
                if (Q2 && l == (DIR == 0 ? N : M)) {
                    sn = 2 * Ls;
                    lastKind = 1;
                } else {
                    sn = 2 * Ls - 1;
                    lastKind = 2;
                }
            } else {
                sn = 2 * Ls;
                lastKind = 0;
            }
        } else if (tR) {
            if (!b2f) {
                if (qEnd) {
                    sn = 2 * Ls;
                    lastKind = 1;
                } else {
                    sn = 2 * Ls - 1;
                    lastKind = 2;
                }
            } else {
                sn = 2 * Ls;
                lastKind = 0;
            }
        } else {
            if (!b2f) {
                if (qEnd) {
                    sn = 2 * Ls - 1;
                    lastKind = 1;
                } else {
                    sn = 2 * Ls - 2;
                    lastKind = 2;
                }
            } else {
                sn = 2 * Ls - 1;
                lastKind = 0;
            }
        }
        sg.sn[tid] = sn;
        const int rowF = 2 * f;
        if (sn < 0) {
            // single-cell segment on an open edge: the reference solves a negative-size
            // system on stale scratch; nothing is solved here
            flag_status(g, HYD_ST_DEGENERATE);
            for (int r = rowF; r <= 2 * l + 1; r++) {
                A[r] = 0.0;
                B[r] = 1.0;
                C[r] = 0.0;
                D[r] = 0.0;
            }
        } else {
            const int rowL = rowF + sn;
            const double oA = A[rowL], oB = B[rowL], oC = C[rowL], oD = D[rowL];
            if (!b1f) {
                if (tR) D[rowF] = D[rowF] - A[rowF] * bq_first;
                else D[rowF] = D[rowF] - A[rowF] * sg.tzl[tid];
            }
            if (lastKind == 1) {
                A[rowL] = oA;
                B[rowL] = oB;
                D[rowL] = oD - oC * bq_last;
            } else if (lastKind == 2) {
                A[rowL] = oA;
                B[rowL] = oB;
                D[rowL] = oD - oC * sg.tzr[tid];
            }
            A[rowF] = 0.0;
            C[rowL] = 0.0;
            for (int r = rowL + 1; r <= 2 * l + 1; r++) {
                A[r] = 0.0;
                B[r] = 1.0;
                C[r] = 0.0;
                D[r] = 0.0;
            }
        }
    }
    __syncthreads();

    // ---- C: solve
    if (SOLVER == 0) solve_partitioned<T>(A, B, C, D, m, red);
    else solve_thomas(A, B, C, D, 2 * L + 4);

    // ---- D: extract (_uzSolver_extract_solution 668-723 / _vzSolver_extract_solution 595-665)
    const double* x = B;
    const int QF = DIR == 0 ? g.bienQ[2] : g.bienQ[1];
    const int QL = DIR == 0 ? g.bienQ[3] : g.bienQ[0];
    for (int sI = 0; sI < nseg; sI++) {
        const int f = sg.first[sI], l = sg.last[sI];
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        const int sn = sg.sn[sI];
        const int qfirst = !b1f && QF && f == 2;
        for (int k = f + tid; k <= l; k += T) {
            const int pos = base + k * along;
            if (k < l) {
                if (b1f || qfirst) {
                    g.t_z[pos] = x[2 * k];
                    tvel[pos] = x[2 * k + 1];
                    if (k == f) tvel[pos - along] = b1f ? 0.0 : bq_first;
                } else {
                    if (k == f) {
                        const double tv = x[2 * f];
                        tvel[pos] = tv;
                        tvel[pos - along] = (d2[f] - g.t_z[pos] - c2[f] * tv) / a2[f];
                    } else {
                        g.t_z[pos] = x[2 * k - 1];
                        tvel[pos] = x[2 * k];
                    }
                }
            } else {
                const double xl = sn >= 0 ? x[2 * f + sn] : 0.0;
                if (b2f) {
                    tvel[pos] = 0.0;
                    g.t_z[pos] = xl;
                } else if (QL && l == (DIR == 0 ? N : M)) {
                    tvel[pos] = bq_last;
                    g.t_z[pos] = xl;
                } else {
                    double tprev;
                    if (l > f) tprev = (b1f || qfirst) ? x[2 * l - 1] : x[2 * l - 2];
                    else tprev = tvel[pos - along];
                    tvel[pos] = (d2[l] - a2[l] * tprev - g.t_z[pos]) / c2[l];
                }
            }
        }
    }
    (void)cross;
}

// ---- sediment sweeps --------------------------------------------------------------

__device__ __forceinline__ double source_chs(const DevParams& p, double wsm, double Zf, double fs, double fw,
                                             double vth, double h_moi) {
    // source_chs (Sediment_Transport.cu:12-49)
    double toee = p.Toe;
    const double todd = p.Tod;
    double S = 0;
    const double tob = p.ro * fw * (vth * vth);
    if (h_moi > p.ghtoe) toee = p.Toe * (1 + p.hstoe * ((h_moi - p.ghtoe)));
    if (tob > toee) S = p.Mbochat / p.ros * (tob - toee) / toee;
    else if (tob < todd) {
        const double Pd = 1 - (tob / todd);
        const double beta = 1 + (Zf / (1.25 + 4.75 * pow(Pd, 2.5)));
        const double Cb = beta * fs;
        S = -wsm * Cb * Pd;
    }
    return S;
}

__device__ __forceinline__ double source_nchs(const DevParams& p, double wsm, double Zf, double Uf, double h_moi,
                                              double fs) {
    // source_nchs (Sediment_Transport.cu:52-60)
    const double gamac = 0.434 + 5.975 * Zf + 2.888 * Zf * Zf;
    const double Tx = fmax(0.0, (Uf * Uf - p.ufr * p.ufr) / (p.ufr * p.ufr));
    const double Cac = 0.015 * p.dm * pow(Tx, 1.5) * pow(p.dxr, (-0.3)) / (0.05 * h_moi);
    return wsm * (Cac - gamac * fs);
}

// Suspended-sediment sweep.  DIR 0: FSj (columns j = 3..M-1, rows i), DIR 1: FSi (rows i = 3..N-1).
template <int DIR, int T, int SOLVER>
__global__ void __launch_bounds__(T) k_fs_sweep(DevGrid g, DevParams p, double t, int startidx, int m) {
    extern __shared__ double smem[];
    __shared__ SegInfo sg;
    const int line = startidx + blockIdx.x;
    const int P = g.P;
    const int Rpad = T * m;
    double* A = smem;
    double* B = A + Rpad;
    double* C = B + Rpad;
    double* D = C + Rpad;
    double* red = D + Rpad;
    const int tid = threadIdx.x;
    const int along = DIR == 0 ? P : 1;
    const int base = DIR == 0 ? line : line * P;
    const double s_start = p.bed_change_start;
    if (tid == 0) sg.nseg = DIR == 0 ? g.mocj[line] : g.moci[line];
    for (int r = tid; r < Rpad; r += T) {
        A[r] = 0.0;
        B[r] = 1.0;
        C[r] = 0.0;
        D[r] = 0.0;
    }
    __syncthreads();
    const int nseg = sg.nseg;
    if (tid < nseg) {
        const int f = DIR == 0 ? g.dauj[line * HYD_SEGL + tid] : g.daui[line * HYD_SEGL + tid];
        const int l = DIR == 0 ? g.cuoij[line * HYD_SEGL + tid] : g.cuoii[line * HYD_SEGL + tid];
        int b1, b2;
        if (DIR == 0) seg_flags_u(g, p, line, f, l, b1, b2);
        else seg_flags_v(g, p, line, f, l, b1, b2);
        sg.first[tid] = f;
        sg.last[tid] = l;
        sg.br1[tid] = b1;
        sg.br2[tid] = b2;
    }
    __syncthreads();
    const double* FS = g.FS;
    const double* H = g.H_moi;
    const double sqrtg = sqrt(p.g);
    for (int sI = 0; sI < nseg; sI++) {
        const int f = sg.first[sI], l = sg.last[sI];
        if (l - f < 2) continue;
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        for (int k = f + 1 + tid; k <= l - 1; k += T) {
            const int pos = base + k * along;
            const double c = 18 * log(12 * H[pos] / p.Ks);
            const double Uf = sqrtg * fabs(g.VTH[pos]) / c;
            const double wsm = p.wss * pow((1 - FS[pos]), 4);
            double Zf = 0;
            double S;
            double gamav;
            if (DIR == 0) gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;  // evaluated before Zf (Sediment_Transport.cu:236)
            if (FS[pos] > 0.00001) Zf = wsm / (0.4 * (Uf + 2 * wsm));
            if (p.ketdinh) S = source_chs(p, wsm, Zf, FS[pos], g.Fw[pos], g.VTH[pos], H[pos]);
            else S = source_nchs(p, wsm, Zf, Uf, H[pos], FS[pos]);
            if (t < s_start) S = 0;
            if (DIR == 1) gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
            double aa, bb, cc, dd, pp, qq;
            if (DIR == 0) {
                aa = -gamav * 0.5 * (g.t_u[pos] + g.t_u[pos - P]) / p.dX2 -
                     g.Htdu[pos - P] * g.Kx[pos - P] / (H[pos] * (p.dXbp));
                cc = gamav * 0.5 * (g.t_u[pos] + g.t_u[pos - P]) / p.dX2 - g.Htdu[pos] * g.Kx[pos] / (H[pos] * (p.dXbp));
                bb = p.HaiChiadT + (g.Htdu[pos] * g.Kx[pos] + g.Htdu[pos - P] * g.Kx[pos - P]) / (H[pos] * (p.dXbp));
                pp = 0;
                qq = 0;
                if ((H[pos - 1] > p.H_TINH) && (H[pos + 2] > p.H_TINH)) pp = (FS[pos + 1] - FS[pos]);
                if ((H[pos - 2] > p.H_TINH) && (H[pos + 1] > p.H_TINH)) qq = (FS[pos] - FS[pos - 1]);
                pp = (1 / (H[pos] * p.dYbp)) * (g.Htdv[pos] * g.Ky[pos] * pp - g.Htdv[pos - 1] * g.Ky[pos - 1] * qq);
                if ((H[pos - 2] > p.H_TINH) && (H[pos + 2] > p.H_TINH)) {
                    qq = (FS[pos + 1] - FS[pos - 1]) / p.dY2;
                    qq = (g.t_v[pos] + g.t_v[pos - 1]) * 0.5 * qq * gamav;
                } else
                    qq = 0;
                dd = FS[pos] / (p.dT * 0.5) - qq + pp + (S / H[pos]);
                if (k == f + 1) {
                    if (b1f || g.t_u[base + f * along] == 0) bb += aa;
                    else dd -= aa * FS[base + f * along];
                }
                if (k == l - 1) {
                    if (b2f && g.t_u[base + l * along] == 0) bb += cc;
                    else dd -= cc * FS[base + l * along];
                }
            } else {
                aa = -gamav * 0.5 * (g.t_v[pos - 1] + g.t_v[pos]) / p.dY2 -
                     g.Htdv[pos - 1] * g.Ky[pos - 1] / (H[pos] * p.dYbp);
                cc = gamav * 0.5 * (g.t_v[pos - 1] + g.t_v[pos]) / p.dY2 - g.Htdv[pos] * g.Ky[pos] / (H[pos] * p.dYbp);
                bb = p.HaiChiadT + (g.Htdv[pos] * g.Ky[pos] + g.Htdv[pos - 1] * g.Ky[pos - 1]) / (H[pos] * p.dYbp);
                pp = 0;
                qq = 0;
                if ((H[pos + 2 * P] > p.H_TINH) && (H[pos - P] > p.H_TINH)) pp = (FS[pos + P] - FS[pos]);
                if (H[pos - 2 * P] > p.H_TINH && H[pos + P] > p.H_TINH) qq = (FS[pos] - FS[pos - P]);
                pp = (1 / (H[pos] * p.dXbp)) * (g.Htdu[pos] * g.Kx[pos] * pp - g.Htdu[pos - P] * g.Kx[pos - P] * qq);
                if (H[pos + 2 * P] > p.H_TINH && H[pos - 2 * P] > p.H_TINH) {
                    qq = (FS[pos + P] - FS[pos - P]) / p.dX2;
                    qq = (g.t_u[pos] + g.t_u[pos - P]) * 0.5 * qq * gamav;
                } else
                    qq = 0;
                dd = FS[pos] / (p.dT * 0.5) - qq + pp + (S / H[pos]);
                if (k == f + 1) {
                    if (b1f || g.t_v[base + f * along] == 0) bb = bb + aa;
                    else dd = dd - aa * FS[base + f * along];
                }
                if (k == l - 1) {
                    if (b2f || g.t_v[base + l * along] == 0) bb = bb + cc;
                    else dd = dd - cc * FS[base + l * along];
                }
            }
            A[k] = (k == f + 1) ? 0.0 : aa;
            B[k] = bb;
            C[k] = (k == l - 1) ? 0.0 : cc;
            D[k] = dd;
        }
    }
    __syncthreads();
    if (SOLVER == 0) solve_partitioned<T>(A, B, C, D, m, red);
    else solve_thomas(A, B, C, D, DIR == 0 ? g.N + 3 : g.M + 3);
    const double* x = B;
    double* vel = DIR == 0 ? g.t_u : g.t_v;
    for (int sI = 0; sI < nseg; sI++) {
        const int f = sg.first[sI], l = sg.last[sI];
        if (l - f < 2) continue;
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        for (int k = f + 1 + tid; k <= l - 1; k += T) {
            const int pos = base + k * along;
            double xv = x[k];
            if (xv < 0) xv = p.NDnen;
            g.tFS[pos] = xv;
            if (k == f + 1) {
                // FSj: t_u[pos - width]; FSi: t_v[i*width + first]
                const double vb = DIR == 0 ? vel[pos - P] : vel[base + f * along];
                g.tFS[base + f * along] = (b1f || vb == 0) ? xv : FS[base + f * along];
            }
            if (k == l - 1) {
                const double vb = DIR == 0 ? vel[pos + P] : vel[base + l * along];
                g.tFS[base + l * along] = (b2f || vb == 0) ? xv : FS[base + l * along];
            }
        }
    }
}

// --- launch configuration --------------------------------------------------------
inline int odd_chunk(int rows, int T) {
    int m = (rows + T - 1) / T;
    if (m < 3) m = 3;
    if ((m & 1) == 0) m++;
    return m;
}

template <int DIR>
void launch_hydro(const DevGrid& g, const DevParams& p, int startidx, int endidx, int solver, cudaStream_t s) {
    const int nlines = endidx - startidx + 1;
    if (nlines <= 0) return;
    const int L = DIR == 0 ? g.N : g.M;
    const int rows = 2 * L + 4;
    const int Lc = L + 3;
#define HYD_LAUNCH_T(TT)                                                                                     \
    do {                                                                                                     \
        const int m = odd_chunk(rows, TT);                                                                   \
        const size_t sm = sizeof(double) * ((size_t)4 * TT * m + 3 * (size_t)Lc + kRedBuf * 2 * TT);         \
        if (solver == 0) {                                                                                   \
            cudaFuncSetAttribute(k_hydro_sweep<DIR, TT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
            k_hydro_sweep<DIR, TT, 0><<<nlines, TT, sm, s>>>(g, p, startidx, m);                             \
        } else {                                                                                             \
            cudaFuncSetAttribute(k_hydro_sweep<DIR, TT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
            k_hydro_sweep<DIR, TT, 1><<<nlines, TT, sm, s>>>(g, p, startidx, m);                             \
        }                                                                                                    \
    } while (0)
    if (rows <= 256) HYD_LAUNCH_T(32);
    else if (rows <= 1024) HYD_LAUNCH_T(64);
    else HYD_LAUNCH_T(128);
#undef HYD_LAUNCH_T
    hyd_kernel_launches_add(1);
}

template <int DIR>
void launch_fs(const DevGrid& g, const DevParams& p, double t, int solver, cudaStream_t s) {
    const int startidx = 3;
    const int endidx = DIR == 0 ? g.M - 1 : g.N - 1;
    const int nlines = endidx - startidx + 1;
    if (nlines <= 0) return;
    const int rows = (DIR == 0 ? g.N : g.M) + 3;
#define HYD_LAUNCH_T(TT)                                                                                  \
    do {                                                                                                  \
        const int m = odd_chunk(rows, TT);                                                                \
        const size_t sm = sizeof(double) * ((size_t)4 * TT * m + kRedBuf * 2 * TT);                       \
        if (solver == 0) {                                                                                \
            cudaFuncSetAttribute(k_fs_sweep<DIR, TT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
            k_fs_sweep<DIR, TT, 0><<<nlines, TT, sm, s>>>(g, p, t, startidx, m);                          \
        } else {                                                                                          \
            cudaFuncSetAttribute(k_fs_sweep<DIR, TT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
            k_fs_sweep<DIR, TT, 1><<<nlines, TT, sm, s>>>(g, p, t, startidx, m);                          \
        }                                                                                                 \
    } while (0)
    if (rows <= 128) HYD_LAUNCH_T(32);
    else if (rows <= 512) HYD_LAUNCH_T(64);
    else HYD_LAUNCH_T(128);
#undef HYD_LAUNCH_T
    hyd_kernel_launches_add(1);
}

}  // namespace

void launch_sweep_uz(const DevGrid& g, const DevParams& p, int startidx, int endidx, int solver, cudaStream_t s) {
    launch_hydro<0>(g, p, startidx, endidx, solver, s);
}
void launch_sweep_vz(const DevGrid& g, const DevParams& p, int startidx, int endidx, int solver, cudaStream_t s) {
    launch_hydro<1>(g, p, startidx, endidx, solver, s);
}
void launch_fs_sweep_j(const DevGrid& g, const DevParams& p, double t, int solver, cudaStream_t s) {
    launch_fs<0>(g, p, t, solver, s);
}
void launch_fs_sweep_i(const DevGrid& g, const DevParams& p, double t, int solver, cudaStream_t s) {
    launch_fs<1>(g, p, t, solver, s);
}
