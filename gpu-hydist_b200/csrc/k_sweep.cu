// k_sweep.cu — fused implicit line sweeps of the ADI step.
//
// A line's sweep does what the reference spreads over five kernels and global scratch
// (UZSolver_calculate_preindex/_abcd/_matrix_coeff, tridiagSolver,
// UZSolver_extract_solution, UVZSolver_multithread.cu:881-943 and the VZ twins 818-879;
// Scan_FS*/tridiagSolver/FS*_extract_solution, Sediment_Transport.cu:570-617).
// Only the wet segments of the line are touched: their cells and their tridiagonal rows
// are packed one segment after another, so a line with a few wet cells costs a few rows
// however long it is.
//   A  continuity coefficients a2, c2, d2 of every wet cell (those of the segment ends
//      kept for D)
//   B  momentum coefficients and the interleaved rows of every segment's system
//   C  all segments of the line solved as one block-decoupled tridiagonal system by a
//      partitioned method: each thread eliminates a chunk of rows, the chunk-end
//      unknowns are solved by parallel cyclic reduction, each thread substitutes back
//      (replaces the reference's serial Thomas sweep, UVZSolver_multithread.cu:203-228)
//   D  the solution scattered to t_z / t_u (t_v) with the reference's boundary formulas.
//
// One persistent kernel per sweep: a 512-thread CTA per SM takes every G-th line, one
// per warp.  A short line (at most 3 rows per lane) is swept by its warp alone; a long
// line by the whole CTA in shared memory sized for the longest line the grid can hold (a
// global scratch region per CTA beyond that).  A short line's solve is its warp's: lanes
// eliminate chunks of rows, the chunk ends are solved by shuffle-only cyclic reduction; a
// long line's adds a level (up to 256 threads eliminate chunks, one warp solves the
// chunk-end system as above).
// In the column sweeps the cell-local coefficients come precomputed, stored column-major
// so that a column reads them contiguously (k_coef_bnd<0>, k_coef_fsj).
#include <cuda_runtime.h>

#include <cmath>

#include "hydist_dev.cuh"

namespace {

constexpr int kTL = 512;         // threads of a sweep CTA
constexpr int kWL = kTL / 32;    // lines per group (one per warp)
// A warp's shared-memory slice holds kRowW rows (9 per lane).  Which lines a warp sweeps
// alone is chosen per launch: with at most one group of lines per CTA, lines of at most
// kRowShort rows (kRowShortF for sediment), the rest by the whole CTA (a long line then
// costs the CTA less time than a warp would take); with more lines than that, every line
// that fits the slice, so that a CTA's many medium lines run side by side.
constexpr int kRowW = 288;
constexpr int kRowShort = 96;
constexpr int kRowShortF = 64;
// continuity coefficients (a, c, d) of the first and last cell of every segment of a
// hydrodynamic line, kept for the extraction: 6 doubles per segment
constexpr int kEnds = 6 * HYD_SEGL;
constexpr int kWarpHydro = 4 * kRowW + kEnds;  // doubles per warp (the largest slice)
constexpr int kWarpFs = 4 * kRowW;
constexpr int kRowSlice = 96;  // rows of a slice when warps take lines of up to kRowShort (kRowShortF) rows
// rows of a warp's slice for a launch whose warps take lines of up to roww rows
__host__ __device__ inline int slice_rows(int roww) { return roww > kRowSlice ? kRowW : kRowSlice; }
static_assert(kRowW % 32 == 0 && (kRowW / 32) % 2 == 1, "a warp solve pads R <= kRowW rows to 32 chunk_len(R, 32) <= kRowW");

// A group of threads that sweeps one line: a warp, or a whole CTA for a long line.
// WarpG::exchange() gives lane t the values v of lanes t - h (lo) and t + h (hi).
struct WarpG {
    static constexpr int size = 32;
    __device__ static __forceinline__ int rank() { return threadIdx.x & 31; }
    __device__ static __forceinline__ void sync() { __syncwarp(); }
    template <class R>
    __device__ static __forceinline__ void exchange(const R (&v)[6], int h, R (&lo)[6], R (&hi)[6]) {
#pragma unroll
        for (int k = 0; k < 6; k++) {
            lo[k] = __shfl_up_sync(0xffffffffu, v[k], h);
            hi[k] = __shfl_down_sync(0xffffffffu, v[k], h);
        }
    }
};

struct BlockG {
    static constexpr int size = kTL;
    __device__ static __forceinline__ int rank() { return threadIdx.x; }
    __device__ static __forceinline__ void sync() { __syncthreads(); }
};

// Chunk length for R rows over T threads: at least 3 and odd (odd strides keep the
// chunk-strided shared-memory accesses free of bank conflicts).
__host__ __device__ inline int chunk_len(int R, int T) {
    int m = (R + T - 1) / T;
    if (m < 3) m = 3;
    if ((m & 1) == 0) m++;
    return m;
}

// Partitioned tridiagonal solve.  Row r: A[r] x[r-1] + B[r] x[r] + C[r] x[r+1] = D[r];
// A[0] and C[last] are ignored.  Thread t owns the chunk of rows [t*m, t*m+m) (m >= 3).
//
// chunk_reduce: downward elimination inside the chunk (x_i + c'_i x_{i+1} + a'_i x_s =
// d'_i), then upward (x_i = d''_i - a''_i x_s - c''_i x_e for s < i < e), leaving the two
// chunk-end rows of the reduced system on the chunk-end unknowns, ordered (x_s, x_e)
// chunk after chunk and scaled to a unit diagonal: row 2t is (v[0], 1, v[1] | v[2]), row
// 2t+1 is (v[3], 1, v[4] | v[5]) as (lower, diagonal, upper | right-hand side).
// Every solver function is a template on the arithmetic type R: double for the FP64 form,
// float for the mixed form (the FP64 instantiation is the same code with R = double).
template <class R>
__device__ __forceinline__ void chunk_reduce(R* A, R* B, R* C, R* D, int s, int e, R (&v)[6]) {
    {
        int i = s + 1;
        R r = R(1) / B[i];
        R cp = C[i] * r, dp = D[i] * r, ap = A[i] * r;
        A[i] = ap;
        C[i] = cp;
        D[i] = dp;
        for (i = s + 2; i <= e; i++) {
            const R ai = A[i];
            r = R(1) / (B[i] - ai * cp);
            cp = C[i] * r;
            dp = (D[i] - ai * dp) * r;
            ap = -(ai * ap) * r;
            A[i] = ap;
            C[i] = cp;
            D[i] = dp;
        }
    }
    {
        R an = A[e - 1], cn = C[e - 1], dn = D[e - 1];
        for (int i = e - 2; i >= s + 1; i--) {
            const R ci = C[i];
            dn = D[i] - ci * dn;
            an = A[i] - ci * an;
            cn = -ci * cn;
            A[i] = an;
            C[i] = cn;
            D[i] = dn;
        }
    }
    const R cs = C[s];
    const R ib = R(1) / (B[s] - cs * A[s + 1]);
    v[0] = A[s] * ib;
    v[1] = -cs * C[s + 1] * ib;
    v[2] = (D[s] - cs * D[s + 1]) * ib;
    v[3] = A[e];
    v[4] = C[e];
    v[5] = D[e];
}

// The chunk's inner unknowns from its end values; x goes to B.
template <class R>
__device__ __forceinline__ void chunk_back(R* A, R* B, R* C, R* D, int s, int e, R xs, R xe) {
    for (int i = s + 1; i < e; i++) B[i] = D[i] - A[i] * xs - C[i] * xe;
    B[s] = xs;
    B[e] = xe;
}

// Parallel cyclic reduction of the 64-row reduced system of a warp (two unit-diagonal
// rows per lane, in registers, exchanged by shuffles): at distance d row r eliminates rows
// r - d and r + d, every row rescaled to a unit diagonal (one reciprocal per row and
// level).  On return v[2] = x_s and v[5] = x_e of the lane's chunk.
template <class R>
__device__ __forceinline__ void pcr_warp(R (&v)[6]) {
    constexpr int T = 32, n = 2 * T;
    const int t = threadIdx.x & 31;
    for (int d = 1; d < n; d <<= 1) {
        R lo[6], hi[6];
        const int h = d == 1 ? 1 : d >> 1;
        WarpG::exchange(v, h, lo, hi);
        R la[2], lc[2], ld[2], ha[2], hc[2], hd[2];
        bool lv[2], hv[2];
        if (d == 1) {
            // row 2t: lo = row 2t-1 (lane t-1, second row), hi = row 2t+1 (own second row)
            la[0] = lo[3]; lc[0] = lo[4]; ld[0] = lo[5]; lv[0] = t >= 1;
            ha[0] = v[3]; hc[0] = v[4]; hd[0] = v[5]; hv[0] = true;
            // row 2t+1: lo = row 2t (own first row), hi = row 2t+2 (lane t+1, first row)
            la[1] = v[0]; lc[1] = v[1]; ld[1] = v[2]; lv[1] = true;
            ha[1] = hi[0]; hc[1] = hi[1]; hd[1] = hi[2]; hv[1] = t + 1 < T;
        } else {
#pragma unroll
            for (int q = 0; q < 2; q++) {
                la[q] = lo[3 * q]; lc[q] = lo[3 * q + 1]; ld[q] = lo[3 * q + 2]; lv[q] = t - h >= 0;
                ha[q] = hi[3 * q]; hc[q] = hi[3 * q + 1]; hd[q] = hi[3 * q + 2]; hv[q] = t + h < T;
            }
        }
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const R a = v[3 * q], c = v[3 * q + 1];
            R nA = R(0), nC = R(0), nB = R(1), nD = v[3 * q + 2];
            if (lv[q]) {
                nA = -la[q] * a;
                nB -= lc[q] * a;
                nD -= ld[q] * a;
            }
            if (hv[q]) {
                nC = -hc[q] * c;
                nB -= ha[q] * c;
                nD -= hd[q] * c;
            }
            const R ib = R(1) / nB;
            v[3 * q] = nA * ib;
            v[3 * q + 1] = nC * ib;
            v[3 * q + 2] = nD * ib;
        }
    }
}

// One warp: rows [0, 32 m), chunks of m rows per lane, the reduced system by pcr_warp.
// On return B[r] holds x[r].
template <class R>
__device__ __forceinline__ void solve_warp(R* A, R* B, R* C, R* D, int m) {
    const int t = threadIdx.x & 31;
    const int s = t * m, e = s + m - 1;
    R v[6];
    chunk_reduce(A, B, C, D, s, e, v);
    pcr_warp(v);
    chunk_back(A, B, C, D, s, e, v[2], v[5]);
    __syncwarp();
}

// How a group of threads solves R rows: t1 threads with chunks of m rows.  t1 == 32: one
// warp (solve_warp).  t1 > 32: two levels (solve_block): the 2 t1 chunk-end rows form a
// tridiagonal system that one warp solves in chunks of m2 = chunk_len(2 t1, 32) rows.
// The plan minimises the serial depth, about 3 m + 6 for one warp and 3 m + 3 m2 + 10
// for two levels (their two CTA barriers counted as two steps each).
struct SolvePlan {
    int t1, m;
};
constexpr int kRedRows = 32 * 17;  // reduced rows of the largest two-level plan (t1 = 256)
__host__ __device__ inline SolvePlan solve_plan(int R, int max_t1) {
    SolvePlan best{32, chunk_len(R, 32)};
    int depth = 3 * best.m + 6;
    for (int t1 = 64; t1 <= max_t1 && t1 <= 256; t1 <<= 1) {
        const int m1 = chunk_len(R, t1), m2 = chunk_len(2 * t1, 32);
        const int d = 3 * m1 + 3 * m2 + 10;
        if (d < depth) {
            depth = d;
            best = SolvePlan{t1, m1};
        }
    }
    return best;
}

// Two-level solve by a CTA (rows [0, t1 m)); red holds 4 kRedRows doubles.  Every thread
// of the CTA calls it.  On return B[r] holds x[r].
template <class R>
__device__ __forceinline__ void solve_block(R* A, R* B, R* C, R* D, SolvePlan pl, R* red) {
    const int t = threadIdx.x;
    const int m2 = chunk_len(2 * pl.t1, 32);
    R *rA = red, *rB = red + kRedRows, *rC = red + 2 * kRedRows, *rD = red + 3 * kRedRows;
    if (t < pl.t1) {
        const int s = t * pl.m, e = s + pl.m - 1;
        R v[6];
        chunk_reduce(A, B, C, D, s, e, v);
        rA[2 * t] = v[0];
        rB[2 * t] = R(1);
        rC[2 * t] = v[1];
        rD[2 * t] = v[2];
        rA[2 * t + 1] = v[3];
        rB[2 * t + 1] = R(1);
        rC[2 * t + 1] = v[4];
        rD[2 * t + 1] = v[5];
    }
    for (int r = 2 * pl.t1 + t; r < 32 * m2; r += blockDim.x) {  // identity rows
        rA[r] = R(0);
        rB[r] = R(1);
        rC[r] = R(0);
        rD[r] = R(0);
    }
    __syncthreads();
    if (t < 32) solve_warp(rA, rB, rC, rD, m2);
    __syncthreads();
    if (t < pl.t1) {
        const int s = t * pl.m, e = s + pl.m - 1;
        chunk_back(A, B, C, D, s, e, rB[2 * t], rB[2 * t + 1]);
    }
    __syncthreads();
}

// Serial Thomas over the packed rows by the group's first thread, in the reference's
// operation order (tridiag, UVZSolver_multithread.cu:203-228); decoupled segments solve
// exactly as separate systems.  Used to check the partitioned solver.
template <class G, class R>
__device__ __forceinline__ void solve_thomas(R* A, R* B, R* C, R* D, int rows) {
    if (G::rank() == 0 && rows > 0) {
        R Ap = -C[0] / B[0], Bp = D[0] / B[0];
        C[0] = Ap;
        D[0] = Bp;
        for (int i = 1; i < rows; i++) {
            const R ep = A[i] * Ap + B[i];
            Ap = -C[i] / ep;
            Bp = (D[i] - (A[i] * Bp)) / ep;
            C[i] = Ap;
            D[i] = Bp;
        }
        R x = D[rows - 1];
        B[rows - 1] = x;
        for (int i = rows - 2; i >= 0; i--) {
            x = D[i] + (C[i] * x);
            B[i] = x;
        }
    }
    G::sync();
}

// Solve of a line's packed system (rows padded with identity rows to pl.t1 * pl.m) by
// group G: one warp (a warp group, or a CTA's first warp with the others waiting), or
// the two-level solve of a CTA.
template <class G, int SOLVER, class R>
__device__ __forceinline__ void solve_line(R* A, R* B, R* C, R* D, SolvePlan pl, int rows, R* red) {
    if (SOLVER == 0) {
        if (G::size == 32) {
            solve_warp(A, B, C, D, pl.m);
        } else if (pl.t1 == 32) {
            if (threadIdx.x < 32) solve_warp(A, B, C, D, pl.m);
            G::sync();
        } else {
            solve_block(A, B, C, D, pl, red);
        }
    } else {
        solve_thomas<G, R>(A, B, C, D, rows);
    }
}

struct LineShared {
    int first[HYD_SEGL], last[HYD_SEGL];
    int br1[HYD_SEGL], br2[HYD_SEGL];
    int typeR[HYD_SEGL];     // rows start with continuity (bienrandau) rather than momentum (bienlongdau)
    int sn[HYD_SEGL];        // last row index of the segment's system (the reference's SN)
    int lastKind[HYD_SEGL];  // 0 wall end, 1 discharge end, 2 stage end
    int co[HYD_SEGL + 1];    // packed cell offset of each segment
    int ro[HYD_SEGL + 1];    // packed row offset of each segment
    double tzl[HYD_SEGL], tzr[HYD_SEGL];
    double zl[HYD_SEGL], zr[HYD_SEGL];  // mixed form: z at the segment ends (the increments' base)
    int nseg, R, C;
};

// The segment holding packed cell (seg_of) or packed row (seg_of_row) c: the last s with
// off[s] <= c (binary search over at most 20 offsets).
__device__ __forceinline__ int seg_search(const int* off, int nseg, int c) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int seg_of(const LineShared& sg, int c) { return seg_search(sg.co, sg.nseg, c); }
__device__ __forceinline__ int seg_of_row(const LineShared& sg, int c) { return seg_search(sg.ro, sg.nseg, c); }

// ---- hydrodynamic sweeps ----------------------------------------------------------
// DIR 0: UZ, line = column j, cells i (t_u, ubt/ubp, bienQ[2]/[3]).
// DIR 1: VZ, line = row i, cells j (t_v, vbd/vbt, bienQ[1]/[0]).

// Segments of the line, their system sizes (_calculate_matrix_coeff,
// UVZSolver_multithread.cu:515-592) and packed offsets, into sg.
template <int DIR, class G, bool MIX>
__device__ __forceinline__ void hydro_setup(const DevGrid& g, const DevParams& p, int line, LineShared& sg) {
    const int tid = G::rank();
    const int L = DIR == 0 ? g.N : g.M;
    const int along = DIR == 0 ? g.P : 1;
    const int base = DIR == 0 ? line : line * g.P;
    const int Q1 = DIR == 0 ? g.bienQ[2] : g.bienQ[1];  // dkBienQ_1
    const int Q2 = DIR == 0 ? g.bienQ[3] : g.bienQ[0];  // dkBienQ_2
    const int nseg = DIR == 0 ? g.mocj[line] : g.moci[line];
    if (tid < nseg) {
        const int f = DIR == 0 ? g.dauj[line * HYD_SEGL + tid] : g.daui[line * HYD_SEGL + tid];
        const int l = DIR == 0 ? g.cuoij[line * HYD_SEGL + tid] : g.cuoii[line * HYD_SEGL + tid];
        int b1, b2;
        if (DIR == 0) seg_flags_u(g, p, line, f, l, b1, b2);
        else seg_flags_v(g, p, line, f, l, b1, b2);
        const int Ls = l - f;
        const int tR = b1 || (Q1 && f == 2);
        const int qEnd = Q1 && l == L;
        int sn, kind;
        if (b1) {
            if (!b2) {
                if (Q2 && l == L) { sn = 2 * Ls; kind = 1; }
                else { sn = 2 * Ls - 1; kind = 2; }
            } else { sn = 2 * Ls; kind = 0; }
        } else if (tR) {
            if (!b2) {
                if (qEnd) { sn = 2 * Ls; kind = 1; }
                else { sn = 2 * Ls - 1; kind = 2; }
            } else { sn = 2 * Ls; kind = 0; }
        } else {
            if (!b2) {
                if (qEnd) { sn = 2 * Ls - 1; kind = 1; }
                else { sn = 2 * Ls - 2; kind = 2; }
            } else { sn = 2 * Ls - 1; kind = 0; }
        }
        sg.first[tid] = f;
        sg.last[tid] = l;
        sg.br1[tid] = b1;
        sg.br2[tid] = b2;
        sg.typeR[tid] = tR;
        sg.sn[tid] = sn;
        sg.lastKind[tid] = kind;
        sg.tzl[tid] = g.t_z[base + f * along];
        sg.tzr[tid] = g.t_z[base + l * along];
        if (MIX) {
            sg.zl[tid] = g.z[base + f * along];
            sg.zr[tid] = g.z[base + l * along];
        }
    }
    G::sync();
    if (tid == 0) {
        int c = 0, r = 0;
        for (int s = 0; s < nseg; s++) {
            sg.co[s] = c;
            sg.ro[s] = r;
            c += sg.last[s] - sg.first[s] + 1;
            if (sg.sn[s] >= 0) r += sg.sn[s] + 1;
            else flag_status(g, HYD_ST_DEGENERATE);  // single-cell segment on an open edge
        }
        sg.co[nseg] = c;
        sg.ro[nseg] = r;
        sg.C = c;
        sg.R = r;
        sg.nseg = nseg;
    }
    G::sync();
}

// Phases A-D of one line by group G.  Rows A, B, Cc, D hold at least pl.t1 * pl.m
// entries, ends kEnds; red: the two-level solve's reduced rows.
// R = float: the mixed form.  Its coefficients (k_coef_bnd's FP32 arrays) are those of the
// level increment dz = z' - z: the continuity right-hand side d2 - z and the momentum
// f5 - f4 (z_k - z_k+1), so that the same rows solve for (dz, u) in FP32; the prescribed
// levels enter as increments, and the new level is z + dz in FP64.
template <int DIR, int SOLVER, class G, class R>
__device__ __forceinline__ void hydro_body(const DevGrid& g, const DevParams& p, int line, const LineShared& sg,
                                           R* A, R* B, R* Cc, R* D, R* ends, R* red, SolvePlan pl) {
    constexpr bool MIX = sizeof(R) == sizeof(float);
    constexpr int T = G::size;
    const int tid = G::rank();
    const int N = g.N, M = g.M, P = g.P;
    const int L = DIR == 0 ? N : M;
    (void)M;
    const int along = DIR == 0 ? P : 1;  // offset to the next cell of the line
    const int base = DIR == 0 ? line : line * P;
    double* tvel = DIR == 0 ? g.t_u : g.t_v;
    const R bq_first = R(DIR == 0 ? g.ubt[line] : g.vbd[line]);  // ubt_or_vbd
    const R bq_last = R(DIR == 0 ? g.ubp[line] : g.vbt[line]);   // ubp_or_vbt
    const int nseg = sg.nseg;
    const int C = sg.C, Rn = sg.R;

    // ---- A + B1, one pass over the cells: the continuity coefficients of the cell and of
    // the next one (preindex, UVZSolver_multithread.cu:402-406 / 345-349), the momentum
    // coefficients (preindex f1..f5, _calculate_abcd 409-466) and the rows.  The continuity
    // coefficients of each segment's first and last cell are kept for the extraction.
    auto cont = [&](int k, R& a, R& c, R& d) {
        if (DIR == 0) {
            const size_t t = (size_t)line * g.LT + k;  // precomputed by k_coef_bnd<0>
            a = colTr<R>(g, 0)[t];
            c = colTr<R>(g, 1)[t];
            d = colTr<R>(g, 2)[t];
        } else {
            const int pos = base + k * along;  // precomputed by k_coef_bnd<1>
            a = rowCr<R>(g, 0)[pos];
            c = rowCr<R>(g, 1)[pos];
            d = rowCr<R>(g, 2)[pos];
        }
    };
    for (int r = Rn + tid; r < pl.t1 * pl.m; r += T) {  // identity rows up to the solver's rows
        A[r] = R(0);
        B[r] = R(1);
        Cc[r] = R(0);
        D[r] = R(0);
    }
    const R f4 = R(DIR == 0 ? 2 * p.g * p.dTchia2dX : 2 * p.g * p.dTchia2dY);
    for (int c = tid; c < C; c += T) {
        const int sI = seg_of(sg, c);
        const int f = sg.first[sI], l = sg.last[sI];
        const int k = f + (c - sg.co[sI]);
        const int Ls = l - f;
        const int tR = sg.typeR[sI];
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        const int sn = sg.sn[sI];
        const int r0 = sg.ro[sI];
        const int rel = 2 * (k - f);  // row 2k relative to the segment's first row 2f
        // every coefficient the cell may need, loaded at once (the next cell's and f1..f5
        // are in bounds even where unused: k + 1 <= L + 1 inside the padded line)
        R ac, cc, dc, an, cn, dn, f1, f2, f3, f5;
        cont(k, ac, cc, dc);
        cont(k + 1, an, cn, dn);
        if (DIR == 0) {
            const size_t t = (size_t)line * g.LT + k;
            f1 = colTr<R>(g, 3)[t];
            f2 = colTr<R>(g, 4)[t];
            f3 = colTr<R>(g, 5)[t];
            f5 = colTr<R>(g, 6)[t];
        } else {
            const int pos = base + k * along;
            f1 = rowCr<R>(g, 3)[pos];
            f2 = rowCr<R>(g, 4)[pos];
            f3 = rowCr<R>(g, 5)[pos];
            f5 = rowCr<R>(g, 6)[pos];
        }
        if (k == f) {
            ends[6 * sI] = ac;
            ends[6 * sI + 1] = cc;
            ends[6 * sI + 2] = dc;
        }
        if (k == l) {
            ends[6 * sI + 3] = ac;
            ends[6 * sI + 4] = cc;
            ends[6 * sI + 5] = dc;
        }
        if (tR && rel <= sn) {
            A[r0 + rel] = ac;
            B[r0 + rel] = R(1);
            Cc[r0 + rel] = cc;
            D[r0 + rel] = dc;
        }
        if (k == l) continue;
        if (Ls <= 1 && k != f) continue;
        const int rm = tR ? rel + 1 : rel;  // the momentum row of this cell
        if (rm > sn) continue;
        R ra, rb, rc, rd;
        if (Ls >= 2) {
            if (k == f && b1f) {
                ra = f4;
                rb = f2 - (f3 * an / cn);
                rc = -f4 - (f3 / cn);
                rd = f5 - (f3 * dn / cn);
            } else if (k == l - 1 && b2f) {
                ra = f4 - f1 / ac;
                rb = f2 - (f1 * cc / ac);
                rc = -f4;
                rd = f5 - (f1 * dc / ac);
            } else {
                ra = f4 - f1 / ac;
                rc = -f4 - (f3 / cn);
                rb = f2 - (f1 * cc / ac) - (f3 * an / cn);
                rd = f5 - (f1 * dc / ac) - (f3 * dn / cn);
            }
        } else {
            ra = f4;
            rb = f2;
            rd = f5;
            rc = -f4;
        }
        A[r0 + rm] = ra;
        B[r0 + rm] = rb;
        Cc[r0 + rm] = rc;
        D[r0 + rm] = rd;
        if (!tR && rel + 1 <= sn) {
            A[r0 + rel + 1] = an;
            B[r0 + rel + 1] = R(1);
            Cc[r0 + rel + 1] = cn;
            D[r0 + rel + 1] = dn;
        }
    }
    G::sync();

    // ---- B2: segment end rows (_calculate_matrix_coeff 469-592) and decoupling
    if (tid < nseg && sg.sn[tid] >= 0) {
        const int sn = sg.sn[tid];
        const int rowF = sg.ro[tid], rowL = rowF + sn;
        const R oA = A[rowL], oB = B[rowL], oC = Cc[rowL], oD = D[rowL];
        // the prescribed end levels (increments over z in the mixed form)
        const R tzl = MIX ? R(sg.tzl[tid] - sg.zl[tid]) : R(sg.tzl[tid]);
        const R tzr = MIX ? R(sg.tzr[tid] - sg.zr[tid]) : R(sg.tzr[tid]);
        if (!sg.br1[tid]) {
            if (sg.typeR[tid]) D[rowF] = D[rowF] - A[rowF] * bq_first;
            else D[rowF] = D[rowF] - A[rowF] * tzl;
        }
        // the end-row statement always rewrites AA, BB, DD of the last row; for a
        // single-row system that undoes the first-row override (UVZSolver_multithread.cu:574-590)
        A[rowL] = oA;
        B[rowL] = oB;
        const int kind = sg.lastKind[tid];
        if (kind == 1) D[rowL] = oD - oC * bq_last;
        else if (kind == 2) D[rowL] = oD - oC * tzr;
        else D[rowL] = oD;
        A[rowF] = R(0);
        Cc[rowL] = R(0);
    }
    G::sync();

    // ---- C: solve
    solve_line<G, SOLVER, R>(A, B, Cc, D, pl, Rn, red);

    // ---- D: extract (_uzSolver_extract_solution 668-723 / _vzSolver_extract_solution 595-665)
    const R* x = B;
    // a solved level: the unknown itself, or z + the increment in FP64 (mixed form); a
    // prescribed level as the rows use it
    auto put_z = [&](int pos, R xz) { g.t_z[pos] = MIX ? g.z[pos] + (double)xz : (double)xz; };
    auto row_z = [&](int pos) { return MIX ? R(g.t_z[pos] - g.z[pos]) : R(g.t_z[pos]); };
    const int QF = DIR == 0 ? g.bienQ[2] : g.bienQ[1];
    const int QL = DIR == 0 ? g.bienQ[3] : g.bienQ[0];
    for (int c = tid; c < C; c += T) {
        const int sI = seg_of(sg, c);
        const int f = sg.first[sI], l = sg.last[sI];
        const int k = f + (c - sg.co[sI]);
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        const int sn = sg.sn[sI];
        const int r0 = sg.ro[sI] - 2 * f;  // packed index of global row r is r0 + r
        const int qfirst = !b1f && QF && f == 2;
        const int pos = base + k * along;
        if (k < l) {
            if (b1f || qfirst) {
                put_z(pos, x[r0 + 2 * k]);
                tvel[pos] = x[r0 + 2 * k + 1];
                if (k == f) tvel[pos - along] = b1f ? R(0) : bq_first;
            } else if (k == f) {
                const R tv = x[r0 + 2 * f];
                tvel[pos] = tv;
                tvel[pos - along] = (ends[6 * sI + 2] - row_z(pos) - ends[6 * sI + 1] * tv) / ends[6 * sI];
            } else {
                put_z(pos, x[r0 + 2 * k - 1]);
                tvel[pos] = x[r0 + 2 * k];
            }
        } else {
            const R xl = sn >= 0 ? x[r0 + 2 * f + sn] : R(0);
            if (b2f) {
                tvel[pos] = R(0);
                put_z(pos, xl);
            } else if (QL && l == L) {
                tvel[pos] = bq_last;
                put_z(pos, xl);
            } else {
                R tprev;
                if (l > f) tprev = (b1f || qfirst) ? x[r0 + 2 * l - 1] : x[r0 + 2 * l - 2];
                else tprev = R(tvel[pos - along]);
                tvel[pos] = (ends[6 * sI + 5] - ends[6 * sI + 3] * tprev - row_z(pos)) / ends[6 * sI + 4];
            }
        }
    }
}

// The lines a sweep launch covers: lines start .. start + n - 1 of one grid, or the lines of
// every member of a batch in one list (member m's at list positions lstart[m] ..
// lstart[m + 1] - 1, its lines first[m] onwards).
struct OneGridLines {
    DevGrid g;
    DevParams p;
    int start, n;
    __device__ __forceinline__ int count() const { return n; }
    __device__ __forceinline__ void at(int li, int& m, int& line) const {
        m = 0;
        line = start + li;
    }
    __device__ __forceinline__ const DevGrid& grid(int) const { return g; }
    __device__ __forceinline__ const DevParams& params(int) const { return p; }
};

// Fused sweep of one direction.  CTA b takes lines b, b + G, b + 2G, ... (G = gridDim.x)
// in groups of 16, one line per warp.  Every warp sets its line up; a warp whose line is
// short (at most roww rows) sweeps it alone in its own slice of shared memory; then the
// whole CTA sweeps the group's long lines one after another in the full shared memory
// (RB rows; a CTA's region of global scratch beyond that).
// Adjacent long lines (a wet band) fall on different CTAs.  Warps with nothing to sweep
// wait at the CTA barriers rather than exit: the warp-synchronous steps of a warp whose
// sibling warps had exited were measured an order of magnitude slower on B200.
template <int DIR, int SOLVER, class R, class Lines>
__device__ __forceinline__ void hydro_sweep_loop(const Lines& lines, int RB, double* gscr_d, int RG, int roww) {
    constexpr bool MIX = sizeof(R) == sizeof(float);
    extern __shared__ double dyn_smem_d[];
    R* dyn_smem = reinterpret_cast<R*>(dyn_smem_d);
    R* gscr = reinterpret_cast<R*>(gscr_d);
    __shared__ LineShared sgw[kWL];
    __shared__ int s_long[kWL], s_mem[kWL], s_line[kWL];
    __shared__ int s_nlong;
    __shared__ R s_red[4 * kRedRows];  // reduced rows of the two-level solve
    const int w = threadIdx.x >> 5;
    const int nlines = lines.count();
    const int G = gridDim.x;
    for (int j0 = 0; (int)blockIdx.x + j0 * G < nlines; j0 += kWL) {
        const int li = blockIdx.x + (j0 + w) * G;
        LineShared& sg = sgw[w];
        int m = 0, line = 0;
        if (li < nlines) lines.at(li, m, line);
        if (threadIdx.x == 0) s_nlong = 0;
        if ((threadIdx.x & 31) == 0) {
            s_mem[w] = m;
            s_line[w] = line;
        }
        if (li < nlines) hydro_setup<DIR, WarpG, MIX>(lines.grid(m), lines.params(m), line, sg);  // warp-uniform
        __syncthreads();
        if (li < nlines && sg.nseg > 0) {
            if (sg.R > roww) {
                if ((threadIdx.x & 31) == 0) s_long[atomicAdd(&s_nlong, 1)] = w;
            } else {
                const int wr = slice_rows(roww);
                R* A = dyn_smem + w * (4 * wr + kEnds);
                R* B = A + wr;
                R* Cc = B + wr;
                R* D = Cc + wr;
                hydro_body<DIR, SOLVER, WarpG, R>(lines.grid(m), lines.params(m), line, sg, A, B, Cc, D, D + wr,
                                                  nullptr, SolvePlan{32, chunk_len(sg.R, 32)});
            }
        }
        __syncthreads();
        const int nl = s_nlong;
        for (int q = 0; q < nl; q++) {
            const int wl = s_long[q];
            const LineShared& sl = sgw[wl];
            const int lm = s_mem[wl];
            const SolvePlan pl = solve_plan(sl.R, SOLVER == 0 ? 256 : 32);
            const bool fits = pl.t1 * pl.m <= RB;
            const int rs = fits ? RB : RG;
            R* A = fits ? dyn_smem : gscr + (size_t)blockIdx.x * (4 * (size_t)RG + kEnds);
            R* B = A + rs;
            R* Cc = B + rs;
            R* D = Cc + rs;
            hydro_body<DIR, SOLVER, BlockG, R>(lines.grid(lm), lines.params(lm), s_line[wl], sl, A, B, Cc, D, D + rs,
                                               s_red, pl);
            __syncthreads();  // the slices and sgw are reused
        }
    }
}

template <int DIR, int SOLVER, class R>
__global__ void __launch_bounds__(kTL, 1) k_hydro_sweep(DevGrid g, DevParams p, int startidx, int endidx, int RB,
                                                     double* gscr_d, int RG, int roww) {
    hydro_sweep_loop<DIR, SOLVER, R>(OneGridLines{g, p, startidx, endidx - startidx + 1}, RB, gscr_d, RG, roww);
}
template <int DIR, int SOLVER, class R>
__global__ void __launch_bounds__(kTL, 1) k_hydro_sweep_b(BatchLines bl, int RB, double* gscr_d, int RG, int roww) {
    hydro_sweep_loop<DIR, SOLVER, R>(bl, RB, gscr_d, RG, roww);
}

// ---- sediment sweeps --------------------------------------------------------------

// The sediment rows in the arithmetic type R (double: the FP64 form; float: the mixed
// form).  Every operand is read in FP64 and taken to R at its use; the wet/dry tests on
// the depths compare the stored FP64 values, so both forms take the same branches.

// Row of the FSj system for one interior wet cell before the segment-end terms
// (_FSj_calculate__mactrix_coeff, Sediment_Transport.cu:205-302): aa, bb, cc, dd of the row,
// with the source S gated by t < bed_change_start.
template <class R>
__device__ __forceinline__ void fsj_cell_coeffs(const DevGrid& g, const DevParams& p, double t, int pos, R& aa, R& bb,
                                                R& cc, R& dd) {
    const int P = g.P;
    const double* FS = g.FS;
    const double* H = g.H_moi;
    // FSj runs right after the half-step's state update, which left u = t_u and v = t_v
    // on every cell it reads; reading u and v lets it run beside the next half-step's
    // sweeps, which write t_u and t_v
    const double *u = g.u, *v = g.v;
    // every operand first (one memory round trip; the branches below only select)
    const double Hd = H[pos], FSd = FS[pos], VTHd = g.VTH[pos], Fwd = g.Fw[pos];
    const double u0 = u[pos], u1 = u[pos - P], hu0 = g.Htdu[pos], hu1 = g.Htdu[pos - P], kx0 = g.Kx[pos],
                 kx1 = g.Kx[pos - P];
    const double Hm1 = H[pos - 1], Hp2 = H[pos + 2], Hm2 = H[pos - 2], Hp1 = H[pos + 1];
    const double FSp1 = FS[pos + 1], FSm1 = FS[pos - 1];
    const double hv0 = g.Htdv[pos], hv1 = g.Htdv[pos - 1], ky0 = g.Ky[pos], ky1 = g.Ky[pos - 1];
    const double v0 = v[pos], v1 = v[pos - 1];
    const R Hp = R(Hd), FSp = R(FSd), VTHp = R(VTHd);
    const double s_start = p.bed_change_start;
    const R sqrtg = sqrt(R(p.g));
    const R c = 18 * log(12 * Hp / R(p.Ks));
    const R Uf = sqrtg * fabs(VTHp) / c;
    const R fq = 1 - FSp;
    const R wsm = R(p.wss) * ((fq * fq) * (fq * fq));  // wss (1 - FS)^4
    R Zf = 0;
    R S;
    const R gamav = R(0.98) - R(0.198) * Zf + R(0.032) * Zf * Zf;  // evaluated before Zf (Sediment_Transport.cu:236)
    if (FSd > 0.00001) Zf = wsm / (R(0.4) * (Uf + 2 * wsm));
    if (p.ketdinh) S = source_chs<R>(p, wsm, Zf, FSp, R(Fwd), VTHp, Hp);
    else S = source_nchs<R>(p, wsm, Zf, Uf, Hp, FSp);
    if (t < s_start) S = 0;
    aa = -gamav * R(0.5) * (R(u0) + R(u1)) / R(p.dX2) - R(hu1) * R(kx1) / (Hp * (R(p.dXbp)));
    cc = gamav * R(0.5) * (R(u0) + R(u1)) / R(p.dX2) - R(hu0) * R(kx0) / (Hp * (R(p.dXbp)));
    bb = R(p.HaiChiadT) + (R(hu0) * R(kx0) + R(hu1) * R(kx1)) / (Hp * (R(p.dXbp)));
    R pp = 0, qq = 0;
    if ((Hm1 > p.H_TINH) && (Hp2 > p.H_TINH)) pp = R(FSp1 - FSd);
    if ((Hm2 > p.H_TINH) && (Hp1 > p.H_TINH)) qq = R(FSd - FSm1);
    pp = (1 / (Hp * R(p.dYbp))) * (R(hv0) * R(ky0) * pp - R(hv1) * R(ky1) * qq);
    if ((Hm2 > p.H_TINH) && (Hp2 > p.H_TINH)) {
        qq = R(FSp1 - FSm1) / R(p.dY2);
        qq = (R(v0) + R(v1)) * R(0.5) * qq * gamav;
    } else
        qq = 0;
    dd = FSp / (R(p.dT) * R(0.5)) - qq + pp + (S / Hp);
}

// Row of the FSi system for one interior wet cell before the segment-end terms
// (_FSi_calculate__mactrix_coeff, Sediment_Transport.cu:62-165).  The terms that depend on
// the cell alone (gamav and the gated source over the depth, rowC arrays 0 and 1) were
// computed by the state update that precedes the sweep (fsi_cell_terms).
template <class R>
__device__ __forceinline__ void fsi_cell_coeffs(const DevGrid& g, const DevParams& p, int pos, R& aa, R& bb, R& cc,
                                                R& dd) {
    const int P = g.P;
    const double* FS = g.FS;
    const double* H = g.H_moi;
    // every operand first (one memory round trip; the branches below only select)
    const double Hd = H[pos], FSd = FS[pos];
    const R gamav = rowCr<R>(g, 0)[pos], src = rowCr<R>(g, 1)[pos];
    const double tv0 = g.t_v[pos], tv1 = g.t_v[pos - 1], hv0 = g.Htdv[pos], hv1 = g.Htdv[pos - 1], ky0 = g.Ky[pos],
                 ky1 = g.Ky[pos - 1];
    const double Hp2 = H[pos + 2 * P], Hm1 = H[pos - P], Hm2 = H[pos - 2 * P], Hp1 = H[pos + P];
    const double FSp1 = FS[pos + P], FSm1 = FS[pos - P];
    const double hu0 = g.Htdu[pos], hu1 = g.Htdu[pos - P], kx0 = g.Kx[pos], kx1 = g.Kx[pos - P];
    const double tu0 = g.t_u[pos], tu1 = g.t_u[pos - P];
    const R Hp = R(Hd);
    aa = -gamav * R(0.5) * (R(tv1) + R(tv0)) / R(p.dY2) - R(hv1) * R(ky1) / (Hp * R(p.dYbp));
    cc = gamav * R(0.5) * (R(tv1) + R(tv0)) / R(p.dY2) - R(hv0) * R(ky0) / (Hp * R(p.dYbp));
    bb = R(p.HaiChiadT) + (R(hv0) * R(ky0) + R(hv1) * R(ky1)) / (Hp * R(p.dYbp));
    R pp = 0, qq = 0;
    if ((Hp2 > p.H_TINH) && (Hm1 > p.H_TINH)) pp = R(FSp1 - FSd);
    if (Hm2 > p.H_TINH && Hp1 > p.H_TINH) qq = R(FSd - FSm1);
    pp = (1 / (Hp * R(p.dXbp))) * (R(hu0) * R(kx0) * pp - R(hu1) * R(kx1) * qq);
    if (Hp2 > p.H_TINH && Hm2 > p.H_TINH) {
        qq = R(FSp1 - FSm1) / R(p.dX2);
        qq = (R(tu0) + R(tu1)) * R(0.5) * qq * gamav;
    } else
        qq = 0;
    dd = R(FSd) / (R(p.dT) * R(0.5)) - qq + pp + src;
}

// FSj rows of every interior wet cell (columns 3..M-1), one warp per row of the grid over
// the row's span, written column-major (colT arrays 0..3 in R: aa bb cc dd), with TILE
// through a tile.
template <int TILE, class R>
__device__ __forceinline__ void coef_fsj_body(const DevGrid& g, const DevParams& p, int half, int bx) {
    const double t = g.clock[half];
    if constexpr (!TILE) {
        const int i = 2 + ((bx * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
        if (i > g.N) return;
        const int lo = max(g.rlo[i], 3), hi = min(g.rhi[i], g.M - 1);
        for (int j = lo + lane; j <= hi; j += 32) {
            const int pos = i * g.P + j;
            if (g.khouot[pos] != 0) continue;
            R aa, bb, cc, dd;
            fsj_cell_coeffs<R>(g, p, t, pos, aa, bb, cc, dd);
            const size_t q = (size_t)j * g.LT + i;
            colTr<R>(g, 0)[q] = aa;
            colTr<R>(g, 1)[q] = bb;
            colTr<R>(g, 2)[q] = cc;
            colTr<R>(g, 3)[q] = dd;
        }
    } else {
        R* const dst[4] = {colTr<R>(g, 0), colTr<R>(g, 1), colTr<R>(g, 2), colTr<R>(g, 3)};
        colmajor_tile<4>(
            g, 2 + kTileRows * bx, g.N, 3, g.M - 1,
            [&](int i, int j, R* v) {
                const int pos = i * g.P + j;
                if (g.khouot[pos] != 0) return false;
                fsj_cell_coeffs<R>(g, p, t, pos, v[0], v[1], v[2], v[3]);
                return true;
            },
            dst);
    }
}

template <int TILE, class R>
__global__ void __launch_bounds__(256) k_coef_fsj(DevGrid g, DevParams p, int half) {
    coef_fsj_body<TILE, R>(g, p, half, blockIdx.x);
}
template <int TILE, class R>
__global__ void __launch_bounds__(256) k_coef_fsj_b(BatchRef br, int half) {
    const BatchMember bm(br);
    coef_fsj_body<TILE, R>(bm.g, bm.p, half, bm.bx);
}

// Segments of a sediment line and their row offsets (one row per interior cell
// first+1..last-1, the reference's SN+1 rows).
template <int DIR, class G>
__device__ __forceinline__ void fs_setup(const DevGrid& g, const DevParams& p, int line, LineShared& sg) {
    const int tid = G::rank();
    const int nseg = DIR == 0 ? g.mocj[line] : g.moci[line];
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
    G::sync();
    if (tid == 0) {
        int r = 0;
        for (int s = 0; s < nseg; s++) {
            sg.ro[s] = r;
            const int n = sg.last[s] - sg.first[s] - 1;
            if (n > 0) r += n;
        }
        sg.ro[nseg] = r;
        sg.R = r;
        sg.nseg = nseg;
    }
    G::sync();
}

// Rows, solve and extraction of one sediment line (_FSi/_FSj_calculate__mactrix_coeff
// and _FSi/_FSj_extract_solution, Sediment_Transport.cu:62-340, driven by Scan_FSi/
// Scan_FSj and FSi/FSj_extract_solution 570-618).  DIR 0: FSj (line = column j, cells
// i), DIR 1: FSi (line = row i, cells j).
template <int DIR, int SOLVER, class G, class R>
__device__ __forceinline__ void fs_body(const DevGrid& g, const DevParams& p, int half, int line,
                                        const LineShared& sg, R* A, R* B, R* Cc, R* D, R* red, SolvePlan pl) {
    constexpr int T = G::size;
    const int tid = G::rank();
    const int P = g.P;
    const int along = DIR == 0 ? P : 1;
    const int base = DIR == 0 ? line : line * P;
    (void)half;  // both rows are precomputed (k_coef_fsj, the state update's FSi terms)
    const int Rn = sg.R;
    for (int r = Rn + tid; r < pl.t1 * pl.m; r += T) {  // identity rows up to the solver's rows
        A[r] = R(0);
        B[r] = R(1);
        Cc[r] = R(0);
        D[r] = R(0);
    }
    const double* FS = g.FS;
    for (int rr = tid; rr < Rn; rr += T) {
        const int sI = seg_of_row(sg, rr);
        const int f = sg.first[sI], l = sg.last[sI];
        const int k = f + 1 + (rr - sg.ro[sI]);
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        const int pos = base + k * along;
        R aa, bb, cc, dd;
        if (DIR == 0) {  // precomputed by k_coef_fsj
            const size_t q = (size_t)line * g.LT + k;
            aa = colTr<R>(g, 0)[q];
            bb = colTr<R>(g, 1)[q];
            cc = colTr<R>(g, 2)[q];
            dd = colTr<R>(g, 3)[q];
            if (k == f + 1) {
                if (b1f || g.u[base + f * along] == 0) bb += aa;
                else dd -= aa * R(FS[base + f * along]);
            }
            if (k == l - 1) {
                if (b2f && g.u[base + l * along] == 0) bb += cc;
                else dd -= cc * R(FS[base + l * along]);
            }
        } else {
            fsi_cell_coeffs<R>(g, p, pos, aa, bb, cc, dd);
            if (k == f + 1) {
                if (b1f || g.t_v[base + f * along] == 0) bb = bb + aa;
                else dd = dd - aa * R(FS[base + f * along]);
            }
            if (k == l - 1) {
                if (b2f || g.t_v[base + l * along] == 0) bb = bb + cc;
                else dd = dd - cc * R(FS[base + l * along]);
            }
        }
        A[rr] = (k == f + 1) ? R(0) : aa;
        B[rr] = bb;
        Cc[rr] = (k == l - 1) ? R(0) : cc;
        D[rr] = dd;
    }
    G::sync();
    solve_line<G, SOLVER, R>(A, B, Cc, D, pl, Rn, red);
    const R* x = B;
    const double* vel = DIR == 0 ? g.u : g.t_v;  // FSj: u = t_u here (see fsj_cell_coeffs)
    for (int c = tid; c < Rn; c += T) {
        const int sI = seg_of_row(sg, c);
        const int f = sg.first[sI], l = sg.last[sI];
        const int k = f + 1 + (c - sg.ro[sI]);
        const int b1f = sg.br1[sI], b2f = sg.br2[sI];
        const int pos = base + k * along;
        double xv = x[c];
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

// Fused sediment sweep of one direction: as k_hydro_sweep.
template <int DIR, int SOLVER, class R, class Lines>
__device__ __forceinline__ void fs_sweep_loop(const Lines& lines, int half, int RB, double* gscr_d, int RG, int roww) {
    extern __shared__ double dyn_smem_d[];
    R* dyn_smem = reinterpret_cast<R*>(dyn_smem_d);
    R* gscr = reinterpret_cast<R*>(gscr_d);
    __shared__ LineShared sgw[kWL];
    __shared__ int s_long[kWL], s_mem[kWL], s_line[kWL];
    __shared__ int s_nlong;
    __shared__ R s_red[4 * kRedRows];  // reduced rows of the two-level solve
    const int w = threadIdx.x >> 5;
    const int nlines = lines.count();
    const int G = gridDim.x;
    for (int j0 = 0; (int)blockIdx.x + j0 * G < nlines; j0 += kWL) {
        const int li = blockIdx.x + (j0 + w) * G;
        LineShared& sg = sgw[w];
        int m = 0, line = 0;
        if (li < nlines) lines.at(li, m, line);
        if (threadIdx.x == 0) s_nlong = 0;
        if ((threadIdx.x & 31) == 0) {
            s_mem[w] = m;
            s_line[w] = line;
        }
        if (li < nlines) fs_setup<DIR, WarpG>(lines.grid(m), lines.params(m), line, sg);  // warp-uniform
        __syncthreads();
        if (li < nlines && sg.R > 0) {
            if (sg.R > roww) {
                if ((threadIdx.x & 31) == 0) s_long[atomicAdd(&s_nlong, 1)] = w;
            } else {
                const int wr = slice_rows(roww);
                R* A = dyn_smem + w * 4 * wr;
                fs_body<DIR, SOLVER, WarpG, R>(lines.grid(m), lines.params(m), half, line, sg, A, A + wr, A + 2 * wr,
                                               A + 3 * wr, nullptr, SolvePlan{32, chunk_len(sg.R, 32)});
            }
        }
        __syncthreads();
        const int nl = s_nlong;
        for (int q = 0; q < nl; q++) {
            const int wl = s_long[q];
            const LineShared& sl = sgw[wl];
            const int lm = s_mem[wl];
            const SolvePlan pl = solve_plan(sl.R, SOLVER == 0 ? 256 : 32);
            const bool fits = pl.t1 * pl.m <= RB;
            const int rs = fits ? RB : RG;
            R* A = fits ? dyn_smem : gscr + (size_t)blockIdx.x * 4 * (size_t)RG;
            fs_body<DIR, SOLVER, BlockG, R>(lines.grid(lm), lines.params(lm), half, s_line[wl], sl, A, A + rs,
                                            A + 2 * rs, A + 3 * rs, s_red, pl);
            __syncthreads();
        }
    }
}

template <int DIR, int SOLVER, class R>
__global__ void __launch_bounds__(kTL, 1) k_fs_sweep(DevGrid g, DevParams p, int half, int startidx, int endidx, int RB,
                                                  double* gscr_d, int RG, int roww) {
    fs_sweep_loop<DIR, SOLVER, R>(OneGridLines{g, p, startidx, endidx - startidx + 1}, half, RB, gscr_d, RG, roww);
}
template <int DIR, int SOLVER, class R>
__global__ void __launch_bounds__(kTL, 1) k_fs_sweep_b(BatchLines bl, int half, int RB, double* gscr_d, int RG,
                                                    int roww) {
    fs_sweep_loop<DIR, SOLVER, R>(bl, half, RB, gscr_d, RG, roww);
}

// Largest dynamic shared memory the kernel may be given on this device.
int max_dyn_smem(const void* f) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, f) != cudaSuccess) return 48 * 1024;
    return optin - (int)a.sharedSizeBytes;
}

template <class F>
cudaError_t allow_all(F* const* fs, int n, int* limit) {
    int lim = 1 << 30;
    for (int i = 0; i < n; i++) {
        const int mx = max_dyn_smem((const void*)fs[i]);
        const cudaError_t e = cudaFuncSetAttribute((const void*)fs[i], cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (e != cudaSuccess) return e;
        if (mx < lim) lim = mx;
    }
    *limit = lim;
    return cudaSuccess;
}

using HydroSweepFn = void(DevGrid, DevParams, int, int, int, double*, int, int);
using FsSweepFn = void(DevGrid, DevParams, int, int, int, int, double*, int, int);
using HydroSweepBFn = void(BatchLines, int, double*, int, int);
using FsSweepBFn = void(BatchLines, int, int, double*, int, int);

// [precision: 0 FP64, 1 mixed][direction][solver]
HydroSweepFn* const kHydroSweep[2][2][2] = {
    {{k_hydro_sweep<0, 0, double>, k_hydro_sweep<0, 1, double>},
     {k_hydro_sweep<1, 0, double>, k_hydro_sweep<1, 1, double>}},
    {{k_hydro_sweep<0, 0, float>, k_hydro_sweep<0, 1, float>},
     {k_hydro_sweep<1, 0, float>, k_hydro_sweep<1, 1, float>}}};
FsSweepFn* const kFsSweep[2][2][2] = {
    {{k_fs_sweep<0, 0, double>, k_fs_sweep<0, 1, double>}, {k_fs_sweep<1, 0, double>, k_fs_sweep<1, 1, double>}},
    {{k_fs_sweep<0, 0, float>, k_fs_sweep<0, 1, float>}, {k_fs_sweep<1, 0, float>, k_fs_sweep<1, 1, float>}}};

}  // namespace

// Shared-memory sizes and the long-line grid of a grid of N x M cells on the current
// device; opts the sweep kernels into the shared memory they may need.  max_rows > 0 caps
// the rows a long line may hold in shared memory (longer lines then run in global scratch).
cudaError_t sweep_plan(int N, int M, SweepPlan* sp, int max_rows) {
    cudaError_t e;
    int lim_h, lim_f;
    // the row counts below are planned for FP64 rows; the mixed form's FP32 rows take half
    // the bytes of the same plan
    if ((e = allow_all(&kHydroSweep[0][0][0], 8, &lim_h)) != cudaSuccess) return e;
    if ((e = allow_all(&kFsSweep[0][0][0], 8, &lim_f)) != cudaSuccess) return e;
    const int L = N > M ? N : M;
    const size_t warp_h = (size_t)kWL * kWarpHydro, warp_f = (size_t)kWL * kWarpFs;  // short-line slices
    if ((long long)(sizeof(double) * warp_h) > lim_h || (long long)(sizeof(double) * warp_f) > lim_f)
        return cudaErrorInvalidValue;
    // every row a line can have: rows <= 2 L + 20 (solved by 32 lanes)
    {
        int rg = 0;
        for (int t1 = 32; t1 <= 256; t1 <<= 1) {  // the padded rows of any solve plan
            const int r = t1 * chunk_len(2 * L + HYD_SEGL, t1);
            if (r > rg) rg = r;
        }
        sp->RG = rg;
    }
    sp->need_global = 0;
    sp->wide = 0;
    if ((long long)(sizeof(double) * (4 * (size_t)sp->RG + kEnds)) <= lim_h) {
        sp->RB = sp->RG;
    } else {  // as many rows as fit; longer lines use global scratch
        sp->RB = (int)((lim_h / (int)sizeof(double) - kEnds) / 4);
        sp->need_global = 1;
    }
    if (max_rows > 0 && sp->RB > max_rows) {
        sp->RB = max_rows;
        sp->need_global = 1;
    }
    size_t big = 4 * (size_t)sp->RB + kEnds;
    sp->smem_lines = sizeof(double) * (big > warp_h ? big : warp_h);
    sp->RGf = 0;
    for (int t1 = 32; t1 <= 256; t1 <<= 1) {
        const int r = t1 * chunk_len(L, t1);
        if (r > sp->RGf) sp->RGf = r;
    }
    if ((long long)(sizeof(double) * 4 * (size_t)sp->RGf) <= lim_f) {
        sp->RBf = sp->RGf;
    } else {
        sp->RBf = (int)((lim_f / (int)sizeof(double)) / 4);
        sp->need_global = 1;
    }
    if (max_rows > 0 && sp->RBf > max_rows) {
        sp->RBf = max_rows;
        sp->need_global = 1;
    }
    big = 4 * (size_t)sp->RBf;
    sp->smem_fs_lines = sizeof(double) * (big > warp_f ? big : warp_f);
    int dev = 0, nsm = 0, occ = 0, occf = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kHydroSweep[0][0][0], kTL, sp->smem_lines)) !=
        cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occf, kFsSweep[0][0][0], kTL, sp->smem_fs_lines)) !=
        cudaSuccess)
        return e;
    if (occ < 1) occ = 1;
    if (occf < 1) occf = 1;
    sp->long_grid = nsm * (occ < occf ? occ : occf);
    if (sp->long_grid > L + 3) sp->long_grid = L + 3;
    sp->scratch_doubles =
        sp->need_global ? (size_t)sp->long_grid * (4 * (size_t)(sp->RG > sp->RGf ? sp->RG : sp->RGf) + kEnds) : 1;
    return cudaSuccess;
}

void sweep_plan_throughput(int N, int M, SweepPlan* sp) {
    const int L = N > M ? N : M;
    const int g = (L + 3 + kWL - 1) / kWL;
    if (sp->long_grid > g) sp->long_grid = g;
    sp->wide = 1;
}

namespace {
void hydro_sweep(int dir, const DevGrid& g, const DevParams& p, const SweepPlan& sp, int startidx, int endidx,
                 int solver, double* scratch, cudaStream_t s) {
    const int nlines = endidx - startidx + 1;
    if (nlines <= 0) return;
    const int sv = solver ? 1 : 0;
    const int roww = (sp.wide || nlines > kWL * sp.long_grid) ? kRowW : kRowShort;
    // the long-line rows or the warps' slices, whichever is larger (a smaller request
    // leaves more of the SM's on-chip memory to L1)
    const size_t big = 4 * (size_t)sp.RB + kEnds, slices = (size_t)kWL * (4 * slice_rows(roww) + kEnds);
    const size_t esz = p.mixed ? sizeof(float) : sizeof(double);
    const size_t smem = esz * (big > slices ? big : slices);
    kHydroSweep[p.mixed ? 1 : 0][dir][sv]<<<sp.long_grid, kTL, smem, s>>>(g, p, startidx, endidx, sp.RB, scratch,
                                                                         sp.RG, roww);
    hyd_kernel_launches_add(1);
}

void fs_sweep(int dir, const DevGrid& g, const DevParams& p, const SweepPlan& sp, int half, int startidx,
              int endidx, int solver, double* scratch, cudaStream_t s) {
    const int nlines = endidx - startidx + 1;
    if (nlines <= 0) return;
    const int sv = solver ? 1 : 0;
    const int roww = (sp.wide || nlines > kWL * sp.long_grid) ? kRowW : kRowShortF;
    const size_t big = 4 * (size_t)sp.RBf, slices = (size_t)kWL * 4 * slice_rows(roww);
    const size_t esz = p.mixed ? sizeof(float) : sizeof(double);
    const size_t smem = esz * (big > slices ? big : slices);
    kFsSweep[p.mixed ? 1 : 0][dir][sv]<<<sp.long_grid, kTL, smem, s>>>(g, p, half, startidx, endidx, sp.RBf, scratch,
                                                                      sp.RGf, roww);
    hyd_kernel_launches_add(1);
}
}  // namespace

void launch_coef_fsj(const DevGrid& g, const DevParams& p, int half, cudaStream_t s) {
    const int nb = ((g.N - 1) * 32 + 255) / 256;
    if (p.mixed) {
        if (g.tile_cols) k_coef_fsj<1, float><<<nb, 256, 0, s>>>(g, p, half);
        else k_coef_fsj<0, float><<<nb, 256, 0, s>>>(g, p, half);
    } else {
        if (g.tile_cols) k_coef_fsj<1, double><<<nb, 256, 0, s>>>(g, p, half);
        else k_coef_fsj<0, double><<<nb, 256, 0, s>>>(g, p, half);
    }
    hyd_kernel_launches_add(1);
}

void launch_sweep_uz(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int startidx, int endidx,
                     int solver, double* scratch, cudaStream_t s) {
    hydro_sweep(0, g, p, sp, startidx, endidx, solver, scratch, s);
}

void launch_sweep_vz(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int startidx, int endidx,
                     int solver, double* scratch, cudaStream_t s) {
    hydro_sweep(1, g, p, sp, startidx, endidx, solver, scratch, s);
}

// FSj over columns 3..M-1 (Engine.py:224-237), FSi over rows 3..N-1 (Engine.py:345-358).
void launch_fs_sweep_j(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int half, int solver,
                       double* scratch, cudaStream_t s) {
    fs_sweep(0, g, p, sp, half, 3, g.M - 1, solver, scratch, s);
}

void launch_fs_sweep_i(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int half, int solver,
                       double* scratch, cudaStream_t s) {
    fs_sweep(1, g, p, sp, half, 3, g.N - 1, solver, scratch, s);
}

// ---- batched sweeps: every member's lines in one persistent launch (the common plan of
// the batch: rows kept in shared memory, warp tier wide)
void launch_sweep_batch(int dir, const BatchLines& bl, const SweepPlan& sp, int solver, int mixed, double* scratch,
                        int grid, cudaStream_t s) {
    const int sv = solver ? 1 : 0;
    const int roww = kRowW;
    const size_t big = 4 * (size_t)sp.RB + kEnds, slices = (size_t)kWL * (4 * slice_rows(roww) + kEnds);
    const size_t smem = (mixed ? sizeof(float) : sizeof(double)) * (big > slices ? big : slices);
    if (mixed) {
        if (dir == 0) {
            if (sv) k_hydro_sweep_b<0, 1, float><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
            else k_hydro_sweep_b<0, 0, float><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
        } else {
            if (sv) k_hydro_sweep_b<1, 1, float><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
            else k_hydro_sweep_b<1, 0, float><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
        }
    } else {
        if (dir == 0) {
            if (sv) k_hydro_sweep_b<0, 1, double><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
            else k_hydro_sweep_b<0, 0, double><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
        } else {
            if (sv) k_hydro_sweep_b<1, 1, double><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
            else k_hydro_sweep_b<1, 0, double><<<grid, kTL, smem, s>>>(bl, sp.RB, scratch, sp.RG, roww);
        }
    }
    hyd_kernel_launches_add(1);
}

void launch_fs_sweep_batch(int dir, const BatchLines& bl, const SweepPlan& sp, int half, int solver, int mixed,
                           double* scratch, int grid, cudaStream_t s) {
    const int sv = solver ? 1 : 0;
    const int roww = kRowW;
    const size_t big = 4 * (size_t)sp.RBf, slices = (size_t)kWL * 4 * slice_rows(roww);
    const size_t smem = (mixed ? sizeof(float) : sizeof(double)) * (big > slices ? big : slices);
    if (mixed) {
        if (dir == 0) {
            if (sv) k_fs_sweep_b<0, 1, float><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
            else k_fs_sweep_b<0, 0, float><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
        } else {
            if (sv) k_fs_sweep_b<1, 1, float><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
            else k_fs_sweep_b<1, 0, float><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
        }
    } else {
        if (dir == 0) {
            if (sv) k_fs_sweep_b<0, 1, double><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
            else k_fs_sweep_b<0, 0, double><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
        } else {
            if (sv) k_fs_sweep_b<1, 1, double><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
            else k_fs_sweep_b<1, 0, double><<<grid, kTL, smem, s>>>(bl, half, sp.RBf, scratch, sp.RGf, roww);
        }
    }
    hyd_kernel_launches_add(1);
}

void launch_coef_fsj_batch(const BatchRef& br, int ctas, int half, int mixed, cudaStream_t s) {
    if (mixed) k_coef_fsj_b<0, float><<<ctas, 256, 0, s>>>(br, half);
    else k_coef_fsj_b<0, double><<<ctas, 256, 0, s>>>(br, half);
    hyd_kernel_launches_add(1);
}

// The batched sweeps may use all the shared memory the device allows (their row plans
// are the largest member's).
cudaError_t batch_sweep_setup() {
    HydroSweepBFn* const hb[8] = {k_hydro_sweep_b<0, 0, double>, k_hydro_sweep_b<0, 1, double>,
                                 k_hydro_sweep_b<1, 0, double>, k_hydro_sweep_b<1, 1, double>,
                                 k_hydro_sweep_b<0, 0, float>,  k_hydro_sweep_b<0, 1, float>,
                                 k_hydro_sweep_b<1, 0, float>,  k_hydro_sweep_b<1, 1, float>};
    FsSweepBFn* const fb[8] = {k_fs_sweep_b<0, 0, double>, k_fs_sweep_b<0, 1, double>, k_fs_sweep_b<1, 0, double>,
                              k_fs_sweep_b<1, 1, double>, k_fs_sweep_b<0, 0, float>,  k_fs_sweep_b<0, 1, float>,
                              k_fs_sweep_b<1, 0, float>,  k_fs_sweep_b<1, 1, float>};
    int lim;
    cudaError_t e = allow_all(hb, 8, &lim);
    if (e == cudaSuccess) e = allow_all(fb, 8, &lim);
    return e;
}
