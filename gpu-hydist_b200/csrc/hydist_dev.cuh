// hydist_dev.cuh — device-side state, parameters and helpers of the B200 ADI library.
//
// Layout in HBM: every (N+3) x (M+3) grid field of the reference (Argument_Pointers,
// constant.cuh:6-20) is stored row-major with a pitch P >= M+3 that is a multiple of
// 32 doubles (256 B), so every row starts on a 256-byte boundary.  Element (i, j) is
// at i*P + j; i is the x / "N" direction (u faces, dX), j the y / "M" direction
// (v faces, dY).  Segment tables keep the reference's [line][20] layout.
#pragma once

#include <cstdint>

#define HYD_SEGL 20
#define HYD_MAX_LINE 25000  // largest N or M (a line is staged in shared memory)

// Device status bits (read back by hyd_synchronize).
#define HYD_ST_SEG_OVERFLOW 1u     // more than 20 wet segments on a line
#define HYD_ST_INTERP_RANGE 2u     // edge FS interpolation index left the grid
#define HYD_ST_DEGENERATE 4u       // single-cell segment on an open edge (reference reads stale scratch)
#define HYD_ST_EDGE_REACH 8u       // an edge FS interpolation read the opposite edge row (order-dependent)
#define HYD_ST_STAGE_RANGE 16u     // a line's staged span exceeded its shared-memory bound (not run)

struct DevParams {
    double dX, dY, dT, dXbp, dX2, dYbp, dY2, dTchia2dX, dTchia2dY, HaiChiadT;
    double NANGDAY, H_TINH, heso, mu_mn, NDnen, Tod, Toe, hstoe, ghtoe, Mbochat, ro, ros, dm,
        Dorong, Sx, CORIOLIS_FORCE, g, Ks;
    // device helpers of constant.cuh:126-133, evaluated once
    double windx, windy, ufr, dxr, wss;
    double dxr_m03;  // pow(dxr, -0.3), a constant of the source and bed-load formulas
    double sediment_start, bed_change_start;
    int ketdinh, kenhhepd, kenhhepng, channel;
    // morphodynamic feedback (off: the reference's step): each Exner update's bed change,
    // morfac x bed_period / (1 - Dorong) x rate, is applied to h and the depths re-derived
    int bed_feedback;
    int bed_fixed;         // the bed stays fixed within bed_fixed cells of the grid's edges
    double bed_min_depth;  // and where the water is shallower than this
    double morfac, bed_period;  // bed_period: the Exner period in s (bed_change_start if unset)
    // precision_mode MIXED: coefficient assembly, the line sweeps, the explicit momentum and
    // the sediment transport in FP32; the water level's continuity update, the mass sums
    // and the Exner accumulation in FP64
    int mixed;
};

struct DevGrid {
    int N, M, P;
    int total_time;
    // grid fields (pitch P)
    double *h, *hsnham, *VISC, *Fw, *Tsxw, *Tsyw;
    double *u, *v, *z, *t_u, *t_v, *t_z;
    double *Htdu, *Htdv, *H_moi, *htaiz, *htaiz_bd, *Kx1, *Ky1;
    double *FS, *tFS, *VTH, *Kx, *Ky, *Qbx, *Qby, *dH;
    double *h0, *dHc;  // feedback: h at set-up (h = h0 + dH) and dH's Kahan compensation
    double* dHinc;     // feedback: an update's unfiltered bed change (NaN where none)
    int* khouot;
    // segment tables (reference layout)
    int *daui, *cuoii, *moci, *dauj, *cuoij, *mocj;
    // boundary data
    double *ubt, *ubp, *vbt, *vbd, *hi, *hmax;  // hmax[4]: 1/(ros*hmax) per edge (up, down, left, right)
    int *bienQ, *btype;                          // bienQ[4], btype[4*20]
    double *bc[4], *cc[4];                       // [nseg][total_time] per edge
    unsigned* status;
    // span of the cells whose mask is not 2 (those never change) per row / column
    int *rlo, *rhi, *clo, *chi;
    // extended span per row (every cell within a few cells of those), where the
    // elementwise kernels run once the whole grid has been brought up to date
    int *elo, *ehi;
    int* span_wide;  // set when a velocity lies outside the extended spans
    int* dflag;      // scratch flag of the set-field check
    // lines whose mask changed since their segments were scanned: flags and lists
    int *dirty_r, *dirty_c, *dlist_r, *dlist_c;
    unsigned* dctr;  // [0] listed rows, [1] listed columns, [2] [3] CTAs of the rescans done
    // column-major copies of per-cell quantities for the column sweeps: 7 arrays of
    // (M+3) columns x LT rows (LT = N+3 rounded up to 32), array k at colT + k*colT_stride
    double* colT;
    unsigned char* colB;  // column-major reset bytes of the column resets (stride LT)
    double* rowC;         // row-major VZ coefficients, 7 arrays of (N+3) x P
    // the mixed form's FP32 copies of colT and rowC (same layout and strides; null in FP64)
    float* colTf;
    float* rowCf;
    size_t rowC_stride;
    size_t colT_stride;
    int LT;
    int wpr;  // warps per row of the extended-span kernels (1 until the spans are known)
    // doubles of shared memory the explicit-momentum kernels stage a row (sv_cap) or column
    // (su_cap) in: the longest span of cells that are not land, plus the three cells around
    // the segments they read or write (M + 3 / N + 3 until the spans are known)
    int sv_cap, su_cap;
    // column-major stores through shared-memory tiles (colmajor_tile): set for grids whose
    // column-major arrays are too large to stay in L2, where one 32-byte sector per stored
    // value costs DRAM traffic; smaller grids store straight from the per-row warps
    int tile_cols;
    double* clock;  // [0] time of half-step 1, [1] time of half-step 2, [2] time at the step start
    // water volume budget since hyd_init (kBud* slots): per edge the net, gross inflow and
    // gross outflow volumes through its faces as the sweeps' continuity rows used them, each
    // a Kahan sum with its compensation; the volumes of cells opened and closed by the
    // wet/dry resets (depth sums, atomically added)
    double* budget;
};

// Slots of DevGrid::budget.  Edge e = 0 up, 1 down, 2 left, 3 right.  An edge's half-step
// volumes are summed by kEdgeCtas CTAs, each writing its (in, out) partial to kBudPart +
// 2 (e kEdgeCtas + c); the last CTA of the edge to finish (counted in the unsigned words
// at kBudCount) adds the partials in CTA order to the edge's Kahan sums.
constexpr int kBudNet = 0, kBudNetC = 4, kBudIn = 8, kBudInC = 12, kBudOut = 16, kBudOutC = 20;
constexpr int kBudOpen = 24, kBudClose = 25, kBudBed = 26, kBudJump = 27, kBudLeak = 28;
constexpr int kEdgeCtas = 8, kBudPart = 32, kBudCount = kBudPart + 8 * kEdgeCtas, kBudSlots = kBudCount + 4;
// the budget CTAs of a half-step: kEdgeCtas per edge
constexpr int kBudCtas = 4 * kEdgeCtas;

__device__ __forceinline__ void flag_status(const DevGrid& g, unsigned bit) { atomicOr(g.status, bit); }

// CTAs of 256 threads that give each of `rows` rows g.wpr warps (the extended-span kernels).
__host__ __device__ __forceinline__ int row_warp_ctas(const DevGrid& g, int rows) {
    return (rows * g.wpr * 32 + 255) / 256;
}

// A batch of reaches stepped by batched launches: member m's grid and parameters (device
// arrays), and for one launch the first CTA of each member's share (bstart[m], with
// bstart[nm] the launch's CTAs).  Every CTA of a batched launch works for one member.
struct BatchRef {
    const DevGrid* __restrict__ g;  // read-only during a launch: loads of it need not be repeated
    const DevParams* __restrict__ p;
    const int* __restrict__ bstart;
    int nm;
};

// The last m with bstart[m] <= b.
__device__ __forceinline__ int batch_member_of(const int* bstart, int nm, int b) {
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bstart[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The lines of a batched sweep: every member's lines in one list (member m's at list
// positions lstart[m] .. lstart[m + 1] - 1, its lines first[m] onwards).
struct BatchLines {
    const DevGrid* __restrict__ g;
    const DevParams* __restrict__ p;
    const int* __restrict__ lstart;
    const int* __restrict__ first;
    int nm;
    __device__ __forceinline__ int count() const;
    __device__ __forceinline__ void at(int li, int& m, int& line) const;
    __device__ __forceinline__ const DevGrid& grid(int m) const { return g[m]; }
    __device__ __forceinline__ const DevParams& params(int m) const { return p[m]; }
};

__device__ __forceinline__ int BatchLines::count() const { return lstart[nm]; }
__device__ __forceinline__ void BatchLines::at(int li, int& m, int& line) const {
    m = batch_member_of(lstart, nm, li);
    line = first[m] + (li - lstart[m]);
}

// This CTA's member, and its index bx among the member's gx CTAs (what blockIdx.x and
// gridDim.x are in a launch for that member alone).
struct BatchMember {
    int m, bx, gx;
    const DevGrid& g;
    const DevParams& p;
    __device__ __forceinline__ explicit BatchMember(const BatchRef& br)
        : m(batch_member_of(br.bstart, br.nm, (int)blockIdx.x)),
          bx((int)blockIdx.x - br.bstart[m]),
          gx(br.bstart[m + 1] - br.bstart[m]),
          g(br.g[m]),
          p(br.p[m]) {}
};

// Column-major copy k of a per-cell quantity; (row i, column j) is at [j * g.LT + i].
__device__ __forceinline__ double* colT(const DevGrid& g, int k) { return g.colT + (size_t)k * g.colT_stride; }
__device__ __forceinline__ double* rowC(const DevGrid& g, int k) { return g.rowC + (size_t)k * g.rowC_stride; }
// The same arrays in the arithmetic type R of a kernel instantiation (float: the mixed form's copies).
template <class R>
__device__ __forceinline__ R* colTr(const DevGrid& g, int k);
template <>
__device__ __forceinline__ double* colTr<double>(const DevGrid& g, int k) { return colT(g, k); }
template <>
__device__ __forceinline__ float* colTr<float>(const DevGrid& g, int k) { return g.colTf + (size_t)k * g.colT_stride; }
template <class R>
__device__ __forceinline__ R* rowCr(const DevGrid& g, int k);
template <>
__device__ __forceinline__ double* rowCr<double>(const DevGrid& g, int k) { return rowC(g, k); }
template <>
__device__ __forceinline__ float* rowCr<float>(const DevGrid& g, int k) { return g.rowCf + (size_t)k * g.rowC_stride; }

// Per-cell values of a row-major sweep over the grid stored column-major through a
// shared-memory tile.  The CTA (256 threads) takes rows i0..i0+7, one warp per row as the
// per-row kernels do, and walks the union of those rows' spans (rlo..rhi clipped to
// [jmin, jmax]; rows past ilast have none) in chunks of 32 columns.  cell(i, j, v) fills
// the K values of cell (i, j) and returns whether the cell is stored; the stored values
// of a chunk go out column by column, the 8 rows of a column as one contiguous run, in
// place of one 32-byte sector per cell.  dst[k][j * g.LT + i] receives value k.
constexpr int kTileRows = 8;
template <int K, class T, class Cell>
__device__ __forceinline__ void colmajor_tile(const DevGrid& g, int i0, int ilast, int jmin, int jmax, Cell cell,
                                              T* const (&dst)[K]) {
    __shared__ T s_v[K][kTileRows][33];
    __shared__ unsigned s_m[kTileRows];
    __shared__ int s_lo[kTileRows], s_hi[kTileRows];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = i0 + w;
    int lo = 1 << 30, hi = -1;
    if (i <= ilast) {
        lo = max(g.rlo[i], jmin);
        hi = min(g.rhi[i], jmax);
    }
    if (lane == 0) {
        s_lo[w] = lo;
        s_hi[w] = hi;
    }
    __syncthreads();
    int ulo = 1 << 30, uhi = -1;
#pragma unroll
    for (int r = 0; r < kTileRows; r++) {
        ulo = min(ulo, s_lo[r]);
        uhi = max(uhi, s_hi[r]);
    }
    const int sc = threadIdx.x / kTileRows, sr = threadIdx.x % kTileRows;  // store: column, row
    for (int jc = ulo; jc <= uhi; jc += 32) {
        const int j = jc + lane;
        T v[K];
        bool wr = false;
        if (j >= lo && j <= hi) wr = cell(i, j, v);
        const unsigned m = __ballot_sync(0xffffffffu, wr);
        if (wr) {
#pragma unroll
            for (int k = 0; k < K; k++) s_v[k][w][lane] = v[k];
        }
        if (lane == 0) s_m[w] = m;
        __syncthreads();
        if ((s_m[sr] >> sc) & 1u) {
            const size_t q = (size_t)(jc + sc) * g.LT + i0 + sr;
#pragma unroll
            for (int k = 0; k < K; k++) dst[k][q] = s_v[k][sr][sc];
        }
        __syncthreads();
    }
}

// Wall/open flags of a row segment [first, last] (locate_segment_v, constant.cuh:135-154).
__device__ __forceinline__ void seg_flags_v(const DevGrid& g, const DevParams& p, int row, int first, int last,
                                            int& br1, int& br2) {
    const int P = g.P;
    br1 = (first > 2) ||
          (first == 2 && (g.h[row * P + first - 1] + g.h[(row - 1) * P + first - 1]) * 0.5 == p.NANGDAY);
    br2 = (last < g.M) || (last == g.M && (g.h[row * P + last] + g.h[(row - 1) * P + last]) * 0.5 == p.NANGDAY);
}

// Minimum / maximum in the arithmetic type of a kernel instantiation.
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double rmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float rmin(float a, float b) { return fminf(a, b); }

// Erosion/deposition source terms of the suspended-sediment rows, in the arithmetic type R
// (double: the FP64 form; float: the mixed form's sediment transport).
template <class R>
__device__ __forceinline__ R source_chs(const DevParams& p, R wsm, R Zf, R fs, R fw, R vth, R h_moi) {
    // source_chs (Sediment_Transport.cu:12-49)
    R toee = R(p.Toe);
    const R todd = R(p.Tod);
    R S = 0;
    const R tob = R(p.ro) * fw * (vth * vth);
    if (h_moi > R(p.ghtoe)) toee = R(p.Toe) * (1 + R(p.hstoe) * ((h_moi - R(p.ghtoe))));
    if (tob > toee) S = R(p.Mbochat) / R(p.ros) * (tob - toee) / toee;
    else if (tob < todd) {
        const R Pd = 1 - (tob / todd);
        // Pd^2.5 as Pd^2 sqrt(Pd) (0 < Pd <= 1): the same value to a few ulp, without pow's
        // general path
        const R beta = 1 + (Zf / (R(1.25) + R(4.75) * (Pd * Pd * sqrt(Pd))));
        const R Cb = beta * fs;
        S = -wsm * Cb * Pd;
    }
    return S;
}

template <class R>
__device__ __forceinline__ R source_nchs(const DevParams& p, R wsm, R Zf, R Uf, R h_moi, R fs) {
    // source_nchs (Sediment_Transport.cu:52-60)
    const R gamac = R(0.434) + R(5.975) * Zf + R(2.888) * Zf * Zf;
    const R ufr = R(p.ufr);
    const R Tx = rmax(R(0), (Uf * Uf - ufr * ufr) / (ufr * ufr));
    const R Cac = R(0.015) * R(p.dm) * (Tx * sqrt(Tx)) * R(p.dxr_m03) / (R(0.05) * h_moi);  // Tx^1.5, Tx >= 0
    return wsm * (Cac - gamac * fs);
}

// Wall/open flags of a column segment (locate_segment_u, constant.cuh:156-178).
__device__ __forceinline__ void seg_flags_u(const DevGrid& g, const DevParams& p, int col, int first, int last,
                                            int& br1, int& br2) {
    const int P = g.P;
    br1 = (first > 2) || (first == 2 && (g.h[1 * P + col] + g.h[1 * P + col - 1]) * 0.5 == p.NANGDAY);
    br2 = (last < g.N) || (last == g.N && (g.h[g.N * P + col] + g.h[g.N * P + col - 1]) * 0.5 == p.NANGDAY);
}

// Segment of row `row` holding column `col`, -1 if none.
__device__ __forceinline__ int find_seg_v(const DevGrid& g, int row, int col, int& first, int& last) {
    const int n = g.moci[row];
    for (int k = 0; k < n; k++) {
        const int a = g.daui[row * HYD_SEGL + k], b = g.cuoii[row * HYD_SEGL + k];
        if (a <= col && col <= b) {
            first = a;
            last = b;
            return k;
        }
    }
    return -1;
}

// Segment of column `col` holding row `row`, -1 if none.
__device__ __forceinline__ int find_seg_u(const DevGrid& g, int row, int col, int& first, int& last) {
    const int n = g.mocj[col];
    for (int k = 0; k < n; k++) {
        const int a = g.dauj[col * HYD_SEGL + k], b = g.cuoij[col * HYD_SEGL + k];
        if (a <= row && row <= b) {
            first = a;
            last = b;
            return k;
        }
    }
    return -1;
}

// Host launch wrappers (defined in the .cu files, called by hydist_api.cu).
struct StepLaunch;
void launch_init_kernels(const DevGrid& g, const DevParams& p, const int* keep_mask, cudaStream_t s);
// Launch shapes of the sweeps for one grid (k_sweep.cu).
struct SweepPlan {
    size_t smem_lines, smem_fs_lines;  // dynamic shared memory of the hydrodynamic / sediment sweeps
    int RB, RBf;                       // rows of a long line held in shared memory
    int RG, RGf;                       // rows of a CTA's global scratch region
    int long_grid;                     // CTAs of the sweeps
    int need_global;                   // some line may exceed shared memory
    int wide;                          // warps sweep every line their slice holds (throughput sizing)
    size_t scratch_doubles;            // global scratch to allocate
};
// max_rows > 0: at most that many rows of a long line in shared memory (0: as many as fit)
cudaError_t sweep_plan(int N, int M, SweepPlan* sp, int max_rows);
// Throughput sizing for reaches that share the device with others: as many sweep CTAs as
// give every line of the longer direction its own warp in one pass (each CTA sweeps one
// line per warp), instead of one CTA per SM, and every line a warp's slice holds swept
// by its warp.
void sweep_plan_throughput(int N, int M, SweepPlan* sp);
cudaError_t grid_setup(int N, int M);
void launch_sweep_uz(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int startidx, int endidx,
                     int solver, double* scratch, cudaStream_t s);
void launch_sweep_vz(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int startidx, int endidx,
                     int solver, double* scratch, cudaStream_t s);
// bytes: also write the column reset bytes (the smoothing of u just before the column resets)
// fs_bnd: also apply the concentration part of the second half-step's boundary (span
// passes only)
// budget: also add the half-step's open-edge volumes to the budget (the first smoothing
// after each sweep: isU = 1 after the UZ sweep, isU = 0 after the VZ sweep)
void launch_budget_half(const DevGrid& g, const DevParams& p, int isU, cudaStream_t s);
void launch_smooth(const DevGrid& g, const DevParams& p, int isU, double* out, int full, int bytes, int fs_bnd,
                   int budget, cudaStream_t s);
void launch_widen_spans(const DevGrid& g, cudaStream_t s);
void launch_explicit_v(const DevGrid& g, const DevParams& p, int threads, cudaStream_t s);
void launch_explicit_u(const DevGrid& g, const DevParams& p, int threads, cudaStream_t s);
void launch_coef_eu(const DevGrid& g, const DevParams& p, cudaStream_t s);
// threads: a multiple of 32
void launch_reset_rows(const DevGrid& g, const DevParams& p, int force, int threads, cudaStream_t s);
void launch_reset_cols(const DevGrid& g, const DevParams& p, int force, int threads, cudaStream_t s);
void launch_spans(const DevGrid& g, cudaStream_t s);
// n <= kPutDoubles values from host memory to dst through the launch parameters (returns
// 0, launching nothing, when n is out of range)
constexpr int kPutDoubles = 480;
int launch_put_doubles(double* dst, const double* src, int n, cudaStream_t s);
// rows x cols doubles of a pitched array into a packed one
void launch_pack_rows(const double* src, int pitch, double* dst, int rows, int cols, cudaStream_t s);
void clear_rescan_lists(const DevGrid& g, cudaStream_t s);
// 1 if a and b differ outside the extended spans on [i0, i1] x [j0, j1], 0 if not, -1 on error
int outside_differs(const DevGrid& g, const double* a, const double* b, int i0, int i1, int j0, int j1, int* dflag,
                    cudaStream_t s);
void launch_mark_all_cols(const DevGrid& g, cudaStream_t s);
void launch_post(const DevGrid& g, const DevParams& p, int full, cudaStream_t s);
void launch_scan_cols(const DevGrid& g, const DevParams& p, cudaStream_t s);
void launch_scan_rows(const DevGrid& g, const DevParams& p, cudaStream_t s);
// fsi: the second half-step's, which also leaves the FSi cell terms
void launch_vth_hesok(const DevGrid& g, const DevParams& p, int full, int fsi, cudaStream_t s);
void launch_post_fused(const DevGrid& g, const DevParams& p, int rows, int vth, cudaStream_t s);
// The first launch of half-step `half`: its line coefficients (UZ column-major / VZ
// row-major) and its boundary values (`writes`: 1 velocities/levels, 2 inflow
// concentrations, 3 both; ignored in channel mode).  Half-step 1 also advances the clock.
void launch_coef_bnd(const DevGrid& g, const DevParams& p, int half, int writes, cudaStream_t s);
void launch_coef_fsj(const DevGrid& g, const DevParams& p, int half, cudaStream_t s);
void launch_fs_sweep_j(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int half, int solver,
                       double* scratch, cudaStream_t s);
void launch_fs_sweep_i(const DevGrid& g, const DevParams& p, const SweepPlan& sp, int half, int solver,
                       double* scratch, cudaStream_t s);
void launch_update_fs(const DevGrid& g, int full, cudaStream_t s);
void launch_bed(const DevGrid& g, const DevParams& p, int startidx, int endidx, cudaStream_t s);
// feedback: h0 = h (the bed the applied changes start from), dH and its compensation zeroed
void launch_bed_reset(const DevGrid& g, cudaStream_t s);
// hyd_add_levels: increments added to z, u, v on the wet cells of rows i0.. x columns j0..,
// the depths and face depths re-derived around them
void launch_add_levels(const DevGrid& g, const DevParams& p, const float* du, const float* dv, const float* dz,
                       int i0, int j0, int rows, int cols, long long ld, cudaStream_t s);
// hyd_steady_residual: per-CTA sums over the wet cells (4 per CTA), then the totals in
// out[0..3] added in CTA order; snapshot: u0, v0, z0 = u, v, z afterwards
void launch_steady_residual(const DevGrid& g, double* u0, double* v0, double* z0, int snapshot, double* part,
                            int nblocks, double* out, cudaStream_t s);
long long hyd_kernel_launches_add(long long n);

// Batched launches (k_grid.cu, k_sweep.cu): one launch for every member of a batch, each
// CTA working for one member; `ctas` = the members' CTAs together.
void launch_coef_bnd_batch(const BatchRef& br, int ctas, int half, int writes, int mixed, cudaStream_t s);
void launch_smooth_batch(const BatchRef& br, int ctas, int isU, double* const* outs, int bytes, int fs_bnd, int budget,
                         cudaStream_t s);
void launch_explicit_v_batch(const BatchRef& br, int ctas, int threads, size_t smem, int mixed, cudaStream_t s);
void launch_coef_eu_batch(const BatchRef& br, int ctas, int mixed, cudaStream_t s);
void launch_explicit_u_batch(const BatchRef& br, int ctas, int threads, size_t smem, int mixed, cudaStream_t s);
void launch_reset_batch(const BatchRef& br, int ctas, int rows, int threads, size_t smem, cudaStream_t s);
void launch_post_fused_batch(const BatchRef& br, int ctas, int rows, int vth, int mixed, size_t smem, cudaStream_t s);
void launch_update_fs_batch(const BatchRef& br, int ctas, cudaStream_t s);
void launch_coef_fsj_batch(const BatchRef& br, int ctas, int half, int mixed, cudaStream_t s);
void launch_sweep_batch(int dir, const BatchLines& bl, const SweepPlan& sp, int solver, int mixed, double* scratch,
                        int grid, cudaStream_t s);
void launch_fs_sweep_batch(int dir, const BatchLines& bl, const SweepPlan& sp, int half, int solver, int mixed,
                           double* scratch, int grid, cudaStream_t s);
cudaError_t batch_grid_setup(size_t smem_ev, size_t smem_eu, size_t smem_rr, size_t smem_rc, size_t smem_pf);
cudaError_t batch_sweep_setup();
void line_smem(int N, int M, size_t* ev, size_t* eu, size_t* rr, size_t* rc, size_t* pf);
