// hydist_api.cu — the C ABI of include/hydist_b200.h.
//
// Replaces the reference's Python host (rep.py gpu_init, Pointers.py struct packing,
// Engine.hydraulic_Calculation's time loop): one handle owns a device arena, a stream
// and the launch sequence of a full ADI step.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <utility>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydist_b200.h"
#include "hydist_dev.cuh"

namespace {

thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess) return fail(HYD_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr double kPiRef = 3.14159265359;

}  // namespace

long long hyd_kernel_launches_add(long long n) { return g_launches.fetch_add(n) + n; }

struct FieldDesc {
    const char* name;
    int kind;     // 0 grid double, 1 grid int, 2 row table int (N+2)*20, 3 col table int (M+2)*20,
                  // 4 int N+2, 5 int M+2, 6 double M+2, 7 double N+2, 8 hi, 9 hmax[4]
    size_t off;   // offset of the pointer member in DevGrid
};

#define FD(n, k) {#n, k, offsetof(DevGrid, n)}
static const FieldDesc kFieldTable[] = {
    FD(h, 0),     FD(hsnham, 0), FD(Fw, 0),    FD(Tsxw, 0),    FD(Tsyw, 0),  FD(u, 0),
    FD(v, 0),     FD(z, 0),      FD(t_u, 0),   FD(t_v, 0),     FD(t_z, 0),   FD(Htdu, 0),
    FD(Htdv, 0),  FD(H_moi, 0),  FD(htaiz, 0), FD(htaiz_bd, 0), FD(Kx1, 0),  FD(Ky1, 0),
    FD(FS, 0),    FD(tFS, 0),    FD(VTH, 0),   FD(Kx, 0),      FD(Ky, 0),    FD(Qbx, 0),
    FD(Qby, 0),   FD(dH, 0),     FD(khouot, 1), FD(daui, 2),   FD(cuoii, 2), FD(moci, 4),
    FD(dauj, 3),  FD(cuoij, 3),  FD(mocj, 5),  FD(ubt, 6),     FD(ubp, 6),   FD(vbt, 7),
    FD(vbd, 7),   FD(hi, 8),     FD(hmax, 9),
};
#undef FD

struct HydSim {
    HydCaseParams P;
    int N, M, pitch;
    int device;
    cudaStream_t stream;
    DevGrid g;
    DevParams dp;
    double* scratch_u;  // smoothing ping-pong partners
    double* scratch_v;
    double* sweep_scratch;  // rows/cells of lines too long for shared memory
    double* fs_scratch;     // the same for the sediment sweeps (which may run beside the others)
    SweepPlan plan;         // launch shapes of the sweeps
    int plan_grid;          // the sweeps' CTAs as planned at creation (the most allowed)
    void* arena;
    size_t arena_bytes;
    std::vector<void*> extra;
    double t;
    int have_boundary;
    int bnd_nseg[4];  // segments per edge of the boundary tables
    // the eight tables in one device block (bc 0-3, cc 0-3), a pinned staging copy for
    // hyd_update_boundary and the event of its last upload
    double* bnd_block;
    double* bnd_stage;
    size_t bnd_doubles;
    cudaEvent_t ev_bnd;
    int initialized;
    int solver;
    int start_idx, end_idx;
    unsigned* h_status;
    double* run_part;  // hyd_run's non-finite check: partial sums, allocated at its first use
    // phase timing (instrumentation): bit k set = phase k bracketed by events
    unsigned timing;
    struct Mark {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> event_pool;
    double phase_ms[32];
    long long phase_n[32];
    // CUDA graphs of one full step, one per variant (bit 0: sediment in half-step 1,
    // bit 1: sediment in half-step 2, bit 2: Exner update)
    int use_graphs;
    int force_rescan;  // the next step rescans every line (mask or segment tables were set)
    // elementwise kernels still owed one whole-grid pass before they may run on the
    // extended spans: bit 0 hydrodynamics (smoothing, state update), bit 1 sediment
    int full_pending;
    // CTA widths of the row and column line kernels, from the longest span of each
    // direction (about two cells per thread)
    int thr_r, thr_c;
    // second stream for work that runs beside the main chain (forked and joined by events)
    cudaStream_t side;
    cudaEvent_t ev_fork, ev_join;
    // third stream: a half-step's water budget beside the launches that follow its sweep
    cudaStream_t side2;
    cudaEvent_t ev_bfork, ev_bjoin;
    // asynchronous field reads: two device snapshots, copied out on their own stream
    cudaStream_t copy_stream;
    cudaEvent_t ev_snap, ev_copied[2];
    void* snap[2];
    int snap_i;
    // whole-grid events (set-up, field writes, whole-grid steps): after one, any cell of a
    // field may have changed; between them only the cells of the extended spans can
    unsigned long long epoch;
    // rows [box_r0, box_r1] x columns [box_c0, box_c1]: every cell with a non-empty
    // extended span, as of whole-grid event count box_epoch
    unsigned long long box_epoch;
    int box_r0, box_r1, box_c0, box_c1;
    // host mirror of one grid field (hyd_mirror_*): two pinned copies handed out in turn,
    // each up to date as of whole-grid event count mir_epoch[k]; device staging of a copy
    const FieldDesc* mir_f;
    double* mir[2];
    void* mir_snap[2];
    unsigned long long mir_epoch[2];
    cudaEvent_t ev_mir[2];
    int mir_i, mir_open;
    cudaGraphExec_t graph[8];
    long long graph_kernels[8];
    // timing with graphs: one graph per variant with the phase events captured in it
    cudaGraphExec_t tgraph[8];
    std::vector<Mark> tmarks[8];
    std::vector<Mark>* mark_sink;  // where PhaseScope files its events (null: marks)
    // hyd_checkpoint: a device copy of the arena and the column-major mask bytes, with the
    // host-side step state at the time (allocated at the first save)
    void* ck_arena;
    int ck_valid;
    double ck_t;
    int ck_start, ck_end, ck_full, ck_force;
    // hyd_steady_residual: snapshot of u, v, z (three pitched grid fields), per-CTA sums and
    // the totals (allocated at the first call)
    double* res_buf;
    int res_valid;
};

static const char* kPhaseNames[] = {"boundary", "sweep_uz", "sweep_vz", "smooth", "explicit_v", "explicit_u",
                                    "reset_rows", "reset_cols", "post", "scan", "vth_hesok", "fs_sweep_j",
                                    "fs_sweep_i", "update_fs", "bed", "coef_uz", "coef_fsj", "coef_eu"};
enum Phase { PH_BOUNDARY, PH_SWEEP_UZ, PH_SWEEP_VZ, PH_SMOOTH, PH_EXPL_V, PH_EXPL_U, PH_RESET_ROWS,
             PH_RESET_COLS, PH_POST, PH_SCAN, PH_VTH, PH_FS_J, PH_FS_I, PH_UPDATE_FS, PH_BED, PH_COEF_UZ,
             PH_COEF_FSJ, PH_COEF_EU, PH_COUNT };
static_assert(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]) == PH_COUNT, "one name per phase");

namespace {
void drop_graphs(HydSim* s) {
    for (int k = 0; k < 8; k++) {
        if (s->graph[k]) cudaGraphExecDestroy(s->graph[k]);
        s->graph[k] = nullptr;
        if (s->tgraph[k]) cudaGraphExecDestroy(s->tgraph[k]);
        s->tgraph[k] = nullptr;
        for (auto& m : s->tmarks[k]) {
            cudaEventDestroy(m.a);
            cudaEventDestroy(m.b);
        }
        s->tmarks[k].clear();
    }
}

// Widths of the row / column line kernels from the spans (read back once per mask).
static int refresh_widths(HydSim* s) {
    std::vector<int> lo((size_t)(s->N > s->M ? s->N : s->M) + 3), hi(lo.size());
    auto longest = [&](const int* dlo, const int* dhi, int n) -> int {
        if (cudaMemcpyAsync(lo.data(), dlo, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaMemcpyAsync(hi.data(), dhi, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            return -1;
        int best = 0;
        for (int i = 0; i < n; i++)
            if (hi[i] >= lo[i] && hi[i] - lo[i] + 1 > best) best = hi[i] - lo[i] + 1;
        return best;
    };
    auto pick = [](int len) {
        int t = ((len + 1) / 2 + 31) / 32 * 32;
        return t < 64 ? 64 : (t > 512 ? 512 : t);
    };
    const int lr = longest(s->g.rlo, s->g.rhi, s->N + 3), lc = longest(s->g.clo, s->g.chi, s->M + 3);
    const int le = longest(s->g.elo, s->g.ehi, s->N + 3);
    if (lr < 0 || lc < 0 || le < 0) return fail(HYD_ECUDA, "reading the spans back failed");
    const int tr = pick(lr), tc = pick(lc);
    int wpr = (le + 31) / 32;
    wpr = wpr < 1 ? 1 : (wpr > 8 ? 8 : wpr);
    // a segment's cells are not land, so a staged line [first - 2, last + 1] spans at most
    // the longest run of such cells plus 3
    const int svc = std::min(lr + 3, s->M + 3), suc = std::min(lc + 3, s->N + 3);
    if (tr != s->thr_r || tc != s->thr_c || wpr != s->g.wpr || svc != s->g.sv_cap || suc != s->g.su_cap)
        drop_graphs(s);
    s->thr_r = tr;
    s->thr_c = tc;
    s->g.wpr = wpr;
    s->g.sv_cap = svc;
    s->g.su_cap = suc;
    return HYD_OK;
}


int set_clock(HydSim* s, double t) {
    const double c[3] = {t, t, t};
    cudaError_t e = cudaMemcpyAsync(s->g.clock, c, sizeof c, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? HYD_OK : fail(HYD_ECUDA, std::string("clock: ") + cudaGetErrorString(e));
}

cudaEvent_t pool_event(HydSim* s) {
    if (!s->event_pool.empty()) {
        cudaEvent_t e = s->event_pool.back();
        s->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
struct PhaseScope {
    HydSim* s;
    int ph;
    cudaStream_t st;  // the stream the phase's launches go to
    cudaEvent_t a = nullptr;
    // inside a capture an event record is an ordering edge unless marked external
    void record(cudaEvent_t e) {
        if (s->mark_sink) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
        else cudaEventRecord(e, st);
    }
    PhaseScope(HydSim* s_, int ph_, cudaStream_t st_) : s(s_), ph(ph_), st(st_) {
        if ((s->timing >> ph) & 1u) {
            a = pool_event(s);
            record(a);
        }
    }
    ~PhaseScope() {
        if (a) {
            cudaEvent_t b = pool_event(s);
            record(b);
            (s->mark_sink ? *s->mark_sink : s->marks).push_back({ph, a, b});
        }
    }
};
}  // namespace
#define PHASE(ph) PhaseScope phase_scope_##__LINE__(s, ph, s->stream)
#define PHASE_ON(ph, stream) PhaseScope phase_scope_##__LINE__(s, ph, stream)

namespace {

size_t field_count(const HydSim* s, int kind) {
    const size_t N = s->N, M = s->M;
    switch (kind) {
        case 0:
        case 1: return (N + 3) * (M + 3);
        case 2: return (N + 2) * HYD_SEGL;
        case 3: return (M + 2) * HYD_SEGL;
        case 4: return N + 2;
        case 5: return M + 2;
        case 6: return M + 2;
        case 7: return N + 2;
        case 9: return 4;
        default: return 2 * (N + 3) + 2 * (M + 3);
    }
}

const FieldDesc* find_field(const char* name) {
    if (!strcmp(name, "VISCOIDX") || !strcmp(name, "VISCOINDX")) {
        static const FieldDesc visc = {"VISCOIDX", 0, offsetof(DevGrid, VISC)};
        return &visc;
    }
    for (const FieldDesc& f : kFieldTable)
        if (!strcmp(f.name, name)) return &f;
    return nullptr;
}

void* member(HydSim* s, const FieldDesc* f) { return *(void**)((char*)&s->g + f->off); }

DevParams make_dev_params(const HydCaseParams& P) {
    DevParams d;
    d.dX = P.dX;
    d.dY = P.dY;
    d.dT = P.dT;
    d.dXbp = P.dXbp;
    d.dX2 = P.dX2;
    d.dYbp = P.dYbp;
    d.dY2 = P.dY2;
    d.dTchia2dX = P.dTchia2dX;
    d.dTchia2dY = P.dTchia2dY;
    d.HaiChiadT = P.HaiChiadT;
    d.NANGDAY = P.NANGDAY;
    d.H_TINH = P.H_TINH;
    d.heso = P.heso;
    d.mu_mn = P.mu_mn;
    d.NDnen = P.NDnen;
    d.Tod = P.Tod;
    d.Toe = P.Toe;
    d.hstoe = P.hstoe;
    d.ghtoe = P.ghtoe;
    d.Mbochat = P.Mbochat;
    d.ro = P.ro;
    d.ros = P.ros;
    d.dm = P.dm;
    d.Dorong = P.Dorong;
    d.Sx = P.Sx;
    d.CORIOLIS_FORCE = P.CORIOLIS_FORCE;
    d.g = P.g;
    d.Ks = P.Ks;
    // device helpers of constant.cuh:126-133
    d.windx = 0.0013 * (0.00075 + 0.000067 * std::fabs(P.Wind)) * std::fabs(P.Wind) * P.Wind *
              std::cos(P.huonggio * (kPiRef / 180));
    d.windy = 0.0013 * (0.00075 + 0.000067 * std::fabs(P.Wind)) * std::fabs(P.Wind) * P.Wind *
              std::sin(P.huonggio * (kPiRef / 180));
    d.ufr = 0.25 * std::pow((P.Sx - 1) * P.g, 8.0 / 15.0) * std::pow(P.dm, 9.0 / 15.0) * std::pow(P.muy, -1.0 / 15.0);
    d.dxr = P.dm * std::pow(P.g * (P.Sx - 1) / P.muy * P.muy, (1.0 / 3.0));
    d.dxr_m03 = std::pow(d.dxr, -0.3);
    d.wss = 10 * P.muy / P.dm * (std::sqrt(1 + 0.01 * (P.Sx - 1) * 9.81 * std::pow(P.dm, 3) / std::pow(P.muy, 2)) - 1);
    d.sediment_start = P.sediment_start;
    d.bed_change_start = P.bed_change_start;
    d.ketdinh = P.ketdinh;
    d.kenhhepd = P.kenhhepd;
    d.kenhhepng = P.kenhhepng;
    d.channel = (P.kenhhepd || P.kenhhepng) ? 1 : 0;
    d.bed_feedback = P.bed_feedback ? 1 : 0;
    d.bed_fixed = P.bed_fixed > 0 ? P.bed_fixed : 0;
    d.bed_min_depth = P.bed_min_depth > 0 ? P.bed_min_depth : 0.0;
    d.morfac = P.morfac;
    d.bed_period = P.bed_period > 0 ? P.bed_period : P.bed_change_start;
    d.mixed = P.precision_mode == HYD_PRECISION_MIXED ? 1 : 0;
    return d;
}

int check_device_status(HydSim* s) {
    unsigned st = 0;
    CUDA_TRY(cudaMemcpyAsync(&st, s->g.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (st & HYD_ST_SEG_OVERFLOW)
        return fail(HYD_EDEVICE, "a grid line has more than 20 wet segments (segment_limit)");
    if (st & HYD_ST_STAGE_RANGE)
        return fail(HYD_EDEVICE, "a line's wet span exceeded the explicit kernels' staging bound");
    return HYD_OK;
}

// mass balance: per-block partial sums, then one block adds them in a fixed order
__global__ void k_mass_partial(DevGrid g, double* part) {
    __shared__ double sh[5][256];
    const int tid = threadIdx.x;
    double a = 0, b = 0, c = 0, wet = 0, bad = 0;
    const long long ncell = (long long)(g.N + 3) * (g.M + 3);
    for (long long q = (long long)blockIdx.x * blockDim.x + tid; q < ncell; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / (g.M + 3)), j = (int)(q % (g.M + 3));
        const int gp = i * g.P + j;
        if (i <= g.N && j <= g.M) {
            if (!isfinite(g.z[gp]) || !isfinite(g.u[gp]) || !isfinite(g.v[gp]) || !isfinite(g.FS[gp])) bad += 1;
        }
        if (i < 2 || j < 2 || i > g.N || j > g.M) continue;
        if (g.khouot[gp] == 0) {
            a += g.H_moi[gp];
            b += g.FS[gp] * g.H_moi[gp];
            wet += 1;
        }
        if (isfinite(g.dH[gp])) c += g.dH[gp];
    }
    sh[0][tid] = a;
    sh[1][tid] = b;
    sh[2][tid] = c;
    sh[3][tid] = wet;
    sh[4][tid] = bad;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (tid < w)
            for (int k = 0; k < 5; k++) sh[k][tid] += sh[k][tid + w];
        __syncthreads();
    }
    if (tid == 0)
        for (int k = 0; k < 5; k++) part[blockIdx.x * 5 + k] = sh[k][0];
}

__global__ void k_mass_final(const double* part, int nblocks, double* out) {
    if (threadIdx.x != 0) return;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < nblocks; b++)
        for (int k = 0; k < 5; k++) acc[k] += part[b * 5 + k];
    for (int k = 0; k < 5; k++) out[k] = acc[k];
}

// Scratch of hyd_mass_balance_noalloc: up to HYD_MASS_NOALLOC_MAX_BLOCKS blocks of five
// partial sums, then the five totals.  Looked up once per device.
static __device__ __align__(256) double g_mass_scratch[HYD_MASS_NOALLOC_MAX_BLOCKS * 5 + 5];
constexpr int kMaxDevices = 64;
double* g_mass_scratch_ptr[kMaxDevices];
std::mutex g_mass_scratch_mu;

// The device address of g_mass_scratch on `device` (current), looked up once per device.
// The lookup loads this file's module on that device (with lazy module loading it is not
// loaded before), which places the array in device memory: hyd_create does it, so that a
// later hyd_mass_balance_noalloc call finds the module loaded and allocates nothing.
cudaError_t mass_scratch_address(int device, double** out) {
    std::lock_guard<std::mutex> lock(g_mass_scratch_mu);
    if (!g_mass_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_mass_scratch);
        if (e != cudaSuccess) return e;
        g_mass_scratch_ptr[device] = (double*)p;
    }
    *out = g_mass_scratch_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" {

const char* hyd_last_error(void) { return g_last_error.c_str(); }

const char* hyd_version(void) {
    return "hydist_b200 1.1 (sm_100a, FP64 ADI and FP32-bulk mixed form, partitioned line solver)";
}

void hyd_params_derive(HydCaseParams* p) {
    p->dXbp = p->dX * p->dX;
    p->dX2 = 2 * p->dX;
    p->dYbp = p->dY * p->dY;
    p->dY2 = 2 * p->dY;
    p->dTchia2dX = p->dT / (2 * p->dX);
    p->dTchia2dY = p->dT / (2 * p->dY);
    p->QuyDoiTime = 1.0 / 3600;
    p->QuyDoiPi = 1.0 / kPiRef;
    p->HaiChiadT = 2.0 / p->dT;
}

void hyd_params_default(HydCaseParams* p) {
    memset(p, 0, sizeof(*p));
    p->dX = 10.0;
    p->dY = 10.0;
    p->dT = 2.0;
    p->NANGDAY = 0.0;
    p->H_TINH = 0.02;
    p->Wind = 0.0;
    p->huonggio = 0.0;
    p->Zbandau = 0.0;
    p->heso = 0.94;
    p->mu_mn = 0.2;
    p->NDnen = 0.0;
    p->NDbphai = p->NDbtrai = p->NDbtren = p->NDbduoi = 0.5;
    p->Tod = 0.06;
    p->Toe = 0.15;
    p->hstoe = 0;
    p->ghtoe = 3;
    p->Mbochat = 0.00001;
    p->ro = 1000;
    p->ros = 2000;
    p->dm = 0.00001;
    p->d90 = 0.002;
    p->muy = 1.01e-06;
    p->Dorong = 0.5;
    p->Sx = 2;
    p->sohn = 8;
    p->soha = 3;
    p->sohn1 = 3;
    p->CORIOLIS_FORCE = 0.0;
    p->g = 9.81;
    p->Ks = 2.5 * 0.00001;
    p->sediment_start = 36000;
    p->bed_change_start = 72000;
    p->ketdinh = 1;
    p->precision_mode = HYD_PRECISION_FP64;
    p->morfac = 1.0;
    p->bed_period = 0.0;
    p->bed_feedback = 0;
    hyd_params_derive(p);
}

// Free what a handle holds (any of it may be missing on a failed create) and the handle.
static void release(HydSim* s) {
    cudaFree(s->run_part);
    cudaFree(s->ck_arena);
    cudaFree(s->res_buf);
    cudaFree(s->sweep_scratch);
    cudaFree(s->fs_scratch);
    cudaFree(s->g.colT);
    cudaFree(s->g.rowC);
    cudaFree(s->g.colTf);
    cudaFree(s->g.rowCf);
    cudaFree(s->arena);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    if (s->ev_bfork) cudaEventDestroy(s->ev_bfork);
    if (s->ev_bjoin) cudaEventDestroy(s->ev_bjoin);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    cudaFree(s->snap[0]);
    cudaFree(s->snap[1]);
    for (int k = 0; k < 2; k++) {
        if (s->mir[k]) cudaFreeHost(s->mir[k]);
        cudaFree(s->mir_snap[k]);
        if (s->ev_mir[k]) cudaEventDestroy(s->ev_mir[k]);
        s->mir[k] = nullptr;
        s->mir_snap[k] = nullptr;
        s->ev_mir[k] = nullptr;
    }
    s->mir_open = 0;
    if (s->ev_snap) cudaEventDestroy(s->ev_snap);
    if (s->ev_copied[0]) cudaEventDestroy(s->ev_copied[0]);
    if (s->ev_copied[1]) cudaEventDestroy(s->ev_copied[1]);
    if (s->ev_bnd) cudaEventDestroy(s->ev_bnd);
    cudaFree(s->bnd_block);
    if (s->bnd_stage) cudaFreeHost(s->bnd_stage);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->side2) cudaStreamDestroy(s->side2);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int hyd_create(const HydCaseParams* p, int N, int M, int device, hyd_handle* out) {
    if (!p || !out) return fail(HYD_EINVAL, "null argument");
    if (N < 6 || M < 6) return fail(HYD_EINVAL, "grid too small (N, M >= 6)");
    // a line of the grid is staged in shared memory by several kernels (8 B per cell)
    if (N > HYD_MAX_LINE || M > HYD_MAX_LINE) return fail(HYD_EINVAL, "grid too large (N, M <= 25000)");
    if (p->dT <= 0 || p->dX <= 0 || p->dY <= 0) return fail(HYD_EINVAL, "dX, dY, dT must be positive");
    if (p->precision_mode != HYD_PRECISION_FP64 && p->precision_mode != HYD_PRECISION_MIXED)
        return fail(HYD_EINVAL, "precision_mode must be HYD_PRECISION_FP64 or HYD_PRECISION_MIXED");
    if (p->bed_feedback && !(p->morfac > 0)) return fail(HYD_EINVAL, "bed_feedback needs morfac > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(HYD_ECUDA, "no CUDA device: this library has no CPU path");
    if (device < 0 || device >= ndev) return fail(HYD_EINVAL, "bad device index");
    CUDA_TRY(cudaSetDevice(device));
    HydSim* s = new HydSim();
    s->thr_r = s->thr_c = 128;
    s->P = *p;
    s->N = N;
    s->M = M;
    s->pitch = ((M + 3) + 31) / 32 * 32;
    s->device = device;
    s->t = 0;
    s->have_boundary = 0;
    s->initialized = 0;
    const char* sv = getenv("HYD_SOLVER");
    s->solver = (sv && !strcmp(sv, "thomas")) ? 1 : 0;
    s->start_idx = 2;
    s->end_idx = N;
    s->timing = 0;
    {
        const char* gv = getenv("HYD_GRAPHS");
        s->use_graphs = !(gv && !strcmp(gv, "0"));
    }
    for (int k = 0; k < 8; k++) {
        s->graph[k] = nullptr;
        s->graph_kernels[k] = 0;
    }
    for (int k = 0; k < 32; k++) {
        s->phase_ms[k] = 0;
        s->phase_n[k] = 0;
    }
    // the side stream's work (the first half-step's sediment) has the slack: it runs at a
    // lower priority than the main chain it runs beside
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    cudaError_t e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, prio_lo);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->side2, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_bfork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_bjoin, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_snap, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_copied[0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_copied[1], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_bnd, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        release(s);
        return fail(HYD_ECUDA, std::string("streams: ") + cudaGetErrorString(e));
    }
    // arena: grid fields (double and int), smoothing partners, tables, boundary arrays
    const size_t nrow = (size_t)N + 3;
    const size_t gbytes = nrow * s->pitch * sizeof(double);
    const size_t ngrid = 29;  // double grid fields in kFieldTable + VISC, h0, dHc, dHinc
    const size_t nseg_rows = ((size_t)N + 3) * HYD_SEGL, nseg_cols = ((size_t)M + 3) * HYD_SEGL;
    auto a256 = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t total = a256(gbytes) * (ngrid + 1 + 2) + a256(nrow * s->pitch * sizeof(int));
    total += 2 * a256(nseg_rows * 4) + a256((N + 3) * 4) + 2 * a256(nseg_cols * 4) + a256((M + 3) * 4);
    total += 2 * a256((M + 3) * 8) + 2 * a256((N + 3) * 8) + a256((2 * (N + 3) + 2 * (M + 3)) * 8);
    total += a256(4 * 8) + a256(4 * 4) + a256(4 * HYD_SEGL * 4) + a256(64) + a256(64);
    total += 4 * a256((N + 3) * 4) + 4 * a256((M + 3) * 4) + a256(64);  // spans, rescan flags and lists
    total += 2 * a256((N + 3) * 4) + 2 * a256(64);                      // extended spans, flags
    total += a256(kBudSlots * 8);                                       // water budget
    e = cudaMalloc(&s->arena, total);
    if (e != cudaSuccess) {
        release(s);
        return fail(HYD_ENOMEM, std::string("device arena: ") + cudaGetErrorString(e));
    }
    s->arena_bytes = total;
    cudaMemset(s->arena, 0, total);
    char* cur = (char*)s->arena;
    auto take = [&](size_t b) {
        char* q = cur;
        cur += a256(b);
        return (void*)q;
    };
    DevGrid& g = s->g;
    memset(&g, 0, sizeof g);
    g.N = N;
    g.M = M;
    g.P = s->pitch;
    g.wpr = 1;
    g.sv_cap = M + 3;
    g.su_cap = N + 3;
    double** gd[] = {&g.h,   &g.hsnham, &g.VISC,  &g.Fw,   &g.Tsxw,  &g.Tsyw,     &g.u,   &g.v,   &g.z,
                     &g.t_u, &g.t_v,    &g.t_z,   &g.Htdu, &g.Htdv,  &g.H_moi,    &g.htaiz, &g.htaiz_bd,
                     &g.Kx1, &g.Ky1,    &g.FS,    &g.tFS,  &g.VTH,   &g.Kx,       &g.Ky,  &g.Qbx, &g.Qby,
                     &g.dH,  &g.h0,     &g.dHc,    &g.dHinc};
    for (double** q : gd) *q = (double*)take(gbytes);
    s->scratch_u = (double*)take(gbytes);
    s->scratch_v = (double*)take(gbytes);
    g.khouot = (int*)take(nrow * s->pitch * sizeof(int));
    g.daui = (int*)take(nseg_rows * 4);
    g.cuoii = (int*)take(nseg_rows * 4);
    g.moci = (int*)take((N + 3) * 4);
    g.dauj = (int*)take(nseg_cols * 4);
    g.cuoij = (int*)take(nseg_cols * 4);
    g.mocj = (int*)take((M + 3) * 4);
    g.ubt = (double*)take((M + 3) * 8);
    g.ubp = (double*)take((M + 3) * 8);
    g.vbt = (double*)take((N + 3) * 8);
    g.vbd = (double*)take((N + 3) * 8);
    g.hi = (double*)take((2 * (N + 3) + 2 * (M + 3)) * 8);
    g.hmax = (double*)take(4 * 8);
    g.bienQ = (int*)take(4 * 4);
    g.btype = (int*)take(4 * HYD_SEGL * 4);
    g.status = (unsigned*)take(64);
    g.rlo = (int*)take((N + 3) * 4);
    g.rhi = (int*)take((N + 3) * 4);
    g.dirty_r = (int*)take((N + 3) * 4);
    g.dlist_r = (int*)take((N + 3) * 4);
    g.clo = (int*)take((M + 3) * 4);
    g.chi = (int*)take((M + 3) * 4);
    g.dirty_c = (int*)take((M + 3) * 4);
    g.dlist_c = (int*)take((M + 3) * 4);
    g.dctr = (unsigned*)take(64);
    g.elo = (int*)take((N + 3) * 4);
    g.ehi = (int*)take((N + 3) * 4);
    g.span_wide = (int*)take(64);
    g.dflag = (int*)take(64);
    g.clock = (double*)take(64);
    g.budget = (double*)take(kBudSlots * 8);
    if ((size_t)(cur - (char*)s->arena) > total) {
        release(s);
        return fail(HYD_ENOMEM, "arena layout overflow");
    }
    s->dp = make_dev_params(s->P);
    {
        // HYD_SWEEP_ROWS caps the rows a long line keeps in shared memory, so that tests can
        // send lines of a moderate grid through the global-scratch sweeps
        const char* rv = getenv("HYD_SWEEP_ROWS");
        e = sweep_plan(N, M, &s->plan, rv ? atoi(rv) : 0);
        s->plan_grid = s->plan.long_grid;
    }
    if (e == cudaSuccess) e = grid_setup(N, M);
    if (e == cudaSuccess && device < kMaxDevices) {
        // the fixed scratch of hyd_mass_balance_noalloc: its module is loaded now, while
        // creating a handle allocates anyway
        double* scratch = nullptr;
        e = mass_scratch_address(device, &scratch);
    }
    if (e != cudaSuccess) {
        release(s);
        return fail(HYD_ECUDA, std::string("shared-memory set-up: ") + cudaGetErrorString(e));
    }
    s->g.LT = (N + 3 + 31) / 32 * 32;
    // the seven column-major coefficient arrays outgrow L2 from about 4M cells
    s->g.tile_cols = (size_t)N * M >= ((size_t)1 << 22);
    s->g.colT_stride = (size_t)(M + 3) * s->g.LT;
    e = cudaMalloc(&s->g.colT, 7 * s->g.colT_stride * sizeof(double) + s->g.colT_stride);
    s->g.colB = (unsigned char*)(s->g.colT + 7 * s->g.colT_stride);
    s->g.rowC_stride = (size_t)(N + 3) * s->pitch;
    if (e == cudaSuccess) e = cudaMalloc(&s->g.rowC, 7 * s->g.rowC_stride * sizeof(double));
    if (e == cudaSuccess && p->precision_mode == HYD_PRECISION_MIXED) {
        // the mixed form's FP32 coefficient arrays (the FP64 ones stay for the set-up paths)
        e = cudaMalloc(&s->g.colTf, 7 * s->g.colT_stride * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&s->g.rowCf, 7 * s->g.rowC_stride * sizeof(float));
    }
    if (e != cudaSuccess) {
        release(s);
        return fail(HYD_ENOMEM, std::string("column-major scratch: ") + cudaGetErrorString(e));
    }
    s->sweep_scratch = nullptr;
    e = cudaMalloc(&s->sweep_scratch, s->plan.scratch_doubles * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s->fs_scratch, s->plan.scratch_doubles * sizeof(double));
    if (e != cudaSuccess) {
        release(s);
        return fail(HYD_ENOMEM, std::string("sweep scratch: ") + cudaGetErrorString(e));
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        release(s);
        return fail(HYD_ECUDA, std::string("create: ") + cudaGetErrorString(e));
    }
    *out = s;
    return HYD_OK;
}

int hyd_destroy(hyd_handle h) {
    if (!h) return HYD_OK;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    for (void* q : h->extra) cudaFree(q);
    for (auto& m : h->marks) {
        cudaEventDestroy(m.a);
        cudaEventDestroy(m.b);
    }
    for (cudaEvent_t e : h->event_pool) cudaEventDestroy(e);
    drop_graphs(h);
    release(h);
    return HYD_OK;
}

int hyd_set_field(hyd_handle h, const char* name, const void* host, size_t count) {
    if (!h || !name || !host) return fail(HYD_EINVAL, "null argument");
    const FieldDesc* f = find_field(name);
    if (!f) return fail(HYD_EINVAL, std::string("unknown field ") + name);
    if (count != field_count(h, f->kind)) return fail(HYD_EINVAL, std::string("wrong element count for ") + name);
    CUDA_TRY(cudaSetDevice(h->device));
    void* dst = member(h, f);
    if (f->kind == 0 || f->kind == 1) {
        const size_t es = f->kind == 0 ? 8 : 4;
        CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)h->pitch * es, host, (size_t)(h->M + 3) * es, (size_t)(h->M + 3) * es,
                                   (size_t)h->N + 3, cudaMemcpyHostToDevice, h->stream));
    } else {
        const size_t es = (f->kind >= 6) ? 8 : 4;
        CUDA_TRY(cudaMemcpyAsync(dst, host, count * es, cudaMemcpyHostToDevice, h->stream));
    }
    if (dst == (void*)h->g.khouot) {
        // new mask: new spans, and every line is rescanned at the next step
        launch_spans(h->g, h->stream);
        clear_rescan_lists(h->g, h->stream);
        h->force_rescan = 1;
        const int rc = refresh_widths(h);
        if (rc) return rc;
    } else if (f->kind >= 2 && f->kind <= 5) {
        h->force_rescan = 1;  // segment tables
    }
    // A field the elementwise kernels may read or bring up to date outside the extended
    // spans owes whole-grid passes, unless it is one of z, u, v, FS and equals there what
    // those passes would leave (t_z, t_u, t_v; tFS once a sediment pass has run).
    const DevGrid& G = h->g;
    int owed = 3;
    if (h->initialized) {
        const double* partner = nullptr;
        int i0 = 0, j0 = 0;
        if (dst == (void*)G.u) partner = G.t_u;
        else if (dst == (void*)G.v) partner = G.t_v;
        else if (dst == (void*)G.z) partner = G.t_z;
        else if (dst == (void*)G.FS) {
            owed = 2;  // read by the sediment kernels only
            if (!(h->full_pending & 2)) {
                partner = G.tFS;
                i0 = j0 = 1;
            }
        }
        if (partner) {
            const int d = outside_differs(G, (const double*)dst, partner, i0, h->N, j0, h->M, G.dflag, h->stream);
            if (d < 0) return fail(HYD_ECUDA, "set-field span check failed");
            if (!d) owed = 0;
        }
    }
    h->full_pending |= owed;
    h->epoch++;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return HYD_OK;
}

int hyd_get_field(hyd_handle h, const char* name, void* host, size_t count) {
    if (!h || !name || !host) return fail(HYD_EINVAL, "null argument");
    const FieldDesc* f = find_field(name);
    if (!f) return fail(HYD_EINVAL, std::string("unknown field ") + name);
    if (count != field_count(h, f->kind)) return fail(HYD_EINVAL, std::string("wrong element count for ") + name);
    CUDA_TRY(cudaSetDevice(h->device));
    const void* src = member(h, f);
    if (f->kind == 0 || f->kind == 1) {
        const size_t es = f->kind == 0 ? 8 : 4;
        CUDA_TRY(cudaMemcpy2DAsync(host, (size_t)(h->M + 3) * es, src, (size_t)h->pitch * es, (size_t)(h->M + 3) * es,
                                   (size_t)h->N + 3, cudaMemcpyDeviceToHost, h->stream));
    } else {
        const size_t es = (f->kind >= 6) ? 8 : 4;
        CUDA_TRY(cudaMemcpyAsync(host, src, count * es, cudaMemcpyDeviceToHost, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return HYD_OK;
}

int hyd_get_field_device(hyd_handle h, const char* name, void* dst, size_t count) {
    if (!h || !name || !dst) return fail(HYD_EINVAL, "null argument");
    const FieldDesc* f = find_field(name);
    if (!f) return fail(HYD_EINVAL, std::string("unknown field ") + name);
    if (count != field_count(h, f->kind)) return fail(HYD_EINVAL, std::string("wrong element count for ") + name);
    CUDA_TRY(cudaSetDevice(h->device));
    const void* src = member(h, f);
    if (f->kind == 0 || f->kind == 1) {
        const size_t es = f->kind == 0 ? 8 : 4;
        CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)(h->M + 3) * es, src, (size_t)h->pitch * es, (size_t)(h->M + 3) * es,
                                   (size_t)h->N + 3, cudaMemcpyDeviceToDevice, h->stream));
    } else {
        const size_t es = (f->kind >= 6) ? 8 : 4;
        CUDA_TRY(cudaMemcpyAsync(dst, src, count * es, cudaMemcpyDeviceToDevice, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return HYD_OK;
}

int hyd_get_field_async(hyd_handle h, const char* name, void* host, size_t count) {
    if (!h || !name || !host) return fail(HYD_EINVAL, "null argument");
    const FieldDesc* f = find_field(name);
    if (!f) return fail(HYD_EINVAL, std::string("unknown field ") + name);
    if (f->kind != 0) return fail(HYD_EINVAL, std::string("asynchronous reads take grid fields of doubles: ") + name);
    if (count != field_count(h, f->kind)) return fail(HYD_EINVAL, std::string("wrong element count for ") + name);
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t row = (size_t)(h->M + 3) * sizeof(double);
    const int i = h->snap_i;
    if (!h->snap[i]) CUDA_TRY(cudaMalloc(&h->snap[i], row * (h->N + 3)));
    // the read two calls back must have left this snapshot before it is overwritten
    CUDA_TRY(cudaEventSynchronize(h->ev_copied[i]));
    // packed on the device (the host copy is then one contiguous transfer)
    launch_pack_rows((const double*)member(h, f), h->pitch, (double*)h->snap[i], h->N + 3, h->M + 3, h->stream);
    CUDA_TRY(cudaEventRecord(h->ev_snap, h->stream));
    CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->ev_snap, 0));
    CUDA_TRY(cudaMemcpyAsync(host, h->snap[i], row * (h->N + 3), cudaMemcpyDeviceToHost, h->copy_stream));
    CUDA_TRY(cudaEventRecord(h->ev_copied[i], h->copy_stream));
    h->snap_i = i ^ 1;
    return HYD_OK;
}

int hyd_wait_fields(hyd_handle h) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaEventSynchronize(h->ev_copied[0]));
    CUDA_TRY(cudaEventSynchronize(h->ev_copied[1]));
    if (h->mir_open) {
        CUDA_TRY(cudaEventSynchronize(h->ev_mir[0]));
        CUDA_TRY(cudaEventSynchronize(h->ev_mir[1]));
    }
    return HYD_OK;
}

// The box of the extended spans, read back from the device (waits for the queued steps).
static int mirror_box(HydSim* h) {
    const int n = h->N + 3;
    std::vector<int> lo(n), hi(n);
    CUDA_TRY(cudaMemcpyAsync(lo.data(), h->g.elo, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaMemcpyAsync(hi.data(), h->g.ehi, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    int r0 = n, r1 = -1, c0 = h->M + 3, c1 = -1;
    for (int i = 0; i < n; i++) {
        if (hi[i] < lo[i]) continue;
        r0 = std::min(r0, i);
        r1 = std::max(r1, i);
        c0 = std::min(c0, lo[i]);
        c1 = std::max(c1, hi[i]);
    }
    h->box_r0 = r0;
    h->box_r1 = r1;
    h->box_c0 = c0;
    h->box_c1 = c1;
    h->box_epoch = h->epoch;
    return HYD_OK;
}

int hyd_mirror_open(hyd_handle h, const char* name) {
    if (!h || !name) return fail(HYD_EINVAL, "null argument");
    if (strcmp(name, "z") && strcmp(name, "u") && strcmp(name, "v"))
        return fail(HYD_EINVAL, std::string("mirrors hold z, u or v: ") + name);
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_mirror_open");
    CUDA_TRY(cudaSetDevice(h->device));
    if (h->mir_open) {
        const int rc = hyd_mirror_close(h);
        if (rc) return rc;
    }
    const size_t count = (size_t)(h->N + 3) * (h->M + 3);
    for (int k = 0; k < 2; k++) {
        CUDA_TRY(cudaMallocHost(&h->mir[k], count * sizeof(double)));
        CUDA_TRY(cudaMalloc(&h->mir_snap[k], count * sizeof(double)));
        CUDA_TRY(cudaEventCreateWithFlags(&h->ev_mir[k], cudaEventDisableTiming));
    }
    h->mir_open = 1;
    h->mir_f = find_field(name);
    int rc = hyd_get_field(h, name, h->mir[0], count);
    if (rc) return rc;
    memcpy(h->mir[1], h->mir[0], count * sizeof(double));
    h->mir_epoch[0] = h->mir_epoch[1] = h->epoch;
    h->mir_i = 0;
    return HYD_OK;
}

int hyd_mirror_update_async(hyd_handle h, const double** view, size_t* bytes) {
    if (!h || !view) return fail(HYD_EINVAL, "null argument");
    if (!h->mir_open) return fail(HYD_ESTATE, "hyd_mirror_open must precede hyd_mirror_update_async");
    CUDA_TRY(cudaSetDevice(h->device));
    const int k = h->mir_i;
    // the previous call's copy is complete on return (its view may be read from then on),
    // and the copy before it, in the slot reused here, with it (the copies run in order)
    CUDA_TRY(cudaEventSynchronize(h->ev_mir[k ^ 1]));
    const int W = h->M + 3;
    const double* src = (const double*)member(h, h->mir_f);
    size_t moved = 0;
    if (h->mir_epoch[k] != h->epoch) {
        // a whole-grid event since this copy was last brought up to date: all of it
        launch_pack_rows(src, h->pitch, (double*)h->mir_snap[k], h->N + 3, W, h->stream);
        CUDA_TRY(cudaEventRecord(h->ev_snap, h->stream));
        CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->ev_snap, 0));
        moved = sizeof(double) * (size_t)(h->N + 3) * W;
        CUDA_TRY(cudaMemcpyAsync(h->mir[k], h->mir_snap[k], moved, cudaMemcpyDeviceToHost, h->copy_stream));
    } else {
        if (h->box_epoch != h->epoch || h->box_r1 < 0) {
            const int rc = mirror_box(h);
            if (rc) return rc;
        }
        if (h->box_r1 >= h->box_r0 && h->box_c1 >= h->box_c0) {
            const int nr = h->box_r1 - h->box_r0 + 1, nc = h->box_c1 - h->box_c0 + 1;
            launch_pack_rows(src + (size_t)h->box_r0 * h->pitch + h->box_c0, h->pitch, (double*)h->mir_snap[k], nr, nc,
                             h->stream);
            CUDA_TRY(cudaEventRecord(h->ev_snap, h->stream));
            CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->ev_snap, 0));
            CUDA_TRY(cudaMemcpy2DAsync(h->mir[k] + (size_t)h->box_r0 * W + h->box_c0, sizeof(double) * W,
                                       h->mir_snap[k], sizeof(double) * nc, sizeof(double) * nc, nr,
                                       cudaMemcpyDeviceToHost, h->copy_stream));
            moved = sizeof(double) * (size_t)nr * nc;
        }
    }
    CUDA_TRY(cudaEventRecord(h->ev_mir[k], h->copy_stream));
    h->mir_epoch[k] = h->epoch;
    h->mir_i = k ^ 1;
    *view = h->mir[k];
    if (bytes) *bytes = moved;
    return HYD_OK;
}

int hyd_mirror_close(hyd_handle h) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    if (!h->mir_open) return HYD_OK;
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->copy_stream));
    for (int k = 0; k < 2; k++) {
        cudaFreeHost(h->mir[k]);
        cudaFree(h->mir_snap[k]);
        cudaEventDestroy(h->ev_mir[k]);
        h->mir[k] = nullptr;
        h->mir_snap[k] = nullptr;
        h->ev_mir[k] = nullptr;
    }
    h->mir_open = 0;
    return HYD_OK;
}

int hyd_set_boundary(hyd_handle h, const int* boundary_type, const double* const* tables, const double* const* cc,
                     const int* nseg, int total_time) {
    if (!h || !boundary_type || !tables || !cc || !nseg) return fail(HYD_EINVAL, "null argument");
    if (total_time < 2) return fail(HYD_EINVAL, "total_time must be >= 2");
    CUDA_TRY(cudaSetDevice(h->device));
    int bienQ[4];
    for (int e = 0; e < 4; e++) {
        bienQ[e] = 0;
        for (int k = 0; k < HYD_SEGL; k++) {
            const int bt = boundary_type[e * HYD_SEGL + k];
            if (bt < 0 || bt > 2) return fail(HYD_EINVAL, "boundary_type values must be 0, 1 or 2");
            if (bt == 2) bienQ[e] = 1;
        }
        if (nseg[e] < 0 || nseg[e] > HYD_SEGL) return fail(HYD_EINVAL, "nseg out of range");
    }
    CUDA_TRY(cudaMemcpyAsync(h->g.bienQ, bienQ, sizeof bienQ, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->g.btype, boundary_type, 4 * HYD_SEGL * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    // one block for the eight tables (each padded as the reference's reads allow: an edge
    // without segments still gets one zero row, and two spare values)
    size_t off[8], total = 0;
    for (int q = 0; q < 8; q++) {
        const int e = q & 3;
        off[q] = total;
        total += ((size_t)(nseg[e] > 0 ? nseg[e] : 1) * total_time + 2 + 31) / 32 * 32;
    }
    for (int e = 0; e < 4; e++)
        if (nseg[e] > 0 && (!tables[e] || !cc[e])) return fail(HYD_EINVAL, "missing boundary table");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->bnd_block) {
        cudaFree(h->bnd_block);
        h->bnd_block = nullptr;
    }
    if (h->bnd_stage) {
        cudaFreeHost(h->bnd_stage);
        h->bnd_stage = nullptr;
    }
    CUDA_TRY(cudaMalloc(&h->bnd_block, total * sizeof(double)));
    CUDA_TRY(cudaMallocHost(&h->bnd_stage, total * sizeof(double)));
    h->bnd_doubles = total;
    memset(h->bnd_stage, 0, total * sizeof(double));
    for (int e = 0; e < 4; e++) {
        if (nseg[e] <= 0) continue;
        memcpy(h->bnd_stage + off[e], tables[e], (size_t)nseg[e] * total_time * 8);
        memcpy(h->bnd_stage + off[4 + e], cc[e], (size_t)nseg[e] * total_time * 8);
    }
    CUDA_TRY(cudaMemcpyAsync(h->bnd_block, h->bnd_stage, total * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    for (int e = 0; e < 4; e++) {
        h->g.bc[e] = h->bnd_block + off[e];
        h->g.cc[e] = h->bnd_block + off[4 + e];
    }
    h->g.total_time = total_time;
    for (int e = 0; e < 4; e++) h->bnd_nseg[e] = nseg[e];
    h->have_boundary = 1;
    h->epoch++;  // the tables moved
    drop_graphs(h);
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return HYD_OK;
}

int hyd_update_boundary(hyd_handle h, const double* const* tables, const double* const* cc) {
    if (!h || !tables || !cc) return fail(HYD_EINVAL, "null argument");
    if (!h->have_boundary) return fail(HYD_ESTATE, "hyd_set_boundary must precede hyd_update_boundary");
    for (int e = 0; e < 4; e++)
        if (h->bnd_nseg[e] > 0 && (!tables[e] || !cc[e])) return fail(HYD_EINVAL, "missing boundary table");
    CUDA_TRY(cudaSetDevice(h->device));
    // the staging copy is reused: the previous upload must have left it
    CUDA_TRY(cudaEventSynchronize(h->ev_bnd));
    for (int e = 0; e < 4; e++) {
        if (h->bnd_nseg[e] <= 0) continue;
        const size_t n = (size_t)h->bnd_nseg[e] * h->g.total_time;
        memcpy(h->bnd_stage + (h->g.bc[e] - h->bnd_block), tables[e], n * 8);
        memcpy(h->bnd_stage + (h->g.cc[e] - h->bnd_block), cc[e], n * 8);
    }
    // small tables travel in a kernel's parameters (no copy engine, and the staging copy is
    // free again at once); larger ones as one copy, which the next call waits for
    if (!launch_put_doubles(h->bnd_block, h->bnd_stage, (int)h->bnd_doubles, h->stream)) {
        CUDA_TRY(cudaMemcpyAsync(h->bnd_block, h->bnd_stage, h->bnd_doubles * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
        CUDA_TRY(cudaEventRecord(h->ev_bnd, h->stream));
    }
    CUDA_TRY(cudaGetLastError());
    return HYD_OK;
}

static int init_common(HydSim* h, double t_start, int pickup) {
    if (!h->have_boundary) return fail(HYD_ESTATE, "hyd_set_boundary must precede hyd_init");
    CUDA_TRY(cudaSetDevice(h->device));
    const int* keep = nullptr;
    if (pickup) {
        // the caller's mask, parked in a smoothing partner (rewritten by the first step)
        CUDA_TRY(cudaMemcpyAsync(h->scratch_u, h->g.khouot, sizeof(int) * (size_t)(h->N + 3) * h->pitch,
                                 cudaMemcpyDeviceToDevice, h->stream));
        keep = (const int*)h->scratch_u;
    }
    launch_init_kernels(h->g, h->dp, keep, h->stream);
    CUDA_TRY(cudaMemsetAsync(h->g.budget, 0, kBudSlots * sizeof(double), h->stream));
    launch_bed_reset(h->g, h->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->t = t_start;
    h->initialized = 1;
    h->force_rescan = 0;  // the set-up scanned every line
    h->full_pending = 3;
    h->epoch++;
    int rc = refresh_widths(h);
    if (rc) return rc;
    rc = set_clock(h, t_start);
    if (rc) return rc;
    return check_device_status(h);
}

int hyd_init(hyd_handle h, double t_start) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    return init_common(h, t_start, 0);
}

int hyd_init_pickup(hyd_handle h, double t_start) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    return init_common(h, t_start, 1);
}

// The launch sequence of one full step (Engine.py:144-366).  sed1/sed2: sediment phase
// active in the first/second half-step (t >= sediment_start); bed: Exner update at the end.
static void launch_step(HydSim* s, int sed1, int sed2, int bed, int force = 0, int full_h = 0, int full_s = 0) {
    DevGrid& g = s->g;
    const DevParams& p = s->dp;
    cudaStream_t st = s->stream;
    // channel mode writes levels at table-dependent places: always the whole grid
    const int fh = full_h || p.channel, fsd = full_s || p.channel;
    // ---- half-step 1: implicit along i (columns), explicit v
    // (the first launch advances the clock and applies the boundary values)
    int start_idx = 2, end_idx = s->M;
    if (p.channel && s->P.kenhhepd == 1) {
        start_idx = 3;
        end_idx = s->M - 1;
    }
    { PHASE(PH_COEF_UZ); launch_coef_bnd(g, p, 0, 3, st); }
    { PHASE(PH_SWEEP_UZ); launch_sweep_uz(g, p, s->plan, start_idx, end_idx, s->solver, s->sweep_scratch, st); }
    // span-limited passes: the half-step's water budget beside the smoothing and explicit v
    // (joined before the row resets change the mask); whole-grid passes keep it in the
    // smoothing's launches
    if (!fh) {
        cudaEventRecord(s->ev_bfork, st);
        cudaStreamWaitEvent(s->side2, s->ev_bfork, 0);
        launch_budget_half(g, p, 1, s->side2);
        cudaEventRecord(s->ev_bjoin, s->side2);
    }
    { PHASE(PH_SMOOTH); launch_smooth(g, p, 1, s->scratch_u, fh, 0, 0, fh, st); }
    std::swap(g.t_u, s->scratch_u);
    { PHASE(PH_EXPL_V); launch_explicit_v(g, p, s->thr_r, st); }
    { PHASE(PH_SMOOTH); launch_smooth(g, p, 0, s->scratch_v, fh, 0, 0, 0, st); }
    std::swap(g.t_v, s->scratch_v);
    if (force) launch_mark_all_cols(g, st);
    if (!fh) cudaStreamWaitEvent(st, s->ev_bjoin, 0);
    { PHASE(PH_RESET_ROWS); launch_reset_rows(g, p, force, s->thr_r, st); }
    // after a span-limited pass the update, the column rescan and (with sediment) VTH/K
    // share one launch; whole-grid passes keep them apart
    const int fuse1 = !fh && !fsd;
    if (!fh) {
        PHASE(PH_POST);
        launch_post_fused(g, p, 0, sed1 && fuse1, st);
    } else {
        { PHASE(PH_POST); launch_post(g, p, fh, st); }
        { PHASE(PH_SCAN); launch_scan_cols(g, p, st); }
    }
    // With span-limited passes the first half-step's sediment (FSj coefficients, sweep and
    // update) runs on the side stream beside the second half-step up to its explicit u: it
    // reads u, v (equal to t_u, t_v after the update above), FS, H_moi, VTH, K and the
    // column segments, none of which those launches write, and its coefficients live in
    // column-major slots they do not use.  The second half-step's boundary then writes
    // velocities and levels only; its inflow concentrations (FS) follow the join, in the
    // smoothing launch that precedes the column resets.
    const int overlap = sed1 && fuse1 && !p.channel;
    if (overlap) {
        cudaEventRecord(s->ev_fork, st);
        cudaStreamWaitEvent(s->side, s->ev_fork, 0);
        { PHASE_ON(PH_COEF_FSJ, s->side); launch_coef_fsj(g, p, 0, s->side); }
        { PHASE_ON(PH_FS_J, s->side); launch_fs_sweep_j(g, p, s->plan, 0, s->solver, s->fs_scratch, s->side); }
        { PHASE_ON(PH_UPDATE_FS, s->side); launch_update_fs(g, fsd, s->side); }
        cudaEventRecord(s->ev_join, s->side);
    } else if (sed1) {
        if (!(sed1 && fuse1)) { PHASE(PH_VTH); launch_vth_hesok(g, p, fsd, 0, st); }
        { PHASE(PH_COEF_FSJ); launch_coef_fsj(g, p, 0, st); }
        { PHASE(PH_FS_J); launch_fs_sweep_j(g, p, s->plan, 0, s->solver, s->fs_scratch, st); }
        { PHASE(PH_UPDATE_FS); launch_update_fs(g, fsd, st); }
    }
    // ---- half-step 2: implicit along j (rows), explicit u
    { PHASE(PH_BOUNDARY); launch_coef_bnd(g, p, 1, overlap ? 1 : 3, st); }
    start_idx = 2;
    end_idx = s->N;
    if (p.channel && s->P.kenhhepng == 1) {
        start_idx = 3;
        end_idx = s->N;
    }
    { PHASE(PH_SWEEP_VZ); launch_sweep_vz(g, p, s->plan, start_idx, end_idx, s->solver, s->sweep_scratch, st); }
    if (!fh) {  // the budget beside the launches up to the column resets
        cudaEventRecord(s->ev_bfork, st);
        cudaStreamWaitEvent(s->side2, s->ev_bfork, 0);
        launch_budget_half(g, p, 0, s->side2);
        cudaEventRecord(s->ev_bjoin, s->side2);
    }
    { PHASE(PH_SMOOTH); launch_smooth(g, p, 0, s->scratch_v, fh, 0, 0, fh, st); }
    std::swap(g.t_v, s->scratch_v);
    { PHASE(PH_COEF_EU); launch_coef_eu(g, p, st); }
    { PHASE(PH_EXPL_U); launch_explicit_u(g, p, s->thr_c, st); }
    if (overlap) cudaStreamWaitEvent(st, s->ev_join, 0);
    { PHASE(PH_SMOOTH); launch_smooth(g, p, 1, s->scratch_u, fh, 1, overlap, 0, st); }
    std::swap(g.t_u, s->scratch_u);
    if (!fh) cudaStreamWaitEvent(st, s->ev_bjoin, 0);
    { PHASE(PH_RESET_COLS); launch_reset_cols(g, p, 0, s->thr_c, st); }
    if (!fh) {
        PHASE(PH_POST);
        launch_post_fused(g, p, 1, sed2 && fuse1, st);
    } else {
        { PHASE(PH_POST); launch_post(g, p, fh, st); }
        { PHASE(PH_SCAN); launch_scan_rows(g, p, st); }
    }
    if (sed2) {
        if (!(sed2 && fuse1)) { PHASE(PH_VTH); launch_vth_hesok(g, p, fsd, 1, st); }
        { PHASE(PH_FS_I); launch_fs_sweep_i(g, p, s->plan, 1, s->solver, s->fs_scratch, st); }
        { PHASE(PH_UPDATE_FS); launch_update_fs(g, fsd, st); }
        start_idx = 3;
        end_idx = s->N - 1;
    }
    if (bed) {
        PHASE(PH_BED);
        launch_bed(g, p, start_idx, end_idx, st);
    }
    if (full_h && !p.channel) launch_widen_spans(g, st);
    s->start_idx = start_idx;
    s->end_idx = end_idx;
}

// The captured graph of one step variant (built on first use).  timed: the variant with
// the phase events captured in it (their pairs are read after each replay).
static cudaGraphExec_t step_graph(HydSim* s, int mask, int timed = 0) {
    cudaGraphExec_t* slot = timed ? &s->tgraph[mask] : &s->graph[mask];
    if (*slot) return *slot;
    const long long before = hyd_kernel_launches_add(0);
    if (timed) s->mark_sink = &s->tmarks[mask];
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        s->mark_sink = nullptr;
        return nullptr;
    }
    launch_step(s, mask & 1, (mask >> 1) & 1, (mask >> 2) & 1);
    s->mark_sink = nullptr;
    cudaGraph_t graph = nullptr;
    if (cudaStreamEndCapture(s->stream, &graph) != cudaSuccess || !graph) return nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return nullptr;
    const long long after = hyd_kernel_launches_add(0);
    s->graph_kernels[mask] = after - before;
    hyd_kernel_launches_add(-(after - before));
    *slot = exec;
    return exec;
}

int hyd_step(hyd_handle h, int nsteps, int sync, double* t_out) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_step");
    if (nsteps < 0) return fail(HYD_EINVAL, "nsteps < 0");
    CUDA_TRY(cudaSetDevice(h->device));
    // the hourly tables must cover the last hour index reached (support_funcs.cu:565)
    const double t_end = h->t + nsteps * h->P.dT;
    if ((int)(t_end / 3600) + 1 >= h->g.total_time)
        return fail(HYD_EINVAL, "boundary tables too short for the requested time span");
    double t = h->t;
    for (int n = 0; n < nsteps; n++) {
        const double t1 = t + h->P.dT * 0.5;
        const double t2 = t1 + h->P.dT * 0.5;
        const int sed1 = t1 >= h->P.sediment_start;
        const int sed2 = t2 >= h->P.sediment_start;
        // Engine.py:364: int(t) % bed_change_start == 0 and t integral; with a bed period,
        // every bed_period s from bed_change_start on
        const double it = (double)(long long)t2;
        const int bed = h->P.bed_period > 0
                            ? (t2 - it == 0 && t2 >= h->P.bed_change_start && std::fmod(it, h->P.bed_period) == 0)
                            : (std::fmod(it, h->P.bed_change_start) == 0 && t2 - it == 0);
        const int mask = sed1 | (sed2 << 1) | (bed << 2);
        const int force = h->force_rescan;
        h->force_rescan = 0;
        const int full_h = h->full_pending & 1;
        const int full_s = (sed1 || sed2) ? (h->full_pending >> 1) & 1 : 0;
        h->full_pending &= ~(full_h | (full_s << 1));
        const int special = force || full_h || full_s;
        // channel mode writes levels at table-dependent places every step
        if (special || h->dp.channel) h->epoch++;
        cudaGraphExec_t exec = (h->use_graphs && !special) ? step_graph(h, mask, h->timing) : nullptr;
        if (exec) {
            CUDA_TRY(cudaGraphLaunch(exec, h->stream));
            hyd_kernel_launches_add(h->graph_kernels[mask]);
            if (h->timing) {
                // the replay's phase events, read before the next replay reuses them
                CUDA_TRY(cudaStreamSynchronize(h->stream));
                for (auto& m : h->tmarks[mask]) {
                    float ms = 0;
                    cudaEventElapsedTime(&ms, m.a, m.b);
                    h->phase_ms[m.phase] += ms;
                    h->phase_n[m.phase] += 1;
                }
            }
        } else {
            launch_step(h, sed1, sed2, bed, force, full_h, full_s);
        }
        t = t2;
    }
    h->t = t;
    CUDA_TRY(cudaGetLastError());
    if (t_out) *t_out = t;
    if (sync) return check_device_status(h);
    return HYD_OK;
}

// Non-finite values in z, u, v, FS (the mass-balance kernels' count), on the handle's
// stream; -1 on error.
static long long count_nonfinite(HydSim* h) {
    const int nb = 148;
    if (!h->run_part && cudaMalloc(&h->run_part, ((size_t)nb * 5 + 5) * sizeof(double)) != cudaSuccess) return -1;
    k_mass_partial<<<nb, 256, 0, h->stream>>>(h->g, h->run_part);
    k_mass_final<<<1, 32, 0, h->stream>>>(h->run_part, nb, h->run_part + nb * 5);
    hyd_kernel_launches_add(2);
    double r[5];
    if (cudaMemcpyAsync(r, h->run_part + nb * 5, sizeof r, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return -1;
    return (long long)r[4];
}

// An output time of hyd_run: t integral and a whole multiple of interval (Engine.py:398).
static bool run_output_time(double t, double interval) {
    if (!(interval > 0)) return false;
    const double it = (double)(long long)t;
    return t - it == 0 && std::fmod(it, interval) == 0;
}

int hyd_run(hyd_handle h, double Tmax, double interval, hyd_run_callback cb, void* user, double* t_out) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_run");
    CUDA_TRY(cudaSetDevice(h->device));
    double t = h->t;
    while (t < Tmax) {
        // the steps up to the next output time or the end (the host's time arithmetic:
        // two half-step increments per step, Engine.py:146,260)
        int n = 0;
        double tn = t;
        do {
            tn = tn + h->P.dT * 0.5;
            tn = tn + h->P.dT * 0.5;
            n++;
        } while (tn < Tmax && !run_output_time(tn, interval));
        int rc = hyd_step(h, n, 0, &t);
        if (rc) return rc;
        if (run_output_time(t, interval) || t >= Tmax) {
            const long long bad = count_nonfinite(h);
            if (bad < 0) return fail(HYD_ECUDA, "hyd_run: the non-finite check failed");
            rc = check_device_status(h);
            if (rc) return rc;
            if (bad > 0) {
                if (t_out) *t_out = t;
                return fail(HYD_EDEVICE, "non-finite values in z, u, v or FS at t = " + std::to_string(t) + " s (" +
                                             std::to_string(bad) + " values)");
            }
            if (cb && cb(h, t, user)) break;
        }
    }
    if (t_out) *t_out = t;
    return HYD_OK;
}

int hyd_set_params(hyd_handle h, const HydCaseParams* p) {
    if (!h || !p) return fail(HYD_EINVAL, "null argument");
    if (p->dT <= 0 || p->dX <= 0 || p->dY <= 0) return fail(HYD_EINVAL, "dX, dY, dT must be positive");
    if (p->precision_mode != HYD_PRECISION_FP64 && p->precision_mode != HYD_PRECISION_MIXED)
        return fail(HYD_EINVAL, "precision_mode must be HYD_PRECISION_FP64 or HYD_PRECISION_MIXED");
    if (p->precision_mode != h->P.precision_mode)
        return fail(HYD_EINVAL, "precision_mode is fixed when the handle is created");
    if (p->bed_feedback && !(p->morfac > 0)) return fail(HYD_EINVAL, "bed_feedback needs morfac > 0");
    CUDA_TRY(cudaSetDevice(h->device));
    const int feedback_on = p->bed_feedback && !h->P.bed_feedback;
    h->P = *p;
    h->dp = make_dev_params(h->P);
    h->full_pending = 3;
    h->epoch++;
    drop_graphs(h);
    if (feedback_on && h->initialized) {  // the applied changes start from the bed as it is
        launch_bed_reset(h->g, h->stream);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    return HYD_OK;
}

int hyd_get_time(hyd_handle h, double* t) {
    if (!h || !t) return fail(HYD_EINVAL, "null argument");
    *t = h->t;
    return HYD_OK;
}

int hyd_set_time(hyd_handle h, double t) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_set_time");
    if (!(t >= 0.0)) return fail(HYD_EINVAL, "t must be >= 0");
    if ((int)(t / 3600) + 1 >= h->g.total_time) return fail(HYD_EINVAL, "boundary tables too short for t");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->t = t;
    return set_clock(h, t);
}

int hyd_checkpoint(hyd_handle h, int restore) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_checkpoint");
    CUDA_TRY(cudaSetDevice(h->device));
    const size_t bytes = h->arena_bytes + h->g.colT_stride;  // arena, then the mask bytes
    unsigned char* colB = h->g.colB;
    if (!restore) {
        if (!h->ck_arena) CUDA_TRY(cudaMalloc(&h->ck_arena, bytes));
        char* dst = (char*)h->ck_arena;
        CUDA_TRY(cudaMemcpyAsync(dst, h->arena, h->arena_bytes, cudaMemcpyDeviceToDevice, h->stream));
        CUDA_TRY(cudaMemcpyAsync(dst + h->arena_bytes, colB, h->g.colT_stride, cudaMemcpyDeviceToDevice, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->ck_t = h->t;
        h->ck_start = h->start_idx;
        h->ck_end = h->end_idx;
        h->ck_full = h->full_pending;
        h->ck_force = h->force_rescan;
        h->ck_valid = 1;
        return HYD_OK;
    }
    if (!h->ck_valid) return fail(HYD_ESTATE, "no checkpoint saved on this handle");
    const char* src = (const char*)h->ck_arena;
    CUDA_TRY(cudaMemcpyAsync(h->arena, src, h->arena_bytes, cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(colB, src + h->arena_bytes, h->g.colT_stride, cudaMemcpyDeviceToDevice, h->stream));
    h->t = h->ck_t;
    h->start_idx = h->ck_start;
    h->end_idx = h->ck_end;
    h->full_pending = h->ck_full;
    h->force_rescan = h->ck_force;
    h->epoch++;
    return set_clock(h, h->t);  // synchronises the stream
}

// The steady residual; with `status`, the device status word is read back in the same
// synchronisation (the quasi-steady period's warm steps run without a check of their own).
static int steady_residual(HydSim* h, int snapshot, double* out, unsigned* status) {
    const size_t field = (size_t)(h->N + 3) * h->pitch;
    const int nb = 2 * 148;
    if (!h->res_buf) {
        CUDA_TRY(cudaMalloc(&h->res_buf, (3 * field + (size_t)nb * 4 + 4) * sizeof(double)));
        h->res_valid = 0;
    }
    double *u0 = h->res_buf, *v0 = u0 + field, *z0 = v0 + field, *part = z0 + field, *tot = part + (size_t)nb * 4;
    launch_steady_residual(h->g, u0, v0, z0, snapshot, part, nb, tot, h->stream);
    CUDA_TRY(cudaGetLastError());
    double sums[4];
    CUDA_TRY(cudaMemcpyAsync(sums, tot, sizeof sums, cudaMemcpyDeviceToHost, h->stream));
    if (status) CUDA_TRY(cudaMemcpyAsync(status, h->g.status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (!h->res_valid || !(sums[1] > 0) || !(sums[3] > 0)) {
        out[0] = out[1] = HUGE_VAL;  // no snapshot yet, no wet cell or no flow: not steady
    } else {
        out[0] = std::sqrt(sums[0] / sums[1]);
        out[1] = std::sqrt(sums[2] / sums[3]);
        if (!std::isfinite(out[0])) out[0] = HUGE_VAL;
        if (!std::isfinite(out[1])) out[1] = HUGE_VAL;
    }
    if (snapshot) h->res_valid = 1;
    return HYD_OK;
}

int hyd_steady_residual(hyd_handle h, int snapshot, double* out, int n) {
    if (!h || !out || n < 2) return fail(HYD_EINVAL, "need 2 output slots");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_steady_residual");
    CUDA_TRY(cudaSetDevice(h->device));
    return steady_residual(h, snapshot, out, nullptr);
}

int hyd_quasi_steady_period(hyd_handle h, double period, int warm, int min_warm, double gate, const float* du,
                            const float* dv, const float* dz, int i0, int j0, int rows, int cols, long long ld,
                            int retry, int* result) {
    if (!h || !result) return fail(HYD_EINVAL, "null argument");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_quasi_steady_period");
    const double dT = h->P.dT;
    if (!(period > 0) || warm < 2) return fail(HYD_EINVAL, "period must be > 0 and warm >= 2");
    const long long nper = llround(period / dT);
    if (nper < warm || std::fabs((double)nper * dT - period) > 1e-9 * period)
        return fail(HYD_EINVAL, "period must be a whole number of steps, at least warm");
    if (min_warm < 1) min_warm = 1;
    if (min_warm > warm - 1) min_warm = warm - 1;
    const double t_end = h->t + period;
    int rc = hyd_checkpoint(h, 0);
    if (rc) return rc;
    long long steps = 0;
    // the warm steps from the current state: ok once the gate passes (and the period's last
    // step, with its bed update, is taken); a device check that fails (e.g. a line with
    // more than 20 wet segments) rejects the state like a residual above the gate
    auto warm_phase = [&](int& ok) -> int {
        ok = 0;
        int e = hyd_set_time(h, t_end - warm * dT);
        if (e) return e;
        double r[2], t;
        e = hyd_steady_residual(h, 1, r, 2);
        if (e) return e;
        for (int k = 1; k < warm; k++) {
            e = hyd_step(h, 1, 0, &t);
            if (e) return e;
            unsigned st = 0;
            e = steady_residual(h, 1, r, &st);
            if (e) return e;
            if (st & HYD_ST_SEG_OVERFLOW) break;
            if (k >= min_warm && r[0] < gate && r[1] < gate) {
                double mb[5];
                e = hyd_mass_balance(h, mb, 5);
                if (e) return e;
                if (mb[4] != 0) continue;
                e = hyd_set_time(h, t_end - dT);
                if (e) return e;
                e = hyd_step(h, 1, 1, &t);  // the period's last step: the bed update on the accepted state
                if (e == HYD_EDEVICE) break;
                if (e) return e;
                steps += k + 1;
                ok = 1;
                return HYD_OK;
            }
        }
        steps += warm - 1;
        return HYD_OK;
    };
    int jumped = 0, ok = 0;
    if (du && dv && dz && rows > 0 && cols > 0) {
        rc = hyd_add_levels(h, du, dv, dz, i0, j0, rows, cols, ld);
        if (rc) return rc;
        jumped = 1;
    }
    rc = warm_phase(ok);
    if (rc) return rc;
    if (!ok && jumped && retry) {  // the jump rejected: the previous state as the warm start
        rc = hyd_checkpoint(h, 1);
        if (rc) return rc;
        jumped = 0;
        rc = warm_phase(ok);
        if (rc) return rc;
    }
    if (!ok) {  // not steady within the warm steps: the period stepped plainly
        rc = hyd_checkpoint(h, 1);
        if (rc) return rc;
        double t;
        rc = hyd_step(h, (int)nper, 1, &t);
        if (rc) return rc;
        steps += nper;
    }
    result[0] = ok;
    result[1] = ok && jumped;
    result[2] = (int)steps;
    return HYD_OK;
}

int hyd_add_levels(hyd_handle h, const float* du, const float* dv, const float* dz, int i0, int j0, int rows,
                   int cols, long long ld) {
    if (!h || !du || !dv || !dz) return fail(HYD_EINVAL, "null argument");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_add_levels");
    if (rows < 0 || cols < 0 || ld < cols || i0 < 0 || j0 < 0 || i0 + rows > h->N + 3 || j0 + cols > h->M + 3)
        return fail(HYD_EINVAL, "rectangle outside the grid");
    if (!rows || !cols) return HYD_OK;
    CUDA_TRY(cudaSetDevice(h->device));
    launch_add_levels(h->g, h->dp, du, dv, dz, i0, j0, rows, cols, ld, h->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->epoch++;
    return HYD_OK;
}

int hyd_synchronize(hyd_handle h) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaGetLastError());
    return check_device_status(h);
}

int hyd_mass_balance(hyd_handle h, double* out, int n) {
    if (!h || !out || n < 5) return fail(HYD_EINVAL, "need 5 output slots");
    CUDA_TRY(cudaSetDevice(h->device));
    const int nb = 148;
    double* part = nullptr;
    CUDA_TRY(cudaMallocAsync(&part, (size_t)nb * 5 * 8 + 5 * 8, h->stream));
    k_mass_partial<<<nb, 256, 0, h->stream>>>(h->g, part);
    k_mass_final<<<1, 32, 0, h->stream>>>(part, nb, part + nb * 5);
    hyd_kernel_launches_add(2);
    double r[5];
    CUDA_TRY(cudaMemcpyAsync(r, part + nb * 5, sizeof r, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaFreeAsync(part, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const double area = h->P.dX * h->P.dY;
    out[0] = r[0] * area;
    out[1] = r[1] * area;
    out[2] = r[2] * area;
    out[3] = r[3];
    out[4] = r[4];
    return HYD_OK;
}

int hyd_mass_budget(hyd_handle h, double* out, int n) {
    if (!h || !out || n < 10) return fail(HYD_EINVAL, "need at least 10 output slots");
    if (!h->initialized) return fail(HYD_ESTATE, "hyd_init must precede hyd_mass_budget");
    CUDA_TRY(cudaSetDevice(h->device));
    double b[kBudSlots];
    CUDA_TRY(cudaMemcpyAsync(b, h->g.budget, sizeof b, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const double area = h->P.dX * h->P.dY;
    double net = 0, gin = 0, gout = 0;
    for (int e = 0; e < 4; e++) {
        net += b[kBudNet + e];
        gin += b[kBudIn + e];
        gout += b[kBudOut + e];
        out[6 + e] = b[kBudNet + e];
    }
    out[0] = net;
    out[1] = gin;
    out[2] = gout;
    out[3] = b[kBudOpen] * area;
    out[4] = b[kBudClose] * area;
    out[5] = b[kBudBed] * area;
    if (n > 10) out[10] = b[kBudJump] * area;
    if (n > 11) out[11] = b[kBudLeak];
    return HYD_OK;
}

int hyd_mass_balance_noalloc(hyd_handle h, int nblocks, double* out, int n) {
    if (!h || !out || n < 5) return fail(HYD_EINVAL, "need 5 output slots");
    if (nblocks < 1 || nblocks > HYD_MASS_NOALLOC_MAX_BLOCKS)
        return fail(HYD_EINVAL, "nblocks must be in 1.." + std::to_string(HYD_MASS_NOALLOC_MAX_BLOCKS) +
                                    " (the static scratch holds that many blocks of partial sums)");
    if (h->device < 0 || h->device >= kMaxDevices) return fail(HYD_EINVAL, "device index beyond the scratch table");
    CUDA_TRY(cudaSetDevice(h->device));
    double* part = nullptr;
    {
        // found by hyd_create already; looked up here only if that failed
        const cudaError_t e = mass_scratch_address(h->device, &part);
        if (e != cudaSuccess) return fail(HYD_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    k_mass_partial<<<nblocks, 256, 0, h->stream>>>(h->g, part);
    k_mass_final<<<1, 32, 0, h->stream>>>(part, nblocks, part + nblocks * 5);
    hyd_kernel_launches_add(2);
    CUDA_TRY(cudaGetLastError());
    double r[5];
    CUDA_TRY(cudaMemcpyAsync(r, part + nblocks * 5, sizeof r, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const double area = h->P.dX * h->P.dY;
    out[0] = r[0] * area;
    out[1] = r[1] * area;
    out[2] = r[2] * area;
    out[3] = r[3];
    out[4] = r[4];
    return HYD_OK;
}

int hyd_state_size(hyd_handle h, size_t* bytes) {
    if (!h || !bytes) return fail(HYD_EINVAL, "null argument");
    size_t b = 64;
    for (const FieldDesc& f : kFieldTable) {
        const size_t es = (f.kind == 0 || f.kind >= 6) ? 8 : 4;
        b += field_count(h, f.kind) * es;
    }
    b += (size_t)(h->N + 3) * (h->M + 3) * 8;  // VISCOIDX
    *bytes = b;
    return HYD_OK;
}

int hyd_get_state(hyd_handle h, void* buf, size_t bytes) {
    size_t need = 0;
    int rc = hyd_state_size(h, &need);
    if (rc) return rc;
    if (!buf || bytes < need) return fail(HYD_EINVAL, "state buffer too small");
    char* p = (char*)buf;
    memset(p, 0, 64);
    memcpy(p, &h->t, 8);
    memcpy(p + 8, &h->N, 4);
    memcpy(p + 12, &h->M, 4);
    memcpy(p + 16, &h->start_idx, 4);
    memcpy(p + 20, &h->end_idx, 4);
    p += 64;
    for (const FieldDesc& f : kFieldTable) {
        const size_t es = (f.kind == 0 || f.kind >= 6) ? 8 : 4;
        const size_t n = field_count(h, f.kind);
        rc = hyd_get_field(h, f.name, p, n);
        if (rc) return rc;
        p += n * es;
    }
    rc = hyd_get_field(h, "VISCOIDX", p, (size_t)(h->N + 3) * (h->M + 3));
    if (rc) return rc;
    return HYD_OK;
}

int hyd_set_state(hyd_handle h, const void* buf, size_t bytes) {
    size_t need = 0;
    int rc = hyd_state_size(h, &need);
    if (rc) return rc;
    if (!buf || bytes < need) return fail(HYD_EINVAL, "state buffer too small");
    const char* p = (const char*)buf;
    int n0, m0;
    memcpy(&n0, p + 8, 4);
    memcpy(&m0, p + 12, 4);
    if (n0 != h->N || m0 != h->M) return fail(HYD_EINVAL, "state image is for a different grid");
    memcpy(&h->t, p, 8);
    memcpy(&h->start_idx, p + 16, 4);
    memcpy(&h->end_idx, p + 20, 4);
    p += 64;
    for (const FieldDesc& f : kFieldTable) {
        const size_t es = (f.kind == 0 || f.kind >= 6) ? 8 : 4;
        const size_t n = field_count(h, f.kind);
        rc = hyd_set_field(h, f.name, p, n);
        if (rc) return rc;
        p += n * es;
    }
    rc = hyd_set_field(h, "VISCOIDX", p, (size_t)(h->N + 3) * (h->M + 3));
    if (rc) return rc;
    h->initialized = 1;
    launch_bed_reset(h->g, h->stream);  // h0 = h - dH for the restored bed
    CUDA_TRY(cudaGetLastError());
    rc = set_clock(h, h->t);
    if (rc) return rc;
    return HYD_OK;
}

int hyd_device_status(hyd_handle h, unsigned* status) {
    if (!h || !status) return fail(HYD_EINVAL, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpyAsync(status, h->g.status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return HYD_OK;
}

int hyd_get_stream(hyd_handle h, void** stream) {
    if (!h || !stream) return fail(HYD_EINVAL, "null argument");
    *stream = (void*)h->stream;
    return HYD_OK;
}

int hyd_set_timing_phases(hyd_handle h, unsigned phase_mask) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    phase_mask &= (1u << PH_COUNT) - 1u;
    if (phase_mask != h->timing) {
        // the timed graphs hold the event records of the previous selection
        CUDA_TRY(cudaSetDevice(h->device));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        for (int k = 0; k < 8; k++) {
            if (h->tgraph[k]) cudaGraphExecDestroy(h->tgraph[k]);
            h->tgraph[k] = nullptr;
            for (auto& m : h->tmarks[k]) {
                cudaEventDestroy(m.a);
                cudaEventDestroy(m.b);
            }
            h->tmarks[k].clear();
        }
    }
    h->timing = phase_mask;
    return HYD_OK;
}

int hyd_set_timing(hyd_handle h, int enable) { return hyd_set_timing_phases(h, enable ? ~0u : 0u); }

int hyd_phase_name(int phase, const char** name) {
    if (!name || phase < 0 || phase >= PH_COUNT) return fail(HYD_EINVAL, "phase out of range");
    *name = kPhaseNames[phase];
    return HYD_OK;
}

int hyd_timing_report(hyd_handle h, char* buf, size_t buflen) {
    if (!h || !buf || buflen == 0) return fail(HYD_EINVAL, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (auto& m : h->marks) {
        float ms = 0;
        cudaEventElapsedTime(&ms, m.a, m.b);
        h->phase_ms[m.phase] += ms;
        h->phase_n[m.phase] += 1;
        h->event_pool.push_back(m.a);
        h->event_pool.push_back(m.b);
    }
    h->marks.clear();
    std::string out;
    char line[128];
    for (int k = 0; k < PH_COUNT; k++) {
        if (h->phase_n[k] == 0) continue;
        snprintf(line, sizeof line, "%s %lld %.6f\n", kPhaseNames[k], h->phase_n[k], h->phase_ms[k]);
        out += line;
        h->phase_ms[k] = 0;
        h->phase_n[k] = 0;
    }
    snprintf(buf, buflen, "%s", out.c_str());
    return HYD_OK;
}

int hyd_launch_count(hyd_handle h, long long* count) {
    (void)h;
    if (!count) return fail(HYD_EINVAL, "null argument");
    *count = g_launches.load();
    return HYD_OK;
}

// ---- batches of independent reaches (one persistent handle per member)

// Phases of a batched step with their own per-member CTA counts.
enum BatchPhase { BP_CB, BP_SM_BUD, BP_SM, BP_SM_FSB, BP_EV, BP_CEU, BP_EU, BP_RR, BP_RC, BP_PF, BP_FSJC, BP_UFS,
                  BP_COUNT };
// Line lists of the batched sweeps.
enum BatchLineSet { BL_UZ, BL_VZ, BL_FSJ, BL_FSI, BL_COUNT };

// The batched form of a batch step: every phase of the step one launch for all members
// (each CTA working for one member), the whole step one CUDA graph per step variant.
struct BatchFused {
    int nm = 0, mixed = 0, solver = 0;
    void* dev = nullptr;    // the device tables below, one allocation
    DevGrid* gS[3] = {};    // the members' grids as the step sees them: t_u / t_v as at the
                            // step start (S0), after the first smoothing of u (S1), and of v (S2)
    DevParams* p = nullptr;
    double** outs[4] = {};  // smoothing outputs: half-step 1 u, v; half-step 2 v, u
    int* bst[BP_COUNT] = {};
    int ctas[BP_COUNT] = {};
    int* lst[BL_COUNT] = {};
    int* lfirst[BL_COUNT] = {};
    SweepPlan plan{};
    int grid = 0;
    double* gscr = nullptr;     // sweep rows of lines too long for shared memory (if any)
    double* gscr_fs = nullptr;  // the same for the sediment sweep beside the main chain
    int thr_r = 64, thr_c = 64;
    size_t sm_ev = 0, sm_eu = 0, sm_rr = 0, sm_rc = 0, sm_pf = 0;
    cudaStream_t st = nullptr, side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, done = nullptr;
    std::vector<cudaEvent_t> mev;  // per member: its stream's work before a batched run
    std::vector<unsigned long long> epochs;  // the members' whole-grid event counts the tables were built at
    cudaGraphExec_t graph[8] = {};
    long long graph_kernels[8] = {};
    long long steps = 0;
    int built = 0;
};

struct HydBatch {
    std::vector<hyd_handle> members;
    int fused = 0;
    BatchFused bf;
};

int hyd_set_sweep_shape(hyd_handle h, int ctas, int wide) {
    if (!h) return fail(HYD_EINVAL, "null handle");
    if (ctas < 0 || (wide != 0 && wide != 1)) return fail(HYD_EINVAL, "ctas must be >= 0 and wide 0 or 1");
    const int g = ctas == 0 || ctas > h->plan_grid ? h->plan_grid : ctas;
    if (g != h->plan.long_grid || wide != h->plan.wide) {
        h->plan.long_grid = g;
        h->plan.wide = wide;
        drop_graphs(h);
    }
    return HYD_OK;
}

int hyd_get_sweep_shape(hyd_handle h, int* ctas, int* wide) {
    if (!h || !ctas || !wide) return fail(HYD_EINVAL, "null argument");
    *ctas = h->plan.long_grid;
    *wide = h->plan.wide;
    return HYD_OK;
}

int hyd_batch_create(int count, const HydCaseParams* params, const int* dims, int device, hyd_batch* out) {
    if (!params || !dims || !out || count < 1) return fail(HYD_EINVAL, "batch: null argument or empty batch");
    HydBatch* b = new HydBatch();
    for (int k = 0; k < count; k++) {
        hyd_handle h = nullptr;
        const int rc = hyd_create(&params[k], dims[2 * k], dims[2 * k + 1], device, &h);
        if (rc) {
            const std::string msg = "batch member " + std::to_string(k) + ": " + hyd_last_error();
            for (hyd_handle m : b->members) hyd_destroy(m);
            delete b;
            return fail(rc, msg);
        }
        // the members run side by side: sweeps sized by their lines, not the device
        sweep_plan_throughput(h->N, h->M, &h->plan);
        b->members.push_back(h);
    }
    *out = b;
    return HYD_OK;
}

int hyd_batch_size(hyd_batch b, int* count) {
    if (!b || !count) return fail(HYD_EINVAL, "null argument");
    *count = (int)b->members.size();
    return HYD_OK;
}

int hyd_batch_member(hyd_batch b, int k, hyd_handle* h) {
    if (!b || !h) return fail(HYD_EINVAL, "null argument");
    if (k < 0 || k >= (int)b->members.size()) return fail(HYD_EINVAL, "batch member index out of range");
    *h = b->members[k];
    return HYD_OK;
}

}  // extern "C"

namespace {

void fused_release(BatchFused& f) {
    for (int k = 0; k < 8; k++) {
        if (f.graph[k]) cudaGraphExecDestroy(f.graph[k]);
        f.graph[k] = nullptr;
    }
    if (f.st) cudaStreamSynchronize(f.st);
    if (f.side) cudaStreamSynchronize(f.side);
    cudaFree(f.dev);
    cudaFree(f.gscr);
    cudaFree(f.gscr_fs);
    f.dev = nullptr;
    f.gscr = f.gscr_fs = nullptr;
    for (cudaEvent_t e : f.mev) cudaEventDestroy(e);
    f.mev.clear();
    if (f.fork) cudaEventDestroy(f.fork);
    if (f.join) cudaEventDestroy(f.join);
    if (f.done) cudaEventDestroy(f.done);
    f.fork = f.join = f.done = nullptr;
    if (f.side) cudaStreamDestroy(f.side);
    if (f.st) cudaStreamDestroy(f.st);
    f.st = f.side = nullptr;
    f.built = 0;
}

// Whether the batch can take its next step as batched launches: every member initialised,
// at the same time with the same step and schedule, in the same precision, none in
// channel mode, owed whole-grid passes or a rescan of every line (those steps run per
// member first), none timed, and no grid large enough for the tiled column-major stores.
bool fused_eligible(HydBatch* b, int sed) {
    const HydSim* a = b->members[0];
    for (HydSim* s : b->members) {
        if (!s->initialized || s->dp.channel || s->force_rescan || s->timing || s->g.tile_cols) return false;
        if (s->full_pending & 1) return false;
        if (sed && (s->full_pending & 2)) return false;
        if (s->device != a->device || s->t != a->t || s->P.dT != a->P.dT ||
            s->P.sediment_start != a->P.sediment_start || s->P.bed_change_start != a->P.bed_change_start ||
            s->P.bed_period != a->P.bed_period || s->dp.mixed != a->dp.mixed || s->solver != a->solver)
            return false;
    }
    return true;
}

// The device tables of the batched form (from the members' current pointers: a step
// leaves them as it found them).
int fused_build(HydBatch* b) {
    BatchFused& f = b->bf;
    const int nm = (int)b->members.size();
    f.nm = nm;
    const HydSim* a0 = b->members[0];
    f.mixed = a0->dp.mixed;
    f.solver = a0->solver;
    std::vector<DevGrid> gs[3];
    std::vector<DevParams> ps;
    std::vector<double*> outs[4];
    std::vector<int> counts[BP_COUNT];
    std::vector<int> lines[BL_COUNT], firsts[BL_COUNT];
    int Nmax = 0, Mmax = 0;
    for (HydSim* s : b->members) {
        const DevGrid g0 = s->g;
        double *A = g0.t_u, *Bu = s->scratch_u, *C = g0.t_v, *D = s->scratch_v;
        DevGrid g1 = g0, g2 = g0;
        g1.t_u = Bu;
        g2.t_u = Bu;
        g2.t_v = D;
        gs[0].push_back(g0);
        gs[1].push_back(g1);
        gs[2].push_back(g2);
        ps.push_back(s->dp);
        outs[0].push_back(Bu);
        outs[1].push_back(D);
        outs[2].push_back(C);
        outs[3].push_back(A);
        const int N = s->N, M = s->M;
        const int rw = row_warp_ctas(g0, N + 3);
        counts[BP_CB].push_back(((N - 1) * 32 + 255) / 256 + 1);
        counts[BP_SM_BUD].push_back(rw + kBudCtas);
        counts[BP_SM].push_back(rw);
        counts[BP_SM_FSB].push_back(rw + 1);
        counts[BP_EV].push_back(N - 1);
        counts[BP_CEU].push_back(((N - 2) * 32 + 255) / 256);
        counts[BP_EU].push_back(M - 1);
        counts[BP_RR].push_back(N);
        counts[BP_RC].push_back(M);
        counts[BP_PF].push_back(row_warp_ctas(g0, N + 1) + 32 + 8);
        counts[BP_FSJC].push_back(((N - 1) * 32 + 255) / 256);
        counts[BP_UFS].push_back(row_warp_ctas(g0, N) + 2);
        lines[BL_UZ].push_back(M - 1);
        firsts[BL_UZ].push_back(2);
        lines[BL_VZ].push_back(N - 1);
        firsts[BL_VZ].push_back(2);
        lines[BL_FSJ].push_back(M - 3);
        firsts[BL_FSJ].push_back(3);
        lines[BL_FSI].push_back(N - 3);
        firsts[BL_FSI].push_back(3);
        Nmax = std::max(Nmax, N);
        Mmax = std::max(Mmax, M);
        f.thr_r = std::max(f.thr_r, s->thr_r);
        f.thr_c = std::max(f.thr_c, s->thr_c);
        size_t ev, eu, rr, rc, pf;
        line_smem(N, M, &ev, &eu, &rr, &rc, &pf);
        f.sm_ev = std::max(f.sm_ev, ev);
        f.sm_eu = std::max(f.sm_eu, eu);
        f.sm_rr = std::max(f.sm_rr, rr);
        f.sm_rc = std::max(f.sm_rc, rc);
        f.sm_pf = std::max(f.sm_pf, pf);
    }
    // one device block: grids, parameters, output pointers, CTA starts, line lists
    auto a8 = [](size_t x) { return (x + 255) / 256 * 256; };
    size_t off = 0;
    size_t o_g[3], o_p, o_out[4], o_b[BP_COUNT], o_ls[BL_COUNT], o_lf[BL_COUNT];
    for (int k = 0; k < 3; k++) { o_g[k] = off; off += a8(sizeof(DevGrid) * nm); }
    o_p = off;
    off += a8(sizeof(DevParams) * nm);
    for (int k = 0; k < 4; k++) { o_out[k] = off; off += a8(sizeof(double*) * nm); }
    for (int k = 0; k < BP_COUNT; k++) { o_b[k] = off; off += a8(sizeof(int) * (nm + 1)); }
    for (int k = 0; k < BL_COUNT; k++) {
        o_ls[k] = off;
        off += a8(sizeof(int) * (nm + 1));
        o_lf[k] = off;
        off += a8(sizeof(int) * nm);
    }
    std::vector<char> host(off, 0);
    for (int k = 0; k < 3; k++) memcpy(host.data() + o_g[k], gs[k].data(), sizeof(DevGrid) * nm);
    memcpy(host.data() + o_p, ps.data(), sizeof(DevParams) * nm);
    for (int k = 0; k < 4; k++) memcpy(host.data() + o_out[k], outs[k].data(), sizeof(double*) * nm);
    for (int k = 0; k < BP_COUNT; k++) {
        int* q = (int*)(host.data() + o_b[k]);
        q[0] = 0;
        for (int m = 0; m < nm; m++) q[m + 1] = q[m] + counts[k][m];
        f.ctas[k] = q[nm];
    }
    for (int k = 0; k < BL_COUNT; k++) {
        int* q = (int*)(host.data() + o_ls[k]);
        q[0] = 0;
        for (int m = 0; m < nm; m++) q[m + 1] = q[m] + std::max(lines[k][m], 0);
        memcpy(host.data() + o_lf[k], firsts[k].data(), sizeof(int) * nm);
    }
    CUDA_TRY(cudaSetDevice(a0->device));
    CUDA_TRY(cudaMalloc(&f.dev, off));
    CUDA_TRY(cudaMemcpy(f.dev, host.data(), off, cudaMemcpyHostToDevice));
    char* d = (char*)f.dev;
    for (int k = 0; k < 3; k++) f.gS[k] = (DevGrid*)(d + o_g[k]);
    f.p = (DevParams*)(d + o_p);
    for (int k = 0; k < 4; k++) f.outs[k] = (double**)(d + o_out[k]);
    for (int k = 0; k < BP_COUNT; k++) f.bst[k] = (int*)(d + o_b[k]);
    for (int k = 0; k < BL_COUNT; k++) {
        f.lst[k] = (int*)(d + o_ls[k]);
        f.lfirst[k] = (int*)(d + o_lf[k]);
    }
    // the sweeps' plan for the largest member, one persistent CTA per SM
    CUDA_TRY(sweep_plan(Nmax, Mmax, &f.plan, 0));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, a0->device);
    f.grid = nsm;
    if (f.plan.need_global) {
        const size_t rows = 4 * (size_t)std::max(f.plan.RG, f.plan.RGf) + 6 * HYD_SEGL;
        CUDA_TRY(cudaMalloc(&f.gscr, rows * f.grid * sizeof(double)));
        CUDA_TRY(cudaMalloc(&f.gscr_fs, rows * f.grid * sizeof(double)));
    }
    CUDA_TRY(batch_sweep_setup());
    CUDA_TRY(batch_grid_setup(f.sm_ev, f.sm_eu, f.sm_rr, f.sm_rc, f.sm_pf));
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    CUDA_TRY(cudaStreamCreateWithPriority(&f.st, cudaStreamNonBlocking, prio_hi));
    CUDA_TRY(cudaStreamCreateWithPriority(&f.side, cudaStreamNonBlocking, prio_lo));
    CUDA_TRY(cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming));
    f.mev.resize(nm);
    for (int m = 0; m < nm; m++) CUDA_TRY(cudaEventCreateWithFlags(&f.mev[m], cudaEventDisableTiming));
    f.epochs.clear();
    for (HydSim* s : b->members) f.epochs.push_back(s->epoch);
    f.built = 1;
    return HYD_OK;
}

// The launch sequence of one batched step (launch_step's span-limited sequence, every
// phase one launch for all members).
void fused_launch_step(HydBatch* b, int sed1, int sed2, int bed) {
    BatchFused& f = b->bf;
    const int nm = f.nm, mx = f.mixed;
    auto BR = [&](int state, int ph) { return BatchRef{f.gS[state], f.p, f.bst[ph], nm}; };
    auto BL = [&](int state, int set) { return BatchLines{f.gS[state], f.p, f.lst[set], f.lfirst[set], nm}; };
    cudaStream_t st = f.st;
    // ---- half-step 1
    launch_coef_bnd_batch(BR(0, BP_CB), f.ctas[BP_CB], 0, 3, mx, st);
    launch_sweep_batch(0, BL(0, BL_UZ), f.plan, f.solver, mx, f.gscr, f.grid, st);
    launch_smooth_batch(BR(0, BP_SM_BUD), f.ctas[BP_SM_BUD], 1, f.outs[0], 0, 0, 1, st);
    launch_explicit_v_batch(BR(1, BP_EV), f.ctas[BP_EV], f.thr_r, f.sm_ev, mx, st);
    launch_smooth_batch(BR(1, BP_SM), f.ctas[BP_SM], 0, f.outs[1], 0, 0, 0, st);
    launch_reset_batch(BR(2, BP_RR), f.ctas[BP_RR], 1, f.thr_r, f.sm_rr, st);
    launch_post_fused_batch(BR(2, BP_PF), f.ctas[BP_PF], 0, sed1, mx, f.sm_pf, st);
    if (sed1) {  // the first half-step's sediment beside the second half-step (as launch_step)
        cudaEventRecord(f.fork, st);
        cudaStreamWaitEvent(f.side, f.fork, 0);
        launch_coef_fsj_batch(BR(2, BP_FSJC), f.ctas[BP_FSJC], 0, mx, f.side);
        launch_fs_sweep_batch(0, BL(2, BL_FSJ), f.plan, 0, f.solver, mx, f.gscr_fs, f.grid, f.side);
        launch_update_fs_batch(BR(2, BP_UFS), f.ctas[BP_UFS], f.side);
        cudaEventRecord(f.join, f.side);
    }
    // ---- half-step 2
    launch_coef_bnd_batch(BR(2, BP_CB), f.ctas[BP_CB], 1, sed1 ? 1 : 3, mx, st);
    launch_sweep_batch(1, BL(2, BL_VZ), f.plan, f.solver, mx, f.gscr, f.grid, st);
    launch_smooth_batch(BR(2, BP_SM_BUD), f.ctas[BP_SM_BUD], 0, f.outs[2], 0, 0, 1, st);
    launch_coef_eu_batch(BR(1, BP_CEU), f.ctas[BP_CEU], mx, st);
    launch_explicit_u_batch(BR(1, BP_EU), f.ctas[BP_EU], f.thr_c, f.sm_eu, mx, st);
    if (sed1) cudaStreamWaitEvent(st, f.join, 0);
    launch_smooth_batch(BR(1, sed1 ? BP_SM_FSB : BP_SM), f.ctas[sed1 ? BP_SM_FSB : BP_SM], 1, f.outs[3], 1, sed1, 0,
                        st);
    launch_reset_batch(BR(0, BP_RC), f.ctas[BP_RC], 0, f.thr_c, f.sm_rc, st);
    launch_post_fused_batch(BR(0, BP_PF), f.ctas[BP_PF], 1, sed2, mx, f.sm_pf, st);
    if (sed2) {
        launch_fs_sweep_batch(1, BL(0, BL_FSI), f.plan, 1, f.solver, mx, f.gscr, f.grid, st);
        launch_update_fs_batch(BR(0, BP_UFS), f.ctas[BP_UFS], st);
    }
    if (bed) {  // once per bed period: the members' own launches, inside the step's graph
        for (HydSim* s : b->members) {
            const int start = sed2 ? 3 : 2, end = sed2 ? s->N - 1 : s->N;
            launch_bed(s->g, s->dp, start, end, st);
        }
    }
}

cudaGraphExec_t fused_graph(HydBatch* b, int mask) {
    BatchFused& f = b->bf;
    if (f.graph[mask]) return f.graph[mask];
    const long long before = hyd_kernel_launches_add(0);
    if (cudaStreamBeginCapture(f.st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return nullptr;
    fused_launch_step(b, mask & 1, (mask >> 1) & 1, (mask >> 2) & 1);
    cudaGraph_t graph = nullptr;
    if (cudaStreamEndCapture(f.st, &graph) != cudaSuccess || !graph) return nullptr;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return nullptr;
    const long long after = hyd_kernel_launches_add(0);
    f.graph_kernels[mask] = after - before;
    hyd_kernel_launches_add(-(after - before));
    f.graph[mask] = exec;
    return exec;
}

// One batched step of every member; HYD_ESTATE (nothing done) when the batch is not
// eligible for it now.
int fused_step(HydBatch* b) {
    HydSim* a = b->members[0];
    const double t1 = a->t + a->P.dT * 0.5;
    const double t2 = t1 + a->P.dT * 0.5;
    const int sed1 = t1 >= a->P.sediment_start;
    const int sed2 = t2 >= a->P.sediment_start;
    if (!fused_eligible(b, sed1 || sed2)) return HYD_ESTATE;
    for (HydSim* s : b->members)
        if ((int)(t2 / 3600) + 1 >= s->g.total_time) return fail(HYD_EINVAL, "boundary tables too short");
    const double it = (double)(long long)t2;
    const int bed = a->P.bed_period > 0 ? (t2 - it == 0 && t2 >= a->P.bed_change_start &&
                                           std::fmod(it, a->P.bed_period) == 0)
                                        : (std::fmod(it, a->P.bed_change_start) == 0 && t2 - it == 0);
    BatchFused& f = b->bf;
    if (!f.built) {
        const int rc = fused_build(b);
        if (rc) return rc;
    }
    const int mask = sed1 | (sed2 << 1) | (bed << 2);
    cudaGraphExec_t exec = fused_graph(b, mask);
    if (!exec) return fail(HYD_ECUDA, "batched step: graph capture failed");
    CUDA_TRY(cudaGraphLaunch(exec, f.st));
    hyd_kernel_launches_add(f.graph_kernels[mask]);
    for (HydSim* s : b->members) {
        s->t = t2;
        s->start_idx = sed2 ? 3 : 2;
        s->end_idx = sed2 ? s->N - 1 : s->N;
    }
    f.steps++;
    return HYD_OK;
}

}  // namespace

extern "C" {

int hyd_batch_set_fused(hyd_batch b, int on) {
    if (!b) return fail(HYD_EINVAL, "null batch");
    b->fused = on ? 1 : 0;
    return HYD_OK;
}

int hyd_batch_fused_steps(hyd_batch b, long long* steps) {
    if (!b || !steps) return fail(HYD_EINVAL, "null argument");
    *steps = b->bf.steps;
    return HYD_OK;
}

int hyd_batch_step(hyd_batch b, int nsteps, int sync) {
    if (!b) return fail(HYD_EINVAL, "null batch");
    if (nsteps < 0) return fail(HYD_EINVAL, "nsteps < 0");
    if (b->fused && nsteps > 0) {
        // batched steps while the members allow them (a member owing whole-grid passes or
        // a full rescan takes that step on its own first); the members' streams and the
        // batch stream are ordered both ways around the batched run
        BatchFused& f = b->bf;
        int n = 0;
        int ordered = 0;
        while (n < nsteps) {
            HydSim* a = b->members[0];
            const double t1 = a->t + a->P.dT * 0.5, t2 = t1 + a->P.dT * 0.5;
            if (!fused_eligible(b, t1 >= a->P.sediment_start || t2 >= a->P.sediment_start)) {
                if (ordered) {  // the batched steps before this one come first
                    CUDA_TRY(cudaEventRecord(f.done, f.st));
                    for (HydSim* s : b->members) CUDA_TRY(cudaStreamWaitEvent(s->stream, f.done, 0));
                    ordered = 0;
                }
                for (size_t k = 0; k < b->members.size(); k++) {
                    const int rc = hyd_step(b->members[k], 1, 0, nullptr);
                    if (rc) return fail(rc, "batch member " + std::to_string(k) + ": " + hyd_last_error());
                }
                n++;
                continue;
            }
            if (!ordered) {
                // tables built before a member's parameters, fields or spans changed are stale
                bool stale = !f.built;
                for (size_t k = 0; f.built && k < b->members.size(); k++)
                    if (b->members[k]->epoch != f.epochs[k]) stale = true;
                if (stale) {
                    if (f.built) fused_release(f);
                    const int rc = fused_build(b);
                    if (rc) return rc;
                }
                for (size_t k = 0; k < b->members.size(); k++) {
                    CUDA_TRY(cudaEventRecord(f.mev[k], b->members[k]->stream));
                    CUDA_TRY(cudaStreamWaitEvent(f.st, f.mev[k], 0));
                }
                ordered = 1;
            }
            const int rc = fused_step(b);
            if (rc) return rc;
            n++;
        }
        if (ordered) {
            CUDA_TRY(cudaEventRecord(f.done, f.st));
            for (HydSim* s : b->members) CUDA_TRY(cudaStreamWaitEvent(s->stream, f.done, 0));
        }
        CUDA_TRY(cudaGetLastError());
        if (sync) {
            for (size_t k = 0; k < b->members.size(); k++) {
                const int rc = hyd_synchronize(b->members[k]);
                if (rc) return fail(rc, "batch member " + std::to_string(k) + ": " + hyd_last_error());
            }
        }
        return HYD_OK;
    }
    // one step of every member at a time: each member's graphs go to its own stream, so
    // the device runs the members side by side while the host queues the next round
    for (int n = 0; n < nsteps; n++) {
        for (size_t k = 0; k < b->members.size(); k++) {
            const int rc = hyd_step(b->members[k], 1, 0, nullptr);
            if (rc) return fail(rc, "batch member " + std::to_string(k) + ": " + hyd_last_error());
        }
    }
    if (sync) {
        for (size_t k = 0; k < b->members.size(); k++) {
            const int rc = hyd_synchronize(b->members[k]);
            if (rc) return fail(rc, "batch member " + std::to_string(k) + ": " + hyd_last_error());
        }
    }
    return HYD_OK;
}

int hyd_batch_destroy(hyd_batch b) {
    if (!b) return HYD_OK;
    if (!b->members.empty()) {
        cudaSetDevice(b->members[0]->device);
        fused_release(b->bf);
    }
    int rc = HYD_OK;
    for (hyd_handle h : b->members) {
        const int r = hyd_destroy(h);
        if (r && !rc) rc = r;
    }
    delete b;
    return rc;
}

}  // extern "C"
