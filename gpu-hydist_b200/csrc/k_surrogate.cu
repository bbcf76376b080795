// k_surrogate.cu — BF16 convolution kernels of the learned surrogate on the 5th-generation
// tensor cores (tcgen05.mma, FP32 accumulators in tensor memory).  No reference
// counterpart: the reference has no learned part.
//
// The network is a stack of 3x3 convolutions over NHWC BF16 activations.  Every layer is an
// implicit GEMM  D[p][n] = sum_k A[p][k] B[n][k]  with p an output pixel (128 per CTA tile,
// the MMA's M), n an output channel (the MMA's N, 16..256 in steps of 16) and k = (tap,
// input channel) (K = 9 x CIN, consumed 16 at a time).  A is gathered from the input
// activation by a pixel mapping (same-size, its adjoint, stride-2 down, stride-2 up), so the
// forward pass, the data gradient (the adjoint mapping with the channel-transposed weights)
// and the weight gradient (pixels as the reduction) are the same kernels.
//
// Shared-memory operand layout: the canonical K-major layout without swizzle.  A core
// matrix is 8 rows x 16 bytes (8 BF16 along K), stored as 128 contiguous bytes; within one
// K step of 16 the two core matrices of an 8-row group lie 128 B apart (the descriptor's
// leading byte offset) and consecutive 8-row groups 256 B apart (its stride byte offset).
// Both strides keep every core matrix inside the K step's block, whichever of the two
// offsets the hardware applies to which direction, so a layout mistake shows as wrong
// numbers, never as an access outside the operand.
//
// One elected thread issues the MMAs; tcgen05.commit arrives on an mbarrier that the CTA
// waits on with a bounded spin (on timeout: an error flag, a second bounded wait, the
// tensor memory freed, return).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/hydist_b200.h"

long long hyd_kernel_launches_add(long long n);

namespace {

constexpr int kTile = 128;            // output pixels per CTA tile (MMA M)
constexpr int kThreads = 128;         // four warps: one thread per tile row
constexpr int kConvGroups = 3;        // the forward kernel's thread groups: a third of the taps
constexpr int kConvThreads = kTile * kConvGroups;  // and of the output column blocks each
constexpr unsigned kSpinLimit = 1u << 26;  // bounded waits (~seconds); then the error flag

// pixel mappings of a layer (the input pixel that output pixel p, tap t reads)
enum ConvMode { kSame = HYD_CONV_SAME, kSameAdj = HYD_CONV_SAME_ADJ, kDown = HYD_CONV_DOWN, kUp = HYD_CONV_UP };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// sm_100 shared-memory matrix descriptor: start, leading and stride byte offsets (>> 4),
// version 1 (bits 46-47), no swizzle (bits 61-63 = 0), base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12
// = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for phase `parity` of the mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (unsigned it = 0; it < kSpinLimit; it++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Tensor memory of `cols` columns (a power of two >= 32), allocated by warp 0.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 FP32 columns of this thread's tensor-memory lane (32x32b shape: warp w reads lanes
// 32w..32w+31, thread = lane).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// 16-byte asynchronous copy global -> shared, cached in L1 (the two halves of a 32-byte
// sector and the taps of neighbouring pixels read the same lines); src_bytes 0 fills the
// 16 bytes with zeros (nothing is read).  A thread's copies are waited for with
// cp_async_wait_all.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Byte offset of element (row, k) of a K step block (row-major 8-row groups of two core
// matrices, see the file comment).
__device__ __forceinline__ uint32_t op_off(int row, int k) {
    return (uint32_t)((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// The input pixel that output pixel (y, x) reads through tap t, or -1 (zero padding).
template <int MODE>
__device__ __forceinline__ long long map_pixel(int b, int y, int x, int t, int Hin, int Win) {
    const int dy = t / 3 - 1, dx = t % 3 - 1;
    int iy, ix;
    if (MODE == kSame) {
        iy = y + dy;
        ix = x + dx;
    } else if (MODE == kSameAdj) {
        iy = y - dy;
        ix = x - dx;
    } else if (MODE == kDown) {
        iy = 2 * y + dy;
        ix = 2 * x + dx;
    } else {  // kUp: the adjoint of kDown
        const int sy = y - dy, sx = x - dx;
        if ((sy & 1) || (sx & 1)) return -1;
        iy = sy >> 1;
        ix = sx >> 1;
    }
    if (iy < 0 || ix < 0 || iy >= Hin || ix >= Win) return -1;
    return ((long long)b * Hin + iy) * Win + ix;
}

struct ConvArgs {
    const __nv_bfloat16* x;  // input activation, NHWC with cin channels
    int B, Hin, Win;
    const uint4* w;          // packed weights: the shared-memory image of B (ksteps x ncols x 16)
    const float* bias;       // ncols (or null)
    const __nv_bfloat16* mask;  // null, or an NHWC activation with nout channels: output *= (mask > 0)
    void* y;                 // output, NHWC with nout channels (BF16, or FP32 with out_f32)
    int Hout, Wout, nout;
    int relu, out_f32;
    int* err;
};

// Taps t0..t0+2 of row `row` of A for `tile` (output pixel tile * kTile + row): CIN
// channels of the input pixel of each tap, copied asynchronously into the K step blocks
// (zeros for padding and for pixels past the end), one commit group.
template <int MODE, int CIN>
__device__ __forceinline__ void gather_row(const ConvArgs& a, uint32_t sA, long long tile, long long npix, int row,
                                           int t0) {
    constexpr int CB = CIN / 16;
    constexpr int A_STEP = kTile * 32;
    const long long p = tile * kTile + row;
    int b = 0, y = 0, x = 0;
    const bool live = p < npix;
    if (live) {  // the host keeps the pixel count below 2^31
        const int pi = (int)p;
        const int r = pi / a.Wout;
        x = pi - r * a.Wout;
        b = r / a.Hout;
        y = r - b * a.Hout;
    }
#pragma unroll
    for (int dt = 0; dt < 9 / kConvGroups; dt++) {
        const int t = t0 + dt;
        const long long q = live ? map_pixel<MODE>(b, y, x, t, a.Hin, a.Win) : -1;
        const __nv_bfloat16* src = a.x + (q < 0 ? 0 : q) * CIN;
        const uint32_t n = q < 0 ? 0u : 16u;
#pragma unroll
        for (int cb = 0; cb < CB; cb++) {
            const uint32_t blk = sA + (uint32_t)((t * CB + cb) * A_STEP);
            cp_async16(blk + op_off(row, 0), src + 16 * cb, n);
            cp_async16(blk + op_off(row, 8), src + 16 * cb + 8, n);
        }
    }
    cp_async_commit();
}

// zero the BF16 halves of v whose mask value is not > 0
__device__ __forceinline__ uint32_t mask_bf16x2(uint32_t v, uint32_t m) {
    const bool lo = __uint_as_float(m << 16) > 0.0f, hi = __uint_as_float(m & 0xFFFF0000u) > 0.0f;
    return (lo ? (v & 0xFFFFu) : 0u) | (hi ? (v & 0xFFFF0000u) : 0u);
}

// Forward / data-gradient convolution: CTA tiles of 128 output pixels, all output columns
// (NCOL, a multiple of 16) at once.  CIN (16 or 48) input channels per pixel; the weights
// for the whole K stay in shared memory, the tile's whole A (K x 128) is copied in
// asynchronously (every copy of a thread in flight at once), then K/16 MMAs accumulate in
// tensor memory.  Once they have completed, the next tile's copies are issued and run
// under this tile's epilogue, which stages the output tile (bias, ReLU) in shared memory
// and writes it with coalesced 16-byte stores (the mask applied there).  Three groups of
// 128 threads: thread (group g, row r) copies taps 3g..3g+2 of tile row r and, in the
// epilogue, reads column blocks g, g + 3, ... of its row (warp w reads tensor-memory
// lanes 32 (w % 4)..+31, the lanes its sub-partition may access).
template <int MODE, int CIN, int NCOL>
__global__ void __launch_bounds__(kConvThreads, 1) k_conv_tc(ConvArgs a) {
    constexpr int KSTEPS = 9 * CIN / 16;
    constexpr int A_STEP = kTile * 32;           // bytes of A per K step
    constexpr int B_STEP = NCOL * 32;            // bytes of B per K step
    constexpr uint32_t TCOLS = NCOL <= 32 ? 32 : (NCOL <= 64 ? 64 : (NCOL <= 128 ? 128 : 256));
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;
    unsigned char* sB = smem + KSTEPS * A_STEP;
    unsigned char* sO = sB + KSTEPS * B_STEP;    // the output tile, kTile x nout, as in y
    float* sBias = reinterpret_cast<float*>(sO + kTile * NCOL * 4);
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = tid & (kTile - 1), grp = tid / kTile;
    const long long npix = (long long)a.B * a.Hout * a.Wout;
    const long long ntiles = (npix + kTile - 1) / kTile;
    const uint32_t a0 = smem_u32(sA);
    if ((long long)blockIdx.x < ntiles) gather_row<MODE, CIN>(a, a0, blockIdx.x, npix, row, 3 * grp);
    // weights: a straight copy of the packed image; the bias (zero beyond nout)
    {
        const uint4* src = a.w;
        uint4* dst = reinterpret_cast<uint4*>(sB);
        for (int q = tid; q < KSTEPS * B_STEP / 16; q += kConvThreads) dst[q] = src[q];
        for (int c = tid; c < NCOL; c += kConvThreads) sBias[c] = (a.bias && c < a.nout) ? a.bias[c] : 0.0f;
    }
    if (tid == 0) {
        mbar_init(&mbar);
        s_fail = 0;
    }
    if (warp == 0) tmem_alloc(&s_tmem, TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const int nout = a.nout, esz = a.out_f32 ? 4 : 2;
    uint32_t phase = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        cp_async_wait_all();
        fence_async_smem();
        __syncthreads();
        // ---- the MMAs, issued by one thread; their completion arrives on the mbarrier
        if (tid == 0) {
            tc_fence_after();
            const uint32_t b0 = smem_u32(sB);
            constexpr uint32_t idesc = instr_desc(kTile, NCOL);
            for (int s = 0; s < KSTEPS; s++)
                mma_bf16(tmem, smem_desc(a0 + s * A_STEP, 128, 256), smem_desc(b0 + s * B_STEP, 128, 256), idesc,
                         s > 0 ? 1u : 0u);
            mma_commit(&mbar);
        }
        const bool ok = mbar_wait(&mbar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {  // the whole CTA leaves together
            if (tid == 0) s_fail = 1;
            break;
        }
        tc_fence_after();
        // A has been read: the next tile's copies run under this epilogue
        if (tile + gridDim.x < ntiles) gather_row<MODE, CIN>(a, a0, tile + gridDim.x, npix, row, 3 * grp);
        const long long rem = npix - tile * kTile;
        const int live_n = rem < kTile ? (int)rem : kTile;
        // ---- this thread's row from tensor memory, bias and activation, into the staged
        // tile (every thread of a warp takes part in tcgen05.ld, which is .sync.aligned)
#pragma unroll
        for (int c0 = 16 * grp; c0 < NCOL; c0 += 16 * kConvGroups) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0, v);
            if (row < live_n) {
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    v[k] += sBias[c0 + k];
                    if (a.relu) v[k] = fmaxf(v[k], 0.0f);
                }
                if (!a.out_f32 && nout % 8 == 0 && c0 + 16 <= nout) {  // two 16-byte stores
                    uint32_t w[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
                        w[k] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    uint4* d = reinterpret_cast<uint4*>(sO + ((size_t)row * nout + c0) * 2);
                    d[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    d[1] = make_uint4(w[4], w[5], w[6], w[7]);
                } else if (a.out_f32 && nout % 4 == 0 && c0 + 16 <= nout) {  // four 16-byte stores
                    float4* d = reinterpret_cast<float4*>(sO + ((size_t)row * nout + c0) * 4);
#pragma unroll
                    for (int k = 0; k < 4; k++) d[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
                } else {
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const int c = c0 + k;
                        if (c >= nout) break;
                        if (a.out_f32) reinterpret_cast<float*>(sO)[row * nout + c] = v[k];
                        else reinterpret_cast<__nv_bfloat16*>(sO)[row * nout + c] = __float2bfloat16_rn(v[k]);
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();  // the staged tile is complete; the tensor memory has been read
        // ---- the staged tile to y (it is contiguous there), the mask applied
        const long long e0 = tile * kTile * nout;  // first element of the tile in y and the mask
        const int nel = live_n * nout, nbytes = nel * esz;
        unsigned char* yb = reinterpret_cast<unsigned char*>(a.y) + e0 * esz;
        const __nv_bfloat16* mb = a.mask ? a.mask + e0 : nullptr;
        const bool vec = (nbytes % 16 == 0) && !(reinterpret_cast<uintptr_t>(yb) & 15) &&
                         !(reinterpret_cast<uintptr_t>(mb) & (a.out_f32 ? 7 : 15));
        if (vec) {
            for (int q = tid; q < nbytes / 16; q += kConvThreads) {
                uint4 v = reinterpret_cast<const uint4*>(sO)[q];
                if (mb) {
                    if (a.out_f32) {
                        const uint2 m = reinterpret_cast<const uint2*>(mb)[q];
                        v.x = __uint_as_float(m.x << 16) > 0.0f ? v.x : 0u;
                        v.y = __uint_as_float(m.x & 0xFFFF0000u) > 0.0f ? v.y : 0u;
                        v.z = __uint_as_float(m.y << 16) > 0.0f ? v.z : 0u;
                        v.w = __uint_as_float(m.y & 0xFFFF0000u) > 0.0f ? v.w : 0u;
                    } else {
                        const uint4 m = reinterpret_cast<const uint4*>(mb)[q];
                        v.x = mask_bf16x2(v.x, m.x);
                        v.y = mask_bf16x2(v.y, m.y);
                        v.z = mask_bf16x2(v.z, m.z);
                        v.w = mask_bf16x2(v.w, m.w);
                    }
                }
                reinterpret_cast<uint4*>(yb)[q] = v;
            }
        } else {
            for (int e = tid; e < nel; e += kConvThreads) {
                const bool keep = !mb || __bfloat162float(mb[e]) > 0.0f;
                if (a.out_f32) reinterpret_cast<float*>(yb)[e] = keep ? reinterpret_cast<const float*>(sO)[e] : 0.0f;
                else
                    reinterpret_cast<__nv_bfloat16*>(yb)[e] =
                        keep ? reinterpret_cast<const __nv_bfloat16*>(sO)[e] : __float2bfloat16_rn(0.0f);
            }
        }
    }
    cp_async_wait_all();  // no copy in flight past this point
    __syncthreads();
    if (s_fail) {
        if (tid == 0) atomicExch(a.err, 1);
        // the MMAs may still be in flight: one more bounded wait before the memory is freed
        mbar_wait(&mbar, phase ^ 1u);
    }
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, TCOLS);
}

struct WgradArgs {
    const __nv_bfloat16* x;   // the layer's input activation, NHWC, cin channels
    int B, Hin, Win, cin;
    const __nv_bfloat16* dy;  // gradient at the layer's output, NHWC, ncol channels
    int Hout, Wout;
    int nout;                 // output channels to accumulate (<= NCOL)
    float* dw;                // [nout][9][cin] FP32, accumulated atomically
    long long chunk;          // output pixels per CTA (a multiple of 16)
    int* err;
};

// Weight gradient: dW[n][t][ci] = sum_p dY[p][n] X[map(p, t)][ci].  An MMA with M = 128 rows
// (t, ci) of the 9 x cin, N = NCOL output channels and K = output pixels; CTA (m-tile,
// pixel chunk), the chunk's K steps gathered 8 at a time, the partial sums added to dw.
// Each round's 128 pixels are mapped once (thread k: pixel k's input pixel for every tap,
// kept in shared memory), so the gathers do no index division.
template <int MODE, int NCOL>
__global__ void __launch_bounds__(kThreads, 1) k_conv_wgrad_tc(WgradArgs a) {
    constexpr int KB = 8;                 // K steps per gather round
    constexpr int A_STEP = kTile * 32, B_STEP = NCOL * 32;
    constexpr uint32_t TCOLS = NCOL <= 32 ? 32 : (NCOL <= 64 ? 64 : (NCOL <= 128 ? 128 : 256));
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;
    unsigned char* sB = smem + KB * A_STEP;
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    __shared__ long long s_q[9][16 * KB];  // the round's input pixel per tap (-1: none)
    const int tid = threadIdx.x, warp = tid >> 5;
    const int rows = 9 * a.cin;
    const int mt = blockIdx.y;
    const int r = mt * kTile + tid;  // this thread's A row (t, ci)
    const bool rlive = r < rows;
    const int t = rlive ? r / a.cin : 0, ci = rlive ? r % a.cin : 0;
    const long long npix = (long long)a.B * a.Hout * a.Wout;
    const long long p0 = (long long)blockIdx.x * a.chunk;
    long long p1 = p0 + a.chunk;
    if (p1 > npix) p1 = npix;
    if (tid == 0) {
        mbar_init(&mbar);
        s_fail = 0;
    }
    if (warp == 0) tmem_alloc(&s_tmem, TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    uint32_t phase = 0;
    int issued = 0;
    static_assert(16 * KB == kThreads, "one pixel of the round per thread");
    for (long long k0 = p0; k0 < p1; k0 += 16 * KB) {
        {
            const long long p = k0 + tid;
            int x = 0, y = 0, b = 0;
            if (p < p1) {
                x = (int)(p % a.Wout);
                const long long rr = p / a.Wout;
                y = (int)(rr % a.Hout);
                b = (int)(rr / a.Hout);
            }
#pragma unroll
            for (int tt = 0; tt < 9; tt++) s_q[tt][tid] = p < p1 ? map_pixel<MODE>(b, y, x, tt, a.Hin, a.Win) : -1;
        }
        __syncthreads();
        const long long* qrow = s_q[t];
        for (int s = 0; s < KB; s++) {
            // A row r over 16 pixels; B rows (channels) over the same pixels
            __align__(16) __nv_bfloat16 va[16];
            __align__(16) __nv_bfloat16 vb[16];
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const long long p = k0 + s * 16 + k;
                __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
                __nv_bfloat16 w = v;
                if (p < p1) {
                    if (rlive) {
                        const long long q = qrow[s * 16 + k];
                        if (q >= 0) v = a.x[q * a.cin + ci];
                    }
                    if (tid < NCOL) w = a.dy[p * NCOL + tid];
                }
                va[k] = v;
                vb[k] = w;
            }
            unsigned char* blkA = sA + s * A_STEP;
            *reinterpret_cast<uint4*>(blkA + op_off(tid, 0)) = *reinterpret_cast<const uint4*>(&va[0]);
            *reinterpret_cast<uint4*>(blkA + op_off(tid, 8)) = *reinterpret_cast<const uint4*>(&va[8]);
            if (tid < NCOL) {
                unsigned char* blkB = sB + s * B_STEP;
                *reinterpret_cast<uint4*>(blkB + op_off(tid, 0)) = *reinterpret_cast<const uint4*>(&vb[0]);
                *reinterpret_cast<uint4*>(blkB + op_off(tid, 8)) = *reinterpret_cast<const uint4*>(&vb[8]);
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            constexpr uint32_t idesc = instr_desc(kTile, NCOL);
            for (int s = 0; s < KB; s++)
                mma_bf16(tmem, smem_desc(a0 + s * A_STEP, 128, 256), smem_desc(b0 + s * B_STEP, 128, 256), idesc,
                         (issued + s) > 0 ? 1u : 0u);
            mma_commit(&mbar);
        }
        issued += KB;
        const bool ok = mbar_wait(&mbar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {  // the whole CTA leaves together
            if (tid == 0) s_fail = 1;
            break;
        }
        tc_fence_after();
        __syncthreads();  // the operands of the round are free
    }
    __syncthreads();
    if (!s_fail && issued > 0) {
#pragma unroll
        for (int c0 = 0; c0 < NCOL; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (rlive) {
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int n = c0 + k;
                    if (n < a.nout) atomicAdd(&a.dw[((size_t)n * 9 + t) * a.cin + ci], v[k]);
                }
            }
        }
    }
    if (s_fail) {
        if (tid == 0) atomicExch(a.err, 1);
        mbar_wait(&mbar, phase ^ 1u);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, TCOLS);
}

// Bias gradient: db[n] += sum over pixels of dY[p][n] (NHWC, ncol channels), FP32.
__global__ void k_bias_grad(const __nv_bfloat16* dy, long long npix, int ncol, int nout, float* db) {
    __shared__ float acc[256];
    for (int c = threadIdx.x; c < nout; c += blockDim.x) acc[c] = 0.0f;
    __syncthreads();
    for (long long p = blockIdx.x * (long long)blockDim.y + threadIdx.y; p < npix; p += (long long)gridDim.x * blockDim.y)
        for (int c = threadIdx.x; c < nout; c += blockDim.x) atomicAdd(&acc[c], __bfloat162float(dy[p * ncol + c]));
    __syncthreads();
    for (int c = threadIdx.x; c < nout; c += blockDim.x)
        if (threadIdx.y == 0) atomicAdd(&db[c], acc[c]);
}

// Masked mean-squared error of FP32 predictions (npix x nc) against targets, weighted per
// pixel: loss += sum w (pred - tgt)^2 * scale; dY (BF16, npix x ncol, zero beyond nc) =
// 2 w (pred - tgt) * scale.
__global__ void k_mse_grad(const float* pred, const float* tgt, const float* wgt, long long npix, int nc, int ncol,
                           float scale, __nv_bfloat16* dy, float* loss) {
    float l = 0.0f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        const float w = wgt ? wgt[p] : 1.0f;
        for (int c = 0; c < ncol; c++) {
            float g = 0.0f;
            if (c < nc) {
                const float d = pred[p * nc + c] - tgt[p * nc + c];
                l += w * d * d * scale;
                g = 2.0f * w * d * scale;
            }
            dy[p * ncol + c] = __float2bfloat16_rn(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

template <int MODE, int CIN, int NCOL>
cudaError_t launch_conv(const ConvArgs& a, cudaStream_t s) {
    constexpr int KSTEPS = 9 * CIN / 16;
    const size_t smem = (size_t)KSTEPS * (kTile * 32 + NCOL * 32) + (size_t)kTile * NCOL * 4 + NCOL * 4;
    cudaError_t e = cudaFuncSetAttribute(k_conv_tc<MODE, CIN, NCOL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long ntiles = ((long long)a.B * a.Hout * a.Wout + kTile - 1) / kTile;
    const int grid = (int)(ntiles < nsm ? ntiles : nsm);
    k_conv_tc<MODE, CIN, NCOL><<<grid, kConvThreads, smem, s>>>(a);
    hyd_kernel_launches_add(1);
    return cudaGetLastError();
}

template <int MODE>
cudaError_t dispatch_conv(const ConvArgs& a, int cin, int ncol, cudaStream_t s) {
    if (cin == 16 && ncol == 48) return launch_conv<MODE, 16, 48>(a, s);
    if (cin == 48 && ncol == 48) return launch_conv<MODE, 48, 48>(a, s);
    if (cin == 48 && ncol == 16) return launch_conv<MODE, 48, 16>(a, s);
    return cudaErrorInvalidValue;
}

template <int MODE, int NCOL>
cudaError_t launch_wgrad(const WgradArgs& a, cudaStream_t s) {
    const size_t smem = (size_t)8 * (kTile * 32 + NCOL * 32);
    cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad_tc<MODE, NCOL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const long long npix = (long long)a.B * a.Hout * a.Wout;
    const dim3 grid((unsigned)((npix + a.chunk - 1) / a.chunk), (unsigned)((9 * a.cin + kTile - 1) / kTile));
    k_conv_wgrad_tc<MODE, NCOL><<<grid, kThreads, smem, s>>>(a);
    hyd_kernel_launches_add(1);
    return cudaGetLastError();
}

template <int MODE>
cudaError_t dispatch_wgrad(const WgradArgs& a, int ncol, cudaStream_t s) {
    if (ncol == 48) return launch_wgrad<MODE, 48>(a, s);
    if (ncol == 16) return launch_wgrad<MODE, 16>(a, s);
    return cudaErrorInvalidValue;
}

}  // namespace

extern "C" {

int hyd_conv_forward(const void* x, int B, int Hin, int Win, int cin, const void* w_packed, const float* bias,
                     int ncol, int nout, int mode, int relu, const void* mask, void* y, int Hout, int Wout,
                     int out_f32, int* err, void* stream) {
    if (!x || !w_packed || !y || !err || B < 1 || Hin < 1 || Win < 1 || Hout < 1 || Wout < 1) return HYD_EINVAL;
    if (nout < 1 || nout > ncol) return HYD_EINVAL;
    if ((long long)B * Hout * Wout >= (1LL << 31)) return HYD_EINVAL;  // 32-bit pixel indices in the gather
    if ((reinterpret_cast<uintptr_t>(x) & 15) || (reinterpret_cast<uintptr_t>(w_packed) & 15)) return HYD_EINVAL;
    ConvArgs a{(const __nv_bfloat16*)x, B, Hin, Win, (const uint4*)w_packed, bias, (const __nv_bfloat16*)mask, y,
               Hout, Wout, nout, relu, out_f32, err};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    switch (mode) {
        case HYD_CONV_SAME: e = dispatch_conv<kSame>(a, cin, ncol, s); break;
        case HYD_CONV_SAME_ADJ: e = dispatch_conv<kSameAdj>(a, cin, ncol, s); break;
        case HYD_CONV_DOWN: e = dispatch_conv<kDown>(a, cin, ncol, s); break;
        case HYD_CONV_UP: e = dispatch_conv<kUp>(a, cin, ncol, s); break;
        default: return HYD_EINVAL;
    }
    return e == cudaSuccess ? HYD_OK : (e == cudaErrorInvalidValue ? HYD_EINVAL : HYD_ECUDA);
}

int hyd_conv_wgrad(const void* x, int B, int Hin, int Win, int cin, int mode, const void* dy, int Hout, int Wout,
                   int ncol, int nout, float* dw, int* err, void* stream) {
    if (!x || !dy || !dw || !err || B < 1 || (cin != 16 && cin != 48) || nout < 1 || nout > ncol) return HYD_EINVAL;
    WgradArgs a{(const __nv_bfloat16*)x, B, Hin, Win, cin, (const __nv_bfloat16*)dy, Hout, Wout, nout, dw, 2048, err};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    switch (mode) {
        case HYD_CONV_SAME: e = dispatch_wgrad<kSame>(a, ncol, s); break;
        case HYD_CONV_DOWN: e = dispatch_wgrad<kDown>(a, ncol, s); break;
        case HYD_CONV_UP: e = dispatch_wgrad<kUp>(a, ncol, s); break;
        default: return HYD_EINVAL;
    }
    return e == cudaSuccess ? HYD_OK : (e == cudaErrorInvalidValue ? HYD_EINVAL : HYD_ECUDA);
}

int hyd_bias_grad(const void* dy, long long npix, int ncol, int nout, float* db, void* stream) {
    if (!dy || !db || npix < 1 || nout < 1 || nout > ncol || nout > 256) return HYD_EINVAL;
    const dim3 block(64, 4);
    k_bias_grad<<<148, block, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)dy, npix, ncol, nout, db);
    hyd_kernel_launches_add(1);
    return cudaGetLastError() == cudaSuccess ? HYD_OK : HYD_ECUDA;
}

int hyd_mse_grad(const float* pred, const float* target, const float* weight, long long npix, int nc, int ncol,
                 float scale, void* dy, float* loss, void* stream) {
    if (!pred || !target || !dy || !loss || npix < 1 || nc < 1 || nc > ncol) return HYD_EINVAL;
    k_mse_grad<<<296, 256, 0, (cudaStream_t)stream>>>(pred, target, weight, npix, nc, ncol, scale,
                                                      (__nv_bfloat16*)dy, loss);
    hyd_kernel_launches_add(1);
    return cudaGetLastError() == cudaSuccess ? HYD_OK : HYD_ECUDA;
}

}  // extern "C"
