// vpt_unet.cu - the learned denoiser's network kernels: a U-Net of 3x3 convolutions that predicts
// per-pixel 5x5 kernels (a kernel-predicting denoiser), trained on the GPU by these kernels.
//
// The reference runs its learned denoiser through libtorch (src/Denoiser/PyTorchDenoiser.cpp:637-800,
// a TorchScript forward).  It has no training code and no network of its own; this file is new.
//
// Tensors are NHWC bf16 ("pixels x channels", P = N*H*W rows, channels contiguous, every channel
// count a multiple of 16); accumulation is fp32.  A 3x3 convolution (stride 1, zero padding 1) is an
// implicit GEMM with K = 9 * Cin, k = tap * Cin + ci, tap = (dy + 1) * 3 + (dx + 1):
//
//   forward       y[p][co]  = act(bias[co] + sum_k x[p + off(tap)][ci] * w[co][k])       M = pixels
//   input grad    dx[p][ci] = sum_k' dy[p + off(tap')][co] * wrot[ci][k'],  wrot[ci][t'][co]
//                 = w[co][8 - t'][ci] (the same kernel, rotated weights)                   M = pixels
//   weight grad   dw[co][k] = sum_p dy[p][co] * x[p + off(tap)][ci]                      M = k, K = pixels
//
// Tensor-core path (sm_100a tcgen05): one CTA computes a 128 x N tile (N <= 256 output channels) of
// D = A * B^T with the fp32 accumulator in tensor memory (TMEM).  All 128 threads gather the A / B
// tiles of the next K-stages with 16-byte cp.async copies (zero-filled outside the image) into a
// 4-stage shared-memory ring laid out in the UMMA no-swizzle canonical form (8-row x 16-byte core
// matrices); one thread issues tcgen05.mma (kind::f16, bf16 x bf16 -> fp32) per 16-wide K step and
// tcgen05.commit signals a per-stage mbarrier when the stage's MMAs have read their operands, which
// frees the slot for the next gather.  The epilogue reads the accumulator with tcgen05.ld (each warp
// its 32 TMEM lanes = 32 tile rows) and fuses bias, ReLU, the ReLU-derivative mask of the backward
// pass and the bf16 / fp32 store.  Forward and input-gradient tiles have K-major operands (k
// contiguous: channels of one pixel); the weight-gradient tile has MN-major operands (channels
// contiguous, pixels along K) and writes per-split fp32 partial sums that the optimiser reduces in a
// fixed order (deterministic).
//
// Every mbarrier wait is bounded: on expiry the kernel records VPT_ERR_ITER_LIMIT in *err, waits
// (bounded) for the MMAs it issued, frees its TMEM and returns.
#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "../../include/vpt_b200.h"
#include "vpt_kernels.h"

namespace vpt {
namespace unet {

typedef __nv_bfloat16 bf16;

constexpr int kBM = 128;      // tile rows (TMEM lanes)
constexpr int kBK = 64;       // K elements per pipeline stage (4 MMAs of K = 16)
constexpr int kThreads = 128;
constexpr uint32_t kWaitLimit = 1u << 22;  // bounded mbarrier waits (error flag on expiry)

// ---------------------------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;  // n = 0 writes 16 zero bytes and reads nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async16_stream(uint32_t dst, const void* src) {  // L2 only
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 4 : 0;  // n = 0 writes 4 zero bytes and reads nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// make this thread's generic-proxy shared-memory writes visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// waits until the phase with the given parity has completed; false after kWaitLimit polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// whole warp: allocate `cols` TMEM columns (power of two >= 32), address written to shared memory
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle: start address, leading-dimension byte offset (between
// core matrices adjacent along K), stride-dimension byte offset (between core matrices adjacent
// along M/N), all in 16-byte units; bits 46-47 = 1 (descriptor version of sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// Instruction descriptor of kind::f16: D fp32 (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1),
// A / B major (bit 15 / 16: 0 = K-major, 1 = MN-major), N >> 3 (bits 17-22), M >> 4 (bits 24-28).
__host__ __device__ constexpr uint32_t instr_desc(int m, int n, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns: lane i of the warp gets TMEM lane (base + i)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------------------------
// the implicit-GEMM convolution tile
// ---------------------------------------------------------------------------------------------
enum Mode : int { kConv = 0, kWgrad = 1 };

struct ConvArgs {
    const bf16* x;       // conv: input [P][cin]; wgrad: forward input [P][cin]
    const bf16* w;       // conv: weights [cout][9][cin]; wgrad: output gradient dy [P][cout]
    const float* bias;   // conv: [cout] or null
    const bf16* mask;    // conv: [P][cout]; output multiplied by (mask > 0) (ReLU derivative) or null
    void* y;             // conv: [P][cout] bf16 or fp32; wgrad: fp32 partials [splits][m_pad][cout]
    int* err;            // device error word (VPT_ERR_ITER_LIMIT on an expired wait) or null
    int n, h, w_;        // batch and image size (pixels P = n * h * w_)
    int cin, cout;       // channel counts (multiples of 16)
    int n_tile;          // output columns per CTA (multiple of 16, <= 256)
    int tmem_cols;       // power of two >= n_tile, >= 32
    int relu, out_f32;   // conv epilogue
    int pix_per_split;   // wgrad: pixels (K) per CTA, multiple of kBK
    int m_pad;           // wgrad: rows of a partial (multiple of kBM)
    int ksplit;          // conv: K stages split over blockIdx.z (> 1: raw sums to `partial`)
    float* partial;      // conv split-K: fp32 [ksplit][P][cout]
};

__device__ __forceinline__ void pixel_coords(int p, int h, int w, int& n, int& y, int& x) {
    x = p % w;
    const int t = p / w;
    y = t % h;
    n = t / h;
}

template <int MODE, int kStages>
__global__ void __launch_bounds__(kThreads) conv_tile_kernel(const ConvArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bars[kStages];
    __shared__ uint32_t tmem_slot;

    const int tid = threadIdx.x;
    const int P = a.n * a.h * a.w_;
    const int n_tile = a.n_tile;
    const uint32_t a_bytes = kBM * kBK * 2;
    const uint32_t b_bytes = (uint32_t)n_tile * kBK * 2;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    const uint32_t sbase = smem_u32(smem);
    const int n0 = blockIdx.y * n_tile;

    // K extent and tile origin
    int K, m0, kbeg = 0, kend = 0;
    int s_first = 0;  // conv split-K: first K stage of this CTA
    if (MODE == kConv) {
        K = 9 * a.cin;
        m0 = blockIdx.x * kBM;
    } else {
        m0 = blockIdx.x * kBM;  // rows m = tap * cin + ci
        kbeg = blockIdx.z * a.pix_per_split;
        kend = min(P, kbeg + a.pix_per_split);
        K = kend - kbeg;
    }
    const int M = (MODE == kConv) ? P : 9 * a.cin;
    int nk = (K + kBK - 1) / kBK;
    if (MODE == kConv && a.ksplit > 1) {
        const int per = (nk + a.ksplit - 1) / a.ksplit;
        s_first = blockIdx.z * per;
        nk = max(0, min(nk, s_first + per) - s_first);
    }

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(smem_u32(&bars[s]), 1);
        fence_mbar_init();
    }
    if (tid < 32) tmem_alloc(smem_u32(&tmem_slot), (uint32_t)a.tmem_cols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    // per-thread gather state
    int pn = 0, py = 0, px = 0;
    bool p_ok = false;
    int wg_tap = 0, wg_ci = 0;
    bool wg_m_ok = false;
    if (MODE == kConv) {
        const int p = m0 + tid;  // this thread's A row
        p_ok = p < P;
        if (p_ok) pixel_coords(p, a.h, a.w_, pn, py, px);
    } else {
        const int m = m0 + ((tid >> 3) & 15) * 8;  // this thread's 8 A rows
        wg_m_ok = m < M;
        if (wg_m_ok) {
            wg_tap = m / a.cin;
            wg_ci = m - wg_tap * a.cin;
        }
    }

    // incremental gather state (stages are loaded in increasing order, so nothing is divided by a
    // runtime value inside the loop)
    int ld_tap = (s_first * kBK) / a.cin, ld_ci = (s_first * kBK) % a.cin;  // conv: next stage's first k
    int b_r0 = tid % n_tile, b_kc0 = tid / n_tile;   // conv: first B unit of this thread
    int wq_n = 0, wq_y = 0, wq_x = 0, wq_p = kbeg + (tid & 7);  // wgrad: this thread's next A pixel
    if (MODE == kWgrad && wq_p < P) pixel_coords(wq_p, a.h, a.w_, wq_n, wq_y, wq_x);
    const int nch = n_tile / 8;
    const int wb_rest0 = tid >> 3;
    const int wb_nc0 = wb_rest0 % nch, wb_kph0 = wb_rest0 / nch;

    auto load_stage = [&](int slot, int s) {
        const uint32_t sA = sbase + slot * stage_bytes;
        const uint32_t sB = sA + a_bytes;
        if (MODE == kConv) {
            const int k0 = (s_first + s) * kBK;
            // A: row tid, 8 chunks of 8 channels; unit (r, kc) at kc * kBM * 16 + r * 16
            int tap = ld_tap, ci = ld_ci;
#pragma unroll
            for (int kc = 0; kc < 8; ++kc) {
                const int kk = k0 + kc * 8;
                const bf16* src = a.x;
                bool v = false;
                if (p_ok && kk < K) {
                    const int dy = (tap * 11) >> 5, dx = tap - 3 * dy;  // tap / 3, tap % 3 for tap < 9
                    const int yy = py + dy - 1, xx = px + dx - 1;
                    if (yy >= 0 && yy < a.h && xx >= 0 && xx < a.w_) {
                        v = true;
                        src = a.x + ((size_t)(pn * a.h + yy) * a.w_ + xx) * a.cin + ci;
                    }
                }
                cp_async16(sA + kc * (kBM * 16) + tid * 16, src, v);
                ci += 8;
                while (ci >= a.cin) {
                    ci -= a.cin;
                    ++tap;
                }
            }
            ld_tap = tap;
            ld_ci = ci;
            // B: weight rows n0 .. n0 + n_tile; unit (r, kc) at kc * n_tile * 16 + r * 16
            int r = b_r0, kc = b_kc0;
            for (int q = tid; q < n_tile * 8; q += kThreads) {
                const int kk = k0 + kc * 8, co = n0 + r;
                const bool v = co < a.cout && kk < K;
                cp_async16(sB + kc * (n_tile * 16) + r * 16, v ? a.w + (size_t)co * K + kk : a.w, v);
                r += kThreads;
                while (r >= n_tile) {
                    r -= n_tile;
                    ++kc;
                }
            }
        } else {
            const int pbase = kbeg + s * kBK;
            // A (MN-major): unit (mc, kp) at (kp / 8) * 2048 + mc * 128 + (kp % 8) * 16 = 16 * q; this
            // thread's pixels advance by 8 per unit
            const int tdy = (wg_tap * 11) >> 5, tdx = wg_tap - 3 * tdy;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const bf16* src = a.x;
                bool v = false;
                if (wg_m_ok && wq_p < kend) {
                    const int yy = wq_y + tdy - 1, xx = wq_x + tdx - 1;
                    if (yy >= 0 && yy < a.h && xx >= 0 && xx < a.w_) {
                        v = true;
                        src = a.x + ((size_t)(wq_n * a.h + yy) * a.w_ + xx) * a.cin + wg_ci;
                    }
                }
                cp_async16(sA + (i * kThreads + tid) * 16, src, v);
                wq_p += 8;
                wq_x += 8;
                while (wq_x >= a.w_) {
                    wq_x -= a.w_;
                    if (++wq_y == a.h) {
                        wq_y = 0;
                        ++wq_n;
                    }
                }
            }
            // B (MN-major): dy rows; unit (nc, kp) at (kp / 8) * n_tile * 16 + nc * 128 + (kp % 8) * 16
            int nc = wb_nc0, kph = wb_kph0;
            for (int q = tid; q < n_tile * 8; q += kThreads) {
                const int p = pbase + kph * 8 + (tid & 7), co = n0 + nc * 8;
                const bool v = p < kend && co < a.cout;
                cp_async16(sB + q * 16, v ? a.w + (size_t)p * a.cout + co : a.w, v);
                nc += kThreads / 8;
                while (nc >= nch) {
                    nc -= nch;
                    ++kph;
                }
            }
        }
    };

    const uint32_t idesc = (MODE == kConv) ? instr_desc(kBM, n_tile, 0, 0) : instr_desc(kBM, n_tile, 1, 1);
    const uint32_t a_lbo = (MODE == kConv) ? kBM * 16 : (kBM / 8) * 128;
    const uint32_t b_lbo = (uint32_t)n_tile * 16;

    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) load_stage(s, s);
        cp_async_commit();
    }
    int aborted = 0;
    int issued = -1;  // last stage whose MMAs were committed
    for (int s = 0; s < nk; ++s) {
        const int slot = s % kStages;
        cp_async_wait<kStages - 2>();
        fence_proxy_async();
        if (__syncthreads_or(aborted)) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sA = sbase + slot * stage_bytes;
            const uint32_t sB = sA + a_bytes;
            const int steps = min(kBK / 16, (K - (s_first + s) * kBK + 15) / 16);
            for (int j = 0; j < steps; ++j) {
                const uint64_t da = smem_desc(sA + j * 2 * a_lbo, a_lbo, 128);
                const uint64_t db = smem_desc(sB + j * 2 * b_lbo, b_lbo, 128);
                mma_bf16(tmem, da, db, idesc, (s > 0 || j > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&bars[slot]));
        }
        issued = s;
        const int nxt = s + kStages - 1;
        if (nxt < nk) {
            bool ok = true;
            if (s >= 1) {  // the slot of stage s - 1 is refilled: its MMAs must have read it
                const int ps = s - 1;
                ok = mbar_wait(smem_u32(&bars[ps % kStages]), (uint32_t)((ps / kStages) & 1));
            }
            if (ok) load_stage(nxt % kStages, nxt);
            else aborted = 1;
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    // the last commit tracks every MMA this CTA issued
    bool done = true;
    if (issued >= 0) done = mbar_wait(smem_u32(&bars[issued % kStages]), (uint32_t)((issued / kStages) & 1));
    const bool fail = __syncthreads_or(aborted || !done || (issued != nk - 1 && nk > 0));
    tc_fence_after();

    if (!fail && nk == 0 && MODE == kConv && a.partial) {  // an empty K range contributes zeros
        const int p = m0 + tid;
        if (p < P)
            for (int co = n0; co < min(a.cout, n0 + n_tile); co += 4)
                *reinterpret_cast<float4*>(a.partial + ((size_t)blockIdx.z * P + p) * a.cout + co) =
                    make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (!fail && nk > 0) {
        const int warp = tid >> 5, lane = tid & 31;
        const int r = warp * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < n_tile; c0 += 16) {
            float v[16];
            tmem_ld16(trow + (uint32_t)c0, v);  // whole warp, uniform
            const int co = n0 + c0;
            if (co >= a.cout) continue;
            if (MODE == kConv) {
                const int p = m0 + r;
                if (p >= P) continue;
                if (a.partial) {  // split-K: raw sums, finished by conv_finalize_kernel
                    float4* dst = reinterpret_cast<float4*>(a.partial + ((size_t)blockIdx.z * P + p) * a.cout + co);
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                    continue;
                }
                if (a.bias) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] += a.bias[co + i];
                }
                if (a.relu) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
                }
                if (a.mask) {
                    const uint4* mp = reinterpret_cast<const uint4*>(a.mask + (size_t)p * a.cout + co);
                    const uint4 m4[2] = {mp[0], mp[1]};
                    const bf16* mb = reinterpret_cast<const bf16*>(m4);
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = __bfloat162float(mb[i]) > 0.0f ? v[i] : 0.0f;
                }
                if (a.out_f32) {
                    float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.y) + (size_t)p * a.cout + co);
#pragma unroll
                    for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                } else {
                    uint4 o[2];
                    __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(o);
#pragma unroll
                    for (int i = 0; i < 8; ++i) ob[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                    uint4* dst = reinterpret_cast<uint4*>(static_cast<bf16*>(a.y) + (size_t)p * a.cout + co);
                    dst[0] = o[0];
                    dst[1] = o[1];
                }
            } else {
                const int m = m0 + r;
                if (m >= M) continue;
                float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.y) +
                                                        ((size_t)blockIdx.z * a.m_pad + m) * a.cout + co);
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
    }
    if (fail && tid == 0 && a.err) atomicExch(a.err, (int)VPT_ERR_ITER_LIMIT);
    tc_fence_before();
    __syncthreads();
    if (tid < 32) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)a.tmem_cols);
    }
}

// Split-K convolution: y = act(bias + sum over the splits of partial[s]) (fixed order), times the
// ReLU-derivative mask, stored bf16 or fp32; 4 channels per thread.
__global__ void conv_finalize_kernel(const float* __restrict__ partial, int ksplit, long P, int cout,
                                     const float* __restrict__ bias, const bf16* __restrict__ mask, int relu,
                                     int out_f32, void* __restrict__ y) {
    const long total = P * (cout / 4);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long p = i / (cout / 4);
        const int c = (int)(i % (cout / 4)) * 4;
        float4 acc = reinterpret_cast<const float4*>(partial + p * cout + c)[0];
        for (int k = 1; k < ksplit; ++k) {
            const float4 u = reinterpret_cast<const float4*>(partial + ((size_t)k * P + p) * cout + c)[0];
            acc.x += u.x;
            acc.y += u.y;
            acc.z += u.z;
            acc.w += u.w;
        }
        float v[4] = {acc.x, acc.y, acc.z, acc.w};
        for (int j = 0; j < 4; ++j) {
            if (bias) v[j] += bias[c + j];
            if (relu) v[j] = fmaxf(v[j], 0.0f);
            if (mask) v[j] = __bfloat162float(mask[p * cout + c + j]) > 0.0f ? v[j] : 0.0f;
        }
        if (out_f32) {
            reinterpret_cast<float4*>(static_cast<float*>(y) + p * cout + c)[0] = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(y) + p * cout + c);
            o[0] = __floats2bfloat162_rn(v[0], v[1]);
            o[1] = __floats2bfloat162_rn(v[2], v[3]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// the row-strip convolution (forward and input gradient on images at least 128 pixels wide)
// ---------------------------------------------------------------------------------------------
// A persistent CTA owns segments of consecutive rows of one 128-pixel-wide image column
// (n, x0 .. x0 + 127).  The output tile of row y needs input rows y-1, y, y+1 at x0-1 .. x0+128: each
// input row is gathered once into a ring of 5 shared-memory row strips (130 pixels per 8-channel
// plane, 16 bytes per pixel, planes 2080 bytes apart), so that a row stays resident for the three
// output rows that use it and the row two ahead is in flight.  In the UMMA K-major no-swizzle layout
// (8-row core matrices of 16-byte rows, SBO = 128 between 8-pixel groups, LBO = plane stride between
// 8-channel chunks) the A operand of tap (dy, dx) is the strip of row y+dy with its start address
// moved by dx * 16 bytes: the three horizontal taps share one gather.  All 9 taps of the weights are
// resident in shared memory for the CTA's lifetime.  Two TMEM accumulators alternate: the epilogue
// of tile i-1 (tcgen05.ld, bias, ReLU, mask, store) runs while the tensor core computes tile i.
constexpr int kStripPix = kBM + 2;          // 130 pixels: x0-1 .. x0+128
constexpr int kPlane = kStripPix * 16;      // bytes per 8-channel plane of a row strip
constexpr int kRing = 5;                    // row strips resident

struct StripArgs {
    const bf16* x;       // [n][h][w][cin]
    const bf16* w;       // [cout][9][cin]
    const float* bias;   // [cout] or null
    const bf16* mask;    // [n][h][w][cout] or null
    void* y;             // [n][h][w][cout] bf16 / fp32
    int* err;
    int n, h, w_, cin, cout;   // cin: input channels of this pass (a group of the tensor's channels)
    int cin_total, c0;         // channels per pixel of x (and per tap of w); first channel of this pass
    const float* part_in;      // fp32 [n][h][w][cout] partial sum added before the epilogue, or null
    float* part_out;           // non-null: store the raw fp32 sum here (an intermediate pass), no epilogue
    int relu, out_f32;
    int xtiles;          // ceil(w / 128)
    int seg_rows;        // rows per segment
    int segs_per_col;
    int tmem_cols;
};

// TMEM lane quarter `quarter` (the warp's index mod 4) holds pixels x0 + 32 quarter .. + 31
__device__ __forceinline__ void strip_epilogue(const StripArgs& a, uint32_t tacc, int n_img, int yrow, int x0,
                                               int quarter, int lane) {
    const int x = x0 + quarter * 32 + lane;
    const bool ok = x < a.w_;
    const size_t p = ((size_t)n_img * a.h + yrow) * a.w_ + (ok ? x : 0);
    const uint32_t trow = tacc + ((uint32_t)(quarter * 32) << 16);
    for (int c0 = 0; c0 < a.cout; c0 += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c0, v);
        if (!ok) continue;
        if (a.part_in) {
            const float4* src = reinterpret_cast<const float4*>(a.part_in + p * a.cout + c0);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float4 u = src[i];
                v[4 * i] += u.x;
                v[4 * i + 1] += u.y;
                v[4 * i + 2] += u.z;
                v[4 * i + 3] += u.w;
            }
        }
        if (a.part_out) {
            float4* dst = reinterpret_cast<float4*>(a.part_out + p * a.cout + c0);
#pragma unroll
            for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            continue;
        }
        if (a.bias) {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] += a.bias[c0 + i];
        }
        if (a.relu) {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
        }
        if (a.mask) {
            const uint4* mp = reinterpret_cast<const uint4*>(a.mask + p * a.cout + c0);
            const uint4 m4[2] = {mp[0], mp[1]};
            const bf16* mb = reinterpret_cast<const bf16*>(m4);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = __bfloat162float(mb[i]) > 0.0f ? v[i] : 0.0f;
        }
        if (a.out_f32) {
            float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.y) + p * a.cout + c0);
#pragma unroll
            for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        } else {
            uint4 o[2];
            __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(o);
#pragma unroll
            for (int i = 0; i < 8; ++i) ob[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
            uint4* dst = reinterpret_cast<uint4*>(static_cast<bf16*>(a.y) + p * a.cout + c0);
            dst[0] = o[0];
            dst[1] = o[1];
        }
    }
}

__global__ void __launch_bounds__(kThreads) conv_strip_kernel(const StripArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x;
    const int nkc = a.cin / 8;
    const uint32_t w_bytes = 9u * (uint32_t)a.cin * (uint32_t)a.cout * 2u;
    const uint32_t row_bytes = (uint32_t)nkc * kPlane;
    const uint32_t sw = smem_u32(smem);
    const uint32_t sring = sw + ((w_bytes + 127u) & ~127u);

    if (tid == 0) {
        mbar_init(smem_u32(&bars[0]), 1);
        mbar_init(smem_u32(&bars[1]), 1);
        fence_mbar_init();
    }
    if (tid < 32) tmem_alloc(smem_u32(&tmem_slot), (uint32_t)a.tmem_cols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    // resident weights: unit (t, kc, co) at ((t * nkc + kc) * cout + co) * 16
    for (int q = tid; q < 9 * nkc * a.cout; q += kThreads) {
        const int co = q % a.cout, rest = q / a.cout;
        const int kc = rest % nkc, t = rest / nkc;
        cp_async16(sw + (uint32_t)q * 16u, a.w + ((size_t)co * 9 + t) * a.cin_total + a.c0 + kc * 8, true);
    }
    cp_async_commit();

    auto load_row = [&](int n_img, int yy, int x0) {
        const uint32_t base = sring + (uint32_t)(((yy + 1) % kRing + kRing) % kRing) * row_bytes;
        const bool row_ok = yy >= 0 && yy < a.h;
        for (int q = tid; q < kStripPix * nkc; q += kThreads) {
            const int r = q % kStripPix, kc = q / kStripPix;
            const int xx = x0 - 1 + r;
            const bool v = row_ok && xx >= 0 && xx < a.w_;
            const bf16* src = v ? a.x + (((size_t)n_img * a.h + yy) * a.w_ + xx) * a.cin_total + a.c0 + kc * 8 : a.x;
            cp_async16(base + (uint32_t)kc * kPlane + (uint32_t)r * 16u, src, v);
        }
    };

    const uint32_t idesc = instr_desc(kBM, a.cout, 0, 0);
    const uint32_t b_lbo = (uint32_t)a.cout * 16u;
    const int total_segs = a.n * a.xtiles * a.segs_per_col;
    long g = 0;          // tiles computed by this CTA (accumulator index and mbarrier parity)
    int fail = 0;
    int pend_n = 0, pend_y = 0, pend_x0 = 0;
    bool pending = false;  // a tile whose epilogue has not run

    for (int seg = blockIdx.x; seg < total_segs && !fail; seg += gridDim.x) {
        const int col = seg / a.segs_per_col, part = seg % a.segs_per_col;
        const int n_img = col / a.xtiles, x0 = (col % a.xtiles) * kBM;
        const int y0 = part * a.seg_rows, y1 = min(a.h, y0 + a.seg_rows);
        if (y0 >= y1) continue;
        // every MMA of the previous segment has finished reading the ring
        if (pending) {
            if (!mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail = 1;
            if (__syncthreads_or(fail)) break;
            tc_fence_after();
            strip_epilogue(a, tmem + (uint32_t)(((g - 1) & 1) * a.cout), pend_n, pend_y, pend_x0, tid >> 5, tid & 31);
            pending = false;
        }
        load_row(n_img, y0 - 1, x0);
        load_row(n_img, y0, x0);
        load_row(n_img, y0 + 1, x0);
        cp_async_commit();
        if (y0 + 2 <= y1) load_row(n_img, y0 + 2, x0);
        cp_async_commit();
        for (int yrow = y0; yrow < y1; ++yrow, ++g) {
            cp_async_wait<1>();  // rows yrow-1 .. yrow+1 (and the weights) have landed
            fence_proxy_async();
            tc_fence_before();
            if (__syncthreads_or(fail)) break;
            const int buf = (int)(g & 1);
            if (tid == 0) {
                tc_fence_after();
                const uint32_t dacc = tmem + (uint32_t)(buf * a.cout);
                int first = 1;
                for (int dy = 0; dy < 3; ++dy) {
                    const uint32_t rb = sring + (uint32_t)((yrow + dy) % kRing) * row_bytes;  // slot of row yrow+dy-1
                    for (int dx = 0; dx < 3; ++dx) {
                        const int t = dy * 3 + dx;
                        for (int j = 0; j < nkc / 2; ++j) {
                            const uint64_t da = smem_desc(rb + (uint32_t)(2 * j) * kPlane + (uint32_t)dx * 16u, kPlane,
                                                          128);
                            const uint64_t db = smem_desc(sw + (uint32_t)((t * nkc + 2 * j) * a.cout) * 16u, b_lbo, 128);
                            mma_bf16(dacc, da, db, idesc, first ? 0u : 1u);
                            first = 0;
                        }
                    }
                }
                mma_commit(smem_u32(&bars[buf]));
            }
            if (pending) {  // epilogue of the previous tile while this one computes
                if (!mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail = 1;
                if (__syncthreads_or(fail)) break;
                tc_fence_after();
                strip_epilogue(a, tmem + (uint32_t)(((g - 1) & 1) * a.cout), pend_n, pend_y, pend_x0, tid >> 5, tid & 31);
            }
            pending = true;
            pend_n = n_img;
            pend_y = yrow;
            pend_x0 = x0;
            // the previous tile's MMAs are done: the slot of row yrow-2 is free for row yrow+3
            if (yrow + 3 <= y1) load_row(n_img, yrow + 3, x0);
            cp_async_commit();
        }
    }
    cp_async_wait<0>();
    if (pending && !fail) {
        if (!mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail = 1;
        if (!__syncthreads_or(fail)) {
            tc_fence_after();
            strip_epilogue(a, tmem + (uint32_t)(((g - 1) & 1) * a.cout), pend_n, pend_y, pend_x0, tid >> 5, tid & 31);
        }
    } else if (pending) {
        // bounded wait for the MMAs in flight before the accumulator is freed
        mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1));
    }
    if (__syncthreads_or(fail) && tid == 0 && a.err) atomicExch(a.err, (int)VPT_ERR_ITER_LIMIT);
    tc_fence_before();
    __syncthreads();
    if (tid < 32) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)a.tmem_cols);
    }
}

// ---------------------------------------------------------------------------------------------
// the warp-specialised row-strip convolution (TMA-fed)
// ---------------------------------------------------------------------------------------------
// The tiling of conv_strip_kernel (persistent CTAs over segments of consecutive rows of one
// 128-pixel column; row strips of 130 pixels; A of tap (dy, dx) = the strip of row y+dy-1 with its
// start moved by dx pixel rows; the weights of all 9 taps resident), with the work split over warps
// and no CTA-wide barrier after the weights have landed:
//   warp 0     one lane loads input rows into a ring of `ring` slots with the tensor-memory-access
//              unit: one box {64 / 32 / 16 channels, 130 pixels} per channel group, written in the
//              swizzled K-major layout of that line width (pixel rows of 128 / 64 / 32 bytes), rows and
//              pixels outside the image arriving as zeros; full[s] completes on the bytes, empty[s] is
//              signalled by the tensor core once the last MMA reading the slot has completed;
//   warps 1, 6 one lane each issues the 9 x cin/16 MMAs of every other output row (accumulator
//              index g: warp 1 the even, warp 6 the odd) into TMEM accumulator g % 2 (acc_full[b] on
//              completion, after acc_empty[b]): one issuing thread is the bound for small N (about 93
//              cycles per MMA against the tensor core's 48), two overlap their issue;
//   warps 2-5  the epilogue; warp w reads TMEM lane quarter w % 4 (pixels x0 + 32 (w % 4) .. + 31).
// All roles walk the same segment sequence, so ring and accumulator positions agree without
// communication.  Every wait is bounded: on expiry the role records the error and stops, and the
// CTA waits (bounded) for its copies and MMAs in flight before TMEM is released.
constexpr int kWsThreads = 224;  // 7 warps: producer, MMA issuer, 4 epilogue warps, second MMA issuer
constexpr int kWsMaxRing = 8;

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
// tiled 4-D load (coordinates innermost first) into this CTA's shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

struct WsSegment {
    int n_img, x0, y0, y1;
};
__device__ __forceinline__ WsSegment ws_segment(const StripArgs& a, int seg) {
    const int col = seg / a.segs_per_col, part = seg % a.segs_per_col;
    WsSegment g;
    g.n_img = col / a.xtiles;
    g.x0 = (col % a.xtiles) * kBM;
    g.y0 = part * a.seg_rows;
    g.y1 = min(a.h, g.y0 + a.seg_rows);
    return g;
}

// Channel groups of a row: widths 64 / 32 / 16 channels = lines of 128 / 64 / 32 bytes per pixel in
// the 128B / 64B / 32B-swizzled K-major layout (what one TMA box of {width, 130 pixels} writes);
// each group buffer starts on a 1024-byte boundary.
constexpr int kWsMaxGroups = 4;
struct WsArgs {
    StripArgs s;
    int ngroups;
    int gc[kWsMaxGroups];    // first channel of the group (within this pass)
    int gw[kWsMaxGroups];    // channels of the group: 64, 32 or 16
    int goff[kWsMaxGroups];  // byte offset of the group buffer in a ring slot
    int row_bytes;           // ring slot size
    int tx_bytes;            // bytes the boxes of one row deliver
};

// K-major swizzled shared-memory descriptor: line = 128 / 64 / 32 bytes per row, 8-row groups
// `8 * line` apart (SBO), LBO unused (1), layout type 2 / 4 / 6 (bits 61-63).  The swizzle acts on
// absolute shared-memory address bits (as the TMA's does), so a start moved by whole rows (the dx
// taps) needs no base offset (measured: base offset 0 matches the oracle for every line width).
__device__ __forceinline__ uint64_t smem_desc_sw(uint32_t addr, uint32_t line) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(((8u * line) >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    const uint64_t layout = line == 128 ? 2 : (line == 64 ? 4 : 6);
    d |= layout << 61;
    return d;
}

// tcgen05.mma from descriptor halves.  No memory clobber: the MMA reads shared memory asynchronously
// and is ordered by the mbarrier waits, tcgen05 fences and commits around it (which carry clobbers);
// without one the issuing loop keeps its loop-invariant values in registers.
__device__ __forceinline__ void mma_bf16_halves(uint32_t tmem_d, uint32_t a_lo, uint32_t a_hi, uint32_t b_lo,
                                                uint32_t b_hi, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\n.reg .b64 da, db;\nmov.b64 da, {%1, %2};\nmov.b64 db, {%3, %4};\n"
        "setp.ne.b32 p, %6, 0;\ntcgen05.mma.cta_group::1.kind::f16 [%0], da, db, %5, p;\n}\n" ::"r"(tmem_d),
        "r"(a_lo), "r"(a_hi), "r"(b_lo), "r"(b_hi), "r"(idesc), "r"(acc));
}

// high word of smem_desc_sw: SBO = 8 lines, version, layout type of the line width (2 * channels)
__device__ __forceinline__ uint32_t a_hi_of(int channels) {
    return (uint32_t)(smem_desc_sw(0, (uint32_t)channels * 2u) >> 32);
}

__global__ void __launch_bounds__(kWsThreads, 2) conv_ws_kernel(const __grid_constant__ CUtensorMap map64,
                                                             const __grid_constant__ CUtensorMap map32,
                                                             const __grid_constant__ CUtensorMap map16,
                                                             const __grid_constant__ WsArgs wa, int ring) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t full[kWsMaxRing], empty[kWsMaxRing], acc_full[2], acc_empty[2], done_bar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int fail_any;
    const StripArgs& a = wa.s;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nkc = a.cin / 8;
    const uint32_t w_bytes = 9u * (uint32_t)a.cin * (uint32_t)a.cout * 2u;
    const uint32_t row_bytes = (uint32_t)wa.row_bytes;
    const uint32_t sw = smem_u32(smem);
    const uint32_t sring = sw + ((w_bytes + 1023u) & ~1023u);
    const uint32_t acc_cols = (uint32_t)a.tmem_cols / 2;
    if (tid == 0) {
        for (int s = 0; s < ring; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 2);  // one release per MMA-issuing warp
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 4);  // one arrival per epilogue warp
            mbar_init(smem_u32(&done_bar[b]), 1);
        }
        fail_any = 0;
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(smem_u32(&tmem_slot), (uint32_t)a.tmem_cols);
    // resident weights: unit (t, kc, co) at ((t * nkc + kc) * cout + co) * 16
    for (int q = tid; q < 9 * nkc * a.cout; q += kWsThreads) {
        const int co = q % a.cout, rest = q / a.cout;
        const int kc = rest % nkc, t = rest / nkc;
        cp_async16(sw + (uint32_t)q * 16u, a.w + ((size_t)co * 9 + t) * a.cin_total + a.c0 + kc * 8, true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const int total_segs = a.n * a.xtiles * a.segs_per_col;
    bool fail = false;

    if (warp == 0) {
        if (lane == 0) {
            int slot = 0;
            uint32_t phase = 0;
            long issued = 0;
            for (int seg = blockIdx.x; seg < total_segs && !fail; seg += gridDim.x) {
                const WsSegment g = ws_segment(a, seg);
                if (g.y0 >= g.y1) continue;
                for (int yy = g.y0 - 1; yy <= g.y1; ++yy) {
                    if (!mbar_wait(smem_u32(&empty[slot]), phase ^ 1u)) {
                        fail = true;
                        break;
                    }
                    const uint32_t dst = sring + (uint32_t)slot * row_bytes;
                    const uint32_t fb = smem_u32(&full[slot]);
                    mbar_arrive_expect_tx(fb, (uint32_t)wa.tx_bytes);
                    for (int k = 0; k < wa.ngroups; ++k) {
                        const CUtensorMap* m = wa.gw[k] == 64 ? &map64 : (wa.gw[k] == 32 ? &map32 : &map16);
                        tma_load_4d(dst + (uint32_t)wa.goff[k], m, a.c0 + wa.gc[k], g.x0 - 1, yy, g.n_img, fb);
                    }
                    ++issued;
                    if (++slot == ring) {
                        slot = 0;
                        phase ^= 1u;
                    }
                }
            }
            // the last loads (one per slot at most) have landed before the CTA can exit
            const long tail = issued < ring ? issued : ring;
            for (long k = 1; k <= tail; ++k) {
                int s = slot - (int)k;
                uint32_t ph = phase;
                if (s < 0) {
                    s += ring;
                    ph ^= 1u;
                }
                if (!mbar_wait(smem_u32(&full[s]), ph)) fail = true;
            }
        }
    } else if (warp == 1 || warp == 6) {
        if (lane == 0) {
            const int mw = warp == 1 ? 0 : 1;  // this warp's accumulator parity
            const uint32_t idesc = instr_desc(kBM, a.cout, 0, 0);
            // descriptor words: A (swizzled, start field added per row / group / dx / step; LBO 1),
            // B (no swizzle, LBO = one 8-channel plane of the weights, SBO 128)
            const uint64_t bd0 = smem_desc(sw, (uint32_t)a.cout * 16u, 128);
            const uint32_t b_hi = (uint32_t)(bd0 >> 32), b_lo0 = (uint32_t)bd0;
            const uint32_t a_lo1 = 1u << 16;  // LBO field of the A descriptors
            const uint32_t b_step = 2u * (uint32_t)a.cout, b_tap = (uint32_t)(nkc * a.cout), b_row = 3u * b_tap;
            // per channel group (registers: every index below is a compile-time constant)
            const int ngroups = wa.ngroups;
            uint32_t g_ahi[kWsMaxGroups], g_aoff[kWsMaxGroups], g_line[kWsMaxGroups], g_boff[kWsMaxGroups];
            int g_steps[kWsMaxGroups];
#pragma unroll
            for (int k = 0; k < kWsMaxGroups; ++k) {
                const bool on = k < ngroups;
                const int gw = on ? wa.gw[k] : 16;
                g_ahi[k] = a_hi_of(gw);
                g_aoff[k] = on ? (uint32_t)wa.goff[k] >> 4 : 0u;
                g_line[k] = (uint32_t)gw >> 3;  // line bytes / 16
                g_boff[k] = on ? (uint32_t)((wa.gc[k] >> 3) * a.cout) : 0u;
                g_steps[k] = gw / 16;
            }
            int slot = 0;        // ring position of the segment's first row
            uint32_t phase = 0;
            long g = 0;          // accumulators used (both warps count every output row)
            // Ring slots are released by both issuing warps (empty[] counts 2): after output row i
            // its warp releases input rows i and i+1 (its last uses of them: it also computed row
            // i-2, the other warp rows i-1 and i+1).  Rows without such a row get the arrival at the
            // segment's start (input row 0 from the warp of row -1) or end (rows `rows`, `rows`+1).
            auto own = [&](long gi) { return (int)(gi & 1) == mw; };
            auto slot_of = [&](int r) { return (uint32_t)((slot + r) % ring); };
            for (int seg = blockIdx.x; seg < total_segs && !fail; seg += gridDim.x) {
                const WsSegment sgm = ws_segment(a, seg);
                if (sgm.y0 >= sgm.y1) continue;
                const int rows = sgm.y1 - sgm.y0;
                const long g0 = g;
                if (own(g0 - 1)) mbar_arrive(smem_u32(&empty[slot_of(0)]));
                for (int i = 0; i < rows && !fail; ++i, ++g) {
                    if (!own(g)) continue;
                    // input rows i, i+1, i+2 of the segment (y-1, y, y+1)
                    for (int k = 0; k <= 2; ++k) {
                        const int pos = slot + i + k;
                        const uint32_t ph = phase ^ (uint32_t)((pos / ring) & 1);
                        if (!mbar_wait(smem_u32(&full[pos % ring]), ph)) fail = true;
                    }
                    const int b = (int)(g & 1);
                    if (!fail && !mbar_wait(smem_u32(&acc_empty[b]), (uint32_t)(((g >> 1) & 1) ^ 1))) fail = true;
                    if (fail) break;
                    tc_fence_after();
                    const uint32_t dacc = tmem + (uint32_t)b * acc_cols;
                    // descriptors walk affinely: per channel group, A's start advances by one pixel
                    // row per dx and 32 bytes per 16-channel step, B's by a tap (nkc * cout * 16
                    // bytes) per dx and two 8-channel planes per step
                    uint32_t acc = 0;
#pragma unroll 1
                    for (int dy = 0; dy < 3; ++dy) {
                        const uint32_t row16 = (sring + slot_of(i + dy) * row_bytes) >> 4;
#pragma unroll
                        for (int k = 0; k < kWsMaxGroups; ++k) {
                            if (k >= ngroups) break;
                            const uint32_t al0 = a_lo1 + row16 + g_aoff[k];
                            const uint32_t bl0 = b_lo0 + (uint32_t)dy * b_row + g_boff[k];
#pragma unroll
                            for (int dx = 0; dx < 3; ++dx) {
                                const uint32_t al = al0 + (uint32_t)dx * g_line[k], bl = bl0 + (uint32_t)dx * b_tap;
#pragma unroll
                                for (int j = 0; j < 4; ++j) {
                                    if (j >= g_steps[k]) break;
                                    mma_bf16_halves(dacc, al + 2u * (uint32_t)j, g_ahi[k], bl + (uint32_t)j * b_step,
                                                    b_hi, idesc, acc);
                                    acc = 1;
                                }
                            }
                        }
                    }
                    mma_commit(smem_u32(&acc_full[b]));
                    mma_commit(smem_u32(&empty[slot_of(i)]));
                    mma_commit(smem_u32(&empty[slot_of(i + 1)]));
                }
                if (fail) break;
                if (own(g0 + rows - 1)) mma_commit(smem_u32(&empty[slot_of(rows + 1)]));
                if (own(g0 + rows)) {
                    mma_commit(smem_u32(&empty[slot_of(rows)]));
                    mma_commit(smem_u32(&empty[slot_of(rows + 1)]));
                }
                const int adv = slot + rows + 2;
                slot = adv % ring;
                phase ^= (uint32_t)((adv / ring) & 1);
            }
            // every MMA this warp issued has completed before TMEM is released
            mma_commit(smem_u32(&done_bar[mw]));
            if (!mbar_wait(smem_u32(&done_bar[mw]), 0)) fail = true;
        }
    } else if (warp >= 2 && warp <= 5) {
        const int quarter = warp & 3;
        long g = 0;
        for (int seg = blockIdx.x; seg < total_segs && !fail; seg += gridDim.x) {
            const WsSegment sgm = ws_segment(a, seg);
            for (int y = sgm.y0; y < sgm.y1; ++y, ++g) {
                const int b = (int)(g & 1);
                const bool ok = mbar_wait(smem_u32(&acc_full[b]), (uint32_t)((g >> 1) & 1));
                if (!__all_sync(0xffffffffu, ok)) {
                    fail = true;
                    break;
                }
                tc_fence_after();
                strip_epilogue(a, tmem + (uint32_t)b * acc_cols, sgm.n_img, y, sgm.x0, quarter, lane);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
            }
        }
    }
    if (fail) atomicOr(&fail_any, 1);
    tc_fence_before();
    __syncthreads();
    if (fail_any && tid == 0 && a.err) atomicExch(a.err, (int)VPT_ERR_ITER_LIMIT);
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)a.tmem_cols);
    }
}

// ---------------------------------------------------------------------------------------------
// the row-strip weight gradient (images at least 128 pixels wide)
// ---------------------------------------------------------------------------------------------
// dw[co][t][ci] = sum over pixels p of dy[p][co] * x[p + off(t)][ci].  Per output row y of a 128-pixel
// column: the 128 pixels are the K dimension; for tap (dy, dx) the x operand is the row strip of
// input row y+dy-1 shifted by dx pixels (descriptor start + dx * 16 bytes, as in the forward strip
// kernel), the dy operand is output-gradient row y.  Both operands are MN-major (8-channel planes of
// 16-byte pixel rows: LBO = 128 between 8-pixel groups, SBO = plane stride between channel groups).
// ROLE 0: A = x (M = input channels m0 .. m0+ma, zero planes beyond), B = dy (N = output channels);
// ROLE 1: A = dy (M = output channels m0 .. m0+ma), B = x (N = input channels).  Each tap t of
// [t0, t1) accumulates in its own TMEM block (columns (t - t0) * N) over every row the CTA owns; the
// CTA writes its sums to partial[blockIdx.x][t * cin + ci][co] at the end (reduced in fixed order by
// reduce_grads_kernel).  M = 64 accumulators occupy lanes 0-15 of each 32-lane quarter of TMEM.
constexpr int kDyRing = 3;
constexpr int kDyPlane = kBM * 16;  // 2048 bytes: 128 pixels x 16 bytes

struct WgradStripArgs {
    const bf16* x;      // [n][h][w][cin]
    const bf16* dy;     // [n][h][w][cout]
    float* partial;     // [splits][m_pad][cout]
    int* err;
    int n, h, w_, cin, cout;
    int m0, ma;         // A channel range (input channels for role 0, output channels for role 1), ma 64 / 128
    int t0, t1;         // taps of this pass
    int xplanes, dyplanes;  // 8-channel planes per x strip / dy row in shared memory
    int m_pad;
    int xtiles, seg_rows, segs_per_col, tmem_cols;
};

template <int ROLE>
__global__ void __launch_bounds__(kThreads) wgrad_strip_kernel(const WgradStripArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x;
    const int N = ROLE == 0 ? a.cout : a.cin;
    const uint32_t xrow = (uint32_t)a.xplanes * kPlane, dyrow = (uint32_t)a.dyplanes * kDyPlane;
    const uint32_t sx = smem_u32(smem);
    const uint32_t sdy = sx + kRing * xrow;
    // channels gathered into the strips: x planes [x_c0, x_c0 + 8 * x_real), dy planes likewise
    const int x_c0 = ROLE == 0 ? a.m0 : 0;
    const int x_real = ROLE == 0 ? min(a.ma, a.cin - a.m0) / 8 : a.cin / 8;
    const int dy_c0 = ROLE == 0 ? 0 : a.m0;
    const int dy_real = ROLE == 0 ? a.cout / 8 : min(a.ma, a.cout - a.m0) / 8;

    if (tid == 0) {
        mbar_init(smem_u32(&bars[0]), 1);
        mbar_init(smem_u32(&bars[1]), 1);
        fence_mbar_init();
    }
    if (tid < 32) tmem_alloc(smem_u32(&tmem_slot), (uint32_t)a.tmem_cols);
    // zero the padding planes of every ring slot once (the gathers never write them)
    {
        uint4* base = reinterpret_cast<uint4*>(smem);
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (int slot = 0; slot < kRing; ++slot)
            for (int q = tid; q < (a.xplanes - x_real) * kStripPix; q += kThreads)
                base[(slot * xrow + (uint32_t)(x_real + q / kStripPix) * kPlane) / 16 + q % kStripPix] = z;
        for (int slot = 0; slot < kDyRing; ++slot)
            for (int q = tid; q < (a.dyplanes - dy_real) * kBM; q += kThreads)
                base[(kRing * xrow + slot * dyrow + (uint32_t)(dy_real + q / kBM) * kDyPlane) / 16 + q % kBM] = z;
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    auto load_x = [&](int n_img, int yy, int x0) {
        const uint32_t base = sx + (uint32_t)(((yy + 1) % kRing + kRing) % kRing) * xrow;
        const bool row_ok = yy >= 0 && yy < a.h;
        for (int q = tid; q < kStripPix * x_real; q += kThreads) {
            const int r = q % kStripPix, kc = q / kStripPix;
            const int xx = x0 - 1 + r;
            const bool v = row_ok && xx >= 0 && xx < a.w_;
            const bf16* src = v ? a.x + (((size_t)n_img * a.h + yy) * a.w_ + xx) * a.cin + x_c0 + kc * 8 : a.x;
            cp_async16(base + (uint32_t)kc * kPlane + (uint32_t)r * 16u, src, v);
        }
    };
    auto load_dy = [&](int n_img, int yy, int x0) {
        const uint32_t base = sdy + (uint32_t)(yy % kDyRing) * dyrow;
        for (int q = tid; q < kBM * dy_real; q += kThreads) {
            const int r = q % kBM, kc = q / kBM;
            const int xx = x0 + r;
            const bool v = yy < a.h && xx < a.w_;
            const bf16* src = v ? a.dy + (((size_t)n_img * a.h + yy) * a.w_ + xx) * a.cout + dy_c0 + kc * 8 : a.dy;
            cp_async16(base + (uint32_t)kc * kDyPlane + (uint32_t)r * 16u, src, v);
        }
    };

    const uint32_t idesc = instr_desc(a.ma, N, 1, 1);
    // MN-major descriptor words (LBO = 128 between 8-pixel groups, SBO = plane stride); start fields 0
    const uint64_t xd0 = smem_desc(0, 128, kPlane), dd0 = smem_desc(0, 128, kDyPlane);
    const uint32_t x_lo = (uint32_t)xd0, x_hi = (uint32_t)(xd0 >> 32);
    const uint32_t d_lo = (uint32_t)dd0, d_hi = (uint32_t)(dd0 >> 32);
    const int total_segs = a.n * a.xtiles * a.segs_per_col;
    long g = 0;
    int fail = 0;
    for (int seg = blockIdx.x; seg < total_segs && !fail; seg += gridDim.x) {
        const int col = seg / a.segs_per_col, part = seg % a.segs_per_col;
        const int n_img = col / a.xtiles, x0 = (col % a.xtiles) * kBM;
        const int y0 = part * a.seg_rows, y1 = min(a.h, y0 + a.seg_rows);
        if (y0 >= y1) continue;
        if (g > 0) {  // the previous segment's MMAs have read their rows
            if (!mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail = 1;
            if (__syncthreads_or(fail)) break;
        }
        load_x(n_img, y0 - 1, x0);
        load_x(n_img, y0, x0);
        load_x(n_img, y0 + 1, x0);
        load_dy(n_img, y0, x0);
        cp_async_commit();
        if (y0 + 2 <= y1) load_x(n_img, y0 + 2, x0);
        if (y0 + 1 < y1) load_dy(n_img, y0 + 1, x0);
        cp_async_commit();
        for (int yrow = y0; yrow < y1; ++yrow, ++g) {
            cp_async_wait<1>();
            fence_proxy_async();
            tc_fence_before();
            if (__syncthreads_or(fail)) break;
            if (tid == 0) {
                tc_fence_after();
                // descriptor halves: the start fields walk 256 bytes (16 pixels) per K step; the x
                // strip of tap (dyy, dxx) starts dxx pixels (16 bytes) into the slot of row yrow+dyy
                const uint32_t d16 = (sdy + (uint32_t)(yrow % kDyRing) * dyrow) >> 4;
                for (int t = a.t0; t < a.t1; ++t) {
                    const int dyy = t / 3, dxx = t - 3 * dyy;
                    const uint32_t x16 = ((sx + (uint32_t)((yrow + dyy) % kRing) * xrow) >> 4) + (uint32_t)dxx;
                    const uint32_t dacc = tmem + (uint32_t)((t - a.t0) * N);
#pragma unroll
                    for (int j = 0; j < kBM / 16; ++j) {
                        const uint32_t xl = x_lo + x16 + 16u * (uint32_t)j, dl = d_lo + d16 + 16u * (uint32_t)j;
                        const uint32_t acc = (g == 0 && j == 0) ? 0u : 1u;
                        if (ROLE == 0) mma_bf16_halves(dacc, xl, x_hi, dl, d_hi, idesc, acc);
                        else mma_bf16_halves(dacc, dl, d_hi, xl, x_hi, idesc, acc);
                    }
                }
                mma_commit(smem_u32(&bars[g & 1]));
            }
            if (yrow > y0) {  // the previous row's MMAs are done: its x and dy slots are free
                if (!mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail = 1;
                if (__syncthreads_or(fail)) break;
            }
            if (yrow + 3 <= y1) load_x(n_img, yrow + 3, x0);
            if (yrow + 2 < y1) load_dy(n_img, yrow + 2, x0);
            cp_async_commit();
        }
    }
    cp_async_wait<0>();
    bool done = true;
    if (g > 0) done = mbar_wait(smem_u32(&bars[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1));
    fail = __syncthreads_or(fail || !done);
    tc_fence_after();
    if (!fail) {
        // accumulator rows: M = 128 -> lane = row; M = 64 -> lanes 0-15 of each warp quarter
        const int warp = tid >> 5, lane = tid & 31;
        const int row = a.ma == 128 ? warp * 32 + lane : (lane < 16 ? warp * 16 + lane : -1);
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        float* part = a.partial + (size_t)blockIdx.x * a.m_pad * a.cout;
        for (int t = a.t0; t < a.t1; ++t) {
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tmem_ld16(trow + (uint32_t)((t - a.t0) * N + c0), v);
                if (row < 0) continue;
                if (g == 0) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = 0.0f;
                }
                if (ROLE == 0) {
                    const int ci = a.m0 + row;
                    if (ci >= a.cin) continue;
                    float4* dst = reinterpret_cast<float4*>(part + (size_t)(t * a.cin + ci) * a.cout + c0);
#pragma unroll
                    for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                } else {
                    const int co = a.m0 + row;
                    if (co >= a.cout) continue;
#pragma unroll
                    for (int i = 0; i < 16; ++i) part[(size_t)(t * a.cin + c0 + i) * a.cout + co] = v[i];
                }
            }
        }
    }
    if (fail && tid == 0 && a.err) atomicExch(a.err, (int)VPT_ERR_ITER_LIMIT);
    tc_fence_before();
    __syncthreads();
    if (tid < 32) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)a.tmem_cols);
    }
}

// ---------------------------------------------------------------------------------------------
// small kernels around the convolutions (NHWC bf16, 8 channels = 16 bytes per thread)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void load8(const bf16* p, float (&f)[8]) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 t = __bfloat1622float2(b[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}
__device__ __forceinline__ void store8(bf16* p, const float (&f)[8]) {
    uint4 u;
    __nv_bfloat162* b = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) b[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    *reinterpret_cast<uint4*>(p) = u;
}

// wrot[ci][t][co] = w[co][8 - t][ci]
__global__ void rotate_weights_kernel(const bf16* __restrict__ w, bf16* __restrict__ wrot, int cin, int cout) {
    const int total = cout * 9 * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int ci = i % cin, t = (i / cin) % 9, co = i / (9 * cin);
        wrot[((size_t)ci * 9 + (8 - t)) * cout + co] = w[i];
    }
}

// 2x2 average pooling, [n][h][w][c] -> [n][h/2][w/2][c]
__global__ void pool2_kernel(const bf16* __restrict__ in, bf16* __restrict__ out, int n, int h, int w, int c) {
    const int ho = h / 2, wo = w / 2, c8 = c / 8;
    const long total = (long)n * ho * wo * c8;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int cc = (int)(i % c8) * 8;
        const long pix = i / c8;
        const int x = (int)(pix % wo), y = (int)((pix / wo) % ho), b = (int)(pix / ((long)wo * ho));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float f[8];
                load8(in + (((size_t)b * h + 2 * y + dy) * w + 2 * x + dx) * c + cc, f);
#pragma unroll
                for (int k = 0; k < 8; ++k) acc[k] += f[k];
            }
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] *= 0.25f;
        store8(out + pix * c + cc, acc);
    }
}

// out[n][y][x] = (lo[n][y/2][x/2] (ca channels), skip[n][y][x] (cs channels)): nearest upsampling
// of the coarser level concatenated with the skip connection
__global__ void upcat_kernel(const bf16* __restrict__ lo, const bf16* __restrict__ skip, bf16* __restrict__ out,
                             int n, int h, int w, int ca, int cs) {
    const int c = ca + cs, c8 = c / 8;
    const long total = (long)n * h * w * c8;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int cc = (int)(i % c8) * 8;
        const long pix = i / c8;
        const int x = (int)(pix % w), y = (int)((pix / w) % h), b = (int)(pix / ((long)w * h));
        const uint4* src;
        if (cc < ca)
            src = reinterpret_cast<const uint4*>(lo + (((size_t)b * (h / 2) + y / 2) * (w / 2) + x / 2) * ca + cc);
        else
            src = reinterpret_cast<const uint4*>(skip + (size_t)pix * cs + (cc - ca));
        *reinterpret_cast<uint4*>(out + (size_t)pix * c + cc) = *src;
    }
}

// backward of upcat for the coarse part: dlo[n][y][x][k] = (lo > 0) * sum of the 2x2 children's
// gradient d[.][k] (k < ca); lo is the coarse level's ReLU output
__global__ void upcat_grad_lo_kernel(const bf16* __restrict__ d, const bf16* __restrict__ lo, bf16* __restrict__ dlo,
                                     int n, int h, int w, int ca, int cs) {
    const int ho = h / 2, wo = w / 2, c = ca + cs, c8 = ca / 8;
    const long total = (long)n * ho * wo * c8;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int cc = (int)(i % c8) * 8;
        const long pix = i / c8;
        const int x = (int)(pix % wo), y = (int)((pix / wo) % ho), b = (int)(pix / ((long)wo * ho));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float f[8];
                load8(d + (((size_t)b * h + 2 * y + dy) * w + 2 * x + dx) * c + cc, f);
#pragma unroll
                for (int k = 0; k < 8; ++k) acc[k] += f[k];
            }
        float m[8];
        load8(lo + pix * ca + cc, m);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = m[k] > 0.0f ? acc[k] : 0.0f;
        store8(dlo + pix * ca + cc, acc);
    }
}

// gradient at an encoder level's ReLU output e (c channels): the skip part of the decoder's
// concatenated gradient (d_cat[p][cat_off + k], row stride cat_c; may be null) plus the pooled
// branch's gradient d_pool[n][y/2][x/2][k] / 4 (may be null), times (e > 0)
__global__ void encoder_grad_kernel(const bf16* __restrict__ d_cat, int cat_c, int cat_off,
                                    const bf16* __restrict__ d_pool, const bf16* __restrict__ e,
                                    bf16* __restrict__ out, int n, int h, int w, int c) {
    const int c8 = c / 8;
    const long total = (long)n * h * w * c8;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int cc = (int)(i % c8) * 8;
        const long pix = i / c8;
        const int x = (int)(pix % w), y = (int)((pix / w) % h), b = (int)(pix / ((long)w * h));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f[8];
        if (d_cat) {
            load8(d_cat + (size_t)pix * cat_c + cat_off + cc, f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
        if (d_pool) {
            load8(d_pool + (((size_t)b * (h / 2) + y / 2) * (w / 2) + x / 2) * c + cc, f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += 0.25f * f[k];
        }
        load8(e + (size_t)pix * c + cc, f);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = f[k] > 0.0f ? acc[k] : 0.0f;
        store8(out + (size_t)pix * c + cc, acc);
    }
}

// per-block column sums of dy [P][c] (bias gradient, first pass): partial[block][c]
__global__ void bias_grad_kernel(const bf16* __restrict__ dy, float* __restrict__ partial, int P, int c) {
    extern __shared__ float red[];  // [blockDim.x / c8 groups][c]
    const int c8 = c / 8;
    const int lane_c = threadIdx.x % c8, group = threadIdx.x / c8, groups = blockDim.x / c8;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (group < groups) {
        for (long p = (long)blockIdx.x * groups + group; p < P; p += (long)gridDim.x * groups) {
            float f[8];
            load8(dy + p * c + lane_c * 8, f);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) red[group * c + lane_c * 8 + k] = acc[k];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        float s = 0.0f;
        for (int g = 0; g < groups; ++g) s += red[g * c + j];
        partial[(size_t)blockIdx.x * c + j] = s;
    }
}

// gradient of one layer into the flat fp32 gradient: g[co][t][ci] = sum_s wpart[s][t*cin+ci][co]
// (fixed order over the splits) and gb[co] = sum_b bpart[b][co]
__global__ void reduce_grads_kernel(const float* __restrict__ wpart, int splits, int m_pad, int cin, int cout,
                                    const float* __restrict__ bpart, int bblocks, float* __restrict__ gw,
                                    float* __restrict__ gb) {
    const int nw = cout * 9 * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw + cout; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        if (i < nw) {
            const int ci = i % cin, t = (i / cin) % 9, co = i / (9 * cin);
            const size_t off = (size_t)(t * cin + ci) * cout + co;
            for (int k = 0; k < splits; ++k) s += wpart[(size_t)k * m_pad * cout + off];
            gw[i] = s;
        } else {
            const int co = i - nw;
            if (bpart)
                for (int k = 0; k < bblocks; ++k) s += bpart[(size_t)k * cout + co];
            gb[co] = s;
        }
    }
}

// Adam (Kingma & Ba 2015, Algorithm 1) on the flat fp32 master parameters; the bf16 copy the
// convolutions read is written in the same pass
__global__ void adam_kernel(float* __restrict__ param, bf16* __restrict__ param_bf16, float* __restrict__ m1,
                            float* __restrict__ m2, const float* __restrict__ grad, long count, float lr, float beta1,
                            float beta2, float eps, float bias1, float bias2, float grad_scale) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        const float g = grad[i] * grad_scale;
        const float a = beta1 * m1[i] + (1.0f - beta1) * g;
        const float b = beta2 * m2[i] + (1.0f - beta2) * g * g;
        m1[i] = a;
        m2[i] = b;
        const float mhat = a / bias1, vhat = b / bias2;
        const float p = param[i] - lr * mhat / (sqrtf(vhat) + eps);
        param[i] = p;
        if (param_bf16) param_bf16[i] = __float2bfloat16_rn(p);
    }
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ in, bf16* __restrict__ out, long count) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(in[i]);
}

// ---------------------------------------------------------------------------------------------
// network input and the kernel-prediction head
// ---------------------------------------------------------------------------------------------
constexpr int kInputChannels = 16;  // 15 used: log radiance 3, albedo 3, normal 3, depth 1, transmittance 1,
                                    // noise level 1, log standard error of the pixel mean 3

// planes: [n][3][h][w] radiance (mean of the frames rendered so far), albedo [n][3][h][w], normal
// [n][3][h][w], depth [n][h][w], transmittance [n][h][w] (each may be null -> zeros); noise_level
// [n] (1 / sqrt(frames) of each image; may be null -> zeros); second_moment [n][3][h][w] (mean of the
// squared per-frame radiance; with noise_level gives log1p of the standard error of the pixel mean,
// sqrt(max(0, m2 - mean^2)) / sqrt(frames); may be null -> zeros)
__global__ void pack_input_kernel(const float* __restrict__ radiance, const float* __restrict__ albedo,
                                  const float* __restrict__ normal, const float* __restrict__ depth,
                                  const float* __restrict__ transmittance, const float* __restrict__ noise_level,
                                  const float* __restrict__ second_moment, bf16* __restrict__ out, int n, int h,
                                  int w) {
    const long plane = (long)h * w, total = (long)n * plane;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long b = i / plane, q = i % plane;
        float f[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int c = 0; c < 3; ++c) {
            const float r = radiance[(b * 3 + c) * plane + q];
            f[c] = log1pf(fmaxf(r, 0.0f));
            if (albedo) f[3 + c] = albedo[(b * 3 + c) * plane + q];
            if (normal) f[6 + c] = normal[(b * 3 + c) * plane + q];
        }
        if (depth) f[9] = depth[b * plane + q];
        if (transmittance) f[10] = transmittance[b * plane + q];
        if (noise_level) {
            f[11] = noise_level[b];
            if (second_moment)
                for (int c = 0; c < 3; ++c) {
                    const float m1 = radiance[(b * 3 + c) * plane + q];
                    const float m2 = second_moment[(b * 3 + c) * plane + q];
                    f[12 + c] = log1pf(sqrtf(fmaxf(0.0f, m2 - m1 * m1)) * noise_level[b]);
                }
        }
        float lo[8], hi[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            lo[k] = f[k];
            hi[k] = f[8 + k];
        }
        store8(out + i * kInputChannels, lo);
        store8(out + i * kInputChannels + 8, hi);
    }
}

// Per-pixel k x k kernel application with the tap softmax fused, and (target != null) the relative
// MSE loss and its gradient with respect to the logits:
//   s = softmax(logits[p][0 .. k*k-1]);  d[c][p] = sum_j s_j x[c][p + off_j]  (taps outside skipped)
//   loss = sum_{p,c} (d - t)^2 / (t^2 + eps) * inv_count
//   dL/dlogit_j = s_j (g . x_j - g . d),  g_c = 2 (d_c - t_c) / (t_c^2 + eps) * inv_count
// logits: [P][hc] fp32 (NHWC, hc >= k*k a multiple of 8, channels k*k.. unused, their gradient 0);
// x, t, out: [n][3][h][w] fp32.  The softmax is recomputed per pass (no per-tap arrays in registers).
// One block per 64-pixel row segment at a time (grid-stride): the segment's logits (contiguous in
// NHWC) are staged in shared memory by asynchronous copies, a warp per pixel row, at a row stride of
// hc + 4 floats; the KS x (64 + KS - 1) radiance window likewise, with zeros outside the image (an
// out-of-image tap adds to the normalisation only).  Four lanes per pixel take the kernel rows
// sub, sub + 4, ... (columns unrolled: window offsets are immediates) and combine by shuffles.  Bank
// spread: the logit stride is 4 (mod 8) with an odd quotient, so the warp's 8 pixels start on banks
// 0, 4, .., 28 and the lanes' rows (KS odd) add 0..3; the window row length is 8 (mod 16), so the
// lanes' window rows start 8 banks apart.  The logit gradients overwrite the staged logits and leave
// as coalesced bf16 rows.
constexpr int kHeadSeg = 64;

__host__ __device__ constexpr int head_window_row(int ks) {  // >= kHeadSeg + ks - 1, = 8 (mod 16)
    return (kHeadSeg + ks - 1 + 7) / 16 * 16 + 8;
}

__device__ __forceinline__ float quad_sum(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v + __shfl_xor_sync(0xffffffffu, v, 2);
}

template <int KS>
__global__ void __launch_bounds__(256) kpn_head_kernel(const float* __restrict__ logits, int hc,
                                                       const float* __restrict__ x, const float* __restrict__ target,
                                                       float* __restrict__ out, bf16* __restrict__ dlogits,
                                                       float* __restrict__ loss_partial, int n, int h, int w,
                                                       float eps, float inv_count) {
    constexpr int RW = head_window_row(KS), WIN = KS * RW, TAPS = KS * KS, RAD = KS / 2;
    extern __shared__ float hsm[];
    const int stride = hc + 4;
    float* lsm = hsm;                       // [kHeadSeg][stride]
    float* rsm = hsm + kHeadSeg * stride;   // [3][KS][RW]
    const long plane = (long)h * w;
    const int segs_w = (w + kHeadSeg - 1) / kHeadSeg;
    const long nseg = (long)n * h * segs_w;
    const int t = threadIdx.x, pl = t >> 2, sub = t & 3, warp = t >> 5, lane = t & 31;
    const int q4 = hc / 4;
    float local = 0.0f;
    for (long sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        const int sx = (int)(sg % segs_w);
        const long row = sg / segs_w;
        const int y = (int)(row % h);
        const long b = row / h;
        const int x0 = sx * kHeadSeg, np = min(kHeadSeg, w - x0);
        const long p0 = (b * h + y) * w + x0;
        __syncthreads();  // the previous segment is done with shared memory
        // asynchronous copies: every copy of the block is in flight before the first wait
        const float4* lg4 = reinterpret_cast<const float4*>(logits + p0 * hc);
        for (int p = warp; p < np; p += 8) {
            const float4* src = lg4 + (long)p * q4;
            const uint32_t dst = smem_u32(lsm + p * stride);
            for (int c = lane; c < q4; c += 32) cp_async16_stream(dst + 16 * c, src + c);
        }
        const float* xb = x + b * 3 * plane;
        for (int rr = warp; rr < 3 * KS; rr += 8) {  // window row rr = c * KS + r
            const int c = rr / KS, r = rr - c * KS;
            const int yy = y + r - RAD;
            const bool row_ok = yy >= 0 && yy < h;
            const float* src = xb + c * plane + (long)(row_ok ? yy : 0) * w;
            const uint32_t dst = smem_u32(rsm + rr * RW);
            for (int xx = lane; xx < kHeadSeg + KS - 1; xx += 32) {
                const int xq = x0 + xx - RAD;
                const bool v = row_ok && xq >= 0 && xq < w;
                cp_async4(dst + 4 * xx, v ? src + xq : xb, v);
            }
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        const bool pv = pl < np;
        const float* lp = lsm + pl * stride;
        const float* rp = rsm + pl;
        float mx = -INFINITY;
        if (pv)
            for (int r = sub; r < KS; r += 4) {
#pragma unroll
                for (int c = 0; c < KS; ++c) mx = fmaxf(mx, lp[r * KS + c]);
            }
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
        float sum = 0.0f, d0 = 0.0f, d1 = 0.0f, d2 = 0.0f;
        if (pv)
            for (int r = sub; r < KS; r += 4) {
                const float* lr = lp + r * KS;
                const float* xr = rp + r * RW;
#pragma unroll
                for (int c = 0; c < KS; ++c) {
                    const float e = __expf(lr[c] - mx);
                    sum += e;
                    d0 += e * xr[c];
                    d1 += e * xr[WIN + c];
                    d2 += e * xr[2 * WIN + c];
                }
            }
        sum = quad_sum(sum);
        d0 = quad_sum(d0);
        d1 = quad_sum(d1);
        d2 = quad_sum(d2);
        const float inv = 1.0f / sum;
        const float d[3] = {d0 * inv, d1 * inv, d2 * inv};
        const long q = (long)y * w + x0 + pl;
        if (pv && out && sub < 3) out[(b * 3 + sub) * plane + q] = sub == 0 ? d[0] : (sub == 1 ? d[1] : d[2]);
        if (target) {
            float g[3] = {0.0f, 0.0f, 0.0f};
            if (pv) {
                for (int c = 0; c < 3; ++c) {
                    const float tg = target[(b * 3 + c) * plane + q];
                    const float den = tg * tg + eps;
                    const float e = d[c] - tg;
                    if (sub == 0) local += e * e / den * inv_count;
                    g[c] = 2.0f * e / den * inv_count;
                }
            }
            const float gd = g[0] * d[0] + g[1] * d[1] + g[2] * d[2];
            float* lw = lsm + pl * stride;
            for (int r = sub; r < KS; r += 4) {
                float* lr = lw + r * KS;
                const float* xr = rp + r * RW;
#pragma unroll
                for (int c = 0; c < KS; ++c) {
                    const float gx = g[0] * xr[c] + g[1] * xr[WIN + c] + g[2] * xr[2 * WIN + c];
                    lr[c] = pv ? __expf(lr[c] - mx) * inv * (gx - gd) : 0.0f;
                }
            }
            for (int j = TAPS + sub; j < hc; j += 4) lw[j] = 0.0f;
            __syncthreads();
            for (int p = warp; p < np; p += 8) {
                const float* srow = lsm + p * stride;
                bf16* drow = dlogits + (p0 + p) * hc;
                for (int c = lane * 8; c < hc; c += 256) {
                    const float4 u = *reinterpret_cast<const float4*>(srow + c);
                    const float4 v = *reinterpret_cast<const float4*>(srow + c + 4);
                    const float f[8] = {u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w};
                    store8(drow + c, f);
                }
            }
        }
    }
    if (loss_partial) {
        // block reduction (fixed order)
        __shared__ float red[256];
        red[threadIdx.x] = local;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) loss_partial[blockIdx.x] = red[0];
    }
}

// ---------------------------------------------------------------------------------------------
// multi-scale reconstruction
// ---------------------------------------------------------------------------------------------
// Level l (l = 0 full resolution) has the noisy input x_l (x_{l+1} = 2x2 average of x_l), its kernel
// output d_l = apply(x_l, K_l), and the reconstruction
//     c_l = d_l + a_l * (up(c_{l+1}) - up(pool(d_l))),   a_l = sigmoid(logit_l[alpha channel])
// (the coarsest level: c = d): the low frequencies of the fine estimate are replaced, in the
// proportion a, by the coarser level's estimate.  up = nearest (each coarse pixel to its 2x2
// children), pool = 2x2 average.  Images are planar [n][3][h][w] fp32; logits NHWC [p][hc] fp32.
__device__ __forceinline__ float sigmoidf_(float v) { return 1.0f / (1.0f + __expf(-v)); }

__global__ void kpn_combine_kernel(const float* __restrict__ d, const float* __restrict__ c_coarse,
                                   const float* __restrict__ logits, int hc, int alpha_ch, float* __restrict__ c,
                                   int n, int h, int w) {
    const long plane = (long)h * w, total = (long)n * plane;
    const int hh = h / 2, wh = w / 2;
    const long cplane = (long)hh * wh;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long b = i / plane, q = i % plane;
        const int y = (int)(q / w), x = (int)(q % w);
        const int y0 = y & ~1, x0 = x & ~1;
        const float a = sigmoidf_(logits[i * hc + alpha_ch]);
        for (int ch = 0; ch < 3; ++ch) {
            const float* dp = d + (b * 3 + ch) * plane;
            const float pool = 0.25f * ((dp[(long)y0 * w + x0] + dp[(long)y0 * w + x0 + 1]) +
                                        (dp[(long)(y0 + 1) * w + x0] + dp[(long)(y0 + 1) * w + x0 + 1]));
            const float cc = c_coarse[(b * 3 + ch) * cplane + (long)(y / 2) * wh + x / 2];
            c[(b * 3 + ch) * plane + q] = dp[q] + a * (cc - pool);
        }
    }
}

// Backward of one level.  g = dL/dc_l is read from g_in, or (level 0, target != null) computed here
// from the relative-MSE loss of c = c_l against the target (whose partial sums go to loss_partial).
// With a blend (alpha_ch >= 0): dL/dd = g - pool^T(up^T(a g)) (each pixel minus a quarter of its
// 2x2 family's sum of a g), dL/dc_{l+1} = up^T(a g) (written by the family's first pixel),
// dL/dlogit_alpha = a (1 - a) g . (up(c_{l+1}) - up(pool(d))); without: dL/dd = g.  Then the kernel
// application's gradient dL/dlogit_j = s_j (gd . x_j - gd . d) (taps outside skipped), all written
// to dlogits [p][hc] bf16 (0 in unused channels).
__global__ void kpn_level_grad_kernel(const float* __restrict__ logits, int hc, int ks, int alpha_ch,
                                      const float* __restrict__ x, const float* __restrict__ d,
                                      const float* __restrict__ c_coarse, const float* __restrict__ g_in,
                                      const float* __restrict__ c_out, const float* __restrict__ target, float eps,
                                      float inv_count, bf16* __restrict__ dlogits, float* __restrict__ g_coarse,
                                      float* __restrict__ loss_partial, int n, int h, int w) {
    const long plane = (long)h * w, total = (long)n * plane;
    const int taps = ks * ks, rad = ks / 2;
    const int hh = h / 2, wh = w / 2;
    const long cplane = (long)hh * wh;
    float local = 0.0f;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long b = i / plane, q = i % plane;
        const int y = (int)(q / w), xx = (int)(q % w);
        // gradient at c for a pixel of this image
        auto g_at = [&](long qq, int ch) -> float {
            if (target) {
                const float t = target[(b * 3 + ch) * plane + qq];
                return 2.0f * (c_out[(b * 3 + ch) * plane + qq] - t) / (t * t + eps) * inv_count;
            }
            return g_in[(b * 3 + ch) * plane + qq];
        };
        float g[3], gd[3];
        for (int ch = 0; ch < 3; ++ch) g[ch] = g_at(q, ch);
        if (target) {
            for (int ch = 0; ch < 3; ++ch) {
                const float t = target[(b * 3 + ch) * plane + q];
                const float e = c_out[(b * 3 + ch) * plane + q] - t;
                local += e * e / (t * t + eps) * inv_count;
            }
        }
        float dalpha = 0.0f;
        bool has_alpha = alpha_ch >= 0;
        if (has_alpha) {
            const int y0 = y & ~1, x0 = xx & ~1;
            const long fam[4] = {(long)y0 * w + x0, (long)y0 * w + x0 + 1, (long)(y0 + 1) * w + x0,
                                 (long)(y0 + 1) * w + x0 + 1};
            const long base = i - q;  // first pixel of this image in NHWC order
            float sag[3] = {0.0f, 0.0f, 0.0f};
            for (int k = 0; k < 4; ++k) {
                const float ak = sigmoidf_(logits[(base + fam[k]) * hc + alpha_ch]);
                for (int ch = 0; ch < 3; ++ch) sag[ch] += ak * g_at(fam[k], ch);
            }
            const float a = sigmoidf_(logits[i * hc + alpha_ch]);
            const long parent = (long)(y / 2) * wh + xx / 2;
            for (int ch = 0; ch < 3; ++ch) {
                gd[ch] = g[ch] - 0.25f * sag[ch];
                const float* dp = d + (b * 3 + ch) * plane;
                const float pool = 0.25f * ((dp[fam[0]] + dp[fam[1]]) + (dp[fam[2]] + dp[fam[3]]));
                dalpha += g[ch] * (c_coarse[(b * 3 + ch) * cplane + parent] - pool);
            }
            dalpha *= a * (1.0f - a);
            if (g_coarse && (y & 1) == 0 && (xx & 1) == 0)
                for (int ch = 0; ch < 3; ++ch) g_coarse[(b * 3 + ch) * cplane + parent] = sag[ch];
        } else {
            for (int ch = 0; ch < 3; ++ch) gd[ch] = g[ch];
        }
        // kernel application backward
        const float* lg = logits + i * hc;
        float mx = -INFINITY;
        for (int j = 0; j < taps; ++j) mx = fmaxf(mx, lg[j]);
        float sum = 0.0f;
        for (int j = 0; j < taps; ++j) sum += __expf(lg[j] - mx);
        const float inv = 1.0f / sum;
        const float* xb = x + b * 3 * plane;
        const float gdd = gd[0] * d[(b * 3 + 0) * plane + q] + gd[1] * d[(b * 3 + 1) * plane + q] +
                          gd[2] * d[(b * 3 + 2) * plane + q];
        for (int j0 = 0; j0 < hc; j0 += 8) {
            float f[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = j0 + k;
                f[k] = 0.0f;
                if (j < taps) {
                    const float sj = __expf(lg[j] - mx) * inv;
                    const int yy = y + j / ks - rad, xq = xx + j % ks - rad;
                    float gx = 0.0f;
                    if (yy >= 0 && yy < h && xq >= 0 && xq < w) {
                        const long o = (long)yy * w + xq;
                        gx = gd[0] * xb[o] + gd[1] * xb[plane + o] + gd[2] * xb[2 * plane + o];
                    }
                    f[k] = sj * (gx - gdd);
                } else if (j == alpha_ch) {
                    f[k] = dalpha;
                }
            }
            store8(dlogits + i * hc + j0, f);
        }
    }
    if (loss_partial) {
        __shared__ float red[256];
        red[threadIdx.x] = local;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) loss_partial[blockIdx.x] = red[0];
    }
}

// out = a + b (bf16, count a multiple of 8)
__global__ void add_bf16_kernel(const bf16* __restrict__ a, const bf16* __restrict__ b, bf16* __restrict__ out,
                                long count8) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count8; i += (long)gridDim.x * blockDim.x) {
        float fa[8], fb[8];
        load8(a + i * 8, fa);
        load8(b + i * 8, fb);
#pragma unroll
        for (int k = 0; k < 8; ++k) fa[k] += fb[k];
        store8(out + i * 8, fa);
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
inline int grid_for(long work, int threads) {
    long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148L * 16) b = 148L * 16;
    return (int)b;
}

inline int pow2_cols(int n) {
    int c = 32;
    while (c < n) c <<= 1;
    return c;
}

template <int MODE, int STAGES>
cudaError_t launch_tile_n(const ConvArgs& a, dim3 grid, cudaStream_t s) {
    const size_t smem = (size_t)STAGES * (kBM * kBK * 2 + (size_t)a.n_tile * kBK * 2);
    cudaError_t e = cudaFuncSetAttribute(conv_tile_kernel<MODE, STAGES>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    conv_tile_kernel<MODE, STAGES><<<grid, kThreads, smem, s>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

static int g_gather_stages = 0;  // 0: 3 stages, except 4 for 64-column convolution tiles (measured)

template <int MODE>
cudaError_t launch_tile(const ConvArgs& a, dim3 grid, cudaStream_t s) {
    int st = g_gather_stages;
    if (st == 0) st = (MODE == kConv && a.n_tile == 64) ? 4 : 3;
    return st == 3 ? launch_tile_n<MODE, 3>(a, grid, s) : launch_tile_n<MODE, 4>(a, grid, s);
}

inline bool chan_ok(int c) { return c > 0 && c % 16 == 0; }

inline int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

constexpr size_t kStripSmemLimit = 200 * 1024;

inline size_t strip_smem_bytes(int cin, int cout) {
    return ((9ul * cin * cout * 2 + 127) & ~(size_t)127) + (size_t)kRing * (cin / 8) * kPlane;
}

// the row-strip kernel serves images at least one tile wide with at most 256 output channels; the
// input channels are split into groups whose weights and ring fit in shared memory (one pass each,
// summed through an fp32 partial)
inline int strip_groups(int width, int cin, int cout, bool any = false) {
    if (width < kBM || cout > 256) return 0;
    for (int g = 1; g <= 4; ++g) {
        const int cg = (cin / 16 + g - 1) / g * 16;
        // grouped passes re-stream an fp32 partial; they beat the gather kernel only for narrow
        // outputs (measured: 176 -> 32 faster, 160 -> 64 slower)
        if (strip_smem_bytes(cg, cout) <= kStripSmemLimit) return (g == 1 || cout <= 32 || any) ? g : 0;
    }
    return 0;
}

// Weight-gradient plan on row strips: the role (which tensor is A), the A channel chunks of at most
// 128 (M = 64 or 128), tap groups so that taps x N <= 512 TMEM columns, and the shared memory of the
// largest pass; 0 passes = not eligible (the gather kernel serves it).
struct WgradPlan {
    int role = 0, chunks = 0, taps_per = 9, groups = 1, passes = 0;
    size_t smem = 0;
};

constexpr size_t kWgradSmemLimit = 220 * 1024;

inline WgradPlan wgrad_plan(int width, int cin, int cout, bool any_width = false) {
    WgradPlan best;
    if (width < kBM) return best;
    // with fewer than 64 channels on both sides the per-row MMAs are too small (M = 64, N = 32) to
    // beat the gather kernel (measured); any_width lifts the rule
    if (!any_width && cin < 64 && cout < 64) return best;
    for (int role = 0; role < 2; ++role) {
        const int mtot = role == 0 ? cin : cout, N = role == 0 ? cout : cin;
        if (N > 256) continue;
        WgradPlan p;
        p.role = role;
        p.chunks = (mtot + 127) / 128;
        const int ma = mtot > 64 ? 128 : 64;  // largest chunk
        p.taps_per = min(9, 512 / N);
        p.groups = (9 + p.taps_per - 1) / p.taps_per;
        p.passes = p.chunks * p.groups;
        const int xplanes = role == 0 ? ma / 8 : cin / 8, dyplanes = role == 0 ? cout / 8 : ma / 8;
        p.smem = (size_t)kRing * xplanes * kPlane + (size_t)kDyRing * dyplanes * kDyPlane;
        if (p.smem > kWgradSmemLimit) continue;
        if (best.passes == 0 || p.passes < best.passes) best = p;
    }
    return best;
}

inline void strip_segments(int n, int h, int w, int slots, int& xtiles, int& seg_rows, int& segs_per_col,
                           int& total) {
    xtiles = (w + kBM - 1) / kBM;
    const int cols = n * xtiles;
    const int want = max(cols, 2 * slots);
    int spc = (want + cols - 1) / cols;
    spc = min(spc, max(1, h / 4));
    seg_rows = (h + spc - 1) / spc;
    segs_per_col = (h + seg_rows - 1) / seg_rows;
    total = cols * segs_per_col;
}

inline int wgrad_strip_grid(int n, int h, int w) {
    int xt, sr, spc, total;
    strip_segments(n, h, w, sm_count(), xt, sr, spc, total);
    return min(total, sm_count());
}

cudaError_t launch_wgrad_strip(const bf16* x, const bf16* dy, float* partial, int* err, int n, int h, int w, int cin,
                               int cout, const WgradPlan& plan, cudaStream_t s) {
    WgradStripArgs a{};
    a.x = x;
    a.dy = dy;
    a.partial = partial;
    a.err = err;
    a.n = n;
    a.h = h;
    a.w_ = w;
    a.cin = cin;
    a.cout = cout;
    a.m_pad = (9 * cin + kBM - 1) / kBM * kBM;
    const int slots = sm_count();
    int total = 0;
    strip_segments(n, h, w, slots, a.xtiles, a.seg_rows, a.segs_per_col, total);
    const int grid = min(total, slots);
    const int mtot = plan.role == 0 ? cin : cout, N = plan.role == 0 ? cout : cin;
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < plan.chunks && e == cudaSuccess; ++c) {
        a.m0 = c * 128;
        a.ma = (mtot - a.m0) > 64 ? 128 : 64;
        a.xplanes = plan.role == 0 ? a.ma / 8 : cin / 8;
        a.dyplanes = plan.role == 0 ? cout / 8 : a.ma / 8;
        const size_t smem = (size_t)kRing * a.xplanes * kPlane + (size_t)kDyRing * a.dyplanes * kDyPlane;
        for (int gidx = 0; gidx < plan.groups && e == cudaSuccess; ++gidx) {
            a.t0 = gidx * plan.taps_per;
            a.t1 = min(9, a.t0 + plan.taps_per);
            a.tmem_cols = pow2_cols((a.t1 - a.t0) * N);
            if (plan.role == 0) {
                e = cudaFuncSetAttribute(wgrad_strip_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e == cudaSuccess) wgrad_strip_kernel<0><<<grid, kThreads, smem, s>>>(a);
            } else {
                e = cudaFuncSetAttribute(wgrad_strip_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e == cudaSuccess) wgrad_strip_kernel<1><<<grid, kThreads, smem, s>>>(a);
            }
            count_launches(1);
            if (e == cudaSuccess) e = cudaGetLastError();
        }
    }
    return e;
}

cudaError_t launch_strip_pass(StripArgs a, cudaStream_t s) {
    a.xtiles = (a.w_ + kBM - 1) / kBM;
    a.tmem_cols = pow2_cols(2 * a.cout);
    const size_t smem = strip_smem_bytes(a.cin, a.cout);
    int per_sm = (int)(220 * 1024 / smem);
    per_sm = per_sm < 1 ? 1 : per_sm;
    per_sm = min(per_sm, 512 / a.tmem_cols);
    const int slots = sm_count() * per_sm;
    const int cols = a.n * a.xtiles;
    const int want = max(cols, 2 * slots);
    int spc = (want + cols - 1) / cols;
    spc = min(spc, max(1, a.h / 4));  // segments of at least 4 rows (2 halo rows per segment)
    a.seg_rows = (a.h + spc - 1) / spc;
    a.segs_per_col = (a.h + a.seg_rows - 1) / a.seg_rows;
    const int total = cols * a.segs_per_col;
    const int grid = min(total, slots);
    cudaError_t e = cudaFuncSetAttribute(conv_strip_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    conv_strip_kernel<<<grid, kThreads, smem, s>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

// ---- the warp-specialised strip kernel ----
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// NHWC bf16 activation [n][h][w][c] as a 4-D tensor (c, w, h, n) with boxes of `width` channels x
// 130 pixels, swizzled for lines of 2 * width bytes (the channel coordinate of every load is a
// multiple of 16 channels, i.e. 32 bytes)
bool encode_rows(CUtensorMap* map, const bf16* x, int n, int h, int w, int c, int width) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn || reinterpret_cast<uintptr_t>(x) % 16) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2, (cuuint64_t)h * w * c * 2};
    const cuuint32_t box[4] = {(cuuint32_t)width, (cuuint32_t)kStripPix, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapSwizzle sz = width == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                              : (width == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(x), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, sz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr size_t kSmPerSm = 233472;   // shared memory of one SM (bytes)
constexpr size_t kSmPerCta = 232448;  // largest dynamic shared memory of one CTA
constexpr size_t kWsStatic = 2048;    // static shared memory + the per-CTA reservation, rounded up

// a pass's channels as groups of 64, then 32, then 16 (each a 1024-byte aligned buffer of 130 lines)
struct WsGroups {
    int n = 0, c[kWsMaxGroups] = {}, w[kWsMaxGroups] = {}, off[kWsMaxGroups] = {}, row_bytes = 0, tx = 0;
};
inline WsGroups ws_groups_of(int cin) {
    WsGroups g;
    int c = 0, off = 0;
    while (c < cin && g.n < kWsMaxGroups) {
        const int rem = cin - c, width = rem >= 64 ? 64 : (rem >= 32 ? 32 : 16);
        g.c[g.n] = c;
        g.w[g.n] = width;
        g.off[g.n] = off;
        off += (kStripPix * width * 2 + 1023) / 1024 * 1024;
        g.tx += kStripPix * width * 2;
        c += width;
        ++g.n;
    }
    g.row_bytes = c == cin ? off : 0;  // 0: more groups than supported
    return g;
}

inline size_t ws_weight_bytes(int cin, int cout) { return (9ul * cin * cout * 2 + 1023) & ~(size_t)1023; }
inline size_t ws_row_bytes(int cin) { return (size_t)ws_groups_of(cin).row_bytes; }

// CTAs per SM and ring depth: the most rows in flight per SM (CTAs x (ring - 3)), then more CTAs;
// TMEM holds two accumulators per CTA.  false when not even one CTA with a 4-slot ring fits.
bool ws_config(int cin, int cout, int& per_sm, int& ring) {
    const int acc = pow2_cols(cout);
    const size_t rb = ws_row_bytes(cin);
    per_sm = 0;
    ring = 0;
    if (rb == 0) return false;
    int best = -1;
    for (int occ = 1; occ <= 2 && occ * 2 * acc <= 512; ++occ) {  // 2: the registers of 2 CTAs fit an SM
        const size_t budget = kSmPerSm / occ - kWsStatic;
        const size_t wb = ws_weight_bytes(cin, cout);
        if (budget > kSmPerCta || wb >= budget) continue;
        const int r = (int)std::min<size_t>(kWsMaxRing, (budget - wb) / rb);
        if (r < 4) continue;
        const int score = occ * (r - 3);
        if (score > best || (score == best && occ > per_sm)) {
            best = score;
            per_sm = occ;
            ring = r;
        }
    }
    return per_sm > 0;
}

// input-channel passes for the warp-specialised kernel (0 = not eligible).  Several passes re-stream
// an fp32 partial: measured faster than the gather kernel for up to 64 output channels (176 -> 32,
// 160 -> 64), slower for 96 -> 96 and 224 -> 96.
inline int ws_groups(int width, int cin, int cout, bool any = false) {
    if (width < kBM || cout > 256) return 0;
    for (int g = 1; g <= 4; ++g) {
        const int cg = (cin / 16 + g - 1) / g * 16;
        int occ, ring;
        if (ws_config(cg, cout, occ, ring)) return (g == 1 || cout <= 64 || any) ? g : 0;
    }
    return 0;
}

cudaError_t launch_ws_pass(StripArgs a, cudaStream_t s) {
    int per_sm = 0, ring = 0;
    if (!ws_config(a.cin, a.cout, per_sm, ring)) return cudaErrorInvalidValue;
    WsArgs wa{};
    const WsGroups gr = ws_groups_of(a.cin);
    CUtensorMap maps[3];  // widths 64, 32, 16
    memset(maps, 0, sizeof(maps));
    bool have[3] = {false, false, false};
    for (int k = 0; k < gr.n; ++k) {
        const int mi = gr.w[k] == 64 ? 0 : (gr.w[k] == 32 ? 1 : 2);
        if (!have[mi] && !encode_rows(&maps[mi], a.x, a.n, a.h, a.w_, a.cin_total, gr.w[k]))
            return cudaErrorInvalidValue;
        have[mi] = true;
        wa.gc[k] = gr.c[k];
        wa.gw[k] = gr.w[k];
        wa.goff[k] = gr.off[k];
    }
    wa.ngroups = gr.n;
    wa.row_bytes = gr.row_bytes;
    wa.tx_bytes = gr.tx;
    a.tmem_cols = 2 * pow2_cols(a.cout);
    const int slots = sm_count() * per_sm;
    int total = 0;
    strip_segments(a.n, a.h, a.w_, slots, a.xtiles, a.seg_rows, a.segs_per_col, total);
    const int grid = min(total, slots);
    wa.s = a;
    // at least the shared memory that holds the CTAs per SM to per_sm (TMEM is sized for that many)
    const size_t need = ws_weight_bytes(a.cin, a.cout) + (size_t)ring * ws_row_bytes(a.cin);
    const size_t smem = std::max(need, std::min(kSmPerCta, kSmPerSm / (per_sm + 1) - kWsStatic + 1024));
    cudaError_t e = cudaFuncSetAttribute(conv_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    conv_ws_kernel<<<grid, kWsThreads, smem, s>>>(maps[0], maps[1], maps[2], wa, ring);
    count_launches(1);
    return cudaGetLastError();
}

static int g_strip_kernel = 0;  // 0: warp-specialised (TMA) strips, 1: the cp.async strip kernel

cudaError_t launch_strip(const ConvArgs& c, int groups, cudaStream_t s) {
    StripArgs a{};
    a.x = c.x;
    a.w = c.w;
    a.err = c.err;
    a.n = c.n;
    a.h = c.h;
    a.w_ = c.w_;
    a.cout = c.cout;
    a.cin_total = c.cin;
    if (groups <= 1) {
        a.cin = c.cin;
        a.bias = c.bias;
        a.mask = c.mask;
        a.y = c.y;
        a.relu = c.relu;
        a.out_f32 = c.out_f32;
        return g_strip_kernel == 0 ? launch_ws_pass(a, s) : launch_strip_pass(a, s);
    }
    // fp32 partial sum of the earlier groups (stream-ordered scratch)
    float* part = nullptr;
    const size_t bytes = (size_t)c.n * c.h * c.w_ * c.cout * sizeof(float);
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&part), bytes, s);
    if (e != cudaSuccess) return e;
    const int cg = (c.cin / 16 + groups - 1) / groups * 16;
    for (int g = 0, c0 = 0; c0 < c.cin && e == cudaSuccess; ++g, c0 += cg) {
        const bool last = c0 + cg >= c.cin;
        StripArgs p = a;
        p.c0 = c0;
        p.cin = min(cg, c.cin - c0);
        p.part_in = g > 0 ? part : nullptr;
        p.part_out = last ? nullptr : part;
        if (last) {
            p.bias = c.bias;
            p.mask = c.mask;
            p.y = c.y;
            p.relu = c.relu;
            p.out_f32 = c.out_f32;
        }
        e = g_strip_kernel == 0 ? launch_ws_pass(p, s) : launch_strip_pass(p, s);
    }
    const cudaError_t f = cudaFreeAsync(part, s);
    return e != cudaSuccess ? e : f;
}

}  // namespace unet
}  // namespace vpt

using namespace vpt::unet;

static bool g_force_gather = false;  // conv path 1: the gather kernels everywhere
static bool g_force_strip = false;   // conv path 2: the strip kernels wherever they apply
static int g_conv_ksplit = 0;        // gather convolution K splits: 0 automatic, 1 none, k > 1 forced

extern "C" {

VptStatus vpt_unet_conv3x3(const void* x, const void* w, const float* bias, const void* mask, void* y, int n, int h,
                           int width, int cin, int cout, int relu, int out_f32, int* err, void* stream) {
    if (!x || !w || !y || n <= 0 || h <= 0 || width <= 0 || !chan_ok(cin) || !chan_ok(cout) || cout > 4096 ||
        (long)n * h * width > (1L << 30))
        return VPT_ERR_ARG;
    ConvArgs a{};
    a.x = static_cast<const bf16*>(x);
    a.w = static_cast<const bf16*>(w);
    a.bias = bias;
    a.mask = static_cast<const bf16*>(mask);
    a.y = y;
    a.err = err;
    a.n = n;
    a.h = h;
    a.w_ = width;
    a.cin = cin;
    a.cout = cout;
    const int ntiles = (cout + 255) / 256;
    a.n_tile = ((cout + ntiles - 1) / ntiles + 15) / 16 * 16;
    a.tmem_cols = pow2_cols(a.n_tile);
    a.relu = relu;
    a.out_f32 = out_f32;
    // row strips: the warp-specialised kernel's tensor map wants a 16-byte aligned base
    const bool aligned = reinterpret_cast<uintptr_t>(x) % 16 == 0;
    const int groups = g_strip_kernel == 0 ? (aligned ? ws_groups(width, cin, cout, g_force_strip) : 0)
                                           : strip_groups(width, cin, cout, g_force_strip);
    if (groups > 0 && !g_force_gather)
        return launch_strip(a, groups, static_cast<cudaStream_t>(stream)) == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
    const long P = (long)n * h * width;
    const unsigned gx = (unsigned)((P + kBM - 1) / kBM), gy = (unsigned)((cout + a.n_tile - 1) / a.n_tile);
    // small grids (the deep levels): split the K stages over more CTAs, raw fp32 sums finished by
    // conv_finalize_kernel in a fixed order
    const int nk = (9 * cin + kBK - 1) / kBK;
    const int sms = sm_count();
    const long tiles = (long)gx * gy;
    int ksplit = 1;
    if (g_conv_ksplit > 1) ksplit = std::min(g_conv_ksplit, nk);
    else if (g_conv_ksplit == 0 && 2 * tiles <= sms)  // under half a wave: about two CTAs per SM (measured)
        ksplit = (int)std::max<long>(1, std::min<long>(std::min<long>(8, (2L * sms + tiles - 1) / tiles), nk / 2));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (ksplit == 1)
        return launch_tile<kConv>(a, dim3(gx, gy, 1), s) == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
    float* part = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&part), (size_t)ksplit * P * cout * sizeof(float), s) != cudaSuccess)
        return VPT_ERR_OOM;
    a.ksplit = ksplit;
    a.partial = part;
    cudaError_t e = launch_tile<kConv>(a, dim3(gx, gy, (unsigned)ksplit), s);
    if (e == cudaSuccess) {
        conv_finalize_kernel<<<grid_for(P * (cout / 4), 256), 256, 0, s>>>(part, ksplit, P, cout, bias,
                                                                          static_cast<const bf16*>(mask), relu,
                                                                          out_f32, y);
        e = cudaGetLastError();
    }
    const cudaError_t f = cudaFreeAsync(part, s);
    return (e == cudaSuccess && f == cudaSuccess) ? VPT_OK : VPT_ERR_CUDA;
}

// 0: the warp-specialised (TMA) row-strip kernel, 1: the cp.async row-strip kernel (comparisons)
VptStatus vpt_unet_set_strip_kernel(int kind) {
    if (kind < 0 || kind > 1) return VPT_ERR_ARG;
    g_strip_kernel = kind;
    return VPT_OK;
}

// K splits of the gather convolution: 0 chosen by grid size, 1 never split, k > 1 always k (tests)
VptStatus vpt_unet_set_conv_ksplit(int ksplit) {
    if (ksplit < 0 || ksplit > 64) return VPT_ERR_ARG;
    g_conv_ksplit = ksplit;
    return VPT_OK;
}

// 1: every convolution uses the per-tile gather kernel (for comparisons); 0: row strips where eligible
VptStatus vpt_unet_set_conv_path(int path) {
    if (path < 0 || path > 2) return VPT_ERR_ARG;
    g_force_gather = path == 1;
    g_force_strip = path == 2;
    return VPT_OK;
}

// shared-memory ring depth of the gather kernel (3 or 4; 0 = by shape)
VptStatus vpt_unet_set_gather_stages(int stages) {
    if (stages != 0 && stages != 3 && stages != 4) return VPT_ERR_ARG;
    g_gather_stages = stages;
    return VPT_OK;
}

VptStatus vpt_unet_conv3x3_wgrad(const void* x, const void* dy, float* partial, int n, int h, int width, int cin,
                                 int cout, int pixels_per_split, int* err, void* stream) {
    if (!x || !dy || !partial || n <= 0 || h <= 0 || width <= 0 || !chan_ok(cin) || !chan_ok(cout) ||
        cout > 4096 || pixels_per_split <= 0 || pixels_per_split % kBK != 0 || (long)n * h * width > (1L << 30))
        return VPT_ERR_ARG;
    ConvArgs a{};
    a.x = static_cast<const bf16*>(x);
    a.w = static_cast<const bf16*>(dy);
    a.y = partial;
    a.err = err;
    a.n = n;
    a.h = h;
    a.w_ = width;
    a.cin = cin;
    a.cout = cout;
    const int ntiles = (cout + 255) / 256;
    a.n_tile = ((cout + ntiles - 1) / ntiles + 15) / 16 * 16;
    a.tmem_cols = pow2_cols(a.n_tile);
    a.pix_per_split = pixels_per_split;
    const int mtiles = (9 * cin + kBM - 1) / kBM;
    a.m_pad = mtiles * kBM;
    const WgradPlan plan = wgrad_plan(width, cin, cout, g_force_strip);
    if (plan.passes > 0 && !g_force_gather)
        return launch_wgrad_strip(a.x, a.w, partial, err, n, h, width, cin, cout, plan,
                                  static_cast<cudaStream_t>(stream)) == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
    const long P = (long)n * h * width;
    const dim3 grid((unsigned)mtiles, (unsigned)((cout + a.n_tile - 1) / a.n_tile),
                    (unsigned)((P + pixels_per_split - 1) / pixels_per_split));
    return launch_tile<kWgrad>(a, grid, static_cast<cudaStream_t>(stream)) == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

int vpt_unet_wgrad_rows(int cin) { return (9 * cin + kBM - 1) / kBM * kBM; }

int vpt_unet_wgrad_splits(int n, int h, int width, int cin, int cout, int pixels_per_split) {
    if (n <= 0 || h <= 0 || width <= 0 || pixels_per_split <= 0) return 0;
    if (!g_force_gather && wgrad_plan(width, cin, cout, g_force_strip).passes > 0) return wgrad_strip_grid(n, h, width);
    const long P = (long)n * h * width;
    return (int)((P + pixels_per_split - 1) / pixels_per_split);
}

VptStatus vpt_unet_rotate_weights(const void* w, void* wrot, int cin, int cout, void* stream) {
    if (!w || !wrot || !chan_ok(cin) || !chan_ok(cout)) return VPT_ERR_ARG;
    rotate_weights_kernel<<<grid_for((long)cout * 9 * cin, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(w), static_cast<bf16*>(wrot), cin, cout);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_pool2(const void* in, void* out, int n, int h, int w, int c, void* stream) {
    if (!in || !out || n <= 0 || h <= 1 || w <= 1 || h % 2 || w % 2 || c <= 0 || c % 8) return VPT_ERR_ARG;
    pool2_kernel<<<grid_for((long)n * (h / 2) * (w / 2) * (c / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(in), static_cast<bf16*>(out), n, h, w, c);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_upcat(const void* lo, const void* skip, void* out, int n, int h, int w, int ca, int cs,
                         void* stream) {
    if (!lo || !skip || !out || n <= 0 || h <= 1 || w <= 1 || h % 2 || w % 2 || ca <= 0 || ca % 8 || cs <= 0 ||
        cs % 8)
        return VPT_ERR_ARG;
    upcat_kernel<<<grid_for((long)n * h * w * ((ca + cs) / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(lo), static_cast<const bf16*>(skip), static_cast<bf16*>(out), n, h, w, ca, cs);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_upcat_grad_lo(const void* d, const void* lo, void* dlo, int n, int h, int w, int ca, int cs,
                                 void* stream) {
    if (!d || !lo || !dlo || n <= 0 || h <= 1 || w <= 1 || h % 2 || w % 2 || ca <= 0 || ca % 8 || cs <= 0 ||
        cs % 8)
        return VPT_ERR_ARG;
    upcat_grad_lo_kernel<<<grid_for((long)n * (h / 2) * (w / 2) * (ca / 8), 256), 256, 0,
                           static_cast<cudaStream_t>(stream)>>>(static_cast<const bf16*>(d),
                                                                static_cast<const bf16*>(lo), static_cast<bf16*>(dlo),
                                                                n, h, w, ca, cs);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_encoder_grad(const void* d_cat, int cat_c, int cat_off, const void* d_pool, const void* e,
                                void* out, int n, int h, int w, int c, void* stream) {
    if (!e || !out || n <= 0 || h <= 0 || w <= 0 || c <= 0 || c % 8 || (d_cat && (cat_off % 8 || cat_c % 8)) ||
        (d_pool && (h % 2 || w % 2)))
        return VPT_ERR_ARG;
    encoder_grad_kernel<<<grid_for((long)n * h * w * (c / 8), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(d_cat), cat_c, cat_off, static_cast<const bf16*>(d_pool),
        static_cast<const bf16*>(e), static_cast<bf16*>(out), n, h, w, c);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_bias_grad(const void* dy, float* partial, int pixels, int c, int blocks, void* stream) {
    if (!dy || !partial || pixels <= 0 || c <= 0 || c % 8 || c > 2048 || blocks <= 0) return VPT_ERR_ARG;
    const int c8 = c / 8;
    int threads = 256 / c8 * c8;
    if (threads < c8) threads = c8;
    const size_t smem = (size_t)(threads / c8) * c * sizeof(float);
    bias_grad_kernel<<<blocks, threads, smem, static_cast<cudaStream_t>(stream)>>>(static_cast<const bf16*>(dy),
                                                                                   partial, pixels, c);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_reduce_grads(const float* wpartial, int splits, int cin, int cout, const float* bpartial,
                                int bblocks, float* grad_w, float* grad_b, void* stream) {
    if (!wpartial || !grad_w || !grad_b || splits <= 0 || !chan_ok(cin) || !chan_ok(cout) ||
        (bpartial && bblocks <= 0))
        return VPT_ERR_ARG;
    const int m_pad = (9 * cin + kBM - 1) / kBM * kBM;
    reduce_grads_kernel<<<grid_for((long)cout * 9 * cin + cout, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        wpartial, splits, m_pad, cin, cout, bpartial, bblocks, grad_w, grad_b);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_adam(float* param, void* param_bf16, float* m1, float* m2, const float* grad, long count, float lr,
                        float beta1, float beta2, float eps, int step, float grad_scale, void* stream) {
    if (!param || !m1 || !m2 || !grad || count <= 0 || step <= 0) return VPT_ERR_ARG;
    const float bias1 = 1.0f - powf(beta1, (float)step), bias2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        param, static_cast<bf16*>(param_bf16), m1, m2, grad, count, lr, beta1, beta2, eps, bias1, bias2, grad_scale);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_to_bf16(const float* in, void* out, long count, void* stream) {
    if (!in || !out || count <= 0) return VPT_ERR_ARG;
    f32_to_bf16_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        in, static_cast<bf16*>(out), count);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_pack_input(const float* radiance, const float* albedo, const float* normal, const float* depth,
                              const float* transmittance, const float* noise_level, const float* second_moment,
                              void* out, int n, int h, int w, void* stream) {
    if (!radiance || !out || n <= 0 || h <= 0 || w <= 0) return VPT_ERR_ARG;
    pack_input_kernel<<<grid_for((long)n * h * w, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        radiance, albedo, normal, depth, transmittance, noise_level, second_moment, static_cast<bf16*>(out), n, h, w);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

int vpt_unet_head_blocks(int n, int h, int w) { return grid_for((long)n * h * w, 256); }

VptStatus vpt_unet_kpn_head(const float* logits, int head_channels, int kernel_size, const float* radiance,
                            const float* target, float* out, void* dlogits, float* loss_partial, int n, int h, int w,
                            float eps, void* stream) {
    if (!logits || !radiance || n <= 0 || h <= 0 || w <= 0 || (target && !dlogits) || eps <= 0.0f ||
        kernel_size <= 0 || kernel_size % 2 == 0 || kernel_size > 15 || head_channels % 8 ||
        head_channels < kernel_size * kernel_size || head_channels > 512 || reinterpret_cast<uintptr_t>(logits) % 16)
        return VPT_ERR_ARG;
    // the loss partials are per block: as many blocks as vpt_unet_head_blocks (never more than the
    // row segments, which the blocks stride over)
    const int blocks = grid_for((long)n * h * w, 256);
    const float inv_count = 1.0f / (3.0f * (float)n * (float)h * (float)w);
    const size_t smem =
        ((size_t)kHeadSeg * (head_channels + 4) + 3 * kernel_size * head_window_row(kernel_size)) * sizeof(float);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bf16* dl = static_cast<bf16*>(dlogits);
    cudaError_t e = cudaErrorInvalidValue;
    auto go = [&](auto kernel) {
        if (smem > 48 * 1024 &&
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return cudaErrorInvalidValue;
        kernel<<<blocks, 256, smem, s>>>(logits, head_channels, radiance, target, out, dl, loss_partial, n, h, w,
                                         eps, inv_count);
        return cudaGetLastError();
    };
    switch (kernel_size) {
        case 1: e = go(kpn_head_kernel<1>); break;
        case 3: e = go(kpn_head_kernel<3>); break;
        case 5: e = go(kpn_head_kernel<5>); break;
        case 7: e = go(kpn_head_kernel<7>); break;
        case 9: e = go(kpn_head_kernel<9>); break;
        case 11: e = go(kpn_head_kernel<11>); break;
        case 13: e = go(kpn_head_kernel<13>); break;
        case 15: e = go(kpn_head_kernel<15>); break;
        default: return VPT_ERR_ARG;
    }
    if (e != cudaSuccess) return VPT_ERR_CUDA;
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_kpn_combine(const float* d, const float* c_coarse, const float* logits, int head_channels,
                               int alpha_channel, float* c, int n, int h, int w, void* stream) {
    if (!d || !c_coarse || !logits || !c || n <= 0 || h <= 1 || w <= 1 || h % 2 || w % 2 || alpha_channel < 0 ||
        alpha_channel >= head_channels)
        return VPT_ERR_ARG;
    kpn_combine_kernel<<<grid_for((long)n * h * w, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d, c_coarse, logits, head_channels, alpha_channel, c, n, h, w);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_kpn_level_grad(const float* logits, int head_channels, int kernel_size, int alpha_channel,
                                  const float* x, const float* d, const float* c_coarse, const float* g_in,
                                  const float* c_out, const float* target, float eps, void* dlogits, float* g_coarse,
                                  float* loss_partial, int n, int h, int w, void* stream) {
    if (!logits || !x || !d || !dlogits || n <= 0 || h <= 0 || w <= 0 || kernel_size <= 0 || kernel_size % 2 == 0 ||
        kernel_size > 15 || head_channels % 8 || head_channels < kernel_size * kernel_size ||
        (alpha_channel >= 0 && (alpha_channel < kernel_size * kernel_size || alpha_channel >= head_channels ||
                                !c_coarse || h % 2 || w % 2)) ||
        (target ? !c_out : !g_in) || eps <= 0.0f || (loss_partial && !target))
        return VPT_ERR_ARG;
    const float inv_count = 1.0f / (3.0f * (float)n * (float)h * (float)w);
    kpn_level_grad_kernel<<<grid_for((long)n * h * w, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        logits, head_channels, kernel_size, alpha_channel, x, d, c_coarse, g_in, c_out, target, eps, inv_count,
        static_cast<bf16*>(dlogits), g_coarse, loss_partial, n, h, w);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

VptStatus vpt_unet_add(const void* a, const void* b, void* out, long count, void* stream) {
    if (!a || !b || !out || count <= 0 || count % 8) return VPT_ERR_ARG;
    add_bf16_kernel<<<grid_for(count / 8, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(a), static_cast<const bf16*>(b), static_cast<bf16*>(out), count / 8);
    vpt::count_launches(1);
    return cudaGetLastError() == cudaSuccess ? VPT_OK : VPT_ERR_CUDA;
}

}  // extern "C"
