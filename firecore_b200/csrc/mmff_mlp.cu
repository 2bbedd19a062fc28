// mmff_mlp.cu -- learned warm-start proposal for the batched relaxer.
//
// Per-atom descriptors (CUDA cores), a 80(68) -> 128 -> 128 -> 16(3) SiLU MLP
// whose forward and backward products run on the 5th-generation tensor cores
// (tcgen05.mma kind::f16, BF16 operands in shared memory, FP32 accumulators in
// tensor memory), AdamW, and the energy-gated warm-start step.  FireCore has no
// learned component; the network is this project's addition, checked against
// the FP64 restatement in oracle/mlp_oracle.py.
//
// Network kernel: one CTA of 256 threads per SM, persistent over 128-atom
// tiles.  Warps w and w + 4 share TMEM lanes 32 (w % 4) .. + 31 (tile rows)
// and split the columns of every epilogue in halves.  Per tile, all operands stay on chip:
//   Z1 = X W1^T -> H1 = silu(Z1 + b1)                     (TMEM cols 0..127)
//   Z2 = H1 W2^T -> H2 = silu(.), S2 = silu'(.)           (cols 128..255)
//   Y  = H2 W3^T -> dY = 2 (Y + b3 - T) / B
//   dW3^T += H2^T dY ; dH2 = dY W3 -> dZ2 = dH2 * S2
//   dW2 += dZ2^T H1 ; db2 += dZ2^T 1 ; dH1 = dZ2 W2 -> dZ1 = dH1 * silu'(Z1)
//   dW1 += dZ1^T X  ; db1 += dZ1^T 1
// Weight gradients accumulate in TMEM columns 256..511 over all tiles of the
// CTA and are stored once at the end as this CTA's partial sums; a second
// kernel adds the partials of all CTAs in a fixed order (no atomics).  Shared-memory layout
// and the descriptor of every product: mmff_umma.h.  Inference runs the first
// three products only.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "MMFFmulti_lib.h"
#include "mmff_device.cuh"
#include "mmff_host.h"
#include "mmff_umma.h"
#include "mmff_world.h"

namespace mmff {
namespace mlp {

// ------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait on an mbarrier phase (limit in SM clocks: 2^31, about a second,
// in normal launches); false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
    }
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tm_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    // the registers are defined only after wait::ld; tie them to it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float silu_f(float z) { return z / (1.f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
    const float s = 1.f / (1.f + expf(-z));
    return s * fmaf(z, 1.f - s, 1.f);
}
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }
__device__ __forceinline__ float bf_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// 16 values -> row r, columns c..c+15 of a core-matrix tile of row length K (2 x 16 B)
__device__ __forceinline__ void st_row16(uint8_t* base, int r, int c, int K, const float* v) {
    const uint4 a = make_uint4(pack_bf2(v[0], v[1]), pack_bf2(v[2], v[3]), pack_bf2(v[4], v[5]), pack_bf2(v[6], v[7]));
    const uint4 b = make_uint4(pack_bf2(v[8], v[9]), pack_bf2(v[10], v[11]), pack_bf2(v[12], v[13]), pack_bf2(v[14], v[15]));
    *reinterpret_cast<uint4*>(base + cm_off(r, c, K)) = a;
    *reinterpret_cast<uint4*>(base + cm_off(r, c + 8, K)) = b;
}
__device__ __forceinline__ void ld_row16(const uint8_t* base, int r, int c, int K, float* v) {
    const uint4 a = *reinterpret_cast<const uint4*>(base + cm_off(r, c, K));
    const uint4 b = *reinterpret_cast<const uint4*>(base + cm_off(r, c + 8, K));
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int j = 0; j < 8; j++) { v[2 * j] = bf_lo(w[j]); v[2 * j + 1] = bf_hi(w[j]); }
}

// issue one product chain (single thread)
__device__ __forceinline__ void issue(uint32_t sb, uint32_t tbase, int op, bool acc_prev) {
    const MmaOp o = mma_op(op);
    const uint32_t idesc = instr_desc(o.N, o.a_mn, o.b_mn);
    for (int k = 0; k < o.nk; k++) {
        const uint64_t a = smem_desc(sb + o.a_off + k * o.a_step, o.a_lbo, o.a_sbo);
        const uint64_t b = smem_desc(sb + o.b_off + k * o.b_step, o.b_lbo, o.b_sbo);
        tc_mma(tbase + o.dcol, a, b, idesc, (k > 0 || acc_prev) ? 1u : 0u);
    }
}

// flat parameter vector: W1 [128x80] b1 [128] W2 [128x128] b2 [128] W3 [16x128] b3 [16]
constexpr int P_W1 = 0, P_B1 = P_W1 + HID * K0, P_W2 = P_B1 + HID, P_B2 = P_W2 + HID * HID, P_W3 = P_B2 + HID,
              P_B3 = P_W3 + NOP * HID, P_TOTAL = P_B3 + NOP;
// packed bf16 weight image: W1 | W2 | W3, laid out exactly as in shared memory
constexpr int WP_W1 = 0, WP_W2 = HID * K0 * 2, WP_W3 = WP_W2 + HID * HID * 2, WP_BYTES = WP_W3 + NOP * HID * 2;
static_assert(SM_W2 - SM_W1 == WP_W2 && SM_W3 - SM_W1 == WP_W3, "weight image must match the smem map");
static_assert(P_W1 % 4 == 0 && P_W2 % 4 == 0 && K0 % 4 == 0 && HID % 4 == 0 && P_TOTAL % 4 == 0,
              "16-byte gradient stores need 16-byte aligned rows");

struct NetArgs {
    const uint4* X;          // packed input tiles [ntile][128 x 80 bf16]
    const float4* T;         // targets (x, y, z, weight) [ntile*128]; training only
    const uint4* Wp;         // packed bf16 weights
    const float* prm;        // flat FP32 parameters (biases read from here)
    float* gpart;            // training: per-CTA gradient sums [gridDim.x][P_TOTAL]
    double* lpart;           // training: per-CTA loss sums [gridDim.x]
    float4* out;             // inference: network output (3 comps, scaled) per row
    int* err;
    int ntile, nrows;
    float inv_batch, out_scale;
    long long wait_limit;    // SM clocks per completion wait before the CTA gives up
    int no_issue;            // wait test only: issue no product and no commit, so the first wait runs out
};

constexpr int NET_THREADS = 256;

template <bool TRAIN>
__global__ void __launch_bounds__(NET_THREADS, 1) mlp_kernel(NetArgs A) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sb = smem_u32(sm);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int r = 32 * (warp & 3) + (tid & 31);   // tile row = TMEM lane of this thread
    const int half = warp >> 2;                   // which half of the columns
    float* sbias = reinterpret_cast<float*>(sm + SM_BIAS);
    const uint32_t bar = sb + SM_MISC;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SM_MISC + 8);

    {   // weights, ones and biases into shared memory
        uint4* dst = reinterpret_cast<uint4*>(sm + SM_W1);
        for (int i = tid; i < WP_BYTES / 16; i += NET_THREADS) dst[i] = A.Wp[i];
        uint4* one = reinterpret_cast<uint4*>(sm + SM_ONE);
        for (int i = tid; i < NOP * TILE * 2 / 16; i += NET_THREADS) one[i] = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
        for (int i = tid; i < HID; i += NET_THREADS) { sbias[i] = A.prm[P_B1 + i]; sbias[HID + i] = A.prm[P_B2 + i]; }
        if (tid < NOP) sbias[2 * HID + tid] = A.prm[P_B3 + tid];
    }
    if (tid == 0) mbar_init(bar, 1);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tbase = *tslot;
    const uint32_t trow = tbase + ((uint32_t)(32 * (warp & 3)) << 16);   // this warp's 32 TMEM lanes
    const int c0 = half * (HID / 2), c1 = c0 + HID / 2;                   // this thread's epilogue columns

    uint32_t phase = 0;
    bool failed = false;
    int done = 0;
    float lsum = 0.f, db3[NOUT] = {0.f, 0.f, 0.f};

    // commit the issued chain and wait for it with every thread; uniform failure
    auto complete = [&]() -> bool {
        if (tid == 0 && !A.no_issue) tc_commit(bar);
        const bool ok = mbar_wait(bar, phase, A.wait_limit);
        phase ^= 1u;
        const int bad = __syncthreads_or(!ok);
        tc_after();
        return bad == 0;
    };
    // shared-memory writes and TMEM reads of all threads done before the next product
    auto sync_for_mma = [&]() {
        fence_async_smem();
        tc_before();
        __syncthreads();
        tc_after();
    };

    float v[16], w[16];
    for (int tile = blockIdx.x; tile < A.ntile; tile += gridDim.x) {
        const bool acc = done > 0;
        const int row = tile * TILE + r;
        {
            const uint4* src = A.X + (size_t)tile * (TILE * K0 * 2 / 16);
            uint4* dst = reinterpret_cast<uint4*>(sm + SM_X);
            for (int i = tid; i < TILE * K0 * 2 / 16; i += NET_THREADS) dst[i] = src[i];
        }
        sync_for_mma();
        if (tid == 0 && !A.no_issue) issue(sb, tbase, OP_L1, false);
        if (!complete()) { failed = true; break; }
        for (int c = c0; c < c1; c += 16) {          // H1 = silu(Z1 + b1)
            tm_ld16(trow + TM_Z1 + c, v);
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] = silu_f(v[j] + sbias[c + j]);
            st_row16(sm + SM_H1, r, c, HID, v);
        }
        sync_for_mma();
        if (tid == 0 && !A.no_issue) issue(sb, tbase, OP_L2, false);
        if (!complete()) { failed = true; break; }
        for (int c = c0; c < c1; c += 16) {          // H2 = silu(Z2 + b2), S2 = silu'(Z2 + b2)
            tm_ld16(trow + TM_WORK + c, v);
#pragma unroll
            for (int j = 0; j < 16; j++) { const float z = v[j] + sbias[HID + c + j]; v[j] = silu_f(z); w[j] = dsilu_f(z); }
            st_row16(sm + SM_H2, r, c, HID, v);
            if (TRAIN) st_row16(sm + SM_S2, r, c, HID, w);
        }
        sync_for_mma();
        if (tid == 0 && !A.no_issue) issue(sb, tbase, OP_L3, false);
        if (!complete()) { failed = true; break; }
        if (half == 0) {
            tm_ld16(trow + TM_WORK, v);
#pragma unroll
            for (int j = 0; j < NOP; j++) v[j] += sbias[2 * HID + j];
        }
        if (!TRAIN) {
            if (half == 0 && row < A.nrows)
                A.out[row] = make_float4(v[0] * A.out_scale, v[1] * A.out_scale, v[2] * A.out_scale, 0.f);
            done++;
            sync_for_mma();      // TMEM reads of this tile finish before the next tile's products
            continue;
        }
        if (half == 0) {   // loss and dY = 2 (y - t) w / B (padding rows have w = 0)
            const float4 t = A.T[row];
            const float d0 = (v[0] - t.x) * t.w, d1 = (v[1] - t.y) * t.w, d2 = (v[2] - t.z) * t.w;
            lsum += d0 * d0 + d1 * d1 + d2 * d2;
            const float s = 2.f * A.inv_batch;
#pragma unroll
            for (int j = 0; j < 16; j++) w[j] = 0.f;
            w[0] = bf_round(s * d0); w[1] = bf_round(s * d1); w[2] = bf_round(s * d2);
            db3[0] += w[0]; db3[1] += w[1]; db3[2] += w[2];
            st_row16(sm + SM_DY, r, 0, NOP, w);
        }
        sync_for_mma();
        if (tid == 0 && !A.no_issue) { issue(sb, tbase, OP_DW3, acc); issue(sb, tbase, OP_DH2, false); }
        if (!complete()) { failed = true; break; }
        for (int c = c0; c < c1; c += 16) {          // dZ2 = dH2 * S2 (in place of S2)
            tm_ld16(trow + TM_WORK + c, v);
            ld_row16(sm + SM_S2, r, c, HID, w);
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] *= w[j];
            st_row16(sm + SM_S2, r, c, HID, v);
        }
        sync_for_mma();
        if (tid == 0 && !A.no_issue) { issue(sb, tbase, OP_DW2, acc); issue(sb, tbase, OP_DB2, acc); issue(sb, tbase, OP_DH1, false); }
        if (!complete()) { failed = true; break; }
        for (int c = c0; c < c1; c += 16) {          // dZ1 = dH1 * silu'(Z1 + b1), into the H2 buffer
            tm_ld16(trow + TM_WORK + c, v);
            tm_ld16(trow + TM_Z1 + c, w);
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] *= bf_round(dsilu_f(w[j] + sbias[c + j]));
            st_row16(sm + SM_H2, r, c, HID, v);
        }
        sync_for_mma();
        if (tid == 0 && !A.no_issue) { issue(sb, tbase, OP_DW1, acc); issue(sb, tbase, OP_DB1, acc); }
        if (!complete()) { failed = true; break; }
        done++;
    }

    if (TRAIN) {
        // this CTA's gradient sums, plain stores into its own slice (reduced
        // over CTAs by reduce_grad_kernel: no atomics, deterministic order)
        float* g = A.gpart + (size_t)blockIdx.x * P_TOTAL;
        float* red = reinterpret_cast<float*>(sm + SM_X);      // X tile no longer needed: 8 warps x 4 floats
        if (!failed && done > 0) {
            // 16-byte stores (every row start and chunk is 64-byte aligned)
            for (int c = c0; c < c1; c += 16) {
                tm_ld16(trow + TM_DW2 + c, v);
                float4* d = reinterpret_cast<float4*>(g + P_W2 + r * HID + c);
#pragma unroll
                for (int j = 0; j < 4; j++) d[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            }
            // dW1: 5 chunks of 16 columns, 3 in the first half, 2 in the second
            for (int c = half ? 48 : 0; c < (half ? K0 : 48); c += 16) {
                tm_ld16(trow + TM_DW1 + c, v);
                float4* d = reinterpret_cast<float4*>(g + P_W1 + r * K0 + c);
#pragma unroll
                for (int j = 0; j < 4; j++) d[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            }
            if (half == 0) {
                tm_ld16(trow + TM_DW3, v);
#pragma unroll
                for (int j = 0; j < NOP; j++) g[P_W3 + j * HID + r] = v[j];
                tm_ld16(trow + TM_DB1, v);
                g[P_B1 + r] = v[0];
                tm_ld16(trow + TM_DB2, v);
                g[P_B2 + r] = v[0];
            }
        } else {
            for (int i = tid; i < P_B3; i += NET_THREADS) g[i] = 0.f;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
#pragma unroll
            for (int k = 0; k < NOUT; k++) db3[k] += __shfl_xor_sync(0xffffffffu, db3[k], o);
        }
        __syncthreads();
        if ((tid & 31) == 0) {
            red[4 * warp] = lsum;
#pragma unroll
            for (int k = 0; k < NOUT; k++) red[4 * warp + 1 + k] = db3[k];
        }
        __syncthreads();
        if (tid < NOP) {
            float b = 0.f;
            if (tid < NOUT) for (int q = 0; q < NET_THREADS / 32; q++) b += red[4 * q + 1 + tid];
            g[P_B3 + tid] = b;
        }
        if (tid == 0) {
            double l = 0.0;
            for (int q = 0; q < NET_THREADS / 32; q++) l += (double)red[4 * q];
            A.lpart[blockIdx.x] = l * (double)A.inv_batch;
        }
    }
    if (failed && tid == 0) atomicExch(A.err, 1);
    tc_before();
    __syncthreads();
    tc_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TM_COLS) : "memory");
}

// sum of the per-CTA gradient slices (fixed order) and of the loss partials
__global__ void reduce_grad_kernel(const float* __restrict__ gpart, const double* __restrict__ lpart, int nblk,
                                   float* __restrict__ grad, double* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P_TOTAL) {
        float acc = 0.f;
        for (int b = 0; b < nblk; b++) acc += gpart[(size_t)b * P_TOTAL + i];
        grad[i] = acc;
    }
    if (i == 0) {
        double l = 0.0;
        for (int b = 0; b < nblk; b++) l += lpart[b];
        *loss = l;
    }
}

// standardise raw features and pack them into bf16 core-matrix tiles
__global__ void pack_input_kernel(const float* __restrict__ F, int n, int ntile, const float* __restrict__ mean,
                                  const float* __restrict__ istd, uint8_t* __restrict__ X) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;     // (row, 8-column chunk)
    const long nchunk = (long)ntile * TILE * (K0 / 8);
    if (i >= nchunk) return;
    const int r = (int)(i / (K0 / 8)), kc = (int)(i % (K0 / 8));
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int k = kc * 8 + j;
        v[j] = (r < n && k < NFEAT) ? (F[(long)r * NFEAT + k] - mean[k]) * istd[k] : 0.f;
    }
    uint8_t* base = X + (size_t)(r / TILE) * TILE * K0 * 2;
    *reinterpret_cast<uint4*>(base + cm_off(r % TILE, kc * 8, K0)) =
        make_uint4(pack_bf2(v[0], v[1]), pack_bf2(v[2], v[3]), pack_bf2(v[4], v[5]), pack_bf2(v[6], v[7]));
}

// AdamW on the flat FP32 parameters (step t >= 1; t == 0 packs only), then the
// packed bf16 weight image.  Weight decay on W1, W2, W3, not on the biases.
__global__ void adamw_pack_kernel(float* __restrict__ prm, const float* __restrict__ g, float* __restrict__ m,
                                  float* __restrict__ vv, int t, float lr, float b1, float b2, float eps, float wd,
                                  uint8_t* __restrict__ Wp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P_TOTAL) return;
    float p = prm[i];
    const bool isW = (i < P_B1) || (i >= P_W2 && i < P_B2) || (i >= P_W3 && i < P_B3);
    if (t > 0) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * vv[i] + (1.f - b2) * gi * gi;
        m[i] = mi; vv[i] = vi;
        const float mh = mi / (1.f - powf(b1, (float)t));
        const float vh = vi / (1.f - powf(b2, (float)t));
        float upd = mh / (sqrtf(vh) + eps);
        if (isW) upd += wd * p;
        p -= lr * upd;
        // padding: W1 inputs >= 68, W3 / b3 outputs >= 3 stay zero
        if ((i < P_B1 && (i % K0) >= NFEAT) || (i >= P_W3 && i < P_B3 && (i - P_W3) / HID >= NOUT) ||
            (i >= P_B3 && i - P_B3 >= NOUT))
            p = 0.f;
        prm[i] = p;
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(p);
    if (i < P_B1) {
        *reinterpret_cast<__nv_bfloat16*>(Wp + WP_W1 + cm_off(i / K0, i % K0, K0)) = h;
    } else if (i >= P_W2 && i < P_B2) {
        const int e = i - P_W2;
        *reinterpret_cast<__nv_bfloat16*>(Wp + WP_W2 + cm_off(e / HID, e % HID, HID)) = h;
    } else if (i >= P_W3 && i < P_B3) {
        const int e = i - P_W3;
        *reinterpret_cast<__nv_bfloat16*>(Wp + WP_W3 + cm_off(e / HID, e % HID, HID)) = h;
    }
}

// ------------------------------------------------------------ descriptors
constexpr int DESC_WARPS = 8;
constexpr int DESC_CAP = 192;           // candidates within 5 A kept per atom

// one warp per atom: candidates within 5 A over the pair-term image set, the
// 32 nearest by (r, image, j), Gaussian radial bins per element channel,
// height above the slab, GridFF force (the relaxer's sampler)
__global__ void __launch_bounds__(DESC_WARPS * 32) descriptor_kernel(Params P, Systems Y, const int* __restrict__ atom_sys,
                                                                    const int* __restrict__ elem, int NA, float zoff,
                                                                    float* __restrict__ feat, int* __restrict__ err) {
    __shared__ float cr[DESC_WARPS][DESC_CAP];
    __shared__ int ck[DESC_WARPS][DESC_CAP];
    __shared__ unsigned char csel[DESC_WARPS][DESC_CAP];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ga = blockIdx.x * DESC_WARPS + wib;
    if (ga >= NA) return;
    const int s = atom_sys[ga];
    const int4 d = Y.desc[s];
    const int aoff = d.x, voff = d.z, N = d.w, i = ga - aoff;
    const float4 pi = Y.pos[voff + i];
    const float* lv = Y.lvec + 9 * s;
    const bool pbc = (P.flags & F_PBC) != 0;
    const int npx = pbc ? P.npbc[0] : 0, npy = pbc ? P.npbc[1] : 0, npz = pbc ? P.npbc[2] : 0;
    const float RC = 5.0f;
    int count = 0, k = 0;
    for (int iz = -npz; iz <= npz; iz++)
        for (int iy = -npy; iy <= npy; iy++)
            for (int ix = -npx; ix <= npx; ix++, k++) {
                const float shx = lv[0] * ix + lv[3] * iy + lv[6] * iz;
                const float shy = lv[1] * ix + lv[4] * iy + lv[7] * iz;
                const float shz = lv[2] * ix + lv[5] * iy + lv[8] * iz;
                const bool central = (ix | iy | iz) == 0;
                for (int j0 = 0; j0 < N; j0 += 32) {
                    const int j = j0 + lane;
                    bool ok = false;
                    float r = 0.f;
                    if (j < N) {
                        const float4 pj = Y.pos[voff + j];
                        const float dx = pj.x + shx - pi.x, dy = pj.y + shy - pi.y, dz = pj.z + shz - pi.z;
                        r = sqrtf(dx * dx + dy * dy + dz * dz);
                        ok = (r < RC) && !(central && j == i);
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, ok);
                    const int slot = count + __popc(bal & ((1u << lane) - 1u));
                    if (ok && slot < DESC_CAP) { cr[wib][slot] = r; ck[wib][slot] = k * N + j; }
                    count += __popc(bal);
                }
            }
    if (count > DESC_CAP && lane == 0) atomicExch(err, 2);
    const int C = min(count, DESC_CAP);
    __syncwarp();
    for (int c = lane; c < C; c += 32) {
        const float r = cr[wib][c];
        const int key = ck[wib][c];
        int rank = 0;
        for (int q = 0; q < C; q++) {
            const float rq = cr[wib][q];
            rank += (rq < r) || (rq == r && ck[wib][q] < key);
        }
        csel[wib][c] = rank < 32;
    }
    __syncwarp();
    const int ch0 = lane >> 4, ch1 = 2 + (lane >> 4);
    const float mu = (float)(lane & 15) * (5.0f / 15.0f);
    const float ig = 1.f / (2.f * 0.3f * 0.3f);
    float f0 = 0.f, f1 = 0.f;
    for (int c = 0; c < C; c++) {
        if (!csel[wib][c]) continue;
        const int j = ck[wib][c] % N;
        const int ch = min(elem[aoff + j], 3);
        const float t = cr[wib][c] - mu;
        const float e = expf(-t * t * ig);
        if (ch == ch0) f0 += e;
        if (ch == ch1) f1 += e;
    }
    float* out = feat + (size_t)ga * NFEAT;
    out[lane] = f0;
    out[32 + lane] = f1;
    if (lane == 0) {
        const float4 go = Y.gorg[s];
        out[64] = pi.z + go.z + zoff;
        float4 fg = make_float4(0.f, 0.f, 0.f, 0.f);
        if (P.flags & F_GRID) {
            const float3 u = make_float3((pi.x + go.x) * P.ginv[0], (pi.y + go.y) * P.ginv[1], (pi.z + go.z) * P.ginv[2]);
            fg = grid_atom(P, u, Y.PLQ[aoff + i]);
        }
        out[65] = fg.x; out[66] = fg.y; out[67] = fg.z;
    }
}

// ------------------------------------------------------------ warm start
// start of a learned step: remember the atoms' positions, no system decided yet
__global__ void save_kernel(Systems Y, const int* __restrict__ atom_sys, int NA, float4* __restrict__ save) {
    const int ga = blockIdx.x * blockDim.x + threadIdx.x;
    if (ga >= NA) return;
    const int4 d = Y.desc[atom_sys[ga]];
    save[ga] = Y.pos[d.z + ga - d.x];
}

// trial position save + alpha * proposal for the systems still undecided
// (world and local frames differ by a translation only)
__global__ void apply_kernel(Systems Y, const int* __restrict__ atom_sys, int NA, const float4* __restrict__ disp,
                             const float4* __restrict__ save, float alpha, const int* __restrict__ done) {
    const int ga = blockIdx.x * blockDim.x + threadIdx.x;
    if (ga >= NA) return;
    const int s = atom_sys[ga];
    if (done[s]) return;
    const int4 d = Y.desc[s];
    const float4 p = save[ga], u = disp[ga];
    Y.pos[d.z + ga - d.x] = make_float4(p.x + alpha * u.x, p.y + alpha * u.y, p.z + alpha * u.z, p.w);
}

// per undecided system: keep the trial if the total energy dropped (NaN rejects)
__global__ void gate_sys_kernel(int nsys, const double4* __restrict__ E1, double4* __restrict__ E0,
                                int* __restrict__ done, int* __restrict__ accepted) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys || done[s]) return;
    if (E1[s].w < E0[s].w) { E0[s] = E1[s]; accepted[s] += 1; done[s] = 1; }
}

// undecided systems go back to the saved positions
__global__ void revert_kernel(Systems Y, const int* __restrict__ atom_sys, int NA, const int* __restrict__ done,
                              const float4* __restrict__ save) {
    const int ga = blockIdx.x * blockDim.x + threadIdx.x;
    if (ga >= NA) return;
    const int s = atom_sys[ga];
    if (done[s]) return;
    const int4 d = Y.desc[s];
    Y.pos[d.z + ga - d.x] = save[ga];
}

// Rigid-body projection of the proposal, one warp per system: the translation
// t and rotation vector w that best reproduce the per-atom displacements d_i
// in least squares (minimise sum |d_i - t - w x u_i|^2, u_i = p_i - centroid:
// t = mean d, (sum |u|^2 1 - u u^T) w = sum u x (d - t), FP64), then d_i is
// replaced by t + (R(w) - 1) u_i with R the rotation by |w| about w (Rodrigues).
// A rigid move keeps every bond, angle and pi term of the molecule, so the
// energy gate only weighs the molecule's placement against the substrate and
// its own images: the network's per-atom outputs act as a vote on one
// translation and one rotation per molecule.
__global__ void rigid_kernel(Systems Y, int nsys, const float4* __restrict__ save, float4* __restrict__ disp) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nsys) return;                      // whole warps
    const int4 d = Y.desc[w];
    const int a0 = d.x, n = d.w;
    auto red = [](double v) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    };
    double c[3] = {0, 0, 0}, t[3] = {0, 0, 0};
    for (int i = lane; i < n; i += 32) {
        const float4 p = save[a0 + i], q = disp[a0 + i];
        c[0] += p.x; c[1] += p.y; c[2] += p.z; t[0] += q.x; t[1] += q.y; t[2] += q.z;
    }
    for (int k = 0; k < 3; k++) { c[k] = red(c[k]) / n; t[k] = red(t[k]) / n; }
    double A[6] = {0, 0, 0, 0, 0, 0}, b[3] = {0, 0, 0};     // xx yy zz xy xz yz
    for (int i = lane; i < n; i += 32) {
        const float4 p = save[a0 + i], q = disp[a0 + i];
        const double u0 = p.x - c[0], u1 = p.y - c[1], u2 = p.z - c[2];
        const double e0 = q.x - t[0], e1 = q.y - t[1], e2 = q.z - t[2];
        const double uu = u0 * u0 + u1 * u1 + u2 * u2;
        A[0] += uu - u0 * u0; A[1] += uu - u1 * u1; A[2] += uu - u2 * u2;
        A[3] -= u0 * u1; A[4] -= u0 * u2; A[5] -= u1 * u2;
        b[0] += u1 * e2 - u2 * e1; b[1] += u2 * e0 - u0 * e2; b[2] += u0 * e1 - u1 * e0;
    }
    for (int k = 0; k < 6; k++) A[k] = red(A[k]);
    for (int k = 0; k < 3; k++) b[k] = red(b[k]);
    const double tr = A[0] + A[1] + A[2];
    for (int k = 0; k < 3; k++) A[k] += 1e-9 * tr + 1e-12;       // collinear / single-atom systems
    // symmetric 3x3 solve by the adjugate
    const double c00 = A[1] * A[2] - A[5] * A[5], c01 = A[4] * A[5] - A[3] * A[2], c02 = A[3] * A[5] - A[4] * A[1];
    const double c11 = A[0] * A[2] - A[4] * A[4], c12 = A[3] * A[4] - A[0] * A[5], c22 = A[0] * A[1] - A[3] * A[3];
    const double det = A[0] * c00 + A[3] * c01 + A[4] * c02;
    double om[3] = {0, 0, 0};
    if (det > 0) {
        om[0] = (c00 * b[0] + c01 * b[1] + c02 * b[2]) / det;
        om[1] = (c01 * b[0] + c11 * b[1] + c12 * b[2]) / det;
        om[2] = (c02 * b[0] + c12 * b[1] + c22 * b[2]) / det;
    }
    const double th = sqrt(om[0] * om[0] + om[1] * om[1] + om[2] * om[2]);
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (th > 1e-12) {
        const double x = om[0] / th, y = om[1] / th, z = om[2] / th, cs = cos(th), sn = sin(th), cc = 1 - cs;
        R[0] = cs + x * x * cc;     R[1] = x * y * cc - z * sn; R[2] = x * z * cc + y * sn;
        R[3] = y * x * cc + z * sn; R[4] = cs + y * y * cc;     R[5] = y * z * cc - x * sn;
        R[6] = z * x * cc - y * sn; R[7] = z * y * cc + x * sn; R[8] = cs + z * z * cc;
    }
    for (int i = lane; i < n; i += 32) {
        const float4 p = save[a0 + i];
        const double u0 = p.x - c[0], u1 = p.y - c[1], u2 = p.z - c[2];
        disp[a0 + i] = make_float4((float)(t[0] + R[0] * u0 + R[1] * u1 + R[2] * u2 - u0),
                                   (float)(t[1] + R[3] * u0 + R[4] * u1 + R[5] * u2 - u1),
                                   (float)(t[2] + R[6] * u0 + R[7] * u1 + R[8] * u2 - u2), 0.f);
    }
}

}  // namespace mlp
}  // namespace mmff

// ===================================================================== C-ABI
using namespace mmff;
using namespace mmff::mlp;

namespace {

int fail(const std::string& m) { mmff_set_error(m.c_str()); return -1; }
#define MCK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(std::string(#x) + ": " + cudaGetErrorString(e_)); } while (0)

template <class X> struct Buf {
    X* p = nullptr; size_t n = 0;
    int ensure(size_t cnt) {
        if (cnt <= n && p) return 0;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        if (!cnt) return 0;
        if (cudaMalloc(&p, cnt * sizeof(X)) != cudaSuccess) return fail("cudaMalloc failed (learned proposal buffers)");
        n = cnt;
        return 0;
    }
};

struct Net {
    bool has_params = false;
    int t = 0;                              // AdamW step count
    Buf<float> prm, grad, m, v, mean, istd, feat, gpart;
    Buf<uint8_t> Wp, Xs, Xd;
    Buf<float4> Td, outs, save;
    Buf<double> loss, losses, lpart;
    Buf<double4> E0;
    Buf<int> err, atom_sys, elem, accepted, keep;
    float out_scale = 1.f;
    int ndata = 0, ntile_data = 0, na_elem = 0;
    int projection = 0;                     // warm start: 0 per-atom moves, 1 rigid-body projection
    bool attr_set = false;
};
Net N;

int set_attr() {
    if (N.attr_set) return 0;
    MCK(cudaFuncSetAttribute(mlp_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_ALLOC));
    MCK(cudaFuncSetAttribute(mlp_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_ALLOC));
    N.attr_set = true;
    return 0;
}

int num_sms() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

int check_err(cudaStream_t st, const char* what) {
    int h = 0;
    MCK(cudaMemcpyAsync(&h, N.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    if (h == 1) return fail(std::string(what) + ": tensor-core completion wait timed out");
    if (h == 2) return fail(std::string(what) + ": more than 192 descriptor neighbours within 5 A");
    return 0;
}

int pack_input(const float* d_feat, int n, int ntile, uint8_t* X, cudaStream_t st) {
    const long nchunk = (long)ntile * TILE * (K0 / 8);
    pack_input_kernel<<<(unsigned)((nchunk + 255) / 256), 256, 0, st>>>(d_feat, n, ntile, N.mean.p, N.istd.p, X);
    mmff_count_launches(1);
    MCK(cudaGetLastError());
    return 0;
}

int run_net(bool train, const uint8_t* X, const float4* T, int ntile, int nrows, float inv_batch, float4* out,
            cudaStream_t st) {
    if (set_attr()) return -1;
    const int grid = std::max(1, std::min(ntile, num_sms()));
    if (train && (N.gpart.ensure((size_t)grid * P_TOTAL) || N.lpart.ensure(grid))) return -1;
    NetArgs a;
    a.X = reinterpret_cast<const uint4*>(X); a.T = T; a.Wp = reinterpret_cast<const uint4*>(N.Wp.p);
    a.prm = N.prm.p; a.gpart = N.gpart.p; a.lpart = N.lpart.p; a.out = out; a.err = N.err.p;
    a.ntile = ntile; a.nrows = nrows; a.inv_batch = inv_batch; a.out_scale = N.out_scale;
    a.wait_limit = 1ll << 31; a.no_issue = 0;
    if (train) {
        mlp_kernel<true><<<grid, NET_THREADS, SM_ALLOC, st>>>(a);
        mmff_count_launches(1);
        reduce_grad_kernel<<<(P_TOTAL + 255) / 256, 256, 0, st>>>(N.gpart.p, N.lpart.p, grid, N.grad.p, N.loss.p);
        mmff_count_launches(1);
    } else {
        mlp_kernel<false><<<grid, NET_THREADS, SM_ALLOC, st>>>(a);
        mmff_count_launches(1);
    }
    MCK(cudaGetLastError());
    return 0;
}

int adamw(int t, double lr, double wd, cudaStream_t st) {
    adamw_pack_kernel<<<(P_TOTAL + 255) / 256, 256, 0, st>>>(N.prm.p, N.grad.p, N.m.p, N.v.p, t, (float)lr, 0.9f,
                                                             0.999f, 1e-8f, (float)wd, N.Wp.p);
    mmff_count_launches(1);
    MCK(cudaGetLastError());
    return 0;
}

int need_params() { return N.has_params ? 0 : fail("network parameters not set (mmff_mlp_set_params)"); }

// step lengths tried along a learned proposal, longest first
constexpr int kTrials = 4;
constexpr float kAlpha[kTrials] = {1.0f, 0.5f, 0.25f, 0.125f};

// targets in network units, padded to whole tiles with zero weight
std::vector<float4> make_targets(int n, int ntile, const float* target) {
    std::vector<float4> T((size_t)ntile * TILE, make_float4(0, 0, 0, 0));
    const float s = 1.f / N.out_scale;
    for (int r = 0; r < n; r++) T[r] = make_float4(target[3 * r] * s, target[3 * r + 1] * s, target[3 * r + 2] * s, 1.f);
    return T;
}

int features_device(const WorldView& V, double z_top) {
    if (!N.elem.p || N.na_elem != V.NA) return fail("element channels not set for these systems (mmff_mlp_set_elements)");
    if (N.feat.ensure((size_t)V.NA * NFEAT) || N.err.ensure(1)) return -1;
    const float zoff = (float)(V.gpos0[2] - z_top);
    descriptor_kernel<<<(V.NA + DESC_WARPS - 1) / DESC_WARPS, DESC_WARPS * 32, 0, V.stream>>>(
        V.P, V.Y, N.atom_sys.p, N.elem.p, V.NA, zoff, N.feat.p, N.err.p);
    mmff_count_launches(1);
    MCK(cudaGetLastError());
    return 0;
}

}  // namespace

extern "C" {

int mmff_mlp_plan(int* ops) {
    for (int i = 0; i < OP_COUNT; i++) {
        const MmaOp o = mma_op(i);
        const int vals[14] = {o.dcol, o.N, o.nk, o.acc_tiles, o.a_off, o.a_lbo, o.a_sbo, o.a_step, o.a_mn,
                              o.b_off, o.b_lbo, o.b_sbo, o.b_step, o.b_mn};
        for (int j = 0; j < 14; j++) ops[14 * i + j] = vals[j];
    }
    return OP_COUNT;
}

int mmff_mlp_layout(int* out) {
    const int v[16] = {P_TOTAL, P_W1, P_B1, P_W2, P_B2, P_W3, P_B3, SM_TOTAL, SM_ALLOC, TM_COLS, NFEAT, K0,
                       SM_W1, SM_X, SM_DY, WP_BYTES};
    for (int i = 0; i < 16; i++) out[i] = v[i];
    return 0;
}

unsigned long long mmff_mlp_smem_desc(unsigned addr, unsigned lbo, unsigned sbo) { return smem_desc(addr, lbo, sbo); }
unsigned mmff_mlp_instr_desc(int n, int a_mn, int b_mn) { return instr_desc(n, a_mn, b_mn); }

int mmff_mlp_set_params(const float* prm, const float* feat_mean, const float* feat_std, double out_scale) {
    cudaStream_t st = world_stream();
    if (!st) return -1;
    if (!prm || !feat_mean || !feat_std) return fail("mmff_mlp_set_params: NULL argument");
    if (!(out_scale > 0)) return fail("mmff_mlp_set_params: out_scale must be > 0");
    if (N.prm.ensure(P_TOTAL) || N.grad.ensure(P_TOTAL) || N.m.ensure(P_TOTAL) || N.v.ensure(P_TOTAL) ||
        N.mean.ensure(NFEAT) || N.istd.ensure(NFEAT) || N.Wp.ensure(WP_BYTES) || N.loss.ensure(1) || N.err.ensure(1))
        return -1;
    std::vector<float> is(NFEAT);
    for (int k = 0; k < NFEAT; k++) {
        if (!(feat_std[k] > 0.f)) return fail("mmff_mlp_set_params: feature std must be > 0");
        is[k] = 1.f / feat_std[k];
    }
    MCK(cudaMemcpyAsync(N.prm.p, prm, P_TOTAL * sizeof(float), cudaMemcpyHostToDevice, st));
    MCK(cudaMemcpyAsync(N.mean.p, feat_mean, NFEAT * sizeof(float), cudaMemcpyHostToDevice, st));
    MCK(cudaMemcpyAsync(N.istd.p, is.data(), NFEAT * sizeof(float), cudaMemcpyHostToDevice, st));
    MCK(cudaMemsetAsync(N.m.p, 0, P_TOTAL * sizeof(float), st));
    MCK(cudaMemsetAsync(N.v.p, 0, P_TOTAL * sizeof(float), st));
    MCK(cudaMemsetAsync(N.Wp.p, 0, WP_BYTES, st));
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), st));
    N.out_scale = (float)out_scale;
    N.t = 0;
    if (adamw(0, 0.0, 0.0, st)) return -1;
    MCK(cudaStreamSynchronize(st));
    N.has_params = true;
    return 0;
}

int mmff_mlp_get_params(float* prm) {
    if (need_params()) return -1;
    cudaStream_t st = world_stream();
    MCK(cudaMemcpyAsync(prm, N.prm.p, P_TOTAL * sizeof(float), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    return 0;
}

int mmff_mlp_grad(int n, const float* feat, const float* target, float* grad_out, double* loss_out) {
    if (need_params()) return -1;
    if (n <= 0 || !feat || !target) return fail("mmff_mlp_grad: need n > 0 rows of features and targets");
    cudaStream_t st = world_stream();
    const int ntile = (n + TILE - 1) / TILE;
    if (N.feat.ensure((size_t)n * NFEAT) || N.Xs.ensure((size_t)ntile * TILE * K0 * 2) || N.outs.ensure((size_t)ntile * TILE))
        return -1;
    const std::vector<float4> T = make_targets(n, ntile, target);
    MCK(cudaMemcpyAsync(N.feat.p, feat, (size_t)n * NFEAT * sizeof(float), cudaMemcpyHostToDevice, st));
    MCK(cudaMemcpyAsync(N.outs.p, T.data(), T.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
    if (pack_input(N.feat.p, n, ntile, N.Xs.p, st)) return -1;
    MCK(cudaMemsetAsync(N.grad.p, 0, P_TOTAL * sizeof(float), st));
    MCK(cudaMemsetAsync(N.loss.p, 0, sizeof(double), st));
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), st));
    if (run_net(true, N.Xs.p, N.outs.p, ntile, n, 1.f / n, nullptr, st)) return -1;
    if (check_err(st, "mmff_mlp_grad")) return -1;
    if (grad_out) MCK(cudaMemcpyAsync(grad_out, N.grad.p, P_TOTAL * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (loss_out) MCK(cudaMemcpyAsync(loss_out, N.loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    return 0;
}

int mmff_mlp_adamw(const float* grad, double lr, double wd) {
    if (need_params()) return -1;
    cudaStream_t st = world_stream();
    if (grad) MCK(cudaMemcpyAsync(N.grad.p, grad, P_TOTAL * sizeof(float), cudaMemcpyHostToDevice, st));
    N.t++;
    if (adamw(N.t, lr, wd, st)) return -1;
    MCK(cudaStreamSynchronize(st));
    return 0;
}

int mmff_mlp_infer(int n, const float* feat, float* out) {
    if (need_params()) return -1;
    if (n <= 0 || !feat || !out) return fail("mmff_mlp_infer: need n > 0 rows of features and an output array");
    cudaStream_t st = world_stream();
    const int ntile = (n + TILE - 1) / TILE;
    if (N.feat.ensure((size_t)n * NFEAT) || N.Xs.ensure((size_t)ntile * TILE * K0 * 2) || N.outs.ensure((size_t)ntile * TILE))
        return -1;
    MCK(cudaMemcpyAsync(N.feat.p, feat, (size_t)n * NFEAT * sizeof(float), cudaMemcpyHostToDevice, st));
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), st));
    if (pack_input(N.feat.p, n, ntile, N.Xs.p, st)) return -1;
    if (run_net(false, N.Xs.p, nullptr, ntile, n, 0.f, N.outs.p, st)) return -1;
    if (check_err(st, "mmff_mlp_infer")) return -1;
    std::vector<float4> h(n);
    MCK(cudaMemcpyAsync(h.data(), N.outs.p, n * sizeof(float4), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    for (int r = 0; r < n; r++) { out[3 * r] = h[r].x; out[3 * r + 1] = h[r].y; out[3 * r + 2] = h[r].z; }
    return 0;
}

int mmff_mlp_set_data(int n, const float* feat, const float* target) {
    if (need_params()) return -1;
    if (n <= 0 || !feat || !target) return fail("mmff_mlp_set_data: need n > 0 rows of features and targets");
    cudaStream_t st = world_stream();
    const int ntile = (n + TILE - 1) / TILE;
    if (N.feat.ensure((size_t)n * NFEAT) || N.Xd.ensure((size_t)ntile * TILE * K0 * 2) || N.Td.ensure((size_t)ntile * TILE))
        return -1;
    const std::vector<float4> T = make_targets(n, ntile, target);
    MCK(cudaMemcpyAsync(N.feat.p, feat, (size_t)n * NFEAT * sizeof(float), cudaMemcpyHostToDevice, st));
    MCK(cudaMemcpyAsync(N.Td.p, T.data(), T.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
    if (pack_input(N.feat.p, n, ntile, N.Xd.p, st)) return -1;
    MCK(cudaStreamSynchronize(st));
    N.ndata = n; N.ntile_data = ntile;
    return 0;
}

int mmff_mlp_train(int nsteps, int batch_tiles, double lr, double wd, double* loss_out) {
    if (need_params()) return -1;
    if (!N.ndata) return fail("mmff_mlp_train: no training set (mmff_mlp_set_data)");
    if (nsteps <= 0 || batch_tiles <= 0) return fail("mmff_mlp_train: nsteps and batch_tiles must be > 0");
    batch_tiles = std::min(batch_tiles, N.ntile_data);
    cudaStream_t st = world_stream();
    if (N.losses.ensure(nsteps)) return -1;
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), st));
    int t0 = 0;
    for (int k = 0; k < nsteps; k++) {
        if (t0 + batch_tiles > N.ntile_data) t0 = 0;
        const int rows = std::min(batch_tiles * TILE, N.ndata - t0 * TILE);
        MCK(cudaMemsetAsync(N.grad.p, 0, P_TOTAL * sizeof(float), st));
        MCK(cudaMemsetAsync(N.loss.p, 0, sizeof(double), st));
        if (run_net(true, N.Xd.p + (size_t)t0 * TILE * K0 * 2, N.Td.p + (size_t)t0 * TILE, batch_tiles, rows,
                    1.f / rows, nullptr, st))
            return -1;
        N.t++;
        if (adamw(N.t, lr, wd, st)) return -1;
        MCK(cudaMemcpyAsync(N.losses.p + k, N.loss.p, sizeof(double), cudaMemcpyDeviceToDevice, st));
        t0 += batch_tiles;
    }
    if (check_err(st, "mmff_mlp_train")) return -1;
    if (loss_out) MCK(cudaMemcpyAsync(loss_out, N.losses.p, nsteps * sizeof(double), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    return 0;
}

int mmff_mlp_set_elements(const int* elem) {
    WorldView V;
    if (world_view(&V)) return -1;
    if (!elem) return fail("mmff_mlp_set_elements: NULL element array");
    if (N.elem.ensure(V.NA) || N.atom_sys.ensure(V.NA) || N.err.ensure(1)) return -1;
    std::vector<int> as(V.NA);
    for (int s = 0; s < V.nsys; s++)
        for (int i = 0; i < V.desc[s].w; i++) as[V.desc[s].x + i] = s;
    MCK(cudaMemcpyAsync(N.elem.p, elem, V.NA * sizeof(int), cudaMemcpyHostToDevice, V.stream));
    MCK(cudaMemcpyAsync(N.atom_sys.p, as.data(), V.NA * sizeof(int), cudaMemcpyHostToDevice, V.stream));
    MCK(cudaStreamSynchronize(V.stream));
    N.na_elem = V.NA;
    return 0;
}

int mmff_mlp_features(double z_top, float* out) {
    WorldView V;
    if (world_view(&V)) return -1;
    if (!out) return fail("mmff_mlp_features: NULL output");
    if (N.err.ensure(1)) return -1;
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), V.stream));
    if (features_device(V, z_top)) return -1;
    if (check_err(V.stream, "mmff_mlp_features")) return -1;
    MCK(cudaMemcpyAsync(out, N.feat.p, (size_t)V.NA * NFEAT * sizeof(float), cudaMemcpyDeviceToHost, V.stream));
    MCK(cudaStreamSynchronize(V.stream));
    return 0;
}

// The bounded completion waits of the tensor-core kernel, exercised: one
// inference launch (one CTA, one tile of zeros) that issues no product and
// no commit, so its first wait on the completion barrier can only run out
// (limit 2^20 SM clocks, about half a millisecond).  Nothing asynchronous is
// in flight when it does, so the CTA sets the error flag, frees its TMEM and
// returns.  Returns 1 when the timeout came back as the error status (the
// flag is cleared again), 0 if it did not.
int mmff_mlp_wait_test(void) {
    if (need_params()) return -1;
    cudaStream_t st = world_stream();
    if (!st) return -1;
    if (set_attr() || N.Xs.ensure((size_t)TILE * K0 * 2) || N.outs.ensure(TILE) || N.err.ensure(1)) return -1;
    MCK(cudaMemsetAsync(N.Xs.p, 0, (size_t)TILE * K0 * 2, st));
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), st));
    NetArgs a;
    memset(&a, 0, sizeof a);
    a.X = reinterpret_cast<const uint4*>(N.Xs.p); a.Wp = reinterpret_cast<const uint4*>(N.Wp.p); a.prm = N.prm.p;
    a.out = N.outs.p; a.err = N.err.p; a.ntile = 1; a.nrows = 1; a.out_scale = N.out_scale;
    a.wait_limit = 1ll << 20; a.no_issue = 1;
    mlp_kernel<false><<<1, NET_THREADS, SM_ALLOC, st>>>(a);
    mmff_count_launches(1);
    MCK(cudaGetLastError());
    int h = 0;
    MCK(cudaMemcpyAsync(&h, N.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), st));
    MCK(cudaStreamSynchronize(st));
    return h == 1 ? 1 : 0;
}

// How warm-start moves use the network's per-atom displacements: 0 as they
// are, 1 projected on one rigid-body move per system (rigid_kernel).
int mmff_mlp_set_projection(int mode) {
    if (mode != 0 && mode != 1) return fail("mmff_mlp_set_projection: mode must be 0 or 1");
    N.projection = mode;
    return 0;
}

// The rigid-body projection of displacements disp [NA][3] (host, FP64) at the
// systems' current positions -> out [NA][3]: the kernel the warm start uses,
// for checks against a restatement.
int mmff_mlp_project(const double* disp, double* out) {
    WorldView V;
    if (world_view(&V)) return -1;
    if (!disp || !out) return fail("mmff_mlp_project: NULL array");
    if (N.outs.ensure(V.NA) || N.save.ensure(V.NA) || N.atom_sys.ensure(V.NA)) return -1;
    std::vector<int> as(V.NA);
    for (int s = 0; s < V.nsys; s++)
        for (int i = 0; i < V.desc[s].w; i++) as[V.desc[s].x + i] = s;
    std::vector<float4> h(V.NA);
    for (int i = 0; i < V.NA; i++) h[i] = make_float4((float)disp[3 * i], (float)disp[3 * i + 1], (float)disp[3 * i + 2], 0.f);
    MCK(cudaMemcpyAsync(N.atom_sys.p, as.data(), V.NA * sizeof(int), cudaMemcpyHostToDevice, V.stream));
    MCK(cudaMemcpyAsync(N.outs.p, h.data(), V.NA * sizeof(float4), cudaMemcpyHostToDevice, V.stream));
    const unsigned ga = (V.NA + 255) / 256;
    save_kernel<<<ga, 256, 0, V.stream>>>(V.Y, N.atom_sys.p, V.NA, N.save.p);
    rigid_kernel<<<(unsigned)((V.nsys + 3) / 4), 128, 0, V.stream>>>(V.Y, V.nsys, N.save.p, N.outs.p);
    mmff_count_launches(2);
    MCK(cudaGetLastError());
    MCK(cudaMemcpyAsync(h.data(), N.outs.p, V.NA * sizeof(float4), cudaMemcpyDeviceToHost, V.stream));
    MCK(cudaStreamSynchronize(V.stream));
    for (int i = 0; i < V.NA; i++) { out[3 * i] = h[i].x; out[3 * i + 1] = h[i].y; out[3 * i + 2] = h[i].z; }
    return 0;
}

int mmff_mlp_warmstart(int nsteps, double z_top, int* accepted) {
    if (need_params()) return -1;
    WorldView V;
    if (world_view(&V)) return -1;
    if (nsteps < 0) return fail("mmff_mlp_warmstart: nsteps must be >= 0");
    const int ntile = (V.NA + TILE - 1) / TILE;
    if (N.Xs.ensure((size_t)ntile * TILE * K0 * 2) || N.outs.ensure((size_t)ntile * TILE) || N.save.ensure(V.NA) ||
        N.E0.ensure(V.nsys) || N.accepted.ensure(V.nsys) || N.keep.ensure(V.nsys))
        return -1;
    MCK(cudaMemsetAsync(N.err.p, 0, sizeof(int), V.stream));
    MCK(cudaMemsetAsync(N.accepted.p, 0, V.nsys * sizeof(int), V.stream));
    if (mmff_eval(1) < 0) return -1;
    MCK(cudaMemcpyAsync(N.E0.p, V.Y.energy, V.nsys * sizeof(double4), cudaMemcpyDeviceToDevice, V.stream));
    const unsigned ga = (V.NA + 255) / 256, gs = (V.nsys + 255) / 256;
    for (int k = 0; k < nsteps; k++) {
        if (features_device(V, z_top)) return -1;
        if (pack_input(N.feat.p, V.NA, ntile, N.Xs.p, V.stream)) return -1;
        if (run_net(false, N.Xs.p, nullptr, ntile, V.NA, 0.f, N.outs.p, V.stream)) return -1;
        save_kernel<<<ga, 256, 0, V.stream>>>(V.Y, N.atom_sys.p, V.NA, N.save.p);
        mmff_count_launches(1);
        if (N.projection == 1) {
            rigid_kernel<<<(unsigned)((V.nsys + 3) / 4), 128, 0, V.stream>>>(V.Y, V.nsys, N.save.p, N.outs.p);
            mmff_count_launches(1);
        }
        MCK(cudaMemsetAsync(N.keep.p, 0, V.nsys * sizeof(int), V.stream));
        // step-length search along the proposal: the first length that lowers
        // a system's energy is kept, otherwise the system stays where it was
        for (int t = 0; t < kTrials; t++) {
            apply_kernel<<<ga, 256, 0, V.stream>>>(V.Y, N.atom_sys.p, V.NA, N.outs.p, N.save.p, kAlpha[t], N.keep.p);
            mmff_count_launches(1);
            MCK(cudaGetLastError());
            if (mmff_eval(1) < 0) return -1;
            gate_sys_kernel<<<gs, 256, 0, V.stream>>>(V.nsys, V.Y.energy, N.E0.p, N.keep.p, N.accepted.p);
            mmff_count_launches(1);
            MCK(cudaGetLastError());
        }
        revert_kernel<<<ga, 256, 0, V.stream>>>(V.Y, N.atom_sys.p, V.NA, N.keep.p, N.save.p);
        mmff_count_launches(1);
        MCK(cudaGetLastError());
    }
    if (check_err(V.stream, "mmff_mlp_warmstart")) return -1;
    if (accepted) MCK(cudaMemcpyAsync(accepted, N.accepted.p, V.nsys * sizeof(int), cudaMemcpyDeviceToHost, V.stream));
    MCK(cudaStreamSynchronize(V.stream));
    return 0;
}

}  // extern "C"
