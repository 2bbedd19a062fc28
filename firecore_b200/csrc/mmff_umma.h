// mmff_umma.h -- shared-memory operand layout and the tcgen05.mma plan of the
// learned-proposal network (host + device; the host side exports the plan so
// that a CPU test can replay every descriptor against packed matrices).
//
// Network 80(68) -> 128 -> 128 -> 16(3), SiLU, BF16 operands, FP32 TMEM
// accumulators, one 128-atom tile per CTA iteration (M = 128, cta_group::1).
//
// Operand layout ("core-matrix tiles", SWIZZLE_NONE): an R x K bf16 matrix
// (R, K multiples of 8) is stored as 8-row x 16-byte core matrices,
//   byte(r, k) = (r/8) * (16 K) + (k/8) * 128 + (r%8) * 16 + (k%8) * 2.
// Read K-major (rows = M or N index, k = reduction), the descriptor has
// leading byte offset 128 (next 8 k) and stride byte offset 16 K (next 8
// rows).  The same bytes read MN-major give the transpose: the MN index is
// k (core matrices 128 B apart: stride byte offset 128) and the reduction
// index is r (leading byte offset 16 K).  Every backward product uses that
// transpose view instead of a second copy of an operand.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define MMFF_HD __host__ __device__
#else
#define MMFF_HD
#endif

namespace mmff {
namespace mlp {

constexpr int TILE = 128;     // atoms per tile (MMA M)
constexpr int NFEAT = 68;     // descriptor features
constexpr int K0 = 80;        // padded input width (multiple of 16)
constexpr int HID = 128;
constexpr int NOUT = 3;
constexpr int NOP = 16;       // padded output width (MMA N)

MMFF_HD constexpr int cm_off(int r, int k, int K) {
    return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// shared-memory map of the network kernels (bytes from the 1024-aligned base)
constexpr int SM_W1 = 0;                          // W1  [128 x 80]
constexpr int SM_W2 = SM_W1 + HID * K0 * 2;       // W2  [128 x 128]
constexpr int SM_W3 = SM_W2 + HID * HID * 2;      // W3  [16 x 128]
constexpr int SM_ONE = SM_W3 + NOP * HID * 2;     // ones [16 x 128] (bias gradients)
constexpr int SM_X = SM_ONE + NOP * TILE * 2;     // X   [128 x 80]
constexpr int SM_H1 = SM_X + TILE * K0 * 2;       // H1  [128 x 128]
constexpr int SM_H2 = SM_H1 + TILE * HID * 2;     // H2, later dZ1
constexpr int SM_S2 = SM_H2 + TILE * HID * 2;     // silu'(Z2), later dZ2
constexpr int SM_DY = SM_S2 + TILE * HID * 2;     // dY  [128 x 16]
constexpr int SM_BIAS = SM_DY + TILE * NOP * 2;   // b1[128] b2[128] b3[16] (fp32)
constexpr int SM_MISC = SM_BIAS + (2 * HID + NOP) * 4;
constexpr int SM_TOTAL = SM_MISC + 64;            // + mbarrier, TMEM base
constexpr int SM_ALLOC = SM_TOTAL + 1024;         // slack for the 1024-B alignment

// tensor-memory columns
constexpr int TM_Z1 = 0;      // Z1 (kept until dZ1)
constexpr int TM_WORK = 128;  // Z2 / Y / dH2 / dH1
constexpr int TM_DW2 = 256;   // accumulators over all tiles of the CTA
constexpr int TM_DW1 = 384;
constexpr int TM_DW3 = 464;   // dW3 transposed [hid x out]
constexpr int TM_DB1 = 480;
constexpr int TM_DB2 = 496;
constexpr int TM_COLS = 512;

// one tcgen05.mma chain: D[128 x N] (+)= sum over nk k-steps of A_k B_k^T
struct MmaOp {
    int dcol, N, nk, acc_tiles;     // acc_tiles: accumulate across tiles (gradient sums)
    int a_off, a_lbo, a_sbo, a_step, a_mn;
    int b_off, b_lbo, b_sbo, b_step, b_mn;
};

// K-major read of a core-matrix tile of row length K, starting at k = 0
#define MMFF_KM(off, K) (off), 128, (K) * 16, 256, 0
// MN-major (transposed) read of a core-matrix tile of row length K: MN = k, reduction = rows
#define MMFF_MN(off, K) (off), (K) * 16, 128, 2 * (K) * 16, 1

enum { OP_L1 = 0, OP_L2, OP_L3, OP_DW3, OP_DH2, OP_DW2, OP_DB2, OP_DH1, OP_DW1, OP_DB1, OP_COUNT };

MMFF_HD inline MmaOp mma_op(int i) {
    switch (i) {
        // forward: Z1 = X W1^T, Z2 = H1 W2^T, Y = H2 W3^T
        case OP_L1: return {TM_Z1, HID, K0 / 16, 0, MMFF_KM(SM_X, K0), MMFF_KM(SM_W1, K0)};
        case OP_L2: return {TM_WORK, HID, HID / 16, 0, MMFF_KM(SM_H1, HID), MMFF_KM(SM_W2, HID)};
        case OP_L3: return {TM_WORK, NOP, HID / 16, 0, MMFF_KM(SM_H2, HID), MMFF_KM(SM_W3, HID)};
        // dW3^T += H2^T dY  (M = hidden, N = out, reduction over the tile's atoms)
        case OP_DW3: return {TM_DW3, NOP, TILE / 16, 1, MMFF_MN(SM_H2, HID), MMFF_MN(SM_DY, NOP)};
        // dH2 = dY W3  (reduction over the 16 padded outputs)
        case OP_DH2: return {TM_WORK, HID, NOP / 16, 0, MMFF_KM(SM_DY, NOP), MMFF_MN(SM_W3, HID)};
        // dW2 += dZ2^T H1, db2 += dZ2^T 1
        case OP_DW2: return {TM_DW2, HID, TILE / 16, 1, MMFF_MN(SM_S2, HID), MMFF_MN(SM_H1, HID)};
        case OP_DB2: return {TM_DB2, NOP, TILE / 16, 1, MMFF_MN(SM_S2, HID), MMFF_KM(SM_ONE, TILE)};
        // dH1 = dZ2 W2
        case OP_DH1: return {TM_WORK, HID, HID / 16, 0, MMFF_KM(SM_S2, HID), MMFF_MN(SM_W2, HID)};
        // dW1 += dZ1^T X, db1 += dZ1^T 1  (dZ1 lives in the H2 buffer)
        case OP_DW1: return {TM_DW1, K0, TILE / 16, 1, MMFF_MN(SM_H2, HID), MMFF_MN(SM_X, K0)};
        default: return {TM_DB1, NOP, TILE / 16, 1, MMFF_MN(SM_H2, HID), MMFF_KM(SM_ONE, TILE)};
    }
}

// shared-memory matrix descriptor (tcgen05 "matrix descriptor"): start, leading
// and stride byte offsets in 16-byte units, version 1 (bits 46-47), base
// offset 0, SWIZZLE_NONE (bits 61-63 = 0)
MMFF_HD inline uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor, kind::f16: D format F32 (bits 4-5), A and B BF16
// (bits 7-9, 10-12), A/B major (bits 15, 16), N/8 (bits 17-22), M/16 (bits 24-28)
MMFF_HD inline uint32_t instr_desc(int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}

}  // namespace mlp
}  // namespace mmff
