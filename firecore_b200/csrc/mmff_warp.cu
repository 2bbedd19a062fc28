// mmff_warp.cu -- warp-per-system relaxation for systems of up to 64 atoms.
//
// One warp owns one system.  Lane l owns atoms {l, l+32} (APL = atoms per
// lane, 1 or 2), the pi orbitals of nodes {l, l+32} and their velocities
// (kept in registers across the whole relaxation).  Shared memory per warp
// holds only what other lanes read: positions (atoms + pi), non-bonded
// parameters and the node recoil slots.  A FIRE step is
//   bonded (own nodes) -> pair sum (own atoms x all j, smem broadcast,
//   64-bit exclusion masks) -> B-spline GridFF (own atoms, 64 float4 L2
//   gathers each) -> __syncwarp -> recoil assembly -> FP64 warp reductions
//   -> FIRE scalars (FP64, once per warp) -> move -> __syncwarp
// with no block-level barrier, so the SM interleaves many independent
// systems.  Physics is identical to mmff_relax.cu (same device functions,
// same order of operations per term); see mmff_device.cuh for the reference
// file:line of every term.
#include "mmff_device.cuh"
#include <cfloat>

namespace mmff {

__device__ __forceinline__ double wsum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float wmax_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float wmin_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// MMFFsp3_loc::eval_atom (MMFFsp3_loc.h:250-575) for node ia, same arithmetic as
// mmff_device.cuh eval_atom, but every recoil contribution goes straight into
// the node's own slots in shared memory (only this lane touches them), which
// keeps the register footprint small.  fbs: sigma slots of the node, fps: pi.
template <bool ENERGY>
__device__ __forceinline__ float eval_atom_slots(int ia, int natoms, int nnode, int flags, float Fmax2,
                                                 const float4* sp, const float4* sREQ, int4 ng, int4 ngC,
                                                 const float4* gap, const float* gbL, const float* gbK,
                                                 const float* gKsp, const float* gKpp, const float* lv, int npx, int npy,
                                                 int npz, int a13, const Cut13& cu, float4* fbs, float4* fps,
                                                 float3& fa_out, float3& fpi_out, float& E13) {
    const float3 pa = f3(sp[ia]);
    const float3 hpi = f3(sp[natoms + ia]);
    const float4 apar = *gap;
    float3 fa = make_float3(0, 0, 0), fpi = make_float3(0, 0, 0);
    float3 hf[4];
    float he[4], hl[4];
    float E = 0.f;
    E13 = 0.f;
    const int ings[4] = {ng.x, ng.y, ng.z, ng.w};
    const int ingC[4] = {ngC.x, ngC.y, ngC.z, ngC.w};
    auto addslot = [](float4* slot, float3 v) { float4 t = *slot; t.x += v.x; t.y += v.y; t.z += v.z; *slot = t; };
#pragma unroll
    for (int i = 0; i < 4; i++) { fbs[i] = make_float4(0, 0, 0, 0); fps[i] = make_float4(0, 0, 0, 0); hf[i] = make_float3(0, 0, 1); he[i] = 1.f; hl[i] = 1.f; }
    int nb = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int ing = ings[i];
        if (ing < 0) break;
        nb = i + 1;
        float3 h = f3(sp[ing]) - pa;
        if (flags & F_PBC) {
            const int c = ingC[i];
            const float3 cell = image_cell(c, npx, npy, npz);
            const float ix = cell.x, iy = cell.y, iz = cell.z;
            h.x += lv[0] * ix + lv[3] * iy + lv[6] * iz;
            h.y += lv[1] * ix + lv[4] * iy + lv[7] * iz;
            h.z += lv[2] * ix + lv[5] * iy + lv[8] * iz;
        }
        const float l2 = dot3(h, h);
        const float il = rsqrtf(l2);
        const float l = l2 * il;
        h = h * il;
        hf[i] = h; he[i] = il; hl[i] = l;
        if (ia < ing) {
            if (flags & F_BONDS) {
                const float dl = l - gbL[i];
                const float fr = dl * gbK[i];
                float3 f1 = h * fr;
                if (ENERGY) E += fr * dl * 0.5f;
                if (flags & F_SUB_BOND_NB) {
                    const float4 Ri = sREQ[ia], Rj = sREQ[ing];
                    float e;
                    const float F = ljqh<ENERGY>(l * l, Ri.x + Rj.x, Ri.y * Rj.y, Ri.z * Rj.z, fminf(Ri.w * Rj.w, 0.f), e);
                    float3 fij = (h * l) * F;
                    if (flags & F_CLAMP_NB) { float f2 = dot3(fij, fij); if (f2 > Fmax2) fij = fij * sqrtf(Fmax2 / f2); }
                    if (ENERGY) E -= e;
                    f1 = f1 - fij;
                }
                addslot(fbs + i, make_float3(-f1.x, -f1.y, -f1.z));
                fa = fa + f1;
            }
            const float kk = gKpp[i];
            if ((flags & F_PIPI) && (ing < nnode) && (kk > 1e-6f)) {
                const float3 h2 = f3(sp[natoms + ing]);
                float c = dot3(hpi, h2);
                const float3 a = fma3(hpi, -c, h2);
                const float3 b = fma3(h2, -c, hpi);
                const bool sign = c < 0.f;
                if (sign) c = -c;
                if (ENERGY) E += kk * (1.f - c);
                const float fang = sign ? -kk : kk;
                fpi = fpi + a * fang;
                addslot(fps + i, b * fang);
            }
        }
        const float ks = gKsp[i];
        if ((flags & F_PISIGMA) && (ks > 1e-6f)) {
            const float c = dot3(hpi, h);
            const float3 a = fma3(hpi, -c, h);
            const float3 b = fma3(h, -c, hpi);
            const float c_ = c - apar.w;
            if (ENERGY) E += ks * c_ * c_;
            const float fang = -ks * c_ * 2.f;
            fpi = fpi + a * fang;
            const float3 f2 = b * (fang * il);
            fa = fa - f2;
            addslot(fbs + i, f2);
        }
    }
    if (flags & F_ANGLES) {
        const float ssK = apar.z;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (i >= nb) break;
#pragma unroll
            for (int j = i + 1; j < 4; j++) {
                if (j >= nb) break;
                const float3 h = hf[i] + hf[j];
                float c2 = dot3(h, h) * 0.25f;
                const float s2 = 1.f - c2 + 1e-14f;
                const float c = sqrtf(c2);
                const float s = sqrtf(fmaxf(s2, 0.f));
                const float csx = fmaf(apar.x, c, apar.y * s);
                const float csy = fmaf(apar.y, c, -apar.x * s);
                if (ENERGY) E += ssK * (1.f - csx);
                float fr = -ssK * csy;
                c2 *= -2.f;
                fr = __fdividef(fr, 4.f * c * s);
                const float fr1 = fr * he[i];
                const float fr2 = fr * he[j];
                float3 f1 = make_float3(h.x * fr1 + hf[i].x * (fr1 * c2), h.y * fr1 + hf[i].y * (fr1 * c2), h.z * fr1 + hf[i].z * (fr1 * c2));
                float3 f2 = make_float3(h.x * fr2 + hf[j].x * (fr2 * c2), h.y * fr2 + hf[j].y * (fr2 * c2), h.z * fr2 + hf[j].z * (fr2 * c2));
                fa = fa - (f1 + f2);
                if (flags & F_SUB_ANGLE_NB) {
                    const float3 dp = hf[j] * hl[j] - hf[i] * hl[i];
                    // x13: the pair sum skipped this central-image pair (pair13, mmff_device.cuh)
                    const bool x13 = (flags & F_EXCL13) && ((a13 >> angle_slot(i, j)) & 1) &&
                                     (!(flags & F_PBC) || ingC[i] == ingC[j]);
                    float e = 0.f, ep = 0.f;
                    const float F = pair13<ENERGY>(dot3(dp, dp), sREQ[ings[i]], sREQ[ings[j]], x13, cu.Rc2, cu.kq, cu.rc, e, ep);
                    float3 fij = dp * F;
                    if (flags & F_CLAMP_NB) { float ff = dot3(fij, fij); if (ff > Fmax2) fij = fij * sqrtf(Fmax2 / ff); }
                    if (ENERGY) { E += e; E13 += ep; }
                    f1 = f1 + fij;
                    f2 = f2 - fij;
                }
                addslot(fbs + i, f1);
                addslot(fbs + j, f2);
            }
        }
    }
    fa_out = fa; fpi_out = fpi;
    return E;
}

// pair-sum inner loop over all j for (up to) two owned atoms, one image.
// One code path for cutoff / no cutoff keeps the instruction footprint small
// (the kernel is instruction-fetch bound otherwise): without a cutoff Rc2 is
// +inf and kq 0.  HB: the system has H-bond pseudo-charges (a warp-uniform
// choice; without them the H term is identically 0 and is not evaluated).
// Excluded and out-of-range pairs get r^2 = 1e30: every term then underflows
// to zero except the shifted-force constant kq Q / r, below 1e-16 eV/A, so no
// final select is needed.
template <int APL, bool ENERGY, bool COUNT, bool HB>
__device__ __forceinline__ void pair_image(const Params& P, int N, const float4* __restrict__ sp,
                                           const float4* __restrict__ sR, float3 p0, float3 p1, float4 R0i,
                                           float4 R1i, uint32_t m0lo, uint32_t m0hi, uint32_t m1lo, uint32_t m1hi,
                                           float3& f0, float3& f1, float& e0, float& e1, unsigned long long& np) {
    const bool CUT = P.Rc2 > 0.f;
    const float Rc2 = CUT ? P.Rc2 : 3.0e38f, kq = P.kq_rc2;
    const float rc = CUT ? sqrtf(1.f / kq) : 0.f;
    for (int j = 0; j < N; j++) {
        const float4 pj = sp[j];
        const float4 Rj = sR[j];
        const uint32_t b = 1u << (j & 31);
        // atom 0
        {
            const float dx = pj.x - p0.x, dy = pj.y - p0.y, dz = pj.z - p0.z;
            float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool ok = (((j < 32 ? m0lo : m0hi) & b) == 0) && (r2 < Rc2);
            r2 = ok ? r2 : 1e30f;
            const float ir = rsqrtf(r2);
            const float ir2 = ir * ir;
            const float R0 = R0i.x + Rj.x;
            const float E0 = R0i.y * Rj.y;
            const float Q = R0i.z * Rj.z;
            const float Eel = Q * ir;
            const float u2 = R0 * R0 * ir2;
            const float u6 = u2 * u2 * u2;
            const float vdW = u6 * E0;
            const float H = HB ? u6 * vdW * fminf(R0i.w * Rj.w, 0.f) : 0.f;
            float F = -fmaf(12.f * ir2, HB ? fmaf(u6 - 1.f, vdW, H) : (u6 - 1.f) * vdW, Eel * ir2);
            F = fmaf(Q * kq, ir, F);
            f0.x = fmaf(dx, F, f0.x); f0.y = fmaf(dy, F, f0.y); f0.z = fmaf(dz, F, f0.z);
            if (ENERGY && ok) {
                float e = fmaf(u6 - 2.f, vdW, Eel + H);
                if (CUT) e += Q * kq * (r2 * ir - 2.f * rc);
                e0 += e;
            }
            if (COUNT && ok) np++;
        }
        if (APL == 2) {
            const float dx = pj.x - p1.x, dy = pj.y - p1.y, dz = pj.z - p1.z;
            float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool ok = (((j < 32 ? m1lo : m1hi) & b) == 0) && (r2 < Rc2);
            r2 = ok ? r2 : 1e30f;
            const float ir = rsqrtf(r2);
            const float ir2 = ir * ir;
            const float R0 = R1i.x + Rj.x;
            const float E0 = R1i.y * Rj.y;
            const float Q = R1i.z * Rj.z;
            const float Eel = Q * ir;
            const float u2 = R0 * R0 * ir2;
            const float u6 = u2 * u2 * u2;
            const float vdW = u6 * E0;
            const float H = HB ? u6 * vdW * fminf(R1i.w * Rj.w, 0.f) : 0.f;
            float F = -fmaf(12.f * ir2, HB ? fmaf(u6 - 1.f, vdW, H) : (u6 - 1.f) * vdW, Eel * ir2);
            F = fmaf(Q * kq, ir, F);
            f1.x = fmaf(dx, F, f1.x); f1.y = fmaf(dy, F, f1.y); f1.z = fmaf(dz, F, f1.z);
            if (ENERGY && ok) {
                float e = fmaf(u6 - 2.f, vdW, Eel + H);
                if (CUT) e += Q * kq * (r2 * ir - 2.f * rc);
                e1 += e;
            }
            if (COUNT && ok) np++;
        }
    }
}

// Central-image pairs, each unordered pair once (Newton's third law).  Lane l
// owns atoms A = l and B = l + 32; at rotation step s it meets the atoms of
// lane p = l + s (mod 32): (A, A') and (B, B') for s = 1..15 (s = 16: lanes
// l < 16 only), (A, B') for s = 1..16, (B, A') for s = 1..15, and (A, B) of
// its own lane at s = 0 - every pair of the 64 slots exactly once.  The
// reaction forces on the partner's atoms travel back by one shuffle per
// component.  Exclusions come from the own atom's mask (bonded neighbours in
// the central cell are symmetric in MMFFsp3_loc topologies); slots >= N are
// masked.  Energies are full pair energies (not halved).
template <bool ENERGY, bool COUNT, bool HB>
__device__ __forceinline__ void central_pairs(const Params& P, int N, int lane, const float4* __restrict__ sp,
                                              const float4* __restrict__ sR, uint32_t m0lo, uint32_t m0hi,
                                              uint32_t m1lo, uint32_t m1hi, float3& f0, float3& f1, float& ec,
                                              unsigned long long& np) {
    const bool CUT = P.Rc2 > 0.f;
    const float Rc2 = CUT ? P.Rc2 : 3.0e38f, kq = P.kq_rc2;
    const float rc = CUT ? sqrtf(1.f / kq) : 0.f;
    const int a0 = lane, a1 = lane + 32;
    const float4 q0 = sp[min(a0, N - 1)], q1 = sp[min(a1, N - 1)];
    const float4 R0 = sR[min(a0, N - 1)], R1 = sR[min(a1, N - 1)];
    // slots beyond the system are excluded for everybody
    const uint32_t inv_lo = (N >= 32) ? 0u : ~((1u << N) - 1u);
    const uint32_t inv_hi = (N >= 64) ? 0u : (N <= 32 ? ~0u : ~((1u << (N - 32)) - 1u));
    m0lo |= inv_lo; m0hi |= inv_hi; m1lo |= inv_lo; m1hi |= inv_hi;
    if (a0 >= N) { m0lo = ~0u; m0hi = ~0u; }
    if (a1 >= N) { m1lo = ~0u; m1hi = ~0u; }
    bool ok;
    float e = 0.f;
    {   // s = 0: (A, B) of this lane
        const float dx = q1.x - q0.x, dy = q1.y - q0.y, dz = q1.z - q0.z;
        const float F = pair_force<ENERGY, HB>(dx, dy, dz, R0, R1, (m0hi >> lane) & 1u, Rc2, kq, rc, CUT, ok, e);
        f0.x = fmaf(dx, F, f0.x); f0.y = fmaf(dy, F, f0.y); f0.z = fmaf(dz, F, f0.z);
        f1.x = fmaf(-dx, F, f1.x); f1.y = fmaf(-dy, F, f1.y); f1.z = fmaf(-dz, F, f1.z);
        if (ENERGY) ec += e;
        if (COUNT && ok) np += 2;
    }
#ifndef MMFF_CENTRAL_UNROLL
#define MMFF_CENTRAL_UNROLL 1
#endif
    constexpr int kUnroll = MMFF_CENTRAL_UNROLL;      // rotation-step unrolling (build option)
#pragma unroll kUnroll
    for (int s = 1; s <= 16; s++) {
        const int p = (lane + s) & 31;
        const int src = (lane - s) & 31;      // lane whose partner is this lane
        const bool half = (s < 16) || (lane < 16);
        {   // partner atom A' = p: pairs (A, A') and (B, A')
            const float4 qA = sp[min(p, N - 1)], RA = sR[min(p, N - 1)];
            float3 rA = make_float3(0.f, 0.f, 0.f);
            {
                const float dx = qA.x - q0.x, dy = qA.y - q0.y, dz = qA.z - q0.z;
                const float F = pair_force<ENERGY, HB>(dx, dy, dz, R0, RA, ((m0lo >> p) & 1u) || !half, Rc2, kq, rc, CUT, ok, e);
                f0.x = fmaf(dx, F, f0.x); f0.y = fmaf(dy, F, f0.y); f0.z = fmaf(dz, F, f0.z);
                rA.x = -dx * F; rA.y = -dy * F; rA.z = -dz * F;
                if (ENERGY) ec += e;
                if (COUNT && ok) np += 2;
            }
            {   // s = 16: this is (A', B) of lane p, done there
                const float dx = qA.x - q1.x, dy = qA.y - q1.y, dz = qA.z - q1.z;
                const float F = pair_force<ENERGY, HB>(dx, dy, dz, R1, RA, ((m1lo >> p) & 1u) || (s == 16), Rc2, kq, rc, CUT, ok, e);
                f1.x = fmaf(dx, F, f1.x); f1.y = fmaf(dy, F, f1.y); f1.z = fmaf(dz, F, f1.z);
                rA.x = fmaf(-dx, F, rA.x); rA.y = fmaf(-dy, F, rA.y); rA.z = fmaf(-dz, F, rA.z);
                if (ENERGY) ec += e;
                if (COUNT && ok) np += 2;
            }
            f0.x += __shfl_sync(0xffffffffu, rA.x, src); f0.y += __shfl_sync(0xffffffffu, rA.y, src);
            f0.z += __shfl_sync(0xffffffffu, rA.z, src);
        }
        {   // partner atom B' = p + 32: pairs (B, B') and (A, B')
            const float4 qB = sp[min(p + 32, N - 1)], RB = sR[min(p + 32, N - 1)];
            float3 rB = make_float3(0.f, 0.f, 0.f);
            {
                const float dx = qB.x - q1.x, dy = qB.y - q1.y, dz = qB.z - q1.z;
                const float F = pair_force<ENERGY, HB>(dx, dy, dz, R1, RB, ((m1hi >> p) & 1u) || !half, Rc2, kq, rc, CUT, ok, e);
                f1.x = fmaf(dx, F, f1.x); f1.y = fmaf(dy, F, f1.y); f1.z = fmaf(dz, F, f1.z);
                rB.x = -dx * F; rB.y = -dy * F; rB.z = -dz * F;
                if (ENERGY) ec += e;
                if (COUNT && ok) np += 2;
            }
            {
                const float dx = qB.x - q0.x, dy = qB.y - q0.y, dz = qB.z - q0.z;
                const float F = pair_force<ENERGY, HB>(dx, dy, dz, R0, RB, (m0hi >> p) & 1u, Rc2, kq, rc, CUT, ok, e);
                f0.x = fmaf(dx, F, f0.x); f0.y = fmaf(dy, F, f0.y); f0.z = fmaf(dz, F, f0.z);
                rB.x = fmaf(-dx, F, rB.x); rB.y = fmaf(-dy, F, rB.y); rB.z = fmaf(-dz, F, rB.z);
                if (ENERGY) ec += e;
                if (COUNT && ok) np += 2;
            }
            f1.x += __shfl_sync(0xffffffffu, rB.x, src); f1.y += __shfl_sync(0xffffffffu, rB.y, src);
            f1.z += __shfl_sync(0xffffffffu, rB.z, src);
        }
    }
}

// exclusion bits of atom a for image ipbc: itself (every image, NBFF.h:590) and
// its bonded neighbours whose cell is ipbc (NBFF.h:593-607); without PBC every
// bonded neighbour (NBFF::evalLJQs_ng4_atom_omp)
__device__ __forceinline__ void excl_mask(int a, int4 ng, int4 ngC, int ipbc, bool pbc, uint32_t& lo, uint32_t& hi) {
    lo = 0; hi = 0;
    auto setb = [&](int j) { if (j >= 0) { if (j < 32) lo |= 1u << j; else hi |= 1u << (j - 32); } };
    setb(a);
    if (!pbc || ngC.x == ipbc) setb(ng.x);
    if (!pbc || ngC.y == ipbc) setb(ng.y);
    if (!pbc || ngC.z == ipbc) setb(ng.z);
    if (!pbc || ngC.w == ipbc) setb(ng.w);
}

template <int APL, bool ENERGY, bool COUNT>
struct WarpEngine {
    const Params& P;
    const Systems& Y;
    float4* sp;      // [maxNA+maxNN] positions (atoms, then pi)
    float4* sR;      // [maxNA]
    float4* fng;     // [8*maxNN]  sigma slots [4*maxNN], pi slots after
    int4* sng;       // [maxNA] neighbours, cells, back-neighbours
    int4* sngC;
    int4* sbk;
    float4* spar;    // [5*maxNN] node parameters: apars, bLs, bKs, Ksp, Kpp (node-major)
    int maxNN;
    int lane;
    // current system
    int isys, N, NN, NV, aoff, noff, voff;
    float* lv;       // [9] lattice vectors, then 3 floats grid offset, in the warp's region
    bool hasH;
    // owned state (k = 0, 1): atom a_k = lane + 32k, node n_k = a_k if < NN
    float3 va[APL], vp[APL];        // velocities of own atoms / own pi vectors
    float3 fasm_a[APL], fasm_p[APL];// assembled forces of the current step
    const uint32_t* xrow;           // central-image exclusion rows of the system (ceil(N/32) words per atom)
    int nbw;                        // words per row
    double e13 = 0.0;               // ENERGY: pair energies of the skipped 1-3 pairs (energy split)
    unsigned long long npair = 0;

    __device__ WarpEngine(const Params& p, const Systems& y, char* region, const WarpLayout& L, int maxNN_)
        : P(p), Y(y), maxNN(maxNN_) {
        sp = reinterpret_cast<float4*>(region + L.pos);
        sR = reinterpret_cast<float4*>(region + L.REQ);
        fng = reinterpret_cast<float4*>(region + L.fng);
        lv = reinterpret_cast<float*>(region + L.misc);
        sng = reinterpret_cast<int4*>(region + L.ng);
        sngC = reinterpret_cast<int4*>(region + L.ngC);
        sbk = reinterpret_cast<int4*>(region + L.bk);
        spar = reinterpret_cast<float4*>(region + L.npar);
        lane = threadIdx.x & 31;
    }

    __device__ void load(int s) {
        isys = s;
        const int4 d = Y.desc[s];
        aoff = d.x; noff = d.y; voff = d.z; N = d.w;
        NN = Y.nnode[s]; NV = N + NN;
        xrow = Y.xmask + Y.moff[s];
        nbw = (N + 31) >> 5;
        if (lane < 9) lv[lane] = Y.lvec[9 * s + lane];
        if (lane >= 9 && lane < 12) lv[lane] = comp(Y.gorg[s], lane - 9);
        bool h = false;
        for (int v = lane; v < NV; v += 32) sp[v] = Y.pos[voff + v];
        for (int a = lane; a < N; a += 32) {
            const float4 r = Y.REQ[aoff + a]; sR[a] = r; h |= (r.w != 0.f);
            sng[a] = Y.neighs[aoff + a]; sngC[a] = Y.neighCell[aoff + a]; sbk[a] = Y.bkneighs[aoff + a];
        }
        for (int n = lane; n < NN; n += 32) {
            spar[5 * n + 0] = Y.apars[noff + n]; spar[5 * n + 1] = Y.bLs[noff + n]; spar[5 * n + 2] = Y.bKs[noff + n];
            spar[5 * n + 3] = Y.Ksp[noff + n]; spar[5 * n + 4] = Y.Kpp[noff + n];
        }
        hasH = __any_sync(0xffffffffu, h);
#pragma unroll
        for (int k = 0; k < APL; k++) {
            const int a = lane + 32 * k;
            const bool va_ok = a < N, vp_ok = a < NN;
            const float4 v1 = va_ok ? Y.vel[voff + a] : make_float4(0, 0, 0, 0);
            const float4 v2 = vp_ok ? Y.vel[voff + N + a] : make_float4(0, 0, 0, 0);
            va[k] = f3(v1); vp[k] = f3(v2);
        }
        __syncwarp();
    }

    // bounding box of the atoms (identical in all lanes)
    __device__ void bbox(float* mn, float* mx) {
        float a[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, b[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = lane; i < N; i += 32) {
            const float4 p = sp[i];
            a[0] = fminf(a[0], p.x); a[1] = fminf(a[1], p.y); a[2] = fminf(a[2], p.z);
            b[0] = fmaxf(b[0], p.x); b[1] = fmaxf(b[1], p.y); b[2] = fmaxf(b[2], p.z);
        }
#pragma unroll
        for (int k = 0; k < 3; k++) { mn[k] = wmin_f(a[k]); mx[k] = wmax_f(b[k]); }
    }

    // central-image exclusion words of atom a (all set beyond the system)
    __device__ __forceinline__ void central_rows(int a, uint32_t& lo, uint32_t& hi) const {
        if (a >= N) { lo = hi = ~0u; return; }
        lo = __ldg(xrow + a * nbw);
        hi = nbw > 1 ? __ldg(xrow + a * nbw + 1) : ~0u;
    }

    // forces of one step; assembled forces of owned vectors end in fasm_a/fasm_p
    __device__ void forces(double& Eb, double& Enb, double& Eg) {
        const int flags = P.flags;
        // ---- bonded, own nodes
        float3 fa_own[APL], fpi_own[APL];
#pragma unroll
        for (int k = 0; k < APL; k++) {
            fa_own[k] = make_float3(0, 0, 0); fpi_own[k] = make_float3(0, 0, 0);
            const int ia = lane + 32 * k;
            if (ia < NN) {
                const float4* np_ = spar + 5 * ia;
                float E13;
                const float e = eval_atom_slots<ENERGY>(
                    ia, N, NN, flags, P.Fmax2NB, sp, sR, sng[ia], sngC[ia], np_, reinterpret_cast<const float*>(np_ + 1),
                    reinterpret_cast<const float*>(np_ + 2), reinterpret_cast<const float*>(np_ + 3),
                    reinterpret_cast<const float*>(np_ + 4), lv, P.npbc[0], P.npbc[1], P.npbc[2],
                    __ldg(Y.a13 + noff + ia), Cut13(P), fng + ia * 4, fng + 4 * maxNN + ia * 4, fa_own[k], fpi_own[k],
                    E13);
                if (ENERGY) { Eb += (double)e; e13 += (double)E13; }
            }
        }
        // ---- pairs, own atoms x all j
        float3 f0 = make_float3(0, 0, 0), f1 = make_float3(0, 0, 0);
        if (flags & F_NONBONDED) {
            const bool pbc = (flags & F_PBC) != 0;
            const int npx = pbc ? P.npbc[0] : 0, npy = pbc ? P.npbc[1] : 0, npz = pbc ? P.npbc[2] : 0;
            const int nxi = 2 * npx + 1, nyi = 2 * npy + 1;
            const bool cut = P.Rc2 > 0.f;
            float mn[3], mx[3];
            if (cut && (npx | npy | npz)) bbox(mn, mx);
            const int a0 = lane, a1 = lane + 32;
            const float4 q0 = a0 < N ? sp[a0] : make_float4(0, 0, 0, 0);
            const float4 q1 = (APL == 2 && a1 < N) ? sp[a1] : make_float4(0, 0, 0, 0);
            const float4 Ri0 = a0 < N ? sR[a0] : make_float4(0, 0, 0, 0);
            const float4 Ri1 = (APL == 2 && a1 < N) ? sR[a1] : make_float4(0, 0, 0, 0);
            float e0 = 0.f, e1 = 0.f, ec = 0.f;
            for (int iz = -npz; iz <= npz; iz++)
                for (int iy = -npy; iy <= npy; iy++)
                    for (int ix = -npx; ix <= npx; ix++) {
                        const float shx = lv[0] * ix + lv[3] * iy + lv[6] * iz;
                        const float shy = lv[1] * ix + lv[4] * iy + lv[7] * iz;
                        const float shz = lv[2] * ix + lv[5] * iy + lv[8] * iz;
                        if (cut && (ix | iy | iz)) {
                            const float gx = fmaxf(0.f, fabsf(shx) - (mx[0] - mn[0]));
                            const float gy = fmaxf(0.f, fabsf(shy) - (mx[1] - mn[1]));
                            const float gz = fmaxf(0.f, fabsf(shz) - (mx[2] - mn[2]));
                            if (gx * gx + gy * gy + gz * gz >= P.Rc2) continue;   // image out of reach (uniform)
                        }
                        const int ipbc = ((iz + npz) * nyi + (iy + npy)) * nxi + (ix + npx);
                        uint32_t m0lo, m0hi, m1lo, m1hi;
                        if ((ix | iy | iz) == 0) {      // central image: the exclusion rows (bonded and 1-3 pairs)
                            central_rows(a0, m0lo, m0hi);
                            if (APL == 2) central_rows(a1, m1lo, m1hi); else { m1lo = m1hi = ~0u; }
                        } else {
                            if (a0 < N) excl_mask(a0, sng[a0], sngC[a0], ipbc, pbc, m0lo, m0hi); else { m0lo = m0hi = ~0u; }
                            if (APL == 2 && a1 < N) excl_mask(a1, sng[a1], sngC[a1], ipbc, pbc, m1lo, m1hi); else { m1lo = m1hi = ~0u; }
                        }
                        if (APL == 2 && (ix | iy | iz) == 0) {      // central image: each pair once
                            if (hasH) central_pairs<ENERGY, COUNT, true>(P, N, lane, sp, sR, m0lo, m0hi, m1lo, m1hi, f0, f1, ec, npair);
                            else central_pairs<ENERGY, COUNT, false>(P, N, lane, sp, sR, m0lo, m0hi, m1lo, m1hi, f0, f1, ec, npair);
                            continue;
                        }
                        const float3 p0 = make_float3(q0.x - shx, q0.y - shy, q0.z - shz);
                        const float3 p1 = make_float3(q1.x - shx, q1.y - shy, q1.z - shz);
                        if (hasH)
                            pair_image<APL, ENERGY, COUNT, true>(P, N, sp, sR, p0, p1, Ri0, Ri1, m0lo, m0hi, m1lo, m1hi, f0, f1, e0, e1, npair);
                        else
                            pair_image<APL, ENERGY, COUNT, false>(P, N, sp, sR, p0, p1, Ri0, Ri1, m0lo, m0hi, m1lo, m1hi, f0, f1, e0, e1, npair);
                    }
            if (ENERGY) Enb += 0.5 * ((double)e0 + (double)e1) + (double)ec;
        }
        // ---- GridFF, own atoms
        float3 g0 = make_float3(0, 0, 0), g1 = make_float3(0, 0, 0);
        if (flags & F_GRID) {
#pragma unroll
            for (int k = 0; k < APL; k++) {
                const int a = lane + 32 * k;
                if (a < N) {
                    const float4 p = sp[a];
                    const float3 u = make_float3((p.x + lv[9]) * P.ginv[0], (p.y + lv[10]) * P.ginv[1], (p.z + lv[11]) * P.ginv[2]);
                    const float4 r = grid_atom(P, u, __ldg(&Y.PLQ[aoff + a]));
                    if (k == 0) g0 = make_float3(r.x, r.y, r.z); else g1 = make_float3(r.x, r.y, r.z);
                    if (ENERGY) Eg += (double)r.w;
                }
            }
        }
        if (flags & F_SURF) {           // direct substrate term (getSurfMorse)
#pragma unroll
            for (int k = 0; k < APL; k++) {
                const int a = lane + 32 * k;
                if (a < N) {
                    const float4 p = sp[a];
                    const float4 r = surf_atom(P, make_float3(p.x + lv[9], p.y + lv[10], p.z + lv[11]), sR[a]);
                    if (k == 0) g0 = g0 + make_float3(r.x, r.y, r.z); else g1 = g1 + make_float3(r.x, r.y, r.z);
                    if (ENERGY) Eg += (double)r.w;
                }
            }
        }
        __syncwarp();   // recoil slots of every node written
        // ---- assembly (MMFFsp3_loc::assemble_atom)
#pragma unroll
        for (int k = 0; k < APL; k++) {
            const int a = lane + 32 * k;
            float3 f = fa_own[k];
            const int4 bkk = (a < N) ? sbk[a] : make_int4(-1, -1, -1, -1);
            if (a < N) {
                f = f + (k == 0 ? f0 : f1) + (k == 0 ? g0 : g1);
                const int bks[4] = {bkk.x, bkk.y, bkk.z, bkk.w};
#pragma unroll
                for (int q = 0; q < 4; q++) { if (bks[q] < 0) break; f = f + f3(fng[bks[q]]); }
            }
            fasm_a[k] = f;
            float3 fp = fpi_own[k];
            if (a < NN) {
                const int bks[4] = {bkk.x, bkk.y, bkk.z, bkk.w};
#pragma unroll
                for (int q = 0; q < 4; q++) { if (bks[q] < 0) break; fp = fp + f3(fng[4 * maxNN + bks[q]]); }
                const float3 u = f3(sp[N + a]);
                fp = fma3(u, -dot3(fp, u), fp);
            }
            fasm_p[k] = fp;
        }
    }

    // clamp + FIRE sums of owned vectors, then warp totals (identical in all lanes)
    __device__ void fire_sums(double& vf, double& vv, double& ff, float& fmax2, bool& bad) {
        const float Fl = P.Flim;
        vf = 0; vv = 0; ff = 0; fmax2 = 0.f; bool b = false;
#pragma unroll
        for (int k = 0; k < APL; k++) {
            const int a = lane + 32 * k;
#pragma unroll
            for (int w = 0; w < 2; w++) {
                const bool valid = (w == 0) ? (a < N) : (a < NN);
                if (!valid) continue;
                float3 f = (w == 0) ? fasm_a[k] : fasm_p[k];
                const float3 v = (w == 0) ? va[k] : vp[k];
                if ((P.flags & F_BCONS) && w == 0) f = bond_constraint_force(Y, isys, a, sp, lv, f);
                if (Fl > 0.f) {
                    const float fr2 = dot3(f, f);
                    if (fr2 > Fl * Fl) f = f * (Fl * rsqrtf(fr2));
                }
                if ((P.flags & F_CONSTR) && w == 0) f = constraint_force(Y, aoff + a, f3(sp[a]), f);
                // a system whose atoms left any sensible range is retired like a non-finite one
                if (w == 0) { const float4 p = sp[a]; b |= !(fabsf(p.x) + fabsf(p.y) + fabsf(p.z) < 1e5f); }
                if (w == 0) fasm_a[k] = f; else fasm_p[k] = f;
                vf += (double)v.x * f.x + (double)v.y * f.y + (double)v.z * f.z;
                vv += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z;
                const double f2 = (double)f.x * f.x + (double)f.y * f.y + (double)f.z * f.z;
                ff += f2;
                fmax2 = fmaxf(fmax2, (float)f2);
                b |= !isfinite(f.x + f.y + f.z);
            }
        }
        vf = wsum_d(vf); vv = wsum_d(vv); ff = wsum_d(ff); fmax2 = wmax_f(fmax2);
        bad = __any_sync(0xffffffffu, b);
    }

    __device__ void move(double dt, double cv, double cfm) {
        const float dtf = (float)dt;
        const float cvf = (float)cv;
        const float kf = (float)((double)dtf + cfm);
#pragma unroll
        for (int k = 0; k < APL; k++) {
            const int a = lane + 32 * k;
            if (a < N) {
                float3 v = va[k] * cvf;
                v = fma3(fasm_a[k], kf, v);
                float3 p = f3(sp[a]);
                p = fma3(v, dtf, p);
                sp[a] = make_float4(p.x, p.y, p.z, 0.f);
                va[k] = v;
            }
            if (a < NN) {
                float3 p = f3(sp[N + a]);
                float3 f = fasm_p[k];
                f = fma3(p, -dot3(p, f), f);
                float3 v = vp[k] * cvf;
                v = fma3(f, kf, v);
                v = fma3(p, -dot3(p, v), v);
                p = fma3(v, dtf, p);
                p = p * rsqrtf(dot3(p, p));
                sp[N + a] = make_float4(p.x, p.y, p.z, 0.f);
                vp[k] = v;
            }
        }
        __syncwarp();
    }

    // Langevin step (MMFFsp3_loc::move_atom_Langevin, MMFFsp3_loc.h:1191-1216)
    __device__ void move_md(int step) {
        const float dt = P.md_dt, g = P.md_gamma, nz = P.md_noise;
#pragma unroll
        for (int k = 0; k < APL; k++) {
            const int a = lane + 32 * k;
#pragma unroll
            for (int w = 0; w < 2; w++) {
                const bool valid = (w == 0) ? (a < N) : (a < NN);
                if (!valid) continue;
                const int v = (w == 0) ? a : N + a;
                float3 p = f3(sp[v]);
                float3 f = (w == 0) ? fasm_a[k] : fasm_p[k];
                float3 ve = (w == 0) ? va[k] : vp[k];
                if (w == 1) f = fma3(p, -dot3(p, f), f);
                f = fma3(ve, -g, f);
                const long long gv = (long long)voff + v;
                f.x = fmaf(langevin_rand(P.md_seed, gv, step, 0), nz, f.x);
                f.y = fmaf(langevin_rand(P.md_seed, gv, step, 1), nz, f.y);
                f.z = fmaf(langevin_rand(P.md_seed, gv, step, 2), nz, f.z);
                ve = fma3(f, dt, ve);
                if (w == 1) ve = fma3(p, -dot3(p, ve), ve);
                p = fma3(ve, dt, p);
                if (w == 1) p = p * rsqrtf(dot3(p, p));
                sp[v] = make_float4(p.x, p.y, p.z, 0.f);
                if (w == 0) va[k] = ve; else vp[k] = ve;
            }
        }
        __syncwarp();
    }

    // copy of the positions just moved (move ends with __syncwarp)
    __device__ void snapshot() {
        for (int v = lane; v < NV; v += 32) Y.minpos[voff + v] = sp[v];
    }

    __device__ void store(int status, int steps, float meas, double dt, double damping, int lastNeg, double total) {
        for (int v = lane; v < NV; v += 32) Y.pos[voff + v] = sp[v];
#pragma unroll
        for (int k = 0; k < APL; k++) {
            const int a = lane + 32 * k;
            if (a < N) { Y.vel[voff + a] = make_float4(va[k].x, va[k].y, va[k].z, 0.f); Y.force[voff + a] = make_float4(fasm_a[k].x, fasm_a[k].y, fasm_a[k].z, 0.f); }
            if (a < NN) { Y.vel[voff + N + a] = make_float4(vp[k].x, vp[k].y, vp[k].z, 0.f); Y.force[voff + N + a] = make_float4(fasm_p[k].x, fasm_p[k].y, fasm_p[k].z, 0.f); }
        }
        if (lane == 0) {
            Y.fire[isys] = make_double4(dt, damping, (double)lastNeg, total);
            Y.status[isys] = status;
            Y.nsteps[isys] = steps;
            Y.fconv[isys] = meas;
        }
    }
};

// Persistent: every warp claims systems from queue[] until it is empty.
// minimum resident CTAs per SM the register allocation targets (build option)
#ifndef MMFF_WARP_MINB
#define MMFF_WARP_MINB 4
#endif
// EXPL: the exploring cycle (P.md_mode 2) instead of plain FIRE or the drive.
template <int APL, bool COUNT, bool EXPL = false>
__global__ void __launch_bounds__(128, MMFF_WARP_MINB) relax_warp_kernel(Params P, Systems Y, const int* __restrict__ queue, int nqueue,
                                                         int* counter, int maxNA, int maxNN) {
    extern __shared__ __align__(16) char smem[];
    const WarpLayout L = warp_layout(maxNA, maxNN);
    char* region = smem + (threadIdx.x >> 5) * L.per_warp;
    WarpEngine<APL, false, COUNT> E(P, Y, region, L, maxNN);
    const int lane = threadIdx.x & 31;
    while (true) {
        int q = 0;
        if (lane == 0) q = atomicAdd(counter, 1);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= nqueue) break;
        const int s = queue[q];
        E.load(s);
        const double4 fs = Y.fire[s];
        double dt = fs.x, damping = fs.y, total = fs.w;
        int lastNeg = (int)fs.z;
        int status = ST_MAXSTEPS, itr = 0;
        float meas = 0.f;
        int ph = 0;                 // exploring cycle: 2 * (steps in the phase) + exploring
        if constexpr (EXPL) { const int4 g = Y.gopt[s]; ph = 2 * g.y + (g.x != 0); }
        for (itr = 0; itr < P.nstep_max; itr++) {
            bool lang = false;      // an exploring step (Langevin instead of FIRE)
            if constexpr (EXPL) {
                const int ev = explore_step(ph, P.n_explore, P.n_relax);
                lang = ev & 1;
                if ((ev & 2) && lane == 0) Y.gopt[s].w++;
            }
            double d0 = 0, d1 = 0, d2 = 0;
            E.forces(d0, d1, d2);
            double vf, vv, ff;
            float fmax2;
            bool bad;
            E.fire_sums(vf, vv, ff, fmax2, bad);
            if (bad) { status = ST_NAN; break; }
            if (!EXPL && P.md_mode) {   // Langevin drive: fixed number of steps, no FIRE
                E.move_md(P.md_step0 + itr);
                total += 1.0;
                meas = sqrtf(fmax2);
                continue;
            }
            // DynamicOpt::FIRE_update_params (DynamicOpt.cpp:250-267), FP64; in the
            // exploring cycle the FIRE scalars evolve in exploring steps too
            // (MolWorld_sp3.h:2401-2424)
            const double f_len = sqrt(ff), v_len = sqrt(vv);
            const double cos_vf = vf / (f_len * v_len + 1e-32);
            const double renorm_vf = v_len / (f_len + 1e-32);
            double cv, cf;
            if (cos_vf < 0.0) { cv = P.cv_kill; cf = 0.0; } else { cv = 1.0 - damping; cf = damping; }
            cf = renorm_vf * cf;
            if (cos_vf < 0.0) {
                dt = fmax(dt * P.fdec, P.dt_min);
                lastNeg = 0;
                damping = P.damp_max;
            } else {
                if (lastNeg > P.minLastNeg) { dt = fmin(dt * P.finc, P.dt_max); damping = damping * P.falpha; }
                lastNeg++;
            }
            if (EXPL && lang) E.move_md(P.md_step0 + itr);
            else E.move(dt, cv, P.fire_variant == 1 ? cf : renorm_vf * cf);
            total += 1.0;
            const double m = (P.conv_mode == 0) ? ff : (double)fmax2;
            meas = (float)sqrt(m);
            if constexpr (EXPL) {
                if (!lang && m < P.Fconv2) {
                    // a minimum (MolWorld_sp3.h:2465-2473): keep it, start exploring
                    E.snapshot();
                    if (lane == 0) Y.gopt[s].z++;
                    ph = 1;
                }
            } else {
                if (m < P.Fconv2) { status = ST_CONVERGED; itr++; break; }
            }
        }
        const int steps = (status == ST_CONVERGED) ? itr - 1 : itr;
        E.store(status, steps, meas, dt, damping, lastNeg, total);
        if (EXPL && lane == 0) { Y.gopt[s].x = ph & 1; Y.gopt[s].y = ph >> 1; }
        if (COUNT && lane == 0) {
            atomicAdd(Y.counters + 1, (unsigned long long)itr * (unsigned long long)E.N);
            atomicAdd(Y.counters + 2, (unsigned long long)itr);
        }
        __syncwarp();
    }
    if (COUNT) {
        unsigned long long np = E.npair;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) np += __shfl_xor_sync(0xffffffffu, np, o);
        if (lane == 0) atomicAdd(Y.counters, np);
    }
}

// One force (and energy) evaluation; warp w of block b takes queue[b*4 + w].
template <int APL, bool ENERGY>
__global__ void __launch_bounds__(128) eval_warp_kernel(Params P, Systems Y, const int* __restrict__ queue, int nqueue,
                                                        int maxNA, int maxNN) {
    extern __shared__ __align__(16) char smem[];
    const WarpLayout L = warp_layout(maxNA, maxNN);
    char* region = smem + (threadIdx.x >> 5) * L.per_warp;
    const int q = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (q >= nqueue) return;
    WarpEngine<APL, ENERGY, false> E(P, Y, region, L, maxNN);
    const int s = queue[q];
    E.load(s);
    double Eb = 0, Enb = 0, Eg = 0;
    E.forces(Eb, Enb, Eg);
    const int lane = threadIdx.x & 31;
    float fm = 0.f;
#pragma unroll
    for (int k = 0; k < APL; k++) {
        const int a = lane + 32 * k;
        if (a < E.N) { Y.force[E.voff + a] = make_float4(E.fasm_a[k].x, E.fasm_a[k].y, E.fasm_a[k].z, 0.f); fm = fmaxf(fm, dot3(E.fasm_a[k], E.fasm_a[k])); }
        if (a < E.NN) { Y.force[E.voff + E.N + a] = make_float4(E.fasm_p[k].x, E.fasm_p[k].y, E.fasm_p[k].z, 0.f); fm = fmaxf(fm, dot3(E.fasm_p[k], E.fasm_p[k])); }
    }
    fm = wmax_f(fm);
    if (ENERGY) {
        // the reference's split: the skipped 1-3 pair energies belong to the
        // pair sum and their subtraction to the bonded part; the total is
        // summed without them
        const double e13 = wsum_d(E.e13);
        Eb = wsum_d(Eb); Enb = wsum_d(Enb); Eg = wsum_d(Eg);
        if (lane == 0) Y.energy[s] = make_double4(Eb - e13, Enb + e13, Eg, Eb + Enb + Eg);
    }
    if (lane == 0) Y.fconv[s] = sqrtf(fm);
}

void* relax_warp_fn(int apl, bool count) {
    if (apl == 1) return count ? (void*)relax_warp_kernel<1, true> : (void*)relax_warp_kernel<1, false>;
    if (apl == 2) return count ? (void*)relax_warp_kernel<2, true> : (void*)relax_warp_kernel<2, false>;
    return nullptr;
}
void* relax_warp_explore_fn(int apl) {
    if (apl == 1) return (void*)relax_warp_kernel<1, false, true>;
    if (apl == 2) return (void*)relax_warp_kernel<2, false, true>;
    return nullptr;
}
void* eval_warp_fn(int apl, bool energy) {
    if (apl == 1) return energy ? (void*)eval_warp_kernel<1, true> : (void*)eval_warp_kernel<1, false>;
    if (apl == 2) return energy ? (void*)eval_warp_kernel<2, true> : (void*)eval_warp_kernel<2, false>;
    return nullptr;
}

}  // namespace mmff
