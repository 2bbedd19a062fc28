// mmff_relax.cu -- system-resident relaxation kernels for sm_100a.
//
// One CTA owns one system at a time.  The system's whole state (positions,
// velocities, topology, force-field parameters, recoil slots) is staged in
// shared memory, and every FIRE step runs inside the CTA:
//   phase 1  bonded terms (thread per node), non-bonded pairs (S threads per
//            atom, j-split, warp-shuffle reduction) and the B-spline GridFF
//            sample (4 lanes per atom, one x-slice of the 4x4x4 stencil each,
//            float4 gathers that stay resident in L2)
//   phase 2  recoil assembly (MMFFsp3_loc::assemble_atom), optional force clamp,
//            FP64 block reduction of (f.v, v.v, f.f) and max|f|^2
//   phase 3  FIRE_update_params in FP64 (every thread computes the same
//            scalars), move_atom_FIRE, bounding box for PBC-image culling
// The persistent variant claims systems from a device work queue (atomic
// counter): a CTA that finishes a system (converged, failed or out of steps)
// writes it back and claims the next one, so converged systems retire and
// their slots refill without a host round trip.
#include "mmff_device.cuh"
#include <cfloat>

// blocks of at least this many threads unroll the pair tiles and the GridFF
// columns; smaller ones (four or eight per SM, instruction-fetch bound) do
// not: measured +5-7 % at 64 threads, +1.7 % at 128 threads (C2 class of
// 65-128 atoms), while the 256-thread blocks gain 5 % from unrolling
#ifndef MMFF_UNROLL_MIN_T
#define MMFF_UNROLL_MIN_T 256
#endif

namespace mmff {

// warp-level sums / extrema
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float wmax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float wmin(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Image shift for cell index (ix, iy, iz)
__device__ __forceinline__ float3 image_shift(const float* lv, int ix, int iy, int iz) {
    return make_float3(lv[0] * ix + lv[3] * iy + lv[6] * iz, lv[1] * ix + lv[4] * iy + lv[7] * iz,
                       lv[2] * ix + lv[5] * iy + lv[8] * iz);
}

// ---------------------------------------------------------------------------
// The per-system engine.  T threads, S threads per atom in the pair sum.
template <int T, int S, bool ENERGY, bool COUNT = false>
struct Engine {
    static_assert(T % 32 == 0 && 32 % S == 0, "bad tile");
    const Params& P;
    const Systems& Y;
    SmemLayout L;
    char* sm;
    int tid, lane, warp;
    // current system
    int isys, natoms, nnode, nvecs, aoff, noff, voff;
    float lv[9];
    float3 gorg;
    // per-step image culling
    float bbmin[3], bbmax[3];
    bool hasH = false;          // any H-bond pseudo-charge in the system (block-uniform)
    const uint32_t* xrow;       // central-image exclusion rows (ceil(natoms/32) words per atom)
    int nbw;                    // words per row
    bool pairbad = false;       // a non-finite pair force reached the fixed-point sums
    double e13 = 0.0;           // ENERGY: pair energies of the skipped 1-3 pairs (energy split)
    // pair-images evaluated by this thread (COUNT builds only)
    unsigned long long npair = 0;
    // shifted-image pair lists of the current system (relax launches with
    // P.vlist): entries (i | j << 12 | image << 24) in this CTA's slot of global
    // scratch, then the positions at the last build.  Their state is
    // block-uniform and sits in shared memory: [0] usable for this system (no
    // overflow), [1] built and no atom moved more than half the skin since,
    // [2] entries.
    __device__ __forceinline__ uint32_t* vslot() const { return P.vlist + (size_t)blockIdx.x * P.vstride; }
    __device__ __forceinline__ int* vstate() const {
        __shared__ int st[3];
        return st;
    }

    __device__ Engine(const Params& p, const Systems& y, char* smem, const SmemLayout& l)
        : P(p), Y(y), L(l), sm(smem) {
        tid = threadIdx.x; lane = tid & 31; warp = tid >> 5;
    }
    template <class X> __device__ __forceinline__ X* at(int off) { return reinterpret_cast<X*>(sm + off); }
    // per-atom / per-node arrays that a compact layout leaves in global memory
    static constexpr bool kMayCompact = T >= kCompactMinThreads;
    __device__ __forceinline__ bool compact() const { return kMayCompact && L.ng < 0; }
    __device__ __forceinline__ int4 ngs(int a) { return compact() ? __ldg(Y.neighs + aoff + a) : at<int4>(L.ng)[a]; }
    __device__ __forceinline__ int4 ngc(int a) { return compact() ? __ldg(Y.neighCell + aoff + a) : at<int4>(L.ngC)[a]; }
    __device__ __forceinline__ int4 bks(int a) { return compact() ? __ldg(Y.bkneighs + aoff + a) : at<int4>(L.bk)[a]; }
    __device__ __forceinline__ float4 plq(int a) { return compact() ? __ldg(Y.PLQ + aoff + a) : at<float4>(L.PLQ)[a]; }
    __device__ __forceinline__ float4 npar(int off, const float4* g, int n) {
        return compact() ? __ldg(g + noff + n) : at<float4>(off)[n];
    }
    // image tiles for long candidate lists (else ordered rows only)
    static constexpr bool kImgTiles = T >= kImageTileMinThreads;

    __device__ void load(int s) {
        isys = s;
        const int4 d = Y.desc[s];
        aoff = d.x; noff = d.y; voff = d.z; natoms = d.w;
        nnode = Y.nnode[s];
        nvecs = natoms + nnode;
        xrow = Y.xmask + Y.moff[s];
        nbw = (natoms + 31) >> 5;
        pairbad = false;
        if (tid == 0) { int* vs = vstate(); vs[0] = P.vlist != nullptr && natoms <= 4096; vs[1] = 0; vs[2] = 0; }
#pragma unroll
        for (int k = 0; k < 9; k++) lv[k] = Y.lvec[9 * s + k];
        const float4 g = Y.gorg[s];
        gorg = make_float3(g.x, g.y, g.z);
        float4* spos = at<float4>(L.pos); float4* svel = at<float4>(L.vel);
        for (int v = tid; v < nvecs; v += T) { spos[v] = Y.pos[voff + v]; svel[v] = Y.vel[voff + v]; }
        float4* sREQ = at<float4>(L.REQ);
        const bool full = !compact();         // else topology stays in global memory
        int h = 0;
        for (int a = tid; a < natoms; a += T) {
            const float4 r = Y.REQ[aoff + a];
            sREQ[a] = r; h |= (r.w != 0.f);
            if (full) {
                at<float4>(L.PLQ)[a] = Y.PLQ[aoff + a];
                at<int4>(L.ng)[a] = Y.neighs[aoff + a];
                at<int4>(L.ngC)[a] = Y.neighCell[aoff + a];
                at<int4>(L.bk)[a] = Y.bkneighs[aoff + a];
            }
        }
        hasH = __syncthreads_or(h) != 0;
        if (full)
            for (int n = tid; n < nnode; n += T) {
                at<float4>(L.apar)[n] = Y.apars[noff + n]; at<float4>(L.bL)[n] = Y.bLs[noff + n];
                at<float4>(L.bK)[n] = Y.bKs[noff + n]; at<float4>(L.ksp)[n] = Y.Ksp[noff + n];
                at<float4>(L.kpp)[n] = Y.Kpp[noff + n];
            }
    }

    // bounding box of the atoms (all threads end with the same box); needs a barrier inside
    __device__ void bbox_from_smem() {
        const float4* spos = at<float4>(L.pos);
        float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int a = tid; a < natoms; a += T) {
            const float4 p = spos[a];
            mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
            mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
        }
        bbox_reduce(mn, mx);
    }
    // reduce per-thread boxes: warp shuffle, warp partials in smem, barrier, redundant final
    __device__ void bbox_reduce(float* mn, float* mx) {
        float* red = at<float>(L.red) + 8 * 2 * L.nwarps;   // after the 4 doubles per warp
#pragma unroll
        for (int k = 0; k < 3; k++) { mn[k] = wmin(mn[k]); mx[k] = wmax(mx[k]); }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 3; k++) { red[6 * warp + k] = mn[k]; red[6 * warp + 3 + k] = mx[k]; }
        }
        __syncthreads();
        float a[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, b[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int w = 0; w < L.nwarps; w++) {
#pragma unroll
            for (int k = 0; k < 3; k++) { a[k] = fminf(a[k], red[6 * w + k]); b[k] = fmaxf(b[k], red[6 * w + 3 + k]); }
        }
#pragma unroll
        for (int k = 0; k < 3; k++) { bbmin[k] = a[k]; bbmax[k] = b[k]; }
    }

    // is image (ix,iy,iz) within the cutoff of the molecule's own box?
    __device__ __forceinline__ bool image_active(int ix, int iy, int iz) const { return image_within(ix, iy, iz, P.Rc2); }
    // ... within sqrt(R2) (the cutoff, or the cutoff plus the list skin)
    __device__ __forceinline__ bool image_within(int ix, int iy, int iz, float R2) const {
        if (P.Rc2 <= 0.f) return true;
        if (ix == 0 && iy == 0 && iz == 0) return true;
        const float3 sh = image_shift(lv, ix, iy, iz);
        // gap between [bbmin,bbmax] and [bbmin+sh, bbmax+sh] per axis
        const float gx = fmaxf(0.f, fabsf(sh.x) - (bbmax[0] - bbmin[0]));
        const float gy = fmaxf(0.f, fabsf(sh.y) - (bbmax[1] - bbmin[1]));
        const float gz = fmaxf(0.f, fabsf(sh.z) - (bbmax[2] - bbmin[2]));
        return gx * gx + gy * gy + gz * gz < R2;
    }

    // Candidate lists of the shifted images: atom j is a candidate of image
    // (ix,iy,iz) when its shifted position lies within sqrt(R2) (the cutoff,
    // or the cutoff plus the list skin) of this system's own bounding box (no
    // atom i can reach the others).  Lists are
    // ascending in j (ballot words, per-image prefix sums), so the pair sums
    // keep a fixed order.  All threads; contains barriers.
    __device__ void build_candidates(float R2) {
        const float4* spos = at<float4>(L.pos);
        uint32_t* words = at<uint32_t>(L.cwords);
        int* pref = at<int>(L.cpref);
        int* cnt = at<int>(L.ccnt);
        unsigned short* list = at<unsigned short>(L.clist);
        const int npx = P.npbc[0], npy = P.npbc[1], npz = P.npbc[2];
        const int nw = L.nwords;
        for (int base = warp * 32; base < natoms; base += T) {
            const int j = base + lane;
            const float4 p = (j < natoms) ? spos[j] : make_float4(0, 0, 0, 0);
            int k = 0;
            for (int iz = -npz; iz <= npz; iz++)
                for (int iy = -npy; iy <= npy; iy++)
                    for (int ix = -npx; ix <= npx; ix++) {
                        if ((ix | iy | iz) == 0) continue;
                        bool c = false;
                        if (j < natoms && image_within(ix, iy, iz, R2)) {
                            const float3 sh = image_shift(lv, ix, iy, iz);
                            const float qx = p.x + sh.x, qy = p.y + sh.y, qz = p.z + sh.z;
                            const float gx = fmaxf(0.f, fmaxf(bbmin[0] - qx, qx - bbmax[0]));
                            const float gy = fmaxf(0.f, fmaxf(bbmin[1] - qy, qy - bbmax[1]));
                            const float gz = fmaxf(0.f, fmaxf(bbmin[2] - qz, qz - bbmax[2]));
                            c = gx * gx + gy * gy + gz * gz < R2;
                        }
                        const uint32_t bal = __ballot_sync(0xffffffffu, c);
                        if (lane == 0) words[k * nw + (base >> 5)] = bal;
                        k++;
                    }
        }
        __syncthreads();
        for (int k = warp; k < L.nimg; k += L.nwarps) {
            int run = 0;
            for (int w0 = 0; w0 < nw; w0 += 32) {
                const int w = w0 + lane;
                const uint32_t m = (w < nw && 32 * w < natoms) ? words[k * nw + w] : 0u;
                const int c = __popc(m);
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                if (w < nw) pref[k * nw + w] = run + incl - c;
                run += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) cnt[k] = run;
        }
        __syncthreads();
        for (int j = tid; j < natoms; j += T) {
            const int w = j >> 5;
            const uint32_t below = (1u << (j & 31)) - 1u;
            for (int k = 0; k < L.nimg; k++) {
                const uint32_t m = words[k * nw + w];
                if ((m >> (j & 31)) & 1u) list[k * L.maxNA + pref[k * nw + w] + __popc(m & below)] = (unsigned short)j;
            }
        }
        __syncthreads();
    }

    // pair sum of one atom (already shifted by the image) over j = sub, sub+S, ...
    // Branch-free: excluded and out-of-range pairs get r^2 = 1e30, where every
    // term underflows to zero except the shifted-force constant kq Q / r
    // (< 1e-16 eV/A).  HB: the system has H-bond pseudo-charges (block-uniform).
    // list (nullable): candidate atoms of a shifted image, ascending; else all atoms
    template <bool HB>
    __device__ __forceinline__ void pair_row(const float4* spos, const float4* sREQ, int sub, float4 Ri, float pxs,
                                             float pys, float pzs, int e0, int e1, int e2, int e3, int e4,
                                             const unsigned short* list, int ncand,
                                             float& fx, float& fy, float& fz, float& ei) {
        const bool CUT = P.Rc2 > 0.f;
        const float Rc2 = CUT ? P.Rc2 : 3.0e38f, kq = P.kq_rc2;
        const float rc = CUT ? sqrtf(1.f / kq) : 0.f;
        const int n = list ? ncand : natoms;
        for (int c = sub; c < n; c += S) {
            const int j = list ? (int)list[c] : c;
            const float4 pj = spos[j];
            const float4 Rj = sREQ[j];
            const float dx = pj.x - pxs, dy = pj.y - pys, dz = pj.z - pzs;
            float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool ex = (j == e0) | (j == e1) | (j == e2) | (j == e3) | (j == e4);
            const bool ok = !ex && (r2 < Rc2);
            if (COUNT && ok) npair++;
            r2 = ok ? r2 : 1e30f;
            const float ir = rsqrtf(r2);
            const float ir2 = ir * ir;
            const float R0 = Ri.x + Rj.x;
            const float E0 = Ri.y * Rj.y;
            const float Q = Ri.z * Rj.z;
            const float Eel = Q * ir;
            const float u2 = R0 * R0 * ir2;
            const float u6 = u2 * u2 * u2;
            const float vdW = u6 * E0;
            const float H = HB ? u6 * vdW * fminf(Ri.w * Rj.w, 0.f) : 0.f;
            float F = -fmaf(12.f * ir2, HB ? fmaf(u6 - 1.f, vdW, H) : (u6 - 1.f) * vdW, Eel * ir2);
            F = fmaf(Q * kq, ir, F);
            fx = fmaf(dx, F, fx); fy = fmaf(dy, F, fy); fz = fmaf(dz, F, fz);
            if (ENERGY && ok) {
                float e = fmaf(u6 - 2.f, vdW, Eel + H);
                if (CUT) e += Q * kq * (r2 * ir - 2.f * rc);
                ei += e;
            }
        }
    }

    // atom i (lane sub of its S) against image (ix,iy,iz) of the atoms in list
    // (all atoms if list is null): the exclusions of NBFF::evalLJQs_ng4_PBC_atom
    // (NBFF.h:590-607): i itself, and its bonded neighbours whose cell is ipbc
    __device__ __forceinline__ void pair_image_row(const float4* spos, const float4* sREQ, int i, int sub, float4 pi,
                                                   float4 Ri, int4 ng, int4 ngC, bool pbc, int ipbc, int ix, int iy,
                                                   int iz, const unsigned short* list, int ncand, float& fx, float& fy,
                                                   float& fz, float& ei) {
        const float3 sh = image_shift(lv, ix, iy, iz);
        const float pxs = pi.x - sh.x, pys = pi.y - sh.y, pzs = pi.z - sh.z;
        const int e0 = i;
        const int e1 = (ngC.x == ipbc || !pbc) ? ng.x : -1;
        const int e2 = (ngC.y == ipbc || !pbc) ? ng.y : -1;
        const int e3 = (ngC.z == ipbc || !pbc) ? ng.z : -1;
        const int e4 = (ngC.w == ipbc || !pbc) ? ng.w : -1;
        if (hasH) pair_row<true>(spos, sREQ, sub, Ri, pxs, pys, pzs, e0, e1, e2, e3, e4, list, ncand, fx, fy, fz, ei);
        else pair_row<false>(spos, sREQ, sub, Ri, pxs, pys, pzs, e0, e1, e2, e3, e4, list, ncand, fx, fy, fz, ei);
    }

    // ---- central image, each unordered pair once (Newton's third law) --------
    // 32 x 32 atom tiles: the 32 lanes of a warp own the atoms i of block bi,
    // the atoms j of block bj rotate through the lanes (lane l meets j-slot
    // l + s at step s) and so does the reaction accumulator of the current j,
    // which after 32 steps sits in lane j - 32 bj.  Diagonal tiles take steps
    // 1..16 (s = 16 on lanes < 16 only) and return reactions by shuffle.  Tile
    // sums reach the per-atom totals through 64-bit fixed-point shared-memory
    // adds (2^-32 eV/A resolution): integer addition is associative, so the
    // totals do not depend on which warp finishes first.
    static constexpr float kFix = 4294967296.f;
#ifndef MMFF_TILE_UNROLL_SMALL
#define MMFF_TILE_UNROLL_SMALL 1
#endif
#ifndef MMFF_TILE_UNROLL_LARGE
#define MMFF_TILE_UNROLL_LARGE 4
#endif
    // tile-step unrolling (build options): none in blocks below
    // MMFF_UNROLL_MIN_T threads, whose fused step is instruction-fetch bound
    // (unrolling by 4 measured -6 % at 64 threads), 4 in the larger blocks
    // (+4.7 %)
    static constexpr int kTileUnroll = T >= MMFF_UNROLL_MIN_T ? MMFF_TILE_UNROLL_LARGE : MMFF_TILE_UNROLL_SMALL;
    // Each add is clamped to |f| <= 2^20 eV/A, so the 64-bit sums (2^31 units
    // of range per eV/A) cannot wrap for any system that fits a block; a
    // non-finite force (atoms on top of each other) would convert to an
    // arbitrary integer, so it marks the system bad instead (assemble).
    static constexpr float kFixMax = 1048576.f;
    __device__ __forceinline__ void fix_add(long long* a, float3 f) {
        pairbad |= !isfinite(f.x + f.y + f.z);
        const float x = fminf(fmaxf(f.x, -kFixMax), kFixMax), y = fminf(fmaxf(f.y, -kFixMax), kFixMax);
        const float z = fminf(fmaxf(f.z, -kFixMax), kFixMax);
        atomicAdd(reinterpret_cast<unsigned long long*>(a + 0), (unsigned long long)__float2ll_rn(x * kFix));
        atomicAdd(reinterpret_cast<unsigned long long*>(a + 1), (unsigned long long)__float2ll_rn(y * kFix));
        atomicAdd(reinterpret_cast<unsigned long long*>(a + 2), (unsigned long long)__float2ll_rn(z * kFix));
    }

    // own atom i of a tile: position and parameters; invalid slots exclude everything
    struct TileAtom { float4 p, R; int i; bool v; };
    __device__ __forceinline__ TileAtom tile_atom(int i, const float4* spos, const float4* sREQ) {
        TileAtom t;
        t.v = i < natoms;
        t.i = t.v ? i : 0;
        t.p = spos[t.i]; t.R = sREQ[t.i];
        return t;
    }

    // excluded j-slots of block bj for this lane's atom (the host-built
    // exclusion row: the atom itself, its bonded neighbours in the central
    // cell, the 1-3 pairs the angle terms account for, padding slots of bj);
    // all if the atom is a padding slot
    __device__ __forceinline__ uint32_t tile_mask(const TileAtom& a, int bj) const {
        return a.v ? __ldg(xrow + a.i * nbw + bj) : ~0u;
    }

    template <bool HB>
    __device__ void off_tile(int bi, int bj, const float4* spos, const float4* sREQ, bool pbc, int central,
                             long long* facc, float& ec) {
        const bool CUT = P.Rc2 > 0.f;
        const float Rc2 = CUT ? P.Rc2 : 3.0e38f, kq = P.kq_rc2;
        const float rc = CUT ? sqrtf(1.f / kq) : 0.f;
        const int i = bi * 32 + lane;
        const TileAtom a = tile_atom(i, spos, sREQ);
        const uint32_t xm = tile_mask(a, bj);
        float3 fi = make_float3(0.f, 0.f, 0.f), rj = make_float3(0.f, 0.f, 0.f);
        bool ok;
        float e = 0.f;
#pragma unroll kTileUnroll
        for (int s = 0; s < 32; s++) {
            const int jl = (lane + s) & 31;
            const int j = bj * 32 + jl;
            const int jc = min(j, natoms - 1);
            const float4 pj = spos[jc], Rj = sREQ[jc];
            const bool excl = (xm >> jl) & 1u;
            const float dx = pj.x - a.p.x, dy = pj.y - a.p.y, dz = pj.z - a.p.z;
            const float F = pair_force<ENERGY, HB>(dx, dy, dz, a.R, Rj, excl, Rc2, kq, rc, CUT, ok, e);
            fi.x = fmaf(dx, F, fi.x); fi.y = fmaf(dy, F, fi.y); fi.z = fmaf(dz, F, fi.z);
            rj.x = fmaf(-dx, F, rj.x); rj.y = fmaf(-dy, F, rj.y); rj.z = fmaf(-dz, F, rj.z);
            if (ENERGY) ec += e;
            if (COUNT && ok) npair += 2;
            const int nxt = (lane + 1) & 31;
            rj.x = __shfl_sync(0xffffffffu, rj.x, nxt);
            rj.y = __shfl_sync(0xffffffffu, rj.y, nxt);
            rj.z = __shfl_sync(0xffffffffu, rj.z, nxt);
        }
        if (a.v) fix_add(facc + 3 * i, fi);
        const int jo = bj * 32 + lane;
        if (jo < natoms) fix_add(facc + 3 * jo, rj);
    }

    template <bool HB>
    __device__ void diag_tile(int b, const float4* spos, const float4* sREQ, bool pbc, int central, long long* facc,
                              float& ec) {
        const bool CUT = P.Rc2 > 0.f;
        const float Rc2 = CUT ? P.Rc2 : 3.0e38f, kq = P.kq_rc2;
        const float rc = CUT ? sqrtf(1.f / kq) : 0.f;
        const int i = b * 32 + lane;
        const TileAtom a = tile_atom(i, spos, sREQ);
        const uint32_t xm = tile_mask(a, b);
        float3 fi = make_float3(0.f, 0.f, 0.f);
        bool ok;
        float e = 0.f;
#pragma unroll kTileUnroll
        for (int s = 1; s <= 16; s++) {
            const int jl = (lane + s) & 31;
            const int jc = min(b * 32 + jl, natoms - 1);
            const float4 pj = spos[jc], Rj = sREQ[jc];
            const bool excl = ((xm >> jl) & 1u) || (s == 16 && lane >= 16);
            const float dx = pj.x - a.p.x, dy = pj.y - a.p.y, dz = pj.z - a.p.z;
            const float F = pair_force<ENERGY, HB>(dx, dy, dz, a.R, Rj, excl, Rc2, kq, rc, CUT, ok, e);
            fi.x = fmaf(dx, F, fi.x); fi.y = fmaf(dy, F, fi.y); fi.z = fmaf(dz, F, fi.z);
            if (ENERGY) ec += e;
            if (COUNT && ok) npair += 2;
            const int src = (lane - s) & 31;     // the lane whose partner this lane's atom was
            fi.x += __shfl_sync(0xffffffffu, -dx * F, src);
            fi.y += __shfl_sync(0xffffffffu, -dy * F, src);
            fi.z += __shfl_sync(0xffffffffu, -dz * F, src);
        }
        if (a.v) fix_add(facc + 3 * i, fi);
    }

    // position of atom e in the candidate list of image k, or -1
    __device__ __forceinline__ int cand_slot(int k, int e) {
        if (e < 0) return -1;
        const int w = k * L.nwords + (e >> 5);
        const uint32_t m = at<uint32_t>(L.cwords)[w];
        if (!((m >> (e & 31)) & 1u)) return -1;
        return at<int>(L.cpref)[w] + __popc(m & ((1u << (e & 31)) - 1u));
    }

    // ---- shifted images, each unordered image pair once -----------------------
    // Atom i meets image +k of atom j exactly when atom j meets image -k of
    // atom i, with the opposite force.  So for long candidate lists only the
    // images k < nimg / 2 are visited (image nimg-1-k is the mirror of k), as
    // 32 x 32 tiles of (candidates i of image -k) x (candidates j of image +k),
    // each pair once, the reaction on j rotating through the lanes as in
    // off_tile.  Excluded (NBFF::evalLJQs_ng4_PBC_atom, NBFF.h:590-607): i
    // itself, and the bonded neighbours of i whose cell is this image; both
    // are symmetric under the mirror.  k: image index without the central
    // one (iz, iy, ix order).
    template <bool HB>
    __device__ void image_tile(int k, int ti, int tj, const float4* spos, const float4* sREQ, long long* facc,
                               float& ec) {
        const bool CUT = P.Rc2 > 0.f;
        const float Rc2 = CUT ? P.Rc2 : 3.0e38f, kq = P.kq_rc2;
        const float rc = CUT ? sqrtf(1.f / kq) : 0.f;
        const int nxi = 2 * P.npbc[0] + 1, nyi = 2 * P.npbc[1] + 1;
        const int ipbc = k;                                   // k < central: same index with the central one
        const int ix = ipbc % nxi - P.npbc[0], iy = (ipbc / nxi) % nyi - P.npbc[1], iz = ipbc / (nxi * nyi) - P.npbc[2];
        const int kI = L.nimg - 1 - k;
        const unsigned short* Il = at<unsigned short>(L.clist) + kI * L.maxNA;
        const unsigned short* Jl = at<unsigned short>(L.clist) + k * L.maxNA;
        const int nI = at<int>(L.ccnt)[kI], nJ = at<int>(L.ccnt)[k];
        const int ci = 32 * ti + lane;
        const bool vi = ci < nI;
        const int i = vi ? (int)Il[ci] : 0;
        const float3 sh = image_shift(lv, ix, iy, iz);
        float4 pi = spos[i];
        pi.x -= sh.x; pi.y -= sh.y; pi.z -= sh.z;
        const float4 Ri = sREQ[i];
        // excluded j-slots of this tile
        const int j0 = 32 * tj;
        uint32_t xm = ~0u;
        if (vi) {
            const int nvalid = nJ - j0;
            xm = nvalid >= 32 ? 0u : ~((1u << nvalid) - 1u);
            const int4 ng = ngs(i), ngC = ngc(i);
            const int e[5] = {i, ngC.x == ipbc ? ng.x : -1, ngC.y == ipbc ? ng.y : -1, ngC.z == ipbc ? ng.z : -1,
                              ngC.w == ipbc ? ng.w : -1};
#pragma unroll
            for (int q = 0; q < 5; q++) {
                const int d = cand_slot(k, e[q]) - j0;
                if (d >= 0 && d < 32) xm |= 1u << d;
            }
        }
        float3 fi = make_float3(0.f, 0.f, 0.f), rj = make_float3(0.f, 0.f, 0.f);
        bool ok;
        float e = 0.f;
        const int jlast = nJ - 1;
        // the tile's 32 candidates j into this warp's staging slots (one
        // indirect load per lane instead of one per rotation step)
        float4* stg = at<float4>(L.stage) + 64 * warp;
        {
            const int jj = Jl[min(j0 + lane, jlast)];
            stg[lane] = spos[jj];
            stg[32 + lane] = sREQ[jj];
        }
        __syncwarp();
#pragma unroll kTileUnroll
        for (int s = 0; s < 32; s++) {
            const int jl = (lane + s) & 31;
            const float4 pj = stg[jl], Rj = stg[32 + jl];
            const bool excl = (xm >> jl) & 1u;
            const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            const float F = pair_force<ENERGY, HB>(dx, dy, dz, Ri, Rj, excl, Rc2, kq, rc, CUT, ok, e);
            fi.x = fmaf(dx, F, fi.x); fi.y = fmaf(dy, F, fi.y); fi.z = fmaf(dz, F, fi.z);
            rj.x = fmaf(-dx, F, rj.x); rj.y = fmaf(-dy, F, rj.y); rj.z = fmaf(-dz, F, rj.z);
            if (ENERGY) ec += e;
            if (COUNT && ok) npair += 2;
            const int nxt = (lane + 1) & 31;
            rj.x = __shfl_sync(0xffffffffu, rj.x, nxt);
            rj.y = __shfl_sync(0xffffffffu, rj.y, nxt);
            rj.z = __shfl_sync(0xffffffffu, rj.z, nxt);
        }
        __syncwarp();                                         // staging slots free for the next tile
        if (vi) fix_add(facc + 3 * i, fi);
        if (j0 + lane < nJ) fix_add(facc + 3 * (int)Jl[j0 + lane], rj);
    }

    // ---- shifted-image pair lists (Verlet lists with a skin) ------------------
    // (skin P.vskin, 1 A by default.)
    // Of the pairs the candidate tiles of the shifted images evaluate, only a
    // few percent lie inside the cutoff: for a large molecule the candidates
    // of an image span its whole cross-section.  With lists, the ordered pairs
    // (i, j + shift of image k) over every shifted image k closer than
    // Rc + skin are collected once and evaluated every step (both orders of a
    // pair are listed, so the force on i sums in registers and no reaction
    // goes through the fixed-point atomics) until some atom has moved more
    // than skin/2 since the build; then they are rebuilt.  The pairs inside
    // the cutoff are the tiles' pairs, so forces differ from the tile path
    // only in summation order.

    // block-wide exclusive scan of one int per thread (total in every thread); tmp: nwarps ints
    __device__ int block_scan(int x, int& total, int* tmp) {
        int incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) tmp[warp] = incl;
        __syncthreads();
        int base = 0;
        total = 0;
        for (int w = 0; w < L.nwarps; w++) {
            const int t = tmp[w];
            if (w < warp) base += t;
            total += t;
        }
        __syncthreads();
        return base + incl - x;
    }

    // rebuild this system's lists from the current positions; false
    // (block-uniform) when they do not fit in the slot.  All threads; barriers.
    __device__ bool list_build(const float4* spos) {
        const float Rv = sqrtf(P.Rc2) + P.vskin, Rv2 = Rv * Rv;
        build_candidates(Rv2);
        const int* ccnt = at<int>(L.ccnt);
        const unsigned short* clist = at<unsigned short>(L.clist);
        uint32_t* ent = vslot();
        // rows: (shifted image k, candidate i of its mirror), k-major; thread tid takes rows [r0, r1)
        int R = 0;
        for (int k = 0; k < L.nimg; k++) R += ccnt[L.nimg - 1 - k];
        const int r0 = (int)((long long)R * tid / T), r1 = (int)((long long)R * (tid + 1) / T);
        int* tmp = reinterpret_cast<int*>(at<long long>(L.facc));   // unused until the pair sums start
        int off = 0, total = 0;
        for (int pass = 0; pass < 2; pass++) {           // count, then write at the scanned offset
            int c = 0, k = 0, base = 0;
            for (int r = r0; r < r1; r++) {
                while (r >= base + ccnt[L.nimg - 1 - k]) { base += ccnt[L.nimg - 1 - k]; k++; }
                const int i = clist[(L.nimg - 1 - k) * L.maxNA + (r - base)];
                const int nxi = 2 * P.npbc[0] + 1, nyi = 2 * P.npbc[1] + 1;
                const int ipbc = k < L.nimg / 2 ? k : k + 1;      // image index with the central one
                const float3 sh = image_shift(lv, ipbc % nxi - P.npbc[0], (ipbc / nxi) % nyi - P.npbc[1],
                                              ipbc / (nxi * nyi) - P.npbc[2]);
                const float4 pi = spos[i];
                const float qx = pi.x - sh.x, qy = pi.y - sh.y, qz = pi.z - sh.z;
                const unsigned short* Jl = clist + k * L.maxNA;
                const int nJ = ccnt[k];
                for (int jj = 0; jj < nJ; jj++) {
                    const int j = Jl[jj];
                    const float4 pj = spos[j];
                    const float dx = pj.x - qx, dy = pj.y - qy, dz = pj.z - qz;
                    if (!(fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < Rv2) || image_excluded(i, j, ipbc)) continue;
                    if (pass == 1) ent[off + c] = (uint32_t)i | ((uint32_t)j << 12) | ((uint32_t)k << 24);
                    c++;
                }
            }
            if (pass == 0) {
                off = block_scan(c, total, tmp);
                if (total > P.vcap) return false;
            }
        }
        float4* vp = reinterpret_cast<float4*>(ent + P.vcap);
        for (int a = tid; a < natoms; a += T) vp[a] = spos[a];
        if (tid == 0) vstate()[2] = total;
        __syncthreads();
        return true;
    }

    // excluded pair of the shifted image ipbc (NBFF::evalLJQs_ng4_PBC_atom,
    // NBFF.h:590-607): i itself, and the bonded neighbours of i whose cell is this image
    __device__ __forceinline__ bool image_excluded(int i, int j, int ipbc) {
        if (j == i) return true;
        const int4 ng = ngs(i), ngC = ngc(i);
        return (ngC.x == ipbc && ng.x == j) || (ngC.y == ipbc && ng.y == j) || (ngC.z == ipbc && ng.z == j) ||
               (ngC.w == ipbc && ng.w == j);
    }

    // the listed pairs of the shifted images into the fixed-point sums.  Each
    // thread takes a contiguous run of entries (equal shares): consecutive
    // entries mostly share atom i and image k, so the force on i adds up in
    // registers and goes to the fixed-point sums once per run of i, the image
    // shift is recomputed only when k changes, and the next entry's load
    // overlaps the current pair.  Every pair is listed in both orders: half
    // of its energy each time, no reaction.
    template <bool HB>
    __device__ void list_pairs(const float4* spos, const float4* sREQ, long long* facc, float& ec) {
        const float Rc2 = P.Rc2, kq = P.kq_rc2, rc = sqrtf(1.f / kq);
        const int nxi = 2 * P.npbc[0] + 1, nyi = 2 * P.npbc[1] + 1;
        const uint32_t* ent = vslot();
        const int n = vstate()[2];
        const int q0 = (int)((long long)n * tid / T), q1 = (int)((long long)n * (tid + 1) / T);
        if (q0 >= q1) return;
        int ci = -1, ck = -1;
        float3 sh = make_float3(0.f, 0.f, 0.f), fi = make_float3(0.f, 0.f, 0.f);
        float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), Ri = pi;
        uint32_t wn = __ldcg(ent + q0);
        for (int q = q0; q < q1; q++) {
            const uint32_t w = wn;
            if (q + 1 < q1) wn = __ldcg(ent + q + 1);
            const int i = (int)(w & 0xFFFu), j = (int)((w >> 12) & 0xFFFu), k = (int)(w >> 24);
            if (i != ci) {
                if (ci >= 0) fix_add(facc + 3 * ci, fi);
                ci = i; fi = make_float3(0.f, 0.f, 0.f);
                pi = spos[i]; Ri = sREQ[i];
            }
            if (k != ck) {
                ck = k;
                const int ipbc = k < L.nimg / 2 ? k : k + 1;
                sh = image_shift(lv, ipbc % nxi - P.npbc[0], (ipbc / nxi) % nyi - P.npbc[1], ipbc / (nxi * nyi) - P.npbc[2]);
            }
            const float4 pj = spos[j];
            const float dx = pj.x + sh.x - pi.x, dy = pj.y + sh.y - pi.y, dz = pj.z + sh.z - pi.z;
            bool ok;
            float e = 0.f;
            const float F = pair_force<ENERGY, HB>(dx, dy, dz, Ri, sREQ[j], false, Rc2, kq, rc, true, ok, e);
            if (ENERGY) ec += 0.5f * e;
            if (!ok) continue;
            if (COUNT) npair++;
            fi.x = fmaf(dx, F, fi.x); fi.y = fmaf(dy, F, fi.y); fi.z = fmaf(dz, F, fi.z);
        }
        fix_add(facc + 3 * ci, fi);
    }

    // mirror pair (k, nimg-1-k): tiles (true) or ordered rows of both images.
    // Cost in pair evaluations: a tile evaluates 32 x 32 pairs at ~1.2 times
    // the cost of an ordered pair (the reaction and its rotation); the rows
    // evaluate the nI x nJ pairs of each image.
    __device__ __forceinline__ bool image_tiled(int nI, int nJ, int& units) const {
        const int nti = (nI + 31) >> 5, ntj = (nJ + 31) >> 5;
        if (kImgTiles && 6 * 1024 * nti * ntj <= 5 * 2 * nI * nJ) { units = nti * ntj; return true; }
        units = 0;
        return false;
    }

    // LISTS: the candidate lists of this step exist (block-uniform; the
    // central-only form keeps the image code out of the tile loop).
    // Warp units: each off-diagonal tile and pairs of diagonal tiles of the
    // central image, then the tiles of the mirror pairs with long candidate
    // lists; all of equal cost (1024 pair evaluations), dealt round-robin to
    // the warps.  Then, thread units: the mirror pairs with short lists as
    // ordered rows of both images, S lanes per candidate atom i (the images
    // that reach a few edge atoms of a small molecule).  No barrier anywhere:
    // every sum goes to the fixed-point accumulators.
    template <bool HB, bool LISTS>
    __device__ void pair_tiles(const float4* spos, const float4* sREQ, bool pbc, int central, long long* facc,
                               float& ec) {
        const int B = (natoms + 31) >> 5;
        const int noff = B * (B - 1) / 2;
        const int ncen = noff + ((B + 1) >> 1);
        int nunits = ncen, nrows = 0;
        const int* ccnt = at<int>(L.ccnt);
        if (LISTS)
            for (int k = 0; k < L.nimg / 2; k++) {
                int n;
                if (image_tiled(ccnt[L.nimg - 1 - k], ccnt[k], n)) nunits += n;
                else nrows += ccnt[L.nimg - 1 - k] + ccnt[k];
            }
        for (int u = warp; u < nunits; u += L.nwarps) {
            if (u < noff) {
                int bi = 0, rem = u;
                while (rem >= B - 1 - bi) { rem -= B - 1 - bi; bi++; }
                off_tile<HB>(bi, bi + 1 + rem, spos, sREQ, pbc, central, facc, ec);
            } else if (u < ncen) {
                const int d = 2 * (u - noff);
                diag_tile<HB>(d, spos, sREQ, pbc, central, facc, ec);
                if (d + 1 < B) diag_tile<HB>(d + 1, spos, sREQ, pbc, central, facc, ec);
            } else if (LISTS && kImgTiles) {
                int rem = u - ncen, k = 0, n = 0;
                for (;; k++) {
                    if (image_tiled(ccnt[L.nimg - 1 - k], ccnt[k], n) && rem < n) break;
                    rem -= n;
                }
                const int ntj = (ccnt[k] + 31) >> 5;
                image_tile<HB>(k, rem / ntj, rem % ntj, spos, sREQ, facc, ec);
            }
        }
        if (LISTS && nrows > 0) {
            const int nxi = 2 * P.npbc[0] + 1, nyi = 2 * P.npbc[1] + 1;
            const unsigned short* clist = at<unsigned short>(L.clist);
            for (int u0 = 0; u0 < nrows * S; u0 += T) {
                const int u = u0 + tid;
                int c = u / S;
                const int sub = u % S;
                float fx = 0.f, fy = 0.f, fz = 0.f, ei = 0.f;
                int i = -1;
                if (c < nrows) {
                    // row c -> image kk (k, then its mirror) and candidate position
                    int kk = -1;
                    for (int k = 0; k < L.nimg / 2; k++) {
                        int n;
                        if (image_tiled(ccnt[L.nimg - 1 - k], ccnt[k], n)) continue;
                        const int nI = ccnt[L.nimg - 1 - k], nJ = ccnt[k];
                        if (c < nI) { kk = k; break; }
                        c -= nI;
                        if (c < nJ) { kk = L.nimg - 1 - k; break; }
                        c -= nJ;
                    }
                    const int ipbc = kk < L.nimg / 2 ? kk : kk + 1;
                    const int ix = ipbc % nxi - P.npbc[0], iy = (ipbc / nxi) % nyi - P.npbc[1];
                    const int iz = ipbc / (nxi * nyi) - P.npbc[2];
                    i = clist[(L.nimg - 1 - kk) * L.maxNA + c];
                    pair_image_row(spos, sREQ, i, sub, spos[i], sREQ[i], ngs(i), ngc(i), pbc, ipbc, ix, iy, iz,
                                   clist + kk * L.maxNA, ccnt[kk], fx, fy, fz, ei);
                }
#pragma unroll
                for (int o = S / 2; o > 0; o >>= 1) {
                    fx += __shfl_xor_sync(0xffffffffu, fx, o);
                    fy += __shfl_xor_sync(0xffffffffu, fy, o);
                    fz += __shfl_xor_sync(0xffffffffu, fz, o);
                }
                if (i >= 0 && sub == 0) fix_add(facc + 3 * i, make_float3(fx, fy, fz));
                if (ENERGY) ec += 0.5f * ei;
            }
        }
    }

    // GridFF B-spline of every atom, 4 lanes per atom (x-slices), by the
    // threads t0 = 0 .. nt-1 of the caller (whole warps); zero without a grid
    __device__ void grid_phase(int t0, int nt, float4* fgr, double& Eg) {
        const float4* spos = at<float4>(L.pos);
        if (!(P.flags & F_GRID)) {
            for (int a = t0; a < natoms; a += nt) fgr[a] = make_float4(0, 0, 0, 0);
            return;
        }
        const int nunits = natoms * 4;
        const bool cached = Y.gkey != nullptr;      // launch-uniform
        for (int u0 = 0; u0 < nunits; u0 += nt) {
            const int u = u0 + t0;
            const int i = u >> 2, a = u & 3;
            float4 r = make_float4(0, 0, 0, 0);
            if (cached) {
                const bool ok = i < natoms;
                const int ic = ok ? i : natoms - 1;
                const float4 p = spos[ic];
                const float3 uu = make_float3((p.x + gorg.x) * P.ginv[0], (p.y + gorg.y) * P.ginv[1],
                                              (p.z + gorg.z) * P.ginv[2]);
                r = grid_slice_cached<(T >= MMFF_UNROLL_MIN_T) ? 4 : 1>(P.grid, P.gn[0], P.gn[1], P.gn[2], uu, plq(ic),
                                                                       a, ok, Y.gkey, Y.gcs, aoff + ic);
            } else if (i < natoms) {
                const float4 p = spos[i];
                const float3 uu = make_float3((p.x + gorg.x) * P.ginv[0], (p.y + gorg.y) * P.ginv[1],
                                              (p.z + gorg.z) * P.ginv[2]);
                r = grid_slice<(T >= MMFF_UNROLL_MIN_T) ? 4 : 1>(P.grid, P.gn[0], P.gn[1], P.gn[2], uu, plq(i), a);
            }
#pragma unroll
            for (int o = 2; o > 0; o >>= 1) {
                r.x += __shfl_xor_sync(0xffffffffu, r.x, o);
                r.y += __shfl_xor_sync(0xffffffffu, r.y, o);
                r.z += __shfl_xor_sync(0xffffffffu, r.z, o);
                r.w += __shfl_xor_sync(0xffffffffu, r.w, o);
            }
            if (i < natoms && a == 0) {
                fgr[i] = make_float4(r.x * P.gmi[0], r.y * P.gmi[1], r.z * P.gmi[2], 0.f);
                if (ENERGY) Eg += (double)r.w;
            }
        }
    }

    // Threads given to the bonded terms when the GridFF runs beside them on
    // the remaining warps; T = no split.  Cost model in units of one grid
    // round (4 lanes x 16 float4 gathers per atom): one bonded pass (one node
    // per thread) costs ~10 rounds.  Split when the longer of the two
    // concurrent parts beats running them one after the other.
    __device__ __forceinline__ int bonded_grid_split() const {
        if (!(P.flags & F_GRID)) return T;
        const int Tb = ((nnode + 31) / 32) * 32;
        if (Tb >= T || Tb == 0) return T;
        const int Tg = T - Tb;
        const int now = 10 * ((nnode + T - 1) / T) + (4 * natoms + T - 1) / T;
        const int par = max(10, (4 * natoms + Tg - 1) / Tg);
        return par < now ? Tb : T;
    }

    // ------------------------------------------------------------------ phase 1
    // returns this thread's energy contributions (only meaningful if ENERGY)
    __device__ void forces(double& Eb, double& Enb, double& Eg) {
        const int flags = P.flags;
        const float4* spos = at<float4>(L.pos);
        float4* fasm = at<float4>(L.fasm);
        float4* fnb = at<float4>(L.fnb);
        float4* fgr = at<float4>(L.fgrid);
        const float4* sREQ = at<float4>(L.REQ);
        float4* fng = at<float4>(L.fng);
        // Bonded terms and the GridFF stencil are independent: when the nodes
        // fill only part of the block, the other warps sample the grid at the
        // same time (block-uniform choice, see bonded_grid_split)
        const int Tb = bonded_grid_split();
        const bool split = Tb < T;
        if (split && tid >= Tb) {
            grid_phase(tid - Tb, T - Tb, fgr, Eg);
        }
        // --- bonded (nodes); caps get a zero own-force
        if (tid < Tb)
        for (int ia = tid; ia < natoms; ia += Tb) {
            if (ia >= nnode) { fasm[ia] = make_float4(0, 0, 0, 0); continue; }
            BondedOut o;
            eval_atom<ENERGY>(ia, natoms, nnode, flags, P.Fmax2NB, spos, sREQ, ngs(ia), ngc(ia),
                              npar(L.apar, Y.apars, ia), npar(L.bL, Y.bLs, ia), npar(L.bK, Y.bKs, ia),
                              npar(L.ksp, Y.Ksp, ia), npar(L.kpp, Y.Kpp, ia), lv, P.npbc[0], P.npbc[1], P.npbc[2],
                              __ldg(Y.a13 + noff + ia), Cut13(P), o);
            fasm[ia] = make_float4(o.fa.x, o.fa.y, o.fa.z, 0.f);
            fasm[natoms + ia] = make_float4(o.fpi.x, o.fpi.y, o.fpi.z, 0.f);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                fng[ia * 4 + k] = make_float4(o.fbs[k].x, o.fbs[k].y, o.fbs[k].z, 0.f);
                fng[4 * L.maxNN + ia * 4 + k] = make_float4(o.fps[k].x, o.fps[k].y, o.fps[k].z, 0.f);
            }
            if (ENERGY) { Eb += (double)o.E; e13 += (double)o.E13; }
        }
        // --- non-bonded pairs: S lanes per atom i, j strided by S
        if (flags & F_NONBONDED) {
            const bool pbc = (flags & F_PBC) != 0;
            const int npx = pbc ? P.npbc[0] : 0, npy = pbc ? P.npbc[1] : 0, npz = pbc ? P.npbc[2] : 0;
            const int nxi = 2 * npx + 1, nyi = 2 * npy + 1;
            // cutoff + PBC: candidate lists per shifted image, built only when the
            // bounding-box test keeps some shifted image (block-uniform)
            bool any_shift = false;
            for (int iz = -npz; iz <= npz; iz++)
                for (int iy = -npy; iy <= npy; iy++)
                    for (int ix = -npx; ix <= npx; ix++)
                        if ((ix | iy | iz) != 0) any_shift |= image_active(ix, iy, iz);
            // pair lists of the shifted images (relax kernels with a scratch slot):
            // kept while no atom moved more than skin/2 since their build
            bool vrows = false;
            int* vs = vstate();
            if (vs[0] && any_shift && P.Rc2 > 0.f && L.nimg > 0 && L.nimg <= kListMaxImages) {
                bool need = !vs[1];
                if (!need) {
                    const float4* vp = reinterpret_cast<const float4*>(vslot() + P.vcap);
                    const float lim2 = 0.25f * P.vskin * P.vskin;
                    int moved = 0;
                    for (int a = tid; a < natoms; a += T) {
                        const float4 p = spos[a], q = vp[a];
                        const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
                        moved |= !(fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= lim2);
                    }
                    need = __syncthreads_or(moved) != 0;
                }
                if (need) {
                    if (COUNT && tid == 0) atomicAdd(Y.counters + 3, 1ull);
                    const bool built = list_build(spos);
                    __syncthreads();                      // every thread has read the state
                    if (tid == 0) { vs[0] = built; vs[1] = built; }
                    __syncthreads();
                }
                vrows = vs[0] != 0;
                if (COUNT && tid == 0 && vrows) atomicAdd(Y.counters + 4, (unsigned long long)vs[2]);
            }
            const bool lists = !vrows && L.nimg > 0 && any_shift;
            if (lists) build_candidates(P.Rc2);
            const int central = (npz * nyi + npy) * nxi + npx;
            // central image and (with candidate lists) the shifted images:
            // every unordered pair once or ordered rows, into fixed-point sums
            long long* facc = at<long long>(L.facc);
            for (int a = tid; a < 3 * natoms; a += T) facc[a] = 0;
            __syncthreads();
            {
                float ec = 0.f;
                if (hasH) {
                    if (lists) pair_tiles<true, true>(spos, sREQ, pbc, central, facc, ec);
                    else pair_tiles<true, false>(spos, sREQ, pbc, central, facc, ec);
                    if (vrows) list_pairs<true>(spos, sREQ, facc, ec);
                } else {
                    if (lists) pair_tiles<false, true>(spos, sREQ, pbc, central, facc, ec);
                    else pair_tiles<false, false>(spos, sREQ, pbc, central, facc, ec);
                    if (vrows) list_pairs<false>(spos, sREQ, facc, ec);
                }
                if (ENERGY) Enb += (double)ec;
            }
            __syncthreads();
            for (int a = tid; a < natoms; a += T)
                fnb[a] = make_float4((float)facc[3 * a] * (1.f / kFix), (float)facc[3 * a + 1] * (1.f / kFix),
                                     (float)facc[3 * a + 2] * (1.f / kFix), 0.f);
            // without candidate lists: the other images of the bounding-box test,
            // ordered pairs (i, j + shift), S lanes per atom
            if (!lists && !vrows && any_shift) {
                __syncthreads();
                const int nunits = natoms * S;
                for (int u0 = 0; u0 < nunits; u0 += T) {
                    const int u = u0 + tid;
                    const int i = u / S, sub = u % S;
                    float fx = 0.f, fy = 0.f, fz = 0.f;
                    double e = 0.0;
                    if (i < natoms) {
                        const float4 pi = spos[i];
                        const float4 Ri = sREQ[i];
                        const int4 ng = ngs(i), ngC = ngc(i);
                        for (int iz = -npz; iz <= npz; iz++)
                            for (int iy = -npy; iy <= npy; iy++)
                                for (int ix = -npx; ix <= npx; ix++) {
                                    const int ipbc = ((iz + npz) * nyi + (iy + npy)) * nxi + (ix + npx);
                                    if (ipbc == central || !image_active(ix, iy, iz)) continue;
                                    float ei = 0.f;
                                    pair_image_row(spos, sREQ, i, sub, pi, Ri, ng, ngC, pbc, ipbc, ix, iy, iz, nullptr, 0, fx, fy, fz, ei);
                                    if (ENERGY) e += (double)ei;
                                }
                    }
#pragma unroll
                    for (int o = S / 2; o > 0; o >>= 1) {
                        fx += __shfl_xor_sync(0xffffffffu, fx, o);
                        fy += __shfl_xor_sync(0xffffffffu, fy, o);
                        fz += __shfl_xor_sync(0xffffffffu, fz, o);
                    }
                    if (i < natoms && sub == 0) {
                        const float4 a = fnb[i];
                        fnb[i] = make_float4(a.x + fx, a.y + fy, a.z + fz, 0.f);
                    }
                    if (ENERGY) Enb += 0.5 * e;
                }
            }
        } else {
            for (int a = tid; a < natoms; a += T) fnb[a] = make_float4(0, 0, 0, 0);
        }
        // --- GridFF B-spline (unless it ran beside the bonded terms)
        if (!split) grid_phase(tid, T, fgr, Eg);
        // --- direct substrate term (getSurfMorse), one thread per atom
        if (flags & F_SURF) {
            __syncthreads();
            const float4* sR = at<float4>(L.REQ);
            for (int a = tid; a < natoms; a += T) {
                const float4 p = spos[a];
                const float4 r = surf_atom(P, make_float3(p.x + gorg.x, p.y + gorg.y, p.z + gorg.z), sR[a]);
                const float4 g = fgr[a];
                fgr[a] = make_float4(g.x + r.x, g.y + r.y, g.z + r.z, 0.f);
                if (ENERGY) Eg += (double)r.w;
            }
        }
    }

    // ------------------------------------------------------------------ phase 2
    // assemble + clamp; FP64 partial sums of (vf, vv, ff) and max|f|^2 for this thread
    __device__ void assemble(double& vf, double& vv, double& ff, float& fmax2, bool& bad) {
        float4* fasm = at<float4>(L.fasm);
        const float4* fnb = at<float4>(L.fnb);
        const float4* fgr = at<float4>(L.fgrid);
        const float4* fng = at<float4>(L.fng);
        const float4* spos = at<float4>(L.pos);
        const float4* svel = at<float4>(L.vel);
        const float Fl2 = P.Flim * P.Flim;
        for (int v = tid; v < nvecs; v += T) {
            float3 f;
            if (v < natoms) {
                const float4 a = fasm[v], b = fnb[v], c = fgr[v];
                f = make_float3(a.x + b.x + c.x, a.y + b.y + c.y, a.z + b.z + c.z);
                const int4 bk = bks(v);
                const int bks[4] = {bk.x, bk.y, bk.z, bk.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (bks[k] < 0) break;
                    f = f + f3(fng[bks[k]]);
                }
            } else {
                const int ia = v - natoms;
                f = f3(fasm[v]);
                const int4 bk = bks(ia);
                const int bks[4] = {bk.x, bk.y, bk.z, bk.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (bks[k] < 0) break;
                    f = f + f3(fng[4 * L.maxNN + bks[k]]);
                }
                const float3 u = f3(spos[v]);
                f = fma3(u, -dot3(f, u), f);      // Vec3::makeOrthoU
            }
            if ((P.flags & F_BCONS) && v < natoms) f = bond_constraint_force(Y, isys, v, spos, lv, f);
            if (P.Flim > 0.f) {
                const float fr2 = dot3(f, f);
                if (fr2 > Fl2) f = f * (P.Flim * rsqrtf(fr2));
            }
            if ((P.flags & F_CONSTR) && v < natoms) f = constraint_force(Y, aoff + v, f3(spos[v]), f);
            // a system whose atoms left any sensible range (no force clamp,
            // bad start) is retired like a non-finite one
            if (v < natoms) { const float4 p = spos[v]; bad |= !(fabsf(p.x) + fabsf(p.y) + fabsf(p.z) < 1e5f); }
            fasm[v] = make_float4(f.x, f.y, f.z, 0.f);
            const float4 vv4 = svel[v];
            vf += (double)vv4.x * f.x + (double)vv4.y * f.y + (double)vv4.z * f.z;
            vv += (double)vv4.x * vv4.x + (double)vv4.y * vv4.y + (double)vv4.z * vv4.z;
            const double f2 = (double)f.x * f.x + (double)f.y * f.y + (double)f.z * f.z;
            ff += f2;
            fmax2 = fmaxf(fmax2, (float)f2);
            bad |= !isfinite(f.x + f.y + f.z);
        }
        bad |= pairbad;
    }

    // block reduction of 3 doubles + one float max (+flag); result in all threads
    __device__ void reduce4(double& a, double& b, double& c, float& m, bool& bad) {
        double* red = at<double>(L.red);
        a = wsum(a); b = wsum(b); c = wsum(c); m = wmax(m);
        const int anybad = __any_sync(0xffffffffu, bad);
        if (lane == 0) {
            red[4 * warp + 0] = a; red[4 * warp + 1] = b; red[4 * warp + 2] = c;
            reinterpret_cast<float*>(red + 4 * warp + 3)[0] = m;
            reinterpret_cast<int*>(red + 4 * warp + 3)[1] = anybad;
        }
        __syncthreads();
        a = 0; b = 0; c = 0; m = 0.f; int nb = 0;
        for (int w = 0; w < L.nwarps; w++) {
            a += red[4 * w + 0]; b += red[4 * w + 1]; c += red[4 * w + 2];
            m = fmaxf(m, reinterpret_cast<const float*>(red + 4 * w + 3)[0]);
            nb |= reinterpret_cast<const int*>(red + 4 * w + 3)[1];
        }
        bad = nb != 0;
    }

    // ------------------------------------------------------------------ phase 3
    __device__ void move(double dt, double cv, double cfm, float* mn, float* mx) {
        float4* spos = at<float4>(L.pos);
        float4* svel = at<float4>(L.vel);
        const float4* fasm = at<float4>(L.fasm);
        const float dtf = (float)dt;
        const float cvf = (float)cv;
        const float kf = (float)((double)dtf + cfm);
        for (int v = tid; v < nvecs; v += T) {
            float3 f = f3(fasm[v]), ve = f3(svel[v]), p = f3(spos[v]);
            const bool bPi = v >= natoms;
            if (bPi) f = fma3(p, -dot3(p, f), f);
            ve = ve * cvf;
            ve = fma3(f, kf, ve);
            if (bPi) ve = fma3(p, -dot3(p, ve), ve);
            p = fma3(ve, dtf, p);
            if (bPi) p = p * rsqrtf(dot3(p, p));
            spos[v] = make_float4(p.x, p.y, p.z, 0.f);
            svel[v] = make_float4(ve.x, ve.y, ve.z, 0.f);
            if (!bPi) {
                mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
                mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
            }
        }
    }

    // Langevin step (MMFFsp3_loc::move_atom_Langevin, MMFFsp3_loc.h:1191-1216):
    // f - gamma v + uniform(-1,1) * sqrt(2 kB T gamma / dt), then v += f dt,
    // p += v dt; pi vectors keep unit length and stay orthogonal to their force
    __device__ void move_md(int step, float* mn, float* mx) {
        float4* spos = at<float4>(L.pos);
        float4* svel = at<float4>(L.vel);
        const float4* fasm = at<float4>(L.fasm);
        const float dt = P.md_dt, g = P.md_gamma, nz = P.md_noise;
        for (int v = tid; v < nvecs; v += T) {
            float3 f = f3(fasm[v]), ve = f3(svel[v]), p = f3(spos[v]);
            const bool bPi = v >= natoms;
            if (bPi) f = fma3(p, -dot3(p, f), f);
            f = fma3(ve, -g, f);
            const long long gv = (long long)voff + v;
            f.x = fmaf(langevin_rand(P.md_seed, gv, step, 0), nz, f.x);
            f.y = fmaf(langevin_rand(P.md_seed, gv, step, 1), nz, f.y);
            f.z = fmaf(langevin_rand(P.md_seed, gv, step, 2), nz, f.z);
            ve = fma3(f, dt, ve);
            if (bPi) ve = fma3(p, -dot3(p, ve), ve);
            p = fma3(ve, dt, p);
            if (bPi) p = p * rsqrtf(dot3(p, p));
            spos[v] = make_float4(p.x, p.y, p.z, 0.f);
            svel[v] = make_float4(ve.x, ve.y, ve.z, 0.f);
            if (!bPi) {
                mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
                mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
            }
        }
    }

    // copy of the positions just moved (each thread its own vectors, as in move)
    __device__ void snapshot() {
        const float4* spos = at<float4>(L.pos);
        for (int v = tid; v < nvecs; v += T) Y.minpos[voff + v] = spos[v];
    }

    __device__ void store_state(int status, int steps, float fconv, double dt, double damping, int lastNeg, double total) {
        const float4* spos = at<float4>(L.pos);
        const float4* svel = at<float4>(L.vel);
        const float4* fasm = at<float4>(L.fasm);
        for (int v = tid; v < nvecs; v += T) {
            Y.pos[voff + v] = spos[v];
            Y.vel[voff + v] = svel[v];
            Y.force[voff + v] = fasm[v];
        }
        if (tid == 0) {
            Y.fire[isys] = make_double4(dt, damping, (double)lastNeg, total);
            Y.status[isys] = status;
            Y.nsteps[isys] = steps;
            Y.fconv[isys] = fconv;
        }
    }
};

// ---------------------------------------------------------------------------
// Persistent relaxation: claims systems from queue[] via counter.
// resident CTAs per SM the register allocation of the relax kernel targets,
// per thread count (build options; without a target ptxas caps at 128
// registers and spills)
#ifndef MMFF_MINB_T64
#define MMFF_MINB_T64 8
#endif
#ifndef MMFF_MINB_T128
#define MMFF_MINB_T128 4
#endif
#ifndef MMFF_MINB_T256
#define MMFF_MINB_T256 2
#endif
template <int T> constexpr int relax_min_blocks() {
    return T == 64 ? MMFF_MINB_T64 : T == 128 ? MMFF_MINB_T128 : T == 256 ? MMFF_MINB_T256 : 1;
}

// P.vlist (null: none): scratch for the shifted-image pair lists, P.vstride
// 32-bit words per CTA (P.vcap entries, then 4 * maxNA words of positions).
// EXPL: the exploring cycle (P.md_mode 2) instead of plain FIRE or the drive.
template <int T, int S, bool COUNT, bool EXPL = false>
__global__ void __launch_bounds__(T, relax_min_blocks<T>()) relax_kernel(Params P, Systems Y, const int* __restrict__ queue, int nqueue,
                                                  int* counter, int maxNA, int maxNN) {
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_claim;
    const SmemLayout L = smem_layout(maxNA, maxNN, T, P.Rc2 > 0.f ? shifted_images(P.flags, P.npbc) : 0);
    Engine<T, S, false, COUNT> E(P, Y, smem, L);
    while (true) {
        if (threadIdx.x == 0) s_claim = atomicAdd(counter, 1);
        __syncthreads();
        const int q = s_claim;
        if (q >= nqueue) break;
        const int s = queue[q];
        E.load(s);
        const double4 fs = Y.fire[s];
        double dt = fs.x, damping = fs.y, total = fs.w;
        int lastNeg = (int)fs.z;
        __syncthreads();
        E.bbox_from_smem();
        int status = ST_MAXSTEPS, itr = 0;
        float meas = 0.f;
        int ph = 0;                 // exploring cycle: 2 * (steps in the phase) + exploring
        if constexpr (EXPL) { const int4 g = Y.gopt[s]; ph = 2 * g.y + (g.x != 0); }
        for (itr = 0; itr < P.nstep_max; itr++) {
            bool lang = false;      // an exploring step (Langevin instead of FIRE)
            if constexpr (EXPL) {
                const int ev = explore_step(ph, P.n_explore, P.n_relax);
                lang = ev & 1;
                if ((ev & 2) && threadIdx.x == 0) Y.gopt[s].w++;
            }
            double d0 = 0, d1 = 0, d2 = 0;
            E.forces(d0, d1, d2);
            __syncthreads();
            double vf = 0, vv = 0, ff = 0;
            float fmax2 = 0.f;
            bool bad = false;
            E.assemble(vf, vv, ff, fmax2, bad);
            E.reduce4(vf, vv, ff, fmax2, bad);
            if (bad) { status = ST_NAN; break; }
            if (!EXPL && P.md_mode) {   // Langevin drive: fixed number of steps, no FIRE
                float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                E.move_md(P.md_step0 + itr, mn, mx);
                total += 1.0;
                meas = sqrtf(fmax2);
                E.bbox_reduce(mn, mx);
                continue;
            }
            // DynamicOpt::FIRE_update_params (FP64, identical in every thread); in the
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
            float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            if (EXPL && lang) E.move_md(P.md_step0 + itr, mn, mx);
            else E.move(dt, cv, P.fire_variant == 1 ? cf : renorm_vf * cf, mn, mx);
            total += 1.0;
            const double m = (P.conv_mode == 0) ? ff : (double)fmax2;
            meas = (float)sqrt(m);
            if constexpr (EXPL) {
                if (!lang && m < P.Fconv2) {
                    // a minimum (MolWorld_sp3.h:2465-2473): keep it, start exploring
                    E.snapshot();
                    if (threadIdx.x == 0) Y.gopt[s].z++;
                    ph = 1;
                }
            } else {
                if (m < P.Fconv2) { status = ST_CONVERGED; itr++; E.bbox_reduce(mn, mx); break; }
            }
            E.bbox_reduce(mn, mx);   // contains the end-of-step barrier
        }
        // converged at step itr-1 (reference returns the loop index at break)
        const int steps = (status == ST_CONVERGED) ? itr - 1 : itr;
        __syncthreads();
        E.store_state(status, steps, meas, dt, damping, lastNeg, total);
        if (EXPL && threadIdx.x == 0) { Y.gopt[s].x = ph & 1; Y.gopt[s].y = ph >> 1; }
        if (COUNT) {
            // force evaluations done for this system: itr loop iterations
            if (threadIdx.x == 0) {
                atomicAdd(Y.counters + 1, (unsigned long long)itr * (unsigned long long)E.natoms);
                atomicAdd(Y.counters + 2, (unsigned long long)itr);
            }
        }
        __syncthreads();
    }
    if (COUNT) atomicAdd(Y.counters, E.npair);
}

// One force (and energy) evaluation per system; blockIdx.x indexes queue[].
template <int T, int S, bool ENERGY>
__global__ void __launch_bounds__(T) eval_kernel(Params P, Systems Y, const int* __restrict__ queue, int nqueue,
                                                 int maxNA, int maxNN) {
    extern __shared__ __align__(16) char smem[];
    const SmemLayout L = smem_layout(maxNA, maxNN, T, P.Rc2 > 0.f ? shifted_images(P.flags, P.npbc) : 0);
    Engine<T, S, ENERGY> E(P, Y, smem, L);
    const int q = blockIdx.x;
    if (q >= nqueue) return;
    const int s = queue[q];
    E.load(s);
    __syncthreads();
    E.bbox_from_smem();
    double Eb = 0, Enb = 0, Eg = 0;
    E.forces(Eb, Enb, Eg);
    __syncthreads();
    // (the host passes Flim <= 0 here: eval reports unclamped forces)
    double vf = 0, vv = 0, ff = 0;
    float fmax2 = 0.f;
    bool bad = false;
    E.assemble(vf, vv, ff, fmax2, bad);
    __syncthreads();
    const float4* fasm = E.template at<float4>(L.fasm);
    for (int v = threadIdx.x; v < E.nvecs; v += T) Y.force[E.voff + v] = fasm[v];
    if (ENERGY) {
        // the reference's split: the skipped 1-3 pair energies belong to the
        // pair sum and their subtraction to the bonded part; the total is
        // summed without them
        double eb = Eb, enb = Enb, eg = Eg, x13 = E.e13, z0 = 0.0, z1 = 0.0;
        float dummy = 0.f;
        bool b2 = false;
        __syncthreads();
        E.reduce4(eb, enb, eg, dummy, b2);
        __syncthreads();
        E.reduce4(x13, z0, z1, dummy, b2);
        if (threadIdx.x == 0) Y.energy[s] = make_double4(eb - x13, enb + x13, eg, eb + enb + eg);
    }
    if (threadIdx.x == 0) Y.fconv[s] = sqrtf(fmax2);
}

// B-spline sample of n points (grid parity tests): fe = (Fx, Fy, Fz, E)
__global__ void grid_sample_kernel(Params P, int n, const float4* __restrict__ pos, const float4* __restrict__ PLQ,
                                   float4* __restrict__ fe) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = u >> 2, a = u & 3;
    float4 r = make_float4(0, 0, 0, 0);
    if (i < n) {
        const float4 p = pos[i];
        const float3 uu = make_float3(p.x * P.ginv[0], p.y * P.ginv[1], p.z * P.ginv[2]);
        r = grid_slice(P.grid, P.gn[0], P.gn[1], P.gn[2], uu, PLQ[i], a);
    }
#pragma unroll
    for (int o = 2; o > 0; o >>= 1) {
        r.x += __shfl_xor_sync(0xffffffffu, r.x, o);
        r.y += __shfl_xor_sync(0xffffffffu, r.y, o);
        r.z += __shfl_xor_sync(0xffffffffu, r.z, o);
        r.w += __shfl_xor_sync(0xffffffffu, r.w, o);
    }
    if (i < n && a == 0) fe[i] = make_float4(r.x * P.gmi[0], r.y * P.gmi[1], r.z * P.gmi[2], r.w);
}


// address of the kernel instantiation for (T, S)
#define MMFF_TS_SWITCH(T, S, ...)                                                            \
    switch (T * 16 + S) {                                                                     \
        case 64 * 16 + 1: { constexpr int T_ = 64, S_ = 1; __VA_ARGS__; }                            \
        case 64 * 16 + 2: { constexpr int T_ = 64, S_ = 2; __VA_ARGS__; }                            \
        case 64 * 16 + 4: { constexpr int T_ = 64, S_ = 4; __VA_ARGS__; }                            \
        case 64 * 16 + 8: { constexpr int T_ = 64, S_ = 8; __VA_ARGS__; }                            \
        case 128 * 16 + 1: { constexpr int T_ = 128, S_ = 1; __VA_ARGS__; }                          \
        case 128 * 16 + 2: { constexpr int T_ = 128, S_ = 2; __VA_ARGS__; }                          \
        case 128 * 16 + 4: { constexpr int T_ = 128, S_ = 4; __VA_ARGS__; }                          \
        case 128 * 16 + 8: { constexpr int T_ = 128, S_ = 8; __VA_ARGS__; }                          \
        case 256 * 16 + 1: { constexpr int T_ = 256, S_ = 1; __VA_ARGS__; }                          \
        case 256 * 16 + 2: { constexpr int T_ = 256, S_ = 2; __VA_ARGS__; }                          \
        case 256 * 16 + 4: { constexpr int T_ = 256, S_ = 4; __VA_ARGS__; }                          \
        case 256 * 16 + 8: { constexpr int T_ = 256, S_ = 8; __VA_ARGS__; }                          \
        case 512 * 16 + 1: { constexpr int T_ = 512, S_ = 1; __VA_ARGS__; }                          \
        case 512 * 16 + 2: { constexpr int T_ = 512, S_ = 2; __VA_ARGS__; }                          \
        case 512 * 16 + 4: { constexpr int T_ = 512, S_ = 4; __VA_ARGS__; }                          \
        case 512 * 16 + 8: { constexpr int T_ = 512, S_ = 8; __VA_ARGS__; }                          \
        default: return nullptr;                                                              \
    }

void* relax_fn(int T, int S, bool count) {
    if (count) { MMFF_TS_SWITCH(T, S, return (void*)relax_kernel<T_, S_, true>) }
    MMFF_TS_SWITCH(T, S, return (void*)relax_kernel<T_, S_, false>)
}
// the exploring cycle runs one pair lane per atom (S = 1) at any block size
void* relax_explore_fn(int T) {
    switch (T) {
        case 64: return (void*)relax_kernel<64, 1, false, true>;
        case 128: return (void*)relax_kernel<128, 1, false, true>;
        case 256: return (void*)relax_kernel<256, 1, false, true>;
        case 512: return (void*)relax_kernel<512, 1, false, true>;
        default: return nullptr;
    }
}
void* eval_fn(int T, int S, bool energy) {
    if (energy) { MMFF_TS_SWITCH(T, S, return (void*)eval_kernel<T_, S_, true>) }
    MMFF_TS_SWITCH(T, S, return (void*)eval_kernel<T_, S_, false>)
}

}  // namespace mmff
