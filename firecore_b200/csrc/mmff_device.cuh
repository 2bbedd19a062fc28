// mmff_device.cuh -- device-side physics of the multi-system MMFF relaxer.
//
// Every function restates, in FP32, the reference C++ physics the FP64 oracle
// (oracle/mmff_oracle.c) follows:
//   bonded  : MMFFsp3_loc::eval_atom        cpp/common/molecular/MMFFsp3_loc.h:250-575
//             (Forces.h evalBond :137, evalAngleCosHalf :190, evalAngleCos :217,
//              evalPiAling :230, getLJQH :341)
//   pair    : NBFF::evalLJQs_ng4_PBC_atom_omp cpp/common/molecular/NBFF.h:575-618
//   grid    : Bspline::fe3d_pbc_comb3        cpp/common/math/Bspline.h:742-809
//             via GridFF::getForce_Bspline    cpp/common/molecular/GridFF.h:355-402
//   assemble: MMFFsp3_loc::assemble_atom     cpp/common/molecular/MMFFsp3_loc.h:998-1021
//   FIRE    : DynamicOpt::FIRE_update_params cpp/common/math/DynamicOpt.cpp:250-267
//             MMFFsp3_loc::move_atom_FIRE    cpp/common/molecular/MMFFsp3_loc.h:1264-1281
// Precision: forces in FP32; the per-system FIRE sums, the FIRE decision and the
// convergence test in FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define MMFF_COULOMB 14.3996448915f

namespace mmff {

// ---- flags (same bit meaning as the oracle's ORC_* flags)
enum : int {
    F_BONDS = 1 << 0, F_PIPI = 1 << 1, F_PISIGMA = 1 << 2, F_ANGLES = 1 << 3,
    F_SUB_ANGLE_NB = 1 << 4, F_SUB_BOND_NB = 1 << 5, F_CLAMP_NB = 1 << 6,
    F_NONBONDED = 1 << 7, F_GRID = 1 << 8, F_PBC = 1 << 9, F_SURF = 1 << 10,
    // set by the host (never by callers): the 1-3 pairs of the angle terms
    // are left out of the central-image pair sum instead of being added there
    // and subtracted again in the angle term (see pair13)
    F_EXCL13 = 1 << 11,
    // set by the host for relaxations when position constraints are uploaded
    F_CONSTR = 1 << 12,
    F_BCONS = 1 << 13,   // distance / angle constraints between atoms (Constrains bonds / angles)
};

// The host turns F_EXCL13 on exactly when the angle terms subtract the 1-3
// pair term that the pair sum adds and nothing clamps the pair forces.
__host__ __device__ inline bool excl13_active(int flags) {
    return (flags & F_SUB_ANGLE_NB) && (flags & F_ANGLES) && (flags & F_NONBONDED) && !(flags & F_CLAMP_NB);
}

// status codes per system
enum : int { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXSTEPS = 2, ST_NAN = -1 };

struct Params {
    int flags;
    int npbc[3];
    float Rc2;           // cutoff^2 (<=0: none)
    float kq_rc2;        // 1/Rcut^2 for the shifted-force Coulomb
    float Fmax2NB;       // bClampNonBonded
    // grid
    int gn[3];
    float ginv[3];       // 1/step
    float gmi[3];        // -1/step
    const float4* __restrict__ grid;   // [nx][ny][nz] (P, L, Q, 0)
    // FIRE
    double dt_max, dt_min, damp_max, finc, fdec, falpha, cv_kill;
    int minLastNeg;
    int fire_variant;    // 0: run_no_omp mixing f*(dt + renorm*cf); 1: Bitzek 2006 mixing f*(dt + cf)
    float Flim;          // <=0: no force clamp
    double Fconv2;
    int conv_mode;       // 0: sum f^2 ; 1: max |f|^2
    int nstep_max;       // steps allowed in this call
    // Langevin drive (md_mode 1) instead of FIRE: MMFFsp3_loc::move_atom_Langevin;
    // md_mode 2: the exploring cycle of GOpt (Langevin for n_explore steps after
    // every minimum found, or after n_relax FIRE steps without one)
    int md_mode;
    float md_dt, md_gamma, md_noise;   // noise = sqrt(2 kB T gamma / dt)
    unsigned long long md_seed;
    int md_step0;                      // step index of the call's first step (random stream)
    int n_explore, n_relax;            // md_mode 2 (n_relax <= 0: no give-up)
    // direct substrate term (F_SURF): substrate atoms in world coordinates
    const float4* __restrict__ surf_pos;
    const float4* __restrict__ surf_REQ;   // (R0, sqrt(E0), Q sqrt(k_e), H)
    int nsurf;
    int snpbc[3];
    float slv[9];                          // substrate lattice vectors a, b, c
    float sK, sR2damp;                     // -alphaMorse, Rdamp^2
    float sg0[3];                          // grid origin: world = local + gorg + sg0
    // shifted-image pair lists of the CTA relax kernels (null: none): vstride
    // 32-bit words per CTA, the first vcap of them list entries
    uint32_t* vlist;
    int vstride, vcap;
    float vskin;                           // list skin [A]
};

// Counter-based uniform random number in [-1, 1) for the Langevin force:
// SplitMix64 (Steele, Lea & Flood 2014) of (seed, vector, step, component);
// 24 random bits, so the value is exact in float and double.
__host__ __device__ inline unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ inline float langevin_rand(unsigned long long seed, long long vec, int step, int comp) {
    const unsigned long long key =
        seed ^ mix64(((unsigned long long)(unsigned)step << 32) ^ ((unsigned long long)vec << 2) ^ (unsigned long long)comp);
    return (float)(mix64(key) >> 40) * (2.0f / 16777216.0f) - 1.0f;
}

// Exploring cycle of the global optimiser (md_mode 2), one call per step before
// the forces: a FIRE phase longer than n_relax steps is given up
// (MolWorld_sp3_multi.h:797-803), then GOpt::update (GOpt.h:46-56) counts the
// step and ends an exploring phase once it reaches n_explore steps.
// ph = 2 * (steps in the phase) + exploring; returns bit 0: this step explores
// (Langevin instead of FIRE), bit 1: a FIRE phase was given up.
__device__ __forceinline__ int explore_step(int& ph, int n_explore, int n_relax) {
    int ev = 0;
    if (!(ph & 1) && n_relax > 0 && (ph >> 1) > n_relax) { ph = 1; ev = 2; }
    ph += 2;
    if ((ph & 1) && (ph >> 1) >= n_explore) ph = 0;
    return ev | (ph & 1);
}

struct Systems {
    int nsys;
    const int4* __restrict__ desc;      // (aoff, noff, voff, natoms)
    const int* __restrict__ nnode;
    const float* __restrict__ lvec;     // [nsys*9]
    const float4* __restrict__ gorg;    // grid offset of the local frame: orig - pos0
    const float4* __restrict__ REQ;     // (R0, sqrt(E0), Q*sqrt(k_e), Hb)
    const float4* __restrict__ PLQ;     // (P, L, Q, H) for the grid
    const int4* __restrict__ neighs;
    const int4* __restrict__ neighCell;
    const int4* __restrict__ bkneighs;
    const float4* __restrict__ apars;
    const float4* __restrict__ bLs;
    const float4* __restrict__ bKs;
    const float4* __restrict__ Ksp;
    const float4* __restrict__ Kpp;
    const int* __restrict__ a13;        // per node: angle pairs (bit t of slots i<j) whose 1-3 pair the pair sum skips
    const uint32_t* __restrict__ xmask; // central-image exclusion words: row (atom i) of ceil(natoms/32) words per system
    const int* __restrict__ moff;       // per system: first word of its exclusion rows
    const float4* __restrict__ constr;  // per atom: spring anchor (local frame) and w > 0 = on (F_CONSTR)
    const float4* __restrict__ constrK; // per atom: spring constants (kx, ky, kz)
    // distance / angle constraints (F_BCONS): (system, or -1 for every system; local atom indices)
    const int4* __restrict__ dcon_i;    // (system, i0, i1, -)
    const float4* __restrict__ dcon_a;  // (lmax, lmin, kmax, kmin)
    const float4* __restrict__ dcon_b;  // (shift along a, b, c in cell units, flim)
    int ndcon;
    const int4* __restrict__ acon_i;    // (system, centre, end 1, end 2)
    const float4* __restrict__ acon_a;  // (cos a0/2, sin a0/2, k, -)
    int nacon;
    unsigned int* gkey;                 // per atom: stencil cell of its GridFF cache (0xffffffff: empty); null: no cache
    float4* gcs;                        // per atom: 16 float4 = PLQ . C of its 4x4x4 stencil ([x][y] rows of 4 z)
    float4* pos;                        // local frame
    float4* vel;
    float4* force;                      // assembled forces (written by eval / at exit)
    double4* fire;                      // (dt, damping, lastNeg, total steps)
    int* status;
    int* nsteps;                        // steps done in the last call
    float* fconv;                       // convergence measure at exit (sqrt)
    double4* energy;                    // eval only: (bonded, non-bonded, grid, total)
    unsigned long long* counters;       // counting builds: pair-images, atom grid samples, force evaluations
    // exploring cycle (md_mode 2): per system (exploring, steps in the phase,
    // minima found, relax phases given up); per vector the last minimum found
    int4* gopt;
    float4* minpos;                     // local frame, like pos
};

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float f) { return make_float3(a.x * f, a.y * f, a.z * f); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ float3 fma3(float3 a, float f, float3 c) { return make_float3(fmaf(a.x, f, c.x), fmaf(a.y, f, c.y), fmaf(a.z, f, c.z)); }

// image index c (NBFF.h:42 ordering: x fastest, then y, then z) -> shift
// in lattice units.  Quotients by the small image counts go through a float
// reciprocal: (c + 1/2) / n stays >= 1/(2n) away from an integer, far beyond
// the 2-ulp error of __fdividef, so the integer parts are exact.
__device__ __forceinline__ float3 image_cell(int c, int npx, int npy, int npz) {
    const int nx = 2 * npx + 1, ny = 2 * npy + 1;
    const int q = (int)__fdividef((float)c + 0.5f, (float)nx);
    const int r = (int)__fdividef((float)q + 0.5f, (float)ny);
    return make_float3((float)(c - q * nx - npx), (float)(q - r * ny - npy), (float)(r - npz));
}

// i mod n into [0, n) for grid indices (same float-reciprocal argument)
__device__ __forceinline__ int wrap_index(int i, int n) {
    const int q = (int)floorf(__fdividef((float)i + 0.5f, (float)n));
    return i - q * n;
}

// Forces.h:341 getLJQH with undamped Coulomb; REQ holds the pair-mixed values with
// Q = k_e*Qi*Qj.  Returns the scalar F with f = dp * F (the reference's -F).
template <bool ENERGY>
__device__ __forceinline__ float ljqh(float r2, float R0, float E0, float Q, float hw, float& E) {
    const float ir = rsqrtf(r2);
    const float ir2 = ir * ir;
    const float Eel = Q * ir;
    const float u2 = R0 * R0 * ir2;
    const float u6 = u2 * u2 * u2;
    const float vdW = u6 * E0;
    const float H = u6 * vdW * hw;              // u6*u6*(w<0 ? w*E0 : 0)
    if (ENERGY) E = fmaf(u6 - 2.f, vdW, Eel + H);
    return -fmaf(12.f * ir2, fmaf(u6 - 1.f, vdW, H), Eel * ir2);
}

// 1-3 pair (ends of an angle) of the angle term, MMFFsp3_loc.h:525-538.  The
// reference adds this pair in the pair sum and subtracts getLJQH of it here;
// both are ~10^2-10^3 eV/A for close 1-3 contacts, so in FP32 the difference
// keeps the rounding of the large terms.  With x13 the pair sum skipped the
// pair (central image), and this adds what the pair term has beyond getLJQH:
// the shifted-force Coulomb part inside the cutoff (zero without one), or
// -getLJQH beyond it.  Either way the total equals the reference's sum in
// exact arithmetic.  Returns the scalar F of the force on the first atom
// (dp * F, dp = p_second - p_first); e: energy change, ep (x13 only): the
// pair energy the pair sum would have counted (for the energy split).
template <bool ENERGY>
__device__ __forceinline__ float pair13(float r2, float4 Ri, float4 Rj, bool x13, float Rc2, float kq, float rc,
                                        float& e, float& ep) {
    const float R0 = Ri.x + Rj.x, E0 = Ri.y * Rj.y, Q = Ri.z * Rj.z, hw = fminf(Ri.w * Rj.w, 0.f);
    if (x13 && r2 < Rc2) {
        const float ir = rsqrtf(r2);
        if (ENERGY) {
            float eL;
            ljqh<true>(r2, R0, E0, Q, hw, eL);
            e = Q * kq * (r2 * ir - 2.f * rc);
            ep = eL + e;
        }
        return Q * kq * ir;
    }
    float eL = 0.f;
    const float F = ljqh<ENERGY>(r2, R0, E0, Q, hw, eL);
    if (ENERGY) { e = -eL; ep = 0.f; }
    return -F;
}

// scalar pair force F (f_i += d F with d = p_j - p_i) of one pair-image, the
// arithmetic of the pair loops (rsqrt form of getLJQH, Forces.h:341-360, plus
// the shifted-force Coulomb term); ok: inside the cutoff and not excluded.
// Excluded / out-of-range pairs are evaluated at r^2 = 1e30, where every term
// underflows to zero except kq Q / r (< 1e-16 eV/A).
template <bool ENERGY, bool HB>
__device__ __forceinline__ float pair_force(float dx, float dy, float dz, float4 Ri, float4 Rj, bool excl, float Rc2,
                                            float kq, float rc, bool cut, bool& ok, float& e) {
    float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    ok = !excl && (r2 < Rc2);
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
    if (ENERGY) {
        e = 0.f;
        if (ok) {
            e = fmaf(u6 - 2.f, vdW, Eel + H);
            if (cut) e += Q * kq * (r2 * ir - 2.f * rc);
        }
    }
    return F;
}

// Direct substrate term of one atom, getSurfMorse / getMorseQH
// (relax_multi.cl:2741-2877, :166-181): Morse E0 e (e - 2), e = exp(K (r - R0)),
// plus Coulomb k Q / sqrt(r^2 + Rdamp^2), over every substrate atom and its
// images.  pw: atom position relative to the grid origin.  Returns (F, E).
__device__ __forceinline__ float4 surf_atom(const Params& P, float3 pw, float4 Ri) {
    const float K = P.sK, R2d = P.sR2damp;
    pw = make_float3(pw.x + P.sg0[0], pw.y + P.sg0[1], pw.z + P.sg0[2]);
    float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
    for (int j = 0; j < P.nsurf; j++) {
        const float4 sp = __ldg(P.surf_pos + j), Rj = __ldg(P.surf_REQ + j);
        const float R0 = Ri.x + Rj.x, E0 = Ri.y * Rj.y, Q = Ri.z * Rj.z;
        for (int iz = -P.snpbc[2]; iz <= P.snpbc[2]; iz++)
            for (int iy = -P.snpbc[1]; iy <= P.snpbc[1]; iy++)
                for (int ix = -P.snpbc[0]; ix <= P.snpbc[0]; ix++) {
                    const float dx = pw.x - (sp.x + P.slv[0] * ix + P.slv[3] * iy + P.slv[6] * iz);
                    const float dy = pw.y - (sp.y + P.slv[1] * ix + P.slv[4] * iy + P.slv[7] * iz);
                    const float dz = pw.z - (sp.z + P.slv[2] * ix + P.slv[5] * iy + P.slv[8] * iz);
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    const float ir2d = 1.f / (r2 + R2d);
                    const float ir = rsqrtf(r2);
                    const float r = r2 * ir;
                    const float e = expf(K * (r - R0));
                    const float Ae = E0 * e;
                    const float fM = Ae * 2.f * K * (e - 1.f);
                    const float Eel = Q * sqrtf(ir2d);
                    const float fr = fM * ir - Eel * ir2d;
                    fx = fmaf(-dx, fr, fx); fy = fmaf(-dy, fr, fy); fz = fmaf(-dz, fr, fz);
                    E += fmaf(Ae, e - 2.f, Eel);
                }
    }
    return make_float4(fx, fy, fz, E);
}

// ----- bonded terms (one node atom), MMFFsp3_loc::eval_atom
struct BondedOut {
    float3 fa, fpi;
    float3 fbs[4], fps[4];
    float E;
    float E13;      // ENERGY: pair energies of the 1-3 pairs the pair sum skipped
};

// cutoff constants of the pair term as the 1-3 residual needs them
struct Cut13 {
    float Rc2, kq, rc;
    __device__ __forceinline__ Cut13(const Params& P) {
        const bool cut = P.Rc2 > 0.f;
        Rc2 = cut ? P.Rc2 : 3.0e38f;
        kq = P.kq_rc2;
        rc = cut ? sqrtf(1.f / kq) : 0.f;
    }
};

// Position constraint of one atom (relax_multi.cl:995-1010, updateAtomsMMFFf4):
// with anchor.w > 0 the force gains (anchor - p) * max(K, 0) per component,
// after the force clamp; pi orbitals have none.
__device__ __forceinline__ float3 constraint_force(const Systems& Y, int ia, float3 p, float3 f) {
    const float4 c = __ldg(Y.constr + ia);
    if (c.w > 0.f) {
        const float4 k = __ldg(Y.constrK + ia);
        f.x = fmaf(c.x - p.x, fmaxf(k.x, 0.f), f.x);
        f.y = fmaf(c.y - p.y, fmaxf(k.y, 0.f), f.y);
        f.z = fmaf(c.z - p.z, fmaxf(k.z, 0.f), f.z);
    }
    return f;
}

// Distance and angle constraints acting on atom ia of system isys
// (constrains.h: DistConstr::apply with Forces.h:161 spring, AngleConstr::apply
// with evalAngleCosHalf; applied by MolWorld_sp3::run_no_omp after the force
// field, MolWorld_sp3.h:2391-2395, so before the force clamp).  sp: the system's
// positions, lv: its cell (rows a, b, c).  Each constraint is evaluated by each
// of its atoms for its own share.
static __device__ __forceinline__ float3 bond_constraint_force(const Systems& Y, int isys, int ia, const float4* sp, const float* lv,
                                                     float3 f) {
    for (int c = 0; c < Y.ndcon; c++) {
        const int4 d = __ldg(Y.dcon_i + c);
        if ((d.x >= 0 && d.x != isys) || (d.y != ia && d.z != ia)) continue;
        const float4 A = __ldg(Y.dcon_a + c), B = __ldg(Y.dcon_b + c);
        const float3 p0 = f3(sp[d.y]), p1 = f3(sp[d.z]);
        const float3 dd = make_float3(p1.x - p0.x + (lv[0] * B.x + lv[3] * B.y + lv[6] * B.z),
                                      p1.y - p0.y + (lv[1] * B.x + lv[4] * B.y + lv[7] * B.z),
                                      p1.z - p0.z + (lv[2] * B.x + lv[5] * B.y + lv[8] * B.z));
        const float l = sqrtf(dot3(dd, dd));
        float fs = 0.f;                                   // flat-bottom spring between lmin and lmax
        if (l > A.x) fs = fminf((l - A.x) * A.z, B.w);
        else if (l < A.y) fs = fmaxf((l - A.y) * A.w, -B.w);
        const float3 g = dd * (fs / l);
        if (ia == d.y) f = f + g;
        if (ia == d.z) f = f - g;
    }
    for (int c = 0; c < Y.nacon; c++) {
        const int4 a = __ldg(Y.acon_i + c);
        if ((a.x >= 0 && a.x != isys) || (a.y != ia && a.z != ia && a.w != ia)) continue;
        const float4 A = __ldg(Y.acon_a + c);
        const float3 pc = f3(sp[a.y]);
        float3 h1 = pc - f3(sp[a.z]), h2 = pc - f3(sp[a.w]);
        const float ir1 = rsqrtf(dot3(h1, h1)), ir2 = rsqrtf(dot3(h2, h2));
        h1 = h1 * ir1; h2 = h2 * ir2;
        const float3 h = h1 + h2;                          // evalAngleCosHalf (Forces.h:190)
        float c2 = dot3(h, h) * 0.25f;
        const float s2 = 1.f - c2 + 1e-14f;
        const float cc = sqrtf(c2), ss = sqrtf(fmaxf(s2, 0.f));
        const float csy = fmaf(A.y, cc, -A.x * ss);
        float fr = -A.z * csy;
        c2 *= -2.f;
        fr = fr / (4.f * cc * ss);
        const float fr1 = fr * ir1, fr2 = fr * ir2;
        const float3 f1 = h * fr1 + h1 * (fr1 * c2), f2 = h * fr2 + h2 * (fr2 * c2);
        if (ia == a.y) f = f + f1 + f2;
        if (ia == a.z) f = f - f1;
        if (ia == a.w) f = f - f2;
    }
    return f;
}

// angle pair index of neighbour slots i < j (0..5): (0,1) (0,2) (0,3) (1,2) (1,3) (2,3)
__host__ __device__ constexpr int angle_slot(int i, int j) { return i * (7 - i) / 2 + (j - i - 1); }

template <bool ENERGY>
__device__ __forceinline__ void eval_atom(int ia, int natoms, int nnode, int flags, float Fmax2,
                                          const float4* sp, const float4* sREQ, int4 ng, int4 ngC,
                                          float4 apar, float4 bL, float4 bK, float4 ksp, float4 kpp,
                                          const float* lv, int npx, int npy, int npz, int a13, const Cut13& cu,
                                          BondedOut& o) {
    const float3 pa = f3(sp[ia]);
    const float3 hpi = f3(sp[natoms + ia]);
    float3 fa = make_float3(0, 0, 0), fpi = make_float3(0, 0, 0);
    float3 fbs[4], fps[4];
    float3 hf[4];
    float he[4], hl[4];
    float E = 0.f, E13 = 0.f;
    const int ings[4] = {ng.x, ng.y, ng.z, ng.w};
    const int ingC[4] = {ngC.x, ngC.y, ngC.z, ngC.w};
    const float bLa[4] = {bL.x, bL.y, bL.z, bL.w};
    const float bKa[4] = {bK.x, bK.y, bK.z, bK.w};
    const float Kspa[4] = {ksp.x, ksp.y, ksp.z, ksp.w};
    const float Kppa[4] = {kpp.x, kpp.y, kpp.z, kpp.w};
#pragma unroll
    for (int i = 0; i < 4; i++) { fbs[i] = make_float3(0, 0, 0); fps[i] = make_float3(0, 0, 0); hf[i] = make_float3(0, 0, 1); he[i] = 1.f; hl[i] = 1.f; }
    int nb = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int ing = ings[i];
        if (ing < 0) break;
        nb = i + 1;
        float3 h = f3(sp[ing]) - pa;
        if (flags & F_PBC) {
            // shift of image ingC (NBFF.h:42 ordering: iz outer, iy, ix inner)
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
                const float dl = l - bLa[i];
                const float fr = dl * bKa[i];
                float3 f1 = h * fr;
                if (ENERGY) E += fr * dl * 0.5f;
                if (flags & F_SUB_BOND_NB) {
                    const float4 Ri = sREQ[ia], Rj = sREQ[ing];
                    const float hw = fminf(Ri.w * Rj.w, 0.f);
                    float e;
                    const float3 dp = h * l;
                    const float F = ljqh<ENERGY>(l * l, Ri.x + Rj.x, Ri.y * Rj.y, Ri.z * Rj.z, hw, e);
                    float3 fij = dp * F;
                    if (flags & F_CLAMP_NB) { float f2 = dot3(fij, fij); if (f2 > Fmax2) fij = fij * sqrtf(Fmax2 / f2); }
                    if (ENERGY) E -= e;
                    f1 = f1 - fij;
                }
                fbs[i] = fbs[i] - f1; fa = fa + f1;
            }
            const float kk = Kppa[i];
            if ((flags & F_PIPI) && (ing < nnode) && (kk > 1e-6f)) {
                // Forces.h:230 evalPiAling with ir1 = ir2 = 1
                const float3 h2 = f3(sp[natoms + ing]);
                float c = dot3(hpi, h2);
                const float3 a = fma3(hpi, -c, h2);
                const float3 b = fma3(h2, -c, hpi);
                const bool sign = c < 0.f;
                if (sign) c = -c;
                if (ENERGY) E += kk * (1.f - c);
                const float fang = sign ? -kk : kk;
                fpi = fpi + a * fang;
                fps[i] = fps[i] + b * fang;
            }
        }
        const float ks = Kspa[i];
        if ((flags & F_PISIGMA) && (ks > 1e-6f)) {
            // Forces.h:217 evalAngleCos(hpi, h, 1, 1/l, ksp, piC0)
            const float c = dot3(hpi, h);
            const float3 a = fma3(hpi, -c, h);
            const float3 b = fma3(h, -c, hpi);
            const float c_ = c - apar.w;
            if (ENERGY) E += ks * c_ * c_;
            const float fang = -ks * c_ * 2.f;
            fpi = fpi + a * fang;
            const float3 f2 = b * (fang * il);
            fa = fa - f2;
            fbs[i] = fbs[i] + f2;
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
                // Forces.h:190 evalAngleCosHalf
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
                    const int ing = ings[i], jng = ings[j];
                    const float3 dp = hf[j] * hl[j] - hf[i] * hl[i];
                    // x13: the pair sum skipped this central-image pair
                    const bool x13 = (flags & F_EXCL13) && ((a13 >> angle_slot(i, j)) & 1) &&
                                     (!(flags & F_PBC) || ingC[i] == ingC[j]);
                    float e = 0.f, ep = 0.f;
                    const float F = pair13<ENERGY>(dot3(dp, dp), sREQ[ing], sREQ[jng], x13, cu.Rc2, cu.kq, cu.rc, e, ep);
                    float3 fij = dp * F;
                    if (flags & F_CLAMP_NB) { float ff = dot3(fij, fij); if (ff > Fmax2) fij = fij * sqrtf(Fmax2 / ff); }
                    if (ENERGY) { E += e; E13 += ep; }
                    f1 = f1 + fij;
                    f2 = f2 - fij;
                }
                fbs[i] = fbs[i] + f1;
                fbs[j] = fbs[j] + f2;
            }
        }
    }
    o.fa = fa; o.fpi = fpi;
#pragma unroll
    for (int i = 0; i < 4; i++) { o.fbs[i] = fbs[i]; o.fps[i] = fps[i]; }
    o.E = E;
    o.E13 = E13;
}

// ----- cubic B-spline basis (Bspline.h:254, :267)
__device__ __forceinline__ float4 bs_basis(float u) {
    const float u2 = u * u, t = 1.f - u;
    const float inv6 = 1.f / 6.f;
    return make_float4(inv6 * t * t * t, inv6 * fmaf(3.f * u2, u - 2.f, 4.f), inv6 * fmaf(3.f * u, 1.f + u - u2, 1.f), inv6 * u2 * u);
}
__device__ __forceinline__ float4 bs_dbasis(float u) {
    const float u2 = u * u, t = 1.f - u;
    return make_float4(-0.5f * t * t, 0.5f * (3.f * u2 - 4.f * u), 0.5f * (-3.f * u2 + 2.f * u + 1.f), 0.5f * u2);
}
__device__ __forceinline__ float comp(float4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }

// Grid coordinates of an atom far outside any grid (|u| >= 2^20 voxels: only
// in a system that has blown up, which the relax kernels retire) or not
// finite are replaced by the origin, so that the int conversions and the
// periodic wraps below stay in range for every input.
__device__ __forceinline__ float3 grid_safe(float3 u) {
    const float lim = 1048576.f;
    return (fabsf(u.x) < lim && fabsf(u.y) < lim && fabsf(u.z) < lim) ? u : make_float3(0.f, 0.f, 0.f);
}

// One x-slice (a = 0..3) of the 4x4x4 stencil of Bspline::fe3d_pbc_comb3 for
// grid coordinate u (already in voxel units).  Returns the slice's partial
// (dE/dx*bx', E-channel combos) as (Fx, Fy, Fz, E) *before* the -1/step scale.
// UNROLL: y-columns of the slice unrolled (their 16 loads in flight together).
// In the fused relax step of small blocks (four or eight per SM) the step's
// code, not its loads, is the limit: there no unrolling measured 5-7 % faster;
// the 256-thread blocks keep all four (5 % faster there).
template <int UNROLL = 4>
__device__ __forceinline__ float4 grid_slice(const float4* __restrict__ G, int nx, int ny, int nz, float3 u,
                                             float4 PLQ, int a) {
    u = grid_safe(u);
    int ix = (int)u.x, iy = (int)u.y, iz = (int)u.z;
    if (u.x < 0.f) ix--;
    if (u.y < 0.f) iy--;
    const float tx = u.x - (float)ix, ty = u.y - (float)iy, tz = u.z - (float)iz;
    iz = min(max(iz, 3), nz - 5);
    ix = wrap_index(ix - 1, nx);
    iy = wrap_index(iy - 1, ny);
    // x index of this slice with periodic wrap (Bspline.h:36-53 choose_inds_pbc)
    int xa = ix + a; if (xa >= nx) xa -= nx;
    const float4 bz = bs_basis(tz), dz = bs_dbasis(tz);
    const float4 by = bs_basis(ty), dy = bs_dbasis(ty);
    float ex = 0.f, ey = 0.f, ez = 0.f;   // per slice: d/dy combo, d/dz combo, value
#pragma unroll UNROLL
    for (int b = 0; b < 4; b++) {
        int yb = iy + b; if (yb >= ny) yb -= ny;
        const float4* col = G + ((size_t)(xa * ny + yb) * nz + (iz - 1));
        const float4 c0 = __ldg(col), c1 = __ldg(col + 1), c2 = __ldg(col + 2), c3 = __ldg(col + 3);
        const float cs0 = fmaf(PLQ.x, c0.x, fmaf(PLQ.y, c0.y, PLQ.z * c0.z));
        const float cs1 = fmaf(PLQ.x, c1.x, fmaf(PLQ.y, c1.y, PLQ.z * c1.z));
        const float cs2 = fmaf(PLQ.x, c2.x, fmaf(PLQ.y, c2.y, PLQ.z * c2.z));
        const float cs3 = fmaf(PLQ.x, c3.x, fmaf(PLQ.y, c3.y, PLQ.z * c3.z));
        const float v = fmaf(bz.x, cs0, fmaf(bz.y, cs1, fmaf(bz.z, cs2, bz.w * cs3)));
        const float d = fmaf(dz.x, cs0, fmaf(dz.y, cs1, fmaf(dz.z, cs2, dz.w * cs3)));
        const float byb = comp(by, b), dyb = comp(dy, b);
        ex = fmaf(v, dyb, ex);
        ey = fmaf(d, byb, ey);
        ez = fmaf(v, byb, ez);
    }
    const float4 bx = bs_basis(tx), dx = bs_dbasis(tx);
    const float bxa = comp(bx, a), dxa = comp(dx, a);
    return make_float4(dxa * ez, bxa * ex, bxa * ey, bxa * ez);
}

// grid_slice with a per-atom cache of the 64 channel-combined coefficients
// PLQ . C of the atom's stencil (PLQ is constant per atom).  An atom whose
// stencil cell is the cached one reads its 16 numbers of slice a (4 float4,
// 64 contiguous bytes) instead of gathering 16 float4 of the grid (256 B from
// four columns); on a cell change the slice is gathered, combined and stored
// as before.  The arithmetic is the same as grid_slice's, so results are
// bit-identical.  All 32 lanes of the warp call it (a shuffle inside); the
// four lanes of an atom are consecutive (lane a = lane & 3); ok = the lane
// holds a real atom.  The cache of an atom is read and written only by the
// block that owns its system in this launch; a block barrier separates steps.
template <int UNROLL = 4>
__device__ __forceinline__ float4 grid_slice_cached(const float4* __restrict__ G, int nx, int ny, int nz, float3 u,
                                                    float4 PLQ, int a, bool ok, unsigned int* gkey, float4* gcs,
                                                    int atom) {
    u = grid_safe(u);
    int ix = (int)u.x, iy = (int)u.y, iz = (int)u.z;
    if (u.x < 0.f) ix--;
    if (u.y < 0.f) iy--;
    const float tx = u.x - (float)ix, ty = u.y - (float)iy, tz = u.z - (float)iz;
    iz = min(max(iz, 3), nz - 5);
    ix = wrap_index(ix - 1, nx);
    iy = wrap_index(iy - 1, ny);
    const unsigned key = ((unsigned)ix * 4096u + (unsigned)iy) * 256u + (unsigned)iz;
    unsigned old = 0xffffffffu;
    if (ok && a == 0) old = gkey[atom];
    old = __shfl_sync(0xffffffffu, old, (threadIdx.x & 31) & ~3);
    const bool hit = ok && old == key;
    float4* mine = gcs + (size_t)atom * 16 + 4 * a;
    int xa = ix + a; if (xa >= nx) xa -= nx;
    const float4 bz = bs_basis(tz), dz = bs_dbasis(tz);
    const float4 by = bs_basis(ty), dy = bs_dbasis(ty);
    float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll UNROLL
    for (int b = 0; b < 4; b++) {
        float4 cs;
        if (hit) {
            cs = mine[b];
        } else {
            int yb = iy + b; if (yb >= ny) yb -= ny;
            const float4* col = G + ((size_t)(xa * ny + yb) * nz + (iz - 1));
            const float4 c0 = __ldg(col), c1 = __ldg(col + 1), c2 = __ldg(col + 2), c3 = __ldg(col + 3);
            cs.x = fmaf(PLQ.x, c0.x, fmaf(PLQ.y, c0.y, PLQ.z * c0.z));
            cs.y = fmaf(PLQ.x, c1.x, fmaf(PLQ.y, c1.y, PLQ.z * c1.z));
            cs.z = fmaf(PLQ.x, c2.x, fmaf(PLQ.y, c2.y, PLQ.z * c2.z));
            cs.w = fmaf(PLQ.x, c3.x, fmaf(PLQ.y, c3.y, PLQ.z * c3.z));
            if (ok) mine[b] = cs;
        }
        const float v = fmaf(bz.x, cs.x, fmaf(bz.y, cs.y, fmaf(bz.z, cs.z, bz.w * cs.w)));
        const float d = fmaf(dz.x, cs.x, fmaf(dz.y, cs.y, fmaf(dz.z, cs.z, dz.w * cs.w)));
        const float byb = comp(by, b), dyb = comp(dy, b);
        ex = fmaf(v, dyb, ex);
        ey = fmaf(d, byb, ey);
        ez = fmaf(v, byb, ez);
    }
    if (ok && !hit && a == 0) gkey[atom] = key;
    const float4 bx = bs_basis(tx), dx = bs_dbasis(tx);
    const float bxa = comp(bx, a), dxa = comp(dx, a);
    return make_float4(dxa * ez, bxa * ex, bxa * ey, bxa * ez);
}

// B-spline GridFF force + energy of one atom, the whole 4x4x4 stencil in this
// lane (Bspline::fe3d_pbc_comb3, Bspline.h:742-809; the same index and basis
// arithmetic as grid_slice)
__device__ __forceinline__ float4 grid_atom(const Params& P, float3 u, float4 PLQ) {
    const int nx = P.gn[0], ny = P.gn[1], nz = P.gn[2];
    const float4* __restrict__ G = P.grid;
    u = grid_safe(u);
    int ix = (int)u.x, iy = (int)u.y, iz = (int)u.z;
    if (u.x < 0.f) ix--;
    if (u.y < 0.f) iy--;
    const float tx = u.x - (float)ix, ty = u.y - (float)iy, tz = u.z - (float)iz;
    iz = min(max(iz, 3), nz - 5);
    ix = wrap_index(ix - 1, nx);
    iy = wrap_index(iy - 1, ny);
    const float4 bz = bs_basis(tz), dz = bs_dbasis(tz);
    const float4 by = bs_basis(ty), dy = bs_dbasis(ty);
    const float4 bx = bs_basis(tx), dx = bs_dbasis(tx);
    float Fx = 0.f, Fy = 0.f, Fz = 0.f, E = 0.f;
#pragma unroll 1
    for (int a = 0; a < 4; a++) {
        int xa = ix + a; if (xa >= nx) xa -= nx;
        float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            int yb = iy + b; if (yb >= ny) yb -= ny;
            const float4* col = G + ((size_t)(xa * ny + yb) * nz + (iz - 1));
            const float4 c0 = __ldg(col), c1 = __ldg(col + 1), c2 = __ldg(col + 2), c3 = __ldg(col + 3);
            const float cs0 = fmaf(PLQ.x, c0.x, fmaf(PLQ.y, c0.y, PLQ.z * c0.z));
            const float cs1 = fmaf(PLQ.x, c1.x, fmaf(PLQ.y, c1.y, PLQ.z * c1.z));
            const float cs2 = fmaf(PLQ.x, c2.x, fmaf(PLQ.y, c2.y, PLQ.z * c2.z));
            const float cs3 = fmaf(PLQ.x, c3.x, fmaf(PLQ.y, c3.y, PLQ.z * c3.z));
            const float v = fmaf(bz.x, cs0, fmaf(bz.y, cs1, fmaf(bz.z, cs2, bz.w * cs3)));
            const float d = fmaf(dz.x, cs0, fmaf(dz.y, cs1, fmaf(dz.z, cs2, dz.w * cs3)));
            const float byb = comp(by, b), dyb = comp(dy, b);
            ex = fmaf(v, dyb, ex);
            ey = fmaf(d, byb, ey);
            ez = fmaf(v, byb, ez);
        }
        const float bxa = (a == 0) ? bx.x : (a == 1) ? bx.y : (a == 2) ? bx.z : bx.w;
        const float dxa = (a == 0) ? dx.x : (a == 1) ? dx.y : (a == 2) ? dx.z : dx.w;
        Fx = fmaf(dxa, ez, Fx); Fy = fmaf(bxa, ex, Fy); Fz = fmaf(bxa, ey, Fz); E = fmaf(bxa, ez, E);
    }
    return make_float4(Fx * P.gmi[0], Fy * P.gmi[1], Fz * P.gmi[2], E);
}


// ---- shared-memory carve-up of one system (byte offsets)
struct SmemLayout {
    int maxNA, maxNN, maxNV, nwarps, nimg, nwords;
    // offsets in bytes
    int pos, vel, fasm, fnb, fgrid, REQ, PLQ, ng, ngC, bk, apar, bL, bK, ksp, kpp, fng, red;
    int cwords, cpref, ccnt, clist;     // per-image candidate lists (cutoff + PBC only)
    int facc, total;                    // fixed-point force sums of the central image [3 * maxNA] int64
    int stage;                          // image tiles: per warp the 32 j of the current tile (pos, REQ), or -1
};

// number of shifted (non-central) PBC images of the pair term
__host__ __device__ inline int shifted_images(int flags, const int* npbc) {
    if (!(flags & F_PBC)) return 0;
    return (2 * npbc[0] + 1) * (2 * npbc[1] + 1) * (2 * npbc[2] + 1) - 1;
}

// Layouts above this size would hold one CTA per SM.  Above it, the arrays
// read once per atom (or node) per step stay in global memory and are read
// through L1: neighbours, their cells, back-neighbour slots, GridFF
// coefficients and the node parameters (offset -1 in the layout).  That
// brings a 400-atom system under half of the SM's shared memory.  Only
// blocks of >= 256 threads take it (smaller blocks compile without the
// global-memory branch).
constexpr int kCompactAbove = 112 * 1024;
constexpr int kCompactMinThreads = 256;

// Image tiles are compiled into blocks of >= 128 threads only: the 64-thread
// blocks serve molecules of <= 64 atoms, whose images reach a few edge atoms
// (short candidate lists, ordered rows), and without the tile code there the
// code of their central tiles stays as it is.
constexpr int kImageTileMinThreads = 128;
// shifted-image pair lists of the CTA relax kernels: shifted images handled
// (2-D cells have 8) and the average list entries per atom a slot holds
constexpr int kListMaxImages = 12;
constexpr int kListEntriesPerAtom = 48;

__host__ __device__ inline SmemLayout smem_layout_(int maxNA, int maxNN, int T, int nimg, bool compact) {
    SmemLayout L;
    L.maxNA = maxNA; L.maxNN = maxNN; L.maxNV = maxNA + maxNN; L.nwarps = T / 32;
    L.nimg = nimg; L.nwords = (maxNA + 31) / 32;
    int o = 0;
    auto take = [&](int bytes) { int r = o; o += (bytes + 15) & ~15; return r; };
    auto opt = [&](int bytes) { return compact ? -1 : take(bytes); };
    L.pos = take(16 * L.maxNV);
    L.vel = take(16 * L.maxNV);
    L.fasm = take(16 * L.maxNV);
    L.fnb = take(16 * maxNA);
    L.fgrid = take(16 * maxNA);
    L.REQ = take(16 * maxNA);
    L.PLQ = opt(16 * maxNA);
    L.ng = opt(16 * maxNA);
    L.ngC = opt(16 * maxNA);
    L.bk = opt(16 * maxNA);
    L.apar = opt(16 * maxNN);
    L.bL = opt(16 * maxNN);
    L.bK = opt(16 * maxNN);
    L.ksp = opt(16 * maxNN);
    L.kpp = opt(16 * maxNN);
    L.fng = take(16 * 8 * maxNN);
    L.red = take(128 * L.nwarps + 64);     // per warp: 4 doubles (32 B) at 0, bbox 6 floats at 64*nwarps
    L.cwords = take(4 * nimg * L.nwords);   // candidate bit words per image
    L.cpref = take(4 * nimg * L.nwords);    // exclusive prefix of their popcounts
    L.ccnt = take(4 * nimg);                // candidates per image
    L.clist = take(2 * nimg * maxNA);       // candidate atom indices per image, ascending
    L.facc = take(8 * 3 * maxNA);
    // image tiles (blocks >= kImageTileMinThreads with candidate lists): the
    // positions and parameters of a tile's 32 candidates j, copied once per
    // tile so that the 32 rotation steps read them directly instead of through
    // the candidate list
    L.stage = (nimg > 0 && T >= kImageTileMinThreads) ? take(2 * 16 * 32 * L.nwarps) : -1;
    L.total = o;
    return L;
}

// nimg: shifted images that get candidate lists (0: none)
__host__ __device__ inline SmemLayout smem_layout(int maxNA, int maxNN, int T, int nimg) {
    const SmemLayout L = smem_layout_(maxNA, maxNN, T, nimg, false);
    return (T >= kCompactMinThreads && L.total > kCompactAbove) ? smem_layout_(maxNA, maxNN, T, nimg, true) : L;
}

// ---- shared-memory carve-up of one warp-per-system region (byte offsets)
struct WarpLayout {
    int pos, REQ, fng, misc, ng, ngC, bk, npar, per_warp;   // byte offsets inside one warp's region
};
__host__ __device__ inline WarpLayout warp_layout(int maxNA, int maxNN) {
    WarpLayout L;
    int o = 0;
    auto take = [&](int b) { int r = o; o += (b + 15) & ~15; return r; };
    L.pos = take(16 * (maxNA + maxNN));
    L.REQ = take(16 * maxNA);
    L.fng = take(16 * 8 * maxNN);
    L.misc = take(16 * 4);          // lattice vectors (9 floats) + grid offset (3 floats)
    L.ng = take(16 * maxNA);
    L.ngC = take(16 * maxNA);
    L.bk = take(16 * maxNA);
    L.npar = take(16 * 5 * maxNN);  // apars, bLs, bKs, Ksp, Kpp per node
    L.per_warp = o;
    return L;
}

}  // namespace mmff
