/*
 * mmff_oracle.c -- FP64 CPU restatement of the MMFF multi-system relaxation
 * hot path (TEST INFRASTRUCTURE: the checker, never the product).
 *
 * Each function names the reference function (file:line inside the FireCore
 * tree) whose arithmetic it restates.  Operation order follows the reference
 * so that FP64 results agree to rounding with the compiled reference harness
 * (oracle/ref_harness.cpp) on the golden fixtures.
 *
 * Extensions beyond the reference (both off by default): a non-bonded cutoff
 * (P->Rcut > 0, Coulomb in shifted-force form) and a per-vector force clamp in
 * FIRE (F->Flim > 0, as relax_multi.cl:980-983).  With Rcut <= 0 the pair sum
 * is the reference's all-pairs x all-images sum.
 */
#include "mmff_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define COULOMB_CONST 14.3996448915   /* cpp/common_resources/cl/relax_multi.cl:79, constants.h */

typedef struct { double x, y, z; } v3;

static inline v3   v3make(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3   vadd(v3 a, v3 b) { return v3make(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3   vsub(v3 a, v3 b) { return v3make(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3   vmul(v3 a, double f) { return v3make(a.x * f, a.y * f, a.z * f); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* a += b*f  (Vec3::add_mul) */
static inline v3   vaddmul(v3 a, v3 b, double f) { return v3make(a.x + b.x * f, a.y + b.y * f, a.z + b.z * f); }
/* A*fa + B*fb  (Vec3::set_lincomb) */
static inline v3   vlin(double fa, v3 A, double fb, v3 B) { return v3make(A.x * fa + B.x * fb, A.y * fa + B.y * fb, A.z * fa + B.z * fb); }

static inline v3 ld3(const double* p) { return v3make(p[0], p[1], p[2]); }
static inline void st3(double* p, v3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

/* ---------------- scalar force kernels (cpp/common/math/Forces.h) ---------------- */

/* Forces.h:137 evalBond */
static inline double evalBond(v3 h, double dl, double k, v3* f) {
    double fr = dl * k;
    *f = vmul(h, fr);
    return fr * dl * 0.5;
}

/* Forces.h:190 evalAngleCosHalf (Vec2::udiv_cmplx, math/Vec2.h:130) */
static inline double evalAngleCosHalf(v3 h1, v3 h2, double ir1, double ir2,
                                      double cs0x, double cs0y, double k, v3* f1, v3* f2) {
    v3 h = vadd(h1, h2);
    double c2 = vdot(h, h) * 0.25;
    double s2 = 1 - c2 + 1e-14;
    double c = sqrt(c2);
    double s = sqrt(s2);
    double csx = cs0x * c + cs0y * s;
    double csy = cs0y * c - cs0x * s;
    double E = k * (1 - csx);
    double fr = -k * (csy);
    c2 *= -2;
    fr /= 4 * c * s;
    double fr1 = fr * ir1;
    double fr2 = fr * ir2;
    *f1 = vlin(fr1, h, fr1 * c2, h1);
    *f2 = vlin(fr2, h, fr2 * c2, h2);
    return E;
}

/* Forces.h:217 evalAngleCos */
static inline double evalAngleCos(v3 h1, v3 h2, double ir1, double ir2, double K, double c0, v3* f1, v3* f2) {
    double c = vdot(h1, h2);
    v3 a = vaddmul(h2, h1, -c);
    v3 b = vaddmul(h1, h2, -c);
    double c_ = c - c0;
    double E = K * c_ * c_;
    double fang = -K * c_ * 2;
    *f1 = vmul(a, fang * ir1);
    *f2 = vmul(b, fang * ir2);
    return E;
}

/* Forces.h:230 evalPiAling */
static inline double evalPiAling(v3 h1, v3 h2, double K, v3* f1, v3* f2) {
    double c = vdot(h1, h2);
    v3 a = vaddmul(h2, h1, -c);
    v3 b = vaddmul(h1, h2, -c);
    int sign = c < 0; if (sign) c = -c;
    double E = K * (1 - c);
    double fang = K;
    if (sign) fang = -fang;
    *f1 = vmul(a, fang);
    *f2 = vmul(b, fang);
    return E;
}

/* Forces.h:341 getLJQH (undamped Coulomb + H-bond correction); REQ already mixed */
static inline double getLJQH(v3 dp, const double* REQ, v3* f) {
    const double r2 = vdot(dp, dp);
    const double ir2 = 1 / r2;
    double E = COULOMB_CONST * REQ[2] * sqrt(ir2);
    double F = E * ir2;
    const double u2 = REQ[0] * REQ[0] * ir2;
    const double u6 = u2 * u2 * u2;
    const double vdW = u6 * REQ[1];
    const double H = u6 * u6 * ((REQ[3] < 0) ? REQ[3] * REQ[1] : 0.0);
    E += (u6 - 2.) * vdW + H;
    F += ((u6 - 1.) * vdW + H) * ir2 * 12;
    *f = vmul(dp, -F);
    return E;
}

/* Forces.h:270 _mixREQ */
static inline void mixREQ(const double* A, const double* B, double* o) {
    o[0] = A[0] + B[0]; o[1] = A[1] * B[1]; o[2] = A[2] * B[2]; o[3] = A[3] * B[3];
}

/* clampForce (Forces.h) : scale f so |f|^2 <= Fmax2 */
static inline v3 clampForce(v3 f, double Fmax2) {
    double f2 = vdot(f, f);
    if (f2 > Fmax2) { f = vmul(f, sqrt(Fmax2 / f2)); }
    return f;
}

/* NBFF.h:42 makePBCshifts_ ordering: iz outer, iy, ix inner */
static inline v3 pbc_shift(const double* lv, const int* np, int ipbc) {
    int nx = 2 * np[0] + 1, ny = 2 * np[1] + 1;
    int ix = ipbc % nx - np[0];
    int iy = (ipbc / nx) % ny - np[1];
    int iz = ipbc / (nx * ny) - np[2];
    v3 a = ld3(lv), b = ld3(lv + 3), c = ld3(lv + 6);
    return vadd(vadd(vmul(a, ix), vmul(b, iy)), vmul(c, iz));
}

typedef struct {
    int natoms, nnode, nvecs;
    const double* pos;       /* [nvecs*3] */
    const int* neighs; const int* neighCell; const int* bkneighs;
    const double* REQs; const double* apars; const double* bLs; const double* bKs;
    const double* Ksp; const double* Kpp; const double* lvec;
    double* fneigh;          /* [nnode*4*3] */
    double* fneighpi;        /* [nnode*4*3] */
    double* force;           /* [nvecs*3] */
    v3* shifts;              /* [npbc] */
    int npbc;
} sysview;

/* MMFFsp3_loc.h:250-575 eval_atom (non-templated path; no collision damping,
 * bEachAngle=false, bAngleCosHalf=true) */
static double eval_atom(const sysview* S, const ORC_params* P, int ia) {
    const int flags = P->flags;
    double E = 0;
    const double Fmax2 = P->FmaxNonBonded * P->FmaxNonBonded;
    const v3 pa = ld3(S->pos + 3 * ia);
    const v3 hpi = ld3(S->pos + 3 * (S->natoms + ia));
    v3 fa = v3make(0, 0, 0), fpi = v3make(0, 0, 0);
    const int* ings = S->neighs + ia * 4;
    const int* ingC = S->neighCell + ia * 4;
    const double* bK = S->bKs + ia * 4;
    const double* bL = S->bLs + ia * 4;
    const double* Kspi = S->Ksp + ia * 4;
    const double* Kppi = S->Kpp + ia * 4;
    double* fbs = S->fneigh + ia * 12;
    double* fps = S->fneighpi + ia * 12;
    const double* apar = S->apars + ia * 4;
    const double piC0 = apar[3];
    v3 hsf[4]; double hse[4];
    v3 f1, f2;
    v3 fb[4], fp[4];
    for (int i = 0; i < 4; i++) { fb[i] = v3make(0, 0, 0); fp[i] = v3make(0, 0, 0); }

    for (int i = 0; i < 4; i++) {
        int ing = ings[i];
        if (ing < 0) break;
        v3 h = vsub(ld3(S->pos + 3 * ing), pa);
        if (flags & ORC_PBC) { h = vadd(h, S->shifts[ingC[i]]); }
        /* Vec3::normalize (math/Vec3.h:149) */
        double l = sqrt(h.x * h.x + h.y * h.y + h.z * h.z);
        double il = 1.0 / l;
        h = vmul(h, il);
        double he = 1 / l;
        hsf[i] = h; hse[i] = he;
        if (ia < ing) {
            if (flags & ORC_BONDS) {
                E += evalBond(h, l - bL[i], bK[i], &f1);
                if (flags & ORC_SUB_BOND_NB) {
                    double REQij[4]; mixREQ(S->REQs + 4 * ia, S->REQs + 4 * ing, REQij);
                    v3 dp = vmul(h, l);
                    v3 fij;
                    E -= getLJQH(dp, REQij, &fij);
                    if (flags & ORC_CLAMP_NB) fij = clampForce(fij, Fmax2);
                    f1 = vsub(f1, fij);
                }
                fb[i] = vsub(fb[i], f1); fa = vadd(fa, f1);
            }
            double kpp = Kppi[i];
            if ((flags & ORC_PIPI) && (ing < S->nnode) && (kpp > 1e-6)) {
                E += evalPiAling(hpi, ld3(S->pos + 3 * (S->natoms + ing)), kpp, &f1, &f2);
                fpi = vadd(fpi, f1); fp[i] = vadd(fp[i], f2);
            }
        }
        double ksp = Kspi[i];
        if ((flags & ORC_PISIGMA) && (ksp > 1e-6)) {
            E += evalAngleCos(hpi, h, 1., he, ksp, piC0, &f1, &f2);
            fpi = vadd(fpi, f1); fa = vsub(fa, f2); fb[i] = vadd(fb[i], f2);
        }
    }
    if (flags & ORC_ANGLES) {
        const double ssK = apar[2];
        const double cs0x = apar[0], cs0y = apar[1];
        for (int i = 0; i < 3; i++) {
            int ing = ings[i];
            if (ing < 0) break;
            for (int j = i + 1; j < 4; j++) {
                int jng = ings[j];
                if (jng < 0) break;
                E += evalAngleCosHalf(hsf[i], hsf[j], hse[i], hse[j], cs0x, cs0y, ssK, &f1, &f2);
                fa = vsub(fa, vadd(f1, f2));
                if (flags & ORC_SUB_ANGLE_NB) {
                    double REQij[4]; mixREQ(S->REQs + 4 * ing, S->REQs + 4 * jng, REQij);
                    v3 dp = vlin(1. / hse[j], hsf[j], -1. / hse[i], hsf[i]);
                    v3 fij;
                    E -= getLJQH(dp, REQij, &fij);
                    if (flags & ORC_CLAMP_NB) fij = clampForce(fij, Fmax2);
                    f1 = vsub(f1, fij);
                    f2 = vadd(f2, fij);
                }
                fb[i] = vadd(fb[i], f1);
                fb[j] = vadd(fb[j], f2);
            }
        }
    }
    for (int i = 0; i < 4; i++) { st3(fbs + 3 * i, fb[i]); st3(fps + 3 * i, fp[i]); }
    st3(S->force + 3 * ia, fa);
    st3(S->force + 3 * (S->natoms + ia), fpi);
    return E;
}

/* NBFF.h:575-618 evalLJQs_ng4_PBC_atom_omp (returns 0.5*E; adds force) */
static double eval_nb_atom(const sysview* S, const ORC_params* P, int ia) {
    const v3 pi = ld3(S->pos + 3 * ia);
    const double* REQi = S->REQs + 4 * ia;
    const int* ng = S->neighs + 4 * ia;
    const int* ngC = S->neighCell + 4 * ia;
    const int usePBC = (P->flags & ORC_PBC) != 0;
    const int npbc = usePBC ? S->npbc : 1;
    const int cut = P->Rcut > 0;
    const double Rc2 = P->Rcut * P->Rcut;
    double E = 0, fx = 0, fy = 0, fz = 0;
    for (int j = 0; j < S->natoms; j++) {
        if (ia == j) continue;
        double REQij[4]; mixREQ(REQi, S->REQs + 4 * j, REQij);
        const v3 dp = vsub(ld3(S->pos + 3 * j), pi);
        const int bBonded = (j == ng[0]) || (j == ng[1]) || (j == ng[2]) || (j == ng[3]);
        for (int ipbc = 0; ipbc < npbc; ipbc++) {
            const v3 dpc = usePBC ? vadd(dp, S->shifts[ipbc]) : dp;
            if (bBonded) {
                if (usePBC) {
                    if (((j == ng[0]) && (ipbc == ngC[0])) || ((j == ng[1]) && (ipbc == ngC[1])) ||
                        ((j == ng[2]) && (ipbc == ngC[2])) || ((j == ng[3]) && (ipbc == ngC[3]))) continue;
                } else {
                    continue;  /* NBFF::evalLJQs_ng4_atom_omp skips bonded j entirely */
                }
            }
            v3 fij;
            double eij;
            if (cut) {
                /* extension: pairs beyond Rcut dropped; Coulomb in shifted-force
                 * form so the force is continuous at Rcut:
                 * E = kQ (1/r - 1/Rc + (r - Rc)/Rc^2), F = kQ (1/r^2 - 1/Rc^2) */
                double r2 = vdot(dpc, dpc);
                if (r2 >= Rc2) continue;
                eij = getLJQH(dpc, REQij, &fij);
                const double r = sqrt(r2);
                const double kQ = COULOMB_CONST * REQij[2];
                fij = vaddmul(fij, dpc, kQ / (Rc2 * r));
                eij += kQ * (r - 2.0 * P->Rcut) / Rc2;
            } else {
                eij = getLJQH(dpc, REQij, &fij);
            }
            E += eij;
            fx += fij.x; fy += fij.y; fz += fij.z;
        }
    }
    double* f = S->force + 3 * ia;
    f[0] += fx; f[1] += fy; f[2] += fz;
    return 0.5 * E;
}

/* ---------------- B-spline GridFF (cpp/common/math/Bspline.h) ---------------- */

/* Bspline.h:254 basis, :267 dbasis */
static inline void bs_basis(double u, double* b) {
    const double inv6 = 1. / 6.;
    const double u2 = u * u;
    const double t = 1 - u;
    b[0] = inv6 * t * t * t;
    b[1] = inv6 * (3 * u2 * (u - 2) + 4);
    b[2] = inv6 * (3 * u * (1 + u - u2) + 1);
    b[3] = inv6 * u2 * u;
}
static inline void bs_dbasis(double u, double* d) {
    const double u2 = u * u;
    const double t = 1 - u;
    d[0] = -0.5 * t * t;
    d[1] = 0.5 * (3 * u2 - 4 * u);
    d[2] = 0.5 * (-3 * u2 + 2 * u + 1);
    d[3] = 0.5 * u2;
}

static inline int modulo_i(int i, int m) { int r = i % m; if (r < 0) r += m; return r; }

/* Bspline.h:36 make_inds_pbc + :43 choose_inds_pbc */
static inline void choose_inds_pbc(int i, int n, int* q) {
    if (i >= (n - 3)) {
        int ii = i + 4 - n;
        /* iqs[ii] = {0, 1, 2, 3} with the last ii entries wrapped by -n */
        for (int k = 0; k < 4; k++) q[k] = (k >= 4 - ii) ? k - n : k;
        return;
    }
    q[0] = 0; q[1] = 1; q[2] = 2; q[3] = 3;
}

/* Bspline.h:742-809 fe3d_pbc_comb3 with fe2d_comb3 (:527) and fe1Dcomb3 (:519);
 * GridFF.h:355-402 getForce_Bspline (orthorhombic grid, inv_dg2 = -1/step). */
static void grid_fe(const double* C, const int* gn, const double* pos0, const double* step,
                    v3 p, const double* PLQ, double* fe) {
    /* GridFF uses diCell.dot_to(p - pos0) with diCell diagonal = 1/step */
    const double ux = (p.x - pos0[0]) * (1.0 / step[0]);
    const double uy = (p.y - pos0[1]) * (1.0 / step[1]);
    const double uz = (p.z - pos0[2]) * (1.0 / step[2]);
    const int nx = gn[0], ny = gn[1], nz = gn[2];
    int ix = (int)ux, iy = (int)uy, iz = (int)uz;
    if (ux < 0) ix--;
    if (uy < 0) iy--;
    const double tx = ux - ix, ty = uy - iy, tz = uz - iz;
    if (iz < 3) iz = 3; else if (iz > nz - 5) iz = nz - 5;   /* _clamp(iz,3,n.z-5) */
    ix = modulo_i(ix - 1, nx);
    iy = modulo_i(iy - 1, ny);
    const int nyz = nz * ny;
    int qx[4], qy[4];
    choose_inds_pbc(ix, nx, qx);
    choose_inds_pbc(iy, ny, qy);
    for (int k = 0; k < 4; k++) { qx[k] *= nyz; qy[k] *= nz; }
    double bz[4], dz[4], by[4], dy[4], bx[4], dx[4];
    bs_basis(tz, bz); bs_dbasis(tz, dz);
    bs_basis(ty, by); bs_dbasis(ty, dy);
    const int i0 = (iz - 1) + nz * (iy + ny * ix);
    double Ex[4], Ey[4], Ez[4];
    for (int a = 0; a < 4; a++) {
        const int base = i0 + qx[a];
        double fe0[4], fe1[4];   /* per y-column: (value, d/dz) */
        for (int b = 0; b < 4; b++) {
            const double* E = C + 3 * (base + qy[b]);
            double cs[4];
            for (int k = 0; k < 4; k++) {
                const double* e = E + 3 * k;
                cs[k] = PLQ[0] * e[0] + PLQ[1] * e[1] + PLQ[2] * e[2];
            }
            fe0[b] = bz[0] * cs[0] + bz[1] * cs[1] + bz[2] * cs[2] + bz[3] * cs[3];
            fe1[b] = dz[0] * cs[0] + dz[1] * cs[1] + dz[2] * cs[2] + dz[3] * cs[3];
        }
        Ex[a] = fe0[0] * dy[0] + fe0[1] * dy[1] + fe0[2] * dy[2] + fe0[3] * dy[3];
        Ey[a] = fe1[0] * by[0] + fe1[1] * by[1] + fe1[2] * by[2] + fe1[3] * by[3];
        Ez[a] = fe0[0] * by[0] + fe0[1] * by[1] + fe0[2] * by[2] + fe0[3] * by[3];
    }
    bs_basis(tx, bx); bs_dbasis(tx, dx);
    double Fx = dx[0] * Ez[0] + dx[1] * Ez[1] + dx[2] * Ez[2] + dx[3] * Ez[3];
    double Fy = bx[0] * Ex[0] + bx[1] * Ex[1] + bx[2] * Ex[2] + bx[3] * Ex[3];
    double Fz = bx[0] * Ey[0] + bx[1] * Ey[1] + bx[2] * Ey[2] + bx[3] * Ey[3];
    double Ee = bx[0] * Ez[0] + bx[1] * Ez[1] + bx[2] * Ez[2] + bx[3] * Ez[3];
    fe[0] = Fx * (-1.0 / step[0]);
    fe[1] = Fy * (-1.0 / step[1]);
    fe[2] = Fz * (-1.0 / step[2]);
    fe[3] = Ee;
}

/* Forces.h:611 REQ2PLQ_d */
static inline void req2plq(const double* REQ, double K, double* PLQ) {
    double e = exp(K * REQ[0]);
    double cL = e * REQ[1];
    double cP = e * cL;
    double cH = e * e * REQ[3];
    PLQ[0] = cP; PLQ[1] = cL; PLQ[2] = REQ[2]; PLQ[3] = cH;
}

void orc_req2plq(int n, const double* REQ, double K, double* PLQ) {
    for (int i = 0; i < n; i++) req2plq(REQ + 4 * i, K, PLQ + 4 * i);
}

void orc_grid_sample(int n, const double* pos, const double* PLQ, const double* gridC,
                     const ORC_params* P, double* fe) {
    for (int i = 0; i < n; i++) {
        grid_fe(gridC, P->gn, P->gpos0, P->gstep, ld3(pos + 3 * i), PLQ + 4 * i, fe + 4 * i);
    }
}

/* ---------------- one force evaluation of a system ---------------- */

/* Force phase of MolWorld_sp3::run_no_omp (MolWorld_sp3.h:2305-2386):
 * per atom: clear, eval_atom (nodes), evalLJQs_ng4_PBC_atom_omp, gridFF.addAtom;
 * then assemble_atom for all atoms (MMFFsp3_loc.h:997-1021). */
static void eval_system(sysview* S, const ORC_params* P, const double* gridC, double* Eparts) {
    double Eb = 0, Enb = 0, Eg = 0;
    for (int ia = 0; ia < S->natoms; ia++) {
        st3(S->force + 3 * ia, v3make(0, 0, 0));
        if (ia < S->nnode) st3(S->force + 3 * (ia + S->natoms), v3make(0, 0, 0));
        if (ia < S->nnode) Eb += eval_atom(S, P, ia);
        if (P->flags & ORC_NONBONDED) Enb += eval_nb_atom(S, P, ia);
        if (P->flags & ORC_GRID) {
            double PLQ[4], fe[4];
            req2plq(S->REQs + 4 * ia, P->alphaMorse, PLQ);
            grid_fe(gridC, P->gn, P->gpos0, P->gstep, ld3(S->pos + 3 * ia), PLQ, fe);
            double* f = S->force + 3 * ia;
            f[0] += fe[0]; f[1] += fe[1]; f[2] += fe[2];
            Eg += fe[3];
        }
    }
    /* assemble_atom */
    for (int ia = 0; ia < S->natoms; ia++) {
        v3 fa = v3make(0, 0, 0), fp = v3make(0, 0, 0);
        const int* ings = S->bkneighs + 4 * ia;
        int bpi = ia < S->nnode;
        for (int i = 0; i < 4; i++) {
            int j = ings[i];
            if (j < 0) break;
            fa = vadd(fa, ld3(S->fneigh + 3 * j));
            if (bpi) fp = vadd(fp, ld3(S->fneighpi + 3 * j));
        }
        double* f = S->force + 3 * ia;
        st3(f, vadd(ld3(f), fa));
        if (bpi) {
            double* fq = S->force + 3 * (S->natoms + ia);
            v3 fpv = vadd(ld3(fq), fp);
            v3 u = ld3(S->pos + 3 * (S->natoms + ia));
            double c = vdot(fpv, u);          /* Vec3::makeOrthoU */
            fpv = vaddmul(fpv, u, -c);
            st3(fq, fpv);
        }
    }
    Eparts[0] = Eb; Eparts[1] = Enb; Eparts[2] = Eg; Eparts[3] = Eb + Enb + Eg;
}

typedef struct {
    int* aoff; int* noff; int* voff;
} offsets_t;

static offsets_t make_offsets(int nsys, const int* natoms, const int* nnode) {
    offsets_t o;
    o.aoff = (int*)malloc(sizeof(int) * (nsys + 1));
    o.noff = (int*)malloc(sizeof(int) * (nsys + 1));
    o.voff = (int*)malloc(sizeof(int) * (nsys + 1));
    o.aoff[0] = o.noff[0] = o.voff[0] = 0;
    for (int s = 0; s < nsys; s++) {
        o.aoff[s + 1] = o.aoff[s] + natoms[s];
        o.noff[s + 1] = o.noff[s] + nnode[s];
        o.voff[s + 1] = o.voff[s] + natoms[s] + nnode[s];
    }
    return o;
}
static void free_offsets(offsets_t o) { free(o.aoff); free(o.noff); free(o.voff); }

static void setup_view(sysview* S, int s, const offsets_t* o, const int* natoms, const int* nnode,
                       const double* pos, double* force,
                       const int* neighs, const int* neighCell, const int* bkneighs,
                       const double* REQs, const double* apars, const double* bLs,
                       const double* bKs, const double* Ksp, const double* Kpp,
                       const double* lvec, const ORC_params* P) {
    S->natoms = natoms[s]; S->nnode = nnode[s]; S->nvecs = natoms[s] + nnode[s];
    S->pos = pos + 3 * o->voff[s];
    S->force = force + 3 * o->voff[s];
    S->neighs = neighs + 4 * o->aoff[s];
    S->neighCell = neighCell + 4 * o->aoff[s];
    S->bkneighs = bkneighs + 4 * o->aoff[s];
    S->REQs = REQs + 4 * o->aoff[s];
    S->apars = apars + 4 * o->noff[s];
    S->bLs = bLs + 4 * o->noff[s];
    S->bKs = bKs + 4 * o->noff[s];
    S->Ksp = Ksp + 4 * o->noff[s];
    S->Kpp = Kpp + 4 * o->noff[s];
    S->lvec = lvec + 9 * s;
    S->npbc = (2 * P->npbc[0] + 1) * (2 * P->npbc[1] + 1) * (2 * P->npbc[2] + 1);
    S->shifts = (v3*)malloc(sizeof(v3) * S->npbc);
    for (int k = 0; k < S->npbc; k++) S->shifts[k] = pbc_shift(S->lvec, P->npbc, k);
    S->fneigh = (double*)calloc((size_t)S->nnode * 12 + 12, sizeof(double));
    S->fneighpi = (double*)calloc((size_t)S->nnode * 12 + 12, sizeof(double));
}
static void free_view(sysview* S) { free(S->shifts); free(S->fneigh); free(S->fneighpi); }

void orc_eval(int nsys, const int* natoms, const int* nnode,
              const double* pos, double* force, double* Es,
              const int* neighs, const int* neighCell, const int* bkneighs,
              const double* REQs, const double* apars, const double* bLs,
              const double* bKs, const double* Ksp, const double* Kpp,
              const double* lvec, const double* gridC, const ORC_params* P, int nthreads) {
    offsets_t o = make_offsets(nsys, natoms, nnode);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int s = 0; s < nsys; s++) {
        sysview S;
        setup_view(&S, s, &o, natoms, nnode, pos, force, neighs, neighCell, bkneighs, REQs,
                   apars, bLs, bKs, Ksp, Kpp, lvec, P);
        eval_system(&S, P, gridC, Es + 4 * s);
        free_view(&S);
    }
    free_offsets(o);
}

/* Constrains::apply (constrains.h:386-394) for system s: DistConstr::apply
 * (:95-109) with Forces.h:161 spring, AngleConstr::apply (:123-144) with
 * evalAngleCosHalf (Forces.h:190-215), cells of the angle arms zero.  p, f:
 * the system's positions and forces [nvecs*3]; lv: its cell rows a, b, c. */
static void bond_constraints(int s, const double* p, double* f, const double* lv, int ndist, const int* di,
                             const double* dp, int nang, const int* ai, const double* ap) {
    for (int c = 0; c < ndist; c++) {
        const int* x = di + 3 * c;
        const double* q = dp + 8 * c;   /* lmin, lmax, kmin, kmax, flim, shift */
        if (x[0] >= 0 && x[0] != s) continue;
        const int i0 = x[1], i1 = x[2];
        double d[3];
        for (int k = 0; k < 3; k++) d[k] = p[3 * i1 + k] - p[3 * i0 + k] + (lv[k] * q[5] + lv[3 + k] * q[6] + lv[6 + k] * q[7]);
        const double l = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double fs = 0;
        if (l > q[1]) { fs = (l - q[1]) * q[3]; if (fs > q[4]) fs = q[4]; }
        else if (l < q[0]) { fs = (l - q[0]) * q[2]; if (fs < -q[4]) fs = -q[4]; }
        for (int k = 0; k < 3; k++) { const double g = d[k] * (fs / l); f[3 * i1 + k] -= g; f[3 * i0 + k] += g; }
    }
    for (int c = 0; c < nang; c++) {
        const int* x = ai + 4 * c;
        if (x[0] >= 0 && x[0] != s) continue;
        const int ic = x[1], ia = x[2], ib = x[3];
        double h1[3], h2[3], h[3];
        for (int k = 0; k < 3; k++) { h1[k] = p[3 * ic + k] - p[3 * ia + k]; h2[k] = p[3 * ic + k] - p[3 * ib + k]; }
        const double l1 = sqrt(h1[0] * h1[0] + h1[1] * h1[1] + h1[2] * h1[2]);
        const double l2 = sqrt(h2[0] * h2[0] + h2[1] * h2[1] + h2[2] * h2[2]);
        const double ir1 = 1. / l1, ir2 = 1. / l2;
        for (int k = 0; k < 3; k++) { h1[k] *= ir1; h2[k] *= ir2; h[k] = h1[k] + h2[k]; }
        double c2 = (h[0] * h[0] + h[1] * h[1] + h[2] * h[2]) * 0.25;
        const double s2 = 1 - c2 + 1e-14, cc = sqrt(c2), ss = sqrt(s2);
        const double c0 = cos(ap[2 * c] * 0.5), s0 = sin(ap[2 * c] * 0.5), kk = ap[2 * c + 1];
        const double csy = s0 * cc - c0 * ss;
        double fr = -kk * csy;
        c2 *= -2;
        fr /= 4 * cc * ss;
        const double fr1 = fr * ir1, fr2 = fr * ir2;
        for (int k = 0; k < 3; k++) {
            const double f1 = h[k] * fr1 + h1[k] * (fr1 * c2), f2 = h[k] * fr2 + h2[k] * (fr2 * c2);
            f[3 * ia + k] -= f1; f[3 * ic + k] += f1 + f2; f[3 * ib + k] -= f2;
        }
    }
}

/* DynamicOpt.cpp:250-267 FIRE_update_params, then MMFFsp3_loc.h:1264-1281
 * move_atom_FIRE for every vector, as called from MolWorld_sp3::run_no_omp
 * (MolWorld_sp3.h:2401-2430): move_atom_FIRE(i, (float)opt.dt, 1e4, opt.cv,
 * opt.renorm_vf*opt.cf). */
void orc_relax(int nsys, const int* natoms, const int* nnode,
               double* pos, double* vel, double* fire_state,
               const int* neighs, const int* neighCell, const int* bkneighs,
               const double* REQs, const double* apars, const double* bLs,
               const double* bKs, const double* Ksp, const double* Kpp,
               const double* lvec, const double* gridC, const ORC_params* P,
               const ORC_fire* F, int niter, double Fconv, int conv_mode,
               int* nsteps_out, int* conv_out, double* Fout, double* Eout, int nthreads,
               const double* constr, const double* constrK,
               int ndist, const int* dist_idx, const double* dist_par,
               int nang, const int* ang_idx, const double* ang_par) {
    offsets_t o = make_offsets(nsys, natoms, nnode);
    size_t nvtot = (size_t)o.voff[nsys];
    double* force = (double*)calloc(nvtot * 3 + 3, sizeof(double));
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int s = 0; s < nsys; s++) {
        sysview S;
        setup_view(&S, s, &o, natoms, nnode, pos, force, neighs, neighCell, bkneighs, REQs,
                   apars, bLs, bKs, Ksp, Kpp, lvec, P);
        double* p = pos + 3 * o.voff[s];
        double* v = vel + 3 * o.voff[s];
        double* fst = fire_state + 4 * s;
        double dt = fst[0], damping = fst[1];
        int lastNeg = (int)fst[2];
        const double F2conv = Fconv * Fconv;
        int itr;
        int conv = 0;
        double meas = 0;
        double Ep[4] = {0, 0, 0, 0};
        const int nv = S.nvecs;
        for (itr = 0; itr < niter; itr++) {
            eval_system(&S, P, gridC, Ep);
            if (ndist || nang) bond_constraints(s, p, S.force, lvec + 9 * s, ndist, dist_idx, dist_par, nang, ang_idx, ang_par);
            if (F->Flim > 0) {
                const double Fl2 = F->Flim * F->Flim;
                for (int i = 0; i < nv; i++) {
                    double* fi = S.force + 3 * i;
                    double fr2 = fi[0] * fi[0] + fi[1] * fi[1] + fi[2] * fi[2];
                    if (fr2 > Fl2) { double c = F->Flim / sqrt(fr2); fi[0] *= c; fi[1] *= c; fi[2] *= c; }
                }
            }
            /* position springs of updateAtomsMMFFf4 (relax_multi.cl:995-1010):
             * after the clamp, atoms only, (anchor - p) * max(K, 0) where anchor.w > 0 */
            if (constr) {
                const double* cs = constr + 4 * o.aoff[s];
                const double* ck = constrK + 4 * o.aoff[s];
                for (int i = 0; i < S.natoms; i++) {
                    if (!(cs[4 * i + 3] > 0)) continue;
                    double* fi = S.force + 3 * i;
                    for (int k = 0; k < 3; k++) {
                        const double kk = ck[4 * i + k] > 0 ? ck[4 * i + k] : 0.0;
                        fi[k] += (cs[4 * i + k] - p[3 * i + k]) * kk;
                    }
                }
            }
            double vf = 0, vv = 0, ff = 0, fmax2 = 0;
            for (int i = 0; i < nv; i++) {
                for (int k = 0; k < 3; k++) {
                    double vi = v[3 * i + k], fi = S.force[3 * i + k];
                    vf += vi * fi; vv += vi * vi; ff += fi * fi;
                }
                double f2 = S.force[3 * i] * S.force[3 * i] + S.force[3 * i + 1] * S.force[3 * i + 1] +
                            S.force[3 * i + 2] * S.force[3 * i + 2];
                if (f2 > fmax2 || f2 != f2) fmax2 = f2;
            }
            /* FIRE_update_params */
            double f_len = sqrt(ff), v_len = sqrt(vv);
            double cos_vf = vf / (f_len * v_len + 1e-32);
            double renorm_vf = v_len / (f_len + 1e-32);
            double cv, cf;
            if (cos_vf < 0.0) { cv = F->cv_kill; cf = 0.; } else { cv = 1 - damping; cf = damping; }
            cf = renorm_vf * cf;
            if (cos_vf < 0.0) {
                dt = fmax(dt * F->fdec, F->dt_min);
                lastNeg = 0;
                damping = F->damp_max;
            } else {
                if (lastNeg > F->minLastNeg) {
                    dt = fmin(dt * F->finc, F->dt_max);
                    damping = damping * F->falpha;
                }
                lastNeg++;
            }
            /* move_atom_FIRE(i, (float)dt, Flim, cv, renorm_vf*cf) */
            const double dtf = (double)(float)dt;
            const double cfm = (F->variant == 1) ? cf : renorm_vf * cf;
            for (int i = 0; i < nv; i++) {
                v3 f = ld3(S.force + 3 * i), vi = ld3(v + 3 * i), pi = ld3(p + 3 * i);
                const int bPi = i >= S.natoms;
                if (bPi) f = vaddmul(f, pi, -vdot(pi, f));
                vi = vmul(vi, cv);
                vi = vaddmul(vi, f, dtf + cfm);
                if (bPi) vi = vaddmul(vi, pi, -vdot(pi, vi));
                pi = vaddmul(pi, vi, dtf);
                if (bPi) {
                    double l = sqrt(pi.x * pi.x + pi.y * pi.y + pi.z * pi.z);
                    pi = vmul(pi, 1.0 / l);
                }
                st3(p + 3 * i, pi); st3(v + 3 * i, vi);
            }
            meas = (conv_mode == 0) ? ff : fmax2;
            double thr = F2conv;
            if (meas < thr) { conv = 1; break; }
            if (meas != meas) { conv = -1; break; }   /* NaN: the system blew up */
        }
        fst[0] = dt; fst[1] = damping; fst[2] = (double)lastNeg;
        nsteps_out[s] = itr;
        conv_out[s] = conv;
        Fout[s] = sqrt(meas);
        if (Eout) { for (int k = 0; k < 4; k++) Eout[4 * s + k] = Ep[k]; }
        free_view(&S);
    }
    free(force);
    free_offsets(o);
}

/* ---------------- direct substrate term (relax_multi.cl:2741-2877, :166-181) ---------------- */

void orc_surf(int n, const double* pos, const double* REQ, int nsub, const double* spos,
              const double* sREQ, const double* lvec, const int* nPBC, double alphaMorse,
              double Rdamp, double* fe) {
    const double kC = 14.3996448915, K = -alphaMorse, R2d = Rdamp * Rdamp;
    for (int i = 0; i < n; i++) {
        double F[3] = {0, 0, 0}, E = 0;
        for (int j = 0; j < nsub; j++) {
            const double R0 = REQ[4 * i] + sREQ[4 * j];
            const double E0 = REQ[4 * i + 1] * sREQ[4 * j + 1];
            const double Q = REQ[4 * i + 2] * sREQ[4 * j + 2];
            for (int iz = -nPBC[2]; iz <= nPBC[2]; iz++)
                for (int iy = -nPBC[1]; iy <= nPBC[1]; iy++)
                    for (int ix = -nPBC[0]; ix <= nPBC[0]; ix++) {
                        double d[3];
                        for (int k = 0; k < 3; k++)
                            d[k] = pos[3 * i + k] - (spos[3 * j + k] + lvec[k] * ix + lvec[3 + k] * iy + lvec[6 + k] * iz);
                        const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        const double r = sqrt(r2);
                        const double ir2d = 1.0 / (r2 + R2d);
                        const double e = exp(K * (r - R0));
                        const double Ae = E0 * e;
                        const double fM = Ae * 2 * K * (e - 1);
                        const double Eel = kC * Q * sqrt(ir2d);
                        const double fr = fM / r - Eel * ir2d;
                        for (int k = 0; k < 3; k++) F[k] -= d[k] * fr;
                        E += Ae * (e - 2) + Eel;
                    }
        }
        for (int k = 0; k < 3; k++) fe[4 * i + k] = F[k];
        fe[4 * i + 3] = E;
    }
}

/* ---------------- Langevin dynamics (MMFFsp3_loc.h:1191-1216) ---------------- */

static unsigned long long orc_mix64(unsigned long long z) {   /* SplitMix64 finaliser */
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double orc_langevin_rand(unsigned long long seed, long long vec, int step, int comp) {
    const unsigned long long key = seed ^ orc_mix64(((unsigned long long)(unsigned)step << 32) ^
                                                    ((unsigned long long)vec << 2) ^ (unsigned long long)comp);
    return (double)(orc_mix64(key) >> 40) * (2.0 / 16777216.0) - 1.0;
}

void orc_md(int nsys, const int* natoms, const int* nnode, double* pos, double* vel,
            const int* neighs, const int* neighCell, const int* bkneighs,
            const double* REQs, const double* apars, const double* bLs,
            const double* bKs, const double* Ksp, const double* Kpp,
            const double* lvec, const double* gridC, const ORC_params* P,
            int nsteps, double dt, double gamma, double T, unsigned long long seed, int step0,
            double Flim, int nthreads) {
    offsets_t o = make_offsets(nsys, natoms, nnode);
    size_t nvtot = (size_t)o.voff[nsys];
    double* force = (double*)calloc(nvtot * 3 + 3, sizeof(double));
    const double kB = 8.617333262e-5;
    const double noise = sqrt(2.0 * kB * T * gamma / dt);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int s = 0; s < nsys; s++) {
        sysview S;
        setup_view(&S, s, &o, natoms, nnode, pos, force, neighs, neighCell, bkneighs, REQs,
                   apars, bLs, bKs, Ksp, Kpp, lvec, P);
        double* p = pos + 3 * o.voff[s];
        double* v = vel + 3 * o.voff[s];
        double Ep[4] = {0, 0, 0, 0};
        const int nv = S.nvecs;
        for (int it = 0; it < nsteps; it++) {
            eval_system(&S, P, gridC, Ep);
            for (int i = 0; i < nv; i++) {
                double* fi = S.force + 3 * i;
                if (Flim > 0) {
                    double fr2 = fi[0] * fi[0] + fi[1] * fi[1] + fi[2] * fi[2];
                    if (fr2 > Flim * Flim) { double c = Flim / sqrt(fr2); fi[0] *= c; fi[1] *= c; fi[2] *= c; }
                }
                v3 f = ld3(fi), vi = ld3(v + 3 * i), pi = ld3(p + 3 * i);
                const int bPi = i >= S.natoms;
                if (bPi) f = vaddmul(f, pi, -vdot(pi, f));
                f = vaddmul(f, vi, -gamma);
                const long long gv = (long long)o.voff[s] + i;
                v3 r = {orc_langevin_rand(seed, gv, step0 + it, 0), orc_langevin_rand(seed, gv, step0 + it, 1),
                        orc_langevin_rand(seed, gv, step0 + it, 2)};
                f = vaddmul(f, r, noise);
                vi = vaddmul(vi, f, dt);
                if (bPi) vi = vaddmul(vi, pi, -vdot(pi, vi));
                pi = vaddmul(pi, vi, dt);
                if (bPi) {
                    double l = sqrt(pi.x * pi.x + pi.y * pi.y + pi.z * pi.z);
                    pi = vmul(pi, 1.0 / l);
                }
                st3(p + 3 * i, pi); st3(v + 3 * i, vi);
            }
        }
        free_view(&S);
    }
    free(force);
    free_offsets(o);
}

/* ---------------- exploring cycle (GOpt) ---------------- */

/* GOpt (GOpt.h:25-60) driven per step as MolWorld_sp3::run_no_omp does with
 * bGopt (MolWorld_sp3.h:2290-2296 update at the top of the step, :2397-2424
 * FIRE scalars and the Langevin / FIRE move, :2465-2473 a minimum starts
 * exploring) plus the give-up branch of MolWorld_sp3_multi::updateMultiExploring
 * (MolWorld_sp3_multi.h:797-803: a relax phase longer than nRelax steps starts
 * exploring).  Per step: give-up check; step count + 1 and the end of an
 * exploring phase at n_explore; forces (clamped by F->Flim); FIRE_update_params
 * always; exploring: the Langevin move of orc_md (md_dt, gamma, T, stream
 * (seed, vector, step0 + step)), else move_atom_FIRE; a relaxing system below
 * Fconv has found a minimum: minpos <- positions, count + 1, exploring starts.
 * gopt[s*4] = (exploring, steps in phase, minima found, phases given up), in
 * and out; fire_state as orc_relax. */
void orc_explore(int nsys, const int* natoms, const int* nnode,
                 double* pos, double* vel, double* fire_state, int* gopt, double* minpos,
                 const int* neighs, const int* neighCell, const int* bkneighs,
                 const double* REQs, const double* apars, const double* bLs,
                 const double* bKs, const double* Ksp, const double* Kpp,
                 const double* lvec, const double* gridC, const ORC_params* P,
                 const ORC_fire* F, int nsteps, double Fconv, int conv_mode,
                 int n_explore, int n_relax, double md_dt, double gamma, double T,
                 unsigned long long seed, int step0, int nthreads) {
    offsets_t o = make_offsets(nsys, natoms, nnode);
    size_t nvtot = (size_t)o.voff[nsys];
    double* force = (double*)calloc(nvtot * 3 + 3, sizeof(double));
    const double kB = 8.617333262e-5;
    const double noise = sqrt(2.0 * kB * T * gamma / md_dt);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int s = 0; s < nsys; s++) {
        sysview S;
        setup_view(&S, s, &o, natoms, nnode, pos, force, neighs, neighCell, bkneighs, REQs,
                   apars, bLs, bKs, Ksp, Kpp, lvec, P);
        double* p = pos + 3 * o.voff[s];
        double* v = vel + 3 * o.voff[s];
        double* fst = fire_state + 4 * s;
        int* g = gopt + 4 * s;
        double dt = fst[0], damping = fst[1];
        int lastNeg = (int)fst[2];
        double Ep[4] = {0, 0, 0, 0};
        const int nv = S.nvecs;
        for (int it = 0; it < nsteps; it++) {
            if (!g[0] && n_relax > 0 && g[1] > n_relax) { g[3]++; g[0] = 1; g[1] = 0; }
            g[1]++;
            if (g[0] && g[1] >= n_explore) { g[0] = 0; g[1] = 0; }
            const int expl = g[0];
            eval_system(&S, P, gridC, Ep);
            double vf = 0, vv = 0, ff = 0, fmax2 = 0;
            for (int i = 0; i < nv; i++) {
                double* fi = S.force + 3 * i;
                double f2 = fi[0] * fi[0] + fi[1] * fi[1] + fi[2] * fi[2];
                if (F->Flim > 0 && f2 > F->Flim * F->Flim) {
                    double c = F->Flim / sqrt(f2); fi[0] *= c; fi[1] *= c; fi[2] *= c;
                    f2 = fi[0] * fi[0] + fi[1] * fi[1] + fi[2] * fi[2];
                }
                for (int k = 0; k < 3; k++) { vf += v[3 * i + k] * fi[k]; vv += v[3 * i + k] * v[3 * i + k]; ff += fi[k] * fi[k]; }
                if (f2 > fmax2 || f2 != f2) fmax2 = f2;
            }
            double f_len = sqrt(ff), v_len = sqrt(vv);
            double cos_vf = vf / (f_len * v_len + 1e-32);
            double renorm_vf = v_len / (f_len + 1e-32);
            double cv, cf;
            if (cos_vf < 0.0) { cv = F->cv_kill; cf = 0.; } else { cv = 1 - damping; cf = damping; }
            cf = renorm_vf * cf;
            if (cos_vf < 0.0) {
                dt = fmax(dt * F->fdec, F->dt_min);
                lastNeg = 0;
                damping = F->damp_max;
            } else {
                if (lastNeg > F->minLastNeg) { dt = fmin(dt * F->finc, F->dt_max); damping = damping * F->falpha; }
                lastNeg++;
            }
            const double dtf = (double)(float)dt;
            const double cfm = (F->variant == 1) ? cf : renorm_vf * cf;
            for (int i = 0; i < nv; i++) {
                v3 f = ld3(S.force + 3 * i), vi = ld3(v + 3 * i), pi = ld3(p + 3 * i);
                const int bPi = i >= S.natoms;
                if (bPi) f = vaddmul(f, pi, -vdot(pi, f));
                if (expl) {
                    f = vaddmul(f, vi, -gamma);
                    const long long gv = (long long)o.voff[s] + i;
                    v3 r = {orc_langevin_rand(seed, gv, step0 + it, 0), orc_langevin_rand(seed, gv, step0 + it, 1),
                            orc_langevin_rand(seed, gv, step0 + it, 2)};
                    f = vaddmul(f, r, noise);
                    vi = vaddmul(vi, f, md_dt);
                    if (bPi) vi = vaddmul(vi, pi, -vdot(pi, vi));
                    pi = vaddmul(pi, vi, md_dt);
                } else {
                    vi = vmul(vi, cv);
                    vi = vaddmul(vi, f, dtf + cfm);
                    if (bPi) vi = vaddmul(vi, pi, -vdot(pi, vi));
                    pi = vaddmul(pi, vi, dtf);
                }
                if (bPi) {
                    double l = sqrt(pi.x * pi.x + pi.y * pi.y + pi.z * pi.z);
                    pi = vmul(pi, 1.0 / l);
                }
                st3(p + 3 * i, pi); st3(v + 3 * i, vi);
            }
            const double meas = (conv_mode == 0) ? ff : fmax2;
            if (!expl && meas < Fconv * Fconv) {
                memcpy(minpos + 3 * o.voff[s], p, sizeof(double) * 3 * (size_t)nv);
                g[2]++; g[0] = 1; g[1] = 0;
            }
        }
        fst[0] = dt; fst[1] = damping; fst[2] = (double)lastNeg;
        free_view(&S);
    }
    free(force);
    free_offsets(o);
}

/* ---------------- grid construction (GridFF.h:582-635, 847-891) ---------------- */

void orc_grid_potentials(int nsub, const double* spos, const double* sREQ,
                         const double* lvec, const int* nPBC_mors, const int* nPBC_coul,
                         const ORC_params* P, double* V, int nthreads) {
    const int nx = P->gn[0], ny = P->gn[1], nz = P->gn[2];
    const int nm = (2 * nPBC_mors[0] + 1) * (2 * nPBC_mors[1] + 1) * (2 * nPBC_mors[2] + 1);
    const int nc = (2 * nPBC_coul[0] + 1) * (2 * nPBC_coul[1] + 1) * (2 * nPBC_coul[2] + 1);
    v3* sm = (v3*)malloc(sizeof(v3) * nm);
    v3* sc = (v3*)malloc(sizeof(v3) * nc);
    for (int k = 0; k < nm; k++) sm[k] = pbc_shift(lvec, nPBC_mors, k);
    for (int k = 0; k < nc; k++) sc[k] = pbc_shift(lvec, nPBC_coul, k);
    const double K = -P->alphaMorse;
    const long ntot = (long)nx * ny * nz;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (long i = 0; i < ntot; i++) {
        int iz = (int)(i % nz);
        int iy = (int)((i / nz) % ny);
        int ix = (int)(i / ((long)nz * ny));
        v3 pos = v3make(P->gpos0[0] + P->gstep[0] * ix, P->gpos0[1] + P->gstep[1] * iy,
                        P->gpos0[2] + P->gstep[2] * iz);
        double vp = 0, vl = 0, vc = 0;
        for (int ia = 0; ia < nsub; ia++) {
            v3 dp0 = vsub(pos, ld3(spos + 3 * ia));
            const double* R = sREQ + 4 * ia;
            for (int k = 0; k < nm; k++) {
                v3 dp = vadd(dp0, sm[k]);
                double r2 = vdot(dp, dp);
                double r = sqrt(r2 + 1e-32);
                double e = exp(K * (r - R[0]));
                double eM = e * R[1];
                vp += eM * e;
                vl += eM * -2.;
            }
            for (int k = 0; k < nc; k++) {
                v3 dp = vadd(dp0, sc[k]);
                double r2 = vdot(dp, dp);
                double ir2 = 1 / (r2 + 1e-32);
                vc += COULOMB_CONST * R[2] * sqrt(ir2);
            }
        }
        V[3 * i] = vp; V[3 * i + 1] = vl; V[3 * i + 2] = vc;
    }
    free(sm); free(sc);
}

/* 1-D solves of (c[i-1] + 4 c[i] + c[i+1]) / 6 = v[i] */
static void solve_periodic(int n, double* x, double* work) {
    /* circulant tridiagonal, Sherman-Morrison on the Thomas algorithm */
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    double* cp = work;            /* n */
    double* u = work + n;         /* n */
    double* z = work + 2 * n;     /* n */
    double gamma = -b;
    double bb0 = b - gamma;
    double bbn = b - a * a / gamma;
    /* solve T y = x and T z = u, T = tridiag with modified ends */
    for (int i = 0; i < n; i++) u[i] = 0;
    u[0] = gamma; u[n - 1] = a;
    double* rhs[2] = {x, u};
    double* out[2] = {x, z};
    for (int r = 0; r < 2; r++) {
        double* d = rhs[r];
        double* y = out[r];
        if (r == 1) for (int i = 0; i < n; i++) y[i] = d[i];
        double diag0 = bb0;
        cp[0] = a / diag0;
        y[0] = y[0] / diag0;
        for (int i = 1; i < n; i++) {
            double diag = (i == n - 1 ? bbn : b) - a * cp[i - 1];
            cp[i] = a / diag;
            y[i] = (y[i] - a * y[i - 1]) / diag;
        }
        for (int i = n - 2; i >= 0; i--) y[i] -= cp[i] * y[i + 1];
    }
    double fact = (x[0] + a * x[n - 1] / gamma) / (1.0 + z[0] + a * z[n - 1] / gamma);
    for (int i = 0; i < n; i++) x[i] -= fact * z[i];
}
static void solve_open(int n, double* y, double* cp) {
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    cp[0] = a / b;
    y[0] = y[0] / b;
    for (int i = 1; i < n; i++) {
        double diag = b - a * cp[i - 1];
        cp[i] = a / diag;
        y[i] = (y[i] - a * y[i - 1]) / diag;
    }
    for (int i = n - 2; i >= 0; i--) y[i] -= cp[i] * y[i + 1];
}

void orc_bspline_fit(const int* gn, const double* V, double* C) {
    const int nx = gn[0], ny = gn[1], nz = gn[2];
    const long ntot = (long)nx * ny * nz;
    memcpy(C, V, sizeof(double) * 3 * ntot);
    int nmax = nx > ny ? nx : ny; if (nz > nmax) nmax = nz;
    double* line = (double*)malloc(sizeof(double) * nmax);
    double* work = (double*)malloc(sizeof(double) * 3 * nmax);
    for (int ch = 0; ch < 3; ch++) {
        /* z (open) */
        for (int ix = 0; ix < nx; ix++) for (int iy = 0; iy < ny; iy++) {
            long b = ((long)ix * ny + iy) * nz;
            for (int k = 0; k < nz; k++) line[k] = C[3 * (b + k) + ch];
            solve_open(nz, line, work);
            for (int k = 0; k < nz; k++) C[3 * (b + k) + ch] = line[k];
        }
        /* y (periodic) */
        for (int ix = 0; ix < nx; ix++) for (int iz = 0; iz < nz; iz++) {
            for (int k = 0; k < ny; k++) line[k] = C[3 * (((long)ix * ny + k) * nz + iz) + ch];
            solve_periodic(ny, line, work);
            for (int k = 0; k < ny; k++) C[3 * (((long)ix * ny + k) * nz + iz) + ch] = line[k];
        }
        /* x (periodic) */
        for (int iy = 0; iy < ny; iy++) for (int iz = 0; iz < nz; iz++) {
            for (int k = 0; k < nx; k++) line[k] = C[3 * (((long)k * ny + iy) * nz + iz) + ch];
            solve_periodic(nx, line, work);
            for (int k = 0; k < nx; k++) C[3 * (((long)k * ny + iy) * nz + iz) + ch] = line[k];
        }
    }
    free(line); free(work);
}
