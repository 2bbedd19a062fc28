/*
 * mmff_oracle.h -- FP64 CPU restatement of FireCore's multi-system MMFF
 * relaxation hot path.  TEST INFRASTRUCTURE ONLY: this code is the checker
 * that the CUDA path is compared against.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm may load it; the product library
 * never links it and has no CPU fallback.
 *
 * Parity pin: the restatement is validated against the reference's own C++
 * physics (MMFFsp3_loc::eval_atom, NBFF::evalLJQs_ng4_PBC_atom_omp,
 * GridFF::getForce_Bspline, DynamicOpt::FIRE_update_params,
 * MMFFsp3_loc::move_atom_FIRE driven as in MolWorld_sp3::run_no_omp),
 * compiled from the reference sources by oracle/Makefile into oracle/_ref,
 * through the golden fixtures in tests/golden/.
 *
 * Layout (all arrays FP64 / int32, systems packed back to back, CSR):
 *   system s has natoms[s] atoms (nnode[s] node atoms first, then caps) and
 *   nvecs = natoms + nnode vectors (atoms, then one pi-orbital per node).
 *   pos/vel/force : [sum nvecs][3]
 *   neighs/neighCell/bkneighs : [sum natoms][4]  (indices local to the system,
 *       bkneighs values are ia*4+j into the node recoil slots, as produced by
 *       MMFFsp3_loc::makeBackNeighs, cpp/common/molecular/MMFFsp3_loc.h:1336)
 *   REQs  : [sum natoms][4]  (R0, sqrt(E0), Q, H)
 *   apars/bLs/bKs/Ksp/Kpp : [sum nnode][4]
 *   lvec  : [nsys][9] (rows a,b,c)
 *   grid coefficients : [nx][ny][nz][3] z-fastest, channels (Pauli, London, Coulomb)
 */
#ifndef MMFF_ORACLE_H
#define MMFF_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* flag bits for ORC_params.flags */
enum {
    ORC_BONDS        = 1 << 0,
    ORC_PIPI         = 1 << 1,
    ORC_PISIGMA      = 1 << 2,
    ORC_ANGLES       = 1 << 3,
    ORC_SUB_ANGLE_NB = 1 << 4,   /* bSubtractAngleNonBond */
    ORC_SUB_BOND_NB  = 1 << 5,   /* bSubtractBondNonBond  */
    ORC_CLAMP_NB     = 1 << 6,   /* bClampNonBonded       */
    ORC_NONBONDED    = 1 << 7,
    ORC_GRID         = 1 << 8,
    ORC_PBC          = 1 << 9,
};

/* Scalar parameters shared by every system of a call. */
typedef struct {
    int    flags;
    int    npbc[3];        /* nPBC image counts, images run -n..n        */
    double Rcut;           /* <=0: no cutoff (reference semantics); >0: pairs
                              beyond Rcut dropped, shifted-force Coulomb */
    double Ron;            /* unused (kept for layout)                  */
    double FmaxNonBonded;  /* clamp for bClampNonBonded                 */
    double alphaMorse;     /* REQ -> PLQ conversion exponent            */
    /* grid */
    int    gn[3];
    double gpos0[3];
    double gstep[3];       /* orthorhombic voxel edges                  */
} ORC_params;

/* FIRE parameters (DynamicOpt members used by FIRE_update_params) */
typedef struct {
    double dt_max, dt_min, damp_max, finc, fdec, falpha, cv_kill;
    int    minLastNeg;
    int    variant; /* 0: run_no_omp mixing, velocity gets f*(dt + renorm_vf*cf)
                       (MolWorld_sp3.h:2426, cf already = renorm_vf*damping);
                       1: Bitzek et al. 2006 mixing, f*(dt + cf) */
    double Flim;   /* >0: per-vector force clamp |f|<=Flim after assembly, as in
                      relax_multi.cl:980-983 (updateAtomsMMFFf4); <=0: none, as
                      run_no_omp (MolWorld_sp3.h:2426 passes Flim=1e4, unused) */
} ORC_fire;

/* Forces + energies for every system.
 * Es[s*4+k]: 0 bonded (eval_atom sum), 1 non-bonded (0.5*sum, as the
 * reference returns), 2 grid, 3 total. */
void orc_eval(int nsys, const int* natoms, const int* nnode,
              const double* pos, double* force, double* Es,
              const int* neighs, const int* neighCell, const int* bkneighs,
              const double* REQs, const double* apars, const double* bLs,
              const double* bKs, const double* Ksp, const double* Kpp,
              const double* lvec, const double* gridC, const ORC_params* P,
              int nthreads);

/* FIRE relaxation of every system, MolWorld_sp3::run_no_omp semantics.
 * Distance / angle constraints (optional, ndist / nang = 0: none):
 * dist_idx [ndist*3] = (system or -1 = all, i0, i1), dist_par [ndist*8] =
 * (lmin, lmax, kmin, kmax, flim, shift a, b, c); ang_idx [nang*4] = (system or
 * -1, centre, end 1, end 2), ang_par [nang*2] = (ang0 rad, k); applied after
 * the force field and before the clamp (MolWorld_sp3.h:2391-2395).
 * fire_state[s*4]: dt, damping, lastNeg (as double), unused.
 * conv_mode 0: sum_DOF f^2 < Fconv^2 (reference); 1: max_vec |f| < Fconv.
 * nsteps_out[s]: steps done (the reference's return value), conv_out[s]:
 * 1 if converged. Fout[s]: the convergence measure at exit. */
void orc_relax(int nsys, const int* natoms, const int* nnode,
               double* pos, double* vel, double* fire_state,
               const int* neighs, const int* neighCell, const int* bkneighs,
               const double* REQs, const double* apars, const double* bLs,
               const double* bKs, const double* Ksp, const double* Kpp,
               const double* lvec, const double* gridC, const ORC_params* P,
               const ORC_fire* F, int niter, double Fconv, int conv_mode,
               int* nsteps_out, int* conv_out, double* Fout, double* Eout,
               int nthreads, const double* constr, const double* constrK,
               int ndist, const int* dist_idx, const double* dist_par,
               int nang, const int* ang_idx, const double* ang_par);

/* Langevin dynamics, MMFFsp3_loc::move_atom_Langevin (MMFFsp3_loc.h:1191-1216):
 * per step and vector f -= gamma v; f += u sqrt(2 kB T gamma / dt) with u in
 * [-1,1) from orc_langevin_rand(seed, global vector index, step0 + step,
 * component) (the reference draws randf(-1,1)); v += f dt; p += v dt; pi
 * vectors: force and velocity projected, position renormalised.  Flim > 0
 * clamps each force vector first (as in orc_relax). */
void orc_md(int nsys, const int* natoms, const int* nnode, double* pos, double* vel,
            const int* neighs, const int* neighCell, const int* bkneighs,
            const double* REQs, const double* apars, const double* bLs,
            const double* bKs, const double* Ksp, const double* Kpp,
            const double* lvec, const double* gridC, const ORC_params* P,
            int nsteps, double dt, double gamma, double T, unsigned long long seed, int step0,
            double Flim, int nthreads);
/* Exploring cycle of GOpt on top of FIRE and the Langevin drive (see the
 * definition for the step order); gopt[s*4] = (exploring, steps in phase,
 * minima found, phases given up), minpos [nvecs*3] = last minimum found. */
void orc_explore(int nsys, const int* natoms, const int* nnode,
                 double* pos, double* vel, double* fire_state, int* gopt, double* minpos,
                 const int* neighs, const int* neighCell, const int* bkneighs,
                 const double* REQs, const double* apars, const double* bLs,
                 const double* bKs, const double* Ksp, const double* Kpp,
                 const double* lvec, const double* gridC, const ORC_params* P,
                 const ORC_fire* F, int nsteps, double Fconv, int conv_mode,
                 int n_explore, int n_relax, double md_dt, double gamma, double T,
                 unsigned long long seed, int step0, int nthreads);
/* the uniform random numbers of orc_md (SplitMix64 of seed, vector, step, component) */
double orc_langevin_rand(unsigned long long seed, long long vec, int step, int comp);

/* Direct substrate term, getSurfMorse / getMorseQH (relax_multi.cl:2741-2877,
 * :166-181), FP64: for n atoms at pos [n*3] with REQ [n*4] = (R0, sqrt E0,
 * Q, H), against nsub substrate atoms and their images
 * (-nPBC..nPBC along lvec rows): fe[i*4] = (F, E). */
void orc_surf(int n, const double* pos, const double* REQ, int nsub, const double* spos,
              const double* sREQ, const double* lvec, const int* nPBC, double alphaMorse,
              double Rdamp, double* fe);

/* B-spline GridFF sample of n points: fe[i*4] = (Fx,Fy,Fz,E) for PLQ[i*4]. */
void orc_grid_sample(int n, const double* pos, const double* PLQ,
                     const double* gridC, const ORC_params* P, double* fe);

/* REQ -> PLQ (Forces.h REQ2PLQ_d) */
void orc_req2plq(int n, const double* REQ, double K, double* PLQ);

/* Substrate potentials on grid nodes (GridFF::evalBsplineRef semantics with
 * bUseEwald=false): V[i*3+c], node order z-fastest. */
void orc_grid_potentials(int nsub, const double* spos, const double* sREQ,
                         const double* lvec, const int* nPBC_mors,
                         const int* nPBC_coul, const ORC_params* P,
                         double* V, int nthreads);

/* Exact cubic B-spline interpolation coefficients: periodic in x,y, zero
 * coefficients outside [0,nz) in z (the converged limit of
 * Bspline::fit3D_omp with bPBC=true).  V and C: [nx][ny][nz][3]. */
void orc_bspline_fit(const int* gn, const double* V, double* C);

#ifdef __cplusplus
}
#endif
#endif
