/*
 * MMFFmulti_lib.h -- C-ABI of the B200 multi-system MMFF relaxer
 * (libMMFFmulti_lib.so, built in-tree by firecore_b200/build.py).
 *
 * Two layers:
 *  1. The CSR world API (mmff_*): uneven systems packed back to back, the
 *     additive extension the reference's fixed-replica ABI lacks.  Plain
 *     pointers and sizes; host arrays are FP64 / int32 in the reference's
 *     MMFFsp3_loc layout (cpp/common/molecular/MMFFsp3_loc.h:43-139).
 *  2. The legacy symbols pyBall/MMFF_multi.py binds (init, run, eval, ...;
 *     pyBall/MMFF_multi.py:99-599, cpp/libs_OCL/MMFFmulti_lib.cpp), declared at
 *     the end, implemented on top of layer 1.
 *
 * Error behaviour: every int-returning call returns 0 (or a count) on success
 * and a negative value on failure, with a message in mmff_last_error(); the
 * library never exits the process (the reference prints and exit(0)s,
 * OCL.h OCL_checkError).  Nothing here falls back to the CPU: without a CUDA
 * device every compute call fails.
 */
#ifndef MMFFMULTI_LIB_H
#define MMFFMULTI_LIB_H
#include <stdint.h>
#include <stdbool.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ errors/setup */
const char* mmff_last_error(void);
/* No counterpart in the reference.  Kernels this library has launched so far
 * on the relaxation, evaluation and learned-proposal paths (a replay of the
 * captured relax graph counts each kernel it runs); callers difference two
 * readings to count the launches of a region. */
unsigned long long mmff_kernel_launches(void);
/* Select the CUDA device and create the library stream.
 * Replaces OCLsystem::init (cpp/common/OpenCL/OCL.h:386-410). */
int mmff_init_device(int device);
/* Wait for all queued work; reports asynchronous kernel errors. */
int mmff_sync(void);

/* ------------------------------------------------------------ switches */
/* flags: bit set of BONDS 1, PIPI 2, PISIGMA 4, ANGLES 8, SUB_ANGLE_NB 16,
 * SUB_BOND_NB 32, CLAMP_NB 64, NONBONDED 128, GRID 256, PBC 512 -- the
 * MMFFsp3_loc do* switches and ForceField::setNonBondStrategy flags
 * (cpp/common/molecular/ForceField.h:147-186).  nPBC: image counts
 * (MolWorld_sp3::makePBCshifts, MolWorld_sp3.h:775).  Rcut <= 0: all pairs x
 * all images (NBFF::evalLJQs_ng4_PBC_atom_omp, NBFF.h:575); Rcut > 0: pairs
 * beyond Rcut dropped and Coulomb in shifted-force form.  Set before
 * mmff_systems_upload (neighCell indices are validated against nPBC). */
int mmff_set_params(int flags, const int* nPBC, double Rcut, double alphaMorse, double FmaxNonBonded);
/* FIRE parameters (DynamicOpt members, cpp/common/math/DynamicOpt.h:73-95;
 * set_opt, cpp/libs_OCL/MMFFmulti_lib.cpp:141).  Flim > 0 clamps each
 * assembled force vector to |f| <= Flim (relax_multi.cl:980-983).
 * variant 0: the velocity kick of MolWorld_sp3::run_no_omp, f*(dt + renorm*cf)
 * with cf = renorm*damping (MolWorld_sp3.h:2426); variant 1: the mixing of
 * Bitzek et al. (2006), f*(dt + cf). */
int mmff_set_fire(double dt_max, double dt_min, double damp_max, double finc, double fdec, double falpha,
                  int minLastNeg, double cv_kill, double Flim, int variant);
/* Threads per CTA (64/128/256/512) and lanes per atom in the pair sum
 * (1/2/4/8) of the CTA-per-system kernels; 0 = chosen per size bucket
 * (systems of <= 64 atoms then run one per warp).  A non-zero thread count
 * forces every system onto the CTA-per-system kernels. */
int mmff_set_launch(int threads, int pair_split);

/* ------------------------------------------------------------ substrate grid */
/* Upload FP64 B-spline coefficients [nx][ny][nz][3] (z fastest; Pauli,
 * London, Coulomb), stored on the device as float4.  Replaces the
 * BsplinePLQ buffer upload of MolWorld_sp3_multi::initGridFF
 * (cpp/common/molecular/MolWorld_sp3_multi.h:2576-2581). */
int mmff_grid_upload(int nx, int ny, int nz, const double* pos0, const double* step, const double* coefs);
/* Build the grid on the GPU in FP64: node potentials of the substrate
 * (GridFF::evalBsplineRef with bUseEwald=false, GridFF.h:847-891) and the
 * exact B-spline fit (the limit of Bspline::fit3D_omp, Bspline_fit_3D.h:411).
 * spos [nsub*3], sREQ [nsub*4], lvec [9]; coefs_out (nullable) receives the
 * FP64 coefficients [nx][ny][nz][3]. */
int mmff_grid_build(int nsub, const double* spos, const double* sREQ, const double* lvec, const int* nPBC_mors,
                    const int* nPBC_coul, double alphaMorse, int nx, int ny, int nz, const double* pos0,
                    const double* step, double* coefs_out);
/* No counterpart in the reference.  In-place B-spline fit of a device array
 * the caller owns, for callers that may not allocate device memory (their
 * memory comes from a fixed arena they manage, so a cudaMalloc inside the
 * library would break their budget): d_coefs [nx][ny][nz][3] FP64 holds the
 * node values on entry and the coefficients on exit; nothing is allocated.
 * Limit: at most 4096 points per axis (larger grids return an error).  The
 * solver coefficients live in one static device array per GPU that the
 * library keeps until exit; every call rewrites them before use, and calls
 * whose kernels overlap on the GPU (different streams) race on it.  Every
 * call looks up that array's device address (cudaGetSymbolAddress) on the
 * current device, so a reset or recreated context is picked up; the first
 * call on a device also loads the library's kernels there, so make it before
 * any stream capture.  d_coefs must be device (or managed) memory of the
 * current device; anything else returns an error before any launch.
 * Kernels run on `stream` (a cudaStream_t; NULL = legacy default stream);
 * the call does not synchronise. */
int mmff_bspline_fit_noalloc(double* d_coefs, int nx, int ny, int nz, void* stream);
/* B-spline sample (GridFF::getForce_Bspline, GridFF.h:355) at n points:
 * pos [n*3], PLQ [n*4] -> fe [n*4] = (Fx, Fy, Fz, E). */
int mmff_grid_sample(int n, const double* pos, const double* PLQ, double* fe);

/* ------------------------------------------------------------ systems (CSR) */
/* Upload nsys systems (replaces MolWorld_sp3_multi::pack_system + upload,
 * MolWorld_sp3_multi.h:514-703, for uneven sizes).  Per system natoms[s] atoms
 * (nnode[s] nodes first) and nvecs = natoms + nnode vectors.
 * pos/vel [sum nvecs][3] (vel nullable = 0); neighs/neighCell/bkneighs
 * [sum natoms][4] local indices; REQs [sum natoms][4]; apars/bLs/bKs/Ksp/Kpp
 * [sum nnode][4]; lvec [nsys][9].  Indices are validated. */
int mmff_systems_upload(int nsys, const int* natoms, const int* nnode, const double* pos, const double* vel,
                        const int* neighs, const int* neighCell, const int* bkneighs, const double* REQs,
                        const double* apars, const double* bLs, const double* bKs, const double* Ksp,
                        const double* Kpp, const double* lvec);
/* Per-atom position springs for relaxations (the constr / constrK buffers
 * of updateAtomsMMFFf4, relax_multi.cl:995-1010; MolWorld_sp3_multi.h:
 * 1270-1273 sets them for scan_relaxed): anchor [sum natoms][4] = (x, y, z)
 * world coordinates and w > 0 to switch the spring on, K [sum natoms][4] =
 * (kx, ky, kz, -); the relax kernels add (anchor - p) * max(K, 0) to the
 * atom's force after the force clamp.  mmff_eval reports forces without
 * them.  anchor NULL clears; mmff_systems_upload clears. */
int mmff_set_constraints(const double* anchor, const double* K);
/* Distance and angle constraints between atoms for relaxations (FireCore's
 * Constrains: DistConstr / AngleConstr, cpp/common/molecular/constrains.h:83-146;
 * added by addDistConstrain / addAngConstrain, libMMFF.h:41-47, applied by
 * MolWorld_sp3::run_no_omp after the force field, MolWorld_sp3.h:2391-2395).
 * dist_idx [ndist*3] = (system, or -1 for every system; i0; i1) local atom
 * indices; dist_par [ndist*8] = (lmin, lmax, kmin, kmax, flim, shift along the
 * cell vectors a, b, c): a flat-bottom spring on |p[i1] - p[i0] + shift| with
 * constant kmax above lmax and kmin below lmin, its force capped at flim
 * (Forces.h:161 spring).  ang_idx [nang*4] = (system or -1, centre, end 1,
 * end 2); ang_par [nang*2] = (ang0 [rad], k): E = k (1 - cos((a - ang0)/2))
 * (evalAngleCosHalf).  The forces join each atom's force before the force
 * clamp; mmff_eval reports forces without them.  ndist = nang = 0 clears;
 * mmff_systems_upload clears. */
int mmff_set_bond_constraints(int ndist, const int* dist_idx, const double* dist_par, int nang, const int* ang_idx,
                              const double* ang_par);
/* No counterpart in the reference.  Per-atom cache of the 64 channel-combined
 * B-spline coefficients (PLQ . C) of the atom's GridFF stencil in the CTA
 * relax kernels: on (1, default) an atom re-gathers the grid only when its
 * stencil cell changes; off (0) every step gathers.  Results are
 * bit-identical either way; 260 B of device memory per atom. */
int mmff_set_grid_cache(int on);
/* No counterpart in the reference.  Shifted-image pair lists in the CTA relax
 * kernels (cutoff and a 2-D cell): the pairs (atom, image of atom) closer than
 * Rcut + skin are collected once and evaluated every step until an atom has
 * moved skin/2 since; then they are rebuilt (Verlet lists).  The pairs inside
 * the cutoff are those of the per-step candidate tiles, so results differ
 * only in summation order.  on (1, default) or off (0); skin > 0 sets the
 * skin [A] (default 1, at most 5), skin <= 0 keeps it. */
int mmff_set_pair_lists(int on, double skin);
/* Restore positions, velocities and FIRE state saved at upload (device copy). */
int mmff_systems_restore(void);
/* Overwrite positions (and velocities; NULL = 0); reset_fire != 0 resets dt,
 * damping and lastNeg. */
int mmff_systems_set_state(const double* pos, const double* vel, int reset_fire);

/* ------------------------------------------------------------ compute */
/* One force evaluation per system (forces assembled, unclamped) and, with
 * with_energy, FP64 energies (bonded, non-bonded, grid, total).  The force
 * phase of MolWorld_sp3::run_no_omp (MolWorld_sp3.h:2305-2386). */
int mmff_eval(int with_energy);
/* FIRE relaxation of every system for at most nstep_max steps, stopping a
 * system when sum f^2 < Fconv^2 (conv_mode 0, MolWorld_sp3.h:2460) or
 * max |f| < Fconv (conv_mode 1).  Replaces run_ocl_opt
 * (MolWorld_sp3_multi.h:1694-1846) with per-system FIRE in FP64 on the device
 * and no host round trip.  Asynchronous: mmff_sync / mmff_get_* wait. */
int mmff_relax(int nstep_max, double Fconv, int conv_mode);
/* on != 0: mmff_relax replays one captured CUDA graph (counter reset, fork
 * to the per-bucket streams, every bucket's persistent kernel, join) per
 * (parameters, nstep_max, Fconv, conv_mode); off (default): direct launches.
 * Replaces the reference's host loop of kernel enqueues and round trips
 * every 10 steps (MolWorld_sp3_multi.h:843-908). */
int mmff_set_graph(int on);
/* Langevin drive ("explore" dynamics; replaces MMFFsp3_loc::move_atom_Langevin,
 * MMFFsp3_loc.h:1191-1216, and the GPU drive of updateAtomsMMFFf4,
 * relax_multi.cl:1163-1178): every step f <- f - gamma v + u * sqrt(2 kB T
 * gamma / dt) with u uniform in [-1, 1) per component (counter-based stream
 * of (seed, vector, step)), v += f dt, p += v dt; pi vectors stay unit and
 * orthogonal.  mmff_set_md resets the step count of the random stream. */
int mmff_set_md(double dt, double gamma, double T, unsigned long long seed);
/* Direct substrate term (flag 1024 in mmff_set_params; replaces the kernel
 * getSurfMorse with getMorseQH, relax_multi.cl:2741-2877, :166-181): per atom,
 * Morse E0 e (e - 2), e = exp(-alphaMorse (r - R0)), plus Coulomb
 * k Q / sqrt(r^2 + Rdamp^2), over the substrate atoms and their images.
 * spos [nsub][3] world coordinates, sREQ [nsub][4] (R0, sqrt(E0), Q, H),
 * lvec [9], nPBC [3].  Its energy adds to the grid energy slot. */
int mmff_surf_upload(int nsub, const double* spos, const double* sREQ, const double* lvec, const int* nPBC,
                     double Rdamp);
int mmff_md(int nsteps);
/* Exploring cycle of the global optimiser (replaces GOpt, GOpt.h:25-60, as
 * MolWorld_sp3_multi::updateMultiExploring, MolWorld_sp3_multi.h:770-833, and
 * MolWorld_sp3::run_no_omp with bGopt, MolWorld_sp3.h:2290-2296,2397-2473,
 * drive it; the reference steps it on the host every 10 GPU steps, here it
 * runs per step inside the relax kernels).  Per system and step: a FIRE phase
 * longer than n_relax steps (n_relax <= 0: never) is given up and an exploring
 * phase starts; the step count of the phase advances and an exploring phase
 * ends once it reaches n_explore; forces; the FIRE scalars update; the atoms
 * move by the Langevin drive of mmff_set_md (exploring) or by FIRE; a relaxing
 * system whose convergence measure drops below Fconv has found a minimum: the
 * positions are kept, the count rises and an exploring phase starts.  No
 * system retires: mmff_explore runs nsteps steps for every system.
 * mmff_set_explore resets the state (start_exploring != 0: every system
 * starts in an exploring phase, as MolWorld_sp3_multi does after init with
 * bGopt); mmff_get_explore reads it back: gopt [nsys][4] = (exploring, steps
 * in the phase, minima found, phases given up), minpos (nullable)
 * [sum(natoms+nnode)][3] = the last minimum found, world coordinates (the
 * positions at mmff_set_explore where none was found).  The reference's
 * database of distinct minima and its group drives are not part of it. */
int mmff_set_explore(int n_explore, int n_relax, int start_exploring);
int mmff_explore(int nsteps, double Fconv, int conv_mode);
int mmff_get_explore(int* gopt, double* minpos);
/* Autotuner (no counterpart in the reference, which uses one fixed work-group
 * size): for each size class present (0: <= 32 atoms, 1: <= 64, 3: <= 128,
 * 4: <= 256, 5: larger), time every candidate launch configuration (warp per
 * system, or threads per CTA x lanes per atom in the pair sum) on up to
 * max_sample of its systems for nstep_probe FIRE steps and keep the fastest.
 * State is restored.  report [6 per candidate] (nullable): class, kind,
 * atoms per lane, threads, pair lanes, us per system-step (< 0: not
 * launchable).  Returns the number of candidates tried. */
int mmff_autotune(int nstep_probe, int max_sample, float* report, int report_cap);
/* Tuned configuration of size class cls: out[4] = (kind: -1 heuristic, 0 CTA
 * per system, 1 warp per system; atoms per lane; threads; pair lanes). */
int mmff_get_tuning(int cls, int* out);
int mmff_set_tuning(int cls, int kind, int apl, int threads, int pair_split);

/* ------------------------------------------------------------ results */
int mmff_get_forces(double* force);                 /* [sum nvecs][3] */
int mmff_get_energies(double* E);                   /* [nsys][4] */
/* pos/vel [sum nvecs][3] absolute frame; fire [nsys][4] (dt, damping, lastNeg,
 * total steps); status [nsys] (1 converged, 2 step limit, -1 NaN);
 * nsteps [nsys] (run_no_omp's return value); fconv [nsys] (convergence
 * measure at exit).  Any pointer may be NULL. */
int mmff_get_state(double* pos, double* vel, double* fire, int* status, int* nsteps, double* fconv);

/* ------------------------------------------------------------ timing / info */
int mmff_timer_start(void);                          /* CUDA event on the library stream */
double mmff_timer_stop(void);                        /* ms since mmff_timer_start, <0 on error */
/* Counting mode (on != 0): the relax kernels also count pair-images inside
 * the cutoff, atom B-spline samples and force evaluations; counters reset. */
int mmff_set_counting(int on);
/* out[5] = (pair-images, atom grid samples, force evaluations, shifted-image
 * pair-list builds, listed pairs evaluated) since the reset */
int mmff_get_counters(unsigned long long* out);
/* Measured denominators: FP32 FFMA throughput [TFLOP/s] and L2-resident
 * float4 read bandwidth [GB/s] over an mbytes MiB buffer; < 0 on error. */
double mmff_peak_fp32(void);
double mmff_peak_l2(int mbytes);
int mmff_num_buckets(void);
/* info[7] = (threads, pair_split, nsys, maxNA, maxNN, smem bytes, CTAs);
 * pair_split < 0 marks a warp-per-system bucket with -pair_split atoms per lane */
int mmff_bucket_info(int b, int* info);

/* ------------------------------------------------------------ synthetic workloads */
/* Node count the generator produces for natoms atoms. */
int mmff_gen_nnode(int natoms);
/* Seeded molecules (C:N:O:H = 10:2:2:10 heavy-atom trees with H caps) in the
 * layout above; topo_mode 0 = replicas of one topology, 1 = one per system. */
int mmff_gen_systems(int nsys, const int* natoms, uint64_t seed, int topo_mode, double sigma, int rotate,
                     double zplace, const double* cell_xy, int hbond, double* pos, int* neighs, int* neighCell,
                     int* bkneighs, double* REQs, double* apars, double* bLs, double* bKs, double* Ksp, double* Kpp,
                     int* elements, int central_cell);
/* Rock-salt (001) slab; returns the number of ions. */
int mmff_gen_slab(double a, int ncell, int layers, double z_top, double q, const double* REQ_cation,
                  const double* REQ_anion, double* spos, double* sREQ);

/* ------------------------------------------------------------ FireCore topology builder (host only)
 * Replaces what MolWorld_sp3::init does before any force evaluation
 * (cpp/common/molecular/MolWorld_sp3.h:309-382): initParams (:1298) reads the
 * four tables with MMFFparams (MMFFparams.h:267-541), buildMolecule_xyz
 * (:1323) and makeFFs / makeMMFFs (:1359-1586) type the molecule with
 * MM::Builder (autoBonds, autoConfEPi, assignBondParams, assignTypes,
 * toMMFFsp3_loc: MMFFBuilder.h:2087, 1633, 867, 1444, 4153) and fill
 * MMFFsp3_loc.  Same outputs, bit for bit, on the same files.
 * Arrays are the caller's, sized for cap atoms: apos [2*cap*3] (natoms atoms,
 * then nnode pi orientations), REQs / neighs / neighCell [cap*4], atypes
 * [cap], apars / bLs / bKs / Ksp / Kpp [cap*4] (nnode rows), type_names
 * [cap*8] (NUL-padded); any may be NULL.  counts[4] = natoms, nnode,
 * natoms + nnode, 1 if the xyz carried an "lvs" cell (then neighCell holds the
 * image of each bonded neighbour for the nPBC images, else -1).  bEpairs as in
 * FireCore's init.  Returns natoms; -1 on bad files or a molecule FireCore's
 * builder rejects (message in mmff_last_error), -2 if cap is too small. */
int mmff_build_xyz(const char* fElementTypes, const char* fAtomTypes, const char* fBondTypes, const char* fAngleTypes,
                   const char* xyz, int bEpairs, const int* nPBC, int cap, int* counts, double* apos, double* REQs,
                   int* atypes, int* neighs, int* neighCell, double* apars, double* bLs, double* bKs, double* Ksp,
                   double* Kpp, char* type_names);


/* ============================================================================
 * Legacy symbols: the reference library's ABI as pyBall/MMFF_multi.py binds it
 * (argtypes at pyBall/MMFF_multi.py:99-599).  One global world of nSys
 * replicas of one molecule with host mirrors of the device buffers, served
 * by the CSR API above.  All compute runs on the GPU.
 * ========================================================================== */

/* libUtils.h:16-47 -- name -> host buffer registry */
void   printBuffNames(void);
double* getBuff(const char* name);     /* apos fapos DOFs fDOFs vDOFs pipos fpipos Es */
float*  getfBuff(const char* name);    /* gpu_atoms gpu_aforces gpu_avel gpu_constr gpu_REQs gpu_MMpars
                                          gpu_BLs gpu_BKs gpu_Ksp gpu_Kpp gpu_lvecs gpu_ilvecs gpu_pbcshifts */
int*    getIBuff(const char* name);    /* ndims neighs selection gpu_neighs gpu_neighCell gpu_bkNeighs */

/* cpp/libs_OCL/MMFFmulti_lib.cpp */
void  init_buffers(void);                                                   /* :23 */
void* init(int nSys, char* xyz_name, char* surf_name, char* smile_name, bool bMMFF, bool bEpairs, int* nPBC,
           int* grid_nPBC, double gridStep, char* sElementTypes, char* sAtomTypes, char* sBondTypes,
           char* sAngleTypes, double T, double gamma, int nExplore, int nRelax, double pos_kick, double vel_kick,
           int GridFF);                                                     /* :75 */
/* init: as MolWorld_sp3::init does, the molecule is typed with FireCore's tables
 * from common_resources/{Element,Atom,Bond,Angle}Types.dat under the working
 * directory (the reference ignores the four file arguments, MMFFmulti_lib.cpp:85);
 * when those are absent the four names given are used, and when neither set
 * exists this library's own parameter table (a documented deviation).  Typing
 * with tables = mmff_build_xyz.  T, gamma, nExplore and nRelax set up the
 * exploring cycle of run(iParalel = 2); smile_name is not used, nor are
 * pos_kick and vel_kick (the reference's GOpt::apply_kick is never called). */
int   run(int nstepMax, double dt, double Fconv, int ialg, double* outE, double* outF, int iParalel);   /* :116 */
/* run: FIRE relaxation of every replica for up to nstepMax steps (every
 * iParalel); with init's nExplore > 0 and iParalel 0, 1 or 2, nstepMax steps
 * of the exploring cycle instead (mmff_explore; Langevin time step = the FIRE
 * dt_max, T and gamma from init, every replica starting in an exploring
 * phase), as run_omp_ocl and run_ocl_opt with GOpt do; only iParalel 2 gives
 * up a relax phase after nRelax steps (run_ocl_opt's rule).  dt and ialg are
 * ignored, as by the reference. */
void  MDloop(int perframe, double Ftol, int iParalel, int perVF);           /* :134 */
void  set_opt(double dt_max, double dt_min, double damp_max, double finc, double fdec, double falpha, int minLastNeg,
              double cvf_min, double cvf_max);                              /* :141 */
void  sampleSurf(char* name, int n, double* rs, double* Es, double* fs, int kind, int atyp, double Q, double K,
                 double RQ, double* pos0_, bool bSave);                     /* :168 */
void  sampleSurf_vecs(char* name, int n, double* poss_, double* Es, double* fs_, int kind, int atyp, double Q,
                      double K, double RQ, double* pos0_, bool bSave);      /* :210 */
void  pack_system(int isys, bool bParams, bool bForces, bool bVel, bool blvec);   /* :253 */
void  unpack_system(int isys, bool bForces, bool bVel);                     /* :256 */
void  upload_sys(int isys, bool bParams, bool bForces, bool bVel, bool blvec);    /* :260 */
void  download_sys(int isys, bool bForces, bool bVel);                      /* :263 */
void  upload(bool bParams, bool bForces, bool bVel, bool blvec);            /* :267 */
void  download(bool bForces, bool bVel);                                    /* :270 */
void  change_lvec(double* lvec, bool bAdd, bool bUpdatePi);                 /* :275 */
void  upload_pop(const char* fname);                                        /* :281 */
void  optimizeLattice_1d(double* dlvec, int n1, int n2, int initMode, double tol);         /* :289 */
void  optimizeLattice_2d_multi(double* dlvec, int nstesp, int initMode, double tol);       /* :294 */
void  scan(int nconf, double* poss, double* rots, double* Es, double* aforces, double* aposs, bool omp, bool bRelax,
           int niter_max, double dt, double Fconv, double Flim);            /* :305 */
void  setSwitches_multi(int CheckInvariants, int PBC, int NonBonded, int MMFF, int Angles, int PiSigma, int PiPiI,
                        int dovdW, int bSaveToDatabase);                    /* :316 */

/* cpp/common/molecular/libMMFF.h */
void  setVerbosity(int verbosity_, int idebug_);                            /* :15 */
void  insertSMILES(char* s);                                                /* :25 */
bool  checkInvariants(double maxVcog, double maxFcog, double maxTg);        /* :52 */
void  setOptLog(int n, double* cos, double* f, double* v, double* dt, double* damp);
bool  setTrjName(const char* trj_fname_, int savePerNsteps_);               /* :53 */
int   saveXYZ(const char* fname, const char* comment, int imod);            /* :55 */
const char* getTypeName(int ia, bool fromFF);                               /* :112 */
double eval(void);                                                          /* :98 */
void  addDistConstrain(int i0, int i1, double lmin, double lmax, double kmin, double kmax, double flim, double* shift,
                       bool bOldIndex);                                     /* :41 */
void  addAngConstrain(int i0, int i1, int i2, double ang0, double k);       /* :46 */
void  shift_atoms_ax(int n, int* selection, double* d);                     /* :122 */
void  shift_atoms(int n, int* selection, int ia0, int ia1, double l);       /* :124 */
void  rotate_atoms_ax(int n, int* selection, double* p0, double* ax, double phi);         /* :123 */
void  rotate_atoms(int n, int* selection, int ia0, int iax0, int iax1, double phi);       /* :125 */
void  scanTranslation_ax(int n, int* selection, double* vec, int nstep, double* Es, const char* trjName,
                         bool bAddjustCaps);                                /* :134 */
void  scanTranslation(int n, int* selection, int ia0, int ia1, double l, int nstep, double* Es, const char* trjName,
                      bool bAddjustCaps);                                   /* :138 */
void  scanRotation_ax(int n, int* selection, double* p0, double* ax, double phi, int nstep, double* Es,
                      const char* trjName);                                 /* :141 */
void  scanRotation(int n, int* selection, int ia0, int iax0, int iax1, double phi, int nstep, double* Es,
                   const char* trjName);                                    /* :147 */
void  sample_DistConstr(double lmin, double lmax, double kmin, double kmax, double flim, int n, double* xs, double* Es,
                        double* Fs);                                        /* :426 */
void  sample_evalPiAling(double k, double ang0, double r1, double r2, int n, double* angles, double* Es, double* Fs);   /* :439 */
void  sample_evalAngleCos(double k, double ang0, double r1, double r2, int n, double* angles, double* Es, double* Fs);  /* :451 */
void  sample_evalAngleCosHalf(double k, double ang0, double r1, double r2, int n, double* angles, double* Es,
                              double* Fs);                                  /* :464 */
void  sampleNonBond(int n, double* rs, double* Es, double* fs, int kind, double* REQi_, double* REQj_, double K,
                    double Rdamp);                                          /* :477 */

/* ------------------------------------------------------------ learned warm-start proposal
 * No counterpart in FireCore (its relaxers are plain FIRE,
 * MolWorld_sp3.h:2261-2490); the network is this library's addition: per-atom
 * descriptors (32 nearest neighbours within 5 A: 16 Gaussian radial bins,
 * sigma 0.3 A, x 4 element channels H C N O; height above the slab; GridFF
 * force) -> 68 -> 128 -> 128 -> 3 SiLU MLP predicting a displacement toward the
 * minimum.  BF16 weights and activations, FP32 accumulation on the tensor
 * cores (tcgen05).  Flat FP32 parameter vector: W1 [128][80] (inputs >= 68
 * zero), b1 [128], W2 [128][128], b2 [128], W3 [16][128] (rows >= 3 zero),
 * b3 [16] (see mmff_mlp_layout for the offsets).  Targets and outputs are in
 * A; the network works in units of out_scale. */
/* Parameters (flat vector), feature standardisation (mean, std > 0 per
 * feature) and output scale [A]; resets the AdamW moments and step count. */
int mmff_mlp_set_params(const float* prm, const float* feat_mean, const float* feat_std, double out_scale);
int mmff_mlp_get_params(float* prm);
/* Gradient sums of the mean squared displacement error over n rows of raw
 * features [n][68] and targets [n][3] (no update); loss = sum |y - t|^2 / n. */
int mmff_mlp_grad(int n, const float* feat, const float* target, float* grad_out, double* loss_out);
/* One AdamW step (beta 0.9/0.999, eps 1e-8, decoupled decay wd on W1..W3)
 * with the given flat FP32 gradients (NULL: the last computed ones). */
int mmff_mlp_adamw(const float* grad, double lr, double wd);
/* Network displacement [n][3] (A) for raw features [n][68]. */
int mmff_mlp_infer(int n, const float* feat, float* out);
/* Device-resident training set (rows in the order given) and nsteps AdamW
 * steps over consecutive batches of batch_tiles x 128 rows; per-step losses
 * to loss_out [nsteps] (nullable). */
int mmff_mlp_set_data(int n, const float* feat, const float* target);
int mmff_mlp_train(int nsteps, int batch_tiles, double lr, double wd, double* loss_out);
/* Element channel per atom of the uploaded systems [sum natoms] (0 H, 1 C,
 * 2 N, 3 O; larger values use channel 3). */
int mmff_mlp_set_elements(const int* elem);
/* Raw descriptors [sum natoms][68] of the current positions; z_top = slab top [A]. */
int mmff_mlp_features(double z_top, float* out);
/* No counterpart in the reference.  How warm-start moves use the network's
 * per-atom displacements: 0 as they are (default), 1 projected per system on
 * the least-squares rigid-body move (translation + rotation, FP64 fit), which
 * leaves every bonded term of the molecule unchanged. */
int mmff_mlp_set_projection(int mode);
/* No counterpart in the reference.  Exercises the bounded completion waits of
 * the tensor-core kernel: one launch that issues no product and no commit, so
 * its first wait can only run out (about half a millisecond); the CTA then
 * sets the error flag, frees its TMEM and returns.  1: the timeout came back
 * as the error status (flag cleared again); 0: it did not; < 0: error. */
int mmff_mlp_wait_test(void);
/* No counterpart in the reference.  That rigid-body projection of host
 * displacements disp [sum natoms][3] at the systems' current positions ->
 * out [sum natoms][3] (the warm start's kernel, for checks). */
int mmff_mlp_project(const double* disp, double* out);
/* nsteps learned moves on every system: descriptors -> network proposal d ->
 * trial positions x + a d for a = 1, 1/2, 1/4, 1/8 -> the first trial that
 * lowers the system's total energy is kept, else the system stays at x;
 * accepted [nsys] (nullable) counts the kept moves.  Velocities and FIRE
 * state are left as they are. */
int mmff_mlp_warmstart(int nsteps, double z_top, int* accepted);
/* Introspection for host-side checks: the tcgen05 product plan (14 ints per
 * product; returns the count), sizes/offsets, and the descriptor encoders. */
int mmff_mlp_plan(int* ops);
int mmff_mlp_layout(int* out);
unsigned long long mmff_mlp_smem_desc(unsigned addr, unsigned lbo, unsigned sbo);
unsigned mmff_mlp_instr_desc(int n, int a_mn, int b_mn);

#ifdef __cplusplus
}
#endif
#endif
