// ref_harness.cpp -- drives FireCore's own C++ physics (compiled from the
// reference sources by oracle/Makefile) so that the FP64 restatement in
// mmff_oracle.c can be pinned against it.  TEST INFRASTRUCTURE ONLY.
//
// The harness owns no physics.  It fills a MolWorld_sp3 instance the way
// MolWorld_sp3::makeFFs / initGridFF leave it (cpp/common/molecular/
// MolWorld_sp3.h:1442-1586, 968-1003) and then calls the reference:
//   * MolWorld_sp3::run_no_omp            (MolWorld_sp3.h:2261-2490)
//   * MMFFsp3_loc::eval_atom/assemble_atom (MMFFsp3_loc.h:250, 998)
//   * NBFF::evalLJQs_ng4_PBC_atom_omp      (NBFF.h:575)
//   * GridFF::addAtom / getForce_Bspline   (GridFF.h:355, 459)
//   * Bspline::fit3D_omp                   (Bspline_fit_3D.h:411)
//   * GridFF::evalGridFFPoint_Mors/_Coul   (GridFF.h:582, 614)
#include "globals.h"
#include "testUtils.h"
#include "MolWorld_sp3.h"
#include <cstdio>

static MolWorld_sp3 W;
static double* g_gridC = nullptr;   // Vec3d[nx*ny*nz], z-fastest
static int     g_flags = 0;

enum {
    F_BONDS = 1 << 0, F_PIPI = 1 << 1, F_PISIGMA = 1 << 2, F_ANGLES = 1 << 3,
    F_SUB_ANGLE_NB = 1 << 4, F_SUB_BOND_NB = 1 << 5, F_CLAMP_NB = 1 << 6,
    F_NONBONDED = 1 << 7, F_GRID = 1 << 8, F_PBC = 1 << 9,
};

extern "C" {

// One system. pos: [nvecs*3]; neighs/neighCell: [natoms*4] (cap entries are
// rebuilt by makeBackNeighs); returns bkneighs [natoms*4] and cap neighs.
int ref_setup(int natoms, int nnode, const double* pos,
              const int* neighs, const int* neighCell, const double* REQs,
              const double* apars, const double* bLs, const double* bKs,
              const double* Ksp, const double* Kpp, const double* lvec,
              const int* nPBC, int flags, double alphaMorse,
              const int* gn, const double* gpos0, const double* gstep,
              const double* gridC, int* bkneighs_out, int* neighs_out) {
    verbosity = 0;
    g_flags = flags;
    MMFFsp3_loc& ff = W.ffl;
    ff.realloc(nnode, natoms - nnode);
    for (int i = 0; i < ff.nvecs; i++) { ff.apos[i] = Vec3d{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]}; }
    for (int i = 0; i < natoms; i++) {
        ff.neighs[i]    = Quat4i{neighs[4 * i], neighs[4 * i + 1], neighs[4 * i + 2], neighs[4 * i + 3]};
        ff.neighCell[i] = Quat4i{neighCell[4 * i], neighCell[4 * i + 1], neighCell[4 * i + 2], neighCell[4 * i + 3]};
        ff.REQs[i]      = Quat4d{REQs[4 * i], REQs[4 * i + 1], REQs[4 * i + 2], REQs[4 * i + 3]};
        ff.atypes[i] = 0;
    }
    for (int i = 0; i < nnode; i++) {
        ff.apars[i] = Quat4d{apars[4 * i], apars[4 * i + 1], apars[4 * i + 2], apars[4 * i + 3]};
        ff.bLs[i]   = Quat4d{bLs[4 * i], bLs[4 * i + 1], bLs[4 * i + 2], bLs[4 * i + 3]};
        ff.bKs[i]   = Quat4d{bKs[4 * i], bKs[4 * i + 1], bKs[4 * i + 2], bKs[4 * i + 3]};
        ff.Ksp[i]   = Quat4d{Ksp[4 * i], Ksp[4 * i + 1], Ksp[4 * i + 2], Ksp[4 * i + 3]};
        ff.Kpp[i]   = Quat4d{Kpp[4 * i], Kpp[4 * i + 1], Kpp[4 * i + 2], Kpp[4 * i + 3]};
    }
    ff.makeBackNeighs(true);
    for (int i = 0; i < natoms; i++) {
        for (int k = 0; k < 4; k++) { bkneighs_out[4 * i + k] = ff.bkneighs[i].array[k]; neighs_out[4 * i + k] = ff.neighs[i].array[k]; }
    }
    Mat3d lv; lv.a = Vec3d{lvec[0], lvec[1], lvec[2]}; lv.b = Vec3d{lvec[3], lvec[4], lvec[5]}; lv.c = Vec3d{lvec[6], lvec[7], lvec[8]};
    ff.setLvec(lv);
    const bool bPBC = (flags & F_PBC) != 0;
    if (bPBC) {
        // MolWorld_sp3::makePBCshifts + bindShifts (MolWorld_sp3.h:775, 1413-1414)
        W.nPBC = Vec3i{nPBC[0], nPBC[1], nPBC[2]};
        W.makePBCshifts(W.nPBC, lv);
        ff.bindShifts(W.npbc, W.pbc_shifts);
        ff.bPBC = true;
    } else { ff.bPBC = false; }
    W.bPBC = bPBC;
    // the same flags MolWorld_sp3 keeps for the run_no_omp path
    ff.doBonds   = (flags & F_BONDS) != 0;
    ff.doPiPiI   = (flags & F_PIPI) != 0;
    ff.doPiSigma = (flags & F_PISIGMA) != 0;
    ff.doAngles  = (flags & F_ANGLES) != 0;
    W.bMMFF = true;
    W.bNonBonded = (flags & F_NONBONDED) != 0;
    W.bNonBondNeighs = true;
    W.bGopt = false; W.bGroups = false; W.bConstrains = false; W.bConstrZ = false;
    W.bHardConstrs = false; W.bCheckStuck = false; W.go.bExploring = false;
    // PLQd as makeFFs computes it (NBFF::evalPLQd -> REQ2PLQ_d)
    _realloc(ff.PLQd, natoms);
    for (int i = 0; i < natoms; i++) ff.PLQd[i] = REQ2PLQ_d(ff.REQs[i], alphaMorse);
    // GridFF in BsplineDouble mode over the caller's coefficients
    GridFF& g = W.gridFF;
    g.alphaMorse = alphaMorse;
    g.mode = GridFFmod::BsplineDouble;
    g.grid.n = Vec3i{gn[0], gn[1], gn[2]};
    g.grid.pos0 = Vec3d{gpos0[0], gpos0[1], gpos0[2]};
    g.grid.dCell = Mat3d{gstep[0], 0, 0, 0, gstep[1], 0, 0, 0, gstep[2]};
    g.grid.dCell.invert_T_to(g.grid.diCell);
    g.grid.cell = Mat3d{gstep[0] * gn[0], 0, 0, 0, gstep[1] * gn[1], 0, 0, 0, gstep[2] * gn[2]};
    make_inds_pbc(gn[0], g.cubic_xqis);
    make_inds_pbc(gn[1], g.cubic_yqis);
    size_t ng = (size_t)gn[0] * gn[1] * gn[2];
    delete[] g_gridC;
    g_gridC = new double[ng * 3];
    for (size_t i = 0; i < ng * 3; i++) g_gridC[i] = gridC[i];
    g.Bspline_PLQ = (Vec3d*)g_gridC;
    W.bGridFF = (flags & F_GRID) != 0;
    W.bSurfAtoms = W.bGridFF;
    // optimizer bound to the force field DOFs (MolWorld_sp3::setOptimizer)
    W.opt.bindOrAlloc(ff.nDOFs, ff.DOFs, 0, ff.fDOFs, 0);
    W.opt.initOpt(0.1);
    W.opt.cleanVel();
    ff.vapos = (Vec3d*)W.opt.vel;
    ff.setNonBondStrategy(+1);
    return ff.nvecs;
}

// One force evaluation with the force phase of run_no_omp (MolWorld_sp3.h:2305-2386).
void ref_eval(double* force, double* Es) {
    MMFFsp3_loc& ff = W.ffl;
    ff.bNonBonded = W.bNonBonded; ff.setNonBondStrategy(+1);
    double Eb = 0, Enb = 0, Eg = 0;
    for (int ia = 0; ia < ff.natoms; ia++) {
        ff.fapos[ia] = Vec3dZero;
        if (ia < ff.nnode) ff.fapos[ia + ff.natoms] = Vec3dZero;
        if (ia < ff.nnode) Eb += ff.eval_atom(ia);
        if (W.bNonBonded) {
            if (W.bPBC) Enb += ff.evalLJQs_ng4_PBC_atom_omp(ia);
            else        Enb += ff.evalLJQs_ng4_atom_omp(ia);
        }
        if (W.bGridFF) Eg += W.gridFF.addAtom(ff.apos[ia], ff.PLQd[ia], ff.fapos[ia]);
    }
    for (int ia = 0; ia < ff.natoms; ia++) ff.assemble_atom(ia);
    for (int i = 0; i < ff.nvecs; i++) { force[3 * i] = ff.fapos[i].x; force[3 * i + 1] = ff.fapos[i].y; force[3 * i + 2] = ff.fapos[i].z; }
    Es[0] = Eb; Es[1] = Enb; Es[2] = Eg; Es[3] = Eb + Enb + Eg;
}

// FIRE relaxation through MolWorld_sp3::run_no_omp.
// fire: [dt, damping, lastNeg, dt_max, dt_min, damp_max, finc, fdec, falpha, minLastNeg, cv_kill]
int ref_relax(int niter, double Fconv, double* pos, double* vel, double* fire, double* outE, double* outF) {
    MMFFsp3_loc& ff = W.ffl;
    for (int i = 0; i < ff.nvecs; i++) {
        ff.apos[i] = Vec3d{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        ff.vapos[i] = Vec3d{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    }
    DynamicOpt& o = W.opt;
    o.dt = fire[0]; o.damping = fire[1]; o.lastNeg = (int)fire[2];
    o.dt_max = fire[3]; o.dt_min = fire[4]; o.damp_max = fire[5];
    o.finc = fire[6]; o.fdec = fire[7]; o.falpha = fire[8]; o.minLastNeg = (int)fire[9]; o.cv_kill = fire[10];
    int itr = W.run_no_omp(niter, -1.0, Fconv, 1000, -1.0, outE, outF);
    for (int i = 0; i < ff.nvecs; i++) {
        pos[3 * i] = ff.apos[i].x; pos[3 * i + 1] = ff.apos[i].y; pos[3 * i + 2] = ff.apos[i].z;
        vel[3 * i] = ff.vapos[i].x; vel[3 * i + 1] = ff.vapos[i].y; vel[3 * i + 2] = ff.vapos[i].z;
    }
    fire[0] = o.dt; fire[1] = o.damping; fire[2] = o.lastNeg;
    return itr;
}

// The exploring cycle of run_no_omp with bGopt (MolWorld_sp3.h:2290-2296,
// 2397-2424, 2465-2473): GOpt on / off, its nExplore, the Langevin drive's
// temperature and friction, and its current state (exploring, istep).  A
// minimum found while relaxing makes run_no_omp append the geometry to
// gopt.xyz in the working directory; the caller makes that open fail.
void ref_set_gopt(int on, int nExplore, double T, double gamma, int exploring, int istep) {
    W.bGopt = on != 0;
    W.go.nExplore = nExplore;
    W.go.T_target = T;
    W.go.gamma_damp = gamma;
    W.go.bExploring = exploring != 0;
    W.go.istep = istep;
}
void ref_get_gopt(int* out) { out[0] = W.go.bExploring ? 1 : 0; out[1] = W.go.istep; }

// Distance / angle constraints of the current system (after ref_setup), as
// MolWorld_sp3::addDistConstrain (MolWorld_sp3.h:515-521) and libMMFF.h:45-47
// add them; run_no_omp applies them when bConstrains is on.  dp rows: lmin,
// lmax, kmin, kmax, flim, shift a, b, c; ap rows: ang0, k.  The angle arms'
// cells, which AngleConstr's constructor leaves unset, are zero.
void ref_set_constraints(int nd, const int* di, const double* dp, int na, const int* ai, const double* ap) {
    W.constrs.bonds.clear();
    W.constrs.angles.clear();
    for (int c = 0; c < nd; c++) {
        const double* q = dp + 8 * c;
        W.addDistConstrain(di[2 * c], di[2 * c + 1], q[0], q[1], q[2], q[3], q[4], Vec3d{q[5], q[6], q[7]}, false);
    }
    for (int c = 0; c < na; c++) {
        AngleConstr a(Vec3i{ai[3 * c], ai[3 * c + 1], ai[3 * c + 2]}, Vec2d{cos(ap[2 * c] / 2.), sin(ap[2 * c] / 2.)}, ap[2 * c + 1]);
        a.acell = Vec3iZero; a.bcell = Vec3iZero;
        W.constrs.angles.push_back(a);
    }
    W.bConstrains = nd > 0;
}

void ref_grid_sample(int n, const double* pos, const double* PLQ, double* fe) {
    for (int i = 0; i < n; i++) {
        Quat4d r = W.gridFF.getForce_Bspline(Vec3d{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]},
                                             Quat4d{PLQ[4 * i], PLQ[4 * i + 1], PLQ[4 * i + 2], PLQ[4 * i + 3]});
        fe[4 * i] = r.x; fe[4 * i + 1] = r.y; fe[4 * i + 2] = r.z; fe[4 * i + 3] = r.w;
    }
}

void ref_req2plq(int n, const double* REQ, double K, double* PLQ) {
    for (int i = 0; i < n; i++) {
        Quat4d r = REQ2PLQ_d(Quat4d{REQ[4 * i], REQ[4 * i + 1], REQ[4 * i + 2], REQ[4 * i + 3]}, K);
        PLQ[4 * i] = r.x; PLQ[4 * i + 1] = r.y; PLQ[4 * i + 2] = r.z; PLQ[4 * i + 3] = r.w;
    }
}

// Bspline::fit3D_omp on one channel. ns = (nx,ny,nz) in the fit's own x-fastest
// order; Es/Gs are [nz][ny][nx].
int ref_fit3d(const int* ns, const double* Es, double* Gs, double Ftol, int nmaxiter, double dt) {
    Vec3i n{ns[0], ns[1], ns[2]};
    return Bspline::fit3D_omp(n, Gs, Es, 0, Ftol, nmaxiter, dt, 0.0, true, true);
}

// Grid node potentials with the reference point evaluators.
void ref_grid_points(int npt, const double* pts, int nsub, const double* spos, const double* sREQ,
                     const double* lvec, const int* nPBC_mors, const int* nPBC_coul, double alphaMorse,
                     double* V) {
    GridFF& g = W.gridFF;
    g.alphaMorse = alphaMorse;
    g.shift0 = Vec3dZero;
    Mat3d lv; lv.a = Vec3d{lvec[0], lvec[1], lvec[2]}; lv.b = Vec3d{lvec[3], lvec[4], lvec[5]}; lv.c = Vec3d{lvec[6], lvec[7], lvec[8]};
    Vec3d* sm = 0; Vec3d* sc = 0;
    int nm = makePBCshifts_(Vec3i{nPBC_mors[0], nPBC_mors[1], nPBC_mors[2]}, lv, sm);
    int nc = makePBCshifts_(Vec3i{nPBC_coul[0], nPBC_coul[1], nPBC_coul[2]}, lv, sc);
    std::vector<Vec3d> ap(nsub); std::vector<Quat4d> rq(nsub);
    for (int i = 0; i < nsub; i++) { ap[i] = Vec3d{spos[3 * i], spos[3 * i + 1], spos[3 * i + 2]}; rq[i] = Quat4d{sREQ[4 * i], sREQ[4 * i + 1], sREQ[4 * i + 2], sREQ[4 * i + 3]}; }
    for (int i = 0; i < npt; i++) {
        Vec3d p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
        Quat4d qp, ql;
        g.evalGridFFPoint_Mors(nm, sm, nsub, ap.data(), rq.data(), p, qp, ql);
        Quat4d qe = g.evalGridFFPoint_Coul(nc, sc, nsub, ap.data(), rq.data(), p);
        V[3 * i] = qp.w; V[3 * i + 1] = ql.w; V[3 * i + 2] = qe.w;
    }
    delete[] sm; delete[] sc;
}

// FireCore's own topology / parameter builder on one xyz file, the path the
// drop-in init takes (MolWorld_sp3::init, MolWorld_sp3.h:309-382):
// initParams (:1298-1315) -> buildMolecule_xyz (:1323-1351) -> makeFFs
// (:1442-1586, makeMMFFs -> MM::Builder::assignTypes / toMMFFsp3_loc,
// MMFFBuilder.h:1444, 4153).  A fresh MolWorld_sp3 per call.  Outputs (caller
// capacity cap atoms; returns natoms, or -1 when cap is too small):
//   counts[4] = natoms, nnode, nvecs, bPBC
//   apos [cap*2*3] (nvecs rows), REQs [cap*4], atypes [cap], neighs / neighCell [cap*4],
//   apars / bLs / bKs / Ksp / Kpp [cap*4] (nnode rows), type_names [cap*8] chars
int ref_build_xyz(const char* fElem, const char* fAtom, const char* fBond, const char* fAngle, const char* fDih,
                  const char* xyz, int bEpairs, const int* nPBC, int cap, int* counts, double* apos, double* REQs,
                  int* atypes, int* neighs, int* neighCell, double* apars, double* bLs, double* bKs, double* Ksp,
                  double* Kpp, char* type_names) {
    verbosity = 0;
    MolWorld_sp3* w = new MolWorld_sp3();
    w->bEpairs = bEpairs != 0;
    w->nPBC = Vec3i{nPBC[0], nPBC[1], nPBC[2]};
    w->bOptimizer = false;
    w->initParams(fElem, fAtom, fBond, fAngle, fDih);
    if (w->buildMolecule_xyz(xyz) < 0) return -2;
    w->makeFFs();
    MMFFsp3_loc& f = w->ffl;
    if (f.natoms > cap) return -1;
    counts[0] = f.natoms; counts[1] = f.nnode; counts[2] = f.nvecs; counts[3] = w->bPBC ? 1 : 0;
    for (int i = 0; i < f.nvecs; i++) { apos[3 * i] = f.apos[i].x; apos[3 * i + 1] = f.apos[i].y; apos[3 * i + 2] = f.apos[i].z; }
    for (int i = 0; i < f.natoms; i++) {
        for (int k = 0; k < 4; k++) {
            REQs[4 * i + k] = f.REQs[i].array[k];
            neighs[4 * i + k] = f.neighs[i].array[k];
            neighCell[4 * i + k] = w->bPBC ? f.neighCell[i].array[k] : -1;
        }
        atypes[i] = f.atypes[i];
        const char* nm = (f.atypes[i] >= 0) ? w->params.atypes[f.atypes[i]].name : "?";
        strncpy(type_names + 8 * i, nm, 8);
    }
    for (int i = 0; i < f.nnode; i++) for (int k = 0; k < 4; k++) {
        apars[4 * i + k] = f.apars[i].array[k]; bLs[4 * i + k] = f.bLs[i].array[k]; bKs[4 * i + k] = f.bKs[i].array[k];
        Ksp[4 * i + k] = f.Ksp[i].array[k]; Kpp[4 * i + k] = f.Kpp[i].array[k];
    }
    return f.natoms;
}

}  // extern "C"
