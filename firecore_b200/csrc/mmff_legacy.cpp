// mmff_legacy.cpp -- the symbols pyBall/MMFF_multi.py binds (the reference's
// cpp/libs_OCL/MMFFmulti_lib.cpp + cpp/common/molecular/libMMFF.h +
// cpp/common/libUtils.h), implemented on top of the CSR world API.
//
// The reference keeps one global MolWorld_sp3_multi W holding nSys replicas of
// one molecule, host mirrors of every GPU buffer and a name -> pointer registry
// (libUtils.h:9-47).  Here a global LegacyWorld holds the same mirrors with the
// same names and shapes (pyBall/MMFF_multi.py:210-257); the physics runs on the
// GPU through mmff_systems_upload / mmff_relax / mmff_eval.
//
// Topology: as in the reference (MolWorld_sp3::init -> initParams /
// buildMolecule_xyz / makeFFs), FireCore's parameter tables are read from
// common_resources/{Element,Atom,Bond,Angle}Types.dat under the working
// directory -- the reference reads exactly these and ignores init's four file
// arguments (MMFFmulti_lib.cpp:85 has params.init commented out); if they are
// absent, the caller's four names are tried.  mmff_builder.cpp then reproduces
// MM::Builder's typing and toMMFFsp3_loc bit for bit.  Only when no tables are
// found does a small builder of this project (bond detection by covalent
// radii, nodes = atoms with valence > 1, parameters from mmff_params.h) fill
// the same MMFFsp3_loc arrays with its own values.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "MMFFmulti_lib.h"
#include "mmff_builder.h"
#include "mmff_host.h"
#include "mmff_params.h"

using namespace mmffp;

namespace {

struct V3 { double x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double f) { return {a.x * f, a.y * f, a.z * f}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 unit(V3 a) { double l = norm(a); return l > 0 ? a * (1.0 / l) : V3{0, 0, 1}; }

int g_verbosity = 0;

struct XYZ {
    std::vector<std::string> el;
    std::vector<V3> pos;
    std::vector<double> q;
    bool has_lvs = false;
    double lvs[9] = {0};
};

bool read_xyz(const char* fname, XYZ& X) {
    std::ifstream f(fname);
    if (!f) return false;
    std::string line;
    if (!std::getline(f, line)) return false;
    int n = atoi(line.c_str());
    if (n <= 0) return false;
    std::getline(f, line);
    {
        std::istringstream is(line);
        std::string tag;
        is >> tag;
        if (tag == "lvs") {
            X.has_lvs = true;
            for (int k = 0; k < 9; k++) is >> X.lvs[k];
        }
    }
    for (int i = 0; i < n; i++) {
        if (!std::getline(f, line)) return false;
        std::istringstream is(line);
        std::string e;
        double x, y, z, q = 0.0;
        if (!(is >> e >> x >> y >> z)) return false;
        if (!(is >> q)) q = 0.0;
        X.el.push_back(e);
        X.pos.push_back({x, y, z});
        X.q.push_back(q);
    }
    return true;
}

// one molecule in MMFFsp3_loc layout (nodes first)
struct Molecule {
    int natoms = 0, nnode = 0;
    std::vector<int> el;          // element index (built-in table)
    std::vector<std::string> names;   // atom-type names (FireCore tables); empty with the built-in table
    std::vector<int> neighCell;   // [natoms*4] image index per neighbour (cell read from the xyz); empty otherwise
    std::vector<int> permut;      // input (builder) order -> index here, MM::Builder::atom_permut
    std::vector<V3> pos;          // [natoms + nnode]
    std::vector<int> neighs;      // [natoms*4]
    std::vector<int> bkneighs;    // [natoms*4]
    std::vector<double> REQ;      // [natoms*4]
    std::vector<double> apars, bLs, bKs, Ksp, Kpp;   // [nnode*4]
};

bool build_from_xyz(const XYZ& X, Molecule& M, std::string& err) {
    const int n = (int)X.el.size();
    std::vector<int> el(n);
    for (int i = 0; i < n; i++) {
        el[i] = elem_index(X.el[i].c_str());
        if (el[i] < 0 || kElem[el[i]].valence == 0) { err = "unsupported element " + X.el[i]; return false; }
    }
    // bonds by covalent radii
    std::vector<std::vector<int>> nb(n);
    for (int i = 0; i < n; i++) for (int j = i + 1; j < n; j++) {
        double r = norm(X.pos[j] - X.pos[i]);
        if (r < 1.25 * (kElem[el[i]].rcov + kElem[el[j]].rcov)) { nb[i].push_back(j); nb[j].push_back(i); }
    }
    // nodes: valence > 1; caps: valence 1 bonded to exactly one node
    std::vector<int> order, isnode(n, 0);
    for (int i = 0; i < n; i++) if (kElem[el[i]].valence > 1) { isnode[i] = 1; order.push_back(i); }
    const int nnode = (int)order.size();
    if (nnode == 0) { err = "molecule has no node (heavy) atom"; return false; }
    for (int i = 0; i < n; i++) if (!isnode[i]) {
        if (nb[i].size() != 1 || !isnode[nb[i][0]]) { err = "cap atom " + std::to_string(i) + " must bond to exactly one node"; return false; }
        order.push_back(i);
    }
    std::vector<int> inv(n);
    for (int k = 0; k < n; k++) inv[order[k]] = k;
    M.natoms = n; M.nnode = nnode;
    M.permut = inv;
    M.el.resize(n); M.pos.assign(n + nnode, V3{0, 0, 0});
    M.neighs.assign(4 * n, -1); M.bkneighs.assign(4 * n, -1); M.REQ.assign(4 * n, 0.0);
    M.apars.assign(4 * nnode, 0.0); M.bLs.assign(4 * nnode, 0.0); M.bKs.assign(4 * nnode, 0.0);
    M.Ksp.assign(4 * nnode, 0.0); M.Kpp.assign(4 * nnode, 0.0);
    for (int k = 0; k < n; k++) { M.el[k] = el[order[k]]; M.pos[k] = X.pos[order[k]]; }
    std::vector<int> npi(nnode);
    for (int k = 0; k < nnode; k++) {
        const int i = order[k];
        if (nb[i].size() > 4) { err = "atom " + std::to_string(i) + " has more than 4 bonds"; return false; }
        npi[k] = std::max(0, kElem[el[i]].valence - (int)nb[i].size());
        for (size_t q = 0; q < nb[i].size(); q++) M.neighs[4 * k + q] = inv[nb[i][q]];
    }
    for (int k = nnode; k < n; k++) M.neighs[4 * k] = inv[nb[order[k]][0]];
    // back neighbours (MMFFsp3_loc::makeBackNeighs)
    for (int ia = 0; ia < nnode; ia++) for (int j = 0; j < 4; j++) {
        const int ja = M.neighs[4 * ia + j];
        if (ja < 0) continue;
        int q = 0;
        while (q < 4 && M.bkneighs[4 * ja + q] >= 0) q++;
        if (q == 4) { err = "atom with more than 4 back-neighbours"; return false; }
        M.bkneighs[4 * ja + q] = ia * 4 + j;
    }
    // parameters and pi orientations
    for (int k = 0; k < nnode; k++) {
        const int e = M.el[k];
        const double ang = (npi[k] >= 1) ? 120.0 : kElem[e].sp3ang;
        const double a0 = ang * M_PI / 180.0 * 0.5;
        M.apars[4 * k] = std::cos(a0); M.apars[4 * k + 1] = std::sin(a0); M.apars[4 * k + 2] = 4.0 * kElem[e].Kss; M.apars[4 * k + 3] = 0.0;
        const double kpi = npi[k] > 0 ? kElem[e].Kpp : 0.0;
        int nbk = 0;
        for (int q = 0; q < 4; q++) {
            const int j = M.neighs[4 * k + q];
            if (j < 0) continue;
            nbk++;
            M.bLs[4 * k + q] = bond_l0(e, M.el[j]);
            M.bKs[4 * k + q] = bond_k(e, M.el[j]);
            M.Ksp[4 * k + q] = npi[k] > 0 ? kKsp : 0.0;
            const double kj = (j < nnode && npi[j] > 0) ? kElem[M.el[j]].Kpp : 0.0;
            M.Kpp[4 * k + q] = std::sqrt(kpi * kj);
        }
        V3 p{0, 0, 1};
        if (nbk >= 2) {
            p = cross(M.pos[M.neighs[4 * k]] - M.pos[k], M.pos[M.neighs[4 * k + 1]] - M.pos[k]);
            if (norm(p) < 1e-6) { V3 h = unit(M.pos[M.neighs[4 * k]] - M.pos[k]); p = cross(h, std::fabs(h.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0}); }
        } else if (nbk == 1) {
            V3 h = unit(M.pos[M.neighs[4 * k]] - M.pos[k]);
            p = cross(h, std::fabs(h.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0});
        }
        M.pos[n + k] = unit(p);
    }
    for (int k = 0; k < n; k++) {
        const int e = M.el[k];
        M.REQ[4 * k] = kElem[e].R0; M.REQ[4 * k + 1] = std::sqrt(kElem[e].E0); M.REQ[4 * k + 2] = X.q[order[k]]; M.REQ[4 * k + 3] = 0.0;
    }
    return true;
}

// FireCore-typed molecule (mmff_builder.cpp) -> Molecule, with back neighbours
bool from_built(const fcb::Built& B, const fcb::Tables& T, Molecule& M, std::string& err) {
    M = Molecule();
    M.natoms = B.natoms; M.nnode = B.nnode;
    M.el.assign(B.natoms, EL_C);
    for (int i = 0; i < B.natoms; i++) M.names.push_back(T.types[B.type[i]].name);
    for (int i = 0; i < B.natoms + B.nnode; i++) M.pos.push_back(V3{B.pos[3 * i], B.pos[3 * i + 1], B.pos[3 * i + 2]});
    M.neighs = B.neighs; M.REQ = B.REQ;
    M.apars = B.apars; M.bLs = B.bLs; M.bKs = B.bKs; M.Ksp = B.Ksp; M.Kpp = B.Kpp;
    if (B.pbc) M.neighCell = B.neighCell;
    M.permut = B.permut;
    M.bkneighs.assign(4 * (size_t)B.natoms, -1);
    for (int ia = 0; ia < B.nnode; ia++) for (int j = 0; j < 4; j++) {   // MMFFsp3_loc::makeBackNeighs
        const int ja = M.neighs[4 * ia + j];
        if (ja < 0) continue;
        int q = 0;
        while (q < 4 && M.bkneighs[4 * ja + q] >= 0) q++;
        if (q == 4) { err = "atom with more than 4 back-neighbours"; return false; }
        M.bkneighs[4 * ja + q] = ia * 4 + j;
    }
    return true;
}

bool file_exists(const char* f) { if (!f) return false; FILE* fp = fopen(f, "r"); if (fp) fclose(fp); return fp != nullptr; }

// FireCore's tables: common_resources/ under the working directory (what the
// reference reads), else the four names init was given; false if neither set exists
bool find_tables(const char* e, const char* a, const char* b, const char* g, fcb::Tables& T, std::string& err) {
    const char* cr[4] = {"common_resources/ElementTypes.dat", "common_resources/AtomTypes.dat", "common_resources/BondTypes.dat",
                         "common_resources/AngleTypes.dat"};
    const char* given[4] = {e, a, b, g};
    for (const char** set : {cr, given}) {
        if (!(file_exists(set[0]) && file_exists(set[1]) && file_exists(set[2]) && file_exists(set[3]))) continue;
        if (fcb::load_tables(set[0], set[1], set[2], set[3], T, err)) return true;
        return false;
    }
    err.clear();
    return false;
}

// ---------------------------------------------------------------- the world
struct LegacyWorld {
    bool ready = false;
    int nSys = 0;
    Molecule mol;
    double lvec[9] = {20, 0, 0, 0, 20, 0, 0, 0, 20};
    int nPBC[3] = {1, 1, 0};
    int flags = 1 | 2 | 4 | 8 | 16 | 128 | 256 | 512;
    bool bGrid = false;
    bool fc_tables = false;       // FireCore's tables were found and typed the molecule
    // Constrains of the world (addDistConstrain / addAngConstrain), the same for every replica:
    // dist rows (i0, i1 | lmin, lmax, kmin, kmax, flim, shift a, b, c), angle rows (centre, end1, end2 | ang0, k)
    std::vector<int> dist_i, ang_i;
    std::vector<double> dist_p, ang_p;
    fcb::Tables tables;
    // FIRE (set_opt) -- pyBall/MMFF_multi.py:349 defaults
    double fire[9] = {0.1, 0.02, 0.2, 1.1, 0.5, 0.8, 5, 0.0, 10.0};
    // thermal drive of init(T, gamma) (MolWorld_sp3_multi's TDrive): MDloop runs
    // Langevin dynamics instead of FIRE when both are > 0
    double T = 0.0, gamma = 0.0;
    bool md_set = false;          // Langevin parameters passed to the device world
    // exploring cycle of init(nExplore, nRelax) (GOpt): run(iParalel = 2) drives it
    int nExplore = 0, nRelax = 0;
    int explore_nrelax = -1;      // the give-up rule the device cycle was set up with
    // host mirrors (pyBall/MMFF_multi.py:238-256 shapes)
    std::vector<float> atoms, aforces, avel, constr, REQs, MMpars, BLs, BKs, Ksp, Kpp, lvecs, ilvecs, pbcshifts;
    // spring constants of the constr anchors (MolWorld_sp3_multi::constrK): -1 = no
    // force, as the reference initialises them (MolWorld_sp3_multi.h:224-225)
    std::vector<float> constrK;
    std::vector<int> gneighs, gneighCell, gbkNeighs;
    // single-replica CPU-side buffers (getBuff names), replica iSystemCur
    std::vector<double> DOFs, fDOFs, vDOFs, Es;
    std::vector<int> ndims, neighs1, selection;
    int iSystemCur = 0;
    // opt log / trajectory
    int optlog_n = 0;
    double *log_cos = nullptr, *log_f = nullptr, *log_v = nullptr, *log_dt = nullptr, *log_damp = nullptr;
    std::string trj_name;
    int savePerNsteps = 1;
    // substrate (for sampleSurf*)
    double alphaMorse = 1.5;
    std::unordered_map<std::string, double*> buffers;
    std::unordered_map<std::string, float*> fbuffers;
    std::unordered_map<std::string, int*> ibuffers;
};

LegacyWorld L;

int nvecs() { return L.mol.natoms + L.mol.nnode; }

void set_error(const std::string& m) { mmff_set_error(m.c_str()); if (g_verbosity >= 0) fprintf(stderr, "MMFFmulti_lib: %s\n", m.c_str()); }

int push_bond_constraints();

// pack the CSR arrays of nSys replicas from the mirrors and upload them
int upload_all(bool params) {
    const int ns = L.nSys, na = L.mol.natoms, nn = L.mol.nnode, nv = nvecs();
    std::vector<int> natoms(ns, na), nnode(ns, nn);
    std::vector<double> pos(3 * (size_t)ns * nv), vel(3 * (size_t)ns * nv);
    std::vector<int> ng(4 * (size_t)ns * na), ngC(4 * (size_t)ns * na), bk(4 * (size_t)ns * na);
    std::vector<double> REQ(4 * (size_t)ns * na), ap(4 * (size_t)ns * nn), bL(4 * (size_t)ns * nn), bK(4 * (size_t)ns * nn),
        ks(4 * (size_t)ns * nn), kp(4 * (size_t)ns * nn), lv(9 * (size_t)ns);
    for (int s = 0; s < ns; s++) {
        for (int v = 0; v < nv; v++) for (int k = 0; k < 3; k++) {
            pos[3 * ((size_t)s * nv + v) + k] = L.atoms[4 * ((size_t)s * nv + v) + k];
            vel[3 * ((size_t)s * nv + v) + k] = L.avel[4 * ((size_t)s * nv + v) + k];
        }
        for (int a = 0; a < na; a++) for (int k = 0; k < 4; k++) {
            ng[4 * ((size_t)s * na + a) + k] = L.gneighs[4 * ((size_t)s * nv + a) + k];
            ngC[4 * ((size_t)s * na + a) + k] = L.gneighCell[4 * ((size_t)s * nv + a) + k];
            bk[4 * ((size_t)s * na + a) + k] = L.gbkNeighs[4 * ((size_t)s * nv + a) + k];
            REQ[4 * ((size_t)s * na + a) + k] = L.REQs[4 * ((size_t)s * na + a) + k];
        }
        for (int i = 0; i < nn; i++) for (int k = 0; k < 4; k++) {
            const size_t o = 4 * ((size_t)s * nn + i) + k;
            ap[o] = L.MMpars[o]; bL[o] = L.BLs[o]; bK[o] = L.BKs[o]; ks[o] = L.Ksp[o]; kp[o] = L.Kpp[o];
        }
        for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) lv[9 * s + 3 * r + c] = L.lvecs[12 * s + 4 * r + c];
    }
    (void)params;
    if (mmff_set_params(L.bGrid ? L.flags : (L.flags & ~256), L.nPBC, -1.0, L.alphaMorse, 10.0)) return -1;
    if (mmff_set_fire(L.fire[0], L.fire[1], L.fire[2], L.fire[3], L.fire[4], L.fire[5], (int)L.fire[6], L.fire[7], L.fire[8], 0)) return -1;
    if (mmff_systems_upload(ns, natoms.data(), nnode.data(), pos.data(), vel.data(), ng.data(), ngC.data(), bk.data(),
                            REQ.data(), ap.data(), bL.data(), bK.data(), ks.data(), kp.data(), lv.data()))
        return -1;
    // the gpu_constr mirror (anchors, w > 0 = on) with its spring constants
    std::vector<double> ca(4 * (size_t)ns * na), ck(4 * (size_t)ns * na);
    bool any = false;
    for (size_t i = 0; i < ca.size(); i++) { ca[i] = L.constr[i]; ck[i] = L.constrK[i]; }
    for (size_t i = 0; i < (size_t)ns * na; i++) any |= ca[4 * i + 3] > 0 && (ck[4 * i] > 0 || ck[4 * i + 1] > 0 || ck[4 * i + 2] > 0);
    if (mmff_set_constraints(any ? ca.data() : nullptr, any ? ck.data() : nullptr)) return -1;
    return push_bond_constraints();
}

// the world's distance / angle constraints to the device, for every replica.
// FireCore applies its Constrains only once a distance constraint switched
// bConstrains on (libMMFF.h:41-47: addAngConstrain alone does not)
int push_bond_constraints() {
    const int nd = (int)L.dist_i.size() / 2, nang = nd ? (int)L.ang_i.size() / 3 : 0;
    if (!nd) return mmff_set_bond_constraints(0, nullptr, nullptr, 0, nullptr, nullptr);
    std::vector<int> di(3 * (size_t)nd), ai(4 * (size_t)nang);
    for (int c = 0; c < nd; c++) { di[3 * c] = -1; di[3 * c + 1] = L.dist_i[2 * c]; di[3 * c + 2] = L.dist_i[2 * c + 1]; }
    for (int c = 0; c < nang; c++) { ai[4 * c] = -1; for (int k = 0; k < 3; k++) ai[4 * c + 1 + k] = L.ang_i[3 * c + k]; }
    return mmff_set_bond_constraints(nd, di.data(), L.dist_p.data(), nang, ai.data(), L.ang_p.data());
}

// device state -> mirrors
int download_all(bool forces, bool vel) {
    const int ns = L.nSys, nv = nvecs();
    std::vector<double> pos(3 * (size_t)ns * nv), v(3 * (size_t)ns * nv), f(3 * (size_t)ns * nv);
    if (mmff_get_state(pos.data(), vel ? v.data() : nullptr, nullptr, nullptr, nullptr, nullptr)) return -1;
    if (forces && mmff_get_forces(f.data())) return -1;
    for (size_t i = 0; i < (size_t)ns * nv; i++) for (int k = 0; k < 3; k++) {
        L.atoms[4 * i + k] = (float)pos[3 * i + k];
        if (vel) L.avel[4 * i + k] = (float)v[3 * i + k];
        if (forces) L.aforces[4 * i + k] = (float)f[3 * i + k];
    }
    return 0;
}

void register_buffers() {
    L.buffers.clear(); L.fbuffers.clear(); L.ibuffers.clear();
    const int na = L.mol.natoms, nn = L.mol.nnode;
    L.buffers["DOFs"] = L.DOFs.data(); L.buffers["fDOFs"] = L.fDOFs.data(); L.buffers["vDOFs"] = L.vDOFs.data();
    L.buffers["apos"] = L.DOFs.data(); L.buffers["fapos"] = L.fDOFs.data();
    L.buffers["pipos"] = L.DOFs.data() + 3 * na; L.buffers["fpipos"] = L.fDOFs.data() + 3 * na;
    L.buffers["Es"] = L.Es.data();
    (void)nn;
    L.ibuffers["ndims"] = L.ndims.data(); L.ibuffers["neighs"] = L.neighs1.data(); L.ibuffers["selection"] = L.selection.data();
    L.ibuffers["gpu_neighs"] = L.gneighs.data(); L.ibuffers["gpu_neighCell"] = L.gneighCell.data(); L.ibuffers["gpu_bkNeighs"] = L.gbkNeighs.data();
    L.fbuffers["gpu_atoms"] = L.atoms.data(); L.fbuffers["gpu_aforces"] = L.aforces.data(); L.fbuffers["gpu_avel"] = L.avel.data();
    L.fbuffers["gpu_constr"] = L.constr.data(); L.fbuffers["gpu_REQs"] = L.REQs.data(); L.fbuffers["gpu_MMpars"] = L.MMpars.data();
    L.fbuffers["gpu_BLs"] = L.BLs.data(); L.fbuffers["gpu_BKs"] = L.BKs.data(); L.fbuffers["gpu_Ksp"] = L.Ksp.data();
    L.fbuffers["gpu_Kpp"] = L.Kpp.data(); L.fbuffers["gpu_lvecs"] = L.lvecs.data(); L.fbuffers["gpu_ilvecs"] = L.ilvecs.data();
    L.fbuffers["gpu_pbcshifts"] = L.pbcshifts.data();
}

void invert3(const double* a, double* inv) {
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
    inv[0] = (a[4] * a[8] - a[5] * a[7]) / det; inv[1] = (a[2] * a[7] - a[1] * a[8]) / det; inv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    inv[3] = (a[5] * a[6] - a[3] * a[8]) / det; inv[4] = (a[0] * a[8] - a[2] * a[6]) / det; inv[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    inv[6] = (a[3] * a[7] - a[4] * a[6]) / det; inv[7] = (a[1] * a[6] - a[0] * a[7]) / det; inv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
}

void set_lvec_all(const double* lv) {
    memcpy(L.lvec, lv, sizeof L.lvec);
    double inv[9];
    invert3(lv, inv);
    for (int s = 0; s < L.nSys; s++) for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) {
        L.lvecs[12 * s + 4 * r + c] = (float)lv[3 * r + c];
        L.ilvecs[12 * s + 4 * r + c] = (float)inv[3 * c + r];
    }
}

// replica isys <-> single-replica CPU buffers
void copy_sys_to_cpu(int isys) {
    const int nv = nvecs();
    for (int v = 0; v < nv; v++) for (int k = 0; k < 3; k++) {
        L.DOFs[3 * v + k] = L.atoms[4 * ((size_t)isys * nv + v) + k];
        L.fDOFs[3 * v + k] = L.aforces[4 * ((size_t)isys * nv + v) + k];
        L.vDOFs[3 * v + k] = L.avel[4 * ((size_t)isys * nv + v) + k];
    }
}
void copy_cpu_to_sys(int isys, bool forces, bool vel) {
    const int nv = nvecs();
    for (int v = 0; v < nv; v++) for (int k = 0; k < 3; k++) {
        L.atoms[4 * ((size_t)isys * nv + v) + k] = (float)L.DOFs[3 * v + k];
        if (forces) L.aforces[4 * ((size_t)isys * nv + v) + k] = (float)L.fDOFs[3 * v + k];
        if (vel) L.avel[4 * ((size_t)isys * nv + v) + k] = (float)L.vDOFs[3 * v + k];
    }
}

double eval_energy_sys(int isys) {
    if (mmff_eval(1)) return NAN;
    std::vector<double> E(4 * (size_t)L.nSys);
    if (mmff_get_energies(E.data())) return NAN;
    L.Es[0] = E[4 * isys + 3]; L.Es[1] = E[4 * isys + 0];
    return E[4 * isys + 3];
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ libUtils.h registry
void printBuffNames() {
    printf("#=== Buffers:  \n"); for (auto& it : L.buffers) printf("%s: %p\n", it.first.c_str(), (void*)it.second);
    printf("#=== fBuffers: \n"); for (auto& it : L.fbuffers) printf("%s: %p\n", it.first.c_str(), (void*)it.second);
    printf("#=== IBuffers: \n"); for (auto& it : L.ibuffers) printf("%s: %p\n", it.first.c_str(), (void*)it.second);
}
double* getBuff(const char* name) {
    auto it = L.buffers.find(name);
    if (it == L.buffers.end()) { printf("ERROR: getBuff(%s) NOT FOUND\n", name); printBuffNames(); return nullptr; }
    return it->second;
}
float* getfBuff(const char* name) {
    auto it = L.fbuffers.find(name);
    if (it == L.fbuffers.end()) { printf("ERROR: getfBuff(%s) NOT FOUND\n", name); printBuffNames(); return nullptr; }
    return it->second;
}
int* getIBuff(const char* name) {
    auto it = L.ibuffers.find(name);
    if (it == L.ibuffers.end()) { printf("ERROR: getIBuff(%s) NOT FOUND\n", name); printBuffNames(); return nullptr; }
    return it->second;
}

// ------------------------------------------------------------ MMFFmulti_lib.cpp
void init_buffers() { register_buffers(); }

void setVerbosity(int verbosity_, int idebug_) { g_verbosity = verbosity_; (void)idebug_; }

void* init(int nSys, char* xyz_name, char* surf_name, char* smile_name, bool bMMFF, bool bEpairs, int* nPBC, int* grid_nPBC,
           double gridStep, char* sElementTypes, char* sAtomTypes, char* sBondTypes, char* sAngleTypes, double T, double gamma,
           int nExplore, int nRelax, double pos_kick, double vel_kick, int GridFF) {
    // pos_kick / vel_kick feed GOpt::apply_kick, which the reference never calls
    (void)smile_name; (void)bMMFF; (void)pos_kick; (void)vel_kick;
    L.T = T; L.gamma = gamma; L.md_set = false;
    L.nExplore = nExplore; L.nRelax = nRelax; L.explore_nrelax = -1;
    L.dist_i.clear(); L.dist_p.clear(); L.ang_i.clear(); L.ang_p.clear();
    {   // a new world: the cell of an earlier init (its substrate or xyz) does not carry over
        const double lv0[9] = {20, 0, 0, 0, 20, 0, 0, 0, 20};
        memcpy(L.lvec, lv0, sizeof L.lvec);
    }
    if (nSys < 1 || !xyz_name) { set_error("init: need nSys >= 1 and an xyz file"); return nullptr; }
    if (mmff_init_device(0)) { set_error(std::string("init: ") + mmff_last_error()); return nullptr; }
    XYZ X;
    std::string fn = xyz_name;
    // MolWorld_sp3::insertMolecule appends ".xyz" to a name without extension
    if (!read_xyz(fn.c_str(), X)) {
        fn += ".xyz";
        if (!read_xyz(fn.c_str(), X)) { set_error("init: cannot read " + std::string(xyz_name)); return nullptr; }
    }
    std::string err;
    if (nPBC) for (int k = 0; k < 3; k++) L.nPBC[k] = nPBC[k];
    L.fc_tables = find_tables(sElementTypes, sAtomTypes, sBondTypes, sAngleTypes, L.tables, err);
    if (!L.fc_tables && !err.empty()) { set_error("init: " + err); return nullptr; }
    if (L.fc_tables) {
        fcb::Built B;
        if (!fcb::build_xyz(L.tables, fn.c_str(), bEpairs, L.nPBC, B, err) || !from_built(B, L.tables, L.mol, err)) {
            set_error("init: " + err); return nullptr;
        }
    } else if (!build_from_xyz(X, L.mol, err)) { set_error("init: " + err); return nullptr; }
    L.nSys = nSys;
    const int na = L.mol.natoms, nn = L.mol.nnode, nv = na + nn;
    if (X.has_lvs) memcpy(L.lvec, X.lvs, sizeof L.lvec);
    // substrate and GridFF (GridFF > 0)
    L.bGrid = false;
    if (surf_name && GridFF > 0) {
        XYZ S;
        std::string sn = surf_name;
        if (!read_xyz(sn.c_str(), S) && !read_xyz((sn + ".xyz").c_str(), S)) { set_error("init: cannot read substrate " + sn); return nullptr; }
        if (!S.has_lvs) { set_error("init: substrate file needs an lvs line"); return nullptr; }
        const int nsub = (int)S.el.size();
        std::vector<double> spos(3 * nsub), sREQ(4 * nsub);
        double ztop = -1e300;
        for (int i = 0; i < nsub; i++) {
            spos[3 * i] = S.pos[i].x; spos[3 * i + 1] = S.pos[i].y; spos[3 * i + 2] = S.pos[i].z;
            if (L.fc_tables) {   // MolWorld_sp3::loadSurf reads the substrate through MMFFparams::loadXYZ
                fcb::substrate_REQ(L.tables, S.el[i], S.q[i], 0.0, &sREQ[4 * i]);
            } else {
                const int e = elem_index(S.el[i].c_str());
                const Elem& E = kElem[e < 0 ? EL_C : e];
                sREQ[4 * i] = E.R0; sREQ[4 * i + 1] = std::sqrt(E.E0); sREQ[4 * i + 2] = S.q[i]; sREQ[4 * i + 3] = 0;
            }
            ztop = std::max(ztop, S.pos[i].z);
        }
        const double step = gridStep > 0 ? gridStep : 0.1;
        const int nx = std::max(4, (int)std::lround(S.lvs[0] / step)), ny = std::max(4, (int)std::lround(S.lvs[4] / step));
        const int nz = std::max(8, (int)std::lround(20.0 / step));
        const double pos0[3] = {0, 0, ztop + 0.5};
        const double st[3] = {S.lvs[0] / nx, S.lvs[4] / ny, step};
        const int npm[3] = {grid_nPBC ? grid_nPBC[0] : 1, grid_nPBC ? grid_nPBC[1] : 1, 0};
        const int npc[3] = {25, 25, 0};
        if (mmff_grid_build(nsub, spos.data(), sREQ.data(), S.lvs, npm, npc, L.alphaMorse, nx, ny, nz, pos0, st, nullptr)) {
            set_error(std::string("init: grid build: ") + mmff_last_error()); return nullptr;
        }
        memcpy(L.lvec, S.lvs, sizeof L.lvec);
        L.bGrid = true;
    }
    // mirrors
    L.atoms.assign(4 * (size_t)nSys * nv, 0.f); L.aforces.assign(4 * (size_t)nSys * nv, 0.f); L.avel.assign(4 * (size_t)nSys * nv, 0.f);
    L.constr.assign(4 * (size_t)nSys * na, -1.f); L.REQs.assign(4 * (size_t)nSys * na, 0.f);
    L.constrK.assign(4 * (size_t)nSys * na, -1.f);
    L.MMpars.assign(4 * (size_t)nSys * nn, 0.f); L.BLs.assign(4 * (size_t)nSys * nn, 0.f); L.BKs.assign(4 * (size_t)nSys * nn, 0.f);
    L.Ksp.assign(4 * (size_t)nSys * nn, 0.f); L.Kpp.assign(4 * (size_t)nSys * nn, 0.f);
    L.lvecs.assign(12 * (size_t)nSys, 0.f); L.ilvecs.assign(12 * (size_t)nSys, 0.f);
    const int np = (2 * L.nPBC[0] + 1) * (2 * L.nPBC[1] + 1) * (2 * L.nPBC[2] + 1);
    L.pbcshifts.assign(4 * (size_t)nSys * np, 0.f);
    L.gneighs.assign(4 * (size_t)nSys * nv, -1); L.gneighCell.assign(4 * (size_t)nSys * nv, -1); L.gbkNeighs.assign(4 * (size_t)nSys * nv, -1);
    const int central = (L.nPBC[2] * (2 * L.nPBC[1] + 1) + L.nPBC[1]) * (2 * L.nPBC[0] + 1) + L.nPBC[0];
    for (int s = 0; s < nSys; s++) {
        for (int v = 0; v < nv; v++) {
            L.atoms[4 * ((size_t)s * nv + v)] = (float)L.mol.pos[v].x; L.atoms[4 * ((size_t)s * nv + v) + 1] = (float)L.mol.pos[v].y;
            L.atoms[4 * ((size_t)s * nv + v) + 2] = (float)L.mol.pos[v].z;
        }
        for (int a = 0; a < na; a++) for (int k = 0; k < 4; k++) {
            const int j = L.mol.neighs[4 * a + k];
            L.gneighs[4 * ((size_t)s * nv + a) + k] = j;
            L.gneighCell[4 * ((size_t)s * nv + a) + k] = j < 0 ? -1 : (L.mol.neighCell.empty() ? central : L.mol.neighCell[4 * a + k]);
            L.gbkNeighs[4 * ((size_t)s * nv + a) + k] = L.mol.bkneighs[4 * a + k];
            L.REQs[4 * ((size_t)s * na + a) + k] = (float)L.mol.REQ[4 * a + k];
        }
        for (int i = 0; i < nn; i++) {
            for (int k = 0; k < 4; k++) L.gbkNeighs[4 * ((size_t)s * nv + na + i) + k] = L.mol.bkneighs[4 * i + k];
            for (int k = 0; k < 4; k++) {
                const size_t o = 4 * ((size_t)s * nn + i) + k;
                L.MMpars[o] = (float)L.mol.apars[4 * i + k]; L.BLs[o] = (float)L.mol.bLs[4 * i + k]; L.BKs[o] = (float)L.mol.bKs[4 * i + k];
                L.Ksp[o] = (float)L.mol.Ksp[4 * i + k]; L.Kpp[o] = (float)L.mol.Kpp[4 * i + k];
            }
        }
    }
    set_lvec_all(L.lvec);
    L.DOFs.assign(3 * (size_t)nv, 0.0); L.fDOFs.assign(3 * (size_t)nv, 0.0); L.vDOFs.assign(3 * (size_t)nv, 0.0);
    L.Es.assign(6, 0.0);
    L.ndims = {3 * nv, nn, na - nn, nv, 0, 0};
    L.neighs1.assign(L.mol.neighs.begin(), L.mol.neighs.begin() + 4 * nn);
    L.selection.assign(na, 0);
    copy_sys_to_cpu(0);
    register_buffers();
    if (upload_all(true)) { set_error(std::string("init: upload: ") + mmff_last_error()); return nullptr; }
    L.ready = true;
    return &L;
}

// Relax every replica on the GPU; returns the largest number of steps any
// replica took (run_ocl_opt's count).  As in MMFFmulti_lib.cpp:116-132, dt
// and ialg are not used (the FIRE time steps come from set_opt).  iParalel
// selects the reference's CPU (-1, 0, 1) or OpenCL (2, 3, 4) drivers there;
// this library has only the device path, so every value runs it.
int run(int nstepMax, double dt, double Fconv, int ialg, double* outE, double* outF, int iParalel) {
    (void)dt; (void)ialg;
    if (!L.ready) { set_error("run: init() first"); return -1; }
    if (iParalel >= 0 && iParalel <= 2 && L.nExplore > 0) {
        // run_omp_ocl (iParalel 0, 1) and run_ocl_opt (2) with GOpt, which init
        // switches on (MMFFmulti_lib.cpp:88; MolWorld_sp3_multi.h:1970-2050,
        // 1694-1846, 770-833): every replica cycles between FIRE and nExplore
        // Langevin steps (time step = the FIRE dt_max, MolWorld_sp3_multi.h:756-760,
        // 2012); only run_ocl_opt gives up a relax phase after nRelax steps.
        // After init every replica starts exploring (MolWorld_sp3_multi.h:278).
        // The cycle's state lives on the device until the systems are uploaded
        // again or the give-up rule changes.
        const int nrelax = iParalel == 2 ? L.nRelax : 0;
        if (mmff_get_explore(nullptr, nullptr) || nrelax != L.explore_nrelax) {
            if (mmff_set_md(L.fire[0], L.gamma, L.T, 12345ull) || mmff_set_explore(L.nExplore, nrelax, 1)) {
                set_error(mmff_last_error()); return -1;
            }
            L.md_set = true;
            L.explore_nrelax = nrelax;
        }
        if (mmff_explore(nstepMax, Fconv, 0)) { set_error(mmff_last_error()); return -1; }
    } else if (mmff_relax(nstepMax, Fconv, 0)) { set_error(mmff_last_error()); return -1; }
    std::vector<int> ns(L.nSys);
    std::vector<double> fc(L.nSys);
    if (mmff_get_state(nullptr, nullptr, nullptr, nullptr, ns.data(), fc.data())) return -1;
    if (download_all(true, true)) return -1;
    copy_sys_to_cpu(L.iSystemCur);
    int mx = 0;
    for (int s = 0; s < L.nSys; s++) mx = std::max(mx, ns[s]);
    if (outF) outF[0] = *std::max_element(fc.begin(), fc.end());
    if (outE) outE[0] = eval_energy_sys(L.iSystemCur);
    if (!L.trj_name.empty()) saveXYZ(L.trj_name.c_str(), "# run", 1);
    return mx;
}

// MolWorld_sp3_multi::MDloop: perframe steps of the path its iParalel selects
// (MolWorld_sp3_multi.h:2236-2243: 0 run_no_omp, 1-2 run_omp_ocl, 3 run_ocl_opt),
// i.e. FIRE relaxation, or with init's nExplore > 0 the exploring cycle; with
// nExplore = 0 and init(T > 0, gamma > 0) the Langevin drive for every replica
// instead (time step = the FIRE dt_max), which FireCore only applies to
// exploring replicas
void MDloop(int perframe, double Ftol, int iParalel, int perVF) {
    (void)perVF;
    if (L.ready && L.nExplore > 0 && iParalel >= 0 && iParalel <= 3) {
        run(perframe, -1, Ftol > 0 ? Ftol : 1e-6, 0, nullptr, nullptr, iParalel == 3 ? 2 : 1);
        return;
    }
    if (L.ready && L.T > 0 && L.gamma > 0) {
        if (!L.md_set && mmff_set_md(L.fire[0], L.gamma, L.T, 12345ull)) { set_error(mmff_last_error()); return; }
        L.md_set = true;
        if (mmff_md(perframe) || mmff_sync()) { set_error(mmff_last_error()); return; }
        if (download_all(true, true)) return;
        copy_sys_to_cpu(L.iSystemCur);
        if (!L.trj_name.empty()) saveXYZ(L.trj_name.c_str(), "# MDloop", 1);
        return;
    }
    run(perframe, -1, Ftol > 0 ? Ftol : 1e-6, 0, nullptr, nullptr, iParalel);
}

void set_opt(double dt_max, double dt_min, double damp_max, double finc, double fdec, double falpha, int minLastNeg,
             double cvf_min, double cvf_max) {
    (void)cvf_min; (void)cvf_max;
    double f[9] = {dt_max, dt_min, damp_max, finc, fdec, falpha, (double)minLastNeg, 0.0, L.fire[8]};
    memcpy(L.fire, f, sizeof f);
    mmff_set_fire(f[0], f[1], f[2], f[3], f[4], f[5], minLastNeg, f[7], f[8], 0);
}

void pack_system(int isys, bool bParams, bool bForces, bool bVel, bool blvec) {
    (void)bParams; (void)blvec;
    if (isys < 0 || isys >= L.nSys) return;
    copy_cpu_to_sys(isys, bForces, bVel);
}
void unpack_system(int isys, bool bForces, bool bVel) {
    (void)bForces; (void)bVel;
    if (isys < 0 || isys >= L.nSys) return;
    L.iSystemCur = isys;
    copy_sys_to_cpu(isys);
}
void upload_sys(int isys, bool bParams, bool bForces, bool bVel, bool blvec) { (void)isys; upload(bParams, bForces, bVel, blvec); }
void download_sys(int isys, bool bForces, bool bVel) { (void)isys; download(bForces, bVel); }
void upload(bool bParams, bool bForces, bool bVel, bool blvec) {
    (void)bForces; (void)bVel; (void)blvec;
    if (!L.ready) return;
    if (upload_all(bParams)) set_error(std::string("upload: ") + mmff_last_error());
}
void download(bool bForces, bool bVel) {
    if (!L.ready) return;
    if (download_all(bForces, bVel)) set_error(std::string("download: ") + mmff_last_error());
}

void change_lvec(double* lvec, bool bAdd, bool bUpdatePi) {
    (void)bUpdatePi;
    double lv[9];
    for (int k = 0; k < 9; k++) lv[k] = bAdd ? L.lvec[k] + lvec[k] : lvec[k];
    set_lvec_all(lv);
    if (L.ready) upload_all(false);
}

// population: a multi-frame xyz, one frame per replica
void upload_pop(const char* fname) {
    std::ifstream f(fname);
    if (!f || !L.ready) { set_error(std::string("upload_pop: cannot read ") + (fname ? fname : "")); return; }
    const int na = L.mol.natoms, nv = nvecs();
    for (int s = 0; s < L.nSys; s++) {
        std::string line;
        if (!std::getline(f, line)) break;
        int n = atoi(line.c_str());
        std::getline(f, line);
        if (n != na) { set_error("upload_pop: frame size differs from the molecule"); return; }
        for (int i = 0; i < n; i++) {
            std::getline(f, line);
            std::istringstream is(line); std::string e; double x, y, z;
            is >> e >> x >> y >> z;
            L.atoms[4 * ((size_t)s * nv + i)] = (float)x; L.atoms[4 * ((size_t)s * nv + i) + 1] = (float)y; L.atoms[4 * ((size_t)s * nv + i) + 2] = (float)z;
        }
    }
    upload_all(false);
}

// lattice scans: relax every replica at lvec + i*dlvec (replica i), report in stdout
void optimizeLattice_1d(double* dlvec, int n1, int n2, int initMode, double tol) {
    (void)initMode;
    if (!L.ready) return;
    const double lv0[9] = {L.lvec[0], L.lvec[1], L.lvec[2], L.lvec[3], L.lvec[4], L.lvec[5], L.lvec[6], L.lvec[7], L.lvec[8]};
    for (int i = -n1; i <= n2; i++) {
        double lv[9];
        for (int k = 0; k < 9; k++) lv[k] = lv0[k] + dlvec[k] * i;
        set_lvec_all(lv);
        upload_all(false);
        run(1000, -1, tol > 0 ? tol : 1e-4, 0, nullptr, nullptr, 2);
        printf("optimizeLattice_1d[%i] E=%g\n", i, eval_energy_sys(0));
    }
    set_lvec_all(lv0);
    upload_all(false);
}
void optimizeLattice_2d_multi(double* dlvec, int nstesp, int initMode, double tol) { optimizeLattice_1d(dlvec, 0, nstesp, initMode, tol); }

// MolWorld_sp3_multi::scan_relaxed (MolWorld_sp3_multi.h:1242-1296), which
// MMFFmulti_lib.cpp:305-314 calls for every scan: configuration i is the
// molecule placed by setFromRef (MMFFsp3_loc.h:1543-1551: p = rot^T ref +
// poss[i], pi = rot^T pi_ref) with atom ipicked = 0 pinned to poss[i] by a unit
// spring (constr / constrK), relaxed with niter_max FIRE steps to Fconv;
// Es[i], aforces and aposs [nconf*natoms*3] (nullable) are its energy, forces
// (without the spring) and positions afterwards.  The reference refills each
// relaxed replica slot with the next configuration; here every configuration
// is a system of one uploaded batch and the persistent relax kernels claim
// them from their work queue, so a finished slot takes the next
// configuration without a host round trip.  omp, bRelax, dt and Flim are not
// used (as in the reference).  The replicas of init() are restored afterwards.
void scan(int nconf, double* poss, double* rots, double* Es, double* aforces, double* aposs, bool omp, bool bRelax, int niter_max,
          double dt, double Fconv, double Flim) {
    (void)omp; (void)bRelax; (void)dt; (void)Flim;
    if (!L.ready || nconf < 1 || !poss) return;
    const int na = L.mol.natoms, nn = L.mol.nnode, nv = na + nn;
    const int ipicked = 0;
    std::vector<int> natoms(nconf, na), nnode(nconf, nn);
    std::vector<double> pos(3 * (size_t)nconf * nv), ca(4 * (size_t)nconf * na, -1.0), ck(4 * (size_t)nconf * na, -1.0);
    std::vector<int> ng(4 * (size_t)nconf * na), ngC(4 * (size_t)nconf * na), bk(4 * (size_t)nconf * na);
    std::vector<double> REQ(4 * (size_t)nconf * na), ap(4 * (size_t)nconf * nn), bL(4 * (size_t)nconf * nn),
        bK(4 * (size_t)nconf * nn), ks(4 * (size_t)nconf * nn), kp(4 * (size_t)nconf * nn), lv(9 * (size_t)nconf);
    for (int c = 0; c < nconf; c++) {
        static const double I3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        const double* R = rots ? rots + 9 * c : I3;
        const V3 p0{poss[3 * c], poss[3 * c + 1], poss[3 * c + 2]};
        for (int v = 0; v < nv; v++) {
            const V3 d = L.mol.pos[v];
            // Mat3d::dot_to_T: out_k = sum_j R[3 j + k] d_j
            V3 r{R[0] * d.x + R[3] * d.y + R[6] * d.z, R[1] * d.x + R[4] * d.y + R[7] * d.z, R[2] * d.x + R[5] * d.y + R[8] * d.z};
            if (v < na) r = r + p0;
            pos[3 * ((size_t)c * nv + v)] = r.x; pos[3 * ((size_t)c * nv + v) + 1] = r.y; pos[3 * ((size_t)c * nv + v) + 2] = r.z;
        }
        const size_t ia = 4 * ((size_t)c * na + ipicked);
        ca[ia] = p0.x; ca[ia + 1] = p0.y; ca[ia + 2] = p0.z; ca[ia + 3] = 1.0;
        ck[ia] = ck[ia + 1] = ck[ia + 2] = ck[ia + 3] = 1.0;
        // topology and parameters of replica 0
        for (int a = 0; a < na; a++) for (int k = 0; k < 4; k++) {
            ng[4 * ((size_t)c * na + a) + k] = L.gneighs[4 * (size_t)a + k];
            ngC[4 * ((size_t)c * na + a) + k] = L.gneighCell[4 * (size_t)a + k];
            bk[4 * ((size_t)c * na + a) + k] = L.gbkNeighs[4 * (size_t)a + k];
            REQ[4 * ((size_t)c * na + a) + k] = L.REQs[4 * (size_t)a + k];
        }
        for (int i = 0; i < nn; i++) for (int k = 0; k < 4; k++) {
            const size_t o = 4 * ((size_t)c * nn + i) + k, o0 = 4 * (size_t)i + k;
            ap[o] = L.MMpars[o0]; bL[o] = L.BLs[o0]; bK[o] = L.BKs[o0]; ks[o] = L.Ksp[o0]; kp[o] = L.Kpp[o0];
        }
        for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++) lv[9 * c + 3 * r + q] = L.lvecs[4 * r + q];
    }
    auto check = [](int rc) { if (rc) set_error(std::string("scan: ") + mmff_last_error()); return rc != 0; };
    if (check(mmff_systems_upload(nconf, natoms.data(), nnode.data(), pos.data(), nullptr, ng.data(), ngC.data(), bk.data(),
                                  REQ.data(), ap.data(), bL.data(), bK.data(), ks.data(), kp.data(), lv.data())))
        return;
    if (check(mmff_set_constraints(ca.data(), ck.data())) || check(mmff_relax(niter_max, Fconv, 0)) || check(mmff_eval(1)))
        return;
    std::vector<double> E(4 * (size_t)nconf), F(3 * (size_t)nconf * nv), P(3 * (size_t)nconf * nv);
    if (check(mmff_get_energies(E.data())) || check(mmff_get_forces(F.data())) ||
        check(mmff_get_state(P.data(), nullptr, nullptr, nullptr, nullptr, nullptr)))
        return;
    for (int c = 0; c < nconf; c++) {
        if (Es) Es[c] = E[4 * c + 3];
        for (int a = 0; a < na; a++) for (int k = 0; k < 3; k++) {
            if (aforces) aforces[3 * ((size_t)c * na + a) + k] = F[3 * ((size_t)c * nv + a) + k];
            if (aposs) aposs[3 * ((size_t)c * na + a) + k] = P[3 * ((size_t)c * nv + a) + k];
        }
    }
    check(upload_all(true));
}

// tri-state switches (>0 on, <0 off, 0 keep), MMFFmulti_lib.cpp:316-329
void setSwitches_multi(int CheckInvariants, int PBC, int NonBonded, int MMFF, int Angles, int PiSigma, int PiPiI, int dovdW,
                       int bSaveToDatabase) {
    (void)CheckInvariants; (void)dovdW; (void)bSaveToDatabase;
    auto setbit = [](int v, int bit) { if (v > 0) L.flags |= bit; else if (v < 0) L.flags &= ~bit; };
    setbit(PBC, 512);
    setbit(NonBonded, 128);
    setbit(MMFF, 1);
    setbit(Angles, 8);
    setbit(PiSigma, 4);
    setbit(PiPiI, 2);
    if (L.flags & 128) L.flags |= 16; else L.flags &= ~16;   // bSubtractAngleNonBond = bNonBonded
    if (L.ready) mmff_set_params(L.bGrid ? L.flags : (L.flags & ~256), L.nPBC, -1.0, L.alphaMorse, 10.0);
}

// ------------------------------------------------------------ libMMFF.h
void insertSMILES(char* s) { (void)s; set_error("insertSMILES: SMILES input is not supported; use an xyz file"); }

// net force and torque of the current replica (MolWorld_sp3::checkInvariants)
bool checkInvariants(double maxVcog, double maxFcog, double maxTg) {
    (void)maxVcog;
    if (!L.ready) return false;
    mmff_eval(0);
    download_all(true, false);
    copy_sys_to_cpu(L.iSystemCur);
    const int na = L.mol.natoms;
    V3 F{0, 0, 0}, T{0, 0, 0}, c{0, 0, 0};
    for (int i = 0; i < na; i++) c = c + V3{L.DOFs[3 * i], L.DOFs[3 * i + 1], L.DOFs[3 * i + 2]};
    c = c * (1.0 / na);
    for (int i = 0; i < na; i++) {
        V3 f{L.fDOFs[3 * i], L.fDOFs[3 * i + 1], L.fDOFs[3 * i + 2]}, p{L.DOFs[3 * i], L.DOFs[3 * i + 1], L.DOFs[3 * i + 2]};
        F = F + f; T = T + cross(p - c, f);
    }
    return norm(F) > maxFcog || norm(T) > maxTg;   // true = invariants violated (as the reference)
}

void setOptLog(int n, double* cos, double* f, double* v, double* dt, double* damp) {
    L.optlog_n = n; L.log_cos = cos; L.log_f = f; L.log_v = v; L.log_dt = dt; L.log_damp = damp;
}

bool setTrjName(const char* trj_fname_, int savePerNsteps_) {
    L.trj_name = trj_fname_ ? trj_fname_ : "";
    L.savePerNsteps = savePerNsteps_;
    return true;
}

// append replica isys = imod-1 (0: current) as an xyz frame
int saveXYZ(const char* fname, const char* comment, int imod) {
    if (!L.ready || !fname) return -1;
    FILE* f = fopen(fname, "a");
    if (!f) return -1;
    const int na = L.mol.natoms, nv = nvecs();
    const int s = (imod > 0 && imod <= L.nSys) ? imod - 1 : L.iSystemCur;
    fprintf(f, "%i\n%s\n", na, comment ? comment : "");
    for (int i = 0; i < na; i++)
        fprintf(f, "%s %12.6f %12.6f %12.6f\n", L.mol.names.empty() ? kElem[L.mol.el[i]].sym : L.mol.names[i].c_str(), L.atoms[4 * ((size_t)s * nv + i)],
                L.atoms[4 * ((size_t)s * nv + i) + 1], L.atoms[4 * ((size_t)s * nv + i) + 2]);
    fclose(f);
    return na;
}

const char* getTypeName(int ia, bool fromFF) {
    (void)fromFF;
    if (!L.ready || ia < 0 || ia >= L.mol.natoms) return "?";
    return L.mol.names.empty() ? kElem[L.mol.el[ia]].sym : L.mol.names[ia].c_str();
}

double eval() {
    if (!L.ready) return NAN;
    copy_cpu_to_sys(L.iSystemCur, false, false);
    upload_all(false);
    const double E = eval_energy_sys(L.iSystemCur);
    download_all(true, false);
    copy_sys_to_cpu(L.iSystemCur);
    return E;
}

// libMMFF.h:41-47 (MolWorld_sp3::addDistConstrain, MolWorld_sp3.h:515-521): a
// flat-bottom spring between atoms i0 and i1 of every replica, applied by the
// relaxations from the next run on.  bOldIndex: i0, i1 count atoms in the
// input order (before nodes were sorted first), as the reference's
// builder.atom_permut maps them.
void addDistConstrain(int i0, int i1, double lmin, double lmax, double kmin, double kmax, double flim, double* shift, bool bOldIndex) {
    if (!L.ready) { set_error("addDistConstrain: call init first"); return; }
    const int nperm = (int)L.mol.permut.size();
    if (bOldIndex) {
        if (i0 < 0 || i1 < 0 || i0 >= nperm || i1 >= nperm) { set_error("addDistConstrain: atom index out of range"); return; }
        i0 = L.mol.permut[i0]; i1 = L.mol.permut[i1];
    }
    if (i0 < 0 || i1 < 0 || i0 >= L.mol.natoms || i1 >= L.mol.natoms) { set_error("addDistConstrain: atom index out of range"); return; }
    L.dist_i.push_back(i0); L.dist_i.push_back(i1);
    const double sh[3] = {shift ? shift[0] : 0.0, shift ? shift[1] : 0.0, shift ? shift[2] : 0.0};
    for (double v : {lmin, lmax, kmin, kmax, flim, sh[0], sh[1], sh[2]}) L.dist_p.push_back(v);
    if (push_bond_constraints()) set_error(std::string("addDistConstrain: ") + mmff_last_error());
}
// libMMFF.h:45-47: the angle i1-i0-i2 (i0 the centre) held at ang0 with
// E = k (1 - cos((a - ang0)/2)); active once a distance constraint exists
void addAngConstrain(int i0, int i1, int i2, double ang0, double k) {
    if (!L.ready) { set_error("addAngConstrain: call init first"); return; }
    for (int i : {i0, i1, i2}) if (i < 0 || i >= L.mol.natoms) { set_error("addAngConstrain: atom index out of range"); return; }
    L.ang_i.push_back(i0); L.ang_i.push_back(i1); L.ang_i.push_back(i2);
    L.ang_p.push_back(ang0); L.ang_p.push_back(k);
    if (push_bond_constraints()) set_error(std::string("addAngConstrain: ") + mmff_last_error());
}

// manipulation of the current replica's CPU buffers (DOFs); apply with pack_system + upload
void shift_atoms_ax(int n, int* selection, double* d) {
    for (int k = 0; k < n; k++) { int i = selection ? selection[k] : k; for (int c = 0; c < 3; c++) L.DOFs[3 * i + c] += d[c]; }
}
void shift_atoms(int n, int* selection, int ia0, int ia1, double l) {
    V3 a{L.DOFs[3 * ia0], L.DOFs[3 * ia0 + 1], L.DOFs[3 * ia0 + 2]}, b{L.DOFs[3 * ia1], L.DOFs[3 * ia1 + 1], L.DOFs[3 * ia1 + 2]};
    V3 d = unit(b - a) * l;
    double dd[3] = {d.x, d.y, d.z};
    shift_atoms_ax(n, selection, dd);
}
void rotate_atoms_ax(int n, int* selection, double* p0, double* ax, double phi) {
    V3 u = unit(V3{ax[0], ax[1], ax[2]});
    const double c = std::cos(phi), s = std::sin(phi);
    for (int k = 0; k < n; k++) {
        int i = selection ? selection[k] : k;
        V3 p = V3{L.DOFs[3 * i], L.DOFs[3 * i + 1], L.DOFs[3 * i + 2]} - V3{p0[0], p0[1], p0[2]};
        V3 r = p * c + cross(u, p) * s + u * (dot(u, p) * (1 - c));   // Rodrigues
        L.DOFs[3 * i] = r.x + p0[0]; L.DOFs[3 * i + 1] = r.y + p0[1]; L.DOFs[3 * i + 2] = r.z + p0[2];
    }
}
void rotate_atoms(int n, int* selection, int ia0, int iax0, int iax1, double phi) {
    double p0[3] = {L.DOFs[3 * ia0], L.DOFs[3 * ia0 + 1], L.DOFs[3 * ia0 + 2]};
    double ax[3] = {L.DOFs[3 * iax1] - L.DOFs[3 * iax0], L.DOFs[3 * iax1 + 1] - L.DOFs[3 * iax0 + 1], L.DOFs[3 * iax1 + 2] - L.DOFs[3 * iax0 + 2]};
    rotate_atoms_ax(n, selection, p0, ax, phi);
}

// scans: nstep rigid moves of a selection of the current replica, energy after each
void scanTranslation_ax(int n, int* selection, double* vec, int nstep, double* Es, const char* trjName, bool bAddjustCaps) {
    (void)bAddjustCaps;
    double d[3] = {vec[0] / nstep, vec[1] / nstep, vec[2] / nstep};
    for (int i = 0; i < nstep; i++) {
        shift_atoms_ax(n, selection, d);
        const double E = eval();
        if (Es) Es[i] = E;
        if (trjName) saveXYZ(trjName, "# scanTranslation", 0);
    }
}
void scanTranslation(int n, int* selection, int ia0, int ia1, double l, int nstep, double* Es, const char* trjName, bool bAddjustCaps) {
    V3 a{L.DOFs[3 * ia0], L.DOFs[3 * ia0 + 1], L.DOFs[3 * ia0 + 2]}, b{L.DOFs[3 * ia1], L.DOFs[3 * ia1 + 1], L.DOFs[3 * ia1 + 2]};
    V3 d = unit(b - a) * l;
    double v[3] = {d.x, d.y, d.z};
    scanTranslation_ax(n, selection, v, nstep, Es, trjName, bAddjustCaps);
}
void scanRotation_ax(int n, int* selection, double* p0, double* ax, double phi, int nstep, double* Es, const char* trjName) {
    for (int i = 0; i < nstep; i++) {
        rotate_atoms_ax(n, selection, p0, ax, phi / nstep);
        const double E = eval();
        if (Es) Es[i] = E;
        if (trjName) saveXYZ(trjName, "# scanRotation", 0);
    }
}
void scanRotation(int n, int* selection, int ia0, int iax0, int iax1, double phi, int nstep, double* Es, const char* trjName) {
    double p0[3] = {L.DOFs[3 * ia0], L.DOFs[3 * ia0 + 1], L.DOFs[3 * ia0 + 2]};
    double ax[3] = {L.DOFs[3 * iax1] - L.DOFs[3 * iax0], L.DOFs[3 * iax1 + 1] - L.DOFs[3 * iax0 + 1], L.DOFs[3 * iax1 + 2] - L.DOFs[3 * iax0 + 2]};
    scanRotation_ax(n, selection, p0, ax, phi, nstep, Es, trjName);
}

// ------------------------------------------------------------ scalar samplers (libMMFF.h:426-499)
// Energies and forces of single terms along a coordinate, FP64, host side.
void sample_DistConstr(double lmin, double lmax, double kmin, double kmax, double flim, int n, double* xs, double* Es, double* Fs) {
    // DistConstr: harmonic outside [lmin, lmax], force capped at flim
    for (int i = 0; i < n; i++) {
        const double x = std::fabs(xs[i]);
        double E = 0, f = 0;
        if (x > lmax) { const double d = x - lmax; f = -kmax * d; E = 0.5 * kmax * d * d; }
        else if (x < lmin) { const double d = x - lmin; f = -kmin * d; E = 0.5 * kmin * d * d; }
        if (f > flim) f = flim; else if (f < -flim) f = -flim;
        Es[i] = E; Fs[i] = -f * (xs[i] >= 0 ? 1 : -1);
    }
}
void sample_evalPiAling(double k, double ang0, double r1, double r2, int n, double* angles, double* Es, double* Fs) {
    (void)ang0; (void)r1; (void)r2;
    for (int i = 0; i < n; i++) {
        const double a = angles[i];
        // h1 = (1,0,0), h2 = (cos a, sin a, 0): Forces.h evalPiAling
        double c = std::cos(a);
        const double f1y = std::sin(a) * ((c < 0) ? -k : k);
        if (c < 0) c = -c;
        Es[i] = k * (1 - c);
        Fs[i] = f1y;
    }
}
void sample_evalAngleCos(double k, double ang0, double r1, double r2, int n, double* angles, double* Es, double* Fs) {
    const double c0 = std::cos(ang0);
    for (int i = 0; i < n; i++) {
        const double a = angles[i];
        const double c = std::cos(a), c_ = c - c0;
        Es[i] = k * c_ * c_;
        Fs[i] = std::sin(a) * (-k * c_ * 2) / r1;   // f1 = (h2 - h1*c)*fang*ir1, y component
        (void)r2;
    }
}
void sample_evalAngleCosHalf(double k, double ang0, double r1, double r2, int n, double* angles, double* Es, double* Fs) {
    const double cs0x = std::cos(ang0 / 2.), cs0y = std::sin(ang0 / 2.);
    for (int i = 0; i < n; i++) {
        const double a = angles[i];
        const double hx = 1 + std::cos(a), hy = std::sin(a);
        double c2 = (hx * hx + hy * hy) * 0.25;
        const double s2 = 1 - c2 + 1e-14;
        const double c = std::sqrt(c2), s = std::sqrt(s2);
        const double csx = cs0x * c + cs0y * s, csy = cs0y * c - cs0x * s;
        Es[i] = k * (1 - csx);
        double fr = -k * csy;
        c2 *= -2;
        fr /= 4 * c * s;
        const double fr1 = fr / r1;
        Fs[i] = hy * fr1;      // f1.y = h.y*fr1 + h1.y*(fr1*c2), h1.y = 0
        (void)r2;
    }
}
void sampleNonBond(int n, double* rs, double* Es, double* fs, int kind, double* REQi_, double* REQj_, double K, double Rdamp) {
    (void)Rdamp;
    const double R0 = REQi_[0] + REQj_[0], E0 = std::sqrt(REQi_[1] * REQj_[1]), Q = REQi_[2] * REQj_[2];
    for (int i = 0; i < n; i++) {
        const double r = rs[i];
        double E = 0, F = 0;
        if (kind == 1) {   // Morse + Coulomb
            const double e = std::exp(-K * (r - R0));
            E = E0 * (e * e - 2 * e) + 14.3996448915 * Q / r;
            F = E0 * 2 * K * (e * e - e) + 14.3996448915 * Q / (r * r);
        } else {           // Lennard-Jones + Coulomb
            const double u6 = std::pow(R0 / r, 6);
            E = E0 * (u6 * u6 - 2 * u6) + 14.3996448915 * Q / r;
            F = E0 * 12 * (u6 * u6 - u6) / r + 14.3996448915 * Q / (r * r);
        }
        Es[i] = E; fs[i] = F;
    }
}

// GridFF samples of one probe atom (kind >= 10 uses the device B-spline grid
// built by init): along z at (pos0.x, pos0.y), or at arbitrary points
void sampleSurf(char* name, int n, double* rs, double* Es, double* fs, int kind, int atyp, double Q, double K, double RQ, double* pos0_,
                bool bSave) {
    (void)name; (void)atyp; (void)RQ; (void)bSave; (void)kind;
    std::vector<double> P(3 * (size_t)n), PLQ(4 * (size_t)n), fe(4 * (size_t)n);
    const double R0 = kElem[EL_C].R0, sE = std::sqrt(kElem[EL_C].E0);
    const double e = std::exp(K * R0);
    for (int i = 0; i < n; i++) {
        P[3 * i] = pos0_[0]; P[3 * i + 1] = pos0_[1]; P[3 * i + 2] = rs[i];
        PLQ[4 * i] = e * e * sE; PLQ[4 * i + 1] = e * sE; PLQ[4 * i + 2] = Q; PLQ[4 * i + 3] = 0;
    }
    if (mmff_grid_sample(n, P.data(), PLQ.data(), fe.data())) { set_error(std::string("sampleSurf: ") + mmff_last_error()); return; }
    for (int i = 0; i < n; i++) { Es[i] = fe[4 * i + 3]; fs[i] = fe[4 * i + 2]; }
}
void sampleSurf_vecs(char* name, int n, double* poss_, double* Es, double* fs_, int kind, int atyp, double Q, double K, double RQ,
                     double* pos0_, bool bSave) {
    (void)name; (void)atyp; (void)RQ; (void)bSave; (void)kind; (void)pos0_;
    std::vector<double> PLQ(4 * (size_t)n), fe(4 * (size_t)n);
    const double R0 = kElem[EL_C].R0, sE = std::sqrt(kElem[EL_C].E0);
    const double e = std::exp(K * R0);
    for (int i = 0; i < n; i++) { PLQ[4 * i] = e * e * sE; PLQ[4 * i + 1] = e * sE; PLQ[4 * i + 2] = Q; PLQ[4 * i + 3] = 0; }
    if (mmff_grid_sample(n, poss_, PLQ.data(), fe.data())) { set_error(std::string("sampleSurf_vecs: ") + mmff_last_error()); return; }
    for (int i = 0; i < n; i++) { Es[i] = fe[4 * i + 3]; for (int k = 0; k < 3; k++) fs_[3 * i + k] = fe[4 * i + k]; }
}

}  // extern "C"
