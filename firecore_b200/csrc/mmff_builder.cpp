// mmff_builder.cpp -- xyz + FireCore parameter tables -> MMFFsp3_loc arrays.
//
// What the reference computes, step by step (each step cites the reference
// function whose result it reproduces; the code is this project's):
//   tables   MMFFparams::loadElementTypes / loadAtomTypes / loadBondTypes /
//            loadAngleTypes + assignAllSubTypes (MMFFparams.h:230-470, 509-541)
//   read     MMFFparams::loadXYZ + MM::Builder::loadXYZ_Atoms
//            (MMFFparams.h:844-894, MMFFBuilder.h:3725-3760): atoms of unknown
//            type names are skipped; every non-capping atom gets a
//            configuration holding its electron pairs
//   bonds    MM::Builder::autoBonds / autoBondsPBC (MMFFBuilder.h:2087-2160):
//            |r_ij| < f (Ruff_i + Ruff_j), f = 1.20 (1.35 with a cell, 27 images)
//   checks   checkNumberOfBonds (MMFFBuilder.h:2209-2236), which MolWorld_sp3
//            runs by default (bCheckInit)
//   pi / e   autoConfEPi (MMFFBuilder.h:1633-1680): ne from the type,
//            npi = min(4 - nbond - ne, piMax of the element); with electron
//            pairs also setPiLoop / addAllEpairsByPi (:1598-1631, 1691-1735)
//   bondpar  assignBondParams (MMFFBuilder.h:867-893): order 1 + min(npi_i,
//            npi_j), table lookup by type pair, then by element root types,
//            else (2.0, 10.0)
//   order    sortConfAtomsFirst (MMFFBuilder.h:2448-2458): nodes first
//   types    assignTypes (MMFFBuilder.h:1229-1452): root C/N/O -> X_3/X_2/X_1
//            by npi, then the special-type rules iterated to a fixed point
//   arrays   toMMFFsp3_loc (MMFFBuilder.h:4153-4282) with makeConfGeom
//            (:942-1009) for the pi orientation, flipPis (MMFFsp3_loc.h:1167),
//            makeNeighCells (MMFFsp3_loc.h:1394-1430)
//   nonbond  initNBmol + assignREs + chargeToEpairs (MolWorld_sp3.h:1005-1030,
//            1493-1500; MMFFparams.h:775-794; MMFFsp3_loc.h:1575-1590)
// Floating-point expressions keep the reference's operand order, so the
// results agree bit for bit with FireCore's builder on the same inputs.
#include "mmff_builder.h"
#include "mmff_host.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>

namespace fcb {
namespace {

struct V { double x, y, z; };
inline V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V scale(V a, double f) { return {a.x * f, a.y * f, a.z * f}; }
inline double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm2(V a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V unit(V a) { const double inv = 1.0 / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); return {a.x * inv, a.y * inv, a.z * inv}; }
// two vectors orthogonal to a (not normalised), Vec3::getSomeOrtho
inline void some_ortho(V a, V& u, V& w) {
    const double xx = a.x * a.x, yy = a.y * a.y;
    if (xx < yy) u = {-yy - a.z * a.z, a.x * a.y, a.x * a.z};
    else         u = {a.y * a.x, -a.z * a.z - xx, a.y * a.z};
    w = {a.y * u.z - a.z * u.y, a.z * u.x - a.x * u.z, a.x * u.y - a.y * u.x};
}

const double kDeg = 0.01745329251994329547;   // degrees -> radians, FireCore's constant
// direction cosines of the ideal sp3 / sp2 frames (makeConfGeom literals)
const double kS23 = 0.81649658092, kS13 = 0.57735026919, kS29 = 0.47140452079, kM13 = -0.33333333333;
const double kC30 = 0.86602540378;

unsigned long long bond_key(int a, int b, int order) {
    if (a > b) std::swap(a, b);
    return ((unsigned long long)(unsigned)a << 40) | ((unsigned long long)(unsigned)b << 16) | (unsigned)(order & 0xFFFF);
}

bool is_blank(const char* s) {
    for (; *s; s++) if (!isspace((unsigned char)*s)) return false;
    return true;
}

template <class F>
bool each_line(const char* fname, std::string& err, F f) {
    FILE* fp = fopen(fname, "r");
    if (!fp) { err = std::string("cannot open ") + fname; return false; }
    char buf[1024];
    int ln = 0;
    bool ok = true;
    while (ok && fgets(buf, sizeof buf, fp)) {
        ln++;
        if (buf[0] == '#' || is_blank(buf)) continue;
        ok = f(buf, ln);
    }
    fclose(fp);
    return ok;
}

// ---------------------------------------------------------------- builder state
struct Atom {
    int type;
    V pos;
    double REQ[4];
    int conf;          // configuration (node) index or -1 (capping atom)
};
struct Conf {          // counts are bytes in the reference (AtomConf)
    int atom;
    uint8_t n = 0, nbond = 0, npi = 0, ne = 0, nH = 0;
    int bond[4] = {-1, -1, -1, -1};
    V pidir{0, 0, 0};
};
struct Bond { int a, b; double l0, k; };

struct Work {
    const Tables& T;
    std::vector<Atom> atoms;
    std::vector<Conf> confs;
    std::vector<Bond> bonds;
    std::vector<char> capping;   // per type
    std::string& err;
    Work(const Tables& t, std::string& e) : T(t), err(e) {
        capping.assign(T.types.size(), 0);
        for (size_t i = 0; i < T.types.size(); i++) capping[i] = (T.types[i].iZ == 1 || T.types[i].iZ == 200);
    }
    int other(int ib, int ia) const { const Bond& b = bonds[ib]; return b.a == ia ? b.b : (b.b == ia ? b.a : -1); }

    bool conf_add_bond(int ia, int ib) {
        const int c = atoms[ia].conf;
        if (c < 0) return true;
        Conf& C = confs[c];
        if (C.n >= 4) { err = "atom " + std::to_string(ia) + " (" + T.types[atoms[ia].type].name + ") has no free neighbour slot"; return false; }
        C.bond[C.nbond] = ib;
        C.nbond++; C.n++;
        return true;
    }
    bool add_bond(int i, int j, double l0, double k) {
        const int ib = (int)bonds.size();
        bonds.push_back({i, j, l0, k});
        return conf_add_bond(i, ib) && conf_add_bond(j, ib);
    }
    void add_atom(int type, V p, const double REQ[4], bool with_conf, int ne) {
        Atom A{type, p, {REQ[0], REQ[1], REQ[2], REQ[3]}, -1};
        if (with_conf && !capping[type]) {
            Conf C;
            C.atom = (int)atoms.size();
            C.ne = (uint8_t)ne; C.n = C.ne;
            A.conf = (int)confs.size();
            confs.push_back(C);
        }
        atoms.push_back(A);
    }
    // unit vectors to the bonded neighbours, in configuration order
    void bond_dirs(int ia, V* hs) const {
        const Conf& C = confs[atoms[ia].conf];
        for (int k = 0; k < C.nbond; k++) hs[k] = unit(sub(atoms[other(C.bond[k], ia)].pos, atoms[ia].pos));
    }
};

// ideal directions of the free slots (and the pi axis in hs[3]) of a centre
// with nb sigma bonds hs[0..nb) and npi pi orbitals
void ideal_frame(int nb, int npi, V* hs) {
    if (nb == 3) {
        V b = cross(sub(hs[1], hs[0]), sub(hs[2], hs[0]));
        b = scale(b, -1 / std::sqrt(norm2(b)));
        if (npi == 0 && 0 < dot(b, add(add(hs[0], hs[1]), hs[2]))) b = scale(b, -1.);
        hs[3] = b;
    } else if (nb == 2) {
        V a = unit(sub(hs[1], hs[0])), b = cross(hs[0], hs[1]), c;
        const double r2 = norm2(b);
        if (r2 < 1e-15) some_ortho(a, b, c);
        else { b = scale(b, 1 / std::sqrt(r2)); c = cross(b, a); }
        if (npi == 0) { hs[2] = add(scale(c, kS13), scale(b, kS23)); hs[3] = sub(scale(c, kS13), scale(b, kS23)); }
        else          { hs[2] = c; hs[3] = b; }
    } else if (nb == 1 || nb == 0) {
        const V c = unit(hs[0]);
        V b, a;
        some_ortho(c, b, a);
        if (npi == 0) {
            hs[nb] = add(scale(c, kM13), scale(b, kS29 * 2));
            hs[nb + 1] = add(sub(scale(c, kM13), scale(b, kS29)), scale(a, kS23));
            hs[nb + 2] = sub(sub(scale(c, kM13), scale(b, kS29)), scale(a, kS23));
            if (nb == 0) hs[3] = c;
        } else if (nb == 1) {
            if (npi == 1) { hs[1] = add(scale(c, -0.5), scale(a, kC30)); hs[2] = sub(scale(c, -0.5), scale(a, kC30)); hs[3] = b; }
            else          { hs[1] = scale(c, -1); hs[2] = b; hs[3] = a; }
        }
    }
}

}  // namespace

// ------------------------------------------------------------------- tables
bool load_tables(const char* fe, const char* fa, const char* fb, const char* fang, Tables& T, std::string& err) {
    T = Tables();
    bool ok = each_line(fe, err, [&](const char* s, int ln) {
        ElementRow e;
        char name[64];
        unsigned color;
        int iZ, ne, nv, pm;
        double Rcov, RvdW, EvdW, q[7];
        const int n = sscanf(s, "%63s %i %i %i %i %x %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", name, &iZ, &ne, &nv, &pm, &color, &Rcov,
                             &RvdW, &EvdW, q, q + 1, q + 2, q + 3, q + 4, q + 5, q + 6);
        if (n < 12) { err = std::string(fe) + ":" + std::to_string(ln) + ": incomplete element row"; return false; }
        e.name = name; e.iZ = (uint8_t)iZ; e.neval = (uint8_t)ne; e.valence = (uint8_t)nv; e.piMax = (uint8_t)pm;
        e.Rcov = Rcov; e.RvdW = RvdW; e.EvdW = EvdW;
        if (!T.element_index.emplace(e.name, (int)T.elements.size()).second) { err = "duplicate element " + e.name; return false; }
        T.elements.push_back(e);
        return true;
    });
    if (!ok) return false;
    ok = each_line(fa, err, [&](const char* s, int ln) {
        TypeRow t;
        char name[64], par[64], el[64], ep[64];
        int nv, ne, npi, sym;
        double v[11] = {0};
        const int n = sscanf(s, "%63s %63s %63s %63s %i %i %i %i %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", name, par, el, ep, &nv, &ne,
                             &npi, &sym, v, v + 1, v + 2, v + 3, v + 4, v + 5, v + 6, v + 7, v + 8, v + 9, v + 10);
        if (n < 13) { err = std::string(fa) + ":" + std::to_string(ln) + ": incomplete atom-type row"; return false; }
        t.name = name; t.valence = (uint8_t)nv; t.nepair = (uint8_t)ne; t.npi = (uint8_t)npi; t.sym = (uint8_t)sym;
        t.Ruff = v[0]; t.RvdW = v[1]; t.EvdW = v[2]; t.Qbase = v[3]; t.Hb = v[4];
        if (n >= 19) { t.Ass = v[5]; t.Asp = v[6]; t.Kss = v[7]; t.Ksp = v[8]; t.Kep = v[9]; t.Kpp = v[10]; }
        if (!T.types.empty()) {   // the first row is the wildcard root and resolves nothing
            auto ie = T.element_index.find(el);
            const int ip = T.type(par), iep = T.type(ep);
            if (ie == T.element_index.end()) { err = "atom type " + t.name + ": unknown element " + el; return false; }
            if (ip < 0) { err = "atom type " + t.name + ": unknown parent " + par; return false; }
            if (iep < 0) { err = "atom type " + t.name + ": unknown electron-pair type " + ep; return false; }
            t.element = ie->second; t.parent = ip; t.epair = iep; t.iZ = T.elements[ie->second].iZ;
        }
        if (!T.type_index.emplace(t.name, (int)T.types.size()).second) { err = "duplicate atom type " + t.name; return false; }
        T.types.push_back(t);
        return true;
    });
    if (!ok) return false;
    {   // sub-types of the first type of each element: "<name>_3", "_2", "_1"
        std::vector<char> seen(256, 0);
        for (TypeRow& t : T.types) {
            if (seen[t.iZ & 255]) continue;
            seen[t.iZ & 255] = 1;
            const char* suf[3] = {"_3", "_2", "_1"};
            for (int i = 0; i < 3; i++) { const int it = T.type(t.name + suf[i]); if (it >= 0) t.sub[i] = it; }
        }
    }
    ok = each_line(fb, err, [&](const char* s, int ln) {
        char a[64], b[64];
        int order;
        double l0, k;
        if (sscanf(s, "%63s %63s %i %lf %lf", a, b, &order, &l0, &k) < 5) { err = std::string(fb) + ":" + std::to_string(ln) + ": incomplete bond row"; return false; }
        const int ia = T.type(a), ib = T.type(b);
        if (ia < 0 || ib < 0) { err = std::string("bond type ") + a + "-" + b + ": unknown atom type"; return false; }
        if (!T.bonds.emplace(bond_key(ia, ib, order), std::make_pair(l0, k)).second) { err = std::string("duplicate bond type ") + a + "-" + b; return false; }
        return true;
    });
    if (!ok) return false;
    std::unordered_map<std::string, int> angles;
    return each_line(fang, err, [&](const char* s, int ln) {
        char a[64], b[64], c[64];
        double a0, k;
        if (sscanf(s, "%63s %63s %63s %lf %lf", a, b, c, &a0, &k) < 5) { err = std::string(fang) + ":" + std::to_string(ln) + ": incomplete angle row"; return false; }
        int ia = T.type(a), ib = T.type(b), ic = T.type(c);
        if (ia < 0 || ib < 0 || ic < 0) { err = std::string("angle type ") + a + "-" + b + "-" + c + ": unknown atom type"; return false; }
        if (ia > ic) std::swap(ia, ic);
        const std::string key = T.types[ia].name + "-" + T.types[ib].name + "-" + T.types[ic].name;
        if (!angles.emplace(key, 0).second) { err = "duplicate angle type " + key; return false; }
        return true;
    });
}

void substrate_REQ(const Tables& T, const std::string& name, double Q, double H, double REQ[4]) {
    const int it = T.type(name);
    if (it >= 0) { REQ[0] = T.types[it].RvdW; REQ[1] = std::sqrt(T.types[it].EvdW); REQ[2] = Q; REQ[3] = H; }
    else { REQ[0] = 1.5; REQ[1] = 0.0005; REQ[2] = 0; REQ[3] = 0; }   // MMFFparams::default_REQ, used as is
}

// -------------------------------------------------------------------- build
bool build_xyz(const Tables& T, const char* xyz, bool epairs, const int nPBC[3], Built& M, std::string& err) {
    M = Built();
    if (T.types.empty()) { err = "parameter tables not loaded"; return false; }
    Work W(T, err);
    // ---- read
    FILE* fp = fopen(xyz, "r");
    if (!fp) { err = std::string("cannot open ") + xyz; return false; }
    char buf[1024];
    int n = 0;
    if (!fgets(buf, sizeof buf, fp) || sscanf(buf, "%i", &n) != 1 || n <= 0) { fclose(fp); err = std::string(xyz) + ": no atom count"; return false; }
    if (!fgets(buf, sizeof buf, fp)) { fclose(fp); err = std::string(xyz) + ": truncated"; return false; }
    {
        char c[3];
        double L[9];
        if (sscanf(buf, "%c%c%c %lf %lf %lf %lf %lf %lf %lf %lf %lf", c, c + 1, c + 2, L, L + 1, L + 2, L + 3, L + 4, L + 5, L + 6, L + 7,
                   L + 8) == 12 && c[0] == 'l' && c[1] == 'v' && c[2] == 's') {
            M.pbc = true;
            for (int k = 0; k < 9; k++) M.lvec[k] = L[k];
        }
    }
    for (int i = 0; i < n; i++) {
        if (!fgets(buf, sizeof buf, fp)) { fclose(fp); err = std::string(xyz) + ": fewer atoms than the count"; return false; }
        char name[64];
        double x, y, z, Q = 0, H = 0;
        int npi = -1;
        const int r = sscanf(buf, "%63s %lf %lf %lf %lf %lf %i", name, &x, &y, &z, &Q, &H, &npi);
        if (r < 4) { fclose(fp); err = std::string(xyz) + ": incomplete atom line " + std::to_string(i); return false; }
        if (r < 5) Q = 0;
        if (r < 6) H = 0;
        const int it = T.type(name);
        if (it < 0) continue;                            // unknown names are skipped, as in loadXYZ_Atoms
        const TypeRow& t = T.types[it];
        const double REQ[4] = {t.RvdW, std::sqrt(t.EvdW), Q, H};
        W.add_atom(it, V{x, y, z}, REQ, true, (uint8_t)t.nepair);
    }
    fclose(fp);
    const int na0 = (int)W.atoms.size();
    if (na0 == 0) { err = std::string(xyz) + ": no atom of a known type"; return false; }
    const V La{M.lvec[0], M.lvec[1], M.lvec[2]}, Lb{M.lvec[3], M.lvec[4], M.lvec[5]}, Lc{M.lvec[6], M.lvec[7], M.lvec[8]};
    // ---- bonds by touching Ruff spheres
    {
        const double f = M.pbc ? 1.35 : 1.20;
        const int R = M.pbc ? 1 : 0;
        for (int i = 0; i < na0; i++) {
            const Atom& A = W.atoms[i];
            const double Ri = T.types[A.type].Ruff;
            for (int ix = -R; ix <= R; ix++) for (int iy = -R; iy <= R; iy++) for (int iz = -R; iz <= R; iz++) {
                V p = A.pos;
                if (M.pbc) {
                    const V s{La.x * ix + Lb.x * iy + Lc.x * iz, La.y * ix + Lb.y * iy + Lc.y * iz, La.z * ix + Lb.z * iy + Lc.z * iz};
                    p = sub(A.pos, s);
                }
                for (int j = i + 1; j < na0; j++) {
                    const double Rr = (T.types[W.atoms[j].type].Ruff + Ri) * f;
                    if (!(norm2(sub(W.atoms[j].pos, p)) < Rr * Rr)) continue;
                    if (W.capping[A.type] && W.capping[W.atoms[j].type]) continue;
                    if (!W.add_bond(i, j, 1.5, 10.0)) return false;
                }
            }
        }
    }
    // ---- bond-count checks (MolWorld_sp3 runs them by default and stops on failure)
    {
        std::vector<int> nb(na0, 0);
        for (const Bond& b : W.bonds) { nb[b.a]++; nb[b.b]++; }
        for (int i = 0; i < na0; i++) {
            const Atom& A = W.atoms[i];
            const TypeRow& t = T.types[A.type];
            const std::string who = "atom " + std::to_string(i) + " (" + t.name + ")";
            if (nb[i] <= 0) { err = who + " has no bond"; return false; }
            if (A.conf >= 0) {
                if (nb[i] > 4 || nb[i] > t.valence) { err = who + " has " + std::to_string(nb[i]) + " bonds, valence " + std::to_string(t.valence); return false; }
            } else if (nb[i] > 1) { err = who + " is a capping atom with " + std::to_string(nb[i]) + " bonds"; return false; }
        }
    }
    // ---- electron pairs and pi orbitals per node
    for (int ia = 0; ia < na0; ia++) {
        const Atom& A = W.atoms[ia];
        if (A.conf < 0) continue;
        Conf& C = W.confs[A.conf];
        const TypeRow& t = T.types[A.type];
        const uint8_t ne = (uint8_t)t.nepair;
        if (C.nbond + C.nH + ne > 4) { err = "atom " + std::to_string(ia) + " (" + t.name + "): bonds + electron pairs > 4"; return false; }
        C.ne = ne;
        C.npi = (uint8_t)(4 - C.nbond - C.ne - C.nH);
        C.n = 4;
        C.npi = std::min<int>(C.npi, T.elements[t.element].piMax);
        if (C.nbond >= 2) {
            V hs[4];
            W.bond_dirs(ia, hs);
            ideal_frame(C.nbond, C.npi, hs);
            if (C.npi > 0) C.pidir = hs[3];
        }
    }
    if (epairs) {
        // pi axes of nodes with fewer than two bonds from their neighbours (setPiLoop)
        for (int itr = 0; itr < 10; itr++) {
            int changed = 0;
            for (Conf& C : W.confs) {
                if (norm2(C.pidir) > 0.1) continue;
                V p{0, 0, 0};
                for (int i = 0; i < C.nbond; i++) {
                    const int ja = W.other(C.bond[i], C.atom);
                    const int jc = W.atoms[ja].conf;
                    if (jc < 0) continue;
                    V pi = W.confs[jc].pidir;
                    if (i > 0 && dot(p, pi) < 0) pi = scale(pi, -1.);
                    p = add(p, pi);
                }
                const double r = std::sqrt(norm2(p));
                if (r < 1e-6) continue;
                C.pidir = scale(p, 1. / r);
                changed++;
            }
            if (!changed) break;
        }
        // explicit electron pairs on terminal pi atoms (=O, #N), addAllEpairsByPi
        for (int ia = 0; ia < na0; ia++) {
            const int c = W.atoms[ia].conf;
            if (c < 0) continue;
            Conf& C = W.confs[c];
            const int ne = C.ne;
            if (ne < 1 || C.nbond > 1 || C.npi < 1) continue;
            if (C.nbond < 1) { err = "atom " + std::to_string(ia) + ": electron pairs need one bond"; return false; }
            C.ne = 0;
            C.n = (uint8_t)(C.n - ne);
            V hs[4];
            W.bond_dirs(ia, hs);
            V lf = unit(cross(C.pidir, hs[0]));
            if (C.npi == 1) { hs[1] = add(scale(lf, +kC30), scale(hs[0], -0.5)); hs[2] = add(scale(lf, -kC30), scale(hs[0], -0.5)); }
            else            { hs[1] = scale(hs[0], -1.0); }
            if (ne > 2 || (C.npi != 1 && ne > 1)) { err = "atom " + std::to_string(ia) + ": electron-pair geometry undefined"; return false; }
            const int et = T.types[W.atoms[ia].type].epair;
            const double l = T.types[et].Ruff;
            for (int i = 0; i < ne; i++) {
                const double REQ[4] = {1.4870, 0.026095977, 0., 0.};   // the builder's capping-atom template
                W.add_atom(et, add(W.atoms[ia].pos, scale(hs[1 + i], l)), REQ, false, 0);
                if (!W.add_bond(ia, (int)W.atoms.size() - 1, 1.07, 100 / 16.02176634)) return false;
            }
        }
    }
    // ---- bond parameters from the (input) types and bond orders
    for (Bond& b : W.bonds) {
        const Atom &ai = W.atoms[b.a], &aj = W.atoms[b.b];
        int order = 1;
        if (ai.conf >= 0 && aj.conf >= 0) order += std::min(W.confs[ai.conf].npi, W.confs[aj.conf].npi);
        auto it = T.bonds.find(bond_key(ai.type, aj.type, order));
        if (it == T.bonds.end()) {
            const int ei = T.type(T.elements[T.types[ai.type].element].name), ej = T.type(T.elements[T.types[aj.type].element].name);
            if (ei >= 0 && ej >= 0) it = T.bonds.find(bond_key(ei, ej, order));
        }
        if (it != T.bonds.end()) { b.l0 = it->second.first; b.k = it->second.second; }
        else { b.l0 = 2.0; b.k = 10.0; }
    }
    // ---- nodes first
    const int nA = (int)W.atoms.size(), nC = (int)W.confs.size();
    {
        std::vector<int> perm(nA);
        int j = 0;
        for (int i = 0; i < nA; i++) if (W.atoms[i].conf >= 0) perm[i] = j++;
        for (int i = 0; i < nA; i++) if (W.atoms[i].conf < 0) perm[i] = j++;
        std::vector<Atom> old(W.atoms);
        for (int i = 0; i < nA; i++) {
            W.atoms[perm[i]] = old[i];
            if (old[i].conf >= 0) W.confs[old[i].conf].atom = perm[i];
        }
        for (Bond& b : W.bonds) { b.a = perm[b.a]; b.b = perm[b.b]; if (b.a > b.b) std::swap(b.a, b.b); }
        M.permut = perm;                       // Builder::setup_atom_permut
    }
    // ---- atom types: hybridisation sub-types, then the special-type rules
    {
        const int iC = T.type("C"), iN = T.type("N"), iO = T.type("O");
        if (iC < 0 || iN < 0 || iO < 0) { err = "atom types C, N, O missing from the table"; return false; }
        for (Atom& A : W.atoms) {
            if (T.types[A.type].parent != 0 || A.conf < 0) continue;
            if (A.type != iC && A.type != iN && A.type != iO) continue;
            A.type = T.types[A.type].sub[W.confs[A.conf].npi];
        }
        std::vector<int> ng(4 * (size_t)nA, -1);
        for (int ia = 0; ia < nA; ia++) {
            const int c = W.atoms[ia].conf;
            if (c < 0) continue;
            for (int k = 0; k < W.confs[c].nbond; k++) {
                const int ja = W.other(W.confs[c].bond[k], ia);
                ng[4 * ia + k] = ja;
                if (W.atoms[ja].conf < 0) ng[4 * ja] = ia;
            }
        }
        const char* names[] = {"C_3", "C_2", "C_1", "C_R", "C_ene", "C_yne", "C_CH3", "C_ald", "C_COO", "O", "O_3", "O_2", "O_1", "O_R",
                               "O_OH", "O_ald", "O_sCOO", "O_pCOO", "N", "N_3", "N_2", "N_1", "N_R", "H", "H_OH", "H_COO", "H_NH2",
                               "H_CH3", "H_ene", "H_yne", "H_ald"};
        std::unordered_map<std::string, int> ix;
        for (const char* s : names) {
            const int it = T.type(s);
            if (it < 0) { err = std::string("atom type ") + s + " missing from the table"; return false; }
            ix[s] = it;
        }
        // (neighbour type -> hydrogen type) pairs, tried in this order
        const std::pair<const char*, const char*> hcap[] = {{"O_OH", "H_OH"}, {"N_3", "H_NH2"}, {"N_R", "H_NH2"}, {"C_3", "H_CH3"},
                                                            {"C_CH3", "H_CH3"}, {"C_2", "H_ene"}, {"C_R", "H_ene"}, {"C_ene", "H_ene"},
                                                            {"C_yne", "H_yne"}, {"C_ald", "H_ald"}};
        auto nb_count = [&](int ia, int type) {
            int c = 0;
            for (int k = 0; k < 4; k++) { const int ja = ng[4 * ia + k]; if (ja >= 0 && W.atoms[ja].type == type) c++; }
            return c;
        };
        int itr = 0;
        for (; itr < 10; itr++) {
            int changed = 0;
            for (int ia = 0; ia < nA; ia++) {
                Atom& A = W.atoms[ia];
                const int iZ = T.types[A.type].iZ;
                int pin = 0;                    // bonded neighbours with pi orbitals
                if (A.conf >= 0)
                    for (int k = 0; k < 4; k++) {
                        const int ja = ng[4 * ia + k];
                        if (ja >= 0 && W.atoms[ja].conf >= 0 && W.confs[W.atoms[ja].conf].npi) pin++;
                    }
                int nt = A.type;
                if (iZ == 1) {
                    const int ja = ng[4 * ia];
                    if (ja >= 0 && ja <= nA) {
                        const int jt = W.atoms[ja].type;
                        for (const auto& r : hcap) if (jt == ix[r.first]) { nt = ix[r.second]; break; }
                    }
                } else if (iZ == 6) {
                    if (A.type == ix["C_2"]) {
                        const bool o3 = nb_count(ia, ix["O_3"]) > 0, o2 = nb_count(ia, ix["O_2"]) > 0;
                        if (o3 && o2) nt = ix["C_COO"];
                        else if (o2) nt = ix["C_ald"];
                        else if (pin >= 2) nt = ix["C_R"];
                    }
                } else if (iZ == 7) {
                    if (A.type == ix["N_3"] && pin >= 1) nt = ix["N_R"];
                } else if (iZ == 8) {
                    if (A.conf >= 0 && nb_count(ia, ix["C_COO"]) > 0) {
                        if (A.type == ix["O_3"]) nt = ix["O_sCOO"];
                        else if (A.type == ix["O_2"]) nt = ix["O_pCOO"];
                    } else if (A.conf >= 0 && nb_count(ia, ix["C_ald"]) > 0) nt = ix["O_ald"];
                }
                if (nt >= 0 && nt != A.type) { A.type = nt; changed++; }
            }
            if (!changed) break;
        }
        if (itr == 10) { err = "atom-type rules did not settle in 10 passes"; return false; }
    }
    // ---- MMFFsp3_loc arrays
    int ne_tot = 0;
    if (epairs) for (const Conf& C : W.confs) ne_tot += C.ne;
    const int natoms = nA + ne_tot, nnode = nC;
    M.natoms = natoms; M.nnode = nnode;
    M.pos.assign(3 * (size_t)(natoms + nnode), 0.0);
    M.REQ.assign(4 * (size_t)natoms, 0.0);
    M.type.assign(natoms, -1);
    M.neighs.assign(4 * (size_t)natoms, -1);
    M.neighCell.assign(4 * (size_t)natoms, -1);
    M.apars.assign(4 * (size_t)nnode, 0.0); M.bLs = M.apars; M.bKs = M.apars; M.Ksp = M.apars; M.Kpp = M.apars;
    const int etype = T.type("E");
    std::vector<V> P(natoms + nnode, V{0, 0, 0});
    int ie = nA;
    for (int ia = 0; ia < nA; ia++) {
        const Atom& A = W.atoms[ia];
        P[ia] = A.pos;
        M.type[ia] = A.type;
        for (int k = 0; k < 4; k++) M.REQ[4 * ia + k] = A.REQ[k];
        if (A.conf < 0) continue;
        const Conf& C = W.confs[A.conf];
        const TypeRow& t = T.types[A.type];
        if (C.npi > 2) { err = "atom " + std::to_string(ia) + ": more than 2 pi orbitals"; return false; }
        const double a0 = t.Ass * kDeg * 0.5;
        double* ap = &M.apars[4 * ia];
        ap[0] = std::cos(a0); ap[1] = std::sin(a0); ap[2] = t.Kss * 4.0; ap[3] = std::sin(t.Asp * kDeg);
        V hs[4];
        for (int k = 0; k < C.nbond; k++) {
            const Bond& B = W.bonds[C.bond[k]];
            const int ja = W.other(C.bond[k], ia);
            hs[k] = unit(sub(W.atoms[ja].pos, A.pos));
            M.neighs[4 * ia + k] = ja;
            M.bLs[4 * ia + k] = B.l0;
            M.bKs[4 * ia + k] = B.k;
            M.Ksp[4 * ia + k] = (C.npi > 0 || C.ne > 0) ? t.Ksp : 0;
            M.Kpp[4 * ia + k] = std::sqrt(t.Kpp * T.types[W.atoms[ja].type].Kpp);
        }
        if (C.nbond < 1) { err = "atom " + std::to_string(ia) + " has no bond"; return false; }
        ideal_frame(C.nbond, C.npi, hs);
        if (epairs)
            for (int k = C.nbond; k < C.nbond + C.ne; k++) {
                M.neighs[4 * ia + k] = ie;
                P[ie] = add(A.pos, scale(hs[k], 0.5));
                M.type[ie] = etype;
                M.bKs[4 * ia + k] = 10.0;
                M.bLs[4 * ia + k] = 0.5;
                M.Ksp[4 * ia + k] = C.npi > 0 ? t.Ksp : 0;
                ie++;
            }
        P[natoms + ia] = hs[3];
    }
    // capping atoms point back at their node (makeBackNeighs)
    {
        std::vector<int> back(natoms, -1);
        std::vector<int> nback(natoms, 0);
        for (int ia = 0; ia < nnode; ia++)
            for (int k = 0; k < 4; k++) {
                const int ja = M.neighs[4 * ia + k];
                if (ja < 0) continue;
                if (nback[ja]++ == 0) back[ja] = ia;
                if (nback[ja] > 4) { err = "atom " + std::to_string(ja) + " has more than 4 back-neighbours"; return false; }
            }
        for (int ia = nnode; ia < natoms; ia++) {
            if (back[ia] < 0) { err = "capping atom " + std::to_string(ia) + " has no node"; return false; }
            M.neighs[4 * ia] = back[ia];
        }
    }
    for (int ia = 0; ia < nnode; ia++) {   // pi orientations towards (1,1,1), then unit length
        V& p = P[natoms + ia];             // (flipPis; normalizePis of the first evaluation)
        if (p.x * 1 + p.y * 1 + p.z * 1 < 0) p = scale(p, -1);
        p = unit(p);
    }
    if (M.pbc) {   // nearest image of each bond partner (single-precision distances)
        std::vector<V> shifts;
        for (int iz = -nPBC[2]; iz <= nPBC[2]; iz++) for (int iy = -nPBC[1]; iy <= nPBC[1]; iy++) for (int ix = -nPBC[0]; ix <= nPBC[0]; ix++)
            shifts.push_back(add(add(scale(La, ix), scale(Lb, iy)), scale(Lc, iz)));
        for (int ia = 0; ia < natoms; ia++)
            for (int k = 0; k < 4; k++) {
                const int ja = M.neighs[4 * ia + k];
                if (ja < 0) continue;
                const V d = sub(P[ja], P[ia]);
                int imin = -1;
                float r2min = std::numeric_limits<float>::infinity();
                for (size_t s = 0; s < shifts.size(); s++) {
                    const float r2 = (float)norm2(add(shifts[s], d));
                    if (r2 < r2min) { r2min = r2; imin = (int)s; }
                }
                M.neighCell[4 * ia + k] = imin;
            }
    }
    // non-bonded parameters of the final types; charges onto electron pairs
    for (int ia = 0; ia < natoms; ia++) {
        if (ia >= nA) M.REQ[4 * ia + 2] = 0;
        const TypeRow& t = T.types[M.type[ia]];
        M.REQ[4 * ia] = t.RvdW; M.REQ[4 * ia + 1] = std::sqrt(t.EvdW); M.REQ[4 * ia + 3] = 0;
    }
    for (int ia = 0; ia < nnode; ia++)
        for (int k = 0; k < 4; k++) {
            const int ja = M.neighs[4 * ia + k];
            if (ja >= 0 && M.type[ja] == etype) { M.REQ[4 * ja + 2] += -0.2; M.REQ[4 * ia + 2] -= -0.2; }
        }
    for (int i = 0; i < natoms + nnode; i++) { M.pos[3 * i] = P[i].x; M.pos[3 * i + 1] = P[i].y; M.pos[3 * i + 2] = P[i].z; }
    return true;
}

}  // namespace fcb

// ------------------------------------------------------------------- C-ABI
extern "C" {

// Tables + xyz -> MMFFsp3_loc arrays on the host (no device work).  Arrays are
// the caller's, sized for cap atoms: apos [2*cap*3] (natoms + nnode rows: atoms,
// then pi orientations), REQs / neighs / neighCell [cap*4], atypes [cap],
// apars / bLs / bKs / Ksp / Kpp [cap*4] (nnode rows), type_names [cap*8]
// (NUL-padded).  counts[4] = natoms, nnode, natoms + nnode, pbc.  Returns
// natoms, -1 on an error (message in mmff_last_error), -2 if cap is too small.
int mmff_build_xyz(const char* fElem, const char* fAtom, const char* fBond, const char* fAngle, const char* xyz, int bEpairs,
                   const int* nPBC, int cap, int* counts, double* apos, double* REQs, int* atypes, int* neighs, int* neighCell,
                   double* apars, double* bLs, double* bKs, double* Ksp, double* Kpp, char* type_names) {
    fcb::Tables T;
    fcb::Built M;
    std::string err;
    const int np[3] = {nPBC ? nPBC[0] : 1, nPBC ? nPBC[1] : 1, nPBC ? nPBC[2] : 0};
    if (!fElem || !fAtom || !fBond || !fAngle || !xyz) { mmff_set_error("mmff_build_xyz: null file name"); return -1; }
    if (!fcb::load_tables(fElem, fAtom, fBond, fAngle, T, err) || !fcb::build_xyz(T, xyz, bEpairs != 0, np, M, err)) {
        mmff_set_error(("mmff_build_xyz: " + err).c_str());
        return -1;
    }
    if (M.natoms > cap) { mmff_set_error("mmff_build_xyz: capacity too small"); return -2; }
    if (counts) { counts[0] = M.natoms; counts[1] = M.nnode; counts[2] = M.natoms + M.nnode; counts[3] = M.pbc; }
    if (apos) std::copy(M.pos.begin(), M.pos.end(), apos);
    if (REQs) std::copy(M.REQ.begin(), M.REQ.end(), REQs);
    if (atypes) std::copy(M.type.begin(), M.type.end(), atypes);
    if (neighs) std::copy(M.neighs.begin(), M.neighs.end(), neighs);
    if (neighCell) std::copy(M.neighCell.begin(), M.neighCell.end(), neighCell);
    if (apars) std::copy(M.apars.begin(), M.apars.end(), apars);
    if (bLs) std::copy(M.bLs.begin(), M.bLs.end(), bLs);
    if (bKs) std::copy(M.bKs.begin(), M.bKs.end(), bKs);
    if (Ksp) std::copy(M.Ksp.begin(), M.Ksp.end(), Ksp);
    if (Kpp) std::copy(M.Kpp.begin(), M.Kpp.end(), Kpp);
    if (type_names)
        for (int i = 0; i < M.natoms; i++) {
            memset(type_names + 8 * i, 0, 8);
            strncpy(type_names + 8 * i, T.types[M.type[i]].name.c_str(), 7);
        }
    return M.natoms;
}
}
