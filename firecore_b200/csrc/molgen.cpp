// molgen.cpp -- seeded synthetic workloads for the multi-system MMFF relaxer.
//
// Generates MMFFsp3_loc topologies and parameters directly (the reference gets
// them from MM::Builder::toMMFFsp3_loc, cpp/common/molecular/MMFFBuilder.h:4153,
// reading AtomTypes.dat / BondTypes.dat).  This generator writes arrays with
// the same meaning and layout as toMMFFsp3_loc produces:
//   neighs[ia]   : up to 4 bonded atoms of node ia, -1 padded; caps get
//                  neighs.x = their node (MMFFsp3_loc::makeBackNeighs, bCapNeighs)
//   bkneighs[ia] : ia*4+j back references into node recoil slots
//   apars[ia]    : (cos(a0/2), sin(a0/2), 4*Kss, sin(Asp))
//   bLs/bKs      : per-slot rest length / stiffness
//   Ksp          : per-slot pi-sigma stiffness (only for nodes with pi orbitals)
//   Kpp          : per-slot sqrt(Kpp_i*Kpp_j)
//   REQs         : (R0, sqrt(E0), Q, Hb)
// Parameter values are this project's own table (element x hybridisation),
// chosen in the magnitude ranges of MMFF/UFF; they are inputs to the relaxer,
// not a reproduction of FireCore's parameter files.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <array>
#include <unordered_map>
#include "mmff_host.h"

namespace {

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t& x) {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) { uint64_t x = seed; for (int i = 0; i < 4; i++) s[i] = splitmix(x); }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256**
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    int below(int n) { return (int)(uni() * n); }
    double gauss() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct V3 { double x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double f) { return {a.x * f, a.y * f, a.z * f}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 unit(V3 a) { double l = norm(a); return a * (1.0 / l); }
inline V3 any_perp(V3 u) {
    V3 t = std::fabs(u.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0};
    return unit(cross(u, t));
}

// element codes
enum { EL_H = 0, EL_C = 1, EL_N = 2, EL_O = 3 };
const int kValence[4] = {1, 4, 3, 2};
// non-bonded parameters per element: R0 [A], E0 [eV]
const double kR0[4] = {1.50, 1.90, 1.80, 1.75};
const double kE0[4] = {0.0020, 0.0046, 0.0030, 0.0026};
// angle stiffness Kss [eV/rad^2] per element, and sp3 rest angle [deg]
const double kKss[4] = {0.0, 5.0, 5.5, 6.0};
const double kSp3Ang[4] = {0.0, 109.47, 107.0, 105.0};
// pi-pi stiffness per element for sp2 / sp atoms
const double kKppSp2[4] = {0.0, 1.5, 1.0, 0.5};
const double kKsp = 1.6;

inline double bond_k(int ea, int eb) {
    if (ea == EL_H || eb == EL_H) return 20.0;
    static const double t[4][4] = {{0, 0, 0, 0}, {0, 25.0, 27.0, 28.0}, {0, 27.0, 26.0, 27.5}, {0, 28.0, 27.5, 26.0}};
    return t[ea][eb];
}
inline double bond_l0(int ea, int eb) {
    if (ea == EL_H || eb == EL_H) return 1.09;
    static const double t[4][4] = {{0, 0, 0, 0}, {0, 1.40, 1.38, 1.37}, {0, 1.38, 1.36, 1.35}, {0, 1.37, 1.35, 1.40}};
    return t[ea][eb];
}

// ideal bond directions for n neighbours (first one along +z before rotation)
void ideal_dirs(int n, double ang_deg, V3* d) {
    const double a = ang_deg * M_PI / 180.0;
    d[0] = {0, 0, 1};
    if (n == 2) { d[1] = {std::sin(a), 0, std::cos(a)}; return; }
    if (n == 3) {
        // planar if ang==120, otherwise pyramidal with the given inter-bond angle
        double ca = std::cos(a);
        // bonds 1,2 at polar angle a from d0, azimuths 0 and phi with cos between them = ca
        double st = std::sin(a), ct = std::cos(a);
        double cphi = (ca - ct * ct) / (st * st);
        cphi = std::max(-1.0, std::min(1.0, cphi));
        double phi = std::acos(cphi);
        d[1] = {st, 0, ct};
        d[2] = {st * std::cos(phi), st * std::sin(phi), ct};
        return;
    }
    if (n == 4) {
        double st = std::sin(a), ct = std::cos(a);
        for (int k = 0; k < 3; k++) {
            double ph = 2.0 * M_PI * k / 3.0;
            d[1 + k] = {st * std::cos(ph), st * std::sin(ph), ct};
        }
    }
}

// rotate vector v from local frame (z axis = u, x axis = w) to global
inline V3 to_frame(V3 v, V3 u, V3 w) {
    V3 y = cross(u, w);
    return w * v.x + y * v.y + u * v.z;
}

struct Mol {
    int natoms = 0, nnode = 0;
    std::vector<int> el;          // [natoms]
    std::vector<V3> pos;          // [natoms + nnode] (atoms, then pi vectors)
    std::vector<int> neighs;      // [natoms*4]
    std::vector<double> REQ;      // [natoms*4]
    std::vector<double> apars, bLs, bKs, Ksp, Kpp;  // [nnode*4]
};

// heavy-atom composition for N atoms with C:N:O:H = 10:2:2:10
void composition(int N, int& nC, int& nN, int& nO, int& nH) {
    int nh = (int)std::lround(N * 14.0 / 24.0);
    if (nh < 1) nh = 1;
    if (nh > N) nh = N;
    nH = N - nh;
    nN = (int)std::lround(nh * 2.0 / 14.0);
    nO = (int)std::lround(nh * 2.0 / 14.0);
    nC = nh - nN - nO;
    if (nC < 1) { nC = 1; nN = std::max(0, nh - 1 - nO); nO = nh - nC - nN; }
}

// Heavy-atom tree grown on a diamond lattice (bond 1.40 A): every site has four
// tetrahedral neighbour directions, so bond angles start at 109.47 deg and all
// torsions are staggered.  A site is occupied only if exactly one of its lattice
// neighbours is occupied (its parent), so every lattice-adjacent pair is a bond
// and every 2.29 A pair is a true 1-3 pair.  Hydrogens point into empty sites
// that touch no other heavy atom and no other hydrogen.
bool build_mol(int N, Rng& rng, Mol& M, bool hbond) {
    int nC, nN, nO, nH;
    composition(N, nC, nN, nO, nH);
    const int nh = nC + nN + nO;
    std::vector<int> hel;
    for (int i = 0; i < nC; i++) hel.push_back(EL_C);
    for (int i = 0; i < nN; i++) hel.push_back(EL_N);
    for (int i = 0; i < nO; i++) hel.push_back(EL_O);
    for (int i = nh - 1; i > 1; i--) { int j = 1 + rng.below(i); std::swap(hel[i], hel[j]); }
    M.natoms = N; M.nnode = nh;
    M.el.assign(N, EL_H);
    for (int i = 0; i < nh; i++) M.el[i] = hel[i];
    M.pos.assign(N + nh, V3{0, 0, 0});
    std::vector<std::vector<int>> nb(N);
    // lattice bookkeeping
    struct Site { int x, y, z; };
    auto key = [](int x, int y, int z) -> uint64_t {
        return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) | (uint64_t)(uint32_t)(z + (1 << 20));
    };
    std::unordered_map<uint64_t, int> occ;      // site -> heavy atom
    std::unordered_map<uint64_t, int> hclaim;   // site claimed by a hydrogen
    std::vector<Site> site(nh);
    auto dirs = [](const Site& s, int k, int& dx, int& dy, int& dz) {
        static const int D[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
        int sg = ((s.x & 1) == 0) ? 1 : -1;   // sublattice A (even) / B (odd)
        dx = sg * D[k][0]; dy = sg * D[k][1]; dz = sg * D[k][2];
    };
    auto n_occ_neigh = [&](int x, int y, int z, int skip) {
        Site t{x, y, z};
        int n = 0;
        for (int k = 0; k < 4; k++) {
            int dx, dy, dz; dirs(t, k, dx, dy, dz);
            auto it = occ.find(key(x + dx, y + dy, z + dz));
            if (it != occ.end() && it->second != skip) n++;
        }
        return n;
    };
    // hydrogen targets per heavy atom (C <= 2, N, O <= 1), summing to nH
    std::vector<int> hcount(nh, 0);
    {
        std::vector<int> slots;
        for (int i = 0; i < nh; i++) for (int k = 0; k < (hel[i] == EL_C ? 2 : 1); k++) slots.push_back(i);
        if ((int)slots.size() < nH) return false;
        for (int k = (int)slots.size() - 1; k > 0; k--) { int j = rng.below(k + 1); std::swap(slots[k], slots[j]); }
        for (int k = 0; k < nH; k++) hcount[slots[k]]++;
    }
    // Hydrogens are claimed as soon as their heavy atom is placed: a hydrogen
    // site is an empty lattice site touching only its own heavy atom, with no
    // other hydrogen site next to it; heavy atoms never move next to a claimed
    // hydrogen site.
    std::vector<std::vector<int>> hsites(nh);   // lattice direction index per H
    auto hsite_ok = [&](int x, int y, int z, int owner) {
        uint64_t k2 = key(x, y, z);
        if (occ.count(k2) || hclaim.count(k2)) return false;
        if (n_occ_neigh(x, y, z, owner) != 0) return false;
        Site t{x, y, z};
        for (int q = 0; q < 4; q++) {
            int ex, ey, ez; dirs(t, q, ex, ey, ez);
            if (hclaim.count(key(x + ex, y + ey, z + ez))) return false;
        }
        return true;
    };
    auto claim_H = [&](int a) {
        int want = hcount[a];
        int order[4] = {0, 1, 2, 3};
        for (int k = 3; k > 0; k--) { int j = rng.below(k + 1); std::swap(order[k], order[j]); }
        std::vector<uint64_t> got;
        std::vector<int> gotk;
        for (int kk = 0; kk < 4 && (int)got.size() < want; kk++) {
            int dx, dy, dz; dirs(site[a], order[kk], dx, dy, dz);
            int x = site[a].x + dx, y = site[a].y + dy, z = site[a].z + dz;
            if (!hsite_ok(x, y, z, a)) continue;
            hclaim[key(x, y, z)] = a;
            got.push_back(key(x, y, z)); gotk.push_back(order[kk]);
        }
        if ((int)got.size() < want) { for (auto g : got) hclaim.erase(g); return false; }
        hsites[a] = gotk;
        return true;
    };
    site[0] = {0, 0, 0};
    occ[key(0, 0, 0)] = 0;
    if (!claim_H(0)) return false;
    std::vector<int> hdeg(nh, 0);
    for (int i = 1; i < nh; i++) {
        bool ok = false;
        for (int attempt = 0; attempt < 4000 && !ok; attempt++) {
            // parent: the one nearest the lattice origin of three random picks
            // (keeps big molecules globular); plain random after many failures
            int p = rng.below(i);
            if (attempt < 2000) {
                for (int t = 0; t < 2; t++) {
                    int c = rng.below(i);
                    long rc = (long)site[c].x * site[c].x + (long)site[c].y * site[c].y + (long)site[c].z * site[c].z;
                    long rp = (long)site[p].x * site[p].x + (long)site[p].y * site[p].y + (long)site[p].z * site[p].z;
                    if (rc < rp) p = c;
                }
            }
            if (hdeg[p] + hcount[p] >= kValence[hel[p]]) continue;
            int k = rng.below(4), dx, dy, dz;
            dirs(site[p], k, dx, dy, dz);
            int x = site[p].x + dx, y = site[p].y + dy, z = site[p].z + dz;
            uint64_t kx = key(x, y, z);
            if (occ.count(kx) || hclaim.count(kx)) continue;
            if (n_occ_neigh(x, y, z, p) != 0) continue;   // would close a ring / non-bonded contact
            {   // no foreign hydrogen site next to the new heavy atom
                bool bad = false;
                Site t{x, y, z};
                for (int q = 0; q < 4 && !bad; q++) {
                    int ex, ey, ez; dirs(t, q, ex, ey, ez);
                    auto it = hclaim.find(key(x + ex, y + ey, z + ez));
                    if (it != hclaim.end()) bad = true;
                }
                if (bad) continue;
            }
            if (1 + hcount[i] > kValence[hel[i]]) continue;
            site[i] = {x, y, z};
            occ[kx] = i;
            if (!claim_H(i)) { occ.erase(kx); continue; }
            hdeg[p]++; hdeg[i]++;
            nb[p].push_back(i); nb[i].insert(nb[i].begin(), p);
            ok = true;
        }
        if (!ok) return false;
    }
    int ih = nh;
    for (int a = 0; a < nh; a++) {
        for (int k : hsites[a]) {
            int dx, dy, dz; dirs(site[a], k, dx, dy, dz);
            nb[a].push_back(ih); nb[ih].push_back(a);
            M.pos[ih] = V3{(double)dx, (double)dy, (double)dz};   // direction, scaled below
            ih++;
        }
    }
    if (ih != N) return false;
    // 3) coordinates: lattice unit so that bonds are 1.40 A, +-0.05 A jitter
    const double u = 1.40 / std::sqrt(3.0);
    for (int i = 0; i < nh; i++) {
        M.pos[i] = V3{site[i].x * u, site[i].y * u, site[i].z * u} +
                   V3{0.029 * (2 * rng.uni() - 1), 0.029 * (2 * rng.uni() - 1), 0.029 * (2 * rng.uni() - 1)};
    }
    for (int h = nh; h < N; h++) {
        int a = nb[h][0];
        M.pos[h] = M.pos[a] + unit(M.pos[h]) * 1.09;
    }
    // hybridisation
    std::vector<int> npi(nh), nbt(nh);
    for (int i = 0; i < nh; i++) {
        nbt[i] = (int)nb[i].size();
        npi[i] = kValence[hel[i]] - nbt[i];
        if (hel[i] == EL_C && nbt[i] <= 2) npi[i] = 2;
    }
    // rest angles: sp3 per element, 120 deg for every atom with a pi orbital.
    // Linear (180 deg) centres are never generated: evalAngleCosHalf divides by
    // cos(theta/2), which vanishes at 180 deg.
    auto rest_angle = [&](int i) {
        if (npi[i] >= 1) return 120.0;
        return kSp3Ang[hel[i]];
    };
    // pi orientations
    for (int i = 0; i < nh; i++) {
        int n = nbt[i];
        V3 p;
        if (npi[i] == 1 && n >= 2) {
            p = cross(M.pos[nb[i][0]] - M.pos[i], M.pos[nb[i][1]] - M.pos[i]);
            if (norm(p) < 1e-6) p = any_perp(unit(M.pos[nb[i][0]] - M.pos[i]));
        } else if (n >= 1) {
            p = any_perp(unit(M.pos[nb[i][0]] - M.pos[i]));
        } else {
            p = {0, 0, 1};
        }
        M.pos[N + i] = unit(p);
    }
    // parameters
    M.neighs.assign(N * 4, -1);
    M.REQ.assign(N * 4, 0.0);
    M.apars.assign(nh * 4, 0.0); M.bLs.assign(nh * 4, 0.0); M.bKs.assign(nh * 4, 0.0);
    M.Ksp.assign(nh * 4, 0.0); M.Kpp.assign(nh * 4, 0.0);
    std::vector<double> kpp_at(N, 0.0);
    for (int i = 0; i < nh; i++) if (npi[i] > 0) kpp_at[i] = kKppSp2[hel[i]];
    for (int i = 0; i < nh; i++) {
        double a0 = rest_angle(i) * M_PI / 180.0 * 0.5;
        M.apars[4 * i + 0] = std::cos(a0);
        M.apars[4 * i + 1] = std::sin(a0);
        M.apars[4 * i + 2] = kKss[hel[i]] * 4.0;
        M.apars[4 * i + 3] = 0.0;      // sin(Asp) with Asp = 0: pi orthogonal to sigma
        for (int k = 0; k < nbt[i] && k < 4; k++) {
            int j = nb[i][k];
            M.neighs[4 * i + k] = j;
            M.bLs[4 * i + k] = bond_l0(M.el[i], M.el[j]);
            M.bKs[4 * i + k] = bond_k(M.el[i], M.el[j]);
            M.Ksp[4 * i + k] = (npi[i] > 0) ? kKsp : 0.0;
            M.Kpp[4 * i + k] = std::sqrt(kpp_at[i] * kpp_at[j]);
        }
    }
    for (int i = nh; i < N; i++) M.neighs[4 * i] = nb[i][0];
    double qsum = 0;
    std::vector<double> q(N);
    for (int i = 0; i < N; i++) { q[i] = 0.2 * rng.gauss(); qsum += q[i]; }
    for (int i = 0; i < N; i++) q[i] -= qsum / N;
    for (int i = 0; i < N; i++) {
        int e = M.el[i];
        M.REQ[4 * i + 0] = kR0[e];
        M.REQ[4 * i + 1] = std::sqrt(kE0[e]);
        M.REQ[4 * i + 2] = q[i];
        double hb = 0.0;
        if (hbond) {
            if (e == EL_N || e == EL_O) hb = -0.7;
            if (e == EL_H) { int p = nb[i][0]; if (M.el[p] == EL_N || M.el[p] == EL_O) hb = 0.7; }
        }
        M.REQ[4 * i + 3] = hb;
    }
    return true;
}

// uniform random rotation (quaternion from three uniforms)
void random_rotation(Rng& rng, double R[9]) {
    double u1 = rng.uni(), u2 = rng.uni(), u3 = rng.uni();
    double a = std::sqrt(1 - u1), b = std::sqrt(u1);
    double qx = a * std::sin(2 * M_PI * u2), qy = a * std::cos(2 * M_PI * u2);
    double qz = b * std::sin(2 * M_PI * u3), qw = b * std::cos(2 * M_PI * u3);
    R[0] = 1 - 2 * (qy * qy + qz * qz); R[1] = 2 * (qx * qy - qz * qw);     R[2] = 2 * (qx * qz + qy * qw);
    R[3] = 2 * (qx * qy + qz * qw);     R[4] = 1 - 2 * (qx * qx + qz * qz); R[5] = 2 * (qy * qz - qx * qw);
    R[6] = 2 * (qx * qz - qy * qw);     R[7] = 2 * (qy * qz + qx * qw);     R[8] = 1 - 2 * (qx * qx + qy * qy);
}

}  // namespace

extern "C" {

int mmff_gen_nnode(int natoms) {
    int nC, nN, nO, nH;
    composition(natoms, nC, nN, nO, nH);
    return nC + nN + nO;
}

// See mmff_host.h for the contract.
int mmff_gen_systems(int nsys, const int* natoms, uint64_t seed, int topo_mode,
                     double sigma, int rotate, double zplace, const double* cell_xy,
                     int hbond, double* pos, int* neighs, int* neighCell, int* bkneighs,
                     double* REQs, double* apars, double* bLs, double* bKs, double* Ksp,
                     double* Kpp, int* elements, int central_cell) {
    std::vector<size_t> aoff(nsys + 1, 0), noff(nsys + 1, 0), voff(nsys + 1, 0);
    for (int s = 0; s < nsys; s++) {
        int nh = mmff_gen_nnode(natoms[s]);
        aoff[s + 1] = aoff[s] + natoms[s];
        noff[s + 1] = noff[s] + nh;
        voff[s + 1] = voff[s] + natoms[s] + nh;
    }
    auto build_topo = [&](uint64_t topo_seed, int N, Mol& M) {
        for (int attempt = 0; attempt < 400; attempt++) {
            Rng r(topo_seed * 7919ull + (uint64_t)attempt * 104729ull + 17ull);
            if (build_mol(N, r, M, hbond != 0)) return true;
        }
        return false;
    };
    Mol proto;
    if (topo_mode == 0 && nsys > 0) {
        if (!build_topo(seed, natoms[0], proto)) return -1;
    }
    int fail = 0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int s = 0; s < nsys; s++) {
        if (fail) continue;
        const int N = natoms[s];
        Mol M;
        if (topo_mode == 0) {
            M = proto;
        } else if (!build_topo(seed * 1000003ull + (uint64_t)s, N, M)) {
#pragma omp critical
            { if (!fail) fail = s + 1; }
            continue;
        }
        if ((int)M.natoms != N) {
#pragma omp critical
            { if (!fail) fail = s + 1; }
            continue;
        }
        const size_t ao = aoff[s], no = noff[s], vo = voff[s];
        Rng rp(seed * 2654435761ull + (uint64_t)s * 40503ull + 99991ull);
        const int nh = M.nnode;
        // center, rotate, perturb
        V3 c{0, 0, 0};
        for (int i = 0; i < N; i++) c = c + M.pos[i];
        c = c * (1.0 / N);
        double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (rotate) random_rotation(rp, R);
        std::vector<V3> P(N + nh);
        for (int i = 0; i < N + nh; i++) {
            V3 v = (i < N) ? M.pos[i] - c : M.pos[i];
            P[i] = {R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z, R[6] * v.x + R[7] * v.y + R[8] * v.z};
        }
        for (int i = 0; i < N; i++) P[i] = P[i] + V3{sigma * rp.gauss(), sigma * rp.gauss(), sigma * rp.gauss()};
        double zmin = 1e300, xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
        for (int i = 0; i < N; i++) {
            zmin = std::min(zmin, P[i].z);
            xmin = std::min(xmin, P[i].x); xmax = std::max(xmax, P[i].x);
            ymin = std::min(ymin, P[i].y); ymax = std::max(ymax, P[i].y);
        }
        double cx = 0.5 * cell_xy[0], cy = 0.5 * cell_xy[1];
        V3 shift{cx - 0.5 * (xmin + xmax), cy - 0.5 * (ymin + ymax), zplace - zmin};
        for (int i = 0; i < N; i++) P[i] = P[i] + shift;
        for (int i = 0; i < N + nh; i++) { pos[3 * (vo + i)] = P[i].x; pos[3 * (vo + i) + 1] = P[i].y; pos[3 * (vo + i) + 2] = P[i].z; }
        for (int i = 0; i < N; i++) {
            for (int k = 0; k < 4; k++) {
                neighs[4 * (ao + i) + k] = M.neighs[4 * i + k];
                neighCell[4 * (ao + i) + k] = (M.neighs[4 * i + k] >= 0) ? central_cell : -1;
                REQs[4 * (ao + i) + k] = M.REQ[4 * i + k];
            }
            if (elements) elements[ao + i] = M.el[i];
        }
        // back neighbours (MMFFsp3_loc::makeBackNeighs ordering)
        for (int i = 0; i < N; i++) for (int k = 0; k < 4; k++) bkneighs[4 * (ao + i) + k] = -1;
        bool bad = false;
        for (int ia = 0; ia < nh; ia++) {
            for (int j = 0; j < 4; j++) {
                int ja = M.neighs[4 * ia + j];
                if (ja < 0) continue;
                int* bk = bkneighs + 4 * (ao + ja);
                int k = 0;
                while (k < 4 && bk[k] >= 0) k++;
                if (k == 4) { bad = true; break; }
                bk[k] = ia * 4 + j;
            }
        }
        if (bad) {
#pragma omp critical
            { if (!fail) fail = s + 1; }
            continue;
        }
        for (int i = 0; i < nh; i++) for (int k = 0; k < 4; k++) {
            apars[4 * (no + i) + k] = M.apars[4 * i + k];
            bLs[4 * (no + i) + k] = M.bLs[4 * i + k];
            bKs[4 * (no + i) + k] = M.bKs[4 * i + k];
            Ksp[4 * (no + i) + k] = M.Ksp[4 * i + k];
            Kpp[4 * (no + i) + k] = M.Kpp[4 * i + k];
        }
    }
    return fail ? -fail : 0;
}

// Rock-salt (001) slab, 'layers' layers below z_top, ncell x ncell conventional
// cells of edge a; ions alternate +q/-q.  Writes 4*ncell*ncell*layers ions.
int mmff_gen_slab(double a, int ncell, int layers, double z_top, double q,
                  const double* REQ_cation, const double* REQ_anion,
                  double* spos, double* sREQ) {
    int n = 0;
    const double h = 0.5 * a;
    for (int L = 0; L < layers; L++) {
        double z = z_top - L * h;
        for (int ix = 0; ix < 2 * ncell; ix++) for (int iy = 0; iy < 2 * ncell; iy++) {
            int cation = ((ix + iy + L) % 2) == 0;
            spos[3 * n] = ix * h; spos[3 * n + 1] = iy * h; spos[3 * n + 2] = z;
            const double* R = cation ? REQ_cation : REQ_anion;
            sREQ[4 * n] = R[0]; sREQ[4 * n + 1] = R[1]; sREQ[4 * n + 2] = cation ? q : -q; sREQ[4 * n + 3] = R[3];
            n++;
        }
    }
    return n;
}

}  // extern "C"
